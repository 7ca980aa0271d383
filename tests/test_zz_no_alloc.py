"""The allocation-free FP64 fit entry point (zola_fit_batch_noalloc).

Callers that cannot allocate device memory while they fit (a host application
that owns all device memory and lends the plugin only its own buffers, or an
acquisition thread that cannot stall on cudaMalloc) use this entry point: its
work areas sit in a fixed array inside the library.  It must reproduce the
regular FP64 fit (zola_fit_batch_dev) exactly, on two calls in a row (the
shared array keeps the previous call's contents).  Collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from common import OPTICS, saddle_zernike, synth_rois, tetrapod_zernike

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,R,zern", [(128, 24, saddle_zernike()), (128, 48, tetrapod_zernike())])
def test_noalloc_fit_matches_regular_fp64_fit(zpkg, ctx, N, R, zern):
    import torch
    dev = torch.device("cuda", 0)
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=N, **OPTICS), zern)
    ref = O.OraclePSF(N, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, zern, gauss_f32=False)
    rois_np, truth = synth_rois(ref.model, R, 300, seed=31 + R, zrange=0.6, photons=3000)
    init_np = truth.copy()
    init_np[:, :2] = 0
    init_np[:, 2] = np.round(truth[:, 2] / 0.1) * 0.1
    rois = torch.tensor(rois_np, device=dev)
    init = torch.tensor(init_np, dtype=torch.float64, device=dev)
    prm = zpkg.PSF.fit_params(-1.0, 1.0, R * 0.11 / 2, max_iter=40, tol_xyz=1e-4, precision=zpkg.ZOLA_PREC_FP64)

    def buffers():
        return (torch.zeros((300, 5), dtype=torch.float64, device=dev),
                torch.zeros((300, 5), dtype=torch.float64, device=dev),
                torch.zeros(300, dtype=torch.float64, device=dev),
                torch.zeros(300, dtype=torch.int32, device=dev),
                torch.zeros(300, dtype=torch.int32, device=dev))

    want = buffers()
    psf.fit_dev(rois, init, prm, *want, stream=ctx.stream)   # regular path (also prepares the tables for R)
    torch.cuda.synchronize()
    for call in range(2):
        got = buffers()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        zpkg.fit_noalloc_dev(psf, rois, init, prm, *got, stream=ctx.stream)
        torch.cuda.synchronize()
        if call == 1:  # the first call looked the array up; the second must not allocate
            assert torch.cuda.mem_get_info(dev)[0] == free_before
        assert torch.equal(got[3], want[3])          # status
        assert torch.equal(got[4], want[4])          # evaluations
        for g, w in zip(got[:3], want[:3]):
            assert torch.allclose(g, w, rtol=1e-12, atol=1e-12)
    psf.close()


def test_noalloc_rejects_unprepared_sizes_and_split_precision(zpkg, ctx):
    import torch
    dev = torch.device("cuda", 0)
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=64, **OPTICS), saddle_zernike(15))
    rois = torch.zeros((4, 20, 20), dtype=torch.float32, device=dev)
    init = torch.zeros((4, 5), dtype=torch.float64, device=dev)
    out = torch.zeros((4, 5), dtype=torch.float64, device=dev)
    prm = zpkg.PSF.fit_params(-1.0, 1.0, 1.0, precision=zpkg.ZOLA_PREC_FP64)
    with pytest.raises(zpkg.ZolaError, match="not prepared"):
        zpkg.fit_noalloc_dev(psf, rois, init, prm, out, stream=ctx.stream)
    split = zpkg.PSF.fit_params(-1.0, 1.0, 1.0, precision=zpkg.ZOLA_PREC_SPLIT)
    with pytest.raises(zpkg.ZolaError):
        zpkg.fit_noalloc_dev(psf, rois, init, split, out, stream=ctx.stream)
    psf.close()
