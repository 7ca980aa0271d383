"""GPU tests of the dataflow split fit (ZOLA_SPLIT_FLOW: the whole fit as one
cooperative kernel, stages on their own SMs, device work queue) against the
round-based stage kernels, and of its streaming input and bounded waits."""
import numpy as np
import pytest

import oracle as O
from common import OPTICS, astig_zernike, saddle_zernike, synth_rois, tetrapod_zernike

pytestmark = pytest.mark.gpu

# (N, R, zernike): windows 32 (with 32 and 64 pupil rows), 64 and 128
FLOW_CASES = [
    (64, 16, astig_zernike()),
    (128, 16, astig_zernike()),
    (128, 24, saddle_zernike()),
    (128, 40, tetrapod_zernike()),
    (128, 48, tetrapod_zernike()),
]


def _job(zpkg, ctx, N, R, zern, n, seed):
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=N, **OPTICS), zern)
    ref = O.OraclePSF(N, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, zern, gauss_f32=False)
    rois, truth = synth_rois(ref.model, R, n, seed=seed, zrange=0.6, photons=3000, sigma_ln=0.6)
    init = truth.copy()
    init[:, :2] = 0
    init[:, 2] = np.round(truth[:, 2] / 0.1) * 0.1
    init[:, 3] *= 0.85
    prm = zpkg.PSF.fit_params(-1.0, 1.0, R * 0.11 / 2, max_iter=50, tol_xyz=1e-4, precision=zpkg.ZOLA_PREC_SPLIT)
    return psf, rois, init, prm


@pytest.mark.parametrize("N,R,zern", FLOW_CASES)
def test_flow_equals_staged_bit_for_bit(zpkg, ctx, N, R, zern):
    """The dataflow kernel runs the same stage code as the round-based kernels,
    so each ROI's fit is the same bit for bit, whatever the shape of the
    dataflow kernel (units in flight, CTAs per stage)."""
    psf, rois, init, prm = _job(zpkg, ctx, N, R, zern, 1500, seed=900 + R + N)
    try:
        ctx.set_split_mode("staged")
        staged = psf.fit(rois, init, prm)
        ctx.set_split_mode("flow")
        flow = psf.fit(rois, init, prm)
        import torch
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        ctx.set_flow(units=7, ctas=[sms - 4, 1, 1, 1, 1])
        odd = psf.fit(rois, init, prm)
    finally:
        ctx.set_flow(0, None)
        ctx.set_split_mode("staged")
    assert (staged["status"] == 1).mean() > 0.8
    for r in (flow, odd):
        for k in ("theta", "crlb", "nll", "status", "iters"):
            assert np.array_equal(np.nan_to_num(r[k]), np.nan_to_num(staged[k])), k
    psf.close()


def test_flow_streaming_input_and_wait_limit(zpkg, ctx):
    """Streaming input: a producer's device count says how many ROIs are on the
    device.  The count is left at half the batch and never raised: the fit
    handles every ROI below it (the same results as a plain fit of that half),
    then its bounded wait for more input runs out and the call ends with
    ZOLA_E_TIMEOUT.  The next call on the same context succeeds."""
    import torch
    dev = torch.device("cuda", 0)
    psf, rois, init, prm = _job(zpkg, ctx, 64, 16, astig_zernike(), 800, seed=77)
    n, half = len(rois), len(rois) // 2
    d_rois = torch.tensor(rois, device=dev)
    d_init = torch.tensor(init, device=dev)
    avail = torch.tensor([half], dtype=torch.int32, device=dev)
    out = torch.full((n, 5), -7.0, dtype=torch.float64, device=dev)
    st = torch.zeros(n, dtype=torch.int32, device=dev)
    it = torch.zeros(n, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    ctx.set_wait_limit(40_000_000)  # about 20 ms of GPU clock
    try:
        with pytest.raises(zpkg.ZolaError, match=r"\(-5\)"):
            psf.fit_stream_dev(d_rois, d_init, avail, prm, out, None, None, st, it)
    finally:
        ctx.set_wait_limit(0)
    torch.cuda.synchronize()
    want = psf.fit(rois[:half], init[:half], prm)
    assert np.array_equal(out[:half].cpu().numpy(), want["theta"])
    assert np.array_equal(st[:half].cpu().numpy(), want["status"])
    assert (out[half:].cpu().numpy() == -7.0).all()  # nothing beyond the count was touched
    # the context is usable: the whole batch, streamed with its count already complete
    avail.fill_(n)
    psf.fit_stream_dev(d_rois, d_init, avail, prm, out, None, None, st, it)
    torch.cuda.synchronize()
    full = psf.fit(rois, init, prm)
    assert np.array_equal(out.cpu().numpy(), full["theta"])
    psf.close()


def test_autotuner_changes_timings_only(zpkg, ctx, tmp_path):
    """The autotuner tries a few dataflow-kernel shapes on the first large fits
    of a class and keeps the fastest; every trial gives the same fits bit for
    bit, the tuned shape is written to the cache file, and a new context
    reads it back."""
    import json
    import torch
    dev = torch.device("cuda", 0)
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=64, **OPTICS), astig_zernike())
    n, R = 40000, 16
    rng = np.random.default_rng(5)
    truth = np.c_[rng.uniform(-0.11, 0.11, (n, 2)), rng.uniform(-0.5, 0.5, n), rng.lognormal(np.log(2500.0), 0.5, n),
                  np.full(n, 20.0)]
    psi = torch.empty((n, R, R), dtype=torch.float64, device=dev)
    psf.model_dev(R, torch.tensor(truth[:, :3], device=dev), psi, stream=ctx.stream)
    torch.cuda.synchronize()
    g = torch.Generator(device=dev)
    g.manual_seed(11)
    rois = torch.poisson(torch.tensor(truth[:, 3], device=dev)[:, None, None] * psi + 20.0, generator=g).float()
    init = truth.copy()
    init[:, :2] = 0
    init[:, 2] = np.round(truth[:, 2] / 0.1) * 0.1
    d_init = torch.tensor(init, device=dev)
    prm = zpkg.PSF.fit_params(-1.0, 1.0, 0.88, max_iter=50, tol_xyz=1e-4, precision=zpkg.ZOLA_PREC_SPLIT)

    def run():
        out = [torch.zeros((n, 5), dtype=torch.float64, device=dev), torch.zeros(n, dtype=torch.int32, device=dev)]
        psf.fit_dev(rois, d_init, prm, out[0], None, None, out[1], None, stream=ctx.stream)
        torch.cuda.synchronize()
        return out[0].cpu().numpy(), out[1].cpu().numpy()

    base = run()  # round-based kernels
    cache = str(tmp_path / "flow_tune.json")
    ctx.set_split_mode("flow")
    ctx.set_tuning(True, cache)
    try:
        for _ in range(10):
            got = run()
            assert np.array_equal(got[0], base[0]) and np.array_equal(got[1], base[1])
            if psf.flow_shape(R)[0]:
                break
    finally:
        ctx.set_tuning(False)
        ctx.set_split_mode("staged")
    tuned, units, ctas, ns = psf.flow_shape(R)
    assert tuned and units > 0 and min(ctas) >= 1 and ns > 0
    entry = next(iter(json.load(open(cache)).values()))
    assert entry["units"] == units and entry["ctas"] == ctas
    c2 = zpkg.Context(0)
    try:
        c2.set_tuning(False, cache)
        p2 = zpkg.PSF(c2, zpkg.optics(size_fft=64, **OPTICS), astig_zernike())
        assert p2.flow_shape(R)[:3] == (True, units, ctas)
        p2.close()
    finally:
        c2.close()
    psf.close()


def test_pool_tuner_changes_timings_only(zpkg, tmp_path):
    """With tuning on and an automatic pool, the round-based split fit tries
    four slot pools on the first large fits of a class and keeps the fastest;
    every trial gives the fits of the default pool bit for bit (a fit does not
    depend on its batch), and the choice goes to the cache file and back."""
    import json
    import torch
    dev = torch.device("cuda", 0)
    c = zpkg.Context(0)
    try:
        psf = zpkg.PSF(c, zpkg.optics(size_fft=64, **OPTICS), astig_zernike())
        m, rep, R = 8192, 16, 16
        n = m * rep
        rng = np.random.default_rng(8)
        truth = np.c_[rng.uniform(-0.11, 0.11, (m, 2)), rng.uniform(-0.5, 0.5, m),
                      rng.lognormal(np.log(2500.0), 0.5, m), np.full(m, 20.0)]
        psi = torch.empty((m, R, R), dtype=torch.float64, device=dev)
        psf.model_dev(R, torch.tensor(truth[:, :3], device=dev), psi, stream=c.stream)
        torch.cuda.synchronize()
        g = torch.Generator(device=dev)
        g.manual_seed(12)
        rois = torch.poisson(torch.tensor(truth[:, 3], device=dev)[:, None, None] * psi + 20.0,
                             generator=g).float().repeat(rep, 1, 1).contiguous()
        init = np.tile(truth, (rep, 1))
        init[:, :2] = 0
        init[:, 2] = np.round(init[:, 2] / 0.1) * 0.1
        d_init = torch.tensor(init, device=dev)
        prm = zpkg.PSF.fit_params(-1.0, 1.0, 0.88, max_iter=50, tol_xyz=1e-4, precision=zpkg.ZOLA_PREC_SPLIT)

        def run():
            out = [torch.zeros((n, 5), dtype=torch.float64, device=dev), torch.zeros(n, dtype=torch.int32, device=dev)]
            psf.fit_dev(rois, d_init, prm, out[0], None, None, out[1], None, stream=c.stream)
            torch.cuda.synchronize()
            return out[0].cpu().numpy(), out[1].cpu().numpy()

        c.set_pool(0)
        base = run()
        assert psf.split_pool(R)[0] is False
        cache = str(tmp_path / "pool_tune.json")
        c.set_tuning(True, cache)
        try:
            for _ in range(4):
                got = run()
                assert np.array_equal(got[0], base[0]) and np.array_equal(got[1], base[1])
        finally:
            c.set_tuning(False)
        tuned, pool, ns = psf.split_pool(R)
        assert tuned and pool in (4096, 8192, 16384, 32768) and ns > 0
        got = run()  # the tuned pool
        assert np.array_equal(got[0], base[0]) and np.array_equal(got[1], base[1])
        entries = {k: v for k, v in json.load(open(cache)).items() if k.endswith("_pool")}
        assert list(entries.values())[0]["pool"] == pool
        psf.close()
    finally:
        c.close()
    c2 = zpkg.Context(0)
    try:
        c2.set_tuning(False, cache)
        p2 = zpkg.PSF(c2, zpkg.optics(size_fft=64, **OPTICS), astig_zernike())
        assert p2.split_pool(R)[:2] == (True, pool)
        p2.close()
    finally:
        c2.close()
