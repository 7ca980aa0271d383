"""sCMOS camera model (Localization.java:1132, LocalizationPipeline.java:588-640, 799-820):
the per-pixel var/gain^2 term in the fits and in the frame pipeline, against the oracle."""
import numpy as np
import pytest

import oracle as O
from common import OPTICS, astig_zernike, theta_diff
from test_gpu_detect import make_frames
from test_gpu_pipeline import match

pytestmark = pytest.mark.gpu


def scmos_rois(ref, R, n, seed):
    rng = np.random.default_rng(seed)
    truth = np.c_[rng.uniform(-0.1, 0.1, (n, 2)), rng.uniform(-0.5, 0.5, n), rng.lognormal(np.log(2500), 0.4, n),
                  np.full(n, 15.0)]
    v = rng.uniform(0.5, 12.0, (n, R, R))  # var / gain^2, photons
    mu = truth[:, 3, None, None] * ref.model(R, truth[:, :3]) + truth[:, 4, None, None] + v
    return rng.poisson(mu).astype(np.float32), v.astype(np.float32), truth


@pytest.mark.parametrize("precision", [0, 1])
def test_scmos_fit_matches_oracle(zpkg, ctx, precision):
    zern = astig_zernike()
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=64, **OPTICS), zern)
    ref = O.OraclePSF(64, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, zern, gauss_f32=False)
    rois, v, truth = scmos_rois(ref, 16, 24, seed=5)
    init = truth.copy()
    init[:, :2] = 0
    init[:, 2] = np.round(truth[:, 2] / 0.3) * 0.3
    init[:, 3] *= 0.8
    prm = zpkg.PSF.fit_params(-1.0, 1.0, 0.88, max_iter=40, tol_xyz=1e-4, precision=precision)
    res = psf.fit(rois, init, prm, scmos=v)
    o, nll, st, ev = ref.fit_lm_scmos(rois.astype(np.float64), v.astype(np.float64), init, -1.0, 1.0, 0.88,
                                      tol_xyz=1e-4, max_iter=40)
    ok = (st == 1) & (res["status"] == 1)
    assert ok.mean() > 0.8
    d = theta_diff(res["theta"][ok], o[ok], False)
    assert d[:, :2].max() * 1000 < 0.5 and d[:, 2].max() * 1000 < 1.0
    assert (d[:, 3] / o[ok, 3]).max() < 1e-3
    # without the sCMOS term the fit is biased (the background absorbs it)
    plain = psf.fit(rois, init, prm)
    assert np.median(plain["theta"][ok, 4] - res["theta"][ok, 4]) > 1.0


def test_scmos_pipeline_matches_oracle(zpkg, ctx):
    zern = astig_zernike()
    S, R = 96, 16
    psf_det = zpkg.PSF(ctx, zpkg.optics(size_fft=64, kz_reset=True, **OPTICS), zern)
    psf_fit = zpkg.PSF(ctx, zpkg.optics(size_fft=64, **OPTICS), zern)
    ref_det = O.OraclePSF(64, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, zern, kz_reset=True)
    ref_fit = O.OraclePSF(64, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, zern)
    photons = make_frames(ref_fit.model, S, 6, seed=78, emitters=4, R=32)
    rng = np.random.default_rng(3)
    gain = rng.uniform(1.8, 2.2, (S, S))
    offset = rng.uniform(95.0, 105.0, (S, S))
    var = rng.uniform(2.0, 40.0, (S, S))
    adu = (gain * photons + offset + rng.normal(0, np.sqrt(var), photons.shape)).astype(np.float32)
    minZ, maxZ = -0.6, 0.6
    det = zpkg.Detector(psf_det, S, S, R, minZ, maxZ, 0.11, 0.1)
    odet = O.OracleDetector(ref_det, S, S, R, minZ, maxZ, 0.11, 0.1)
    got = zpkg.localize_frames_scmos(ctx, det, psf_fit, adu, offset, gain, var, minZ, maxZ, photon_threshold=500.0,
                                     precision=0, max_iter=40)
    want = odet.localize_frames_scmos(ref_fit, adu.astype(np.float64), offset, gain, var, minZ, maxZ,
                                      photon_thr=500.0, threads=4)
    assert len(want) > 10
    assert abs(len(got) - len(want)) <= max(2, 0.1 * len(want))
    pairs = match(got, want)
    assert len(pairs) >= 0.9 * len(want)
    dxy = np.array([max(abs(g["x_nm"] - w[1]), abs(g["y_nm"] - w[2])) for g, w in pairs])
    dz = np.array([abs(g["z_nm"] - w[3]) for g, w in pairs])
    assert np.median(dxy) < 0.5 and np.median(dz) < 1.0
    det.close()
