"""GPU Zernike calibration: forward NLL vs the oracle's stack NLL
(ZernikePhaseRetrieval.java:1843-1874), the hand-written adjoint vs central
finite differences (h = 1e-4 lambda) and vs the reference's own
finite-difference step (h = 0.01 rad, :1081-1198), and an LM fit that recovers
known aberrations."""
import numpy as np
import pytest

import oracle as O
from common import OPTICS

pytestmark = pytest.mark.gpu
TWO_PI = 2 * np.pi


def bead_data(nz=15, nb=2, ns=11, R=32, seed=3):
    rng = np.random.default_rng(seed)
    zern = rng.normal(0, 0.05, nz) * TWO_PI
    zern[:3] = 0
    zern[5] += 0.1 * TWO_PI
    dz = (np.arange(ns) - ns // 2) * 0.15
    bead = np.c_[rng.uniform(-0.05, 0.05, (nb, 2)), rng.uniform(-0.05, 0.05, nb), np.full(nb, 20000.0),
                 np.full(nb, 50.0)]
    ref = O.OraclePSF(128, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, zern, gauss_f32=False)
    stacks = np.zeros((nb, ns, R, R))
    for b in range(nb):
        for s in range(ns):
            mu = bead[b, 3] * ref.model_oil(R, bead[b, 0], bead[b, 1], dz[s] + bead[b, 2], 0.0) + bead[b, 4]
            stacks[b, s] = rng.poisson(mu)
    return zern, dz, bead, stacks, ref


def test_forward_nll_matches_oracle(zpkg, ctx):
    zern, dz, bead, stacks, ref = bead_data()
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=128, **OPTICS), np.zeros(15))
    cal = zpkg.Calibration(psf, stacks, dz)
    z_try = zern * 0.7
    want = 0.0
    oref = O.OraclePSF(128, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, z_try, gauss_f32=False)
    for b in range(len(bead)):
        want += oref.calib_nll(32, dz, stacks[b], *bead[b])
    got = cal.forward(z_try, bead)
    assert abs(got - want) <= 1e-9 * abs(want)


def test_adjoint_gradient_vs_central_differences(zpkg, ctx):
    zern, dz, bead, stacks, ref = bead_data()
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=128, **OPTICS), np.zeros(15))
    cal = zpkg.Calibration(psf, stacks, dz)
    z0 = zern * 0.8
    b0 = bead + np.array([0.01, -0.01, 0.02, 500.0, 2.0])
    _, gz, gb = cal.backward(z0, b0)
    h = 1e-4 * TWO_PI  # 1e-4 lambda
    for i in range(3, 15):
        e = np.zeros(15)
        e[i] = h
        fd = (cal.forward(z0 + e, b0) - cal.forward(z0 - e, b0)) / (2 * h)
        assert abs(gz[i] - fd) <= 1e-4 * max(abs(fd), 1e-2 * np.abs(gz[3:]).max()), (i, gz[i], fd)
    hs = [1e-5, 1e-5, 1e-5, 1e-2, 1e-3]
    for b in range(len(b0)):
        for q in range(5):
            e = np.zeros_like(b0)
            e[b, q] = hs[q]
            fd = (cal.forward(z0, b0 + e) - cal.forward(z0, b0 - e)) / (2 * hs[q])
            assert abs(gb[b, q] - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(gb[:, q]).max() + 1e-6), (b, q, gb[b, q], fd)
    assert np.all(gz[:3] == 0)


def test_adjoint_vs_reference_finite_difference_step(zpkg, ctx):
    """The reference's coordinate update takes (lik3 - lik1) / 2h with h = 0.01 rad."""
    zern, dz, bead, stacks, ref = bead_data()
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=128, **OPTICS), np.zeros(15))
    cal = zpkg.Calibration(psf, stacks, dz)
    z0 = zern * 0.5
    _, gz, _ = cal.backward(z0, bead)
    for i in (4, 5, 7, 12):
        lik = []
        for sgn in (-1, 1):
            zz = z0.copy()
            zz[i] += sgn * 0.01
            o = O.OraclePSF(128, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, zz, gauss_f32=False)
            lik.append(sum(o.calib_nll(32, dz, stacks[b], *bead[b]) for b in range(len(bead))))
        fd = (lik[1] - lik[0]) / 0.02
        assert abs(gz[i] - fd) <= 2e-3 * abs(fd) + 1e-6, (i, gz[i], fd)


def test_calibration_fit_recovers_aberrations(zpkg, ctx):
    zern, dz, bead, stacks, ref = bead_data(seed=5)
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=128, **OPTICS), np.zeros(15))
    cal = zpkg.Calibration(psf, stacks, dz)
    z0 = np.zeros(15)
    b0 = bead.copy()
    b0[:, :3] = 0.0
    b0[:, 3] *= 0.8
    nll0 = cal.forward(z0, b0)
    zf, bf, nll, it = cal.fit(z0, b0, max_iter=40)
    assert nll < nll0
    truth_nll = cal.forward(zern, bead)
    assert nll <= truth_nll + 1.0  # at least as good as the truth (noise-limited)
    # defocus Z(2,0) (index 4) trades off with each bead's z offset, so compare
    # the other modes and the fitted stack model itself
    others = [i for i in range(3, 15) if i != 4]
    assert np.abs(zf[others] - zern[others]).max() < 0.05 * TWO_PI
    assert np.abs(bf[:, :2] - bead[:, :2]).max() < 0.01
    _, m_fit = cal.forward(zf, bf, model=True)
    _, m_true = cal.forward(zern, bead, model=True)
    assert np.abs(m_fit - m_true).max() < 0.02 * m_true.max()
