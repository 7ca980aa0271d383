"""GPU Zernike calibration: InitBackgroundAndPhotonNumber against the oracle's
restatement, the forward stack NLL with per-slice photometry, order-2
background and blur width against the oracle (ZernikePhaseRetrieval.java:
1519-1530, 1843-1874), the hand-written adjoint against central finite
differences (h = 1e-4 lambda for the phase) and the reference's own step
(h = 0.01 rad), and an LM fit that recovers known aberrations and sigma."""
import numpy as np
import pytest

import oracle as O
from common import OPTICS
from test_oracle import _bead_stack

pytestmark = pytest.mark.gpu
TWO_PI = 2 * np.pi
NP = 6


def poly_map(c, R):
    i, ii = np.meshgrid(np.arange(R, dtype=float), np.arange(R, dtype=float), indexing="ij")
    return c[0] + c[1] * i + c[2] * i * i + c[3] * ii + c[4] * i * ii + c[5] * ii * ii


def bead_data(nz=15, nb=2, ns=11, R=32, seed=3, sigma=1.0):
    rng = np.random.default_rng(seed)
    zern = rng.normal(0, 0.05, nz) * TWO_PI
    zern[:3] = 0
    zern[5] += 0.1 * TWO_PI
    dz = (np.arange(ns) - ns // 2) * 0.15
    xyz = np.c_[rng.uniform(-0.05, 0.05, (nb, 2)), rng.uniform(-0.05, 0.05, nb)]
    photons = 20000.0 * (1 + 0.2 * np.cos(dz / 0.6))[None, :] * np.ones((nb, 1))
    a = rng.normal(0, 300.0, (nb, ns))
    c = np.zeros((nb, NP))
    c[:, 0] = 50.0
    c[:, 1] = 0.3
    c[:, 3] = -0.2
    c[:, 5] = 0.004
    ref = O.OraclePSF(128, 0.11, 1.4, 0.66, 1.518, 1.518, sigma, zern, gauss_f32=False)
    stacks = np.zeros((nb, ns, R, R))
    for b in range(nb):
        bg = poly_map(c[b], R)
        for s in range(ns):
            mu = (photons[b, s] + a[b, s]) * ref.model_oil(R, xyz[b, 0], xyz[b, 1], dz[s] + xyz[b, 2], 0.0) + bg
            stacks[b, s] = rng.poisson(mu)
    bead = np.c_[xyz, a, c]
    return zern, dz, bead, stacks, photons


def oracle_nll(zern, sigma, dz, bead, stacks, photons, R=32):
    o = O.OraclePSF(128, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, zern, gauss_f32=False)
    ns = len(dz)
    return sum(o.calib_nll_full(R, dz, stacks[b], photons[b], sigma, bead[b, :3], bead[b, 3:3 + ns], bead[b, 3 + ns:])
               for b in range(len(bead)))


def make_cal(zpkg, ctx, stacks, dz, photons):
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=128, **OPTICS), np.zeros(15))
    return zpkg.Calibration(psf, stacks, dz, photons=photons)


def test_calib_init_matches_oracle(zpkg, ctx):
    raw, pts, A, plane, dz = _bead_stack()
    seeds = np.round(pts) + np.array([1.0, -1.0])
    raw32 = raw.astype(np.float32)
    for adu, gain, off in ((1.0, 1.0, 0.0), (0.5, 2.0, 100.0)):
        r = raw32 if off == 0 else ((raw32 - 1.0) / 0.25 + 100.0).astype(np.float32)
        got = zpkg.calib_init(ctx, r, seeds[:, 0], seeds[:, 1], 24, adu=adu, gain=gain, offset=off, zstep=0.1)
        want = O.calib_init(r.astype(np.float64), seeds[:, 0], seeds[:, 1], 24, adu=adu, gain=gain, offset=off,
                            zstep=0.1)
        assert np.array_equal(got["x"], want["x"]) and np.array_equal(got["y"], want["y"])
        for k in ("background", "photons", "patches", "surface"):
            assert np.allclose(got[k], want[k], rtol=1e-9, atol=1e-9 * np.abs(want[k]).max()), k


def test_calib_init_rejects_bad_arguments(zpkg, ctx):
    raw = np.zeros((5, 16, 16), np.float32)
    with pytest.raises(zpkg.ZolaError):
        zpkg.calib_init(ctx, raw, [8.0], [8.0], 2)
    with pytest.raises(zpkg.ZolaError):
        zpkg.calib_init(ctx, raw, [8.0], [8.0], 8, gain=0.0)


def test_forward_nll_matches_oracle(zpkg, ctx):
    zern, dz, bead, stacks, photons = bead_data()
    cal = make_cal(zpkg, ctx, stacks, dz, photons)
    z_try = zern * 0.7
    b_try = bead.copy()
    b_try[:, 3:14] *= 0.5
    for sigma in (1.0, 0.8):
        want = oracle_nll(z_try, sigma, dz, b_try, stacks, photons)
        got = cal.forward(z_try, sigma, b_try)
        assert abs(got - want) <= 1e-9 * abs(want)


def test_adjoint_gradient_vs_central_differences(zpkg, ctx):
    zern, dz, bead, stacks, photons = bead_data()
    cal = make_cal(zpkg, ctx, stacks, dz, photons)
    ns = len(dz)
    z0 = zern * 0.8
    s0 = 0.95
    b0 = bead.copy()
    b0[:, :3] += [0.01, -0.01, 0.02]
    b0[:, 3:3 + ns] += 200.0
    b0[:, 3 + ns] += 2.0
    _, gz, gs, gb = cal.backward(z0, s0, b0)
    h = 1e-4 * TWO_PI  # 1e-4 lambda
    for i in range(3, 15):
        e = np.zeros(15)
        e[i] = h
        fd = (cal.forward(z0 + e, s0, b0) - cal.forward(z0 - e, s0, b0)) / (2 * h)
        assert abs(gz[i] - fd) <= 1e-4 * max(abs(fd), 1e-2 * np.abs(gz[3:]).max()), (i, gz[i], fd)
    fd = (cal.forward(z0, s0 + 1e-5, b0) - cal.forward(z0, s0 - 1e-5, b0)) / 2e-5
    assert abs(gs - fd) <= 1e-4 * abs(fd), (gs, fd)
    cols = [0, 1, 2, 3, 3 + ns // 2, 2 + ns] + list(range(3 + ns, 3 + ns + NP))
    steps = {0: 1e-5, 1: 1e-5, 2: 1e-5}
    for b in range(len(b0)):
        for q in cols:
            hq = steps.get(q, 1e-2 if q < 3 + ns else 1e-4)
            e = np.zeros_like(b0)
            e[b, q] = hq
            fd = (cal.forward(z0, s0, b0 + e) - cal.forward(z0, s0, b0 - e)) / (2 * hq)
            scale = np.abs(gb[:, q]).max()
            assert abs(gb[b, q] - fd) <= 1e-4 * max(abs(fd), 1e-3 * scale) + 1e-6, (b, q, gb[b, q], fd)
    assert np.all(gz[:3] == 0)


def test_adjoint_vs_reference_finite_difference_step(zpkg, ctx):
    """The reference's coordinate update takes (lik3 - lik1) / 2h with h = 0.01 rad."""
    zern, dz, bead, stacks, photons = bead_data()
    cal = make_cal(zpkg, ctx, stacks, dz, photons)
    z0 = zern * 0.5
    _, gz, _, _ = cal.backward(z0, 1.0, bead)
    for i in (4, 5, 7, 12):
        lik = []
        for sgn in (-1, 1):
            zz = z0.copy()
            zz[i] += sgn * 0.01
            lik.append(oracle_nll(zz, 1.0, dz, bead, stacks, photons))
        fd = (lik[1] - lik[0]) / 0.02
        assert abs(gz[i] - fd) <= 2e-3 * abs(fd) + 1e-6, (i, gz[i], fd)


def test_calibration_fit_recovers_aberrations_and_sigma(zpkg, ctx):
    zern, dz, bead, stacks, photons = bead_data(seed=5)
    cal = make_cal(zpkg, ctx, stacks, dz, photons)
    ns = len(dz)
    z0 = np.zeros(15)
    b0 = np.zeros_like(bead)
    b0[:, 3 + ns] = bead[:, 3 + ns]  # constant background term from the init
    nll0 = cal.forward(z0, 0.9, b0)
    zf, sf, bf, nll, it = cal.fit(z0, 0.9, b0, max_iter=60)
    assert nll < nll0
    truth_nll = cal.forward(zern, 1.0, bead)
    assert nll <= truth_nll + 1.0  # at least as good as the truth (noise-limited)
    assert abs(sf - 1.0) < 0.03
    # defocus Z(2,0) (index 4) trades off with each bead's z offset, so compare
    # the other modes and the fitted stack model itself
    others = [i for i in range(3, 15) if i != 4]
    assert np.abs(zf[others] - zern[others]).max() < 0.05 * TWO_PI
    assert np.abs(bf[:, :2] - bead[:, :2]).max() < 0.01
    _, m_fit = cal.forward(zf, sf, bf, model=True)
    _, m_true = cal.forward(zern, 1.0, bead, model=True)
    # the fitted stack model stays within the Poisson noise of the true one at every pixel
    assert (np.abs(m_fit - m_true) / np.sqrt(m_true)).max() < 3.0


def config4_data(seed=3):
    """Bead z-stacks of the calibration benchmark: 5 beads x 61 slices (50 nm
    steps over +-1.5 um) x 32 x 32 px, a PSF from 45 Zernike coefficients
    ~ N(0, 0.05 lambda) plus 0.1 lambda astigmatism, sample index 1.33 with the
    beads at depth 0, 20,000 photons per bead, background 50 / px, Poisson
    noise."""
    rng = np.random.default_rng(seed)
    nz, nb, ns, R = 45, 5, 61, 32
    zern = rng.normal(0, 0.05, nz) * TWO_PI
    zern[:3] = 0
    zern[5] += 0.1 * TWO_PI
    dz = (np.arange(ns) - ns // 2) * 0.05
    xyz = np.c_[rng.uniform(-0.05, 0.05, (nb, 2)), rng.uniform(-0.05, 0.05, nb)]
    photons = np.full((nb, ns), 20000.0)
    a = rng.normal(0, 200.0, (nb, ns))
    c = np.zeros((nb, NP))
    c[:, 0] = 50.0
    ref = O.OraclePSF(128, 0.11, 1.4, 0.66, 1.518, 1.33, 1.0, zern, gauss_f32=False)
    stacks = np.zeros((nb, ns, R, R))
    for b in range(nb):
        for s in range(ns):
            mu = (photons[b, s] + a[b, s]) * ref.model_oil(R, xyz[b, 0], xyz[b, 1], dz[s] + xyz[b, 2], 0.0) + c[b, 0]
            stacks[b, s] = rng.poisson(mu)
    return zern, dz, np.c_[xyz, a, c], stacks, photons


def test_calibration_benchmark_scale_nll_and_adjoint(zpkg, ctx):
    """At the calibration benchmark's scale (45 coefficients, 5 beads x 61
    slices x 32^2, n_sample 1.33): the forward NLL equals the oracle's
    restatement of ZernikePhaseRetrieval's stack likelihood to 1e-9, and the
    hand-written adjoint is within 1e-4 of central finite differences
    (h = 1e-4 lambda for the phase) for every Zernike coefficient, the blur
    width and each bead's x, y, z, photometry and background terms."""
    zern, dz, bead, stacks, photons = config4_data()
    ns, nb = len(dz), len(bead)
    o = dict(OPTICS)
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=128, n_wat=1.33, **o), np.zeros(45))
    cal = zpkg.Calibration(psf, stacks, dz, photons=photons)
    z0 = zern * 0.8
    s0 = 0.95
    b0 = bead.copy()
    b0[:, :3] += [0.01, -0.01, 0.02]
    b0[:, 3 + ns] += 2.0
    ref = O.OraclePSF(128, 0.11, 1.4, 0.66, 1.518, 1.33, 0.9, z0, gauss_f32=False)
    want = sum(ref.calib_nll_full(32, dz, stacks[b], photons[b], s0, b0[b, :3], b0[b, 3:3 + ns], b0[b, 3 + ns:])
               for b in range(nb))
    got = cal.forward(z0, s0, b0)
    assert abs(got - want) <= 1e-9 * abs(want)
    _, gz, gs, gb = cal.backward(z0, s0, b0)
    h = 1e-4 * TWO_PI
    for i in range(3, 45):
        e = np.zeros(45)
        e[i] = h
        fd = (cal.forward(z0 + e, s0, b0) - cal.forward(z0 - e, s0, b0)) / (2 * h)
        assert abs(gz[i] - fd) <= 1e-4 * max(abs(fd), 1e-2 * np.abs(gz[3:]).max()), (i, gz[i], fd)
    fd = (cal.forward(z0, s0 + 1e-5, b0) - cal.forward(z0, s0 - 1e-5, b0)) / 2e-5
    assert abs(gs - fd) <= 1e-4 * abs(fd), (gs, fd)
    cols = [0, 1, 2, 3, 3 + ns // 2, 2 + ns] + list(range(3 + ns, 3 + ns + NP))
    steps = {0: 1e-5, 1: 1e-5, 2: 1e-5}
    for b in range(nb):
        for q in cols:
            hq = steps.get(q, 1e-2 if q < 3 + ns else 1e-4)
            e = np.zeros_like(b0)
            e[b, q] = hq
            fd = (cal.forward(z0, s0, b0 + e) - cal.forward(z0, s0, b0 - e)) / (2 * hq)
            scale = np.abs(gb[:, q]).max()
            assert abs(gb[b, q] - fd) <= 1e-4 * max(abs(fd), 1e-3 * scale) + 1e-6, (b, q, gb[b, q], fd)
    assert np.all(gz[:3] == 0)
