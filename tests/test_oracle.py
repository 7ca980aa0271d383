"""CPU tests of the oracle (known-answer tests; the reference ships no golden vectors)."""
import numpy as np
import pytest

import oracle as O
from common import OPTICS, astig_zernike


def make(N=64, zern=None, **kw):
    o = dict(OPTICS)
    o.update(kw)
    return O.OraclePSF(N, o["xystep"], o["na"], o["wavelength"], o["n_oil"], o.get("n_wat", o["n_oil"]), o["sigma"],
                       np.zeros(15) if zern is None else zern)


def test_disk_sizes():
    # PhaseParameters disk pixel counts for NA 1.4, lambda 0.66, dx 0.11
    assert make(64).K == 708
    assert make(128).K == 2820


def test_in_focus_aberration_free_is_symmetric_and_normalised():
    p = make(64)
    psi = p.model(16, [0.0, 0.0, 0.0])[0]
    assert abs(psi.sum() - 1) < 1e-12
    # centre N/2-0.5 grid and W/2 crop: symmetric under (i -> R-i) about index R/2
    core = psi[1:, 1:]
    assert np.allclose(core, core[::-1, :], rtol=1e-9, atol=1e-15)
    assert np.allclose(core, core[:, ::-1], rtol=1e-9, atol=1e-15)
    assert np.allclose(core, core.T, rtol=1e-9, atol=1e-15)
    assert np.unravel_index(psi.argmax(), psi.shape) == (8, 8)


def test_one_pixel_shift_moves_the_model_by_one_pixel():
    p = make(64, zern=astig_zernike())
    a = p.model(32, [0.0, 0.0, 0.2])[0]
    b = p.model(32, [-0.11, 0.0, 0.2])[0]  # theta_x = -dx moves the PSF by +1 px in x
    # compare the interior (normalisation over the crop differs slightly at the border)
    ia, ib = a[8:-9, 8:-8], b[9:-8, 8:-8]
    assert np.abs(ia / ia.sum() - ib / ib.sum()).max() < 2e-4 * ia.max()


def test_derivatives_match_central_differences():
    p = make(64, zern=astig_zernike())
    th = np.array([0.03, -0.02, 0.15])
    _, d = p.model(16, th, derivs=True)
    for k in range(3):
        e = np.zeros(3)
        e[k] = 1e-5
        fd = (p.model(16, th + e)[0] - p.model(16, th - e)[0]) / 2e-5
        assert np.abs(fd - d[0, k]).max() < 1e-7 * np.abs(d[0, k]).max()


def test_lm_and_reference_coordinate_descent_agree():
    p = make(64, zern=astig_zernike())
    rng = np.random.default_rng(0)
    n = 6
    truth = np.c_[rng.uniform(-.11, .11, (n, 2)), rng.uniform(-.5, .5, n), np.full(n, 3000.), np.full(n, 20.)]
    pat = rng.poisson(truth[:, 3, None, None] * p.model(16, truth[:, :3]) + 20).astype(float)
    init = truth.copy()
    init[:, :3] = 0
    lm, _, st, _ = p.fit_lm(pat, init, -1, 1, 0.88)
    assert (st == 1).all()
    cd, crlb, stc, _ = p.localize_cd(pat, np.c_[init[:, 3], init[:, 4], init[:, :3]], -0.9, 0.9, 20)
    assert (stc == 1).all()
    # accuracy tolerances: 0.5 nm in x/y, 1 nm in z
    assert np.abs(cd[:, :2] - lm[:, :2]).max() < 0.5e-3
    assert np.abs(cd[:, 2] - lm[:, 2]).max() < 1e-3
    assert (crlb > 0).all() and (crlb < 0.1).all()


def test_lm_gradient_is_zero_at_optimum():
    p = make(64, zern=astig_zernike())
    rng = np.random.default_rng(3)
    th = np.array([0.02, -0.01, 0.1, 2500., 20.])
    pat = rng.poisson(th[3] * p.model(16, th[:3])[0] + th[4]).astype(float)
    out, *_ = p.fit_lm(pat[None], th[None], -1, 1, 0.88, tol_xyz=1e-8, max_iter=60)
    v, g, H = p.nll_grad(pat, out[0])
    # scaled gradient g / sqrt(diag H) is ~0 at the optimum
    assert np.abs(g / np.sqrt(np.diag(H))).max() < 1e-3


def test_fft_round_trip_and_unitarity():
    # FFT convention (unitary, forward -i) checked through the blur with sigma -> 0:
    # a very narrow spatial blur leaves the intensity unchanged up to normalisation.
    p_sharp = make(64, sigma=0.05)
    p_none = make(64, sigma=0.05)
    a = p_sharp.model(16, [0.0, 0.0, 0.3])[0]
    b = p_none.model(16, [0.0, 0.0, 0.3])[0]
    assert np.allclose(a, b)
    assert abs(a.sum() - 1) < 1e-12


def test_detection_finds_isolated_emitter():
    p = make(64, zern=astig_zernike())
    det = O.OracleDetector(p, 64, 64, 16, -0.6, 0.6, 0.11, 0.1)
    rng = np.random.default_rng(1)
    img = np.full((64, 64), 20.0)
    psi = p.model(16, [0.0, 0.0, 0.1])[0]
    img[24:40, 30:46] += 5000 * psi
    img = rng.poisson(img).astype(float)
    c = det.detect(img[None])[0]
    assert len(c) >= 1
    assert (int(c[0, 2]), int(c[0, 3])) in [(32, 38), (31, 38), (32, 37), (33, 38), (32, 39)]


def _center_psf(N=64, zfocus=0.4, n_wat=1.33):
    o = OPTICS
    return O.OraclePSF(N, o["xystep"], o["na"], o["wavelength"], o["n_oil"], n_wat, o["sigma"], astig_zernike(),
                       zfocus=zfocus, gauss_f32=False)


def test_fd_fisher_crlb_matches_the_analytic_fisher_with_the_reference_A_row():
    """CRLB.computeFisher: central differences in x, y, z; the A row perturbs the
    formed mean (dmu/dA = mu a_step / h), the B row has dmu/dB = 1."""
    p = _center_psf()
    z = np.array([-0.3, 0.1, 0.45])
    ph, bg, h, ha = 3000.0, 50.0, 5e-4, 5e-4
    c = p.crlb_curve(32, z, ph, bg, h, ha)
    for k, zz in enumerate(z):
        psi, d = p.model(32, [0.0, 0.0, zz], derivs=True)
        mu = ph * psi[0] + bg
        J = [ph * d[0, 0], ph * d[0, 1], ph * d[0, 2], mu * (ha / h), np.ones_like(mu)]
        F = np.array([[np.sum(a * b / mu) for b in J] for a in J])
        assert np.allclose(c[k], np.sqrt(np.diag(np.linalg.inv(F))), rtol=1e-4)


def _center_search_py(p, R, axial, dx, zfocus):
    """SearchPSFcenter.getPosition restated in Python over the oracle's CRLB curve."""
    lat = lambda zs: np.hypot(*p.crlb_curve(R, zs, 3000.0, 50.0, 0.005, 0.5)[:, :2].T)

    def frange(a, b, s, incl=False):
        out, u = [], a
        while (u <= b) if incl else (u < b):
            out.append(u)
            u += s
        return out

    def min_pos(a, b, s):
        zs = frange(a, b, s)
        c = lat(zs)
        best, pos = np.inf, 0.0
        for u, v in zip(zs, c):
            if best > v:
                best, pos = v, u
        return pos

    step = dx * 5
    pos = min_pos(zfocus - 2 * axial - abs(zfocus), zfocus + abs(zfocus) + 2 * axial, step)
    old = np.inf
    for _ in range(10):
        a, b = pos - step * 5, pos + step * 5
        step = step / 2
        pos = min_pos(a, b, step)
        if abs(old - pos) < 1e-5:
            break
        old = pos
    ar = axial / 2
    a, b = pos - 2 * axial, pos + 2 * axial
    crlb = lat(frange(a - ar / 2, b + ar / 2, dx, incl=True))
    best, out = np.inf, 0.0
    nb = int(ar / (2 * dx))
    for u in frange(a, b, dx):
        s, nb2 = 0.0, -int(ar / (2 * dx))
        for _ in frange(-ar / 2, ar / 2, dx, incl=True):
            s += crlb[nb + nb2]
            nb2 += 1
        if best > s:
            best, out = s, u
        nb += 1
    return out


def test_center_search_restatement_agrees():
    p = _center_psf(zfocus=0.4)
    zc = p.center_search(32, 1.0, 0)
    assert zc == _center_search_py(p, 32, 1.0, 0.11, 0.4)


def test_center_search_gpu_form_returns_zfocus_when_index_matched():
    p = _center_psf(zfocus=0.3, n_wat=1.518)
    assert p.center_search(32, 1.0, 1) == 0.3
    assert p.center_search(32, -1.0, 0) == 0.3


def _bead_stack(seed=4, ns=21, W=72, H=64, nb=3, R=24):
    """Synthetic raw stack: tilted-plane background + beads with a z-dependent photon curve."""
    rng = np.random.default_rng(seed)
    o = OPTICS
    p = O.OraclePSF(64, o["xystep"], o["na"], o["wavelength"], o["n_oil"], o["n_oil"], o["sigma"], astig_zernike(),
                    gauss_f32=False)
    ii, jj = np.meshgrid(np.arange(W), np.arange(H), indexing="ij")
    plane = 40.0 + 0.05 * ii - 0.03 * jj
    dz = (np.arange(ns) - ns // 2) * 0.1
    pts = np.array([[18.3, 20.6], [50.2, 21.4], [33.7, 45.1]])[:nb]
    A = 8000.0 * np.exp(-0.5 * (dz / 1.2) ** 2)
    img = np.repeat(plane[None], ns, 0)
    for (px, py) in pts:
        ix, iy = int(px), int(py)
        for s in range(ns):
            # a positive model x moves the PSF towards lower pixel indices
            m = p.model_oil(R, (ix - px) * o["xystep"], (iy - py) * o["xystep"], dz[s], 0.0)
            img[s, ix - R // 2:ix + R // 2, iy - R // 2:iy + R // 2] += A[s] * m
    raw = rng.poisson(img).astype(np.float64)
    return raw, pts, A, plane, dz


def test_calib_init_recovers_background_photons_and_seeds():
    raw, pts, A, plane, dz = _bead_stack()
    seeds = np.round(pts) + np.array([1.0, -1.0])
    out = O.calib_init(raw, seeds[:, 0], seeds[:, 1], 24, zstep=0.1)
    # refined seeds: intensity centroid of the brightest pixels, within a pixel of the bead
    assert np.abs(out["x"] - pts[:, 0]).max() < 1.0 and np.abs(out["y"] - pts[:, 1]).max() < 1.0
    # background surface: the plane + 1 (photon conversion adds 1)
    assert np.abs(out["surface"] - (plane + 1)).max() < 1.5
    for k in range(3):
        x0, y0 = int(out["x"][k]) - 12, int(out["y"][k]) - 12
        assert abs(out["background"][k] - (plane[x0:x0 + 24, y0:y0 + 24].mean() + 1)) < 1.0
    # photon curve: the patch holds most of the bead's photons; the box filter smooths the Gaussian profile
    assert np.all(np.abs(out["photons"][:, len(dz) // 2] / A[len(dz) // 2] - 0.95) < 0.08)
    assert out["patches"].shape == (3, len(dz), 24, 24)


def drift_data(seed=0, nf=1000, nbead=40, n_per=30, L=600.0, Lz=200.0, vel=(0.03, -0.02, 0.01), noise=4.0):
    """Static 3-D structure localized repeatedly while the stage drifts linearly (nm / frame)."""
    rng = np.random.default_rng(seed)
    pts = np.c_[rng.uniform(0, L, (nbead, 2)), rng.uniform(0, Lz, nbead)]
    frames = rng.integers(0, nf, nbead * n_per)
    src = np.repeat(np.arange(nbead), n_per)
    dt = np.outer(frames, vel)
    xyz = pts[src] + dt + rng.normal(0, noise, (len(src), 3))
    return xyz, frames.astype(np.int32), np.full((len(src), 3), noise), dt, np.array(vel)


def test_drift_restatement_recovers_a_linear_drift():
    xyz, fr, cr, dt, vel = drift_data()
    b, l, px = O.drift(xyz, fr, cr, pixel_nm=20.0, bins=6, max_drift_um=0.16)
    assert px == 20.0
    # bin centres: minF + (s / bins)(1 + maxF - minF) + (maxF - minF) / (2 bins)
    fpb = (fr.max() - fr.min()) / 6
    assert np.allclose(b[:, 0], fr.min() + np.arange(6) / 6 * (1 + fr.max() - fr.min()) + fpb / 2)
    want = np.outer(b[:, 0] - b[0, 0], vel)
    assert np.abs(b[:, 1:] - want).max() < 6.0
    # per localization: the spline of the bin drifts at its frame, relative to bin 0's centre
    assert np.abs(l - (dt - np.outer(np.full(len(fr), b[0, 0]), vel))).max() < 7.0


def test_drift_restatement_handles_flat_z():
    xyz, fr, cr, dt, vel = drift_data(seed=1, vel=(0.02, 0.01, 0.0))
    xyz[:, 2] = 0.0
    b, l, px = O.drift(xyz, fr, cr, pixel_nm=20.0, bins=4, max_drift_um=0.16)
    assert np.all(b[:, 3] == 0.0)
    assert np.abs(b[:, 1:3] - np.outer(b[:, 0] - b[0, 0], vel[:2])).max() < 6.0
