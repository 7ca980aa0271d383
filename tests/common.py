"""Shared optics set-ups for the tests (the benchmark optics, at small sizes)."""
import numpy as np

TWO_PI = 2 * np.pi


def astig_zernike(nz=15, seed=0):
    """Astigmatic PSF: Z(2,2) = 0.08 lambda, Z(3,+-1), Z(4,0) ~ N(0, 0.02) lambda (radians)."""
    rng = np.random.default_rng(seed)
    z = np.zeros(nz)
    z[5] = 0.08 * TWO_PI
    for k in (7, 8, 12):
        z[k] = rng.normal(0, 0.02) * TWO_PI
    return z


def tetrapod_zernike(nz=45, seed=1):
    rng = np.random.default_rng(seed)
    z = rng.normal(0, 0.02, nz) * TWO_PI
    z[:3] = 0
    z[5] = 0.6 * TWO_PI
    z[13] = 0.3 * TWO_PI
    z[25] = 0.15 * TWO_PI
    return z


def saddle_zernike(nz=28, seed=2):
    z = np.zeros(nz)
    z[9] = 0.3 * TWO_PI
    return z


OPTICS = dict(xystep=0.11, na=1.4, wavelength=0.66, n_oil=1.518, sigma=0.9)


def synth_rois(model_fn, R, n, seed, zrange=0.6, photons=2000.0, sigma_ln=0.4, bg=20.0, xy_px=1.0, dx=0.11):
    rng = np.random.default_rng(seed)
    truth = np.zeros((n, 5))
    truth[:, :2] = rng.uniform(-xy_px * dx, xy_px * dx, (n, 2))
    truth[:, 2] = rng.uniform(-zrange, zrange, n)
    truth[:, 3] = rng.lognormal(np.log(photons), sigma_ln, n)
    truth[:, 4] = bg
    psi = model_fn(R, truth[:, :3])
    rois = rng.poisson(truth[:, 3, None, None] * psi + bg).astype(np.float32)
    return rois, truth


def z_symmetric(zern):
    """True when only odd Zernike terms (m odd <=> n odd) are non-zero: then
    I(r, -z) = I(r, z) exactly and z is identified up to its sign."""
    idx = 0
    n = 0
    while idx < len(zern):
        for m in range(-n, n + 1, 2):
            if idx < len(zern) and zern[idx] != 0 and n % 2 == 0 and idx > 2:
                return False
            idx += 1
        n += 1
    return True


def theta_diff(a, b, zsym):
    """|a - b| per parameter, comparing |z| when the PSF is z-symmetric."""
    d = np.abs(a - b)
    if zsym:
        d[:, 2] = np.abs(np.abs(a[:, 2]) - np.abs(b[:, 2]))
    return d
