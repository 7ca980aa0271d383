"""GPU detection vs the oracle's restatement of Predetection (process/cpu/Predetection.java):
identical candidate lists (slice, i, j in the same order), scores and parabolic
refinements to rounding (the reference's FFT correlation and this library's
direct FP64 correlation differ only by summation order)."""
import numpy as np
import pytest

import oracle as O
from common import OPTICS, astig_zernike, tetrapod_zernike

pytestmark = pytest.mark.gpu


def make_frames(model, S, n, seed, emitters=5, R=32, zr=0.6, bg=20.0):
    rng = np.random.default_rng(seed)
    frames = np.zeros((n, S, S))
    for f in range(n):
        img = np.full((S + R, S + R), bg)
        k = rng.poisson(emitters)
        for _ in range(k):
            cx, cy = rng.integers(0, S, 2)
            x, y = rng.uniform(-0.055, 0.055, 2)
            z = rng.uniform(-zr, zr)
            A = rng.lognormal(np.log(4000), 0.5)
            img[cx:cx + R, cy:cy + R] += A * model(R, [x, y, z])[0]
        frames[f] = rng.poisson(img[R // 2:R // 2 + S, R // 2:R // 2 + S])
    return frames


@pytest.mark.parametrize("S,R,zern,N", [(96, 16, astig_zernike(), 64), (128, 24, tetrapod_zernike(), 128)])
def test_detection_matches_oracle(zpkg, ctx, S, R, zern, N):
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=N, kz_reset=True, **OPTICS), zern)
    ref = O.OraclePSF(N, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, zern, gauss_f32=False, kz_reset=True)
    frames = make_frames(ref.model, S, 6, seed=S + R, R=2 * R)
    minZ, maxZ, step = -0.7, 0.7, 0.11
    det = zpkg.Detector(psf, S, S, R, minZ, maxZ, step, 0.1)
    odet = O.OracleDetector(ref, S, S, R, minZ, maxZ, step, 0.1)
    rg, lib = det.library()
    org, olib = odet.library()
    assert np.array_equal(rg, org)
    assert np.abs(lib - olib).max() < 1e-12 * olib.max()
    got, counts = det.detect(frames, cap=4096)
    want = odet.detect(frames, cap=4096)
    for f in range(len(frames)):
        g, w = got[f], want[f]
        assert counts[f] == len(w)
        assert len(w) > 0
        assert np.array_equal(g[:, 1:4].astype(int), w[:, 1:4].astype(int)), f"frame {f}: candidate order differs"
        assert np.allclose(g[:, 0], w[:, 0], rtol=1e-10, atol=0)
        assert np.allclose(g[:, 4:], w[:, 4:], rtol=1e-7, atol=1e-12)
    det.close()


def test_detection_empty_and_flat_frames(zpkg, ctx):
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=64, kz_reset=True, **OPTICS), astig_zernike())
    det = zpkg.Detector(psf, 64, 64, 16, -0.5, 0.5, 0.11, 0.1)
    frames = np.zeros((2, 64, 64))
    frames[1] = 7.0  # flat: zero local variance -> score -2 everywhere, no candidates
    got, counts = det.detect(frames, cap=64)
    assert list(counts) == [0, 0]
    det.close()


def test_detection_whole_lists_at_the_reference_threshold(zpkg, ctx):
    """256 x 256 frames against a 41-slice tetrapod library at the reference's
    threshold (0.1) give thousands of candidates per frame.  The lists are the
    oracle's whole sorted lists, the same on every run; a small cap returns
    their first rows, and a cap past the shared-memory sort takes the
    global-memory sort to the same rows."""
    zern = tetrapod_zernike()
    S, R, N = 256, 40, 128
    psf = zpkg.PSF(ctx, zpkg.optics(size_fft=N, kz_reset=True, **OPTICS), zern)
    ref = O.OraclePSF(N, 0.11, 1.4, 0.66, 1.518, 1.518, 0.9, zern, gauss_f32=False, kz_reset=True)
    frames = make_frames(ref.model, S, 2, seed=5, emitters=5, R=64, zr=2.0, bg=30.0)
    det = zpkg.Detector(psf, S, S, R, -2.0, 2.0, 0.1, 0.1)
    odet = O.OracleDetector(ref, S, S, R, -2.0, 2.0, 0.1, 0.1)
    want = odet.detect(frames, cap=100000, threads=8)
    got, counts = det.detect(frames, cap=16384)
    again, _ = det.detect(frames, cap=16384)
    small, counts_small = det.detect(frames, cap=500)
    wide, _ = det.detect(frames, cap=20000)
    for f in range(len(frames)):
        g, w = got[f], want[f]
        assert len(w) > 2000
        assert counts[f] == len(w) and counts_small[f] == len(w)
        assert np.array_equal(g, again[f])
        assert np.array_equal(g[:, 1:4].astype(int), w[:, 1:4].astype(int)), f"frame {f}: candidate order differs"
        assert np.allclose(g[:, 0], w[:, 0], rtol=1e-10, atol=0)
        assert np.array_equal(small[f], g[:500])
        assert np.array_equal(wide[f], g)
    det.close()
