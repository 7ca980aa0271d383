"""ORACLE — test infrastructure only (never imported by the product path).

ctypes wrapper over ``zola_oracle.cpp``, the FP64 CPU restatement of ZOLA-3D's
localization hot path (see the header of that file for the reference file:line
each function follows).  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg may import this module.

PARITY UNPINNED: the reference has no tests or golden vectors for this path and
cannot run here (Java plugin, no JVM); the oracle is pinned by known-answer
tests only.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")
_SRC = os.path.join(_HERE, "zola_oracle.cpp")


def build(force=False):
    """Compile the oracle with g++ (the recipe lives here and in Makefile)."""
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(_SRC):
        subprocess.check_call(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-o", _SO, _SRC, "-lpthread"])
    return _SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_SO)
        d, i, vp = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        P = ctypes.POINTER
        L.orc_psf_create.restype = vp
        L.orc_psf_create.argtypes = [i, d, d, d, d, d, d, i, d, i, i, i, vp]
        L.orc_psf_destroy.argtypes = [vp]
        L.orc_psf_info.argtypes = [vp, vp, vp]
        L.orc_psf_tables.argtypes = [vp] + [vp] * 6
        L.orc_window_size.argtypes = [i, i]
        L.orc_psf_model.argtypes = [vp, i, i, vp, vp, vp]
        L.orc_psf_model_oil.argtypes = [vp, i, d, d, d, d, vp]
        L.orc_localize_cd.argtypes = [vp, i, i, vp, vp, d, d, i, d, vp, vp, vp, vp, i]
        L.orc_localize_cd_eps.argtypes = [vp, i, i, vp, vp, d, d, i, d, d, vp, vp, vp, vp, i]
        L.orc_fit_lm.argtypes = [vp, i, i, vp, vp, vp, i, vp, vp, vp, vp, vp, i]
        L.orc_fit_lm_scmos.argtypes = [vp, i, i, vp, vp, vp, vp, i, vp, vp, vp, vp, vp, i]
        L.orc_nll_grad.restype = d
        L.orc_nll_grad.argtypes = [vp, i, vp, vp, vp, vp]
        L.orc_crlb_fd.argtypes = [vp, i, vp, vp]
        L.orc_center_search.restype = d
        L.orc_center_search.argtypes = [vp, i, d, i, vp]
        L.orc_crlb_curve.argtypes = [vp, i, i, vp, d, d, d, d, vp]
        L.orc_det_create.restype = vp
        L.orc_det_create.argtypes = [vp, i, i, i, d, d, d, d]
        L.orc_det_destroy.argtypes = [vp]
        L.orc_det_nslices.argtypes = [vp]
        L.orc_det_library.argtypes = [vp, vp, vp]
        L.orc_detect.argtypes = [vp, i, vp, i, vp, vp, i]
        L.orc_localize_frames.restype = i
        L.orc_localize_frames.argtypes = [vp, vp, i, vp, d, d, d, d, i, vp, i]
        L.orc_localize_frames_lm.restype = i
        L.orc_localize_frames_lm.argtypes = [vp, vp, i, vp, d, d, d, d, i, d, i, vp, i]
        L.orc_localize_frames_scmos.restype = i
        L.orc_localize_frames_scmos.argtypes = [vp, vp, i, vp, vp, vp, vp, d, d, d, d, i, vp, i]
        L.orc_calib_nll.restype = d
        L.orc_calib_nll.argtypes = [vp, i, i, vp, vp, d, d, d, d, d]
        L.orc_calib_nll_full.restype = d
        L.orc_calib_nll_full.argtypes = [vp, i, i, vp, vp, vp, d, d, d, d, vp, vp]
        L.orc_calib_init.restype = i
        L.orc_drift.restype = i
        L.orc_drift.argtypes = [vp, vp, vp, i, d, i, d, vp, vp, vp]
        L.orc_calib_init.argtypes = [vp, i, i, i, vp, vp, i, i, d, d, d, d, vp, vp, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class OraclePSF:
    """PSFPhase + ZernikePhase (process/cpu/PSFPhase.java, ZernikePhase.java)."""

    def __init__(self, N, dx, na, wavelength, n_oil, n_wat, sigma, zernike, apo=False,
                 zfocus=0.0, kz_reset=False, gauss_f32=True):
        self.zernike = _f64(zernike)
        self.h = lib().orc_psf_create(int(N), dx, na, wavelength, n_oil, n_wat, sigma, int(apo), zfocus,
                                      int(kz_reset), int(gauss_f32), len(self.zernike), _p(self.zernike))
        n = ctypes.c_int()
        k = ctypes.c_int()
        lib().orc_psf_info(self.h, ctypes.byref(n), ctypes.byref(k))
        self.N, self.K = n.value, k.value
        self.dx = dx

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_psf_destroy(self.h)
            self.h = None

    def tables(self):
        out = [np.zeros(self.K) for _ in range(6)]
        lib().orc_psf_tables(self.h, *[_p(o) for o in out])
        return dict(zip(["kx", "ky", "kz", "kzoil", "pupil", "phase"], out))

    def model(self, R, xyz, derivs=False):
        xyz = _f64(np.atleast_2d(xyz))
        n = xyz.shape[0]
        out = np.zeros((n, R, R))
        d = np.zeros((n, 3, R, R)) if derivs else None
        lib().orc_psf_model(self.h, R, n, _p(xyz), _p(out), _p(d) if derivs else None)
        return (out, d) if derivs else out

    def model_oil(self, R, x, y, zoil, zwat):
        out = np.zeros((R, R))
        lib().orc_psf_model_oil(self.h, R, x, y, zoil, zwat, _p(out))
        return out

    def localize_cd(self, patches, init_abxyz, minZ, maxZ, iter_max=20, photon_thr=0.0, threads=1, eps=None):
        """The reference coordinate descent; eps (um) replaces its stopping distance 1e-4 when given."""
        patches = _f64(patches)
        n, R = patches.shape[0], patches.shape[1]
        init = _f64(init_abxyz)
        out = np.zeros((n, 5))
        crlb = np.zeros((n, 3))
        st = np.zeros(n, np.int32)
        ev = np.zeros(n, np.int32)
        if eps is None:
            lib().orc_localize_cd(self.h, R, n, _p(patches), _p(init), minZ, maxZ, iter_max, photon_thr,
                                  _p(out), _p(crlb), _p(st), _p(ev), threads)
        else:
            lib().orc_localize_cd_eps(self.h, R, n, _p(patches), _p(init), minZ, maxZ, iter_max, photon_thr, eps,
                                      _p(out), _p(crlb), _p(st), _p(ev), threads)
        return out, crlb, st, ev

    def fit_lm(self, patches, init_xyzab, zmin, zmax, xymax, tol_xyz=1e-5, step_xy=0.11, step_z=0.22,
               max_iter=30, threads=1, crlb=False):
        patches = _f64(patches)
        n, R = patches.shape[0], patches.shape[1]
        init = _f64(init_xyzab)
        prm = _f64([zmin, zmax, xymax, tol_xyz, step_xy, step_z])
        out = np.zeros((n, 5))
        nll = np.zeros(n)
        st = np.zeros(n, np.int32)
        ev = np.zeros(n, np.int32)
        cr = np.zeros((n, 5)) if crlb else None
        lib().orc_fit_lm(self.h, R, n, _p(patches), _p(init), _p(prm), max_iter, _p(out), _p(nll), _p(st),
                         _p(ev), _p(cr) if crlb else None, threads)
        return (out, nll, st, ev, cr) if crlb else (out, nll, st, ev)

    def fit_lm_scmos(self, patches, scmos, init_xyzab, zmin, zmax, xymax, tol_xyz=1e-5, step_xy=0.11, step_z=0.22,
                     max_iter=30, threads=1):
        """lm_fit with the sCMOS term var/gain^2 (n, R, R) added to the model mean."""
        patches, scmos, init = _f64(patches), _f64(scmos), _f64(init_xyzab)
        n, R = patches.shape[0], patches.shape[1]
        prm = _f64([zmin, zmax, xymax, tol_xyz, step_xy, step_z])
        out = np.zeros((n, 5))
        nll = np.zeros(n)
        st = np.zeros(n, np.int32)
        ev = np.zeros(n, np.int32)
        lib().orc_fit_lm_scmos(self.h, R, n, _p(patches), _p(scmos), _p(init), _p(prm), max_iter, _p(out), _p(nll),
                               _p(st), _p(ev), None, threads)
        return out, nll, st, ev

    def nll_grad(self, patch, theta):
        patch = _f64(patch)
        th = _f64(theta)
        g = np.zeros(5)
        H = np.zeros(25)
        v = lib().orc_nll_grad(self.h, patch.shape[0], _p(patch), _p(th), _p(g), _p(H))
        return v, g, H.reshape(5, 5)

    def crlb_fd(self, R, theta):
        th = _f64(theta)
        out = np.zeros(3)
        lib().orc_crlb_fd(self.h, R, _p(th), _p(out))
        return out

    def center_search(self, R, axial_range, variant=0):
        """SearchPSFcenter.getPosition (variant 0: process/cpu, 1: process/gpu form)."""
        st = ctypes.c_int()
        z = lib().orc_center_search(self.h, int(R), float(axial_range), int(variant), ctypes.byref(st))
        if st.value:
            raise IndexError("center search: range window ran past the CRLB table")
        return z

    def crlb_curve(self, R, z, photons=3000.0, bg=50.0, h=0.005, a_step=0.5):
        """CRLB (x, y, z, A, B) at (0, 0, z) from the finite-difference Fisher matrix."""
        z = _f64(z)
        out = np.zeros((len(z), 5))
        lib().orc_crlb_curve(self.h, int(R), len(z), _p(z), photons, bg, h, a_step, _p(out))
        return out

    def calib_nll_full(self, R, dz, stack, photons, sigma, xyz, a, c):
        """Stack NLL of one bead with per-slice photons + a, order-2 background c[6], blur sigma."""
        dz, stack, a, c = _f64(dz), _f64(stack), _f64(a), _f64(c)
        ph = None if photons is None else _f64(photons)
        return lib().orc_calib_nll_full(self.h, R, len(dz), _p(dz), _p(stack), _p(ph) if ph is not None else None,
                                        sigma, xyz[0], xyz[1], xyz[2], _p(a), _p(c))

    def calib_nll(self, R, dz, stack, x, y, z, A, B):
        dz = _f64(dz)
        stack = _f64(stack)
        return lib().orc_calib_nll(self.h, R, len(dz), _p(dz), _p(stack), x, y, z, A, B)


class OracleDetector:
    """Predetection (process/cpu/Predetection.java) for frames [X][Y]."""

    def __init__(self, psf, SX, SY, R, minZ, maxZ, step, thr=0.1):
        self.psf = psf
        self.SX, self.SY, self.R = SX, SY, R
        self.h = lib().orc_det_create(psf.h, SX, SY, R, minZ, maxZ, step, thr)
        self.nz = lib().orc_det_nslices(self.h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_det_destroy(self.h)
            self.h = None

    def library(self):
        rng = np.zeros(self.nz)
        psfs = np.zeros((self.nz, self.R, self.R))
        lib().orc_det_library(self.h, _p(rng), _p(psfs))
        return rng, psfs

    def localize_frames(self, fit_psf, frames, minZ, maxZ, photon_thr=500.0, max_snr=1.0, threads=1, cap=100000):
        """LocalizationPipeline frame loop with the reference coordinate descent.
        Rows: frame, x_nm, y_nm, z_nm, A, B, chi2, crlbx, crlby, crlbz."""
        frames = _f64(frames)
        rows = np.zeros((cap, 10))
        n = lib().orc_localize_frames(self.h, fit_psf.h, frames.shape[0], _p(frames), minZ, maxZ, photon_thr, max_snr,
                                      cap, _p(rows), threads)
        return rows[:min(n, cap)]

    def localize_frames_lm(self, fit_psf, frames, minZ, maxZ, photon_thr=500.0, max_snr=1.0, max_iter=40,
                           tol_xyz=1e-4, threads=1, cap=100000):
        """The same frame loop with the FP64 LM fit of the library (the oracle of
        zola_localize_frames).  Rows: frame, x_nm, y_nm, z_nm, A, B, chi2, crlbx,
        crlby, crlbz, candidate index, LM status (1 converged, 2 evaluation cap, 3 stalled)."""
        frames = _f64(frames)
        rows = np.zeros((cap, 12))
        n = lib().orc_localize_frames_lm(self.h, fit_psf.h, frames.shape[0], _p(frames), minZ, maxZ, photon_thr,
                                         max_snr, max_iter, tol_xyz, cap, _p(rows), threads)
        return rows[:min(n, cap)]

    def localize_frames_scmos(self, fit_psf, adu, offset, gain, variance, minZ, maxZ, photon_thr=500.0, max_snr=1.0,
                              threads=1, cap=100000):
        """sCMOS pipeline: ADU frames and per-pixel offset / gain / variance maps."""
        adu, off, gn, var = _f64(adu), _f64(offset), _f64(gain), _f64(variance)
        rows = np.zeros((cap, 10))
        n = lib().orc_localize_frames_scmos(self.h, fit_psf.h, adu.shape[0], _p(adu), _p(off), _p(gn), _p(var), minZ,
                                            maxZ, photon_thr, max_snr, cap, _p(rows), threads)
        return rows[:min(n, cap)]

    def detect(self, frames, cap=4096, threads=1):
        frames = _f64(frames)
        nf = frames.shape[0]
        out = np.zeros((nf, cap, 7))
        counts = np.zeros(nf, np.int32)
        lib().orc_detect(self.h, nf, _p(frames), cap, _p(out), _p(counts), threads)
        return [out[f, :min(cap, counts[f])] for f in range(nf)]


def calib_init(raw, xpoints, ypoints, size_patch, adu=1.0, gain=1.0, offset=0.0, zstep=0.05):
    """InitBackgroundAndPhotonNumber restated (raw: (nslice, W, H) ADU)."""
    raw = _f64(raw)
    ns, W, H = raw.shape
    xp = np.array(xpoints, dtype=np.float32)
    yp = np.array(ypoints, dtype=np.float32)
    nb = len(xp)
    ph = np.zeros((nb, ns))
    bg = np.zeros(nb)
    pt = np.zeros((nb, ns, size_patch, size_patch))
    poly = np.zeros((W, H))
    rc = lib().orc_calib_init(_p(raw), ns, W, H, _p(xp), _p(yp), nb, size_patch, adu, gain, offset, zstep, _p(ph),
                              _p(bg), _p(pt), _p(poly))
    if rc:
        raise ValueError("singular background fit")
    return dict(x=xp, y=yp, background=bg, photons=ph, patches=pt, surface=poly)


def drift(xyz_nm, frame, crlb_nm=None, pixel_nm=10.0, bins=20, max_drift_um=0.5):
    """DriftCorrection restated: (bin_drift (bins, 4), per-localization drift (n, 3), voxel size used)."""
    xyz = _f64(xyz_nm)
    fr = np.ascontiguousarray(frame, dtype=np.int32)
    cr = None if crlb_nm is None else _f64(crlb_nm)
    n = len(fr)
    out_b = np.zeros((bins, 4))
    out_l = np.zeros((n, 3))
    px = np.zeros(1)
    rc = lib().orc_drift(_p(xyz), _p(cr) if cr is not None else None, _p(fr), n, pixel_nm, bins, max_drift_um,
                         _p(out_b), _p(out_l), _p(px))
    if rc:
        raise ValueError("bad drift arguments")
    return out_b, out_l, px[0]
