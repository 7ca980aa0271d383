"""Host-side mirror of ZOLA-3D's GPU localization objects over the C-ABI.

The reference drives its GPU path through Java objects (paths relative to its
src/main/java/org/pasteur/imagej/):

  DataPhase_ / DataPhase.loadJSON   process/gpu/DataPhase_.java, process/cpu/DataPhase.java:587-679
  PSFmany_float_.computePSF         process/gpu/PSFmany_float_.java:1626-1720
  Localization_.localize            process/gpu/Localization_.java:633-798

This module exposes the same roles over ``libzola_b200.so`` (include/zola_b200.h):
``Context`` (MyCudaStream), ``PSF`` (DataPhase_ + its model), ``PSF.model``
(computePSF) and ``PSF.fit`` (batched localize).  Host arrays are numpy; the
``*_dev`` forms take torch CUDA tensors and pass raw device pointers.  There is
no CPU fallback: if the library is missing every call raises.
"""
import ctypes
import json
import os
import weakref

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libzola_b200.so")

ZOLA_PREC_FP64 = 0
ZOLA_PREC_SPLIT = 1
ZOLA_SPLIT_STAGED = 0
ZOLA_SPLIT_FUSED = 1
ZOLA_SPLIT_FLOW = 2
ZOLA_CENTER_CPU = 0
ZOLA_CENTER_GPU = 1
FIT_STATUS = {1: "converged", 2: "max_iter", 3: "stalled", -1: "nan"}


class ZolaError(RuntimeError):
    pass


class Optics(ctypes.Structure):
    _fields_ = [("size_fft", ctypes.c_int), ("xystep", ctypes.c_double), ("na", ctypes.c_double),
                ("wavelength", ctypes.c_double), ("n_oil", ctypes.c_double), ("n_wat", ctypes.c_double),
                ("sigma", ctypes.c_double), ("with_apo", ctypes.c_int), ("zfocus", ctypes.c_double),
                ("kz_reset", ctypes.c_int)]


class Localization(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int), ("frame", ctypes.c_int), ("x_nm", ctypes.c_double), ("y_nm", ctypes.c_double),
                ("z_nm", ctypes.c_double), ("intensity", ctypes.c_double), ("background", ctypes.c_double),
                ("chi2", ctypes.c_double), ("crlb_x_nm", ctypes.c_double), ("crlb_y_nm", ctypes.c_double),
                ("crlb_z_nm", ctypes.c_double), ("candidate", ctypes.c_int), ("fit_status", ctypes.c_int)]


class LocParams(ctypes.Structure):
    _fields_ = [("patch", ctypes.c_int), ("minZ", ctypes.c_double), ("maxZ", ctypes.c_double),
                ("photon_threshold", ctypes.c_double), ("max_snr", ctypes.c_double), ("max_iter", ctypes.c_int),
                ("tol_xyz", ctypes.c_double), ("precision", ctypes.c_int), ("cand_cap", ctypes.c_int),
                ("frames_per_batch", ctypes.c_int), ("wave_fits", ctypes.c_int)]


class FitParams(ctypes.Structure):
    _fields_ = [("zmin", ctypes.c_double), ("zmax", ctypes.c_double), ("xymax", ctypes.c_double),
                ("max_iter", ctypes.c_int), ("tol_xyz", ctypes.c_double), ("step_xy", ctypes.c_double),
                ("step_z", ctypes.c_double), ("precision", ctypes.c_int)]


class FitClass(ctypes.Structure):
    _fields_ = [("psf", ctypes.c_void_p), ("R", ctypes.c_int), ("n", ctypes.c_int), ("d_rois", ctypes.c_void_p),
                ("d_init5", ctypes.c_void_p), ("prm", FitParams), ("d_out5", ctypes.c_void_p),
                ("d_crlb5", ctypes.c_void_p), ("d_nll", ctypes.c_void_p), ("d_status", ctypes.c_void_p),
                ("d_iters", ctypes.c_void_p)]


EXPORTS = ["zola_ctx_create", "zola_ctx_destroy", "zola_last_error", "zola_ctx_stream", "zola_ctx_launches",
           "zola_ctx_set_pool", "zola_psf_load", "zola_psf_free", "zola_psf_info", "zola_psf_model",
           "zola_psf_model_dev", "zola_psf_model_prec", "zola_psf_model_prec_dev", "zola_fit_batch",
           "zola_fit_batch_dev", "zola_ctx_profile", "zola_ctx_stage_stats", "zola_fit_batch_noalloc",
           "zola_detector_create", "zola_detector_free", "zola_detector_info", "zola_detect", "zola_detect_dev",
           "zola_localize_frames", "zola_write_csv", "zola_format_double_java", "zola_calib_forward",
           "zola_calib_backward", "zola_calib_fit", "zola_ctx_set_split_mode", "zola_crlb_curve",
           "zola_psf_center_search", "zola_calib_init", "zola_drift", "zola_fit_batch_scmos",
           "zola_fit_batch_scmos_dev", "zola_localize_frames_scmos", "zola_ctx_set_flow", "zola_ctx_set_wait_limit",
           "zola_fit_batch_stream_dev", "zola_ctx_set_tuning", "zola_fit_flow_shape", "zola_ctx_flow_stats",
           "zola_fit_batch_mixed_dev", "zola_detect_u16", "zola_localize_frames_u16", "zola_fit_split_pool",
           "zola_ctx_set_round_graphs", "zola_fit_batch_mixed"]
STAGES = ["split_stage1_pupil_dft", "split_stage2_window_dft", "split_stage3_blur_rows",
          "split_stage4_blur_cols_sums_lm", "split_fused_stages2_5", "fp64_fit", "fp64_model", "other",
          "split_dataflow", "detect"]

_lib = None


def lib():
    """Load libzola_b200.so (built by build.py); raises if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ZolaError(f"{LIB_PATH} not built: run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.zola_ctx_create.argtypes = [i, ctypes.POINTER(vp)]
        L.zola_ctx_destroy.argtypes = [vp]
        L.zola_last_error.argtypes = [vp]
        L.zola_last_error.restype = ctypes.c_char_p
        L.zola_ctx_stream.argtypes = [vp]
        L.zola_ctx_stream.restype = vp
        L.zola_ctx_launches.argtypes = [vp]
        L.zola_ctx_launches.restype = ctypes.c_longlong
        L.zola_psf_load.argtypes = [vp, ctypes.POINTER(Optics), vp, i, ctypes.POINTER(vp)]
        L.zola_psf_free.argtypes = [vp]
        L.zola_psf_info.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(i)]
        L.zola_psf_model.argtypes = [vp, i, vp, i, vp, vp]
        L.zola_psf_model_dev.argtypes = [vp, i, vp, i, vp, vp, vp]
        L.zola_psf_model_prec.argtypes = [vp, i, vp, i, vp, vp, i]
        L.zola_psf_model_prec_dev.argtypes = [vp, i, vp, i, vp, vp, i, vp]
        L.zola_ctx_set_pool.argtypes = [vp, i]
        L.zola_ctx_set_split_mode.argtypes = [vp, i]
        L.zola_ctx_set_flow.argtypes = [vp, i, vp]
        L.zola_ctx_set_wait_limit.argtypes = [vp, ctypes.c_longlong]
        L.zola_ctx_set_tuning.argtypes = [vp, i, ctypes.c_char_p]
        L.zola_fit_flow_shape.argtypes = [vp, i, vp, vp, vp]
        L.zola_ctx_flow_stats.argtypes = [vp, vp, vp, vp]
        L.zola_fit_split_pool.argtypes = [vp, i, vp, vp]
        L.zola_ctx_set_round_graphs.argtypes = [vp, i]
        L.zola_fit_batch_mixed_dev.argtypes = [vp, vp, i, vp]
        L.zola_fit_batch_mixed.argtypes = [vp, vp, i]
        L.zola_crlb_curve.argtypes = [vp, i, vp, i, d, d, d, d, vp]
        L.zola_psf_center_search.argtypes = [vp, i, d, i, ctypes.POINTER(d)]
        L.zola_ctx_profile.argtypes = [vp, i]
        L.zola_detector_create.argtypes = [vp, i, i, i, d, d, d, d, ctypes.POINTER(vp)]
        L.zola_localize_frames.argtypes = [vp, vp, vp, vp, i, i, ctypes.POINTER(LocParams), vp, i, ctypes.POINTER(i)]
        L.zola_write_csv.argtypes = [ctypes.c_char_p, vp, i, i]
        L.zola_calib_forward.argtypes = [vp, ctypes.POINTER(CalibData), vp, d, vp, vp, vp]
        L.zola_calib_backward.argtypes = [vp, ctypes.POINTER(CalibData), vp, d, vp, vp, vp, vp, vp]
        L.zola_calib_fit.argtypes = [vp, ctypes.POINTER(CalibData), vp, vp, vp, i, i, vp, vp]
        L.zola_calib_init.argtypes = [vp, vp, i, i, i, vp, vp, i, i, d, d, d, d, vp, vp, vp, vp]
        L.zola_fit_batch_scmos.argtypes = [vp, vp, i, vp, vp, vp, i, ctypes.POINTER(FitParams), vp, vp, vp, vp, vp]
        L.zola_fit_batch_scmos_dev.argtypes = [vp, vp, i, vp, vp, vp, i, ctypes.POINTER(FitParams), vp, vp, vp, vp,
                                               vp, vp]
        L.zola_localize_frames_scmos.argtypes = [vp, vp, vp, vp, i, i, ctypes.POINTER(LocParams), vp, vp, vp, vp, i,
                                                 ctypes.POINTER(i)]
        L.zola_drift.argtypes = [vp, vp, vp, vp, i, ctypes.POINTER(DriftParams), vp, vp, ctypes.POINTER(d)]
        L.zola_format_double_java.argtypes = [d, ctypes.c_char_p, i]
        L.zola_detector_free.argtypes = [vp]
        L.zola_detector_info.argtypes = [vp, ctypes.POINTER(i), vp, vp]
        L.zola_detect.argtypes = [vp, vp, i, i, vp, vp]
        L.zola_detect_u16.argtypes = [vp, vp, i, i, d, d, d, vp, vp]
        L.zola_localize_frames_u16.argtypes = [vp, vp, vp, vp, i, i, ctypes.POINTER(LocParams), d, d, d, vp, i,
                                               ctypes.POINTER(i)]
        L.zola_detect_dev.argtypes = [vp, vp, i, i, vp, vp, vp]
        L.zola_fit_batch_noalloc.argtypes = [vp, i, vp, vp, i, ctypes.POINTER(FitParams), vp, vp, vp, vp, vp, vp]
        L.zola_ctx_stage_stats.argtypes = [vp, vp, vp, i]
        L.zola_fit_batch.argtypes = [vp, vp, i, vp, vp, i, ctypes.POINTER(FitParams), vp, vp, vp, vp, vp]
        L.zola_fit_batch_dev.argtypes = [vp, vp, i, vp, vp, i, ctypes.POINTER(FitParams), vp, vp, vp, vp, vp, vp]
        L.zola_fit_batch_stream_dev.argtypes = [vp, vp, i, vp, vp, vp, i, ctypes.POINTER(FitParams), vp, vp, vp, vp, vp,
                                                vp]
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


class Context:
    """One device context and stream (replaces MyCudaStream.init/destroy)."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        rc = lib().zola_ctx_create(int(device), ctypes.byref(h))
        if rc != 0:
            raise ZolaError(f"zola_ctx_create failed ({rc}): no usable sm_100 device {device}")
        self.h = h
        self.device = device
        self._psfs = weakref.WeakSet()

    def check(self, rc, what):
        if rc != 0:
            msg = lib().zola_last_error(self.h).decode()
            raise ZolaError(f"{what} failed ({rc}): {msg}")

    @property
    def stream(self):
        return lib().zola_ctx_stream(self.h)

    def set_pool(self, max_slots):
        """Bound the split fit's slot pool (ROIs in flight); 0 = automatic."""
        self.check(lib().zola_ctx_set_pool(self.h, int(max_slots)), "zola_ctx_set_pool")

    def set_split_mode(self, mode):
        """"staged" (default): five stage kernels per LM round; "flow": the whole split fit as one dataflow
        kernel (the same results bit for bit); "fused": stage 1 + one kernel for stages 2-5."""
        code = {"staged": ZOLA_SPLIT_STAGED, "fused": ZOLA_SPLIT_FUSED, "flow": ZOLA_SPLIT_FLOW}[mode]
        self.check(lib().zola_ctx_set_split_mode(self.h, code), "zola_ctx_set_split_mode")

    def set_flow(self, units=0, ctas=None):
        """Dataflow kernel shape: units of slots in flight (0: automatic) and CTAs per stage (None:
        automatic; else five counts adding up to the SM count).  Results do not depend on either."""
        arr = None if ctas is None else (ctypes.c_int * 5)(*[int(c) for c in ctas])
        self.check(lib().zola_ctx_set_flow(self.h, int(units), arr), "zola_ctx_set_flow")

    def set_round_graphs(self, enable=True):
        """Replay the round-based split kernels' 4-round blocks as CUDA graphs (default) or launch them one by one."""
        self.check(lib().zola_ctx_set_round_graphs(self.h, int(bool(enable))), "zola_ctx_set_round_graphs")

    def set_tuning(self, enable=True, cache_path=None):
        """Autotune the dataflow kernel's shape per (pupil grid, ROI side) on large fits; cache_path: JSON cache."""
        self.check(lib().zola_ctx_set_tuning(self.h, int(bool(enable)), cache_path.encode() if cache_path else None),
                   "zola_ctx_set_tuning")

    def flow_stats(self):
        """Last dataflow fit: per stage busy fraction and busy clocks per unit, and the evaluations made."""
        busy = np.zeros(5)
        cpu = np.zeros(5)
        ev = ctypes.c_double()
        self.check(lib().zola_ctx_flow_stats(self.h, _ptr(busy), _ptr(cpu), ctypes.byref(ev)), "zola_ctx_flow_stats")
        return {"busy": busy.tolist(), "clocks_per_unit": cpu.tolist(), "evaluations": ev.value}

    def set_wait_limit(self, clocks):
        """Upper bound (GPU clocks) on the dataflow kernel's waits for a ready unit; 0 = default (2^31)."""
        self.check(lib().zola_ctx_set_wait_limit(self.h, int(clocks)), "zola_ctx_set_wait_limit")

    def profile(self, enable=True):
        """Time every library kernel launch with CUDA events on its stream."""
        self.check(lib().zola_ctx_profile(self.h, int(bool(enable))), "zola_ctx_profile")

    def stage_stats(self, reset=False):
        """{stage: (total device ms, launches)} accumulated while profiling."""
        ms = np.zeros(len(STAGES))
        n = np.zeros(len(STAGES), np.int64)
        self.check(lib().zola_ctx_stage_stats(self.h, _ptr(ms), _ptr(n), int(bool(reset))), "zola_ctx_stage_stats")
        return {s: (float(ms[k]), int(n[k])) for k, s in enumerate(STAGES)}

    @property
    def launches(self):
        return lib().zola_ctx_launches(self.h)

    def close(self):
        if getattr(self, "h", None):
            for p in list(self._psfs):
                p.close()
            lib().zola_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def optics(size_fft=128, xystep=0.11, na=1.4, wavelength=0.66, n_oil=1.518, n_wat=None, sigma=0.9,
           with_apo=False, zfocus=0.0, kz_reset=False):
    return Optics(int(size_fft), float(xystep), float(na), float(wavelength), float(n_oil),
                  float(n_oil if n_wat is None else n_wat), float(sigma), int(bool(with_apo)), float(zfocus),
                  int(bool(kz_reset)))


class PSF:
    """A loaded calibration: pupil tables, Zernike phase and per-ROI-size tables
    on the device (replaces DataPhase_ + PSFmany_float_)."""

    def __init__(self, ctx, opt, zernike):
        self.ctx = ctx
        self.optics = opt
        self.zernike = np.ascontiguousarray(zernike, dtype=np.float64)
        h = ctypes.c_void_p()
        ctx.check(lib().zola_psf_load(ctx.h, ctypes.byref(opt), _ptr(self.zernike), len(self.zernike),
                                      ctypes.byref(h)), "zola_psf_load")
        self.h = h
        ctx._psfs.add(self)
        n, k = ctypes.c_int(), ctypes.c_int()
        lib().zola_psf_info(h, ctypes.byref(n), ctypes.byref(k))
        self.N, self.K = n.value, k.value

    def close(self):
        if getattr(self, "h", None):
            if getattr(self.ctx, "h", None):  # the context frees its PSFs first on close
                lib().zola_psf_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def model(self, R, xyz, derivs=False, precision=ZOLA_PREC_FP64):
        """psi (n, R, R) (and dpsi (n, 3, R, R)) at (x, y, zwat) um on the GPU
        (FP64 CUDA cores, or the tcgen05 split-precision stages)."""
        xyz = np.ascontiguousarray(np.atleast_2d(xyz), dtype=np.float64)
        n = xyz.shape[0]
        out = np.zeros((n, R, R))
        d = np.zeros((n, 3, R, R)) if derivs else None
        self.ctx.check(lib().zola_psf_model_prec(self.h, int(R), _ptr(xyz), n, _ptr(out), _ptr(d), int(precision)),
                       "zola_psf_model_prec")
        return (out, d) if derivs else out

    def model_dev(self, R, xyz, out, dout=None, stream=None):
        """Device form: torch CUDA float64 tensors."""
        n = xyz.shape[0]
        self.ctx.check(lib().zola_psf_model_dev(self.h, int(R), _ptr(xyz), n, _ptr(out), _ptr(dout), stream),
                       "zola_psf_model_dev")

    @staticmethod
    def fit_params(zmin, zmax, xymax, max_iter=30, tol_xyz=1e-5, step_xy=0.11, step_z=0.22,
                   precision=ZOLA_PREC_FP64):
        return FitParams(float(zmin), float(zmax), float(xymax), int(max_iter), float(tol_xyz), float(step_xy),
                         float(step_z), int(precision))

    def fit(self, rois, init, prm, crlb=True, scmos=None, out=None):
        """Batched MLE fit of host ROIs (n, R, R) photons from init (n, 5) = x, y, z, A, B.
        scmos (n, R, R), optional: var/gain^2 of each ROI pixel, added to the model mean.
        out, optional: the result arrays to fill in place, a dict with theta (n, 5) and crlb
        (n, 5) float64 (crlb may be None), nll (n,) float64, status and iters (n,) int32, all
        C-contiguous; views of pinned host memory make the device-to-host copy direct."""
        rois = np.ascontiguousarray(rois, dtype=np.float32)
        init = np.ascontiguousarray(init, dtype=np.float64)
        n, R = rois.shape[0], rois.shape[1]
        if out is None:
            res = dict(theta=np.zeros((n, 5)), crlb=np.zeros((n, 5)) if crlb else None, nll=np.zeros(n),
                       status=np.zeros(n, np.int32), iters=np.zeros(n, np.int32))
        else:
            res = out
            for k, shape, dt in (("theta", (n, 5), np.float64), ("crlb", (n, 5), np.float64),
                                 ("nll", (n,), np.float64), ("status", (n,), np.int32), ("iters", (n,), np.int32)):
                a = res.get(k)
                if a is None and k == "crlb":
                    continue
                if a is None or a.shape != shape or a.dtype != dt or not a.flags["C_CONTIGUOUS"]:
                    raise ValueError(f"out[{k!r}] must be a C-contiguous {np.dtype(dt).name} array of shape {shape}")
        args = (_ptr(res["theta"]), _ptr(res["crlb"]), _ptr(res["nll"]), _ptr(res["status"]), _ptr(res["iters"]))
        if scmos is None:
            self.ctx.check(lib().zola_fit_batch(self.ctx.h, self.h, R, _ptr(rois), _ptr(init), n, ctypes.byref(prm),
                                                *args), "zola_fit_batch")
        else:
            v = np.ascontiguousarray(scmos, dtype=np.float32)
            self.ctx.check(lib().zola_fit_batch_scmos(self.ctx.h, self.h, R, _ptr(rois), _ptr(v), _ptr(init), n,
                                                      ctypes.byref(prm), *args), "zola_fit_batch_scmos")
        return res

    def fit_dev(self, rois, init, prm, out, crlb=None, nll=None, status=None, iters=None, stream=None):
        """Device form over torch CUDA tensors (rois float32, init/out float64).
        stream: a cudaStream_t handle; None runs on the context's stream, which
        CUDA orders with the default stream (torch's default stream)."""
        n, R = rois.shape[0], rois.shape[1]
        self.ctx.check(lib().zola_fit_batch_dev(self.ctx.h, self.h, R, _ptr(rois), _ptr(init), n, ctypes.byref(prm),
                                                _ptr(out), _ptr(crlb), _ptr(nll), _ptr(status), _ptr(iters), stream),
                       "zola_fit_batch_dev")

    def flow_shape(self, R):
        """(tuned, units, [CTAs per stage], ns per evaluation) of the dataflow kernel for R x R ROIs."""
        u = ctypes.c_int()
        c = (ctypes.c_int * 5)()
        ns = ctypes.c_double()
        rc = lib().zola_fit_flow_shape(self.h, int(R), ctypes.byref(u), c, ctypes.byref(ns))
        if rc < 0:
            self.ctx.check(rc, "zola_fit_flow_shape")
        return bool(rc), u.value, list(c), ns.value

    def split_pool(self, R):
        """(tuned, pool slots, ns per evaluation) of the round-based split fit for R x R ROIs."""
        pool = ctypes.c_int()
        ns = ctypes.c_double()
        rc = lib().zola_fit_split_pool(self.h, int(R), ctypes.byref(pool), ctypes.byref(ns))
        if rc < 0:
            self.ctx.check(rc, "zola_fit_split_pool")
        return bool(rc), pool.value, ns.value

    def fit_stream_dev(self, rois, init, avail, prm, out, crlb=None, nll=None, status=None, iters=None, stream=None):
        """Streaming device form (zola_fit_batch_stream_dev): avail is a one-element int32 CUDA tensor holding
        how many leading ROIs of rois are already written; the producer raises it while the fit runs."""
        n, R = rois.shape[0], rois.shape[1]
        self.ctx.check(lib().zola_fit_batch_stream_dev(self.ctx.h, self.h, R, _ptr(rois), _ptr(init), _ptr(avail), n,
                                                       ctypes.byref(prm), _ptr(out), _ptr(crlb), _ptr(nll),
                                                       _ptr(status), _ptr(iters), stream),
                       "zola_fit_batch_stream_dev")

    def crlb_curve(self, R, z, photons=3000.0, background=50.0, h=0.0005, a_step=0.0005):
        """CRLB (x, y, z, A, B) at (0, 0, z) for each depth, finite-difference
        Fisher matrix (CRLB.computeFisher; defaults are CRLB.run's h = 0.5 nm)."""
        z = np.ascontiguousarray(np.atleast_1d(z), dtype=np.float64)
        out = np.zeros((len(z), 5))
        self.ctx.check(lib().zola_crlb_curve(self.h, int(R), _ptr(z), len(z), float(photons), float(background),
                                             float(h), float(a_step), _ptr(out)), "zola_crlb_curve")
        return out

    def center_search(self, axial_range, R=None, variant=ZOLA_CENTER_CPU):
        """SearchPSFcenter.getPosition: the ZfocusCenter depth (um) for an axial range (um)."""
        zc = ctypes.c_double()
        self.ctx.check(lib().zola_psf_center_search(self.h, int(R or self.N), float(axial_range), int(variant),
                                                    ctypes.byref(zc)), "zola_psf_center_search")
        return zc.value


class Detector:
    """PSF-library NCC detection (Predetection / Predetection_cross_).

    psf must be built with kz_reset=True (the reference builds the library from
    its resetKz tables).  Frames are (n, SX, SY) photons, first index x."""

    def __init__(self, psf, SX, SY, R, minZ, maxZ, step, thr=0.1):
        self.psf, self.SX, self.SY, self.R = psf, SX, SY, R
        h = ctypes.c_void_p()
        psf.ctx.check(lib().zola_detector_create(psf.h, SX, SY, R, minZ, maxZ, step, thr, ctypes.byref(h)),
                      "zola_detector_create")
        self.h = h
        nz = ctypes.c_int()
        lib().zola_detector_info(h, ctypes.byref(nz), None, None)
        self.nz = nz.value

    def library(self):
        rng = np.zeros(self.nz)
        psfs = np.zeros((self.nz, self.R, self.R))
        lib().zola_detector_info(self.h, ctypes.byref(ctypes.c_int()), _ptr(rng), _ptr(psfs))
        return rng, psfs

    def detect(self, frames, cap=2048):
        frames = np.ascontiguousarray(frames, dtype=np.float64)
        nf = frames.shape[0]
        out = np.zeros((nf, cap, 7))
        counts = np.zeros(nf, np.int32)
        self.psf.ctx.check(lib().zola_detect(self.h, _ptr(frames), nf, cap, _ptr(out), _ptr(counts)), "zola_detect")
        return [out[f, :min(cap, counts[f])] for f in range(nf)], counts

    def detect_u16(self, frames, adu=1.0, gain=1.0, offset=0.0, cap=2048):
        """detect() on uint16 camera frames, converted to photons on the device."""
        frames = np.ascontiguousarray(frames, dtype=np.uint16)
        nf = frames.shape[0]
        out = np.zeros((nf, cap, 7))
        counts = np.zeros(nf, np.int32)
        self.psf.ctx.check(lib().zola_detect_u16(self.h, _ptr(frames), nf, cap, float(adu), float(gain), float(offset),
                                                 _ptr(out), _ptr(counts)), "zola_detect_u16")
        return [out[f, :min(cap, counts[f])] for f in range(nf)], counts

    def detect_dev(self, frames, cap, out, counts, stream=None):
        self.psf.ctx.check(lib().zola_detect_dev(self.h, _ptr(frames), frames.shape[0], cap, _ptr(out), _ptr(counts),
                                                 stream), "zola_detect_dev")

    def close(self):
        if getattr(self, "h", None) and getattr(self.psf, "h", None):
            lib().zola_detector_free(self.h)
        self.h = None


class DriftParams(ctypes.Structure):
    _fields_ = [("pixel_nm", ctypes.c_double), ("bins", ctypes.c_int), ("max_drift_um", ctypes.c_double)]


def drift(ctx, xyz_nm, frame, crlb_nm=None, pixel_nm=10.0, bins=20, max_drift_um=0.5):
    """DriftCorrection: returns (bin_drift (bins, 4) = frame index, dx, dy, dz nm,
    per-localization drift (n, 3) nm, voxel size used)."""
    xyz = np.ascontiguousarray(xyz_nm, dtype=np.float64)
    fr = np.ascontiguousarray(frame, dtype=np.int32)
    cr = None if crlb_nm is None else np.ascontiguousarray(crlb_nm, dtype=np.float64)
    n = len(fr)
    out_b = np.zeros((int(bins), 4))
    out_l = np.zeros((n, 3))
    px = ctypes.c_double()
    prm = DriftParams(float(pixel_nm), int(bins), float(max_drift_um))
    ctx.check(lib().zola_drift(ctx.h, _ptr(xyz), _ptr(cr), _ptr(fr), n, ctypes.byref(prm), _ptr(out_b), _ptr(out_l),
                               ctypes.byref(px)), "zola_drift")
    return out_b, out_l, px.value


class CalibData(ctypes.Structure):
    _fields_ = [("R", ctypes.c_int), ("nz", ctypes.c_int), ("nbead", ctypes.c_int), ("nslice", ctypes.c_int),
                ("dz", ctypes.c_void_p), ("stacks", ctypes.c_void_p), ("photons", ctypes.c_void_p)]


ZOLA_CALIB_FIT_SIGMA = 1
NPOLY = 6


def calib_init(ctx, raw, xpoints, ypoints, size_patch, adu=1.0, gain=1.0, offset=0.0, zstep=0.05):
    """InitBackgroundAndPhotonNumber: raw stack (nslice, W, H) ADU -> dict with
    refined seeds x/y (pixels), background (nbead,), photons (nbead, nslice),
    patches (nbead, nslice, size_patch, size_patch) and the (W, H) surface."""
    raw = np.ascontiguousarray(raw, dtype=np.float32)
    ns, W, H = raw.shape
    xp = np.array(xpoints, dtype=np.float32)
    yp = np.array(ypoints, dtype=np.float32)
    nb = len(xp)
    ph = np.zeros((nb, ns))
    bg = np.zeros(nb)
    pt = np.zeros((nb, ns, size_patch, size_patch))
    poly = np.zeros((W, H))
    ctx.check(lib().zola_calib_init(ctx.h, _ptr(raw), ns, W, H, _ptr(xp), _ptr(yp), nb, int(size_patch), float(adu),
                                    float(gain), float(offset), float(zstep), _ptr(ph), _ptr(bg), _ptr(pt),
                                    _ptr(poly)), "zola_calib_init")
    return dict(x=xp, y=yp, background=bg, photons=ph, patches=pt, surface=poly)


class Calibration:
    """Bead z-stack calibration (ZernikePhaseRetrieval) on a kz_reset=False PSF.

    stacks: (nbead, nslice, R, R) photons; dz: (nslice,) slice positions (um);
    photons: (nbead, nslice) photon curve from calib_init (or None);
    zernike: (nz,) radians (modes 0-2 unused); sigma: blur width (px);
    bead: (nbead, 3 + nslice + 6) = x, y, z, a[nslice], c[6] (see bead_params)."""

    def __init__(self, psf, stacks, dz, photons=None, nz=None):
        self.psf = psf
        self.stacks = np.ascontiguousarray(stacks, dtype=np.float64)
        self.dz = np.ascontiguousarray(dz, dtype=np.float64)
        self.nb, self.ns, self.R = self.stacks.shape[0], self.stacks.shape[1], self.stacks.shape[2]
        self.photons = None if photons is None else np.ascontiguousarray(photons, dtype=np.float64)
        self.nz = nz

    def _data(self, nz):
        return CalibData(self.R, int(nz), self.nb, self.ns, self.dz.ctypes.data, self.stacks.ctypes.data,
                         None if self.photons is None else self.photons.ctypes.data)

    def bead_params(self, xyz=None, a=None, background=None):
        """Bead parameter array: xyz (nbead, 3), a (nbead, nslice) photon offsets,
        background (nbead,) constant term of the polynomial."""
        b = np.zeros((self.nb, 3 + self.ns + NPOLY))
        if xyz is not None:
            b[:, :3] = xyz
        if a is not None:
            b[:, 3:3 + self.ns] = a
        if background is not None:
            b[:, 3 + self.ns] = background
        return b

    def forward(self, zernike, sigma, bead, model=False):
        z = np.ascontiguousarray(zernike, dtype=np.float64)
        b = np.ascontiguousarray(bead, dtype=np.float64)
        nll = np.zeros(1)
        m = np.zeros_like(self.stacks) if model else None
        data = self._data(len(z))
        self.psf.ctx.check(lib().zola_calib_forward(self.psf.h, ctypes.byref(data), _ptr(z), float(sigma), _ptr(b),
                                                    _ptr(nll), _ptr(m)), "zola_calib_forward")
        return (nll[0], m) if model else nll[0]

    def backward(self, zernike, sigma, bead):
        z = np.ascontiguousarray(zernike, dtype=np.float64)
        b = np.ascontiguousarray(bead, dtype=np.float64)
        nll = np.zeros(1)
        gz = np.zeros(len(z))
        gs = np.zeros(1)
        gb = np.zeros_like(b)
        data = self._data(len(z))
        self.psf.ctx.check(lib().zola_calib_backward(self.psf.h, ctypes.byref(data), _ptr(z), float(sigma), _ptr(b),
                                                     _ptr(nll), _ptr(gz), _ptr(gs), _ptr(gb)), "zola_calib_backward")
        return nll[0], gz, gs[0], gb

    def fit(self, zernike, sigma, bead, max_iter=30, fit_sigma=True):
        z = np.array(zernike, dtype=np.float64)
        sg = np.array([sigma], dtype=np.float64)
        b = np.array(bead, dtype=np.float64)
        nll = np.zeros(1)
        it = ctypes.c_int()
        data = self._data(len(z))
        self.psf.ctx.check(lib().zola_calib_fit(self.psf.h, ctypes.byref(data), _ptr(z), _ptr(sg), _ptr(b),
                                                int(max_iter), ZOLA_CALIB_FIT_SIGMA if fit_sigma else 0, _ptr(nll),
                                                ctypes.byref(it)), "zola_calib_fit")
        return z, sg[0], b, nll[0], it.value


LOC_COLUMNS = ["id", "frame", "x_nm", "y_nm", "z_nm", "intensity", "background", "chi2", "crlb_x_nm", "crlb_y_nm",
               "crlb_z_nm", "candidate", "fit_status"]


LOC_DTYPE = np.dtype([(c, np.int32 if c in ("id", "frame", "candidate", "fit_status") else np.float64)
                      for c in LOC_COLUMNS])
assert LOC_DTYPE.itemsize == ctypes.sizeof(Localization)  # the packed dtype is the C struct's layout


def _loc_params(det, minZ, maxZ, photon_threshold, max_snr, max_iter, tol_xyz, precision, cand_cap,
                frames_per_batch, wave_fits):
    return LocParams(det.R, float(minZ), float(maxZ), float(photon_threshold), float(max_snr), int(max_iter),
                     float(tol_xyz), int(precision), int(cand_cap), int(frames_per_batch), int(wave_fits))


def _loc_rows(ctx, nf, call, name):
    """Run one pipeline entry point into a row buffer and return its rows as a
    structured array (LOC_DTYPE; the buffer is the C array itself)."""
    cap = max(64, nf * 64)
    out = np.empty(cap, dtype=LOC_DTYPE)
    n = ctypes.c_int()
    ctx.check(call(out.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(n)), name)
    return out[:n.value].copy()


def localize_frames(ctx, det, fit_psf, frames, minZ, maxZ, photon_threshold=500.0, max_snr=1.0, max_iter=30,
                    tol_xyz=1e-4, precision=ZOLA_PREC_FP64, frame0=0, cand_cap=0, frames_per_batch=1024, wave_fits=0):
    """Detect and localize every frame (LocalizationPipeline): returns a
    structured numpy array with LOC_COLUMNS, one row per localization."""
    frames = np.ascontiguousarray(frames, dtype=np.float64)
    nf = frames.shape[0]
    prm = _loc_params(det, minZ, maxZ, photon_threshold, max_snr, max_iter, tol_xyz, precision, cand_cap,
                      frames_per_batch, wave_fits)
    return _loc_rows(ctx, nf, lambda out, cap, n: lib().zola_localize_frames(
        ctx.h, det.h, fit_psf.h, _ptr(frames), nf, int(frame0), ctypes.byref(prm), out, cap, n),
        "zola_localize_frames")


def localize_frames_u16(ctx, det, fit_psf, frames, minZ, maxZ, adu=1.0, gain=1.0, offset=0.0, photon_threshold=500.0,
                        max_snr=1.0, max_iter=30, tol_xyz=1e-4, precision=ZOLA_PREC_FP64, frame0=0, cand_cap=0,
                        frames_per_batch=1024, wave_fits=0):
    """The pipeline on uint16 camera frames (n, SX, SY), converted to photons on
    the device as count * adu / gain - offset * adu / gain, clamped at 0."""
    frames = np.ascontiguousarray(frames, dtype=np.uint16)
    nf = frames.shape[0]
    prm = _loc_params(det, minZ, maxZ, photon_threshold, max_snr, max_iter, tol_xyz, precision, cand_cap,
                      frames_per_batch, wave_fits)
    return _loc_rows(ctx, nf, lambda out, cap, n: lib().zola_localize_frames_u16(
        ctx.h, det.h, fit_psf.h, _ptr(frames), nf, int(frame0), ctypes.byref(prm), float(adu), float(gain),
        float(offset), out, cap, n), "zola_localize_frames_u16")


def localize_frames_scmos(ctx, det, fit_psf, adu, offset, gain, variance, minZ, maxZ, photon_threshold=500.0,
                          max_snr=1.0, max_iter=30, tol_xyz=1e-4, precision=ZOLA_PREC_FP64, frame0=0, cand_cap=0,
                          frames_per_batch=1024, wave_fits=0):
    """sCMOS pipeline: ADU frames (n, SX, SY) and offset / gain / variance maps (SX, SY)."""
    adu = np.ascontiguousarray(adu, dtype=np.float32)
    maps = [np.ascontiguousarray(m, dtype=np.float64) for m in (offset, gain, variance)]
    nf = adu.shape[0]
    prm = _loc_params(det, minZ, maxZ, photon_threshold, max_snr, max_iter, tol_xyz, precision, cand_cap,
                      frames_per_batch, wave_fits)
    return _loc_rows(ctx, nf, lambda out, cap, n: lib().zola_localize_frames_scmos(
        ctx.h, det.h, fit_psf.h, _ptr(adu), nf, int(frame0), ctypes.byref(prm), _ptr(maps[0]), _ptr(maps[1]),
        _ptr(maps[2]), out, cap, n), "zola_localize_frames_scmos")


def write_csv(path, locs, append=False):
    """ThunderStorm-style CSV exactly as ZOLA writes it (zola_write_csv)."""
    n = len(locs)
    buf = (Localization * max(1, n))()
    for k in range(n):
        for c in LOC_COLUMNS:
            setattr(buf[k], c, locs[k][c].item() if hasattr(locs[k][c], "item") else locs[k][c])
    rc = lib().zola_write_csv(path.encode(), ctypes.cast(buf, ctypes.c_void_p), n, int(bool(append)))
    if rc != 0:
        raise ZolaError(f"zola_write_csv failed ({rc}) for {path}")


def java_double(v):
    """Java Double.toString of v (the CSV number format)."""
    b = ctypes.create_string_buffer(64)
    if lib().zola_format_double_java(float(v), b, 64) != 0:
        raise ZolaError("zola_format_double_java failed")
    return b.value.decode()


def fit_mixed_dev(ctx, classes, stream=None):
    """Mixed batch (zola_fit_batch_mixed_dev): classes is a list of dicts with psf, rois (n, R, R) float32,
    init (n, 5) float64, prm (split precision), out (n, 5) and optional crlb, nll, status, iters, all torch
    CUDA tensors; every class is fitted in one call."""
    arr = (FitClass * max(1, len(classes)))()
    for k, c in enumerate(classes):
        rois = c["rois"]
        arr[k] = FitClass(c["psf"].h.value if hasattr(c["psf"].h, "value") else c["psf"].h, int(rois.shape[1]),
                          int(rois.shape[0]), rois.data_ptr(), c["init"].data_ptr(), c["prm"], c["out"].data_ptr(),
                          *[c[x].data_ptr() if c.get(x) is not None else None
                            for x in ("crlb", "nll", "status", "iters")])
    ctx.check(lib().zola_fit_batch_mixed_dev(ctx.h, ctypes.cast(arr, ctypes.c_void_p), len(classes), stream),
              "zola_fit_batch_mixed_dev")


def fit_mixed(ctx, classes):
    """Mixed batch from host memory (zola_fit_batch_mixed): classes is a list of dicts with psf, rois (n, R, R)
    float32, init (n, 5) float64, prm (split precision) and out, a dict of host result arrays as PSF.fit takes
    (theta (n, 5); crlb (n, 5), nll, status, iters optional).  Pinned arrays let the copies overlap the fits."""
    arr = (FitClass * max(1, len(classes)))()
    keep = []
    for k, c in enumerate(classes):
        rois = np.ascontiguousarray(c["rois"], dtype=np.float32)
        init = np.ascontiguousarray(c["init"], dtype=np.float64)
        keep += [rois, init]
        res = c["out"]
        n = rois.shape[0]
        for key, shape, dt in (("theta", (n, 5), np.float64), ("crlb", (n, 5), np.float64), ("nll", (n,), np.float64),
                               ("status", (n,), np.int32), ("iters", (n,), np.int32)):
            a = res.get(key)
            if a is None and key != "theta":
                continue
            if a is None or a.shape != shape or a.dtype != dt or not a.flags["C_CONTIGUOUS"]:
                raise ValueError(f"out[{key!r}] must be a C-contiguous {np.dtype(dt).name} array of shape {shape}")
        arr[k] = FitClass(c["psf"].h.value if hasattr(c["psf"].h, "value") else c["psf"].h, int(rois.shape[1]), n,
                          rois.ctypes.data, init.ctypes.data, c["prm"], res["theta"].ctypes.data,
                          *[res[x].ctypes.data if res.get(x) is not None else None
                            for x in ("crlb", "nll", "status", "iters")])
    ctx.check(lib().zola_fit_batch_mixed(ctx.h, ctypes.cast(arr, ctypes.c_void_p), len(classes)),
              "zola_fit_batch_mixed")


def fit_noalloc_dev(psf, rois, init, prm, out, crlb=None, nll=None, status=None, iters=None, stream=None):
    """Allocation-free FP64 fit (zola_fit_batch_noalloc) over torch CUDA tensors.

    For callers that must not allocate device memory while fitting: the work
    areas live in a fixed 64 MiB array inside the library on each GPU.  The
    PSF's tables for this ROI size must have been prepared by an earlier model
    or fit call with the same R; calls that overlap on the GPU race."""
    n, R = rois.shape[0], rois.shape[1]
    psf.ctx.check(lib().zola_fit_batch_noalloc(psf.h, R, _ptr(rois), _ptr(init), n, ctypes.byref(prm), _ptr(out),
                                               _ptr(crlb), _ptr(nll), _ptr(status), _ptr(iters), stream),
                  "zola_fit_batch_noalloc")


def load_calibration_json(path, size_fft=128, n_wat=None, zfocus=0.0, kz_reset=False):
    """Parse a ZOLA calibration JSON (DataPhase.loadJSON, process/cpu/DataPhase.java:587-679).

    Returns (optics, zernike).  As in the reference, the pupil grid is the
    caller's sizeFFT for Zernike calibrations and the file's for pixel phases;
    pixel-phase calibrations are not supported by this library."""
    with open(path) as f:
        js = json.load(f)
    if str(js.get("zernikedPSF", "true")).lower() != "true":
        raise ZolaError("pixel-phase (non-Zernike) calibrations are not supported")
    zern = np.array([float(v) for v in js["zernike"]])
    opt = optics(size_fft=size_fft, xystep=float(js["sizePix"]), na=float(js["NA"]),
                 wavelength=float(js["wavelength"]), n_oil=float(js["index"]), n_wat=n_wat,
                 sigma=float(js["sigmaGaussianKernel"]),
                 with_apo=str(js.get("withApoFactor", "false")).lower() == "true", zfocus=zfocus,
                 kz_reset=kz_reset)
    return opt, zern
