"""Benchmark: batched mixed-size Poisson MLE fits (split precision vs plain FP64 GPU).

Workload (one step): 1,000,000 synthetic ROIs, 50% 16x16 (astigmatic PSF, pupil
64^2), 30% 24x24 (saddle PSF Z(3,3) = 0.3 lambda, pupil 96^2 rounded to 128^2 as
the CPU path does), 20% 48x48 (45-mode tetrapod, pupil 128^2); photons
LogNormal(ln 3000, 0.6), Poisson noise, seed 2 (+ rank).  Every ROI is fitted
with the 5-parameter Levenberg-Marquardt MLE (max 50 model evaluations) through
the library's split-precision tcgen05 path; the plain FP64 GPU form of the same
fit runs on a sample of the same job for the speed-up and the accuracy check.

Usage: python bench.py [--gpus N --steps K --warmup W --impl b200|reference]
Prints one JSON line (rank 0).
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) per model
# evaluation of each round-based kernel of the 48x48 tetrapod class: one launch
# with all 4096 slots of a pool live (profiles/split_kernels_tetra48_dram_traffic.md).
NCU_TRAFFIC = {
    ("tetra48", "split_stage1_pupil_dft"): 117_005,
    ("tetra48", "split_stage2_window_dft"): 284_238,
    ("tetra48", "split_stage3_blur_rows"): 252_620,
    ("tetra48", "split_stage4_blur_cols_sums_lm"): 108_704,
}

METRIC = "MLE ROI fits/sec at ≤0.5 nm vs FP64 oracle (batched split-prec vs plain GPU)"
UNIT = "ROI fits/s"
TWO_PI = 2 * np.pi
DX = 0.11


def zern_astig(rng):
    z = np.zeros(15)
    z[5] = 0.08 * TWO_PI
    for k in (7, 8, 12):
        z[k] = rng.normal(0, 0.02) * TWO_PI
    return z


def zern_saddle(rng):
    z = np.zeros(28)
    z[9] = 0.3 * TWO_PI
    return z


def zern_tetrapod(rng):
    z = rng.normal(0, 0.02, 45) * TWO_PI
    z[:3] = 0
    z[5] = 0.6 * TWO_PI
    z[13] = 0.3 * TWO_PI
    z[25] = 0.15 * TWO_PI
    return z


CLASSES = [
    dict(name="astig16", frac=0.5, R=16, N=64, zern=zern_astig, zr=0.6, bg=20.0, zsym=False),
    dict(name="saddle24", frac=0.3, R=24, N=128, zern=zern_saddle, zr=1.0, bg=20.0, zsym=True),
    dict(name="tetra48", frac=0.2, R=48, N=128, zern=zern_tetrapod, zr=2.0, bg=30.0, zsym=False),
]


def class_counts(n):
    c = [int(round(n * k["frac"])) for k in CLASSES]
    c[0] += n - sum(c)
    return c


def disk_rows(N):
    # disk bounding rows for NA 1.4, lambda 0.66 um, pixel 0.11 um (30 at N=64, 60 at N=128)
    c = N / 2 - 0.5
    ring = (1.4 / 0.66) ** 2
    rows = [i for i in range(N) if ((i - c) / (N * DX)) ** 2 <= ring]
    return len(rows)


def window(R, N):
    w = min(2 * R, N)
    p = 1
    while p < w:
        p <<= 1
    return p


# ----------------------------------------------------------------- data ----
def make_job(z, ctx, torch, n, seed, device, only=None):
    """Synthetic ROIs on the device (FP64 library model + Poisson noise)."""
    rng = np.random.default_rng(seed)
    job = []
    for cls, cnt in zip(CLASSES, class_counts(n)):
        if only and cls["name"] not in only:
            continue
        R, N = cls["R"], cls["N"]
        zern = cls["zern"](np.random.default_rng(seed * 100 + R))
        psf = z.PSF(ctx, z.optics(size_fft=N, xystep=DX, na=1.4, wavelength=0.66, n_oil=1.518, sigma=0.9), zern)
        truth = np.zeros((cnt, 5))
        truth[:, :2] = rng.uniform(-DX, DX, (cnt, 2))
        truth[:, 2] = rng.uniform(-cls["zr"], cls["zr"], cnt)
        truth[:, 3] = rng.lognormal(np.log(3000.0), 0.6, cnt)
        truth[:, 4] = cls["bg"]
        rois = torch.empty((cnt, R, R), dtype=torch.float32, device=device)
        chunk = 1 << 16
        gen = torch.Generator(device=device)
        gen.manual_seed(seed * 1000 + R)
        for s in range(0, cnt, chunk):
            e = min(cnt, s + chunk)
            xyz = torch.tensor(truth[s:e, :3], dtype=torch.float64, device=device)
            psi = torch.empty((e - s, R, R), dtype=torch.float64, device=device)
            psf.model_dev(R, xyz, psi, stream=torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            a = torch.tensor(truth[s:e, 3], dtype=torch.float64, device=device)[:, None, None]
            mu = a * psi + cls["bg"]
            rois[s:e] = torch.poisson(mu, generator=gen).float()
        # initial values: x = y = 0 (ROI centre), z on the 100 nm library grid,
        # B from the ROI border, A from the background-subtracted sum
        init = np.zeros((cnt, 5))
        init[:, 2] = np.round(truth[:, 2] / 0.1) * 0.1
        border = torch.cat([rois[:, 0, :], rois[:, -1, :], rois[:, 1:-1, 0], rois[:, 1:-1, -1]], dim=1)
        b = border.mean(dim=1).double()
        a = (rois.double().sum(dim=(1, 2)) - b * R * R).clamp(min=100.0)
        init[:, 3] = a.cpu().numpy()
        init[:, 4] = b.cpu().numpy()
        # tol 1e-4 um: the reference's stopping distance (Localization.java:31), here on the Newton step
        prm_kw = dict(zmin=-cls["zr"] - 0.3, zmax=cls["zr"] + 0.3, xymax=R * DX / 2, max_iter=50, tol_xyz=1e-4)
        job.append(dict(cls=cls, psf=psf, zern=zern, truth=truth, rois=rois,
                        init=torch.tensor(init, dtype=torch.float64, device=device), init_np=init, prm_kw=prm_kw,
                        out=torch.empty((cnt, 5), dtype=torch.float64, device=device),
                        crlb=torch.empty((cnt, 5), dtype=torch.float64, device=device),
                        nll=torch.empty(cnt, dtype=torch.float64, device=device),
                        status=torch.empty(cnt, dtype=torch.int32, device=device),
                        iters=torch.empty(cnt, dtype=torch.int32, device=device)))
    return job


def render_frames(z, torch, device, psf, emit, nframes, S, P=64, bg=30.0, offset=0.0, seed=1, batch=200):
    """uint16 camera frames (n, S, S): background + emitters (rows frame, x px,
    y px, z um, photons; the FP64 device model on a P x P patch) with Poisson
    noise, plus a camera offset, rendered on the device in batches of frames."""
    cx, cy = emit[:, 1], emit[:, 2]
    ix, iy = cx.astype(int), cy.astype(int)
    frames = np.empty((nframes, S, S), dtype=np.uint16)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    a = torch.arange(P, device=device) - P // 2
    for f0 in range(0, nframes, batch):
        f1 = min(nframes, f0 + batch)
        sel = np.nonzero((emit[:, 0] >= f0) & (emit[:, 0] < f1))[0]
        img = torch.full(((f1 - f0) * S * S,), bg, dtype=torch.float64, device=device)
        if len(sel):
            # a positive model x moves the PSF towards lower pixel indices
            xyz = torch.tensor(np.c_[(ix[sel] - cx[sel]) * DX, (iy[sel] - cy[sel]) * DX, emit[sel, 3]],
                               dtype=torch.float64, device=device)
            psi = torch.empty((len(sel), P, P), dtype=torch.float64, device=device)
            psf.model_dev(P, xyz, psi, stream=torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            fr = torch.tensor(emit[sel, 0] - f0, dtype=torch.int64, device=device)
            ii = torch.tensor(ix[sel], device=device)[:, None, None] + a[None, :, None]
            jj = torch.tensor(iy[sel], device=device)[:, None, None] + a[None, None, :]
            ok = (ii >= 0) & (ii < S) & (jj >= 0) & (jj < S)
            flat = fr[:, None, None] * S * S + ii.clamp(0, S - 1) * S + jj.clamp(0, S - 1)
            amp = torch.tensor(emit[sel, 4], dtype=torch.float64, device=device)[:, None, None]
            img.index_put_((flat[ok],), (amp * psi)[ok], accumulate=True)
        cnt = torch.poisson(img, generator=gen) + offset
        frames[f0:f1] = cnt.clamp(max=65535).to(torch.int32).cpu().numpy().reshape(f1 - f0, S, S).astype(np.uint16)
    return frames


def detect_fit_config(z, ctx, torch, device, nframes, fp64_frames=0, seed=1):
    """Full-frame detect + fit: 256^2 uint16 frames of photon counts with
    Poisson(5) tetrapod emitters (45 modes, pupil 128^2, z in +-2 um,
    A ~ LogNormal(ln 4000, 0.5), B = 30), detected against a 41-slice library
    (0.1 um) with 40 x 40 ROIs and fitted through the frame pipeline
    (zola_localize_frames_u16: host frames in, localization rows out).  The
    split-precision arm runs nframes frames, the plain FP64 arm the first
    fp64_frames of them; the rows of the two arms are joined on (frame,
    candidate index)."""
    S, R, N = 256, 40, 128
    rng = np.random.default_rng(seed)
    zern = zern_tetrapod(np.random.default_rng(seed * 100 + 7))
    base = dict(size_fft=N, xystep=DX, na=1.4, wavelength=0.66, n_oil=1.518, sigma=0.9)
    psf_det = z.PSF(ctx, z.optics(kz_reset=True, **base), zern)
    psf_fit = z.PSF(ctx, z.optics(**base), zern)
    P = 64  # rendering patch
    k = rng.poisson(5, nframes)
    fr = np.repeat(np.arange(nframes), k)
    m = len(fr)
    emit = np.c_[fr, rng.uniform(P / 2, S - P / 2, (m, 2)), rng.uniform(-2.0, 2.0, m),
                 rng.lognormal(np.log(4000.0), 0.5, m)]
    frames = render_frames(z, torch, device, psf_fit, emit, nframes, S, P, seed=seed)
    det = z.Detector(psf_det, S, S, R, -2.0, 2.0, 0.1, 0.1)
    out = {"workload": "256x256 uint16 frames, Poisson(5) tetrapod emitters, R = 40, 0.1 um library over +-2 um; "
                       "host frames in and localization rows out",
           "frames": nframes, "emitters": int(m), "library_slices": det.nz,
           "detect_fp64_flops_per_frame": 2.0 * S * S * R * R * det.nz, "h2d_bytes_per_frame": S * S * 2}
    # detection alone (uint16 frames in, candidate lists out), after a warm-up call of
    # the same size (it sizes the staging and scratch areas)
    det.detect_u16(frames)
    t0 = time.perf_counter()
    det.detect_u16(frames)
    dt = time.perf_counter() - t0
    fp64_issue = 148 * 64 * 2 * 1.965e9  # 148 SMs x 64 DFMA/clk x max SM clock
    out["detect_only"] = {"frames": nframes, "frames_per_s": nframes / dt,
                          "fp64_tflops": out["detect_fp64_flops_per_frame"] * nframes / dt / 1e12,
                          "fp64_frac_of_issue": out["detect_fp64_flops_per_frame"] * nframes / dt / fp64_issue,
                          "note": "host uint16 frames to candidate lists through zola_detect_u16; FP64 issue rate "
                                  "= 148 SMs x 64 DFMA/clk x 1965 MHz (nominal)"}
    rows = {}
    for name, prec, nf in (("split", z.ZOLA_PREC_SPLIT, nframes), ("fp64", z.ZOLA_PREC_FP64, fp64_frames)):
        if nf <= 0:
            continue
        kw = dict(photon_threshold=500.0, precision=prec, max_iter=50, tol_xyz=1e-4)
        z.localize_frames_u16(ctx, det, psf_fit, frames[:min(nf, 64)], -2.0, 2.0, **kw)  # tables, plans, scratch
        t0 = time.perf_counter()
        r = z.localize_frames_u16(ctx, det, psf_fit, frames[:nf], -2.0, 2.0, **kw)
        dt = time.perf_counter() - t0
        rows[name] = r
        out[name] = {"frames": nf, "seconds": dt, "frames_per_s": nf / dt, "localizations": int(len(r)),
                     "localizations_per_s": len(r) / dt}
    if "fp64" in rows:
        a, b = rows["fp64"], rows["split"]
        b = b[b["frame"] < fp64_frames]
        ka = {(int(f), int(c)): i for i, (f, c) in enumerate(zip(a["frame"], a["candidate"]))}
        kb = {(int(f), int(c)): i for i, (f, c) in enumerate(zip(b["frame"], b["candidate"]))}
        both = sorted(set(ka) & set(kb))
        ia, ib = [ka[q] for q in both], [kb[q] for q in both]
        conv = (a["fit_status"][ia] == 1) & (b["fit_status"][ib] == 1)
        dxy = np.maximum(np.abs(a["x_nm"][ia] - b["x_nm"][ib]), np.abs(a["y_nm"][ia] - b["y_nm"][ib]))
        dz = np.abs(a["z_nm"][ia] - b["z_nm"][ib])
        da = np.abs(a["intensity"][ia] - b["intensity"][ib]) / np.abs(a["intensity"][ia])
        out["split_vs_fp64_rows"] = {
            "fp64_rows": int(len(a)), "split_rows": int(len(b)), "same_candidate": len(both),
            "both_converged": int(conv.sum()),
            "converged_within_tolerance": float(((dxy <= 0.5) & (dz <= 1.0) & (da <= 1e-3))[conv].mean())
            if conv.any() else None,
            "converged_max_dxy_nm": float(dxy[conv].max()) if conv.any() else None,
            "converged_max_dz_nm": float(dz[conv].max()) if conv.any() else None}
        out["split_vs_fp64_speedup"] = out["split"]["frames_per_s"] / out["fp64"]["frames_per_s"]
    det.close()
    psf_det.close()
    psf_fit.close()
    return out


def calibration_config(z, ctx, seed=3, fit_iters=10):
    """Calibration benchmark: 5 beads x 61 slices (50 nm, +-1.5 um) x 32^2 px, PSF
    from 45 Zernike coefficients ~ N(0, 0.05 lambda) + 0.1 lambda astigmatism,
    n_sample 1.33 at depth 0, 20,000 photons, background 50, Poisson noise.
    Times the stack NLL (forward), NLL + adjoint gradient (backward) and LM
    iterations of the Zernike fit on the GPU, and the oracle's restatement of
    the reference stack NLL (ZernikePhaseRetrieval.java:1843-1874) on the CPU;
    the reference's coordinate-wise finite-difference update takes about 8
    stack NLLs per coefficient per iteration."""
    import oracle as O
    rng = np.random.default_rng(seed)
    nz, nb, ns, R = 45, 5, 61, 32
    zern = rng.normal(0, 0.05, nz) * TWO_PI
    zern[:3] = 0
    zern[5] += 0.1 * TWO_PI
    dz = (np.arange(ns) - ns // 2) * 0.05
    xyz = np.c_[rng.uniform(-0.05, 0.05, (nb, 2)), rng.uniform(-0.05, 0.05, nb)]
    photons = np.full((nb, ns), 20000.0)
    ref = O.OraclePSF(128, DX, 1.4, 0.66, 1.518, 1.33, 1.0, zern, gauss_f32=False)
    stacks = np.zeros((nb, ns, R, R))
    for b in range(nb):
        for k in range(ns):
            stacks[b, k] = rng.poisson(photons[b, k] * ref.model_oil(R, xyz[b, 0], xyz[b, 1], dz[k] + xyz[b, 2], 0.0)
                                       + 50.0)
    bead = np.zeros((nb, 3 + ns + 6))
    bead[:, 3 + ns] = 50.0
    psf = z.PSF(ctx, z.optics(size_fft=128, xystep=DX, na=1.4, wavelength=0.66, n_oil=1.518, n_wat=1.33, sigma=0.9),
                np.zeros(nz))
    cal = z.Calibration(psf, stacks, dz, photons=photons)
    z0 = np.zeros(nz)
    cal.forward(z0, 0.9, bead)
    cal.backward(z0, 0.9, bead)
    reps = 20
    t0 = time.perf_counter()
    for _ in range(reps):
        cal.forward(z0, 0.9, bead)
    t_fwd = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        cal.backward(z0, 0.9, bead)
    t_bwd = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    _, _, _, nll, it = cal.fit(z0, 0.9, bead, max_iter=fit_iters)
    t_fit = time.perf_counter() - t0
    t0 = time.perf_counter()
    oref = O.OraclePSF(128, DX, 1.4, 0.66, 1.518, 1.33, 0.9, z0, gauss_f32=False)
    for b in range(nb):
        oref.calib_nll_full(R, dz, stacks[b], photons[b], 0.9, bead[b, :3], bead[b, 3:3 + ns], bead[b, 3 + ns:])
    t_cpu = time.perf_counter() - t0
    psf.close()
    return {"workload": "5 beads x 61 slices x 32^2 px, 45 Zernike coefficients, n_sample 1.33, pupil 128^2",
            "forward_nll_per_s": 1.0 / t_fwd, "adjoint_gradient_per_s": 1.0 / t_bwd,
            "lm_iterations": int(it), "lm_iterations_per_s": it / t_fit, "final_nll": float(nll),
            "cpu_oracle_stack_nll_s": t_cpu, "cpu_cores": 1,
            "reference_fd_iteration_s_estimate": t_cpu * 8 * (nz - 3),
            "note": "host C-ABI calls (stacks resident on the device); the reference's finite-difference "
                    "coordinate update needs about 8 stack NLLs per coefficient per iteration (estimate from the "
                    "oracle's single-thread NLL time)"}


def small_roi_config(z, ctx, n=1000, seed=0, reps=5):
    """Plain per-ROI localisation: 1,000 16x16 astigmatic ROIs (pupil 64^2, Z(2,2)
    0.08 lambda + random Z(3,+-1), Z(4,0)), x, y ~ U(-1, 1) px, z ~ U(-0.6, 0.6) um,
    photons LogNormal(ln 2000, 0.4), background 20, Poisson noise, seed 0; at most
    30 evaluations.  The split and FP64 fits run through the host C-ABI (ROIs in
    host memory, results back); the CPU arm is the oracle's restatement of the
    reference CPU localisation (coordinate descent, Localization.java) on the same
    ROIs with all host threads; the FP64 oracle LM of the same fit is the accuracy
    reference for every ROI."""
    import oracle as O
    rng = np.random.default_rng(seed)
    R, N = 16, 64
    zern = zern_astig(np.random.default_rng(seed))
    psf = z.PSF(ctx, z.optics(size_fft=N, xystep=DX, na=1.4, wavelength=0.66, n_oil=1.518, sigma=0.9), zern)
    truth = np.c_[rng.uniform(-DX, DX, (n, 2)), rng.uniform(-0.6, 0.6, n), rng.lognormal(np.log(2000.0), 0.4, n),
                  np.full(n, 20.0)]
    rois = rng.poisson(truth[:, 3, None, None] * psf.model(R, truth[:, :3]) + 20.0).astype(np.float32)
    init = np.zeros((n, 5))
    init[:, 2] = np.round(truth[:, 2] / 0.1) * 0.1
    border = np.concatenate([rois[:, 0, :], rois[:, -1, :], rois[:, 1:-1, 0], rois[:, 1:-1, -1]], axis=1)
    init[:, 4] = border.mean(axis=1)
    init[:, 3] = np.maximum(rois.sum(axis=(1, 2)) - init[:, 4] * R * R, 100.0)
    kw = dict(zmin=-0.9, zmax=0.9, xymax=R * DX / 2, max_iter=30, tol_xyz=1e-4)
    threads = os.cpu_count() or 1
    ref = O.OraclePSF(N, DX, 1.4, 0.66, 1.518, 1.518, 0.9, zern, gauss_f32=False)
    o, _, so, _ = ref.fit_lm(rois.astype(np.float64), init, kw["zmin"], kw["zmax"], kw["xymax"], tol_xyz=kw["tol_xyz"],
                             max_iter=kw["max_iter"], threads=threads)
    out = {"workload": "1,000 16x16 astigmatic ROIs, pupil 64^2, 30 evaluations at most, host ROIs in / results out",
           "rois": n}
    for name, prec in (("split", z.ZOLA_PREC_SPLIT), ("fp64", z.ZOLA_PREC_FP64)):
        prm = z.PSF.fit_params(precision=prec, **kw)
        res = psf.fit(rois, init, prm)
        t0 = time.perf_counter()
        for _ in range(reps):
            res = psf.fit(rois, init, prm)
        dt = (time.perf_counter() - t0) / reps
        out[name] = {"fits_per_s": n / dt, "ms_per_call": dt * 1000,
                     "accuracy_vs_oracle": accuracy_block(o, so, res["theta"], res["status"], False)}
    # the reference CPU path on the same ROIs (its own init: A, B, x, y, z)
    t0 = time.perf_counter()
    ref.localize_cd(rois.astype(np.float64), np.c_[init[:, 3], init[:, 4], init[:, :3]], kw["zmin"], kw["zmax"], 20,
                    0.0, threads=threads)
    dt = time.perf_counter() - t0
    out["cpu_port"] = {"fits_per_s": n / dt, "cores": threads, "kind": "port",
                       "note": "oracle restatement of the reference coordinate descent (Localization.java), FFT model"}
    out["split_vs_cpu_port"] = out["split"]["fits_per_s"] / out["cpu_port"]["fits_per_s"]
    psf.close()
    return out


def filaments(rng, n_curves, lo, hi, zr, n_points):
    """Points on random smooth 3-D curves (cubic Bezier, 4 random control
    points in the box [lo, hi]^2 x [-zr, zr]) with 25 nm Gaussian jitter:
    (n_points, 3) in um."""
    t = rng.uniform(0, 1, n_points)
    c = rng.integers(0, n_curves, n_points)
    ctrl = np.concatenate([rng.uniform(lo, hi, (n_curves, 4, 2)), rng.uniform(-zr, zr, (n_curves, 4, 1))], axis=2)
    b = np.stack([(1 - t) ** 3, 3 * t * (1 - t) ** 2, 3 * t ** 2 * (1 - t), t ** 3], axis=1)
    pts = np.einsum("nk,nkd->nd", b, ctrl[c])
    return pts + rng.normal(0, 0.025, pts.shape)


def stream_drift_config(z, ctx, torch, device, nframes, seed=4):
    """End-to-end stream with drift: 512x512 uint16 frames (camera offset 100
    counts), Poisson(15) emitters a frame on synthetic filaments (random 3-D
    cubic curves, 25 nm jitter), tetrapod PSF (45 modes, pupil 128^2), photons
    LogNormal(ln 4000, 0.5), background 30, and an imposed drift: a random walk
    of 0.5 nm a frame in x, y, z over 100,000 frames (a run of fewer frames
    takes proportionally larger steps, so that it spans the same excursion).
    The split-precision detect -> fit pipeline runs on the uint16 frames (host
    frames in, rows out, timed); then the 3-D drift (20 time bins, 10 nm
    voxels) is estimated from the localizations in a 5.12 x 5.12 um crop at the
    centre (1.5 emitters a frame on average sit on the crop's filaments; the
    others on filaments elsewhere in the frame), and compared with the imposed
    walk."""
    S, R, N, P = 512, 40, 128, 64
    rng = np.random.default_rng(seed)
    zern = zern_tetrapod(np.random.default_rng(seed * 100 + 7))
    base = dict(size_fft=N, xystep=DX, na=1.4, wavelength=0.66, n_oil=1.518, sigma=0.9)
    psf_det = z.PSF(ctx, z.optics(kz_reset=True, **base), zern)
    psf_fit = z.PSF(ctx, z.optics(**base), zern)
    fov = S * DX
    c0, c1 = fov / 2 - 2.56, fov / 2 + 2.56
    inner = filaments(rng, 6, c0 + 0.3, c1 - 0.3, 0.8, 200000)
    outer = filaments(rng, 40, P * DX / 2, fov - P * DX / 2, 1.5, 800000)
    outer = outer[(np.abs(outer[:, 0] - fov / 2) > 2.56 + R * DX / 2) | (np.abs(outer[:, 1] - fov / 2) > 2.56 + R * DX / 2)]
    # the walk's step is scaled so that the run spans the excursion of 100,000 frames at 0.5 nm a frame
    step = 0.5e-3 * np.sqrt(max(1.0, 100000.0 / nframes))
    walk = np.cumsum(rng.normal(0, step, (nframes, 3)), axis=0)  # um
    emit = []
    for f in range(nframes):
        k_in, k_out = rng.poisson(1.5), rng.poisson(13.5)
        pts = np.concatenate([inner[rng.integers(0, len(inner), k_in)], outer[rng.integers(0, len(outer), k_out)]])
        for q in pts:
            emit.append((f, *(q + walk[f]), rng.lognormal(np.log(4000.0), 0.5)))
    emit = np.array(emit)
    emit[:, 1:3] /= DX  # um -> px
    frames = render_frames(z, torch, device, psf_fit, emit, nframes, S, P, offset=100.0, seed=seed)
    det = z.Detector(psf_det, S, S, R, -2.0, 2.0, 0.1, 0.1)
    kw = dict(adu=1.0, gain=1.0, offset=100.0, photon_threshold=500.0, precision=z.ZOLA_PREC_SPLIT, max_iter=50,
              tol_xyz=1e-4)
    z.localize_frames_u16(ctx, det, psf_fit, frames[:8], -2.0, 2.0, **kw)  # warm-up: tables, plans
    t0 = time.perf_counter()
    rows = z.localize_frames_u16(ctx, det, psf_fit, frames, -2.0, 2.0, **kw)
    dt = time.perf_counter() - t0
    out = {"workload": "512x512 uint16 frames, Poisson(15) tetrapod emitters on filaments, drift random walk "
                       "0.5 nm/frame; split-precision pipeline, host frames in / rows out",
           "frames": nframes, "emitters": int(len(emit)), "localizations": int(len(rows)), "seconds": dt,
           "frames_per_s": nframes / dt, "localizations_per_s": len(rows) / dt,
           "h2d_bytes": int(frames.nbytes), "walk_step_nm": step * 1000.0}
    xyz = np.c_[rows["x_nm"], rows["y_nm"], rows["z_nm"]]
    crop = (np.abs(xyz[:, 0] / 1000 - fov / 2) < 2.56) & (np.abs(xyz[:, 1] / 1000 - fov / 2) < 2.56) & \
        (np.abs(xyz[:, 2]) < 1280.0)
    out["crop_localizations"] = int(crop.sum())
    if crop.sum() > 100:
        cr = np.c_[rows["crlb_x_nm"], rows["crlb_y_nm"], rows["crlb_z_nm"]][crop]
        fr = rows["frame"][crop]
        t0 = time.perf_counter()
        b, l, px = z.drift(ctx, xyz[crop], fr, cr, pixel_nm=10.0, bins=20, max_drift_um=0.2)
        out["drift_seconds"] = time.perf_counter() - t0
        err = l - walk[fr] * 1000.0
        err -= err.mean(axis=0)
        out["drift_rms_error_nm"] = [float(v) for v in np.sqrt((err ** 2).mean(axis=0))]
        out["imposed_drift_rms_nm"] = [float(v) for v in (walk * 1000.0 - (walk * 1000.0).mean(0)).std(axis=0)]
        out["drift_voxel_nm"] = px
    det.close()
    psf_det.close()
    psf_fit.close()
    return out


def run_step(z, ctx, job, precision, stream_ptr, mixed=True):
    """One step: the whole mixed job, in one zola_fit_batch_mixed_dev call (split precision), or one
    call per class."""
    if mixed and precision == z.ZOLA_PREC_SPLIT:
        z.fit_mixed_dev(ctx, [dict(psf=j["psf"], rois=j["rois"], init=j["init"],
                                   prm=z.PSF.fit_params(precision=precision, **j["prm_kw"]), out=j["out"],
                                   crlb=j["crlb"], nll=j["nll"], status=j["status"], iters=j["iters"]) for j in job],
                        stream=stream_ptr)
        return
    for j in job:
        p = z.PSF.fit_params(precision=precision, **j["prm_kw"])
        j["psf"].fit_dev(j["rois"], j["init"], p, j["out"], j["crlb"], j["nll"], j["status"], j["iters"],
                         stream=stream_ptr)


# --------------------------------------------------------------- clocks ----
class ClockSampler:
    def __init__(self, device):
        self.p = None
        self.device = device
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(device), "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
        except (OSError, ValueError):
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------ baselines ----
def cpu_baseline(budget_s=15.0, seed=2):
    """The oracle port of the reference's CPU localisation (coordinate descent,
    FFT model, Localization.java) on a bounded sample of the workload, all host
    threads.  Returns fits/s for the job's class mix."""
    import oracle as O
    threads = os.cpu_count() or 1
    per_fit = []
    counts = []
    for cls in CLASSES:
        R, N = cls["R"], cls["N"]
        zern = cls["zern"](np.random.default_rng(seed * 100 + R))
        p = O.OraclePSF(N, DX, 1.4, 0.66, 1.518, 1.518, 0.9, zern)
        rng = np.random.default_rng(seed + 7 * R)
        # four ROIs a host thread per class (64 a class on 16 cores): a sample that takes
        # a few seconds a class, with the GPU job's start (x = y = 0, z on the 0.1 um grid,
        # 0.9 of the photons)
        n1 = 4 * max(threads, 1)
        truth = np.c_[rng.uniform(-DX, DX, (n1, 2)), rng.uniform(-cls["zr"], cls["zr"], n1),
                      rng.lognormal(np.log(3000.0), 0.6, n1), np.full(n1, cls["bg"])]
        rois = rng.poisson(truth[:, 3, None, None] * p.model(R, truth[:, :3]) + cls["bg"]).astype(float)
        init = np.c_[truth[:, 3] * 0.9, truth[:, 4], np.zeros((n1, 2)), np.round(truth[:, 2] / 0.1) * 0.1]
        t0 = time.perf_counter()
        p.localize_cd(rois, init, -cls["zr"] - 0.3, cls["zr"] + 0.3, 20, 0.0, threads=threads)
        dt = time.perf_counter() - t0
        per_fit.append(dt / n1)
        counts.append(n1)
        if sum(per_fit) * threads > budget_s:
            break
    t_job = sum(c["frac"] * t for c, t in zip(CLASSES, per_fit)) / sum(c["frac"] for c in CLASSES[:len(per_fit)])
    sample = ", ".join(f"{n} {c['name']}" for c, n in zip(CLASSES, counts))
    return 1.0 / t_job, threads, sample


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    vals = []
    for i in range(args.warmup + args.steps):
        v, cores, sample = cpu_baseline(budget_s=args.cpu_seconds, seed=2 + i)
        if i >= args.warmup:
            vals.append(v)
    v = float(np.median(vals))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": config_block(args.rois),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"per step: {sample} ROIs fitted by the oracle's restatement of the "
                                       "reference coordinate-descent localisation (Localization.java), "
                                       "throughput weighted by the job's class mix"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_block(n):
    return {"workload": "batched mixed-size 5-parameter Poisson MLE ROI fits, split-precision tcgen05 vs plain "
                        "FP64 GPU", "rois_per_step": n,
            "mix": "50% 16x16 astigmatic (pupil 64^2), 30% 24x24 saddle Z(3,3)=0.3 lambda (pupil 96^2 -> 128^2 as "
                   "the CPU path rounds), 20% 48x48 45-mode tetrapod (pupil 128^2)",
            "photons": "LogNormal(ln 3000, 0.6)", "max_evaluations": 50, "seed": 2,
            "l2": "inputs larger than L2 (float32 ROIs ~3 GB per step)"}


# ----------------------------------------------------------------- main ----
def flops_per_eval(R, N):
    """Algorithmic flops of one model evaluation with x/y/z derivatives (complex MAC = 8 flops)."""
    W, D = window(R, N), disk_rows(N)
    return 3 * 8 * W * D * D + 4 * 8 * W * W * D


def theta_err(a, b, zsym):
    """|a - b| per ROI and parameter, |z| compared for z-symmetric PSFs."""
    d = np.abs(a - b)
    if zsym:
        d[:, 2] = np.abs(np.abs(a[:, 2]) - np.abs(b[:, 2]))
    return d


def accuracy_block(a, sa, b, sb, zsym):
    """Per-ROI error of fits b against reference fits a, over every ROI compared
    (all statuses) and over the ROIs both fits report converged."""
    d = theta_err(a, b, zsym)
    rel = d[:, 3] / np.abs(a[:, 3])
    within = (d[:, :2].max(1) <= 0.5e-3) & (d[:, 2] <= 1e-3) & (rel <= 1e-3)
    conv = (sa == 1) & (sb == 1)
    out = {"compared": int(len(a)), "within_tolerance": float(within.mean()),
           "status_agreement": float((sa == sb).mean()), "both_converged": float(conv.mean()),
           "max_dxy_nm": float(d[:, :2].max() * 1000), "max_dz_nm": float(d[:, 2].max() * 1000),
           "max_dA_rel": float(rel.max()), "p99_dxy_nm": float(np.percentile(d[:, :2].max(1), 99) * 1000),
           "p99_dz_nm": float(np.percentile(d[:, 2], 99) * 1000), "p99_dA_rel": float(np.percentile(rel, 99))}
    if conv.any():
        out.update(converged_max_dxy_nm=float(d[conv, :2].max() * 1000), converged_max_dz_nm=float(d[conv, 2].max() * 1000),
                   converged_max_dA_rel=float(rel[conv].max()), converged_within_tolerance=float(within[conv].mean()))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--rois", type=int, default=1_000_000)
    ap.add_argument("--fp64-sample", type=int, default=20_000)
    ap.add_argument("--oracle-sample", type=int, default=48, help="ROIs per class fitted by the FP64 oracle")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--classes", default="", help="comma list of ROI classes to run (profiling); default all")
    ap.add_argument("--pool", type=int, default=0,
                    help="slots of the split fit's pool per class (0: chosen by the library's autotuner)")
    ap.add_argument("--detect-frames", type=int, default=1024,
                    help="frames of the detect -> fit pipeline measurement (0: skip)")
    ap.add_argument("--split-mode", default="staged", choices=["staged", "flow", "fused"],
                    help="split fit kernels: one dataflow kernel, four stage kernels per round, or stage 1 + fused 2-5")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuning pass (slot pool per class, or the dataflow kernel shape)")
    ap.add_argument("--no-calibration", dest="calibration", action="store_false",
                    help="skip the Zernike calibration measurement")
    ap.add_argument("--detect-fp64-frames", type=int, default=50,
                    help="frames of the detect -> fit pipeline's plain FP64 arm (0: skip)")
    ap.add_argument("--stream-frames", type=int, default=0,
                    help="frames of the 512x512 uint16 stream + drift measurement (0: skip)")
    ap.add_argument("--no-small-rois", dest="small_rois", action="store_false",
                    help="skip the 1,000-ROI 16x16 localisation measurement")
    ap.add_argument("--stage-breakdown", action="store_true",
                    help="also time the round-based stage kernels per stage (explains the dataflow kernel)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist
    import __graft_entry__ as ge
    import oracle as O

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=device)
    z = ge.load_package()
    import zola3d_b200.replicas as rp
    ctx = z.Context(local)
    if args.pool:
        ctx.set_pool(args.pool)
    ctx.set_split_mode(args.split_mode)
    ext = torch.cuda.ExternalStream(ctx.stream, device=device)
    only = [c for c in args.classes.split(",") if c]
    job = make_job(z, ctx, torch, args.rois, seed=2 + rank, device=device, only=only)
    n_total = sum(j["rois"].shape[0] for j in job)
    torch.cuda.synchronize()

    def fit_class(j, precision=None):
        p = z.PSF.fit_params(precision=z.ZOLA_PREC_SPLIT if precision is None else precision, **j["prm_kw"])
        j["psf"].fit_dev(j["rois"], j["init"], p, j["out"], j["crlb"], j["nll"], j["status"], j["iters"],
                         stream=ctx.stream)

    # autotuning pass (outside the timed region): the dataflow kernel's shape per
    # class; fits do not depend on the shape, so this changes timings only
    tuned = {}
    if args.split_mode == "flow" and not args.no_tune:
        ctx.set_tuning(True)
        for j in job:
            for _ in range(10):
                fit_class(j)
                ext.synchronize()
                if j["psf"].flow_shape(j["cls"]["R"])[0]:
                    break
        ctx.set_tuning(False)
    if args.split_mode == "flow":
        for j in job:
            t, units, ctas, ns = j["psf"].flow_shape(j["cls"]["R"])
            tuned[j["cls"]["name"]] = {"tuned": t, "units": units, "ctas_per_stage": ctas, "ns_per_eval": ns}
    # round-based kernels: the slot pool per class (four trial fits of each class
    # alone; the fits are the same bit for bit whatever the pool)
    if args.split_mode == "staged" and not args.no_tune and args.pool == 0:
        ctx.set_tuning(True)
        for j in job:
            for _ in range(4):
                fit_class(j)
                ext.synchronize()
        ctx.set_tuning(False)
    if args.split_mode == "staged":
        for j in job:
            t, pool, ns = j["psf"].split_pool(j["cls"]["R"])
            tuned[j["cls"]["name"]] = {"tuned": t, "pool": pool, "ns_per_eval": ns}

    # warm-up (split path), also primes tables and the slot pool
    for _ in range(args.warmup):
        run_step(z, ctx, job, z.ZOLA_PREC_SPLIT, ctx.stream, mixed=args.split_mode == "staged")
    ext.synchronize()

    # timed steps (device time on the library stream; max over ranks)
    l0 = ctx.launches
    clocks = ClockSampler(local)
    rp.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(ext)
    for _ in range(args.steps):
        run_step(z, ctx, job, z.ZOLA_PREC_SPLIT, ctx.stream, mixed=args.split_mode == "staged")
    ev1.record(ext)
    ev1.synchronize()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    launches = ctx.launches - l0
    ms = rp.max_over_ranks(ms, device)
    rp.barrier()
    ms_step = ms / args.steps
    value = n_total * world / (ms_step / 1000.0)

    # per class: time (CUDA events around the call), then the kernel time of a
    # profiled pass (every launch bracketed by events), evaluations logged per ROI
    per_class, kern_ms = {}, {}
    for j in job:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        fit_class(j)
        e1.record(ext)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1000.0
        name = j["cls"]["name"]
        per_class[name] = {"rois": int(j["rois"].shape[0]), "seconds": t, "fits_per_s": j["rois"].shape[0] / t,
                           "mean_evals": float(j["iters"].double().mean().item())}
        ctx.profile(True)
        ctx.stage_stats(reset=True)
        fit_class(j)
        st = ctx.stage_stats(reset=True)
        ctx.profile(False)
        kern_ms[name] = {k: v for k, v in st.items() if v[1]}
    iters = {j["cls"]["name"]: int(j["iters"].sum().item()) for j in job}
    split_res = {j["cls"]["name"]: (j["out"].cpu().numpy(), j["status"].cpu().numpy()) for j in job}

    # the round-based stage kernels per stage, for the explanation (optional)
    breakdown = None
    if args.stage_breakdown:
        ctx.set_split_mode("staged")
        ctx.set_pool(16384)
        breakdown = {}
        for j in job:
            ctx.profile(True)
            ctx.stage_stats(reset=True)
            fit_class(j)
            st = ctx.stage_stats(reset=True)
            ctx.profile(False)
            ev = iters[j["cls"]["name"]]
            breakdown[j["cls"]["name"]] = {k: {"ms": round(v[0], 3), "launches": v[1],
                                               "sm_clocks_per_eval": round(v[0] * 1e-3 * 1.965e9 * 148 / max(1, ev))}
                                           for k, v in st.items() if v[1]}
        ctx.set_pool(args.pool)
        ctx.set_split_mode(args.split_mode)

    # plain FP64 GPU form on a sample of the same job (speed-up and accuracy, every status)
    fp64, acc64 = {}, {}
    t_job64 = 0.0
    for j in job:
        cnt = j["rois"].shape[0]
        m = min(cnt, max(64, int(args.fp64_sample * j["cls"]["frac"])))
        sl = slice(0, m)
        p64 = z.PSF.fit_params(precision=z.ZOLA_PREC_FP64, **j["prm_kw"])
        out64 = torch.empty((m, 5), dtype=torch.float64, device=device)
        st64 = torch.empty(m, dtype=torch.int32, device=device)
        it64 = torch.empty(m, dtype=torch.int32, device=device)
        j["psf"].fit_dev(j["rois"][:64], j["init"][:64], p64, out64[:64], None, None, st64[:64], it64[:64],
                         stream=ctx.stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        j["psf"].fit_dev(j["rois"][sl], j["init"][sl], p64, out64, None, None, st64, it64, stream=ctx.stream)
        e1.record(ext)
        e1.synchronize()
        t = e0.elapsed_time(e1) / 1000.0
        t_job64 += t / m * cnt
        name = j["cls"]["name"]
        ev64 = int(it64.sum().item())
        fp64[name] = {"sample": m, "seconds": t, "fits_per_s": m / t,
                      "fp64_tflops": round(ev64 * (flops_per_eval(j["cls"]["R"], j["cls"]["N"]) +
                                                   8 * (j["cls"]["R"] * window(j["cls"]["R"], j["cls"]["N"]) ** 2 +
                                                        j["cls"]["R"] ** 2 * window(j["cls"]["R"], j["cls"]["N"])))
                                           / t / 1e12, 3)}
        b, sb = split_res[name]
        acc64[name] = accuracy_block(out64.cpu().numpy(), st64.cpu().numpy(), b[:m], sb[:m], j["cls"]["zsym"])
    fp64_value = n_total / t_job64

    # against the FP64 oracle of the same fit (CPU, all host threads) on a sample, every status
    acc_oracle = {}
    if rank == 0 and args.oracle_sample > 0:
        threads = os.cpu_count() or 1
        for j in job:
            cls = j["cls"]
            m = min(args.oracle_sample, j["rois"].shape[0])
            ref = O.OraclePSF(cls["N"], DX, 1.4, 0.66, 1.518, 1.518, 0.9, j["zern"], gauss_f32=False)
            kw = j["prm_kw"]
            o, _, so, _ = ref.fit_lm(j["rois"][:m].double().cpu().numpy(), j["init_np"][:m], kw["zmin"], kw["zmax"],
                                     kw["xymax"], tol_xyz=kw["tol_xyz"], max_iter=kw["max_iter"], threads=threads)
            b, sb = split_res[cls["name"]]
            acc_oracle[cls["name"]] = accuracy_block(o, so, b[:m], sb[:m], cls["zsym"])

    # roofline: the dataflow kernel (the whole fit) of the class with the most
    # device time, tensor-bound: algorithmic flops of the model evaluations it
    # made / its CUDA-event duration, against the sustained measured bf16 peak
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak_tf = peaks.get("bf16_tflops_sustained", 1400.0)
    peak_gbs = peaks.get("hbm_gbs", 6650.0)
    peak_src = "of measured" if "bf16_tflops_sustained" in peaks and "hbm_gbs" in peaks else "of fallback"
    # algorithmic flops of each kernel per model evaluation: stage 1 the pupil DFT
    # (3*8*W*D^2), stage 2 the window DFT (4*8*W^2*D), the dataflow kernel both
    def stage_flops(R, N):
        W, D = window(R, N), disk_rows(N)
        return {"split_stage1_pupil_dft": 3 * 8 * W * D * D, "split_stage2_window_dft": 4 * 8 * W * W * D,
                "split_dataflow": flops_per_eval(R, N)}
    by_class = {}
    tot_flops = tot_s = 0.0
    best = None
    for j in job:
        name, R, N = j["cls"]["name"], j["cls"]["R"], j["cls"]["N"]
        km, sf = kern_ms[name], stage_flops(R, N)
        ms_all = sum(v[0] for v in km.values())
        ent = {"kernels": {}}
        for k, (ms_k, n_k) in km.items():
            e = {"ms": round(ms_k, 3), "launches": n_k}
            if k in sf and ms_k > 0:
                tf = iters[name] * sf[k] / (ms_k / 1000.0) / 1e12
                e.update(tflops=round(tf, 2), tensor_frac=round(tf / peak_tf, 4))
                if best is None or ms_k > best[2]:
                    best = (name, k, ms_k)
            ent["kernels"][k] = e
        fl = iters[name] * flops_per_eval(R, N)
        ent.update(evaluations=iters[name], fit_ms=round(ms_all, 3),
                   fit_tflops=round(fl / (ms_all / 1000.0) / 1e12, 2),
                   fit_tensor_frac=round(fl / (ms_all / 1000.0) / 1e12 / peak_tf, 4))
        by_class[name] = ent
        tot_flops += fl
        tot_s += ms_all / 1000.0
    dom_cls, dom_k, _ = best
    ent = by_class[dom_cls]["kernels"][dom_k]
    traffic = NCU_TRAFFIC.get((dom_cls, dom_k))
    roofline = {"bound": "tensor", "achieved": ent["tflops"], "peak": peak_tf, "unit": "TFLOP/s",
                "frac": ent["tensor_frac"], "kernel": dom_k, "class": dom_cls,
                "peak_source": peak_src + " (sustained bf16)",
                "traffic": None if traffic is None else int(traffic * iters[dom_cls] / max(1, ent["launches"])),
                "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum per launch: ncu bytes per model "
                                "evaluation of this kernel on this class (profiles/), times the evaluations per launch",
                "hbm_gbs_at_traffic": None if traffic is None else
                round(traffic * iters[dom_cls] / (ent["ms"] / 1000.0) / 1e9, 1),
                "hbm_frac_at_traffic": None if traffic is None else
                round(traffic * iters[dom_cls] / (ent["ms"] / 1000.0) / 1e9 / peak_gbs, 4),
                "whole_job_tflops": round(tot_flops / tot_s / 1e12, 2),
                "whole_job_tensor_frac": round(tot_flops / tot_s / 1e12 / peak_tf, 4),
                "per_class": by_class, "hbm_peak_gbs": peak_gbs,
                "note": "achieved = algorithmic flops of the model evaluations made (pupil DFT 3*8*W*D^2, "
                        "window DFT 4*8*W^2*D per evaluation, complex MAC = 8 flops; evaluations logged per ROI) / "
                        "summed CUDA-event duration of that kernel's launches for that class; whole_job = all "
                        "algorithmic flops / all fit kernels' time; peak = sustained measured bf16 (FP16 runs at the same rate)"}

    # end to end through the host C-ABI (pinned host buffers, H2D + D2H inside the call)
    e2e = None
    host = []
    h2d = d2h = 0
    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    for j in job:
        r = torch.empty(j["rois"].shape, dtype=torch.float32, pin_memory=True)
        r.copy_(j["rois"])
        i0 = torch.empty(j["init"].shape, dtype=torch.float64, pin_memory=True)
        i0.copy_(j["init"])
        m = j["rois"].shape[0]
        res = dict(theta=pinned((m, 5), torch.float64), crlb=pinned((m, 5), torch.float64),
                   nll=pinned((m,), torch.float64), status=pinned((m,), torch.int32), iters=pinned((m,), torch.int32))
        host.append((r.numpy(), i0.numpy(), res))
        h2d += r.numel() * 4 + i0.numel() * 8
        d2h += m * (5 * 8 + 5 * 8 + 8 + 4 + 4)
    # one mixed call from host memory (zola_fit_batch_mixed: each class's H2D copy on the
    # copy stream overlaps the fits of the classes copied before it); one untimed pass
    # sizes the library's staging area, then the timed pass (inputs and results pinned)
    mixed = [dict(psf=j["psf"], rois=r, init=i0, out=res,
                  prm=z.PSF.fit_params(precision=z.ZOLA_PREC_SPLIT, **j["prm_kw"]))
             for j, (r, i0, res) in zip(job, host)]
    z.fit_mixed(ctx, mixed)
    torch.cuda.synchronize()
    rp.barrier()
    t0 = time.perf_counter()
    z.fit_mixed(ctx, mixed)
    t_e2e = rp.max_over_ranks(time.perf_counter() - t0, device)
    e2e = {"value": n_total * world / t_e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "call": "zola_fit_batch_mixed"}

    detect = detect_fit_config(z, ctx, torch, device, args.detect_frames, args.detect_fp64_frames, seed=1 + rank) \
        if args.detect_frames > 0 else None
    calib = calibration_config(z, ctx) if args.calibration and rank == 0 else None
    small = small_roi_config(z, ctx) if args.small_rois and rank == 0 else None
    stream = stream_drift_config(z, ctx, torch, device, args.stream_frames) if args.stream_frames > 0 and rank == 0 \
        else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, sample = cpu_baseline(budget_s=args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{sample} ROIs fitted by the oracle's restatement of the reference coordinate-descent "
                         "localisation (Localization.java), throughput weighted by the job's class mix"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f16x3 (split) / f32 sums / f64 solve", "data": "synthetic",
                "config": dict(config_block(args.rois), parallelism=f"replicas x{world}", split_kernels=args.split_mode,
                               pool=args.pool or "autotuned per class (tuned_shapes)"),
                "e2e": e2e, "gpu_launches": int(launches), "clocks": clk, "roofline": roofline,
                "cpu_baseline": cpu,
                "split_per_class": per_class, "tuned_shapes": tuned,
                "fp64_plain_gpu": {"value": fp64_value, "unit": UNIT, "per_class": fp64},
                "speedup_vs_fp64_plain": value / world / fp64_value,
                "accuracy_vs_oracle": acc_oracle, "accuracy_vs_fp64_gpu": acc64,
                "stage_breakdown_round_based": breakdown,
                "detect_fit_pipeline": detect, "calibration": calib, "small_roi_localisation": small,
                "stream_drift": stream}
        print(json.dumps(line), flush=True)
    for j in job:
        j["psf"].close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
