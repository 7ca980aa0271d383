// Frame localization pipeline: detection -> candidate selection -> fit ->
// filters and mask -> localization rows (process/cpu/LocalizationPipeline.java).
//
// The reference walks each frame's sorted candidate list on a Java thread
// (LocalizationThread.run, LocalizationPipeline.java:720-990):
//   - next candidate whose centre pixel is unmasked and inside the border
//     (myGetMaxPositions, :1218-1250);
//   - skip it if any pixel of its R x R patch is masked;
//   - getAandB init from the library PSF of its slice (:1119-1162); fit only
//     if maxPatch / B > maxSNR (1) and B > 0, else mask the patch pixels above
//     half the patch maximum;
//   - accept if A > photonThreshold, |x|,|y| < 10 px, the rounded position is
//     inside the frame and unmasked, and minZ < z < maxZ (:859-945); then mask
//     the pixels where model - B > 0.2 max(model - B);
//   - otherwise mask the patch pixels above half the patch maximum (:967-977).
// A candidate's fit reads only the raw patch and its getAandB start, never
// the mask, so the fits do not depend on the order.  Frames advance in waves:
// each wave takes, per frame, the next K candidates that need a fit under the
// current mask (one CTA per frame tests candidates in parallel chunks: border,
// centre and patch masks, getAandB, SNR), fits all of them in one batched call
// (FP64 or split), evaluates the model at every fitted position, and then one
// CTA per frame replays the reference's sequential walk over the candidates
// the wave covered: mask tests, acceptance, mask updates.  A candidate masked
// by an earlier one in the same wave was fitted for nothing; masks only grow,
// so a candidate the wave found masked stays skipped.  Accepted localizations
// get chi2 as scoreCompute (:1099-1115) and the CRLB from the Fisher matrix the
// reference forms (Localization.java:317-451: dmu/dA taken as mu, h -> 0
// limit).  Rows come out in frame order and, within a frame, in candidate
// order; x/y/z in nm as 1000*(i*dx - x) (:905-907).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "lm.h"
#include "zola_internal.h"

namespace zola {

struct PipeView {
    int SX, SY, R, cap, nframes;
    double dx, minZ, maxZ, photon_thr, max_snr;
    const double* images;     // nframes x SX x SY: detection images
    const double* fimg;       // nframes x SX x SY: fit images (= images without sCMOS)
    const double* vmap;       // SX x SY sCMOS var/gain^2, or nullptr
    float* slot_v;            // slots x R x R sCMOS patches (with vmap)
    unsigned char* mask;      // nframes x SX x SY
    const double* cand;       // nframes x cap x 7
    const int* counts;        // nframes
    const double* libpsf;     // Z x R x R (normalised library PSFs)
    const double* range;      // Z
    int* cand_slot;           // nframes x cap: fit slot; -1 not fitted (SNR), -2 outside the border,
                              // -3 masked when the wave looked at it
    double* cand_maxp;        // nframes x cap: patch maximum
    int* pointer;             // nframes: first candidate not yet walked
    int* limit;               // nframes: end of the candidates the current wave covers
    int* done;                // nframes
    int* nslots;              // slots of the current wave
    int slot_cap;
    float* rois;              // slots x R x R
    double* init;             // slots x 5
    int* slot_frame;          // slots
    int* slot_cand;           // slots
};

__device__ inline bool pipe_inside(const PipeView& V, int ci, int cj) {
    const int h = V.R / 2;
    return ci > h + 1 && cj > h + 1 && ci < V.SX - h - 1 && cj < V.SY - h - 1;
}

// getAandB with the library PSF of slice r, threshold 10% of its max, on the
// patch minus the sCMOS term when there is one (:1119-1211); returns whether
// the candidate is fitted (maxPatch / B > maxSNR and B > 0).
__device__ bool pipe_a_and_b(const PipeView& V, const double* img, int r, int ci, int cj, double* A_, double* B_,
                             double* maxp_) {
    const double* vm = V.vmap;
    const int R = V.R, h = R / 2, SY = V.SY;
    const double* psf = V.libpsf + (size_t)r * R * R;
    double maxp = -INFINITY, maxi = -INFINITY;
    for (int a = 0; a < R; ++a)
        for (int b = 0; b < R; ++b) {
            const size_t px = (size_t)(ci - h + a) * SY + (cj - h + b);
            maxi = fmax(maxi, psf[a * R + b]);
            maxp = fmax(maxp, img[px] - (vm ? vm[px] : 0.0));
        }
    const double thr = maxi * 0.1;
    double B = 0, A = 0, cb = 0, ca = 0;
    for (int a = 0; a < R; ++a)
        for (int b = 0; b < R; ++b) {
            const size_t px = (size_t)(ci - h + a) * SY + (cj - h + b);
            const double v = img[px] - (vm ? vm[px] : 0.0);
            if (psf[a * R + b] < thr) { B += v; cb += 1; } else { A += v; ca += 1; }
        }
    B = cb != 0 ? B / cb : 0.0;
    A -= ca * B;
    *A_ = A;
    *B_ = B;
    *maxp_ = maxp;
    return maxp / B > V.max_snr && B > 0;
}

// One wave's selection for one frame (one CTA): walking the candidates from
// the frame's pointer in chunks of blockDim, each thread tests one candidate
// under the current mask; the first K that need a fit (in candidate order) get
// slots and their ROI and start.  limit = just past the K-th (or the end).
__global__ void __launch_bounds__(128) k_pipe_wave(PipeView V, int K) {
    const int f = blockIdx.x, SX = V.SX, SY = V.SY, R = V.R, h = R / 2, RR = R * R;
    if (V.done[f]) return;
    const double* img = V.fimg + (size_t)f * SX * SY;
    const unsigned char* mk = V.mask + (size_t)f * SX * SY;
    const double* cand = V.cand + (size_t)f * V.cap * 7;
    const int n = min(V.counts[f], V.cap);
    __shared__ unsigned char sel[128];
    __shared__ int s_got, s_lim, s_base;
    int taken = 0, limit = n;
    for (int c0 = V.pointer[f]; c0 < n && taken < K; c0 += blockDim.x) {
        const int i = c0 + threadIdx.x;
        int code = -4;
        double A = 0, B = 0, maxp = 0;
        if (i < n) {
            const double* row = cand + (size_t)i * 7;
            const int r = (int)llrint(row[1]), ci = (int)llrint(row[2]), cj = (int)llrint(row[3]);
            if (!pipe_inside(V, ci, cj)) {
                code = -2;
            } else {
                bool masked = mk[(size_t)ci * SY + cj] != 0;
                for (int k = 0; k < RR && !masked; ++k) masked = mk[(size_t)(ci - h + k / R) * SY + (cj - h + k % R)] != 0;
                code = masked ? -3 : (pipe_a_and_b(V, img, r, ci, cj, &A, &B, &maxp) ? 0 : -1);
            }
            V.cand_slot[(size_t)f * V.cap + i] = code;
            V.cand_maxp[(size_t)f * V.cap + i] = maxp;
        }
        sel[threadIdx.x] = code == 0;
        __syncthreads();
        if (threadIdx.x == 0) {
            int got = 0, lim = -1;
            for (int t = 0; t < (int)blockDim.x && c0 + t < n; ++t) {
                if (!sel[t]) continue;
                if (got == K - taken) { sel[t] = 0; continue; }
                ++got;
                if (got == K - taken) lim = c0 + t + 1;
            }
            if (lim >= 0)
                for (int t = lim - c0; t < (int)blockDim.x; ++t) sel[t] = 0;
            s_got = got;
            s_lim = lim;
            s_base = got ? atomicAdd(V.nslots, got) : 0;
            int k = 0;
            for (int t = 0; t < (int)blockDim.x && c0 + t < n; ++t)
                if (sel[t]) {
                    const int s = s_base + k++;
                    V.cand_slot[(size_t)f * V.cap + c0 + t] = s < V.slot_cap ? s : -5;
                }
        }
        __syncthreads();
        if (sel[threadIdx.x]) {
            const int s = V.cand_slot[(size_t)f * V.cap + i];
            if (s >= 0) {
                const double* row = cand + (size_t)i * 7;
                const int r = (int)llrint(row[1]), ci = (int)llrint(row[2]), cj = (int)llrint(row[3]);
                float* roi = V.rois + (size_t)s * RR;
                for (int a = 0; a < R; ++a)
                    for (int b = 0; b < R; ++b) roi[a * R + b] = (float)img[(size_t)(ci - h + a) * SY + (cj - h + b)];
                if (V.vmap) {
                    float* sv = V.slot_v + (size_t)s * RR;
                    for (int a = 0; a < R; ++a)
                        for (int b = 0; b < R; ++b) sv[a * R + b] = (float)V.vmap[(size_t)(ci - h + a) * SY + (cj - h + b)];
                }
                double* in = V.init + (size_t)s * 5;  // loc.init(A, B, -dx, -dy, range[r] + dz)
                in[0] = -row[5];
                in[1] = -row[6];
                in[2] = V.range[r] + row[4];
                in[3] = A;
                in[4] = B;
                V.slot_frame[s] = f;
                V.slot_cand[s] = i;
            }
        }
        taken += s_got;
        if (s_lim >= 0) limit = s_lim;
        __syncthreads();
    }
    if (threadIdx.x == 0) V.limit[f] = limit;
}

// The fitted slots that can be accepted whatever the mask: every test of the
// walk's acceptance (k_pipe_replay) but the mask's, with the same arithmetic.
// Only these need the model at their fit (the walk masks by the model only
// where it accepts); they are listed in list[0 .. *count).
__device__ __forceinline__ bool pipe_static_pass(const PipeView& V, const double* theta, const int* status, int slot,
                                                 int ci, int cj) {
    if (status[slot] == ZOLA_FIT_NAN) return false;
    const double* th = theta + (size_t)slot * 5;
    const double x = th[0], y = th[1], z = th[2], A = th[3];
    if (!(A > V.photon_thr && fabs(x) < 10 * V.dx && fabs(y) < 10 * V.dx)) return false;
    const int px = (int)(ci - x / V.dx), py = (int)(cj - y / V.dx);
    return px >= 0 && px < V.SX && py >= 0 && py < V.SY && z > V.minZ && z < V.maxZ;
}

__global__ void k_pipe_need(PipeView V, int n, const double* theta, const int* status, int* list, int* count) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double* row = V.cand + ((size_t)V.slot_frame[s] * V.cap + V.slot_cand[s]) * 7;
    if (pipe_static_pass(V, theta, status, s, (int)llrint(row[2]), (int)llrint(row[3]))) list[atomicAdd(count, 1)] = s;
}

// Model threshold of each listed slot: 0.2 max(0, max(model - B)), model =
// psi A + B (+ sCMOS v) (maxModelThreshold, LocalizationPipeline.java:860-880).
__global__ void k_pipe_mthr(int n, int RR, const double* theta, const double* psi, const float* slot_v, double* mthr,
                            const int* list, const int* count) {
    const int li = blockIdx.x * blockDim.x + threadIdx.x;
    if (li >= min(n, *count)) return;
    const int s = list[li];
    const double A = theta[5 * s + 3], B = theta[5 * s + 4];
    const double* ps = psi + (size_t)s * RR;
    const float* sv = slot_v ? slot_v + (size_t)s * RR : nullptr;
    double m = 0.0;
    for (int k = 0; k < RR; ++k) m = fmax(m, ps[k] * A + B + (sv ? (double)sv[k] : 0.0) - B);
    mthr[s] = m * 0.2;
}

// The reference's sequential walk over one frame's candidates (one CTA per
// frame), with the speculative fits.  Accepted slots are listed with their
// candidate index as the in-frame order.
__global__ void __launch_bounds__(256) k_pipe_replay(PipeView V, const double* theta, const int* status,
                                                     const double* psi, const double* mthr, int* acc_slot,
                                                     int* acc_seq, int* nacc) {
    const int f = blockIdx.x, SX = V.SX, SY = V.SY, R = V.R, h = R / 2, RR = R * R;
    unsigned char* mk = V.mask + (size_t)f * SX * SY;
    const double* img = V.fimg + (size_t)f * SX * SY;
    const double* cand = V.cand + (size_t)f * V.cap * 7;
    if (V.done[f]) return;
    const int n = min(V.counts[f], V.cap), lim = V.limit[f];
    for (int i = V.pointer[f]; i < lim; ++i) {
        const int slot = V.cand_slot[(size_t)f * V.cap + i];
        if (slot == -2 || slot == -3) continue;  // outside the border, or masked (masks only grow)
        const int ci = (int)llrint(cand[(size_t)i * 7 + 2]), cj = (int)llrint(cand[(size_t)i * 7 + 3]);
        if (mk[(size_t)ci * SY + cj]) continue;  // uniform read of the (synchronised) mask
        bool mine = false;
        for (int k = threadIdx.x; k < RR; k += blockDim.x)
            mine |= mk[(size_t)(ci - h + k / R) * SY + (cj - h + k % R)] != 0;
        if (__syncthreads_or(mine)) continue;  // alreadyTreated
        const double maxp = V.cand_maxp[(size_t)f * V.cap + i];
        bool accepted = false;
        if (slot >= 0 && pipe_static_pass(V, theta, status, slot, ci, cj)) {
            const double* th = theta + (size_t)slot * 5;
            const int px = (int)(ci - th[0] / V.dx), py = (int)(cj - th[1] / V.dx);
            accepted = !mk[(size_t)px * SY + py];
        }
        __syncthreads();  // every thread has read the mask before it changes
        if (accepted) {
            if (threadIdx.x == 0) {
                const int o = atomicAdd(nacc, 1);
                acc_slot[o] = slot;
                acc_seq[o] = i;
            }
            const double A = theta[(size_t)slot * 5 + 3], B = theta[(size_t)slot * 5 + 4], thr = mthr[slot];
            const double* ps = psi + (size_t)slot * RR;
            const float* sv = V.vmap ? V.slot_v + (size_t)slot * RR : nullptr;
            for (int k = threadIdx.x; k < RR; k += blockDim.x)
                if (ps[k] * A + B + (sv ? (double)sv[k] : 0.0) - B > thr)
                    mk[(size_t)(ci - h + k / R) * SY + (cj - h + k % R)] = 1;
        } else {
            for (int k = threadIdx.x; k < RR; k += blockDim.x) {
                const size_t px = (size_t)(ci - h + k / R) * SY + (cj - h + k % R);
                if (img[px] > maxp * 0.5) mk[px] = 1;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        V.pointer[f] = lim;
        V.done[f] = lim >= n;
    }
}

struct LocRow {
    int frame, seq, status;
    double x, y, z, A, B, chi2, cx, cy, cz;
};

__global__ void k_take_xyz(int n, const double* theta, double* xyz) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n)
        for (int q = 0; q < 3; ++q) xyz[3 * s + q] = theta[5 * (size_t)s + q];
}

__global__ void k_take_acc(int n, const int* acc_slot, const double* theta, double* xyz) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n)
        for (int q = 0; q < 3; ++q) xyz[3 * k + q] = theta[5 * (size_t)acc_slot[k] + q];
}

// chi2 and CRLB of the accepted localizations (psi, dpsi evaluated at their
// fitted positions, in acceptance-list order).
__global__ void k_pipe_rows(PipeView V, int n, const int* acc_slot, const int* acc_seq, const int* status,
                            const double* theta,
                            const double* psi, const double* dpsi, LocRow* rows) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int s = acc_slot[k], R = V.R, RR = R * R;
    const int f = V.slot_frame[s], i = V.slot_cand[s];
    const double* row = V.cand + ((size_t)f * V.cap + i) * 7;
    const int ci = (int)llrint(row[2]), cj = (int)llrint(row[3]);
    const double* th = theta + (size_t)s * 5;
    const double x = th[0], y = th[1], z = th[2], A = th[3], B = th[4];
    const double* ps = psi + (size_t)k * RR;
    const float* roi = V.rois + (size_t)s * RR;
    const float* sv = V.vmap ? V.slot_v + (size_t)s * RR : nullptr;
    double chi = 0;
    for (int q = 0; q < RR; ++q) {  // scoreCompute against the model (with the sCMOS term)
        const double mu = ps[q] * A + B + (sv ? (double)sv[q] : 0.0);
        const double dd = roi[q] - mu;
        chi += dd * dd / mu;
    }
    chi /= RR;
    double F[25];
    for (int q = 0; q < 25; ++q) F[q] = 0;
    for (int p = 0; p < RR; ++p) {
        const double mu = ps[p] * A + B;
        const double d[5] = {A * dpsi[((size_t)k * 3 + 0) * RR + p], A * dpsi[((size_t)k * 3 + 1) * RR + p],
                             A * dpsi[((size_t)k * 3 + 2) * RR + p], mu, 1.0};
        for (int q = 0; q < 5; ++q)
            for (int r2 = 0; r2 < 5; ++r2) F[q * 5 + r2] += d[q] * d[r2] / mu;
    }
    double cr[5];
    lm_crlb(F, cr);
    for (int q = 0; q < 3; ++q)
        if (!(cr[q] == cr[q])) cr[q] = F[q * 5 + q] != 0 ? sqrt(1.0 / F[q * 5 + q]) : 1.79769313486231570e308;
    LocRow& L = rows[k];
    L.frame = f; L.seq = acc_seq[k]; L.status = status[s];
    L.x = 1000 * (ci * V.dx - x); L.y = 1000 * (cj * V.dx - y); L.z = 1000 * z;
    L.A = A; L.B = B; L.chi2 = chi;
    L.cx = 1000 * cr[0]; L.cy = 1000 * cr[1]; L.cz = 1000 * cr[2];
}

}  // namespace zola

using namespace zola;

namespace {

struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
    Buf() = default;
    Buf(const Buf&) = delete;
    Buf& operator=(const Buf&) = delete;
    ~Buf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t b) {
        if (b <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, b ? b : 1);
        if (e == cudaSuccess) bytes = b ? b : 1;
        return e;
    }
};

constexpr int PIPE_WAVE_FITS = 8;  // speculative fits per frame and wave
// Candidates stored per frame at the start of a call: a 256 x 256 frame against a
// 41-slice library lists up to about 7,500 at the reference's threshold.
constexpr int PIPE_CAND_ROOM = 8192;

}  // namespace

namespace zola {

// sCMOS frames (LocalizationPipeline.java:588-640): c = (ADU - offset)/gain;
// detection image c + vargain[0] clamped at 0, fit image c + vargain.
__global__ void k_pipe_scmos(const float* adu, const double* offset, const double* gain, const double* vg, size_t SS,
                             int nf, double* det_img, double* fit_img) {
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < SS * nf; k += (size_t)gridDim.x * blockDim.x) {
        const size_t px = k % SS;
        const double c = ((double)adu[k] - offset[px]) / gain[px];
        const double d = c + vg[0];
        det_img[k] = d < 0 ? 0 : d;
        fit_img[k] = c + vg[px];
    }
}

}  // namespace zola

namespace {

// frames: photon frames (no sCMOS); or adu + offset/gain/variance maps (sCMOS).
// u16: camera counts (with rescale = {slope, intercept}) instead of photon frames.
int localize_impl(zola_ctx* ctx, zola_detector* det, zola_psf* fit_psf, const double* frames, const float* adu,
                  const double* offset, const double* gain, const double* variance, int nframes, int frame0,
                  const zola_loc_params* prm, zola_localization* out, int out_cap, int* nout,
                  const uint16_t* u16 = nullptr, const double* rescale = nullptr) {
    const bool scmos = adu != nullptr;
    *nout = 0;
    if (nframes <= 0) return ZOLA_OK;
    const int SX = det->v.SX, SY = det->v.SY, R = det->v.R;
    if (det->psf->ctx != ctx || fit_psf->ctx != ctx) { ctx->err = "zola_localize_frames: objects of another context"; return ZOLA_E_ARG; }
    if (prm->patch != R) { ctx->err = "zola_localize_frames: params.patch must equal the detector's R"; return ZOLA_E_ARG; }
    if (fit_psf->o.kz_reset) { ctx->err = "zola_localize_frames: the fit PSF needs kz_reset = 0"; return ZOLA_E_ARG; }
    const std::vector<double>& range = det->range;
    const std::vector<double>& lib = det->h_psf;
    // candidates stored per frame: grows to the longest list met, so that every
    // frame walks its whole list as the reference does
    int cap = prm->cand_cap > 0 ? prm->cand_cap : std::max(PIPE_CAND_ROOM, det->cand_room);
    if (cap > ZOLA_DETECT_MAX_CAP) { ctx->err = "zola_localize_frames: cand_cap above 2^20"; return ZOLA_E_ARG; }
    const int FB = std::max(1, std::min(nframes, prm->frames_per_batch > 0 ? prm->frames_per_batch : 1024));
    const size_t SS = (size_t)SX * SY, RR = (size_t)R * R;
    cudaStream_t st = ctx->stream;
    const int K = prm->wave_fits > 0 ? prm->wave_fits : PIPE_WAVE_FITS;
    const int slot_cap = FB * K;
    Buf b_img, b_mask, b_cand, b_cnt, b_lib, b_rng, b_cslot, b_cmax, b_ptr, b_lim, b_done, b_ns, b_rois, b_init, b_sf,
        b_sc, b_out5, b_st, b_xyz, b_psi, b_mthr, b_acc, b_seq, b_nacc, b_dpsi, b_rows, b_fimg, b_adu, b_off, b_gain,
        b_vg, b_sv, b_u16, b_list, b_nlist;
    cudaError_t e = cudaSuccess;
    auto A = [&](Buf& b, size_t bytes) { if (e == cudaSuccess) e = b.alloc(bytes); };
    A(b_img, SS * FB * 8); A(b_mask, SS * FB); A(b_cand, (size_t)FB * cap * 7 * 8); A(b_cnt, (size_t)FB * 4);
    A(b_lib, lib.size() * 8); A(b_rng, range.size() * 8); A(b_cslot, (size_t)FB * cap * 4);
    A(b_cmax, (size_t)FB * cap * 8); A(b_ptr, (size_t)FB * 4); A(b_lim, (size_t)FB * 4); A(b_done, (size_t)FB * 4);
    A(b_ns, 64); A(b_nacc, 64);
    A(b_rois, RR * slot_cap * 4); A(b_init, (size_t)slot_cap * 40); A(b_sf, (size_t)slot_cap * 4);
    A(b_sc, (size_t)slot_cap * 4); A(b_out5, (size_t)slot_cap * 40); A(b_st, (size_t)slot_cap * 4);
    A(b_xyz, (size_t)slot_cap * 24); A(b_psi, RR * slot_cap * 8); A(b_mthr, (size_t)slot_cap * 8);
    A(b_acc, (size_t)slot_cap * 4); A(b_seq, (size_t)slot_cap * 4);
    if (u16) A(b_u16, SS * FB * 2);
    A(b_list, (size_t)slot_cap * 4); A(b_nlist, 64);
    if (scmos) {
        A(b_fimg, SS * FB * 8); A(b_adu, SS * FB * 4); A(b_off, SS * 8); A(b_gain, SS * 8); A(b_vg, SS * 8);
        A(b_sv, RR * slot_cap * 4);
        std::vector<double> vg(SS);
        for (size_t k = 0; k < SS; ++k) vg[k] = variance[k] / (gain[k] * gain[k]);  // SCMOScamera.java:95
        if (e == cudaSuccess) e = cudaMemcpy(b_vg.p, vg.data(), SS * 8, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b_off.p, offset, SS * 8, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(b_gain.p, gain, SS * 8, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(b_lib.p, lib.data(), lib.size() * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b_rng.p, range.data(), range.size() * 8, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) { ctx->err = std::string("zola_localize_frames: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
    zola_fit_params fp{prm->minZ - 0.3, prm->maxZ + 0.3, 10 * fit_psf->o.xystep + 1e-3, prm->max_iter, prm->tol_xyz,
                       fit_psf->o.xystep, 2 * fit_psf->o.xystep, prm->precision};
    PipeView V{};
    V.SX = SX; V.SY = SY; V.R = R; V.cap = cap;
    V.dx = fit_psf->o.xystep; V.minZ = prm->minZ; V.maxZ = prm->maxZ; V.photon_thr = prm->photon_threshold;
    V.max_snr = prm->max_snr;
    V.images = (double*)b_img.p; V.mask = (unsigned char*)b_mask.p; V.cand = (double*)b_cand.p;
    V.fimg = scmos ? (double*)b_fimg.p : (double*)b_img.p;
    V.vmap = scmos ? (double*)b_vg.p : nullptr;
    V.slot_v = scmos ? (float*)b_sv.p : nullptr;
    V.counts = (int*)b_cnt.p; V.libpsf = (double*)b_lib.p; V.range = (double*)b_rng.p;
    V.cand_slot = (int*)b_cslot.p; V.cand_maxp = (double*)b_cmax.p; V.pointer = (int*)b_ptr.p;
    V.limit = (int*)b_lim.p; V.done = (int*)b_done.p; V.nslots = (int*)b_ns.p; V.slot_cap = slot_cap;
    V.rois = (float*)b_rois.p; V.init = (double*)b_init.p; V.slot_frame = (int*)b_sf.p; V.slot_cand = (int*)b_sc.p;
    std::vector<LocRow> all;
    std::vector<int> done;
    auto fail = [&](cudaError_t err) {
        ctx->err = std::string("zola_localize_frames: ") + cudaGetErrorString(err);
        return ZOLA_E_CUDA;
    };
    for (int f0 = 0; f0 < nframes; f0 += FB) {
        const int nf = std::min(FB, nframes - f0);
        V.nframes = nf;
        if (scmos) {
            e = cudaMemcpyAsync(b_adu.p, adu + (size_t)f0 * SS, SS * nf * 4, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) {
                k_pipe_scmos<<<ctx->num_sms * 8, 256, 0, st>>>((float*)b_adu.p, (double*)b_off.p, (double*)b_gain.p,
                                                              (double*)b_vg.p, SS, nf, (double*)b_img.p,
                                                              (double*)b_fimg.p);
                ctx->launches++;
            }
        } else if (u16) {  // 2 bytes a pixel over the host link, photons made on the device
            e = cudaMemcpyAsync(b_u16.p, u16 + (size_t)f0 * SS, SS * nf * 2, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) rescale_u16(ctx, (const uint16_t*)b_u16.p, SS * nf, rescale, (double*)b_img.p, st);
        } else {
            e = cudaMemcpyAsync(b_img.p, frames + (size_t)f0 * SS, SS * nf * 8, cudaMemcpyHostToDevice, st);
        }
        if (e == cudaSuccess) e = cudaMemsetAsync(b_mask.p, 0, SS * nf, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(b_ptr.p, 0, (size_t)nf * 4, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(b_done.p, 0, (size_t)nf * 4, st);
        if (e != cudaSuccess) return fail(e);
        int rc = zola_detect_dev(det, (double*)b_img.p, nf, cap, (double*)b_cand.p, (int*)b_cnt.p, st);
        if (rc) return rc;
        std::vector<int> counts(nf);
        e = cudaMemcpyAsync(counts.data(), b_cnt.p, (size_t)nf * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(e);
        const int longest = *std::max_element(counts.begin(), counts.end());
        det->cand_room = std::max(det->cand_room, longest);
        if (longest > cap) {  // room for every candidate; the frames whose list was cut are detected again
            if (longest > ZOLA_DETECT_MAX_CAP) {
                ctx->err = "zola_localize_frames: a frame has more than 2^20 candidates";
                return ZOLA_E_ARG;
            }
            const int old = cap;
            cap = longest;
            {
                // the stored rows move to the wider layout; the frames whose whole list
                // fitted keep them (detection is per frame, so they would come out the same)
                Buf wide;
                e = wide.alloc((size_t)FB * cap * 7 * 8);
                if (e == cudaSuccess)
                    e = cudaMemcpy2DAsync(wide.p, (size_t)cap * 7 * 8, b_cand.p, (size_t)old * 7 * 8,
                                          (size_t)old * 7 * 8, nf, cudaMemcpyDeviceToDevice, st);
                if (e != cudaSuccess) return fail(e);
                std::swap(b_cand.p, wide.p);
                std::swap(b_cand.bytes, wide.bytes);
            }  // (freeing the old rows waits for the copy)
            A(b_cslot, (size_t)FB * cap * 4); A(b_cmax, (size_t)FB * cap * 8);
            if (e != cudaSuccess) return fail(e);
            V.cap = cap;
            V.cand = (double*)b_cand.p; V.cand_slot = (int*)b_cslot.p; V.cand_maxp = (double*)b_cmax.p;
            // the cut frames, gathered, are detected again as one batch and their rows scattered back
            std::vector<int> cut;
            for (int f = 0; f < nf; ++f)
                if (counts[f] > old) cut.push_back(f);
            const size_t nc = cut.size();
            Buf g_img, g_out, g_cnt;
            e = g_img.alloc(nc * SS * 8);
            if (e == cudaSuccess) e = g_out.alloc(nc * (size_t)cap * 7 * 8);
            if (e == cudaSuccess) e = g_cnt.alloc(nc * 4);
            for (size_t k = 0; k < nc && e == cudaSuccess; ++k)
                e = cudaMemcpyAsync((double*)g_img.p + k * SS, (double*)b_img.p + (size_t)cut[k] * SS, SS * 8,
                                    cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return fail(e);
            rc = zola_detect_dev(det, (double*)g_img.p, (int)nc, cap, (double*)g_out.p, (int*)g_cnt.p, st);
            if (rc) return rc;
            for (size_t k = 0; k < nc && e == cudaSuccess; ++k) {
                e = cudaMemcpyAsync((double*)b_cand.p + (size_t)cut[k] * cap * 7, (double*)g_out.p + k * cap * 7,
                                    (size_t)cap * 7 * 8, cudaMemcpyDeviceToDevice, st);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync((int*)b_cnt.p + cut[k], (int*)g_cnt.p + k, 4, cudaMemcpyDeviceToDevice, st);
            }
            if (e != cudaSuccess) return fail(e);
        }  // (freeing the gathered buffers waits for the copies)
        for (int wave = 0;; ++wave) {
            e = cudaMemsetAsync(b_ns.p, 0, 4, st);
            if (e == cudaSuccess) e = cudaMemsetAsync(b_nacc.p, 0, 4, st);
            if (e != cudaSuccess) return fail(e);
            k_pipe_wave<<<nf, 128, 0, st>>>(V, K);
            ctx->launches++;
            int nslot = 0;
            e = cudaMemcpyAsync(&nslot, b_ns.p, 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return fail(e);
            if (nslot > 0) {
                rc = scmos ? zola_fit_batch_scmos_dev(ctx, fit_psf, R, (float*)b_rois.p, (float*)b_sv.p,
                                                      (double*)b_init.p, nslot, &fp, (double*)b_out5.p, nullptr,
                                                      nullptr, (int*)b_st.p, nullptr, st)
                           : zola_fit_batch_dev(ctx, fit_psf, R, (float*)b_rois.p, (double*)b_init.p, nslot, &fp,
                                                (double*)b_out5.p, nullptr, nullptr, (int*)b_st.p, nullptr, st);
                if (rc) return rc;
                // psi at the fitted positions the walk may accept (its model masks)
                k_take_xyz<<<(nslot + 127) / 128, 128, 0, st>>>(nslot, (double*)b_out5.p, (double*)b_xyz.p);
                e = cudaMemsetAsync(b_nlist.p, 0, 4, st);
                if (e != cudaSuccess) return fail(e);
                k_pipe_need<<<(nslot + 127) / 128, 128, 0, st>>>(V, nslot, (double*)b_out5.p, (int*)b_st.p,
                                                                 (int*)b_list.p, (int*)b_nlist.p);
                ctx->launches += 2;
                WindowTables* wt = get_window(fit_psf, R, ctx->err);
                if (!wt) return ZOLA_E_ARG;
                rc = launch_model_f64(ctx, fit_psf, wt, (double*)b_xyz.p, nslot, (double*)b_psi.p, nullptr, st,
                                      (const int*)b_list.p, (const int*)b_nlist.p);
                if (rc) return rc;
                k_pipe_mthr<<<(nslot + 127) / 128, 128, 0, st>>>(nslot, (int)RR, (double*)b_out5.p,
                                                                 (double*)b_psi.p, V.slot_v, (double*)b_mthr.p,
                                                                 (const int*)b_list.p, (const int*)b_nlist.p);
                ctx->launches++;
            }
            k_pipe_replay<<<nf, 256, 0, st>>>(V, (double*)b_out5.p, (int*)b_st.p, (double*)b_psi.p,
                                             (double*)b_mthr.p, (int*)b_acc.p, (int*)b_seq.p, (int*)b_nacc.p);
            ctx->launches++;
            int nacc = 0;
            done.assign(nf, 0);
            e = cudaMemcpyAsync(&nacc, b_nacc.p, 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(done.data(), b_done.p, (size_t)nf * 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return fail(e);
            if (nacc > 0) {
                A(b_dpsi, 3 * RR * (size_t)nacc * 8); A(b_rows, (size_t)nacc * sizeof(LocRow));
                if (e != cudaSuccess) return fail(e);
                k_take_acc<<<(nacc + 127) / 128, 128, 0, st>>>(nacc, (int*)b_acc.p, (double*)b_out5.p,
                                                               (double*)b_xyz.p);
                ctx->launches++;
                // the walk has used psi; its buffer now takes the accepted positions' models
                rc = zola_psf_model_dev(fit_psf, R, (double*)b_xyz.p, nacc, (double*)b_psi.p, (double*)b_dpsi.p, st);
                if (rc) return rc;
                k_pipe_rows<<<(nacc + 127) / 128, 128, 0, st>>>(V, nacc, (int*)b_acc.p, (int*)b_seq.p, (int*)b_st.p,
                                                                (double*)b_out5.p, (double*)b_psi.p,
                                                                (double*)b_dpsi.p, (LocRow*)b_rows.p);
                ctx->launches++;
                std::vector<LocRow> rows(nacc);
                e = cudaMemcpyAsync(rows.data(), b_rows.p, (size_t)nacc * sizeof(LocRow), cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) return fail(e);
                for (auto& r : rows) r.frame += f0;
                all.insert(all.end(), rows.begin(), rows.end());
            }
            if (std::all_of(done.begin(), done.end(), [](int d) { return d != 0; })) break;
        }
    }
    std::sort(all.begin(), all.end(), [](const LocRow& a, const LocRow& b) {
        return a.frame != b.frame ? a.frame < b.frame : a.seq < b.seq;
    });
    if ((int)all.size() > out_cap) { ctx->err = "zola_localize_frames: out_cap too small"; *nout = (int)all.size(); return ZOLA_E_ARG; }
    for (size_t k = 0; k < all.size(); ++k) {
        const LocRow& r = all[k];
        zola_localization& L = out[k];
        L.id = (int)k;
        L.frame = frame0 + r.frame;
        L.x_nm = r.x; L.y_nm = r.y; L.z_nm = r.z; L.intensity = r.A; L.background = r.B; L.chi2 = r.chi2;
        L.crlb_x_nm = r.cx; L.crlb_y_nm = r.cy; L.crlb_z_nm = r.cz;
        L.candidate = r.seq;
        L.fit_status = r.status;
    }
    *nout = (int)all.size();
    return ZOLA_OK;
}

}  // namespace

extern "C" int zola_localize_frames(zola_ctx* ctx, zola_detector* det, zola_psf* fit_psf, const double* frames,
                                    int nframes, int frame0, const zola_loc_params* prm, zola_localization* out,
                                    int out_cap, int* nout) {
    if (!ctx || !det || !fit_psf || !prm || !nout || (nframes > 0 && (!frames || !out))) return ZOLA_E_ARG;
    return localize_impl(ctx, det, fit_psf, frames, nullptr, nullptr, nullptr, nullptr, nframes, frame0, prm, out,
                         out_cap, nout);
}

extern "C" int zola_localize_frames_u16(zola_ctx* ctx, zola_detector* det, zola_psf* fit_psf, const uint16_t* frames,
                                        int nframes, int frame0, const zola_loc_params* prm, double adu, double gain,
                                        double offset, zola_localization* out, int out_cap, int* nout) {
    if (!ctx || !det || !fit_psf || !prm || !nout || (nframes > 0 && (!frames || !out))) return ZOLA_E_ARG;
    if (!(gain != 0) || !std::isfinite(adu) || !std::isfinite(gain) || !std::isfinite(offset)) {
        ctx->err = "zola_localize_frames_u16: adu, gain, offset must be finite and gain non-zero";
        return ZOLA_E_ARG;
    }
    double rescale[2];
    camera_rescale(adu, gain, offset, rescale);
    return localize_impl(ctx, det, fit_psf, nullptr, nullptr, nullptr, nullptr, nullptr, nframes, frame0, prm, out,
                         out_cap, nout, frames, rescale);
}

extern "C" int zola_localize_frames_scmos(zola_ctx* ctx, zola_detector* det, zola_psf* fit_psf, const float* adu,
                                          int nframes, int frame0, const zola_loc_params* prm, const double* offset,
                                          const double* gain, const double* variance, zola_localization* out,
                                          int out_cap, int* nout) {
    if (!ctx || !det || !fit_psf || !prm || !nout || (nframes > 0 && (!adu || !out)) || !offset || !gain || !variance)
        return ZOLA_E_ARG;
    return localize_impl(ctx, det, fit_psf, nullptr, adu, offset, gain, variance, nframes, frame0, prm, out, out_cap,
                         nout);
}

// ThunderStorm-style CSV (data/PLocalization.java:224-306): values floored to
// 1e-3 (PLocalization.java:59-72) and printed as Java's Double.toString does.
namespace {

std::string java_double(double v) {
    if (v != v) return "NaN";
    if (std::isinf(v)) return v > 0 ? "Infinity" : "-Infinity";
    if (v == 0) return std::signbit(v) ? "-0.0" : "0.0";
    char buf[64];
    int prec = 1;
    for (; prec <= 17; ++prec) {  // shortest round-trip digits
        std::snprintf(buf, sizeof buf, "%.*e", prec - 1, v);
        if (std::strtod(buf, nullptr) == v) break;
    }
    // buf = d.ddddde[+-]XX ; split into digits and exponent
    std::string s(buf);
    size_t epos = s.find('e');
    int exp10 = std::atoi(s.c_str() + epos + 1);
    std::string mant = s.substr(0, epos);
    bool neg = mant[0] == '-';
    if (neg) mant = mant.substr(1);
    std::string digits;
    for (char c : mant) if (c != '.') digits += c;
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    std::string r;
    const double a = std::fabs(v);
    if (a >= 1e-3 && a < 1e7) {
        int point = exp10 + 1;  // digits before the decimal point
        if (point <= 0) {
            r = "0." + std::string(-point, '0') + digits;
        } else if ((int)digits.size() <= point) {
            r = digits + std::string(point - digits.size(), '0') + ".0";
        } else {
            r = digits.substr(0, point) + "." + digits.substr(point);
        }
    } else {
        r = digits.substr(0, 1) + "." + (digits.size() > 1 ? digits.substr(1) : std::string("0")) + "E" +
            std::to_string(exp10);
    }
    return neg ? "-" + r : r;
}

double floor3(double v) { return std::floor(1000 * v) / 1000; }

}  // namespace

extern "C" int zola_write_csv(const char* path, const zola_localization* locs, int n, int append) {
    if (!path || n < 0 || (n > 0 && !locs)) return ZOLA_E_ARG;
    FILE* fp = std::fopen(path, append ? "a" : "w");
    if (!fp) return ZOLA_E_ARG;
    if (!append)
        std::fputs("id,frame,x [nm],y [nm],z [nm],intensity,background,chi2,crlbX,crlbY,crlbZ,driftX,driftY,driftZ,"
                   "occurrenceMerging\n", fp);
    for (int k = 0; k < n; ++k) {
        const zola_localization& L = locs[k];
        std::string line = std::to_string(L.id) + "," + std::to_string(L.frame) + "," + java_double(floor3(L.x_nm)) +
                           "," + java_double(floor3(L.y_nm)) + "," + java_double(floor3(L.z_nm)) + "," +
                           java_double(floor3(L.intensity)) + "," + java_double(floor3(L.background)) + "," +
                           java_double(floor3(L.chi2)) + "," + java_double(floor3(L.crlb_x_nm)) + "," +
                           java_double(floor3(L.crlb_y_nm)) + "," + java_double(floor3(L.crlb_z_nm)) +
                           ",0.0,0.0,0.0,1\n";
        std::fputs(line.c_str(), fp);
    }
    std::fclose(fp);
    return ZOLA_OK;
}

extern "C" int zola_format_double_java(double v, char* buf, int len) {
    if (!buf || len <= 0) return ZOLA_E_ARG;
    std::string s = java_double(v);
    if ((int)s.size() + 1 > len) return ZOLA_E_ARG;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return ZOLA_OK;
}
