// Frame localization pipeline: detection -> candidate selection -> fit ->
// filters and mask -> localization rows (process/cpu/LocalizationPipeline.java).
//
// The reference walks each frame's sorted candidate list on a Java thread
// (LocalizationThread.run, LocalizationPipeline.java:720-990):
//   - next candidate whose centre pixel is unmasked and inside the border
//     (myGetMaxPositions, :1218-1250);
//   - skip it if any pixel of its R x R patch is masked;
//   - getAandB init from the library PSF of its slice (:1119-1162); fit only
//     if maxPatch / B > maxSNR (1) and B > 0;
//   - accept if A > photonThreshold, |x|,|y| < 10 px, the rounded position is
//     inside the frame and unmasked, and minZ < z < maxZ (:859-945); then mask
//     the pixels where model - B > 0.2 max(model - B);
//   - otherwise mask the patch pixels above half the patch maximum (:967-977).
// The mask makes each frame sequential, so frames are processed in waves:
// every wave advances each frame to its next candidate that needs a fit (one
// per frame) and fits all of them in one batched call (FP64 or split), then
// applies the filters and masks.  Rows come out in frame order and, within a
// frame, in processing order; x/y/z in nm as 1000*(i*dx - x) (:905-907), chi2
// as scoreCompute (:1099-1115), CRLB from the Fisher matrix the reference
// forms (Localization.java:317-451: dmu/dA taken as mu, h -> 0 limit).
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
    const double* images;     // nframes x SX x SY
    unsigned char* mask;      // nframes x SX x SY
    const double* cand;       // nframes x cap x 7
    const int* counts;        // nframes
    int* pointer;             // nframes
    int* done;                // nframes
    const double* libpsf;     // Z x R x R (normalised library PSFs)
    const double* range;      // Z
    // wave outputs
    int* slot_frame;          // n_slots: frame of each fit slot
    int* nslots;
    float* rois;              // slots x R x R
    double* init;             // slots x 5
    double* meta;             // slots x 4: ci, cj, maxPatch, candidate index
};

// Advance every frame to its next candidate that needs a fit.
__global__ void k_pipe_select(PipeView V) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= V.nframes || V.done[f]) return;
    const int SX = V.SX, SY = V.SY, R = V.R, h = R / 2;
    const double* img = V.images + (size_t)f * SX * SY;
    unsigned char* mk = V.mask + (size_t)f * SX * SY;
    const double* cand = V.cand + (size_t)f * V.cap * 7;
    const int n = min(V.counts[f], V.cap);
    int p = V.pointer[f];
    while (true) {
        int sel = -1;
        for (int i = p; i < n; ++i) {  // myGetMaxPositions
            const int ci = (int)llrint(cand[(size_t)i * 7 + 2]), cj = (int)llrint(cand[(size_t)i * 7 + 3]);
            if (mk[(size_t)ci * SY + cj]) continue;
            if (ci > h + 1 && cj > h + 1 && ci < SX - h - 1 && cj < SY - h - 1) {
                sel = i;
                p = i + 1;
                break;
            }
        }
        if (sel < 0) {
            V.done[f] = 1;
            V.pointer[f] = p;
            return;
        }
        const double* row = cand + (size_t)sel * 7;
        const int r = (int)llrint(row[1]), ci = (int)llrint(row[2]), cj = (int)llrint(row[3]);
        bool treated = false;
        for (int a = 0; a < R && !treated; ++a)
            for (int b = 0; b < R; ++b)
                if (mk[(size_t)(ci - h + a) * SY + (cj - h + b)]) { treated = true; break; }
        if (treated) continue;  // alreadyTreated
        // getAandB with the library PSF of slice r, threshold 10% of its max
        const double* psf = V.libpsf + (size_t)r * R * R;
        double maxp = -INFINITY, maxi = -INFINITY;
        for (int a = 0; a < R; ++a)
            for (int b = 0; b < R; ++b) {
                maxi = fmax(maxi, psf[a * R + b]);
                maxp = fmax(maxp, img[(size_t)(ci - h + a) * SY + (cj - h + b)]);
            }
        const double thr = maxi * 0.1;
        double B = 0, A = 0, cb = 0, ca = 0;
        for (int a = 0; a < R; ++a)
            for (int b = 0; b < R; ++b) {
                const double v = img[(size_t)(ci - h + a) * SY + (cj - h + b)];
                if (psf[a * R + b] < thr) { B += v; cb += 1; } else { A += v; ca += 1; }
            }
        B = cb != 0 ? B / cb : 0.0;
        A -= ca * B;
        if (maxp / B > V.max_snr && B > 0) {
            const int s = atomicAdd(V.nslots, 1);
            V.slot_frame[s] = f;
            float* roi = V.rois + (size_t)s * R * R;
            for (int a = 0; a < R; ++a)
                for (int b = 0; b < R; ++b) roi[a * R + b] = (float)img[(size_t)(ci - h + a) * SY + (cj - h + b)];
            double* in = V.init + (size_t)s * 5;  // loc.init(A, B, -dx, -dy, range[r] + dz)
            in[0] = -row[5];
            in[1] = -row[6];
            in[2] = V.range[r] + row[4];
            in[3] = A;
            in[4] = B;
            double* m = V.meta + (size_t)s * 4;
            m[0] = ci; m[1] = cj; m[2] = maxp; m[3] = sel;
            V.pointer[f] = p;
            return;
        }
        // not fitted: mask the patch pixels above half the patch maximum
        for (int a = 0; a < R; ++a)
            for (int b = 0; b < R; ++b)
                if (img[(size_t)(ci - h + a) * SY + (cj - h + b)] > maxp * 0.5) mk[(size_t)(ci - h + a) * SY + (cj - h + b)] = 1;
    }
}

struct LocRow {
    int frame, seq;
    double x, y, z, A, B, chi2, cx, cy, cz;
};

// Filters, mask update and output rows for the fitted slots of one wave.
__global__ void k_pipe_finish(PipeView V, int n, const double* theta, const int* status, const double* psi,
                              const double* dpsi, int wave, LocRow* rows, int* nrows, int rows_cap) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int f = V.slot_frame[s], SX = V.SX, SY = V.SY, R = V.R, h = R / 2, RR = R * R;
    unsigned char* mk = V.mask + (size_t)f * SX * SY;
    const double* m = V.meta + (size_t)s * 4;
    const int ci = (int)m[0], cj = (int)m[1];
    const double maxp = m[2];
    const double* th = theta + (size_t)s * 5;
    const double x = th[0], y = th[1], z = th[2], A = th[3], B = th[4];
    const double* ps = psi + (size_t)s * RR;
    const float* roi = V.rois + (size_t)s * RR;
    bool accepted = false;
    if (status[s] != ZOLA_FIT_NAN) {
        double mmax = 0.0;  // maxModelThreshold starts at 0 (LocalizationPipeline.java:872-880)
        for (int k = 0; k < RR; ++k) mmax = fmax(mmax, ps[k] * A + B - B);
        const double mthr = mmax * 0.2;
        if (A > V.photon_thr && fabs(x) < 10 * V.dx && fabs(y) < 10 * V.dx) {
            const int px = (int)(ci - x / V.dx), py = (int)(cj - y / V.dx);
            if (px >= 0 && px < SX && py >= 0 && py < SY && !mk[(size_t)px * SY + py] && z > V.minZ && z < V.maxZ) {
                accepted = true;
                double chi = 0;
                for (int k = 0; k < RR; ++k) {
                    const double mu = ps[k] * A + B;
                    const double dd = roi[k] - mu;
                    chi += dd * dd / mu;
                }
                chi /= RR;
                // Fisher matrix as the reference forms it: d mu / dA taken as mu
                double F[25];
                for (int q = 0; q < 25; ++q) F[q] = 0;
                for (int k = 0; k < RR; ++k) {
                    const double mu = ps[k] * A + B;
                    const double d[5] = {A * dpsi[((size_t)s * 3 + 0) * RR + k], A * dpsi[((size_t)s * 3 + 1) * RR + k],
                                         A * dpsi[((size_t)s * 3 + 2) * RR + k], mu, 1.0};
                    for (int q = 0; q < 5; ++q)
                        for (int r2 = 0; r2 < 5; ++r2) F[q * 5 + r2] += d[q] * d[r2] / mu;
                }
                double cr[5];
                lm_crlb(F, cr);
                for (int q = 0; q < 3; ++q)
                    if (!(cr[q] == cr[q])) cr[q] = F[q * 5 + q] != 0 ? sqrt(1.0 / F[q * 5 + q]) : 1.79769313486231570e308;
                const int o = atomicAdd(nrows, 1);
                if (o < rows_cap) {
                    LocRow& L = rows[o];
                    L.frame = f; L.seq = wave;
                    L.x = 1000 * (ci * V.dx - x); L.y = 1000 * (cj * V.dx - y); L.z = 1000 * z;
                    L.A = A; L.B = B; L.chi2 = chi;
                    L.cx = 1000 * cr[0]; L.cy = 1000 * cr[1]; L.cz = 1000 * cr[2];
                }
                for (int a = 0; a < R; ++a)
                    for (int b = 0; b < R; ++b)
                        if (ps[a * R + b] * A + B - B > mthr) mk[(size_t)(ci - h + a) * SY + (cj - h + b)] = 1;
            }
        }
    }
    if (!accepted)
        for (int a = 0; a < R; ++a)
            for (int b = 0; b < R; ++b)
                if (roi[a * R + b] > maxp * 0.5) mk[(size_t)(ci - h + a) * SY + (cj - h + b)] = 1;
}

__global__ void k_take_xyz(int n, const double* theta, double* xyz) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n)
        for (int q = 0; q < 3; ++q) xyz[3 * s + q] = theta[5 * s + q];
}

}  // namespace zola

using namespace zola;

namespace {

struct Buf {
    void* p = nullptr;
    ~Buf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t b) { return cudaMalloc(&p, b ? b : 1); }
};

}  // namespace

extern "C" int zola_localize_frames(zola_ctx* ctx, zola_detector* det, zola_psf* fit_psf, const double* frames,
                                    int nframes, int frame0, const zola_loc_params* prm, zola_localization* out,
                                    int out_cap, int* nout) {
    if (!ctx || !det || !fit_psf || !prm || !nout || (nframes > 0 && (!frames || !out))) return ZOLA_E_ARG;
    *nout = 0;
    if (nframes <= 0) return ZOLA_OK;
    const int Z = det->v.Z, SX = det->v.SX, SY = det->v.SY, R = det->v.R;
    if (det->psf->ctx != ctx || fit_psf->ctx != ctx) { ctx->err = "zola_localize_frames: objects of another context"; return ZOLA_E_ARG; }
    if (prm->patch != R) { ctx->err = "zola_localize_frames: params.patch must equal the detector's R"; return ZOLA_E_ARG; }
    if (fit_psf->o.kz_reset) { ctx->err = "zola_localize_frames: the fit PSF needs kz_reset = 0"; return ZOLA_E_ARG; }
    const std::vector<double>& range = det->range;
    const std::vector<double>& lib = det->h_psf;
    const int cap = prm->cand_cap > 0 ? prm->cand_cap : 1024;
    const int FB = std::max(1, std::min(nframes, prm->frames_per_batch > 0 ? prm->frames_per_batch : 1024));
    const size_t SS = (size_t)SX * SY, RR = (size_t)R * R;
    cudaStream_t st = ctx->stream;
    Buf b_img, b_mask, b_cand, b_cnt, b_ptr, b_done, b_lib, b_rng, b_sf, b_ns, b_rois, b_init, b_meta, b_out5, b_st,
        b_xyz, b_psi, b_dpsi, b_rows, b_nrows;
    cudaError_t e = cudaSuccess;
    auto A = [&](Buf& b, size_t bytes) { if (e == cudaSuccess) e = b.alloc(bytes); };
    A(b_img, SS * FB * 8); A(b_mask, SS * FB); A(b_cand, (size_t)FB * cap * 7 * 8); A(b_cnt, (size_t)FB * 4);
    A(b_ptr, (size_t)FB * 4); A(b_done, (size_t)FB * 4); A(b_lib, lib.size() * 8); A(b_rng, range.size() * 8);
    A(b_sf, (size_t)FB * 4); A(b_ns, 64); A(b_rois, RR * FB * 4); A(b_init, (size_t)FB * 40); A(b_meta, (size_t)FB * 32);
    A(b_out5, (size_t)FB * 40); A(b_st, (size_t)FB * 4); A(b_xyz, (size_t)FB * 24); A(b_psi, RR * FB * 8);
    A(b_dpsi, 3 * RR * FB * 8);
    const int rows_cap = FB * 64;
    A(b_rows, (size_t)rows_cap * sizeof(LocRow)); A(b_nrows, 64);
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
    V.counts = (int*)b_cnt.p; V.pointer = (int*)b_ptr.p; V.done = (int*)b_done.p;
    V.libpsf = (double*)b_lib.p; V.range = (double*)b_rng.p;
    V.slot_frame = (int*)b_sf.p; V.nslots = (int*)b_ns.p; V.rois = (float*)b_rois.p; V.init = (double*)b_init.p;
    V.meta = (double*)b_meta.p;
    std::vector<LocRow> all;
    int h_ns = 0, h_nrows = 0;
    for (int f0 = 0; f0 < nframes; f0 += FB) {
        const int nf = std::min(FB, nframes - f0);
        V.nframes = nf;
        e = cudaMemcpyAsync(b_img.p, frames + (size_t)f0 * SS, SS * nf * 8, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(b_mask.p, 0, SS * nf, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(b_ptr.p, 0, (size_t)nf * 4, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(b_done.p, 0, (size_t)nf * 4, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(b_nrows.p, 0, 4, st);
        if (e != cudaSuccess) { ctx->err = std::string("zola_localize_frames: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
        int rc = zola_detect_dev(det, (double*)b_img.p, nf, cap, (double*)b_cand.p, (int*)b_cnt.p, st);
        if (rc) return rc;
        for (int wave = 0;; ++wave) {
            if (cudaMemsetAsync(b_ns.p, 0, 4, st) != cudaSuccess) return ZOLA_E_CUDA;
            k_pipe_select<<<(nf + 127) / 128, 128, 0, st>>>(V);
            ctx->launches++;
            e = cudaMemcpyAsync(&h_ns, b_ns.p, 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) { ctx->err = std::string("zola_localize_frames: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
            if (h_ns == 0) break;
            rc = zola_fit_batch_dev(ctx, fit_psf, R, (float*)b_rois.p, (double*)b_init.p, h_ns, &fp, (double*)b_out5.p,
                                    nullptr, nullptr, (int*)b_st.p, nullptr, st);
            if (rc) return rc;
            k_take_xyz<<<(h_ns + 127) / 128, 128, 0, st>>>(h_ns, (double*)b_out5.p, (double*)b_xyz.p);
            ctx->launches++;
            rc = zola_psf_model_dev(fit_psf, R, (double*)b_xyz.p, h_ns, (double*)b_psi.p, (double*)b_dpsi.p, st);
            if (rc) return rc;
            k_pipe_finish<<<(h_ns + 127) / 128, 128, 0, st>>>(V, h_ns, (double*)b_out5.p, (int*)b_st.p,
                                                              (double*)b_psi.p, (double*)b_dpsi.p, wave,
                                                              (LocRow*)b_rows.p, (int*)b_nrows.p, rows_cap);
            ctx->launches++;
            if (cudaGetLastError() != cudaSuccess) { ctx->err = "zola_localize_frames: kernel launch failed"; return ZOLA_E_CUDA; }
        }
        e = cudaMemcpyAsync(&h_nrows, b_nrows.p, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { ctx->err = std::string("zola_localize_frames: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
        if (h_nrows > rows_cap) { ctx->err = "zola_localize_frames: more than 64 localizations per frame"; return ZOLA_E_ARG; }
        std::vector<LocRow> rows(h_nrows);
        if (h_nrows) {
            e = cudaMemcpy(rows.data(), b_rows.p, (size_t)h_nrows * sizeof(LocRow), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) { ctx->err = std::string("zola_localize_frames: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
        }
        for (auto& r : rows) r.frame += f0;
        all.insert(all.end(), rows.begin(), rows.end());
    }
    std::stable_sort(all.begin(), all.end(), [](const LocRow& a, const LocRow& b) {
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
    }
    *nout = (int)all.size();
    return ZOLA_OK;
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
