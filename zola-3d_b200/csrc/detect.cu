// PSF-library cross-correlation detection (process/cpu/Predetection.java:63-593).
//
// Per frame (S_x x S_y photons, first index x):
//   k_det_var    local mean / variance over the R-wide box by the reference's
//                running sums (Predetection.java:337-405), operation for
//                operation (no FMA contraction), on the float-rounded image
//   k_det_corr   normalised cross-correlation with the zero-mean library PSFs.
//                The reference multiplies unitary FFTs on a zero-padded M x M
//                grid (M = pow2(2S)); with that padding the product is the
//                linear correlation corr(i,j) = sum_uv img[i+u-R/2][j+v-R/2]
//                psf0[u][v], scaled by 1/sqrt(Mx My).  It is computed directly
//                in FP64 here: score = corr / sqrt(varPSF * varImage)
//                (-1 / -2 where a variance is not positive, :459-471).
//   k_det_nms    per slice r in order: tmp = max over j +- 3 where score > 0
//                (tmp keeps the previous slice's value elsewhere, as the
//                reference reuses it), then peaks with score > thr equal to
//                tmp and to the max of tmp over i +- 3, with parabolic x/y/z
//                refinement (:480-560).  Rows: score, r, i, j, topZ, topX, topY,
//                appended in the reference's insertion order (r, then j, then
//                i) by an ordered block scan, so the stored list is the same
//                on every run.
//   k_det_sort   stable sort by descending score (Arrays.sort of the rows in
//                insertion order r, j, i; :447-454): ties keep list order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "zola_internal.h"

namespace zola {



// ---------------------------------------------------------------------------
// Running sums exactly as Predetection.setImage: first along y for every x,
// then along x for every y.  Double arithmetic with explicit rounding
// intrinsics so the compiler cannot fuse multiply-adds.
__global__ void k_det_var(DetView V, const double* frames, double* rowsum, double* rowsq, double* var) {
    const int f = blockIdx.x, SX = V.SX, SY = V.SY, h = V.R / 2;
    const double* img = frames + (size_t)f * SX * SY;
    double* s1 = rowsum + (size_t)f * SX * SY;
    double* s2 = rowsq + (size_t)f * SX * SY;
    double* vr = var + (size_t)f * SX * SY;
    auto F = [&](int i, int j) { return (double)(float)img[(size_t)i * SY + j]; };
    for (int i = threadIdx.x; i < SX; i += blockDim.x) {
        double a = 0.0, b = 0.0;
        for (int t = 0; t < h + 1; ++t)
            if (t < SY) { a = __dadd_rn(a, F(i, t)); b = __dadd_rn(b, __dmul_rn(F(i, t), F(i, t))); }
        s1[(size_t)i * SY] = a;
        s2[(size_t)i * SY] = b;
        for (int ii = 1; ii < SY; ++ii) {
            double v = a, w = b;
            if (ii - h >= 0) { v = __dsub_rn(v, F(i, ii - h)); w = __dsub_rn(w, __dmul_rn(F(i, ii - h), F(i, ii - h))); }
            if (ii + h < SY) { v = __dadd_rn(v, F(i, ii + h)); w = __dadd_rn(w, __dmul_rn(F(i, ii + h), F(i, ii + h))); }
            s1[(size_t)i * SY + ii] = v;
            s2[(size_t)i * SY + ii] = w;
            a = v;
            b = w;
        }
    }
    __syncthreads();
    for (int ii = threadIdx.x; ii < SY; ii += blockDim.x) {
        double a = 0.0, b = 0.0;
        for (int t = 0; t < h + 1; ++t)
            if (t < SX) { a = __dadd_rn(a, s1[(size_t)t * SY + ii]); b = __dadd_rn(b, s2[(size_t)t * SY + ii]); }
        for (int i = 0; i < SX; ++i) {
            if (i > 0) {
                double v = a, w = b;
                if (i - h >= 0) { v = __dsub_rn(v, s1[(size_t)(i - h) * SY + ii]); w = __dsub_rn(w, s2[(size_t)(i - h) * SY + ii]); }
                if (i + h < SX) { v = __dadd_rn(v, s1[(size_t)(i + h) * SY + ii]); w = __dadd_rn(w, s2[(size_t)(i + h) * SY + ii]); }
                a = v;
                b = w;
            }
            const double n = V.norm[(size_t)i * SY + ii];
            const double mean = __ddiv_rn(a, n);
            vr[(size_t)i * SY + ii] = __dsub_rn(__ddiv_rn(b, n), __dmul_rn(mean, mean));
        }
    }
}

// ---------------------------------------------------------------------------
// Direct FP64 correlation of a 16 x 16 output tile against ZC slices.
constexpr int DT = 16;
constexpr int ZC = 8;

__global__ void __launch_bounds__(256) k_det_corr(DetView V, int zc, const double* frames, const double* var,
                                                  double* score) {
    extern __shared__ double sm[];
    const int SX = V.SX, SY = V.SY, R = V.R, Z = V.Z, h = R / 2, TW = DT + R;
    const int f = blockIdx.z;
    const int z0 = blockIdx.y * zc;
    const int tiles_y = (SY + DT - 1) / DT;
    const int i0 = (blockIdx.x / tiles_y) * DT, j0 = (blockIdx.x % tiles_y) * DT;
    double* tile = sm;               // TW x TW image with halo
    double* ps = tile + TW * TW;     // ZC x R x R
    const double* img = frames + (size_t)f * SX * SY;
    for (int k = threadIdx.x; k < TW * TW; k += blockDim.x) {
        const int a = k / TW, b = k % TW;
        const int i = i0 - h + a, j = j0 - h + b;
        tile[k] = (i >= 0 && i < SX && j >= 0 && j < SY) ? img[(size_t)i * SY + j] : 0.0;
    }
    const int nz = min(zc, Z - z0);
    for (int k = threadIdx.x; k < nz * R * R; k += blockDim.x) ps[k] = V.psf0[(size_t)z0 * R * R + k];
    __syncthreads();
    const int ti = threadIdx.x / DT, tj = threadIdx.x % DT;
    const int i = i0 + ti, j = j0 + tj;
    double acc[ZC];
#pragma unroll
    for (int q = 0; q < ZC; ++q) acc[q] = 0.0;
    for (int u = 0; u < R; ++u) {
        const double* trow = tile + (ti + u) * TW + tj;
        for (int v = 0; v < R; ++v) {
            const double x = trow[v];
#pragma unroll
            for (int q = 0; q < ZC; ++q)
                if (q < nz) acc[q] = fma(x, ps[(q * R + u) * R + v], acc[q]);
        }
    }
    if (i >= SX || j >= SY) return;
    const double vi = var[(size_t)f * SX * SY + (size_t)i * SY + j];
    for (int q = 0; q < nz; ++q) {
        const int r = z0 + q;
        const double vp = V.varpsf[r];
        const double s = sqrt(vp * vi);
        double o;
        if (s > 0) o = (acc[q] * V.inv_m) / s;
        else if (vp <= 0) o = -1.0;
        else o = -2.0;
        score[(((size_t)f * Z + r) * SX + i) * SY + j] = o;
    }
}

// ---------------------------------------------------------------------------
// Register-tiled form of the same correlation (same terms, same order per
// output: u outer, v inner, one FMA each), bound by the FP64 FMA pipe instead
// of shared-memory loads.  A CTA of 256 threads covers a 32 x 64 output tile
// and RZC slices; each thread owns 8 consecutive outputs of one row for every
// slice (32 accumulators).  For each kernel row u a thread keeps an 8-wide
// window of the image row in registers and slides it along v, so one image
// load and RZC broadcast library loads feed 8 RZC FMAs.  A half-warp holds
// 16 consecutive rows of one 8-column group; with an odd row stride their
// window loads fall in 16 different bank pairs.
constexpr int RTI = 32, RTJ = 64, RPX = 8, RZC = 4;

__host__ __device__ inline int rt_stride(int R) { return (RTJ + R) | 1; }
__host__ __device__ inline size_t rt_smem(int R, int zc) {
    return (size_t)(RTI + R) * rt_stride(R) * 8 + (size_t)zc * R * R * 8;
}

__global__ void __launch_bounds__(256, 2) k_det_corr_rt(DetView V, int zc, const double* frames, const double* var,
                                                         double* score) {
    extern __shared__ double sm[];
    const int SX = V.SX, SY = V.SY, R = V.R, Z = V.Z, h = R / 2, TS = rt_stride(R), TH = RTI + R;
    const int f = blockIdx.z, z0 = blockIdx.y * zc;
    const int tiles_j = (SY + RTJ - 1) / RTJ;
    const int i0 = (blockIdx.x / tiles_j) * RTI, j0 = (blockIdx.x % tiles_j) * RTJ;
    double* tile = sm;                    // (RTI + R) rows x TS (RTJ + R used, zero-filled)
    double* ps = tile + (size_t)TH * TS;  // zc x R x R
    const double* img = frames + (size_t)f * SX * SY;
    const int TW = RTJ + R;  // the last window load (v = R - 1) reads column RTJ + R - 1
    for (int k = threadIdx.x; k < TH * TW; k += blockDim.x) {
        const int a = k / TW, b = k - a * TW;
        const int i = i0 - h + a, j = j0 - h + b;
        tile[a * TS + b] = (i >= 0 && i < SX && j >= 0 && j < SY) ? img[(size_t)i * SY + j] : 0.0;
    }
    const int nz = min(zc, Z - z0);
    for (int k = threadIdx.x; k < nz * R * R; k += blockDim.x) ps[k] = V.psf0[(size_t)z0 * R * R + k];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ti = (lane & 15) + 16 * (warp & 1), tj = 8 * (2 * (warp >> 1) + (lane >> 4));
    double acc[RZC][RPX];
#pragma unroll
    for (int q = 0; q < RZC; ++q)
#pragma unroll
        for (int k = 0; k < RPX; ++k) acc[q][k] = 0.0;
    const int RR = R * R;
    for (int u = 0; u < R; ++u) {
        const double* trow = tile + (ti + u) * TS + tj;
        const double* prow = ps + u * R;
        double w[RPX];
#pragma unroll
        for (int k = 0; k < RPX; ++k) w[k] = trow[k];
        // unrolled by the window width: the window's shifts become register renames
#pragma unroll 8
        for (int v = 0; v < R; ++v) {
            double p[RZC];
#pragma unroll
            for (int q = 0; q < RZC; ++q) p[q] = q < nz ? prow[q * RR + v] : 0.0;
#pragma unroll
            for (int q = 0; q < RZC; ++q)
#pragma unroll
                for (int k = 0; k < RPX; ++k) acc[q][k] = fma(w[k], p[q], acc[q][k]);
#pragma unroll
            for (int k = 0; k < RPX - 1; ++k) w[k] = w[k + 1];
            w[RPX - 1] = trow[v + RPX];
        }
    }
    const int i = i0 + ti;
    if (i >= SX) return;
    for (int k = 0; k < RPX; ++k) {
        const int j = j0 + tj + k;
        if (j >= SY) break;
        const double vi = var[(size_t)f * SX * SY + (size_t)i * SY + j];
#pragma unroll
        for (int q = 0; q < RZC; ++q) {
            if (q >= nz) break;
            const int r = z0 + q;
            const double vp = V.varpsf[r];
            const double s = sqrt(vp * vi);
            double o;
            if (s > 0) o = (acc[q][k] * V.inv_m) / s;
            else if (vp <= 0) o = -1.0;
            else o = -2.0;
            score[(((size_t)f * Z + r) * SX + i) * SY + j] = o;
        }
    }
}

// ---------------------------------------------------------------------------
// Camera counts to photons as LocalizationPipeline.java:601-605 does it:
// value * (adu / gain) + (-offset * adu / gain), a product then a sum (Java
// does not contract them), negative results set to 0.
__global__ void k_u16_photons(const uint16_t* in, size_t n, double slope, double intercept, double* out) {
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const double v = __dadd_rn(__dmul_rn((double)in[k], slope), intercept);
        out[k] = v < 0 ? 0.0 : v;
    }
}

void rescale_u16(zola_ctx* ctx, const uint16_t* d_in, size_t n, const double* rescale, double* d_out,
                 cudaStream_t st) {
    k_u16_photons<<<ctx->num_sms * 8, 256, 0, st>>>(d_in, n, rescale[0], rescale[1], d_out);
    ctx->launches++;
}

void camera_rescale(double adu, double gain, double offset, double* rescale) {
    rescale[0] = adu / gain;            // rescale_slope (LocalizationPipeline.java:103)
    rescale[1] = -offset * adu / gain;  // rescale_intercept (:104)
}

// ---------------------------------------------------------------------------
__device__ inline double parabola_top(double xa, double ya, double xb, double yb, double xc, double yc) {
    const double a = (yc - ya) / ((xc - xa) * (xc - xb)) - (yb - ya) / ((xb - xa) * (xc - xb));
    const double b = ((yb - ya) / (xb - xa)) - a * (xb + xa);
    return -b / (2 * a);
}

// Exclusive prefix sum of one int per thread over the block, in thread order;
// *total = the block's sum.  wtot: 32 ints of shared memory.
__device__ int block_exclusive_scan(int v, int* wtot, int* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wtot[w] = x;
    __syncthreads();
    if (w == 0) {
        int y = lane < nw ? wtot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += u;
        }
        if (lane < nw) wtot[lane] = y;
    }
    __syncthreads();
    const int base = w ? wtot[w - 1] : 0;
    *total = wtot[nw - 1];
    __syncthreads();  // wtot is reused by the next call
    return base + x - v;
}

// One CTA per frame; slices in order because tmp carries over between them.
// flags: SX x SY bytes per frame of scratch (the peaks of the current slice).
// The first V.cap rows of the frame's list (in insertion order) are stored;
// counts[f] = the length of the whole list.
__global__ void __launch_bounds__(1024) k_det_nms(DetView V, const double* score, double* tmp, unsigned char* flags,
                                                  double* cand, int* counts) {
    const int f = blockIdx.x, SX = V.SX, SY = V.SY, Z = V.Z, dec = 3;
    const int lo = max(dec, V.R / 2);
    const double* sc = score + (size_t)f * Z * SX * SY;
    double* tm = tmp + (size_t)f * SX * SY;
    unsigned char* fl = flags + (size_t)f * SX * SY;
    double* out = cand + (size_t)f * V.cap * 7;
    __shared__ int wtot[32];
    for (int k = threadIdx.x; k < SX * SY; k += blockDim.x) tm[k] = 0.0;
    __syncthreads();
    auto S = [&](int r, int i, int j) { return sc[((size_t)r * SX + i) * SY + j]; };
    int total = 0;
    for (int r = 0; r < Z; ++r) {
        for (int k = threadIdx.x; k < SX * SY; k += blockDim.x) {
            const int i = k / SY, j = k % SY;
            if (i < lo || i >= SX - lo || j < lo || j >= SY - lo) continue;
            if (S(r, i, j) > 0) {
                double t = -INFINITY;
                for (int a = -dec; a <= dec; ++a) t = fmax(S(r, i, j + a), t);
                tm[k] = t;
            }
        }
        __syncthreads();
        for (int k = threadIdx.x; k < SX * SY; k += blockDim.x) {
            const int i = k / SY, j = k % SY;
            unsigned char peak = 0;
            if (i >= lo && i < SX - lo && j >= lo && j < SY - lo) {
                const double v = S(r, i, j);
                if (v > V.thr && v == tm[k]) {
                    double mx = -INFINITY;
                    for (int a = -dec; a <= dec; ++a) mx = fmax(tm[(size_t)(i + a) * SY + j], mx);
                    peak = mx == v;
                }
            }
            fl[k] = peak;
        }
        __syncthreads();
        // append the slice's peaks column by column (thread = column j), rows i in order
        for (int j0 = lo; j0 < SY - lo; j0 += blockDim.x) {
            const int j = j0 + threadIdx.x;
            const bool col = j < SY - lo;
            int c = 0;
            if (col)
                for (int i = lo; i < SX - lo; ++i) c += fl[(size_t)i * SY + j];
            int tot;
            int o = total + block_exclusive_scan(c, wtot, &tot);
            if (col && c)
                for (int i = lo; i < SX - lo; ++i) {
                    if (!fl[(size_t)i * SY + j]) continue;
                    if (o < V.cap) {
                        const double v = S(r, i, j);
                        double tz = 0, tx = 0, ty = 0;
                        if (r > 1 && r < Z - 1) tz = parabola_top(-V.zstep, S(r - 1, i, j), 0, v, V.zstep, S(r + 1, i, j));
                        if (i > 1 && i < SX - 1) tx = parabola_top(-V.dx, S(r, i - 1, j), 0, v, V.dx, S(r, i + 1, j));
                        if (j > 1 && j < SY - 1) ty = parabola_top(-V.dx, S(r, i, j - 1), 0, v, V.dx, S(r, i, j + 1));
                        double* row = out + (size_t)o * 7;
                        row[0] = v; row[1] = r; row[2] = i; row[3] = j; row[4] = tz; row[5] = tx; row[6] = ty;
                    }
                    ++o;
                }
            total += tot;
        }
        __syncthreads();  // tm and the flags change with the next slice
    }
    if (threadIdx.x == 0) counts[f] = total;
}

// Sort keys of up to DET_SORT_SMEM candidates per frame live in shared memory;
// longer lists sort in global scratch (same network).
constexpr int DET_SORT_SMEM = 16384;

__host__ __device__ inline int det_pow2(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

// Sort one frame's stored candidates by (score descending, list position
// ascending) -- a stable sort of the insertion-ordered list -- and write the
// first min(n, cap) rows.  gs / gid: global sort keys (det_pow2(cap) per
// frame) or nullptr for the shared-memory form.
__global__ void __launch_bounds__(1024) k_det_sort(DetView V, const double* cand, const int* counts, double* out,
                                                   double* gs, int* gid) {
    extern __shared__ double smraw[];
    const int f = blockIdx.x, n = min(counts[f], V.cap);
    const int P2 = det_pow2(n);
    double* s = gs ? gs + (size_t)f * det_pow2(V.cap) : smraw;
    int* id = gs ? gid + (size_t)f * det_pow2(V.cap) : (int*)(smraw + P2);
    const double* c = cand + (size_t)f * V.cap * 7;
    for (int t = threadIdx.x; t < P2; t += blockDim.x) {
        if (t < n) { s[t] = c[(size_t)t * 7]; id[t] = t; }
        else { s[t] = -INFINITY; id[t] = 0x7fffffff; }
    }
    __syncthreads();
    // bitonic network: "before" = higher score, then earlier in the list
    for (int size = 2; size <= P2; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < P2; t += blockDim.x) {
                const int o = t ^ stride;
                if (o > t) {
                    const bool up = (t & size) == 0;
                    const bool t_before = s[t] > s[o] || (s[t] == s[o] && id[t] < id[o]);
                    if (up != t_before) {
                        const double ts = s[t]; s[t] = s[o]; s[o] = ts;
                        const int ti = id[t]; id[t] = id[o]; id[o] = ti;
                    }
                }
            }
            __syncthreads();
        }
    double* dst = out + (size_t)f * V.cap * 7;
    for (int t = threadIdx.x; t < n * 7; t += blockDim.x) {
        const int row = t / 7, col = t % 7;
        dst[t] = c[(size_t)id[row] * 7 + col];
    }
}

}  // namespace zola

// ------------------------------------------------------------------ host ----

using namespace zola;

extern "C" {

int zola_detector_create(zola_psf* psf, int SX, int SY, int R, double minZ, double maxZ, double step, double thr,
                         zola_detector** out) {
    if (!psf || !out) return ZOLA_E_ARG;
    zola_ctx* ctx = psf->ctx;
    *out = nullptr;
    if (SX < 8 || SY < 8 || SX > 4096 || SY > 4096 || R < 4 || R % 2 || R > SX || R > SY || R > 96 || !(step > 0) ||
        !(maxZ > minZ)) {
        ctx->err = "zola_detector_create: need 8 <= S <= 4096, even R <= min(S, 96), step > 0, maxZ > minZ";
        return ZOLA_E_ARG;
    }
    int number = (int)std::ceil((maxZ - minZ) / step);  // Predetection.java:120-127
    if (number < 1 || number > 4096) { ctx->err = "zola_detector_create: bad number of library slices"; return ZOLA_E_ARG; }
    zola_detector* d = new zola_detector();
    d->psf = psf;
    double z = minZ;
    for (int i = 0; i < number; ++i) { d->range.push_back(z); z += step; }
    // library PSFs with the FP64 model: x = y = 0, zoil = Zfocus, zwat = range[i]
    std::vector<double> xyz(3 * (size_t)number);
    for (int i = 0; i < number; ++i) { xyz[3 * i] = 0; xyz[3 * i + 1] = 0; xyz[3 * i + 2] = d->range[i]; }
    d->h_psf.resize((size_t)number * R * R);
    int rc = zola_psf_model(psf, R, xyz.data(), number, d->h_psf.data(), nullptr);
    if (rc) { delete d; return rc; }
    std::vector<double> psf0((size_t)number * R * R), varpsf(number), norm((size_t)SX * SY);
    for (int i = 0; i < number; ++i) {  // Predetection.java:178-204
        const double* p = d->h_psf.data() + (size_t)i * R * R;
        double mean = 0;
        for (int k = 0; k < R * R; ++k) mean += p[k];
        mean /= (double)R * R;
        double v = 0;
        for (int k = 0; k < R * R; ++k) {
            double q = p[k] - mean;
            psf0[(size_t)i * R * R + k] = q;
            v += q * q;
        }
        varpsf[i] = v / (double)(R * R);
    }
    for (int i = 0; i < SX; ++i)  // Predetection.java:95-116 (index rules kept)
        for (int ii = 0; ii < SY; ++ii) {
            int vx1 = R / 2, vx2 = R / 2, vy1 = R / 2, vy2 = R / 2;
            if (i < R / 2 - 1) vx1 = i + 1;
            if (i > SX - R / 2 - 2) vx2 = SY - i - 1;
            if (ii < R / 2 - 1) vy1 = ii + 1;
            if (ii > SX - R / 2 - 2) vy2 = SY - ii - 2;
            norm[(size_t)i * SY + ii] = (double)((vx1 + vx2) * (vy1 + vy2));
        }
    size_t total = psf0.size() + varpsf.size() + norm.size();
    cudaError_t e = cudaMalloc(&d->d_lib, total * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(d->d_lib, psf0.data(), psf0.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d->d_lib + psf0.size(), varpsf.data(), varpsf.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d->d_lib + psf0.size() + varpsf.size(), norm.data(), norm.size() * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        ctx->err = std::string("zola_detector_create: ") + cudaGetErrorString(e);
        if (d->d_lib) cudaFree(d->d_lib);
        delete d;
        return ZOLA_E_CUDA;
    }
    int MX = 1, MY = 1;
    while (MX < 2 * SX) MX <<= 1;
    while (MY < 2 * SY) MY <<= 1;
    DetView& v = d->v;
    v.SX = SX; v.SY = SY; v.R = R; v.Z = number; v.cap = 0;
    v.inv_m = 1.0 / std::sqrt((double)MX * (double)MY);
    v.thr = thr; v.zstep = step; v.dx = psf->o.xystep;
    v.psf0 = d->d_lib; v.varpsf = d->d_lib + psf0.size(); v.norm = d->d_lib + psf0.size() + varpsf.size();
    *out = d;
    return ZOLA_OK;
}

int zola_detector_free(zola_detector* d) {
    if (!d) return ZOLA_E_ARG;
    cudaStreamSynchronize(d->psf->ctx->stream);
    cudaFree(d->d_lib);
    delete d;
    return ZOLA_OK;
}

int zola_detector_info(const zola_detector* d, int* nslices, double* range, double* psfs) {
    if (!d || !nslices) return ZOLA_E_ARG;
    *nslices = d->v.Z;
    if (range)
        for (int i = 0; i < d->v.Z; ++i) range[i] = d->range[i];
    if (psfs)
        for (size_t k = 0; k < d->h_psf.size(); ++k) psfs[k] = d->h_psf[k];
    return ZOLA_OK;
}

int zola_detect_dev(zola_detector* d, const double* d_frames, int nframes, int cap, double* d_out, int* d_counts,
                    void* stream) {
    if (!d) return ZOLA_E_ARG;
    zola_ctx* ctx = d->psf->ctx;
    if (nframes < 0 || cap < 1 || cap > ZOLA_DETECT_MAX_CAP || (nframes > 0 && (!d_frames || !d_out || !d_counts))) {
        ctx->err = "zola_detect: bad nframes / cap (1..2^20) or null buffer";
        return ZOLA_E_ARG;
    }
    if (nframes == 0) return ZOLA_OK;
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    DetView v = d->v;
    v.cap = cap;
    const size_t SS = (size_t)v.SX * v.SY;
    const int p2 = det_pow2(cap);
    const bool gsort = p2 > DET_SORT_SMEM;
    // scratch per frame: rowsum (later the peak flags), rowsq, var, tmp, scores (Z x SS),
    // candidates, and the sort keys when they do not fit in shared memory
    const size_t per = (4 + (size_t)v.Z) * SS * 8 + (size_t)cap * 7 * 8 + (gsort ? (size_t)p2 * 12 : 0);
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)nframes, ((size_t)1 << 31) / per));
    if (ensure_scratch(ctx, per * chunk + 1024, ctx->err)) return ZOLA_E_CUDA;
    for (int f0 = 0; f0 < nframes; f0 += chunk) {
        const int nf = std::min(chunk, nframes - f0);
        char* b = (char*)ctx->scratch;
        double* rowsum = (double*)b; b += nf * SS * 8;
        double* rowsq = (double*)b; b += nf * SS * 8;
        double* var = (double*)b; b += nf * SS * 8;
        double* tmp = (double*)b; b += nf * SS * 8;
        double* score = (double*)b; b += nf * v.Z * SS * 8;
        double* cand = (double*)b; b += (size_t)nf * cap * 7 * 8;
        double* gs = gsort ? (double*)b : nullptr;
        int* gid = gsort ? (int*)(gs + (size_t)nf * p2) : nullptr;
        const double* fr = d_frames + (size_t)f0 * SS;
        prof_begin(ctx, 9, st);
        k_det_var<<<nf, 256, 0, st>>>(v, fr, rowsum, rowsq, var);
        // slices per register-tiled CTA: as many (up to RZC) as keep two CTAs per SM
        int zrt = RZC;
        while (zrt > 0 && rt_smem(v.R, zrt) > 112 * 1024) --zrt;
        if (zrt > 0) {
            const int tiles = ((v.SX + RTI - 1) / RTI) * ((v.SY + RTJ - 1) / RTJ);
            const size_t smem = rt_smem(v.R, zrt);
            cudaFuncSetAttribute(k_det_corr_rt, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            dim3 grid(tiles, (v.Z + zrt - 1) / zrt, nf);
            k_det_corr_rt<<<grid, 256, smem, st>>>(v, zrt, fr, var, score);
        } else {
            const int tiles = ((v.SX + DT - 1) / DT) * ((v.SY + DT - 1) / DT);
            const size_t tile_b = (size_t)(DT + v.R) * (DT + v.R) * 8, slice_b = (size_t)v.R * v.R * 8;
            const int zc = (int)std::max<size_t>(1, std::min<size_t>(ZC, (200 * 1024 - tile_b) / slice_b));
            const size_t smem = tile_b + (size_t)zc * slice_b;
            cudaFuncSetAttribute(k_det_corr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            dim3 grid(tiles, (v.Z + zc - 1) / zc, nf);
            k_det_corr<<<grid, 256, smem, st>>>(v, zc, fr, var, score);
        }
        // the row sums are dead after k_det_var: their space holds the peak flags
        k_det_nms<<<nf, 1024, 0, st>>>(v, score, tmp, (unsigned char*)rowsum, cand, d_counts + f0);
        const size_t ssort = gsort ? 0 : (size_t)p2 * 12;
        cudaFuncSetAttribute(k_det_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ssort);
        k_det_sort<<<nf, 1024, ssort, st>>>(v, cand, d_counts + f0, d_out + (size_t)f0 * cap * 7, gs, gid);
        prof_end(ctx, st);
        ctx->launches += 4;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { ctx->err = std::string("zola_detect: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
    }
    return ZOLA_OK;
}

}  // extern "C"

namespace {

// frames (photons) or u16 camera counts with rescale = {slope, intercept}
int detect_impl(zola_detector* d, const double* frames, const uint16_t* u16, const double* rescale, int nframes,
                int cap, double* out, int* counts) {
    if (!d) return ZOLA_E_ARG;
    zola_ctx* ctx = d->psf->ctx;
    if (nframes < 0 || cap < 1 || cap > ZOLA_DETECT_MAX_CAP ||
        (nframes > 0 && ((!frames && !u16) || !out || !counts))) {
        ctx->err = "zola_detect: bad nframes / cap (1..2^20) or null buffer";
        return ZOLA_E_ARG;
    }
    if (nframes == 0) return ZOLA_OK;
    const size_t SS = (size_t)d->v.SX * d->v.SY;
    // Candidates stored per frame in the first pass: at least DETECT_ROOM, so that the
    // usual lists (a few thousand at the reference's threshold) are whole and sorted
    // in one pass whatever cap the caller asks for.
    constexpr int DETECT_ROOM = 8192;
    const int room0 = std::max(cap, DETECT_ROOM);
    // frames, counts, the uint16 frames and the candidate rows come from the
    // context's grow-only staging area, so repeated calls allocate nothing
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t b_df = al(SS * nframes * 8), b_dc = al((size_t)nframes * 4), b_du = u16 ? al(SS * nframes * 2) : 0;
    if (ensure_io(ctx, b_df + b_dc + b_du + al((size_t)nframes * room0 * 7 * 8))) return ZOLA_E_CUDA;
    char* io = (char*)ctx->io;
    double* df = (double*)io;
    int* dc = (int*)(io + b_df);
    uint16_t* du = u16 ? (uint16_t*)(io + b_df + b_dc) : nullptr;
    double* dout = (double*)(io + b_df + b_dc + b_du);
    cudaError_t e = cudaSuccess;
    if (u16) {
        e = cudaMemcpyAsync(du, u16, SS * nframes * 2, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) rescale_u16(ctx, du, SS * nframes, rescale, df, ctx->stream);
    } else {
        e = cudaMemcpyAsync(df, frames, SS * nframes * 8, cudaMemcpyHostToDevice, ctx->stream);
    }
    int rc = e == cudaSuccess ? zola_detect_dev(d, df, nframes, room0, dout, dc, ctx->stream) : ZOLA_OK;
    if (e == cudaSuccess && rc == ZOLA_OK) {
        e = cudaMemcpyAsync(counts, dc, (size_t)nframes * 4, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    // A frame whose list is longer than the room kept the first candidates in scan
    // order, not the best: such frames are gathered and detected again with room
    // for their whole lists, and the first cap rows of each replace theirs.
    std::vector<int> longf;
    int room = room0;
    if (e == cudaSuccess && rc == ZOLA_OK)
        for (int f = 0; f < nframes; ++f)
            if (counts[f] > room0) {
                longf.push_back(f);
                room = std::max(room, counts[f]);
            }
    double* g = nullptr;  // gathered frames, their rows, their counts (rare: one allocation)
    if (!longf.empty() && room > ZOLA_DETECT_MAX_CAP) {
        ctx->err = "zola_detect: a frame has more than 2^20 candidates";
        rc = ZOLA_E_ARG;
    } else if (!longf.empty()) {
        const size_t nl = longf.size();
        e = cudaMalloc(&g, nl * SS * 8 + nl * (size_t)room * 7 * 8 + nl * 4);
        double* g_out = g + nl * SS;
        int* g_cnt = (int*)(g_out + nl * (size_t)room * 7);
        for (size_t k = 0; k < nl && e == cudaSuccess; ++k)
            e = cudaMemcpyAsync(g + k * SS, df + (size_t)longf[k] * SS, SS * 8, cudaMemcpyDeviceToDevice, ctx->stream);
        if (e == cudaSuccess) rc = zola_detect_dev(d, g, (int)nl, room, g_out, g_cnt, ctx->stream);
        for (size_t k = 0; k < nl && e == cudaSuccess && rc == ZOLA_OK; ++k)
            e = cudaMemcpyAsync(dout + (size_t)longf[k] * room0 * 7, g_out + k * room * 7, (size_t)cap * 7 * 8,
                                cudaMemcpyDeviceToDevice, ctx->stream);
    }
    if (e == cudaSuccess && rc == ZOLA_OK) {
        e = cudaMemcpy2DAsync(out, (size_t)cap * 7 * 8, dout, (size_t)room0 * 7 * 8, (size_t)cap * 7 * 8, nframes,
                              cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
    if (g) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(g);
    }
    if (e != cudaSuccess) { ctx->err = std::string("zola_detect: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
    return rc;
}

}  // namespace

extern "C" {

int zola_detect(zola_detector* d, const double* frames, int nframes, int cap, double* out, int* counts) {
    return detect_impl(d, frames, nullptr, nullptr, nframes, cap, out, counts);
}

int zola_detect_u16(zola_detector* d, const uint16_t* frames, int nframes, int cap, double adu, double gain,
                    double offset, double* out, int* counts) {
    if (!d) return ZOLA_E_ARG;
    if (!(gain != 0) || !std::isfinite(adu) || !std::isfinite(gain) || !std::isfinite(offset)) {
        d->psf->ctx->err = "zola_detect_u16: adu, gain, offset must be finite and gain non-zero";
        return ZOLA_E_ARG;
    }
    double rescale[2];
    camera_rescale(adu, gain, offset, rescale);
    return detect_impl(d, nullptr, frames, rescale, nframes, cap, out, counts);
}

}  // extern "C"
