// Zernike PSF calibration from bead z-stacks: FP64 forward model, hand-written
// adjoint (reverse mode), forward-mode tangents, a Gauss-Newton matrix built on
// the device, and an FP64 Levenberg-Marquardt driver.
//
// Model (process/cpu/ZernikePhaseRetrieval.java:1843-1874, background
// :1519-1530): for bead b and slice s, the PSF psi at (x_b, y_b,
// zoil = dz_s + z_b, zwat = 0) with phase sum_i a_i Z_i over modes i >= 3
// (modes 0-2 are the per-bead registration, :93-95, carried here as x_b, y_b,
// z_b) and blur width sigma;
//   mu = psi (A0_bs + a_bs) + sum_k c_bk m_k(i, ii),  m = 1, i, i^2, ii, i ii, ii^2
// (A0 from InitBackgroundAndPhotonNumber, the reference's fit_a + fit_a_each
// folded into a_bs, PolynomialBackground of order 2); mu <= 0 is replaced by
// 1e-8 (:1862-1864) and contributes no gradient; NLL = sum mu - d ln mu.
// The reference updates one parameter at a time by finite-difference Newton
// steps (:225-300, 860-1050, 1081-1198).  Here the gradient of the whole stack
// NLL comes from one adjoint pass per slice:
//   w = 1 - d/mu;  g_psi = At w;  g_m = (g_psi - sum g_psi psi) / S;  g_T = sgn(T) g_m
//   dNLL/dsigma = <g_T, dG I G^T + G I dG^T>
//   g_I = G^T g_T G;  Ebar = g_I o E;  Qbar = C^H Ebar conj(C)
//   g_phi = 2 Im(conj(Q) Qbar)   (per pupil pixel)
//   dNLL/da_i = sum g_phi Z_i,  dNLL/dx_b = sum g_phi kx,  dNLL/dy_b = sum g_phi ky,
//   dNLL/dz_b = -sum g_phi kzoil,  dNLL/da_bs = sum w psi,  dNLL/dc_bk = sum w m_k.
// Tangents (for the Gauss-Newton matrix) push a phase direction dphi through
// dQ = i Q dphi, dE = C dQ C^T, dI = 2 Re(conj E dE), dT = G dI G^T (or
// dT = dG I G^T + G I dG^T for sigma), dpsi = (sgn T dT - psi sum sgn T dT) / S.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "zola_internal.h"

namespace zola {

constexpr int CAL_THREADS = 256;
constexpr int NPOLY = 6;
constexpr int NOUT = 3 + NPOLY;  // per slice: nll, d/da_bs, d/dsigma, d/dc_k
constexpr int CAL_GRID = 1184;   // persistent CTAs (8 per SM), each with its own work area

__host__ __device__ inline double poly_m(int k, int i, int ii) {
    switch (k) {
        case 0: return 1.0;
        case 1: return (double)i;
        case 2: return (double)i * i;
        case 3: return (double)ii;
        case 4: return (double)i * ii;
        default: return (double)ii * ii;
    }
}

struct CalView {
    int D, W, R, nb, ns, pb;    // pb = per-bead stride 3 + ns + NPOLY
    const double* pupil;        // D x D
    const double* kx;           // D
    const double* ky;           // D
    const double* kzoil;        // D x D
    const double2* C;           // W x D
    const double* G;            // R x W at the current sigma
    const double* dG;           // R x W, d G / d sigma
    const double* dz;           // ns
    const double* stacks;       // nb x ns x R x R
    const double* A0;           // nb x ns (nullptr: 0)
};

struct CalWork {
    double2* Q;   // D x D
    double2* S;   // D x W  (also X = C^H Ebar)
    double2* E;   // W x W  (also Ebar)
    double* I;    // W x W  (also g_I)
    double* J;    // R x W
    double* dJ;   // R x W
    double* T;    // R x R
    double* aux;  // R x R
};

__host__ __device__ inline size_t cal_work_bytes(int D, int W, int R) {
    auto al = [](size_t v) { return (v + 255) / 256 * 256; };
    return al((size_t)D * D * 16) + al((size_t)D * W * 16) + al((size_t)W * W * 16) + al((size_t)W * W * 8) +
           al((size_t)R * W * 8) * 2 + al((size_t)R * R * 8) * 2;
}

__device__ inline CalWork cal_carve(char* base, int D, int W, int R) {
    auto al = [](size_t v) { return (v + 255) / 256 * 256; };
    CalWork w;
    size_t o = 0;
    w.Q = (double2*)(base + o); o += al((size_t)D * D * 16);
    w.S = (double2*)(base + o); o += al((size_t)D * W * 16);
    w.E = (double2*)(base + o); o += al((size_t)W * W * 16);
    w.I = (double*)(base + o); o += al((size_t)W * W * 8);
    w.J = (double*)(base + o); o += al((size_t)R * W * 8);
    w.dJ = (double*)(base + o); o += al((size_t)R * W * 8);
    w.T = (double*)(base + o); o += al((size_t)R * R * 8);
    w.aux = (double*)(base + o);
    return w;
}

__device__ inline double block_reduce(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    __syncthreads();
    return s;
}

// Q = pupil exp(i (phase + kx x + ky y - kzoil zoil)) on the disk square.
__device__ void cal_pupil(const CalView& V, const CalWork& w, const double* phase, double x, double y, double zoil) {
    const int D = V.D;
    for (int k = threadIdx.x; k < D * D; k += blockDim.x) {
        const int a = k / D, b = k % D;
        const double p = V.pupil[k];
        double2 q = make_double2(0, 0);
        if (p != 0) {
            double s, c;
            sincos(phase[k] + V.kx[a] * x + V.ky[b] * y - V.kzoil[k] * zoil, &s, &c);
            q = make_double2(p * c, p * s);
        }
        w.Q[k] = q;
    }
    __syncthreads();
}

// E = C X C^T from a pupil field X (D x D); S scratch (D x W).
__device__ void cal_dft(const CalView& V, const double2* X, double2* S, double2* E) {
    const int D = V.D, W = V.W;
    for (int k = threadIdx.x; k < D * W; k += blockDim.x) {
        const int a = k / W, j = k % W;
        double2 s = make_double2(0, 0);
        for (int b = 0; b < D; ++b) {
            const double2 q = X[a * D + b], c = V.C[j * D + b];
            s.x += q.x * c.x - q.y * c.y;
            s.y += q.x * c.y + q.y * c.x;
        }
        S[k] = s;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < W * W; k += blockDim.x) {
        const int i = k / W, j = k % W;
        double2 e = make_double2(0, 0);
        for (int a = 0; a < D; ++a) {
            const double2 c = V.C[i * D + a], s = S[a * W + j];
            e.x += c.x * s.x - c.y * s.y;
            e.y += c.x * s.y + c.y * s.x;
        }
        E[k] = e;
    }
    __syncthreads();
}

// out (R x W) = M (R x W) applied to the W x W matrix I along its first index.
__device__ void cal_rows(const CalView& V, const double* M, const double* I, double* out) {
    const int W = V.W, R = V.R;
    for (int k = threadIdx.x; k < R * W; k += blockDim.x) {
        const int ip = k / W, j = k % W;
        double acc = 0;
        for (int i = 0; i < W; ++i) acc += M[ip * W + i] * I[i * W + j];
        out[k] = acc;
    }
    __syncthreads();
}

// Forward model of one slice into w (J = G I, T = J G^T); returns S = sum |T|.
__device__ double cal_forward(const CalView& V, const CalWork& w, const double* phase, double x, double y, double zoil,
                              double* red) {
    cal_pupil(V, w, phase, x, y, zoil);
    cal_dft(V, w.Q, w.S, w.E);
    const int W = V.W, R = V.R;
    for (int k = threadIdx.x; k < W * W; k += blockDim.x) w.I[k] = w.E[k].x * w.E[k].x + w.E[k].y * w.E[k].y;
    __syncthreads();
    cal_rows(V, V.G, w.I, w.J);
    double s = 0;
    for (int k = threadIdx.x; k < R * R; k += blockDim.x) {
        const int ip = k / R, jp = k % R;
        double acc = 0;
        for (int j = 0; j < W; ++j) acc += V.G[jp * W + j] * w.J[ip * W + j];
        w.T[k] = acc;
        s += fabs(acc);
    }
    return block_reduce(s, red);
}

// Entry k of dT = dG I G^T + G I dG^T, from J = G I and dJ = dG I.
__device__ inline double cal_dT_sigma(const CalView& V, const CalWork& w, int k) {
    const int W = V.W, R = V.R, ip = k / R, jp = k % R;
    double acc = 0;
    for (int j = 0; j < W; ++j) acc += w.dJ[ip * W + j] * V.G[jp * W + j] + w.J[ip * W + j] * V.dG[jp * W + j];
    return acc;
}

// mode 0: NLL (+ model, psi), mode 1: NLL + adjoint.  Items are (bead, slice).
// out_slice: per slice NOUT values; gphi: per slice D x D phase gradient.
__global__ void __launch_bounds__(CAL_THREADS) k_calib(CalView V, const double* phase, const double* bead, int mode,
                                                        char* scratch, size_t per_cta, double* out_slice,
                                                        double* gphi, double* model, double* psi_out) {
    __shared__ double red[CAL_THREADS / 32];
    const int D = V.D, W = V.W, R = V.R, RR = R * R;
    CalWork w = cal_carve(scratch + (size_t)blockIdx.x * per_cta, D, W, R);
    for (int bs = blockIdx.x; bs < V.nb * V.ns; bs += gridDim.x) {
        const int b = bs / V.ns, s = bs % V.ns;
        const double* th = bead + (size_t)b * V.pb;
        const double x = th[0], y = th[1], z = th[2];
        const double At = (V.A0 ? V.A0[bs] : 0.0) + th[3 + s];
        const double* c = th + 3 + V.ns;
        const double Ssum = cal_forward(V, w, phase, x, y, V.dz[s] + z, red);
        const double* d = V.stacks + (size_t)bs * RR;
        double acc[NOUT + 1];  // nll, d/da, (sigma later), d/dc[6], sum g_psi psi
#pragma unroll
        for (int q = 0; q < NOUT + 1; ++q) acc[q] = 0.0;
        for (int k = threadIdx.x; k < RR; k += blockDim.x) {
            const int i = k / R, ii = k % R;
            const double psi = fabs(w.T[k]) / Ssum;
            double bg = 0;
#pragma unroll
            for (int q = 0; q < NPOLY; ++q) bg += c[q] * poly_m(q, i, ii);
            const double mu_raw = psi * At + bg;
            const bool clamped = mu_raw <= 0;
            const double mu = clamped ? 0.00000001 : mu_raw;
            acc[0] += mu - d[k] * log(mu);
            if (model) model[(size_t)bs * RR + k] = mu;
            if (psi_out) psi_out[(size_t)bs * RR + k] = psi;
            const double wgt = clamped ? 0.0 : 1.0 - d[k] / mu;
            acc[1] += wgt * psi;
#pragma unroll
            for (int q = 0; q < NPOLY; ++q) acc[3 + q] += wgt * poly_m(q, i, ii);
            w.aux[k] = At * wgt;  // g_psi
            acc[NOUT] += At * wgt * psi;
        }
        double tot[NOUT + 1];
#pragma unroll
        for (int q = 0; q < NOUT + 1; ++q) tot[q] = q == 2 ? 0.0 : block_reduce(acc[q], red);
        if (mode == 1) {
            // g_T = sgn(T) (g_psi - sum g_psi psi) / S
            for (int k = threadIdx.x; k < RR; k += blockDim.x) {
                const double t = w.T[k];
                w.aux[k] = (t < 0 ? -1.0 : 1.0) * (w.aux[k] - tot[NOUT]) / Ssum;
            }
            __syncthreads();
            // sigma: <g_T, dG I G^T + G I dG^T>
            cal_rows(V, V.dG, w.I, w.dJ);
            double gs = 0;
            for (int k = threadIdx.x; k < RR; k += blockDim.x) gs += w.aux[k] * cal_dT_sigma(V, w, k);
            tot[2] = block_reduce(gs, red);
            // g_I = G^T g_T G:  V1 = g_T G (R x W) into J, then g_I = G^T V1 (W x W) into I
            for (int k = threadIdx.x; k < R * W; k += blockDim.x) {
                const int ip = k / W, j = k % W;
                double a2 = 0;
                for (int jp = 0; jp < R; ++jp) a2 += w.aux[ip * R + jp] * V.G[jp * W + j];
                w.J[k] = a2;
            }
            __syncthreads();
            for (int k = threadIdx.x; k < W * W; k += blockDim.x) {
                const int i = k / W, j = k % W;
                double a2 = 0;
                for (int ip = 0; ip < R; ++ip) a2 += V.G[ip * W + i] * w.J[ip * W + j];
                w.I[k] = a2;
            }
            __syncthreads();
            // Ebar = g_I o E (in place), X = C^H Ebar (D x W, into S), Qbar = X conj(C)
            for (int k = threadIdx.x; k < W * W; k += blockDim.x) {
                w.E[k].x *= w.I[k];
                w.E[k].y *= w.I[k];
            }
            __syncthreads();
            for (int k = threadIdx.x; k < D * W; k += blockDim.x) {
                const int a = k / W, j = k % W;
                double2 a2 = make_double2(0, 0);
                for (int i = 0; i < W; ++i) {
                    const double2 cc = V.C[i * D + a], e = w.E[i * W + j];  // conj(c) * e
                    a2.x += cc.x * e.x + cc.y * e.y;
                    a2.y += cc.x * e.y - cc.y * e.x;
                }
                w.S[k] = a2;
            }
            __syncthreads();
            double* gp = gphi + (size_t)bs * D * D;
            for (int k = threadIdx.x; k < D * D; k += blockDim.x) {
                const int a = k / D, bb = k % D;
                double g = 0;
                if (V.pupil[k] != 0) {
                    double2 qb = make_double2(0, 0);
                    for (int j = 0; j < W; ++j) {
                        const double2 xv = w.S[a * W + j], cc = V.C[j * D + bb];  // x * conj(c)
                        qb.x += xv.x * cc.x + xv.y * cc.y;
                        qb.y += xv.y * cc.x - xv.x * cc.y;
                    }
                    const double2 q = w.Q[k];  // 2 Im(conj(q) qb)
                    g = 2.0 * (q.x * qb.y - q.y * qb.x);
                }
                gp[k] = g;
            }
        }
        if (threadIdx.x == 0)
            for (int q = 0; q < NOUT; ++q) out_slice[(size_t)NOUT * bs + q] = tot[q];
        __syncthreads();
    }
}

// Tangent maps d mu / d theta_t for phase directions (dir_bead >= -1) and for
// sigma (dir_bead == -2).  Items are (direction, bead, slice); a per-bead
// direction leaves other beads' maps at zero.  tan: per (t, bs) R x R.
__global__ void __launch_bounds__(CAL_THREADS) k_calib_tangent(CalView V, const double* phase, const double* bead,
                                                                const double* dirs, const int* dir_bead, int ndir,
                                                                char* scratch, size_t per_cta, double* tan) {
    __shared__ double red[CAL_THREADS / 32];
    const int D = V.D, W = V.W, R = V.R, RR = R * R, nbs = V.nb * V.ns;
    CalWork w = cal_carve(scratch + (size_t)blockIdx.x * per_cta, D, W, R);
    for (int item = blockIdx.x; item < ndir * nbs; item += gridDim.x) {
        const int t = item / nbs, bs = item % nbs, b = bs / V.ns, s = bs % V.ns;
        double* out = tan + ((size_t)t * nbs + bs) * RR;
        if (dir_bead[t] >= 0 && dir_bead[t] != b) {
            for (int k = threadIdx.x; k < RR; k += blockDim.x) out[k] = 0;
            continue;
        }
        const double* th = bead + (size_t)b * V.pb;
        const double At = (V.A0 ? V.A0[bs] : 0.0) + th[3 + s];
        const double Ssum = cal_forward(V, w, phase, th[0], th[1], V.dz[s] + th[2], red);
        if (dir_bead[t] == -2) {
            cal_rows(V, V.dG, w.I, w.dJ);
            for (int k = threadIdx.x; k < RR; k += blockDim.x) {
                const double sg = w.T[k] < 0 ? -1.0 : 1.0;
                w.aux[k] = sg * cal_dT_sigma(V, w, k);
            }
        } else {
            const double* dphi = dirs + (size_t)t * D * D;
            for (int k = threadIdx.x; k < D * D; k += blockDim.x) {
                const double2 q = w.Q[k];
                const double p = dphi[k];
                w.Q[k] = make_double2(-q.y * p, q.x * p);
            }
            __syncthreads();
            for (int k = threadIdx.x; k < D * W; k += blockDim.x) {
                const int a = k / W, j = k % W;
                double2 sacc = make_double2(0, 0);
                for (int bb = 0; bb < D; ++bb) {
                    const double2 q = w.Q[a * D + bb], cc = V.C[j * D + bb];
                    sacc.x += q.x * cc.x - q.y * cc.y;
                    sacc.y += q.x * cc.y + q.y * cc.x;
                }
                w.S[k] = sacc;
            }
            __syncthreads();
            for (int k = threadIdx.x; k < W * W; k += blockDim.x) {
                const int i = k / W, j = k % W;
                double2 e = make_double2(0, 0);
                for (int a = 0; a < D; ++a) {
                    const double2 cc = V.C[i * D + a], sv = w.S[a * W + j];
                    e.x += cc.x * sv.x - cc.y * sv.y;
                    e.y += cc.x * sv.y + cc.y * sv.x;
                }
                const double2 E0 = w.E[k];
                w.I[k] = 2.0 * (E0.x * e.x + E0.y * e.y);  // dI
            }
            __syncthreads();
            cal_rows(V, V.G, w.I, w.J);  // G dI
            for (int k = threadIdx.x; k < RR; k += blockDim.x) {
                const int ip = k / R, jp = k % R;
                double acc = 0;
                for (int j = 0; j < W; ++j) acc += V.G[jp * W + j] * w.J[ip * W + j];
                w.aux[k] = (w.T[k] < 0 ? -1.0 : 1.0) * acc;
            }
        }
        double dsum = 0;
        for (int k = threadIdx.x; k < RR; k += blockDim.x) dsum += w.aux[k];
        dsum = block_reduce(dsum, red);
        for (int k = threadIdx.x; k < RR; k += blockDim.x) {
            const double psi = fabs(w.T[k]) / Ssum;
            out[k] = At * (w.aux[k] - psi * dsum) / Ssum;
        }
        __syncthreads();
    }
}

// Per-slice Gauss-Newton blocks sum_p J_u J_v / mu over the slice's local
// directions: u < nzr Zernike tangents, then sigma, own x, y, z, psi (for
// a_bs) and the NPOLY background monomials; clamped pixels contribute nothing.
// gram: per slice nl (nl + 1) / 2 entries (upper triangle, row-major).
constexpr int GN_CHUNK = 32;
__global__ void __launch_bounds__(CAL_THREADS) k_calib_gn(CalView V, int nzr, const double* tan, const double* model,
                                                           const double* psi, double* gram) {
    extern __shared__ double sm[];  // nl x GN_CHUNK maps + GN_CHUNK inverse mu
    const int R = V.R, RR = R * R, nbs = V.nb * V.ns, nl = nzr + 4 + 1 + NPOLY, ne = nl * (nl + 1) / 2;
    constexpr int EPT = 8;  // Gram entries per thread and pass
    double* L = sm;
    double* inv = sm + (size_t)nl * GN_CHUNK;
    for (int bs = blockIdx.x; bs < nbs; bs += gridDim.x) {
        const int b = bs / V.ns;
        for (int e0 = 0; e0 < ne; e0 += CAL_THREADS * EPT) {
            double acc[EPT];
            int eu[EPT], ev[EPT];
#pragma unroll
            for (int q = 0; q < EPT; ++q) {
                acc[q] = 0;
                int e = e0 + q * CAL_THREADS + threadIdx.x, u = 0;
                // row u of the upper triangle holds nl - u entries
                while (u < nl && e >= nl - u) { e -= nl - u; ++u; }
                eu[q] = u < nl ? u : -1;
                ev[q] = u < nl ? u + e : -1;
            }
            for (int p0 = 0; p0 < RR; p0 += GN_CHUNK) {
                __syncthreads();
                for (int k = threadIdx.x; k < nl * GN_CHUNK; k += blockDim.x) {
                    const int u = k / GN_CHUNK, pp = k % GN_CHUNK, p = p0 + pp;
                    double v = 0;
                    if (p < RR) {
                        const size_t pix = (size_t)bs * RR + p;
                        if (u < nzr + 1) v = tan[((size_t)u * nbs) * RR + pix];
                        else if (u < nzr + 4) v = tan[((size_t)(nzr + 1 + 3 * b + (u - nzr - 1)) * nbs) * RR + pix];
                        else if (u == nzr + 4) v = psi[pix];
                        else v = poly_m(u - nzr - 5, p / R, p % R);
                    }
                    L[k] = v;
                }
                for (int pp = threadIdx.x; pp < GN_CHUNK; pp += blockDim.x) {
                    const int p = p0 + pp;
                    const double m = p < RR ? model[(size_t)bs * RR + p] : 0.0;
                    inv[pp] = (p < RR && m > 0.00000001) ? 1.0 / m : 0.0;
                }
                __syncthreads();
#pragma unroll
                for (int q = 0; q < EPT; ++q) {
                    if (eu[q] < 0) continue;
                    const double* a = L + (size_t)eu[q] * GN_CHUNK;
                    const double* c = L + (size_t)ev[q] * GN_CHUNK;
                    double s = 0;
                    for (int pp = 0; pp < GN_CHUNK; ++pp) s += a[pp] * c[pp] * inv[pp];
                    acc[q] += s;
                }
            }
#pragma unroll
            for (int q = 0; q < EPT; ++q) {
                const int e = e0 + q * CAL_THREADS + threadIdx.x;
                if (eu[q] >= 0 && e < ne) gram[(size_t)bs * ne + e] = acc[q];
            }
        }
        __syncthreads();
    }
}

// Deterministic reductions of per-slice results.  bead_grad: per bead
// (x, y, z, a_0..a_{ns-1}, c_0..c_5); tot = (nll, d/dsigma).
__global__ void __launch_bounds__(256) k_calib_reduce(CalView V, const double* out_slice, const double* gphi,
                                                      double* gphi_sum, double* bead_grad, double* tot) {
    const int D = V.D, nbs = V.nb * V.ns;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < D * D; k += gridDim.x * blockDim.x) {
        double s = 0;
        for (int bs = 0; bs < nbs; ++bs) s += gphi[(size_t)bs * D * D + k];
        gphi_sum[k] = s;
    }
    if (blockIdx.x < V.nb) {  // registration and photometry gradients: one block per bead
        __shared__ double red[3][256 / 32];
        const int b = blockIdx.x;
        double g[3] = {0, 0, 0};
        for (int k = threadIdx.x; k < V.ns * D * D; k += blockDim.x) {
            const int s = k / (D * D), pk = k % (D * D);
            const double v = gphi[((size_t)b * V.ns + s) * D * D + pk];
            g[0] += v * V.kx[pk / D];
            g[1] += v * V.ky[pk % D];
            g[2] -= v * V.kzoil[pk];
        }
        for (int q = 0; q < 3; ++q) {
            double v = g[q];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double* o = bead_grad + (size_t)b * V.pb;
            for (int q = 0; q < 3; ++q) {
                double v = 0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[q][w];
                o[q] = v;
            }
            for (int s = 0; s < V.ns; ++s) o[3 + s] = out_slice[(size_t)NOUT * (b * V.ns + s) + 1];
            for (int q = 0; q < NPOLY; ++q) {
                double v = 0;
                for (int s = 0; s < V.ns; ++s) v += out_slice[(size_t)NOUT * (b * V.ns + s) + 3 + q];
                o[3 + V.ns + q] = v;
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double nll = 0, gs = 0;
        for (int bs = 0; bs < nbs; ++bs) {
            nll += out_slice[(size_t)NOUT * bs];
            gs += out_slice[(size_t)NOUT * bs + 2];
        }
        tot[0] = nll;
        tot[1] = gs;
    }
}

}  // namespace zola

// --------------------------------------------------------------------- host --
using namespace zola;

namespace {

// Zernike basis on the disk square for modes 0..nz-1 (optics.cpp's polynomial),
// cached per (PSF, nz).
struct CalibCache {
    int nz = 0;
    std::vector<double> Z;  // nz x D x D
};

std::map<const zola_psf*, CalibCache> g_cal_cache;

double fact(int n) {
    double f = 1;
    for (int i = 2; i <= n; ++i) f *= i;
    return f;
}

double zern(int n, int m, double th, double rho) {
    int am = m < 0 ? -m : m;
    double s = 0;
    for (int k = 0; k <= (n - am) / 2; ++k)
        s += (((k & 1) ? -1.0 : 1.0) * fact(n - k)) / (fact(k) * fact((n + am) / 2 - k) * fact((n - am) / 2 - k)) *
             std::pow(rho, n - 2 * k);
    return m >= 0 ? s * std::cos(th * am) : s * std::sin(th * am);
}

const CalibCache* basis(zola_psf* p, int nz) {
    CalibCache& c = g_cal_cache[p];
    if (c.nz == nz) return &c;
    c = CalibCache();
    const int D = p->D, N = p->N;
    const double cc = (double)(N / 2) - 0.5;
    const double radius = (p->o.na / p->o.wavelength) * (N * p->o.xystep);
    c.nz = nz;
    c.Z.assign((size_t)nz * D * D, 0.0);
    std::vector<int> zn(nz), zm(nz);
    for (int idx = 0, n = 0; idx < nz; ++n)
        for (int m = -n; m <= n && idx < nz; m += 2, ++idx) { zn[idx] = n; zm[idx] = m; }
    for (int a = 0; a < D; ++a)
        for (int b = 0; b < D; ++b) {
            if (p->pupil[(size_t)a * D + b] == 0) continue;
            const double x = (p->a0 + a - cc) / radius, y = (p->a0 + b - cc) / radius;
            const double rho = std::sqrt(x * x + y * y), th = std::atan2(y, x);
            for (int i = 0; i < nz; ++i) c.Z[((size_t)i * D + a) * D + b] = rho < 1 ? zern(zn[i], zm[i], th, rho) : 0.0;
        }
    return &c;
}

struct CalRun {
    CalView V{};
    size_t per_cta = 0;
    int grid = 0;
    double* d_phase = nullptr;
    double* d_bead = nullptr;
    double* d_slice = nullptr;
    double* d_gphi = nullptr;
    double* d_gsum = nullptr;
    double* d_bgrad = nullptr;
    double* d_tot = nullptr;
    double* d_stacks = nullptr;
    double* d_dz = nullptr;
    double* d_A0 = nullptr;
    double* d_G = nullptr;
    double* d_dG = nullptr;
    double sigma = -1;
    char* scratch = nullptr;
    std::vector<void*> owned;
    CalRun() = default;
    CalRun(const CalRun&) = delete;
    CalRun& operator=(const CalRun&) = delete;
    ~CalRun() { for (void* p : owned) cudaFree(p); }
    cudaError_t alloc(void** p, size_t bytes) {
        cudaError_t e = cudaMalloc(p, bytes ? bytes : 8);
        if (e == cudaSuccess) owned.push_back(*p);
        return e;
    }
};

// Carve the buffers q[k] (bytes[k] each, 256-byte aligned) from a grow-only
// device area of the context; repeated calls of the same size allocate nothing.
cudaError_t carve(void** area, size_t* cap, void** const* q, const size_t* bytes, int n) {
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    size_t total = 0;
    for (int k = 0; k < n; ++k) total += al(bytes[k]);
    if (total > *cap) {
        if (*area) {
            cudaDeviceSynchronize();
            cudaFree(*area);
            *area = nullptr;
            *cap = 0;
        }
        cudaError_t e = cudaMalloc(area, total);
        if (e != cudaSuccess) return e;
        *cap = total;
    }
    char* base = (char*)*area;
    for (int k = 0; k < n; ++k) {
        *q[k] = bytes[k] ? base : nullptr;
        base += al(bytes[k]);
    }
    return cudaSuccess;
}

int cal_setup(zola_psf* p, const zola_calib_data* cd, CalRun& run, const CalibCache** cache) {
    zola_ctx* ctx = p->ctx;
    if (!cd || !cd->dz || !cd->stacks) { ctx->err = "calibration: null data"; return ZOLA_E_ARG; }
    const int R = cd->R, nz = cd->nz, nb = cd->nbead, ns = cd->nslice;
    if (R < 4 || R % 2 || R > p->N || nz < 4 || nz > 231 || nb < 1 || ns < 1) {
        ctx->err = "calibration: need even R <= N, 4 <= nz <= 231, beads and slices >= 1";
        return ZOLA_E_ARG;
    }
    if (p->o.kz_reset) { ctx->err = "calibration: build the PSF with kz_reset = 0"; return ZOLA_E_ARG; }
    WindowTables* w = get_window(p, R, ctx->err);
    if (!w) return ZOLA_E_ARG;
    *cache = basis(p, nz);
    cudaSetDevice(ctx->device);
    CalView& V = run.V;
    V.D = p->D; V.W = w->W; V.R = R; V.nb = nb; V.ns = ns; V.pb = 3 + ns + NPOLY;
    V.pupil = p->view.pupil; V.kx = p->view.kx; V.ky = p->view.ky; V.kzoil = p->view.kzoil;
    V.C = w->d_C;
    const size_t RR = (size_t)R * R, DD = (size_t)p->D * p->D, nbs = (size_t)nb * ns;
    run.per_cta = cal_work_bytes(p->D, w->W, R);
    run.grid = (int)std::min<size_t>(CAL_GRID, nbs);
    // The work buffers are carved from one grow-only area of the context, so that repeated
    // calls (an optimiser's forward / backward evaluations) allocate nothing.
    void** const q[] = {(void**)&run.d_phase, (void**)&run.d_bead, (void**)&run.d_slice, (void**)&run.d_gphi,
                        (void**)&run.d_gsum, (void**)&run.d_bgrad, (void**)&run.d_tot, (void**)&run.d_stacks,
                        (void**)&run.d_dz, (void**)&run.d_G, (void**)&run.d_dG, (void**)&run.scratch,
                        (void**)&run.d_A0};
    const size_t bytes[] = {DD * 8, (size_t)nb * V.pb * 8, nbs * NOUT * 8, nbs * DD * 8, DD * 8,
                            (size_t)nb * V.pb * 8, 16, nbs * RR * 8, (size_t)ns * 8, (size_t)R * w->W * 8,
                            (size_t)R * w->W * 8, (size_t)CAL_GRID * run.per_cta, cd->photons ? nbs * 8 : 0};
    cudaError_t e = carve(&ctx->calib_area, &ctx->calib_bytes, q, bytes, 13);
    if (e == cudaSuccess) e = cudaMemcpy(run.d_stacks, cd->stacks, nbs * RR * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(run.d_dz, cd->dz, (size_t)ns * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && cd->photons) e = cudaMemcpy(run.d_A0, cd->photons, nbs * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { ctx->err = std::string("calibration: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
    V.dz = run.d_dz;
    V.stacks = run.d_stacks;
    V.A0 = run.d_A0;
    V.G = run.d_G;
    V.dG = run.d_dG;
    return ZOLA_OK;
}

// Blur tables at sigma, phase = sum_{i >= 3} a_i Z_i, and bead parameters.
int cal_upload(zola_psf* p, const CalibCache* c, CalRun& run, const double* zern_coef, double sigma,
               const double* bead) {
    zola_ctx* ctx = p->ctx;
    if (!(sigma > 0)) { ctx->err = "calibration: sigma must be positive"; return ZOLA_E_ARG; }
    cudaError_t e = cudaSuccess;
    if (sigma != run.sigma) {
        std::vector<double> G, dG;
        blur_matrix(run.V.R, run.V.W, sigma, G, &dG);
        e = cudaMemcpy(run.d_G, G.data(), G.size() * 8, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(run.d_dG, dG.data(), dG.size() * 8, cudaMemcpyHostToDevice);
        run.sigma = sigma;
    }
    const int D = p->D;
    std::vector<double> ph((size_t)D * D, 0.0);
    for (int i = 3; i < c->nz; ++i) {
        const double a = zern_coef[i];
        if (a == 0) continue;
        const double* Zi = c->Z.data() + (size_t)i * D * D;
        for (size_t k = 0; k < ph.size(); ++k) ph[k] += a * Zi[k];
    }
    if (e == cudaSuccess) e = cudaMemcpy(run.d_phase, ph.data(), ph.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(run.d_bead, bead, (size_t)run.V.nb * run.V.pb * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { ctx->err = std::string("calibration upload: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
    return ZOLA_OK;
}

int cal_eval(zola_psf* p, const CalibCache* c, CalRun& run, const double* zern_coef, double sigma,
             const double* bead, int mode, double* nll, double* gz, double* gsig, double* gb, double* model_dev,
             double* psi_dev) {
    zola_ctx* ctx = p->ctx;
    int rc = cal_upload(p, c, run, zern_coef, sigma, bead);
    if (rc) return rc;
    k_calib<<<run.grid, CAL_THREADS>>>(run.V, run.d_phase, run.d_bead, mode, run.scratch, run.per_cta, run.d_slice,
                                       run.d_gphi, model_dev, psi_dev);
    ctx->launches++;
    if (mode == 0) {
        std::vector<double> sl((size_t)NOUT * run.V.nb * run.V.ns);
        cudaError_t e = cudaMemcpy(sl.data(), run.d_slice, sl.size() * 8, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { ctx->err = std::string("calibration: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
        double s = 0;
        for (int bs = 0; bs < run.V.nb * run.V.ns; ++bs) s += sl[(size_t)NOUT * bs];
        *nll = s;
        return ZOLA_OK;
    }
    k_calib_reduce<<<std::max(64, run.V.nb), 256>>>(run.V, run.d_slice, run.d_gphi, run.d_gsum, run.d_bgrad,
                                                    run.d_tot);
    ctx->launches++;
    double tot[2];
    cudaError_t e = cudaMemcpy(tot, run.d_tot, 16, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { ctx->err = std::string("calibration: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
    *nll = tot[0];
    if (gsig) *gsig = tot[1];
    const int D = p->D;
    std::vector<double> gsum((size_t)D * D);
    e = cudaMemcpy(gsum.data(), run.d_gsum, gsum.size() * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(gb, run.d_bgrad, (size_t)run.V.nb * run.V.pb * 8, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { ctx->err = std::string("calibration: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
    for (int i = 0; i < c->nz; ++i) {
        double s = 0;
        if (i >= 3) {
            const double* Zi = c->Z.data() + (size_t)i * D * D;
            for (size_t k = 0; k < gsum.size(); ++k) s += gsum[k] * Zi[k];
        }
        gz[i] = s;
    }
    return ZOLA_OK;
}

// Damped Cholesky solve (H + lambda max(diag H, floor)) x = -g; false if not positive definite.
bool damped_solve(const std::vector<double>& H, const std::vector<double>& g, int n, double lambda,
                  std::vector<double>& x) {
    std::vector<double> L((size_t)n * n, 0.0), y(n);
    x.assign(n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = H[(size_t)i * n + j] + (i == j ? lambda * std::max(H[(size_t)i * n + i], 1e-12) : 0.0);
            for (int k = 0; k < j; ++k) s -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
            if (i == j) {
                if (!(s > 0)) return false;
                L[(size_t)i * n + i] = std::sqrt(s);
            } else {
                L[(size_t)i * n + j] = s / L[(size_t)j * n + j];
            }
        }
    for (int i = 0; i < n; ++i) {
        double s = -g[i];
        for (int k = 0; k < i; ++k) s -= L[(size_t)i * n + k] * y[k];
        y[i] = s / L[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < n; ++k) s -= L[(size_t)k * n + i] * x[k];
        x[i] = s / L[(size_t)i * n + i];
    }
    return true;
}

}  // namespace

extern "C" {

int zola_calib_forward(zola_psf* psf, const zola_calib_data* data, const double* zernike, double sigma,
                       const double* bead, double* nll, double* model) {
    if (!psf) return ZOLA_E_ARG;
    if (!zernike || !bead || !nll) { psf->ctx->err = "zola_calib_forward: null argument"; return ZOLA_E_ARG; }
    CalRun run;
    const CalibCache* c = nullptr;
    int rc = cal_setup(psf, data, run, &c);
    if (rc) return rc;
    double* d_model = nullptr;
    const size_t nm = (size_t)data->nbead * data->nslice * data->R * data->R;
    if (model && run.alloc((void**)&d_model, nm * 8) != cudaSuccess) return ZOLA_E_CUDA;
    rc = cal_eval(psf, c, run, zernike, sigma, bead, 0, nll, nullptr, nullptr, nullptr, d_model, nullptr);
    if (rc) return rc;
    if (model && cudaMemcpy(model, d_model, nm * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return ZOLA_E_CUDA;
    return ZOLA_OK;
}

int zola_calib_backward(zola_psf* psf, const zola_calib_data* data, const double* zernike, double sigma,
                        const double* bead, double* nll, double* grad_zernike, double* grad_sigma, double* grad_bead) {
    if (!psf) return ZOLA_E_ARG;
    if (!zernike || !bead || !nll || !grad_zernike || !grad_bead) {
        psf->ctx->err = "zola_calib_backward: null argument";
        return ZOLA_E_ARG;
    }
    CalRun run;
    const CalibCache* c = nullptr;
    int rc = cal_setup(psf, data, run, &c);
    if (rc) return rc;
    return cal_eval(psf, c, run, zernike, sigma, bead, 1, nll, grad_zernike, grad_sigma, grad_bead, nullptr, nullptr);
}

// LM over theta = (a_3..a_{nz-1}, [sigma], per bead x, y, z, a_bs, c_bk):
// gradient from the adjoint, Gauss-Newton matrix sum J J^T / mu from device
// tangents and per-slice Gram blocks, FP64 damped solve; a step is accepted
// when the NLL drops.  zernike / sigma / bead are updated in place.
int zola_calib_fit(zola_psf* psf, const zola_calib_data* data, double* zernike, double* sigma, double* bead,
                   int max_iter, int flags, double* nll_out, int* iters_out) {
    if (!psf) return ZOLA_E_ARG;
    zola_ctx* ctx = psf->ctx;
    if (!zernike || !sigma || !bead || !nll_out || max_iter < 0) {
        ctx->err = "zola_calib_fit: null argument or negative max_iter";
        return ZOLA_E_ARG;
    }
    CalRun run;
    const CalibCache* c = nullptr;
    int rc = cal_setup(psf, data, run, &c);
    if (rc) return rc;
    const int D = psf->D, nz = data->nz, nzr = nz - 3, nb = data->nbead, ns = data->nslice, pb = run.V.pb;
    const int RR = data->R * data->R, nbs = nb * ns;
    const bool fit_sigma = (flags & ZOLA_CALIB_FIT_SIGMA) != 0;
    const int gsig = nzr;                         // theta index of sigma (when fitted)
    const int boff = nzr + (fit_sigma ? 1 : 0);   // first bead parameter
    const int npar = boff + nb * pb;
    // tangent directions: Zernike modes (all beads), sigma, x, y, z per bead
    const int ndir = nzr + 1 + 3 * nb;
    std::vector<double> dirs((size_t)ndir * D * D, 0.0);
    std::vector<int> dir_bead(ndir, -1);
    for (int i = 0; i < nzr; ++i)
        std::memcpy(&dirs[(size_t)i * D * D], c->Z.data() + (size_t)(i + 3) * D * D, (size_t)D * D * 8);
    dir_bead[nzr] = -2;
    for (int b = 0; b < nb; ++b)
        for (int q = 0; q < 3; ++q) {
            const int t = nzr + 1 + 3 * b + q;
            dir_bead[t] = b;
            for (int a = 0; a < D; ++a)
                for (int bb = 0; bb < D; ++bb) {
                    const size_t k = (size_t)a * D + bb;
                    if (psf->pupil[k] == 0) continue;
                    dirs[(size_t)t * D * D + k] = q == 0 ? psf->kx[a] : (q == 1 ? psf->ky[bb] : -psf->kzoil[k]);
                }
        }
    const int nl = nzr + 4 + 1 + NPOLY, ne = nl * (nl + 1) / 2;
    double *d_dirs = nullptr, *d_tan = nullptr, *d_model = nullptr, *d_psi = nullptr, *d_gram = nullptr;
    int* d_db = nullptr;
    void** const fq[] = {(void**)&d_dirs, (void**)&d_db, (void**)&d_tan, (void**)&d_model, (void**)&d_psi,
                         (void**)&d_gram};
    const size_t fb[] = {dirs.size() * 8, (size_t)ndir * 4, (size_t)ndir * nbs * RR * 8, (size_t)nbs * RR * 8,
                         (size_t)nbs * RR * 8, (size_t)nbs * ne * 8};
    if (carve(&ctx->calib_fit_area, &ctx->calib_fit_bytes, fq, fb, 6) != cudaSuccess) {
        ctx->err = "zola_calib_fit: device memory";
        return ZOLA_E_CUDA;
    }
    if (cudaMemcpy(d_dirs, dirs.data(), dirs.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_db, dir_bead.data(), (size_t)ndir * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        ctx->err = "zola_calib_fit: upload";
        return ZOLA_E_CUDA;
    }
    const size_t gn_smem = ((size_t)nl + 1) * GN_CHUNK * 8;
    if (gn_smem > 200 * 1024 ||
        cudaFuncSetAttribute(k_calib_gn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gn_smem) != cudaSuccess) {
        ctx->err = "zola_calib_fit: too many Zernike modes for the Gram kernel";
        return ZOLA_E_UNSUPPORTED;
    }
    std::vector<double> th(npar), g(npar), gz(nz), gb((size_t)nb * pb), gram((size_t)nbs * ne);
    std::vector<double> A0;
    if (data->photons) A0.assign(data->photons, data->photons + nbs);
    std::vector<double> zc(zernike, zernike + nz), bd(bead, bead + (size_t)nb * pb);
    double sg = *sigma;
    auto pack = [&](std::vector<double>& t) {
        for (int i = 0; i < nzr; ++i) t[i] = zernike[i + 3];
        if (fit_sigma) t[gsig] = *sigma;
        for (int k = 0; k < nb * pb; ++k) t[boff + k] = bead[k];
    };
    auto unpack = [&](const std::vector<double>& t) {
        for (int i = 0; i < nzr; ++i) zc[i + 3] = t[i];
        if (fit_sigma) sg = t[gsig];
        for (int k = 0; k < nb * pb; ++k) bd[k] = t[boff + k];
    };
    // theta index of each local Gram direction of slice (b, s); -1 when fixed
    auto gidx = [&](int b, int s, int u) -> int {
        if (u < nzr) return u;
        if (u == nzr) return fit_sigma ? gsig : -1;
        if (u < nzr + 4) return boff + b * pb + (u - nzr - 1);
        if (u == nzr + 4) return boff + b * pb + 3 + s;
        return boff + b * pb + 3 + ns + (u - nzr - 5);
    };
    auto evaluate = [&](const std::vector<double>& t, double* f, std::vector<double>& grad, bool with_gn,
                        std::vector<double>& H) -> int {
        unpack(t);
        double gs = 0;
        int r = cal_eval(psf, c, run, zc.data(), sg, bd.data(), 1, f, gz.data(), &gs, gb.data(), d_model, d_psi);
        if (r) return r;
        for (int i = 0; i < nzr; ++i) grad[i] = gz[i + 3];
        if (fit_sigma) grad[gsig] = gs;
        for (int k = 0; k < nb * pb; ++k) grad[boff + k] = gb[k];
        if (!with_gn) return 0;
        k_calib_tangent<<<(unsigned)std::min<size_t>(CAL_GRID, (size_t)ndir * nbs), CAL_THREADS>>>(
            run.V, run.d_phase, run.d_bead, d_dirs, d_db, ndir, run.scratch, run.per_cta, d_tan);
        k_calib_gn<<<(unsigned)std::min(CAL_GRID, nbs), CAL_THREADS, gn_smem>>>(run.V, nzr, d_tan, d_model, d_psi,
                                                                                d_gram);
        ctx->launches += 2;
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(gram.data(), d_gram, gram.size() * 8, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { ctx->err = std::string("zola_calib_fit: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
        H.assign((size_t)npar * npar, 0.0);
        for (int bs = 0; bs < nbs; ++bs) {
            const int b = bs / ns, s = bs % ns;
            const double* gm = &gram[(size_t)bs * ne];
            int e2 = 0;
            for (int u = 0; u < nl; ++u) {
                const int iu = gidx(b, s, u);
                for (int v = u; v < nl; ++v, ++e2) {
                    const int iv = gidx(b, s, v);
                    if (iu < 0 || iv < 0) continue;
                    H[(size_t)iu * npar + iv] += gm[e2];
                    if (iu != iv) H[(size_t)iv * npar + iu] += gm[e2];
                }
            }
        }
        return 0;
    };
    auto constrain = [&](std::vector<double>& t) {
        if (fit_sigma) t[gsig] = std::max(t[gsig], 0.05);
        for (int b = 0; b < nb; ++b)
            for (int s = 0; s < ns; ++s) {
                const double a0 = A0.empty() ? 0.0 : A0[(size_t)b * ns + s];
                double& a = t[boff + b * pb + 3 + s];
                a = std::max(a, 1.0 - a0);  // total photons >= 1
            }
    };
    pack(th);
    double nll = 0, lambda = 1e-3;
    int it = 0;
    std::vector<double> H, Hn, step, g2(npar);
    rc = evaluate(th, &nll, g, true, H);
    if (rc) return rc;
    for (it = 0; it < max_iter; ++it) {
        if (!damped_solve(H, g, npar, lambda, step)) {
            lambda *= 10;
            if (lambda > 1e10) break;
            continue;
        }
        std::vector<double> t2(th);
        for (int i = 0; i < npar; ++i) t2[i] += step[i];
        constrain(t2);
        double nll2;
        rc = evaluate(t2, &nll2, g2, false, Hn);
        if (rc) return rc;
        if (nll2 <= nll) {
            const double dec = nll - nll2;
            th = t2;
            nll = nll2;
            lambda = std::max(lambda * 0.1, 1e-9);
            rc = evaluate(th, &nll, g, true, H);
            if (rc) return rc;
            if (dec < 1e-9 * std::max(1.0, std::fabs(nll))) { ++it; break; }
        } else {
            lambda *= 10;
            if (lambda > 1e10) break;
        }
    }
    unpack(th);
    std::memcpy(zernike, zc.data(), (size_t)nz * 8);
    std::memcpy(bead, bd.data(), bd.size() * 8);
    *sigma = sg;
    *nll_out = nll;
    if (iters_out) *iters_out = it;
    return ZOLA_OK;
}

}  // extern "C"
