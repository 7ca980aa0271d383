// Plain FP64 GPU form of the PSF model and of the per-ROI Poisson MLE fit.
//
// One CTA per ROI (persistent grid pulling ROIs from a device counter), all
// arithmetic in FP64 on the CUDA cores, no tensor cores.  This is the 1x
// reference the split-precision tcgen05 path is measured against, and the
// FP64 device model that the parity tests compare with the CPU oracle.
//
// The model restates process/cpu/PSFPhase.java:557-629 (pupil -> |IFFT|^2 ->
// circular Gaussian blur -> |.| -> crop -> normalise) as partial DFTs:
//   Q  = pupil * exp(i(kx x + ky y + phase + kz zwat - kzoil zoil))   (D x D)
//   S  = Q C^T,  Sy = Q diag(i ky) C^T,  Sz = (i kz o Q) C^T          (D x W)
//   E  = C S,  Ex = C diag(i kx) S,  Ey = C Sy,  Ez = C Sz            (W x W)
//   I  = |E|^2,  I_t = 2 Re(conj(E) E_t)
//   B  = G I G^T (R x R),  psi = |B| / sum|B|,
//   dpsi_t = (sgn(B) B_t - psi sum sgn(B) B_t) / sum|B|.
// The forward field uses the reference's (cos q, sin r) pair (PSFPhase.java:565-569)
// so evanescent tables built with resetKz are reproduced; derivatives assume
// q == r, which holds for the fit tables (kz = 0 where evanescent).
#include <cuda_runtime.h>

#include <mutex>

#include "lm.h"
#include "zola_internal.h"

namespace zola {

constexpr int F64_THREADS = 512;
constexpr int F64_WARPS = F64_THREADS / 32;
constexpr int F64_NRED = 1 + 5 + 15 + 15;  // nll, g, H (lower), F (lower)

struct F64Work {
    double2* Q;  // D*D
    double2* S;  // 3 * D*W
    double* I;   // 4 * W*W
    double* J;   // 4 * R*W
    double* T;   // 4 * R*R
};

__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

__host__ __device__ inline size_t f64_work_bytes(int D, int W, int R) {
    size_t b = 0;
    b += align_up((size_t)D * D * 16, 256);
    b += align_up((size_t)3 * D * W * 16, 256);
    b += align_up((size_t)4 * W * W * 8, 256);
    b += align_up((size_t)4 * R * W * 8, 256);
    b += align_up((size_t)4 * R * R * 8, 256);
    return b;
}

__device__ inline F64Work f64_carve(char* base, int D, int W, int R) {
    F64Work w;
    size_t o = 0;
    w.Q = (double2*)(base + o); o += align_up((size_t)D * D * 16, 256);
    w.S = (double2*)(base + o); o += align_up((size_t)3 * D * W * 16, 256);
    w.I = (double*)(base + o);  o += align_up((size_t)4 * W * W * 8, 256);
    w.J = (double*)(base + o);  o += align_up((size_t)4 * R * W * 8, 256);
    w.T = (double*)(base + o);
    return w;
}

// Block-wide sum of NV doubles per thread; result in red[0..NV) for all threads.
template <int NV>
__device__ inline void block_sum(double (&v)[NV], double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        v[k] = x;
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) red[warp * NV + k] = v[k];
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w * NV + threadIdx.x];
        red[F64_WARPS * NV + threadIdx.x] = s;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = red[F64_WARPS * NV + k];
    __syncthreads();
}

__device__ inline double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ inline double2 cmadd(double2 acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
    return acc;
}

// Computes the four blurred R x R maps T[0..3] = blurred I, I_x, I_y, I_z
// (only T[0] when derivs is false).  All threads of the block participate.
__device__ void eval_maps_f64(const PsfView& P, const WinView& Wn, const F64Work& w, double x, double y,
                              double zoil, double zwat, bool derivs) {
    const int D = P.D, W = Wn.W, R = Wn.R, tid = threadIdx.x, nt = blockDim.x;
    // 1. pupil field on the disk square
    for (int idx = tid; idx < D * D; idx += nt) {
        int a = idx / D, b = idx - a * D;
        double pup = P.pupil[idx];
        double2 q2 = make_double2(0.0, 0.0);
        if (pup != 0.0) {
            double pp = P.kx[a] * x + P.ky[b] * y + P.phase[idx];
            double q = pp + P.kz[idx] * zwat - P.kzoil[idx] * zoil;
            double r = pp + P.kz[idx] * zwat * P.isim[idx] - P.kzoil[idx] * zoil * P.isimoil[idx];
            q2 = make_double2(pup * cos(q), pup * sin(r));
        }
        w.Q[idx] = q2;
    }
    __syncthreads();
    // 2. first contraction over pupil columns b
    double2* S = w.S;
    double2* Sy = w.S + (size_t)D * W;
    double2* Sz = w.S + (size_t)2 * D * W;
    // a thread takes 4 rows a of one column j: each C value it loads serves 4 outputs
    // (every output still sums its terms in the order b = 0, 1, ...)
    constexpr int TA = 4;
    const int DA = (D + TA - 1) / TA;
    for (int idx = tid; idx < DA * W; idx += nt) {
        const int a0 = (idx / W) * TA, j = idx - (idx / W) * W;
        double2 s[TA], sy[TA], sz[TA];
#pragma unroll
        for (int t = 0; t < TA; ++t) { s[t] = make_double2(0, 0); sy[t] = make_double2(0, 0); sz[t] = make_double2(0, 0); }
        const double2* crow = Wn.C + (size_t)j * D;
        for (int b = 0; b < D; ++b) {
            const double2 c = crow[b];
            const double ky = P.ky[b];
#pragma unroll
            for (int t = 0; t < TA; ++t) {
                if (a0 + t >= D) break;
                const double2 q = w.Q[(size_t)(a0 + t) * D + b];
                const double2 qc = cmul(q, c);
                s[t].x += qc.x; s[t].y += qc.y;
                if (derivs) {
                    const double kz = P.kz[(a0 + t) * D + b];
                    sy[t].x -= ky * qc.y; sy[t].y += ky * qc.x;   // (i ky) q c
                    sz[t].x -= kz * qc.y; sz[t].y += kz * qc.x;   // (i kz) q c
                }
            }
        }
#pragma unroll
        for (int t = 0; t < TA; ++t) {
            if (a0 + t >= D) break;
            const size_t o = (size_t)(a0 + t) * W + j;
            S[o] = s[t];
            if (derivs) { Sy[o] = sy[t]; Sz[o] = sz[t]; }
        }
    }
    __syncthreads();
    // 3. second contraction over pupil rows a, then intensities
    double* I0 = w.I;
    double* I1 = w.I + (size_t)W * W;
    double* I2 = w.I + (size_t)2 * W * W;
    double* I3 = w.I + (size_t)3 * W * W;
    // a thread takes 4 rows i of one column j: each S, S_y, S_z value it loads serves 4
    // outputs (every output still sums its terms in the order a = 0, 1, ...)
    constexpr int TI = 4;
    for (int idx = tid; idx < (W / TI) * W; idx += nt) {
        const int i0 = (idx / W) * TI, j = idx - (idx / W) * W;
        double2 e[TI], ex[TI], ey[TI], ez[TI];
#pragma unroll
        for (int t = 0; t < TI; ++t) {
            e[t] = make_double2(0, 0); ex[t] = make_double2(0, 0); ey[t] = make_double2(0, 0); ez[t] = make_double2(0, 0);
        }
        for (int a = 0; a < D; ++a) {
            const double2 s = S[(size_t)a * W + j];
            double2 sy, sz;
            double kx = 0;
            if (derivs) { sy = Sy[(size_t)a * W + j]; sz = Sz[(size_t)a * W + j]; kx = P.kx[a]; }
#pragma unroll
            for (int t = 0; t < TI; ++t) {
                const double2 c = Wn.C[(size_t)(i0 + t) * D + a];
                const double2 cs = cmul(c, s);
                e[t].x += cs.x; e[t].y += cs.y;
                if (derivs) {
                    ex[t].x -= kx * cs.y; ex[t].y += kx * cs.x;
                    ey[t] = cmadd(ey[t], c, sy);
                    ez[t] = cmadd(ez[t], c, sz);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < TI; ++t) {
            const size_t o = (size_t)(i0 + t) * W + j;
            I0[o] = e[t].x * e[t].x + e[t].y * e[t].y;
            if (derivs) {
                I1[o] = 2.0 * (e[t].x * ex[t].x + e[t].y * ex[t].y);
                I2[o] = 2.0 * (e[t].x * ey[t].x + e[t].y * ey[t].y);
                I3[o] = 2.0 * (e[t].x * ez[t].x + e[t].y * ez[t].y);
            }
        }
    }
    __syncthreads();
    // 4. blur along the first index: J[m][i'][j] = sum_i G[i'][i] I[m][i][j]
    const int nm = derivs ? 4 : 1;
    // a thread takes 4 rows i' of one column j (each I value loaded serves 4 outputs)
    constexpr int TR = 4;
    const int RB = (R + TR - 1) / TR;
    for (int idx = tid; idx < nm * RB * W; idx += nt) {
        const int m = idx / (RB * W), rem = idx - m * RB * W, ip0 = (rem / W) * TR, j = rem - (rem / W) * W;
        const double* Im = w.I + (size_t)m * W * W;
        double acc[TR] = {0.0, 0.0, 0.0, 0.0};
        for (int i = 0; i < W; ++i) {
            const double v = Im[(size_t)i * W + j];
#pragma unroll
            for (int t = 0; t < TR; ++t)
                if (ip0 + t < R) acc[t] = fma(Wn.G[(size_t)(ip0 + t) * W + i], v, acc[t]);
        }
#pragma unroll
        for (int t = 0; t < TR; ++t)
            if (ip0 + t < R) w.J[((size_t)m * R + ip0 + t) * W + j] = acc[t];
    }
    __syncthreads();
    // 5. blur along the second index: T[m][i'][j'] = sum_j G[j'][j] J[m][i'][j]
    for (int idx = tid; idx < nm * R * R; idx += nt) {
        int m = idx / (R * R), rem = idx - m * R * R, ip = rem / R, jp = rem - ip * R;
        const double* g = Wn.G + (size_t)jp * W;
        const double* Jm = w.J + (size_t)m * R * W + (size_t)ip * W;
        double acc = 0.0;
        for (int j = 0; j < W; ++j) acc = fma(g[j], Jm[j], acc);
        w.T[idx] = acc;
    }
    __syncthreads();
}

// Normalisation sums: S = sum |T0|, Dt = sum sgn(T0) T_t.
__device__ inline void norm_sums(const F64Work& w, int R, bool derivs, double* red, double (&s)[4]) {
    double v[4] = {0, 0, 0, 0};
    const double* T = w.T;
    for (int k = threadIdx.x; k < R * R; k += blockDim.x) {
        double t0 = T[k];
        double sg = t0 < 0 ? -1.0 : 1.0;
        v[0] += fabs(t0);
        if (derivs) {
            v[1] += sg * T[R * R + k];
            v[2] += sg * T[2 * R * R + k];
            v[3] += sg * T[3 * R * R + k];
        }
    }
    block_sum<4>(v, red);
    for (int k = 0; k < 4; ++k) s[k] = v[k];
}

// Writes psi (and dpsi) of n models; one CTA per model.  With a list, only
// the models list[0 .. *n_dev) are evaluated (position list[m] of xyz, written
// at the same index of out).
__global__ void __launch_bounds__(F64_THREADS) model_f64_kernel(PsfView P, WinView Wn, const double* xyz, int n,
                                                                double* out, double* dout, char* gscratch,
                                                                size_t per_cta, int use_smem, const int* list,
                                                                const int* n_dev) {
    extern __shared__ __align__(256) char smem_raw[];
    double* red = (double*)smem_raw;
    char* base = use_smem ? smem_raw + 8192 : gscratch + (size_t)blockIdx.x * per_cta;
    F64Work w = f64_carve(base, P.D, Wn.W, Wn.R);
    const int R = Wn.R;
    const bool derivs = dout != nullptr;
    const int nn = n_dev ? min(n, *n_dev) : n;
    for (int mi = blockIdx.x; mi < nn; mi += gridDim.x) {
        const int m = list ? list[mi] : mi;
        eval_maps_f64(P, Wn, w, xyz[3 * m], xyz[3 * m + 1], P.zfocus, xyz[3 * m + 2], derivs);
        double s[4];
        norm_sums(w, R, derivs, red, s);
        for (int k = threadIdx.x; k < R * R; k += blockDim.x) {
            double t0 = w.T[k];
            double sg = t0 < 0 ? -1.0 : 1.0;
            double psi = fabs(t0) / s[0];
            out[(size_t)m * R * R + k] = psi;
            if (derivs)
                for (int d = 0; d < 3; ++d)
                    dout[((size_t)m * 3 + d) * R * R + k] = (sg * w.T[(d + 1) * R * R + k] - psi * s[d + 1]) / s[0];
        }
        __syncthreads();
    }
}

// Likelihood, gradient, Gauss-Newton Hessian and Fisher matrix at theta.
// sv (nullable): the ROI's sCMOS term var/gain^2, added to the mean
// (process/cpu/Localization.java:1132).
__device__ void eval_lik_f64(const PsfView& P, const WinView& Wn, const F64Work& w, const float* d, const float* sv,
                             const double* th, double* red, double& nll, double* g, double* H, double* F) {
    const int R = Wn.R;
    eval_maps_f64(P, Wn, w, th[0], th[1], P.zfocus, th[2], true);
    double s[4];
    norm_sums(w, R, true, red, s);
    double v[F64_NRED];
#pragma unroll
    for (int k = 0; k < F64_NRED; ++k) v[k] = 0.0;
    const double A = th[3], B = th[4];
    bool bad = false;
    for (int k = threadIdx.x; k < R * R; k += blockDim.x) {
        double t0 = w.T[k];
        double sg = t0 < 0 ? -1.0 : 1.0;
        double psi = fabs(t0) / s[0];
        double j[5];
        for (int q = 0; q < 3; ++q) j[q] = A * (sg * w.T[(q + 1) * R * R + k] - psi * s[q + 1]) / s[0];
        j[3] = psi;
        j[4] = 1.0;
        double mu = A * psi + B + (sv ? (double)sv[k] : 0.0);
        if (!(mu > 0.0)) { bad = true; continue; }
        double dk = (double)d[k];
        v[0] += dk > 0 ? mu - dk - dk * log(mu / dk) : mu;
        double wg = 1.0 - dk / mu, wh = dk / (mu * mu), wf = 1.0 / mu;
        int o = 1;
#pragma unroll
        for (int q = 0; q < 5; ++q) v[o + q] += wg * j[q];
        o = 6;
#pragma unroll
        for (int q = 0; q < 5; ++q)
#pragma unroll
            for (int r = 0; r <= q; ++r) {
                v[o] += wh * j[q] * j[r];
                v[o + 15] += wf * j[q] * j[r];
                ++o;
            }
    }
    if (bad) v[0] = INFINITY;
    block_sum<F64_NRED>(v, red);
    nll = v[0];
    for (int q = 0; q < 5; ++q) g[q] = v[1 + q];
    int o = 6;
    for (int q = 0; q < 5; ++q)
        for (int r = 0; r <= q; ++r) {
            H[q * 5 + r] = H[r * 5 + q] = v[o];
            F[q * 5 + r] = F[r * 5 + q] = v[o + 15];
            ++o;
        }
}

__global__ void __launch_bounds__(F64_THREADS) fit_f64_kernel(PsfView P, WinView Wn, const float* rois,
                                                              const float* scmos, const double* init, int n,
                                                              FitParamsDev prm,
                                                              double* out5, double* crlb5, double* nll_out,
                                                              int* st_out, int* it_out, char* gscratch,
                                                              size_t per_cta, int use_smem, int* counter) {
    extern __shared__ __align__(256) char smem_raw[];
    double* red = (double*)smem_raw;  // 8192-byte reduction area
    __shared__ LMState st;
    __shared__ int roi;
    __shared__ int go;
    char* base = use_smem ? smem_raw + 8192 : gscratch + (size_t)blockIdx.x * per_cta;
    F64Work w = f64_carve(base, P.D, Wn.W, Wn.R);
    const int R = Wn.R;
    for (;;) {
        if (threadIdx.x == 0) roi = atomicAdd(counter, 1);
        __syncthreads();
        const int r = roi;
        if (r >= n) break;
        const float* d = rois + (size_t)r * R * R;
        const float* sv = scmos ? scmos + (size_t)r * R * R : nullptr;
        if (threadIdx.x == 0) {
            for (int q = 0; q < 5; ++q) st.th[q] = init[5 * r + q];
            lm_clamp(st.th, prm);
        }
        __syncthreads();
        double th[5], nll, g[5], H[25], F[25];
        for (int q = 0; q < 5; ++q) th[q] = st.th[q];
        eval_lik_f64(P, Wn, w, d, sv, th, red, nll, g, H, F);
        if (threadIdx.x == 0) {
            lm_start(st, nll, g, H, F, prm);
            go = lm_propose(st, prm) ? 1 : 0;
        }
        __syncthreads();
        while (go) {
            for (int q = 0; q < 5; ++q) th[q] = st.trial[q];
            eval_lik_f64(P, Wn, w, d, sv, th, red, nll, g, H, F);
            if (threadIdx.x == 0) {
                lm_update(st, nll, g, H, F, prm);
                go = lm_propose(st, prm) ? 1 : 0;
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            for (int q = 0; q < 5; ++q) out5[5 * r + q] = st.th[q];
            if (nll_out) nll_out[r] = st.nll;
            if (st_out) st_out[r] = st.status;
            if (it_out) it_out[r] = st.evals;
            if (crlb5) lm_crlb(st.F, crlb5 + 5 * r);
        }
        __syncthreads();
    }
}

static int f64_layout(zola_ctx* ctx, zola_psf* p, WindowTables* w, int nblocks, size_t& per_cta, int& use_smem,
                      size_t& smem, std::string& err) {
    per_cta = f64_work_bytes(p->D, w->W, w->R);
    use_smem = per_cta + 8192 <= 200 * 1024;
    smem = 8192 + (use_smem ? per_cta : 0);
    if (!use_smem) {
        if (ensure_scratch(ctx, per_cta * (size_t)nblocks, err)) return ZOLA_E_CUDA;
    }
    return 0;
}

int launch_model_f64(zola_ctx* ctx, zola_psf* p, WindowTables* w, const double* d_xyz, int n, double* d_out,
                     double* d_dout, cudaStream_t st, const int* d_list, const int* d_count) {
    if (n <= 0) return ZOLA_OK;
    int nblocks = std::min(n, ctx->num_sms * 2);
    size_t per_cta, smem;
    int use_smem;
    if (f64_layout(ctx, p, w, nblocks, per_cta, use_smem, smem, ctx->err)) return ZOLA_E_CUDA;
    ZOLA_CUDA_CHECK(cudaFuncSetAttribute(model_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), ctx);
    WinView wv{w->R, w->W, w->d_C, w->d_G};
    prof_begin(ctx, 6, st);
    model_f64_kernel<<<nblocks, F64_THREADS, smem, st>>>(p->view, wv, d_xyz, n, d_out, d_dout, (char*)ctx->scratch,
                                                         per_cta, use_smem, d_list, d_count);
    prof_end(ctx, st);
    ctx->launches++;
    ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
    return ZOLA_OK;
}

int launch_fit_f64(zola_ctx* ctx, zola_psf* p, WindowTables* w, const float* d_rois, const float* d_scmos,
                   const double* d_init, int n, const zola_fit_params* prm, double* d_out5, double* d_crlb5,
                   double* d_nll, int* d_status, int* d_iters, cudaStream_t st) {
    if (n <= 0) return ZOLA_OK;
    int nblocks = std::min(n, ctx->num_sms * 2);
    size_t per_cta, smem;
    int use_smem;
    if (f64_layout(ctx, p, w, nblocks, per_cta, use_smem, smem, ctx->err)) return ZOLA_E_CUDA;
    if (use_smem && smem > 110 * 1024) nblocks = std::min(n, ctx->num_sms);
    ZOLA_CUDA_CHECK(cudaFuncSetAttribute(fit_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), ctx);
    FitParamsDev fp{prm->zmin, prm->zmax, prm->xymax, prm->tol_xyz, prm->step_xy, prm->step_z, prm->max_iter};
    WinView wv{w->R, w->W, w->d_C, w->d_G};
    ZOLA_CUDA_CHECK(cudaMemsetAsync(ctx->d_counter, 0, sizeof(int), st), ctx);
    prof_begin(ctx, 5, st);
    fit_f64_kernel<<<nblocks, F64_THREADS, smem, st>>>(p->view, wv, d_rois, d_scmos, d_init, n, fp, d_out5, d_crlb5,
                                                       d_nll,
                                                       d_status, d_iters, (char*)ctx->scratch, per_cta, use_smem,
                                                       ctx->d_counter);
    prof_end(ctx, st);
    ctx->launches++;
    ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
    return ZOLA_OK;
}

}  // namespace zola

// ------------------------------------------------------------------------
// Allocation-free FP64 fit.
//
// Some callers cannot allocate device memory at the time they fit: a host
// application that reserves all device memory for itself at start-up and hands
// plugins only the buffers it owns, or an acquisition thread that must not
// stall on cudaMalloc / cudaFree (both can synchronise the whole device).  For
// them zola_fit_batch_noalloc runs the plain FP64 fit with its per-block work
// areas and its ROI-queue counter in the file-scope array below instead of the
// context's scratch.  The array is part of the library image: every GPU on
// which the library is loaded holds its NOALLOC_SCRATCH_BYTES until the
// process exits.  All calls share it, and it keeps the previous call's
// contents (the counter is cleared at the start of every call), so calls whose
// work overlaps on the GPU (other streams, other host threads) race; serialise
// them.
namespace zola {
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)64 << 20;  // 64 MiB
}  // namespace zola

static __device__ __align__(256) unsigned char g_fit_noalloc_scratch[zola::NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex g_noalloc_mu;
// One cached device address per (device, CUDA context): a context that was
// destroyed and created again (cudaDeviceReset, or the primary context
// released and retained again) gets its address looked up afresh.
struct NoallocEntry {
    void* context = nullptr;
    void* ptr = nullptr;
};
NoallocEntry g_noalloc[64];

// The current CUDA context of the calling thread, through the driver entry
// point the runtime exposes (no link against the driver library).
void* current_context() {
    typedef int (*CtxGetCurrent)(void**);
    static CtxGetCurrent fn = nullptr;
    static bool looked = false;
    if (!looked) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (CtxGetCurrent)f;
        looked = true;
    }
    void* c = nullptr;
    if (fn && fn(&c) != 0) c = nullptr;
    return c;
}

// Device address of the scratch array in the current context (host code must
// not use the array's name as a device pointer).  Looked up once per device
// and context; the caller has made the device current.
void* noalloc_scratch(int device, std::string& err) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (device < 0 || device >= 64) {
        err = "zola_fit_batch_noalloc: device index out of range";
        return nullptr;
    }
    void* c = current_context();
    NoallocEntry& e = g_noalloc[device];
    if (!e.ptr || c != e.context) {
        void* p = nullptr;
        cudaError_t rc = cudaGetSymbolAddress(&p, g_fit_noalloc_scratch);
        if (rc != cudaSuccess || !p) {
            err = std::string("zola_fit_batch_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(rc);
            return nullptr;
        }
        e.ptr = p;
        e.context = c;
    }
    return e.ptr;
}
}  // namespace

extern "C" int zola_fit_batch_noalloc(zola_psf* psf, int R, const float* d_rois, const double* d_init5, int n,
                                      const zola_fit_params* prm, double* d_out5, double* d_crlb5, double* d_nll,
                                      int* d_status, int* d_iters, void* stream) {
    using namespace zola;
    if (!psf) return ZOLA_E_ARG;
    zola_ctx* ctx = psf->ctx;
    if (!prm || prm->precision != ZOLA_PREC_FP64 || prm->max_iter < 1 || prm->max_iter > 1000 ||
        !(prm->zmax >= prm->zmin) || !(prm->xymax > 0) || !(prm->step_xy > 0) || !(prm->step_z > 0) ||
        !(prm->tol_xyz >= 0)) {
        ctx->err = "zola_fit_batch_noalloc: needs valid FP64 fit params (precision = ZOLA_PREC_FP64)";
        return ZOLA_E_ARG;
    }
    if (n < 0 || (n > 0 && (!d_rois || !d_init5 || !d_out5))) {
        ctx->err = "zola_fit_batch_noalloc: bad n or null buffer";
        return ZOLA_E_ARG;
    }
    if (psf->o.kz_reset) {
        ctx->err = "zola_fit_batch_noalloc: fit needs a PSF built with kz_reset = 0";
        return ZOLA_E_ARG;
    }
    // Only look the window tables up: building them would allocate.
    auto it = psf->win.find(R);
    if (it == psf->win.end()) {
        ctx->err = "zola_fit_batch_noalloc: tables for this ROI size are not prepared; call "
                   "zola_psf_model_dev(psf, R, NULL, 0, NULL, NULL, stream) once beforehand";
        return ZOLA_E_ARG;
    }
    WindowTables* w = &it->second;
    if (n == 0) return ZOLA_OK;
    // the PSF's device, as every other entry point (no allocation once its context exists)
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        ctx->err = "zola_fit_batch_noalloc: cudaSetDevice failed";
        return ZOLA_E_CUDA;
    }
    char* base = (char*)noalloc_scratch(ctx->device, ctx->err);
    if (!base) return ZOLA_E_CUDA;
    const size_t per_cta = f64_work_bytes(psf->D, w->W, w->R);
    const int use_smem = per_cta + 8192 <= 200 * 1024;
    const size_t smem = 8192 + (use_smem ? per_cta : 0);
    int* counter = (int*)base;
    char* work = base + 256;
    const size_t room = NOALLOC_SCRATCH_BYTES - 256;
    int nblocks = std::min(n, ctx->num_sms * 2);
    if (use_smem && smem > 110 * 1024) nblocks = std::min(n, ctx->num_sms);
    if (!use_smem) {
        if (per_cta > room) {
            ctx->err = "zola_fit_batch_noalloc: one block's work area (" + std::to_string(per_cta) +
                       " bytes for this ROI size) exceeds the 64 MiB static scratch";
            return ZOLA_E_ARG;
        }
        nblocks = std::min<long long>(nblocks, (long long)(room / per_cta));
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : ctx->stream;
    cudaError_t e = cudaFuncSetAttribute(fit_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) {
        ctx->err = std::string("zola_fit_batch_noalloc: ") + cudaGetErrorString(e);
        return ZOLA_E_CUDA;
    }
    FitParamsDev fp{prm->zmin, prm->zmax, prm->xymax, prm->tol_xyz, prm->step_xy, prm->step_z, prm->max_iter};
    WinView wv{w->R, w->W, w->d_C, w->d_G};
    fit_f64_kernel<<<nblocks, F64_THREADS, smem, st>>>(psf->view, wv, d_rois, nullptr, d_init5, n, fp, d_out5,
                                                       d_crlb5, d_nll,
                                                       d_status, d_iters, work, per_cta, use_smem, counter);
    ctx->launches++;
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        ctx->err = std::string("zola_fit_batch_noalloc: ") + cudaGetErrorString(e);
        return ZOLA_E_CUDA;
    }
    return ZOLA_OK;
}
