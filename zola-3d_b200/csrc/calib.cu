// Zernike PSF calibration from bead z-stacks: FP64 forward model, hand-written
// adjoint (reverse mode) and forward-mode tangents, and an FP64
// Levenberg-Marquardt driver.
//
// Model (process/cpu/ZernikePhaseRetrieval.java:1843-1874): for bead b and
// slice s, the PSF at (x_b, y_b, zoil = dz_s + z_b, zwat = 0) with phase
// sum_i a_i Z_i over modes i >= 3 (modes 0-2 are the per-bead registration,
// :93-95, carried here as x_b, y_b, z_b), mu = A_b psi + B_b, and
//   NLL = sum_{b,s,p} mu - d ln mu.
// The reference optimises one coefficient at a time by finite-difference
// Newton steps (:1081-1198).  Here the gradient of the whole stack NLL comes
// from one adjoint pass per slice:
//   w = 1 - d/mu;  g_psi = A w;  g_m = (g_psi - sum g_psi psi) / S;  g_T = sgn(T) g_m
//   g_I = G^T g_T G;  Ebar = g_I o E;  Qbar = C^H Ebar conj(C)
//   g_phi = 2 Im(conj(Q) Qbar)   (per pupil pixel)
//   dNLL/da_i = sum g_phi Z_i,  dNLL/dx_b = sum g_phi kx,  dNLL/dy_b = sum g_phi ky,
//   dNLL/dz_b = -sum g_phi kzoil,  dNLL/dA_b = sum w psi,  dNLL/dB_b = sum w.
// Tangents (for the Gauss-Newton matrix) push a phase direction dphi through
// dQ = i Q dphi, dE = C dQ C^T, dI = 2 Re(conj E dE), dT = G dI G^T,
// dpsi = (sgn T dT - psi sum sgn T dT) / S.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "lm.h"
#include "zola_internal.h"

namespace zola {

constexpr int CAL_THREADS = 256;

struct CalView {
    int D, W, R, nb, ns, npar;  // npar = nzr (modes >= 3) + 5 nb
    const double* pupil;        // D x D
    const double* kx;           // D
    const double* ky;           // D
    const double* kzoil;        // D x D
    const double2* C;           // W x D
    const double* G;            // R x W
    const double* dz;           // ns
    const double* stacks;       // nb x ns x R x R
};

struct CalWork {
    double2* Q;   // D x D
    double2* S;   // D x W  (also X = C^H Ebar)
    double2* E;   // W x W  (also Ebar)
    double* I;    // W x W  (also g_I)
    double* J;    // R x W
    double* T;    // R x R
    double* aux;  // R x R
};

__host__ __device__ inline size_t cal_work_bytes(int D, int W, int R) {
    auto al = [](size_t v) { return (v + 255) / 256 * 256; };
    return al((size_t)D * D * 16) + al((size_t)D * W * 16) + al((size_t)W * W * 16) + al((size_t)W * W * 8) +
           al((size_t)R * W * 8) + al((size_t)R * R * 8) * 2;
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

// E = C Q C^T from a pupil field X (D x D); S scratch (D x W).
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

// T = G I G^T (R x R); J scratch.
__device__ void cal_blur(const CalView& V, const double* I, double* J, double* T) {
    const int W = V.W, R = V.R;
    for (int k = threadIdx.x; k < R * W; k += blockDim.x) {
        const int ip = k / W, j = k % W;
        double acc = 0;
        for (int i = 0; i < W; ++i) acc += V.G[ip * W + i] * I[i * W + j];
        J[k] = acc;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < R * R; k += blockDim.x) {
        const int ip = k / R, jp = k % R;
        double acc = 0;
        for (int j = 0; j < W; ++j) acc += V.G[jp * W + j] * J[ip * W + j];
        T[k] = acc;
    }
    __syncthreads();
}

// Forward model of one slice into w (T = blurred intensity); returns S = sum |T|.
__device__ double cal_forward(const CalView& V, const CalWork& w, const double* phase, double x, double y, double zoil,
                              double* red) {
    cal_pupil(V, w, phase, x, y, zoil);
    cal_dft(V, w.Q, w.S, w.E);
    const int W = V.W, R = V.R;
    for (int k = threadIdx.x; k < W * W; k += blockDim.x) w.I[k] = w.E[k].x * w.E[k].x + w.E[k].y * w.E[k].y;
    __syncthreads();
    cal_blur(V, w.I, w.J, w.T);
    double s = 0;
    for (int k = threadIdx.x; k < R * R; k += blockDim.x) s += fabs(w.T[k]);
    return block_reduce(s, red);
}

// mode 0: NLL only (+ model), mode 1: NLL + adjoint.  One CTA per (bead, slice).
// out_slice: per slice [nll, gA, gB]; gphi: per slice D x D phase gradient.
__global__ void __launch_bounds__(CAL_THREADS) k_calib(CalView V, const double* phase, const double* bead, int mode,
                                                        char* scratch, size_t per_cta, double* out_slice,
                                                        double* gphi, double* model) {
    __shared__ double red[CAL_THREADS / 32];
    const int bs = blockIdx.x, b = bs / V.ns, s = bs % V.ns;
    const int D = V.D, W = V.W, R = V.R, RR = R * R;
    CalWork w = cal_carve(scratch + (size_t)blockIdx.x * per_cta, D, W, R);
    const double x = bead[5 * b], y = bead[5 * b + 1], z = bead[5 * b + 2], A = bead[5 * b + 3], B = bead[5 * b + 4];
    const double Ssum = cal_forward(V, w, phase, x, y, V.dz[s] + z, red);
    const double* d = V.stacks + (size_t)bs * RR;
    double nll = 0, gA = 0, gB = 0, gpsum = 0;
    for (int k = threadIdx.x; k < RR; k += blockDim.x) {
        const double psi = fabs(w.T[k]) / Ssum;
        double mu = A * psi + B;
        if (mu <= 0) mu = 0.00000001;  // ZernikePhaseRetrieval.java:1862-1864
        nll += mu - d[k] * log(mu);
        if (model) model[(size_t)bs * RR + k] = mu;
        const double wgt = 1.0 - d[k] / mu;
        gA += wgt * psi;
        gB += wgt;
        w.aux[k] = A * wgt;  // g_psi
        gpsum += A * wgt * psi;
    }
    nll = block_reduce(nll, red);
    gA = block_reduce(gA, red);
    gB = block_reduce(gB, red);
    gpsum = block_reduce(gpsum, red);
    if (threadIdx.x == 0) {
        out_slice[3 * bs] = nll;
        out_slice[3 * bs + 1] = gA;
        out_slice[3 * bs + 2] = gB;
    }
    if (mode == 0) return;
    // g_T = sgn(T) (g_psi - sum g_psi psi) / S
    for (int k = threadIdx.x; k < RR; k += blockDim.x) {
        const double t = w.T[k];
        w.aux[k] = (t < 0 ? -1.0 : 1.0) * (w.aux[k] - gpsum) / Ssum;
    }
    __syncthreads();
    // g_I = G^T g_T G:  V1 = g_T G (R x W) into J, then g_I = G^T V1 (W x W) into I
    for (int k = threadIdx.x; k < R * W; k += blockDim.x) {
        const int ip = k / W, j = k % W;
        double acc = 0;
        for (int jp = 0; jp < R; ++jp) acc += w.aux[ip * R + jp] * V.G[jp * W + j];
        w.J[k] = acc;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < W * W; k += blockDim.x) {
        const int i = k / W, j = k % W;
        double acc = 0;
        for (int ip = 0; ip < R; ++ip) acc += V.G[ip * W + i] * w.J[ip * W + j];
        w.I[k] = acc;
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
        double2 acc = make_double2(0, 0);
        for (int i = 0; i < W; ++i) {
            const double2 c = V.C[i * D + a], e = w.E[i * W + j];  // conj(c) * e
            acc.x += c.x * e.x + c.y * e.y;
            acc.y += c.x * e.y - c.y * e.x;
        }
        w.S[k] = acc;
    }
    __syncthreads();
    double* gp = gphi + (size_t)bs * D * D;
    for (int k = threadIdx.x; k < D * D; k += blockDim.x) {
        const int a = k / D, bb = k % D;
        double g = 0;
        if (V.pupil[k] != 0) {
            double2 qb = make_double2(0, 0);
            for (int j = 0; j < W; ++j) {
                const double2 xv = w.S[a * W + j], c = V.C[j * D + bb];  // x * conj(c)
                qb.x += xv.x * c.x + xv.y * c.y;
                qb.y += xv.y * c.x - xv.x * c.y;
            }
            const double2 q = w.Q[k];  // 2 Im(conj(q) qb)
            g = 2.0 * (q.x * qb.y - q.y * qb.x);
        }
        gp[k] = g;
    }
}

// Tangent maps: d mu / d theta_t for a set of phase directions.  One CTA per
// (direction, bead, slice); dirs[t] = D x D phase direction (nullptr rows
// are skipped by the caller).  out: per (t, bs) the R x R tangent of mu.
__global__ void __launch_bounds__(CAL_THREADS) k_calib_tangent(CalView V, const double* phase, const double* bead,
                                                                const double* dirs, const int* dir_bead, int ndir,
                                                                char* scratch, size_t per_cta, double* tan) {
    __shared__ double red[CAL_THREADS / 32];
    const int t = blockIdx.x / (V.nb * V.ns), bs = blockIdx.x % (V.nb * V.ns), b = bs / V.ns, s = bs % V.ns;
    const int D = V.D, W = V.W, R = V.R, RR = R * R;
    double* out = tan + ((size_t)t * V.nb * V.ns + bs) * RR;
    if (dir_bead[t] >= 0 && dir_bead[t] != b) {  // per-bead direction: other beads do not depend on it
        for (int k = threadIdx.x; k < RR; k += blockDim.x) out[k] = 0;
        return;
    }
    CalWork w = cal_carve(scratch + (size_t)blockIdx.x * per_cta, D, W, R);
    const double x = bead[5 * b], y = bead[5 * b + 1], z = bead[5 * b + 2], A = bead[5 * b + 3];
    const double Ssum = cal_forward(V, w, phase, x, y, V.dz[s] + z, red);
    // keep E in E; tangent field dQ = i Q dphi into Q, dE = C dQ C^T into the
    // second half of S's storage is not enough: reuse Q for dQ and build dE in
    // place of E after storing dI = 2 Re(conj E dE)
    const double* dphi = dirs + (size_t)t * D * D;
    for (int k = threadIdx.x; k < D * D; k += blockDim.x) {
        const double2 q = w.Q[k];
        const double p = dphi[k];
        w.Q[k] = make_double2(-q.y * p, q.x * p);
    }
    __syncthreads();
    // dE accumulation needs E: compute dE row by row into I as dI directly
    // (first stage S = dQ C^T, then for each (i, j): dE = sum_a C[i][a] S[a][j])
    {
        const int Dd = D;
        for (int k = threadIdx.x; k < Dd * W; k += blockDim.x) {
            const int a = k / W, j = k % W;
            double2 sacc = make_double2(0, 0);
            for (int bb = 0; bb < Dd; ++bb) {
                const double2 q = w.Q[a * Dd + bb], c = V.C[j * Dd + bb];
                sacc.x += q.x * c.x - q.y * c.y;
                sacc.y += q.x * c.y + q.y * c.x;
            }
            w.S[k] = sacc;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < W * W; k += blockDim.x) {
            const int i = k / W, j = k % W;
            double2 e = make_double2(0, 0);
            for (int a = 0; a < Dd; ++a) {
                const double2 c = V.C[i * Dd + a], sv = w.S[a * W + j];
                e.x += c.x * sv.x - c.y * sv.y;
                e.y += c.x * sv.y + c.y * sv.x;
            }
            const double2 E0 = w.E[k];
            w.I[k] = 2.0 * (E0.x * e.x + E0.y * e.y);
        }
        __syncthreads();
    }
    // dT = G dI G^T into aux
    for (int k = threadIdx.x; k < R * W; k += blockDim.x) {
        const int ip = k / W, j = k % W;
        double acc = 0;
        for (int i = 0; i < W; ++i) acc += V.G[ip * W + i] * w.I[i * W + j];
        w.J[k] = acc;
    }
    __syncthreads();
    double dsum = 0;
    for (int k = threadIdx.x; k < RR; k += blockDim.x) {
        const int ip = k / R, jp = k % R;
        double acc = 0;
        for (int j = 0; j < W; ++j) acc += V.G[jp * W + j] * w.J[ip * W + j];
        const double sg = w.T[k] < 0 ? -1.0 : 1.0;
        w.aux[k] = sg * acc;
        dsum += sg * acc;
    }
    dsum = block_reduce(dsum, red);
    for (int k = threadIdx.x; k < RR; k += blockDim.x) {
        const double psi = fabs(w.T[k]) / Ssum;
        out[k] = A * (w.aux[k] - psi * dsum) / Ssum;
    }
}

// Deterministic reductions of per-slice results.
__global__ void k_calib_reduce(CalView V, const double* out_slice, const double* gphi, double* gphi_sum,
                               double* bead_grad, double* nll) {
    const int D = V.D, nbs = V.nb * V.ns;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < D * D; k += gridDim.x * blockDim.x) {
        double s = 0;
        for (int bs = 0; bs < nbs; ++bs) s += gphi[(size_t)bs * D * D + k];
        gphi_sum[k] = s;
    }
    if (blockIdx.x == 0 && threadIdx.x < V.nb) {
        const int b = threadIdx.x;
        double gx = 0, gy = 0, gz = 0, gA = 0, gB = 0;
        for (int s = 0; s < V.ns; ++s) {
            const double* gp = gphi + (size_t)(b * V.ns + s) * D * D;
            for (int k = 0; k < D * D; ++k) {
                gx += gp[k] * V.kx[k / D];
                gy += gp[k] * V.ky[k % D];
                gz -= gp[k] * V.kzoil[k];
            }
            gA += out_slice[3 * (b * V.ns + s) + 1];
            gB += out_slice[3 * (b * V.ns + s) + 2];
        }
        double* o = bead_grad + 5 * b;
        o[0] = gx; o[1] = gy; o[2] = gz; o[3] = gA; o[4] = gB;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double s = 0;
        for (int bs = 0; bs < nbs; ++bs) s += out_slice[3 * bs];
        *nll = s;
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
    double* d_Z = nullptr;
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

const CalibCache* basis(zola_psf* p, int nz, std::string& err) {
    CalibCache& c = g_cal_cache[p];
    if (c.nz == nz && c.d_Z) return &c;
    if (c.d_Z) cudaFree(c.d_Z);
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
    cudaError_t e = cudaMalloc(&c.d_Z, c.Z.size() * 8);
    if (e == cudaSuccess) e = cudaMemcpy(c.d_Z, c.Z.data(), c.Z.size() * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { err = std::string("calibration basis: ") + cudaGetErrorString(e); return nullptr; }
    return &c;
}

struct CalRun {
    CalView V{};
    size_t per_cta = 0;
    double* d_phase = nullptr;
    double* d_bead = nullptr;
    double* d_slice = nullptr;
    double* d_gphi = nullptr;
    double* d_gsum = nullptr;
    double* d_bgrad = nullptr;
    double* d_nll = nullptr;
    double* d_stacks = nullptr;
    double* d_dz = nullptr;
    char* scratch = nullptr;
    std::vector<void*> owned;
    ~CalRun() { for (void* p : owned) cudaFree(p); }
    cudaError_t alloc(void** p, size_t bytes) {
        cudaError_t e = cudaMalloc(p, bytes ? bytes : 8);
        if (e == cudaSuccess) owned.push_back(*p);
        return e;
    }
};

int cal_setup(zola_psf* p, int R, int nz, int nb, int ns, const double* dz, const double* stacks, CalRun& run,
              const CalibCache** cache) {
    zola_ctx* ctx = p->ctx;
    if (R < 4 || R % 2 || R > p->N || nz < 4 || nz > 231 || nb < 1 || ns < 1 || !dz || !stacks) {
        ctx->err = "calibration: need even R <= N, 4 <= nz <= 231, beads and slices >= 1";
        return ZOLA_E_ARG;
    }
    if (p->o.kz_reset) { ctx->err = "calibration: build the PSF with kz_reset = 0"; return ZOLA_E_ARG; }
    WindowTables* w = get_window(p, R, ctx->err);
    if (!w) return ZOLA_E_ARG;
    *cache = basis(p, nz, ctx->err);
    if (!*cache) return ZOLA_E_CUDA;
    CalView& V = run.V;
    V.D = p->D; V.W = w->W; V.R = R; V.nb = nb; V.ns = ns; V.npar = (nz - 3) + 5 * nb;
    V.pupil = p->view.pupil; V.kx = p->view.kx; V.ky = p->view.ky; V.kzoil = p->view.kzoil;
    V.C = w->d_C; V.G = w->d_G;
    const size_t RR = (size_t)R * R, DD = (size_t)p->D * p->D, nbs = (size_t)nb * ns;
    run.per_cta = cal_work_bytes(p->D, w->W, R);
    cudaError_t e = cudaSuccess;
    auto A = [&](void** q, size_t bytes) { if (e == cudaSuccess) e = run.alloc(q, bytes); };
    A((void**)&run.d_phase, DD * 8); A((void**)&run.d_bead, (size_t)nb * 40); A((void**)&run.d_slice, nbs * 24);
    A((void**)&run.d_gphi, nbs * DD * 8); A((void**)&run.d_gsum, DD * 8); A((void**)&run.d_bgrad, (size_t)nb * 40);
    A((void**)&run.d_nll, 8); A((void**)&run.d_stacks, nbs * RR * 8); A((void**)&run.d_dz, (size_t)ns * 8);
    A((void**)&run.scratch, nbs * run.per_cta);
    if (e == cudaSuccess) e = cudaMemcpy(run.d_stacks, stacks, nbs * RR * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(run.d_dz, dz, (size_t)ns * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { ctx->err = std::string("calibration: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
    V.dz = run.d_dz;
    V.stacks = run.d_stacks;
    return ZOLA_OK;
}

// phase = sum_{i >= 3} a_i Z_i on the host (D x D), uploaded.
int cal_phase(zola_psf* p, const CalibCache* c, const double* zern_coef, CalRun& run) {
    const int D = p->D;
    std::vector<double> ph((size_t)D * D, 0.0);
    for (int i = 3; i < c->nz; ++i) {
        const double a = zern_coef[i];
        if (a == 0) continue;
        const double* Zi = c->Z.data() + (size_t)i * D * D;
        for (size_t k = 0; k < ph.size(); ++k) ph[k] += a * Zi[k];
    }
    return cudaMemcpy(run.d_phase, ph.data(), ph.size() * 8, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : ZOLA_E_CUDA;
}

int cal_eval(zola_psf* p, const CalibCache* c, CalRun& run, const double* zern_coef, const double* bead, int mode,
             double* nll, double* gz, double* gb, double* model_dev) {
    zola_ctx* ctx = p->ctx;
    if (cal_phase(p, c, zern_coef, run)) { ctx->err = "calibration: phase upload failed"; return ZOLA_E_CUDA; }
    if (cudaMemcpy(run.d_bead, bead, (size_t)run.V.nb * 40, cudaMemcpyHostToDevice) != cudaSuccess) return ZOLA_E_CUDA;
    const int nbs = run.V.nb * run.V.ns;
    k_calib<<<nbs, CAL_THREADS>>>(run.V, run.d_phase, run.d_bead, mode, run.scratch, run.per_cta, run.d_slice,
                                  run.d_gphi, model_dev);
    k_calib_reduce<<<64, 256>>>(run.V, run.d_slice, run.d_gphi, run.d_gsum, run.d_bgrad, run.d_nll);
    ctx->launches += 2;
    cudaError_t e = cudaMemcpy(nll, run.d_nll, 8, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { ctx->err = std::string("calibration: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
    if (mode == 1) {
        const int D = p->D;
        std::vector<double> gsum((size_t)D * D);
        e = cudaMemcpy(gsum.data(), run.d_gsum, gsum.size() * 8, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(gb, run.d_bgrad, (size_t)run.V.nb * 40, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { ctx->err = std::string("calibration: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
        for (int i = 0; i < c->nz; ++i) {
            double s = 0;
            if (i >= 3) {
                const double* Zi = c->Z.data() + (size_t)i * D * D;
                for (size_t k = 0; k < gsum.size(); ++k) s += gsum[k] * Zi[k];
            }
            gz[i] = s;
        }
    }
    return ZOLA_OK;
}

}  // namespace

extern "C" {

int zola_calib_forward(zola_psf* psf, int R, int nz, const double* zernike, int nbead, int nslice, const double* dz,
                       const double* bead, const double* stacks, double* nll, double* model) {
    if (!psf || !zernike || !bead || !nll) return ZOLA_E_ARG;
    CalRun run;
    const CalibCache* c = nullptr;
    int rc = cal_setup(psf, R, nz, nbead, nslice, dz, stacks, run, &c);
    if (rc) return rc;
    double* d_model = nullptr;
    const size_t nm = (size_t)nbead * nslice * R * R;
    if (model && run.alloc((void**)&d_model, nm * 8) != cudaSuccess) return ZOLA_E_CUDA;
    rc = cal_eval(psf, c, run, zernike, bead, 0, nll, nullptr, nullptr, d_model);
    if (rc) return rc;
    if (model && cudaMemcpy(model, d_model, nm * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return ZOLA_E_CUDA;
    return ZOLA_OK;
}

int zola_calib_backward(zola_psf* psf, int R, int nz, const double* zernike, int nbead, int nslice, const double* dz,
                        const double* bead, const double* stacks, double* nll, double* grad_zernike,
                        double* grad_bead) {
    if (!psf || !zernike || !bead || !nll || !grad_zernike || !grad_bead) return ZOLA_E_ARG;
    CalRun run;
    const CalibCache* c = nullptr;
    int rc = cal_setup(psf, R, nz, nbead, nslice, dz, stacks, run, &c);
    if (rc) return rc;
    return cal_eval(psf, c, run, zernike, bead, 1, nll, grad_zernike, grad_bead, nullptr);
}

// LM over theta = (a_3..a_{nz-1}, per bead x, y, z, A, B): gradient from the
// adjoint, Gauss-Newton matrix sum J^T J / mu from forward tangents, FP64
// damped solve, accept if the NLL drops (as lm.h).  zernike / bead are updated
// in place; returns the final NLL and the number of iterations.
int zola_calib_fit(zola_psf* psf, int R, int nz, double* zernike, int nbead, int nslice, const double* dz,
                   double* bead, const double* stacks, int max_iter, double* nll_out, int* iters_out) {
    if (!psf || !zernike || !bead || !nll_out) return ZOLA_E_ARG;
    zola_ctx* ctx = psf->ctx;
    CalRun run;
    const CalibCache* c = nullptr;
    int rc = cal_setup(psf, R, nz, nbead, nslice, dz, stacks, run, &c);
    if (rc) return rc;
    const int D = psf->D, nzr = nz - 3, npar = nzr + 5 * nbead, RR = R * R, nbs = nbead * nslice;
    // tangent directions: Zernike modes (all beads) and x, y, z per bead
    const int ndir = nzr + 3 * nbead;
    std::vector<double> dirs((size_t)ndir * D * D, 0.0);
    std::vector<int> dir_bead(ndir, -1);
    for (int i = 0; i < nzr; ++i)
        std::memcpy(&dirs[(size_t)i * D * D], c->Z.data() + (size_t)(i + 3) * D * D, (size_t)D * D * 8);
    for (int b = 0; b < nbead; ++b)
        for (int q = 0; q < 3; ++q) {
            const int t = nzr + 3 * b + q;
            dir_bead[t] = b;
            for (int a = 0; a < D; ++a)
                for (int bb = 0; bb < D; ++bb) {
                    const size_t k = (size_t)a * D + bb;
                    if (psf->pupil[k] == 0) continue;
                    dirs[(size_t)t * D * D + k] = q == 0 ? psf->kx[a] : (q == 1 ? psf->ky[bb] : -psf->kzoil[k]);
                }
        }
    double *d_dirs = nullptr, *d_tan = nullptr, *d_model = nullptr;
    int* d_db = nullptr;
    char* tscratch = nullptr;
    const size_t tblocks = (size_t)ndir * nbs;
    if (run.alloc((void**)&d_dirs, dirs.size() * 8) || run.alloc((void**)&d_db, (size_t)ndir * 4) ||
        run.alloc((void**)&d_tan, tblocks * RR * 8) || run.alloc((void**)&d_model, (size_t)nbs * RR * 8) ||
        run.alloc((void**)&tscratch, tblocks * run.per_cta)) {
        ctx->err = "zola_calib_fit: device memory";
        return ZOLA_E_CUDA;
    }
    cudaMemcpy(d_dirs, dirs.data(), dirs.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_db, dir_bead.data(), (size_t)ndir * 4, cudaMemcpyHostToDevice);
    std::vector<double> th(npar), gz(nz), gb(5 * nbead), g(npar), tanh_((size_t)ndir * nbs * RR),
        mu((size_t)nbs * RR), psi((size_t)nbs * RR);
    auto pack = [&](std::vector<double>& t) {
        for (int i = 0; i < nzr; ++i) t[i] = zernike[i + 3];
        for (int k = 0; k < 5 * nbead; ++k) t[nzr + k] = bead[k];
    };
    auto unpack = [&](const std::vector<double>& t, std::vector<double>& zc, std::vector<double>& bd) {
        zc.assign(zernike, zernike + nz);
        for (int i = 0; i < nzr; ++i) zc[i + 3] = t[i];
        bd.assign(t.begin() + nzr, t.end());
    };
    pack(th);
    std::vector<double> zc, bd;
    double nll = 0, lambda = 1e-3;
    int it = 0;
    auto gradient = [&](const std::vector<double>& t, double* f, std::vector<double>& grad, bool with_tangents,
                        std::vector<double>& H) -> int {
        unpack(t, zc, bd);
        int r = cal_eval(psf, c, run, zc.data(), bd.data(), 1, f, gz.data(), gb.data(), d_model);
        if (r) return r;
        for (int i = 0; i < nzr; ++i) grad[i] = gz[i + 3];
        for (int k = 0; k < 5 * nbead; ++k) grad[nzr + k] = gb[k];
        if (!with_tangents) return 0;
        k_calib_tangent<<<(unsigned)tblocks, CAL_THREADS>>>(run.V, run.d_phase, run.d_bead, d_dirs, d_db, ndir, tscratch,
                                                            run.per_cta, d_tan);
        ctx->launches++;
        if (cudaMemcpy(tanh_.data(), d_tan, tanh_.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(mu.data(), d_model, mu.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
            return ZOLA_E_CUDA;
        // Gauss-Newton matrix sum_p J_p J_p^T / mu_p (Fisher form)
        H.assign((size_t)npar * npar, 0.0);
        for (int bs = 0; bs < nbs; ++bs) {
            const int b = bs / nslice;
            const double A = bd[5 * b + 3], B = bd[5 * b + 4];
            for (int k = 0; k < RR; ++k) {
                const size_t pix = (size_t)bs * RR + k;
                const double m = mu[pix], ps = (m - B) / A;
                double jv[512];
                int idx[512], nj = 0;
                for (int i = 0; i < nzr; ++i) { jv[nj] = tanh_[((size_t)i * nbs) * RR + pix]; idx[nj++] = i; }
                for (int q = 0; q < 3; ++q) {
                    const int t2 = nzr + 3 * b + q;
                    jv[nj] = tanh_[((size_t)t2 * nbs) * RR + pix];
                    idx[nj++] = nzr + 5 * b + q;
                }
                jv[nj] = ps; idx[nj++] = nzr + 5 * b + 3;
                jv[nj] = 1.0; idx[nj++] = nzr + 5 * b + 4;
                for (int u = 0; u < nj; ++u)
                    for (int v = 0; v <= u; ++v) H[(size_t)idx[u] * npar + idx[v]] += jv[u] * jv[v] / m;
            }
        }
        for (int u = 0; u < npar; ++u)
            for (int v = 0; v < u; ++v) H[(size_t)v * npar + u] = H[(size_t)u * npar + v];
        return 0;
    };
    std::vector<double> H, Hn;
    rc = gradient(th, &nll, g, true, H);
    if (rc) return rc;
    for (it = 0; it < max_iter; ++it) {
        // damped Cholesky solve (npar x npar)
        std::vector<double> L((size_t)npar * npar), step(npar), y(npar);
        bool ok = true;
        for (int i = 0; i < npar && ok; ++i)
            for (int j = 0; j <= i; ++j) {
                double s = H[(size_t)i * npar + j] + (i == j ? lambda * std::max(H[(size_t)i * npar + i], 1e-12) : 0.0);
                for (int k = 0; k < j; ++k) s -= L[(size_t)i * npar + k] * L[(size_t)j * npar + k];
                if (i == j) {
                    if (!(s > 0)) { ok = false; break; }
                    L[(size_t)i * npar + i] = std::sqrt(s);
                } else L[(size_t)i * npar + j] = s / L[(size_t)j * npar + j];
            }
        if (!ok) { lambda *= 10; if (lambda > 1e10) break; continue; }
        for (int i = 0; i < npar; ++i) {
            double s = -g[i];
            for (int k = 0; k < i; ++k) s -= L[(size_t)i * npar + k] * y[k];
            y[i] = s / L[(size_t)i * npar + i];
        }
        for (int i = npar - 1; i >= 0; --i) {
            double s = y[i];
            for (int k = i + 1; k < npar; ++k) s -= L[(size_t)k * npar + i] * step[k];
            step[i] = s / L[(size_t)i * npar + i];
        }
        std::vector<double> t2(th), g2(npar);
        for (int i = 0; i < npar; ++i) t2[i] += step[i];
        for (int b = 0; b < nbead; ++b) {
            t2[nzr + 5 * b + 3] = std::max(t2[nzr + 5 * b + 3], 1.0);
            t2[nzr + 5 * b + 4] = std::max(t2[nzr + 5 * b + 4], 0.01);
        }
        double nll2;
        rc = gradient(t2, &nll2, g2, false, Hn);
        if (rc) return rc;
        if (nll2 <= nll) {
            const double dec = nll - nll2;
            th = t2;
            nll = nll2;
            lambda = std::max(lambda * 0.1, 1e-9);
            rc = gradient(th, &nll, g, true, H);
            if (rc) return rc;
            if (dec < 1e-9 * std::max(1.0, std::fabs(nll))) { ++it; break; }
        } else {
            lambda *= 10;
            if (lambda > 1e10) break;
        }
    }
    unpack(th, zc, bd);
    std::memcpy(zernike, zc.data(), (size_t)nz * 8);
    std::memcpy(bead, bd.data(), (size_t)5 * nbead * 8);
    *nll_out = nll;
    if (iters_out) *iters_out = it;
    return ZOLA_OK;
}

}  // extern "C"
