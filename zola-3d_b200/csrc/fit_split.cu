// Split-precision Poisson MLE fit on the sm_100a tensor cores (tcgen05).
//
// The model of process/cpu/PSFPhase.java:557-629 is evaluated for a pool of
// ROI "slots" as four batched tensor-core contractions per Levenberg-Marquardt
// evaluation, each a tcgen05.mma chain from shared memory into TMEM:
//
//   stage 1  S  = Q  C^T  (+ Sy = Q CK^T, Sz = Qz C^T)   rows (roi, a)   K = 2DP
//   stage 2  E^T = S^T C^T (+ Ex, Ey, Ez)                rows (roi, j)   K = 2DP
//            epilogue: I = |E|^2, I_t = 2 Re(conj(E) E_t)
//   stage 3  J^T = I G^T  (blur along the first image index)  rows (roi, j)  K = W
//   stage 4  T^T = G J^T  (blur along the second index, transposed so that a
//            TMEM lane holds one pixel column of all four maps)    K = W
//   stage 5  likelihood, gradient, Gauss-Newton Hessian and Fisher sums in
//            FP32 with Kahan compensation, then the FP64 5x5 LM solve, damping
//            and convergence test; converged slots are retired and refilled
//            from the ROI queue (a device counter).  Stages 4 and 5 run in one
//            kernel.
//
// C is the W x D partial-DFT matrix, CK = C diag(i k) its x/y derivative, Q the
// pupil field (built from the pupil tables and the slot's trial x, y, z), G
// the R x W circular-blur matrix (see optics.cpp).  Complex products are real
// GEMMs on [re | im] operands.  Every operand that sets the likelihood value
// (Q, S, E, I, J of the model itself, and the constants C, G) is an FP16 hi +
// lo pair and multiplied with three products (hi*hi + hi*lo + lo*hi, FP32
// accumulation): about 2^-22 relative.  The derivative maps only enter the
// gradient and the Hessian; their operands are single FP16 products, whose
// rounding moves the optimum by about 2^-11 x CRLB (~0.01 nm), far below the
// 0.5 nm budget.
//
// Every stage is a persistent body that walks "units" of slots (whole stage-1
// and window tiles).  ZOLA_SPLIT_STAGED launches the four bodies (pupil DFT,
// window DFT, row blur, column blur + sums + LM step) as four kernels per LM
// round over the whole pool.  ZOLA_SPLIT_FLOW launches them once, together, as
// one cooperative kernel (k_flow): each stage runs on its own CTAs, a unit
// moves to the next stage as soon as it is done (a state word per unit, one
// scheduler thread per CTA), its operands pass between stages through global
// memory while they are still in L2, and converged fits retire and refill from
// the ROI queue on the device.  Stages 1 and 2 keep the DFT constants in shared
// memory and issue N = 256 MMAs.  All operands use the canonical no-swizzle
// layouts of umma.h.  Intermediate operands travel through global slabs laid
// out as the shared-memory tiles (or K-slabs of them), fetched with 1-D bulk
// (TMA) copies.  Scales are powers of two chosen from host-side bounds so no
// FP16 value overflows; they are exact and undone in FP32.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "lm.h"
#include "umma.h"
#include "zola_internal.h"

namespace zola {

using umma::kmajor_off;
using umma::mnmajor_off;

// Stages 1-4 run 512 threads: four warpgroups share the 128 TMEM lanes (lane
// quadrant = warp % 4, so thread t owns tile row t % 128) and split the column
// work of every epilogue and of the Q build; the LM step runs one thread per slot.
constexpr int SPLIT_THREADS = 512;

// ---------------------------------------------------------------- plan ------
struct SplitScales {
    float q, qz;                 // Q, Qz operand scales
    float c2, c2y, c2z;          // TMEM(S) -> A2 operand factors
    float cI, cIx, cIy, cIz;     // TMEM(E products) -> A3 operand factors
    float cJ[4];                 // TMEM(J) -> A4 operand factors
    float cT[4];                 // TMEM(T) -> true blurred maps
};

struct SplitDev {
    // geometry
    int R, W, D, DP, K1, RP, G1, G2, NT4, P;
    int a0, N;
    double zfocus;
    // constant operands
    const __half* bc2_hi; // NCH2 chunks of 4*16 x K1 (fused kernel)
    const __half* bc2_lo; // NCH2 chunks of 2*16 x K1
    int NCH2;
    const __half* bcs;    // K1/16 K-slabs of 6W x 16 (wide stage kernels)
    const __half* gt_hi;  // RP x W (K-major)
    const __half* gt_lo;
    const __half* g128_hi;  // 128 x W (K-major, rows >= R zero): the column-blur A operand
    const __half* g128_lo;
    // pupil tables padded to DP x DP (row a <-> kx, column b <-> ky; zero
    // beyond the D disk rows and columns), in the warp-load order of stage 1
    const float* pupf;     // pupil (the model uses it in FP32)
    const double* phase0;  // phase - kzoil * zfocus
    const double* kz;
    const double* kx;      // DP
    const double* ky;      // DP
    // pool slabs
    char* a2;      // P/G2 tiles x 4 arrays x 128 x K1 f16
    char* a3;      // P/G2 tiles x 5 arrays x 128 x W f16
    char* a4;      // P x NT4 tiles x 2 arrays x 128 x W f16
    float* tmaps;  // P x 4 x R x R (model-only evaluation)
    double* sums;  // P x NSUM likelihood sums (fit)
    // slot state
    int* slot_roi;
    int* slot_phase;
    LMState* lm;
    int* queue;    // next ROI to hand out
    int* active;   // occupied slots
    int* err;      // bounded-wait timeout flag
    int* navail;   // ROIs [0, *navail) are on the device (all n unless the inputs are still arriving)
    int* ustate;   // per unit of slots: 5 e + s (ready for stage s of evaluation e), or UNIT_DEAD
    long long wait_limit;  // clocks a dataflow scheduler waits for a ready unit before it gives up
    unsigned long long* evals;  // dataflow kernel: model evaluations (LM steps) done
    unsigned long long* clk;    // dataflow kernel: per CTA, clocks without a ready unit, clocks in all, units done
    SplitScales sc;
};

struct SplitPlanHost {
    int R = 0, W = 0, D = 0, DP = 0, K1 = 0, RP = 0, G1 = 0, G2 = 0, NT4 = 0;
    int IC2 = 16, NCH2 = 0;  // fused stage 2-5 kernel: 16-wide i-chunks
    SplitScales sc{};
    __half* d_bc2_hi = nullptr;
    __half* d_bc2_lo = nullptr;
    __half* d_bcs = nullptr;
    __half* d_gt_hi = nullptr;
    __half* d_gt_lo = nullptr;
    __half* d_g128_hi = nullptr;
    __half* d_g128_lo = nullptr;
    double* d_phase0 = nullptr;  // DP x DP
    double* d_kz = nullptr;      // DP x DP
    float* d_pupf = nullptr;     // DP x DP
    double* d_kx = nullptr;      // DP
    double* d_ky = nullptr;      // DP
};

static double pow2scale(double bound) {
    if (!(bound > 0)) return 1.0;
    return std::ldexp(1.0, (int)std::floor(std::log2(16384.0 / bound)));
}

// A2 arrays of a stage-2 tile: S hi, S lo, S_y, S_z
__host__ __device__ inline size_t a2_tile_bytes(int K1) { return (size_t)4 * 128 * K1 * 2; }
__host__ __device__ inline size_t a3_tile_bytes(int W) { return (size_t)5 * 128 * W * 2; }
__host__ __device__ inline size_t a4_tile_bytes(int W) { return (size_t)2 * 128 * W * 2; }
// Row-blurred maps J of one slot as the column-blur B operand: hi then lo, each
// MN-major with N = 4 RP rows n = (map, i') and K = W columns j.
__host__ __device__ inline size_t a4_slot_bytes(int W, int RP) { return (size_t)2 * 4 * RP * W * 2; }
// K order of every operand along a pupil DFT (stage 1: column b, stage 2: row
// a, each with its real and imaginary part): k = 16 (b / 8) + 8 [imaginary] +
// b % 8, so that one 16-wide K step holds both parts of 8 consecutive indices.
__host__ __device__ inline int kperm(int b, bool im) { return 16 * (b >> 3) + (im ? 8 : 0) + (b & 7); }
// the natural K index (real parts 0..DP-1, then imaginary parts) of position kp
__host__ __device__ inline int knat(int kp, int DP) { return ((kp & 8) ? DP : 0) + 8 * (kp >> 4) + (kp & 7); }
// Row stride (floats) of the fused kernel's shared-memory maps: a multiple of 4
// congruent to 4 mod 32, so that 32 lanes storing float4 at consecutive rows
// cover all banks once per 8 lanes.
__host__ __device__ inline int tm_stride(int R) {
    const int s = (R + 3) & ~3;
    return s + (4 - s % 32 + 32) % 32;
}

// Build (once per PSF and ROI size) the constant operands and scales.
static SplitPlanHost* get_plan(zola_psf* p, WindowTables* w, std::string& err) {
    if (w->d_split) return (SplitPlanHost*)w->d_split;
    SplitPlanHost* pl = new SplitPlanHost();
    const int D = p->D, W = w->W, R = w->R;
    pl->R = R; pl->W = W; pl->D = D;
    pl->DP = D <= 32 ? 32 : 64;
    pl->K1 = 2 * pl->DP;
    pl->RP = (R + 15) / 16 * 16;
    pl->G1 = 128 / pl->DP;
    pl->G2 = 128 / W;
    pl->NT4 = (4 * pl->RP + 127) / 128;
    const int DP = pl->DP, K1 = pl->K1, RP = pl->RP;

    // bounds
    double pmax = 0, kmax = 0, kzmax = 0;
    for (size_t i = 0; i < p->pupil.size(); ++i) {
        pmax = std::max(pmax, std::fabs(p->pupil[i]));
        if (p->pupil[i] != 0) kzmax = std::max(kzmax, std::fabs(p->kz[i]));
    }
    for (int a = 0; a < D; ++a) kmax = std::max(kmax, std::fabs(p->kx[a]));
    double sum_pupil = 0;
    for (double v : p->pupil) sum_pupil += std::fabs(v);
    const double sQ = pow2scale(pmax), sQz = pow2scale(pmax * kzmax), sB = pow2scale(std::max(1.0, kmax));
    const double bS = D * pmax, bSy = bS * kmax, bSz = bS * kzmax;
    const double s2 = pow2scale(bS), s2y = pow2scale(bSy), s2z = pow2scale(bSz);
    const double bE = sum_pupil, bI = bE * bE, bIx = 2 * bE * bE * kmax, bIz = 2 * bE * bE * kzmax;
    const double sI = pow2scale(bI), sIx = pow2scale(bIx), sIz = pow2scale(bIz);
    double gmax = 0, gsum = 0;
    for (int ip = 0; ip < R; ++ip) {
        double s = 0;
        for (int i = 0; i < W; ++i) { gmax = std::max(gmax, std::fabs(w->G[(size_t)ip * W + i])); s += std::fabs(w->G[(size_t)ip * W + i]); }
        gsum = std::max(gsum, s);
    }
    const double sG = pow2scale(gmax);
    const double sImap[4] = {sI, sIx, sIx, sIz};
    const double bImap[4] = {bI, bIx, bIx, bIz};
    SplitScales& sc = pl->sc;
    sc.q = (float)sQ; sc.qz = (float)sQz;
    sc.c2 = (float)(s2 / (sQ * sB)); sc.c2y = (float)(s2y / (sQ * sB)); sc.c2z = (float)(s2z / (sQz * sB));
    sc.cI = (float)(sI / ((s2 * sB) * (s2 * sB)));
    sc.cIx = (float)(2 * sIx / ((s2 * sB) * (s2 * sB)));
    sc.cIy = (float)(2 * sIx / ((s2 * sB) * (s2y * sB)));
    sc.cIz = (float)(2 * sIz / ((s2 * sB) * (s2z * sB)));
    for (int m = 0; m < 4; ++m) {
        double sJ = pow2scale(gsum * bImap[m]);
        sc.cJ[m] = (float)(sJ / (sImap[m] * sG));
        sc.cT[m] = (float)(1.0 / (sJ * sG));
    }

    // DFT constant rows, four parts per output index i:
    // part 0: [Re C ; -Im C], 1: [Im C ; Re C], 2: [Re CK ; -Im CK], 3: [Im CK ; Re CK]
    // with data columns k < DP (natural order) multiplying the real and k >= DP
    // the imaginary part of the data; CK[i][b] = C[i][b] * (i k_b).  The packs
    // below place column k at its kperm position.
    auto C = [&](int i, int b, double& re, double& im) {
        re = w->C[((size_t)i * D + b) * 2];
        im = w->C[((size_t)i * D + b) * 2 + 1];
    };
    // scaled constant of part `part` at output index i and data column k (0 beyond the disk)
    auto bc_value = [&](int part, int i, int k) {
        const int b = k < DP ? k : k - DP;
        if (b >= D) return 0.0;
        double cr, ci;
        C(i, b, cr, ci);
        const double kb = p->ky[b];
        const double ckr = -kb * ci, cki = kb * cr;
        const bool re_in = k < DP;
        double v;
        switch (part) {
            case 0: v = re_in ? cr : -ci; break;
            case 1: v = re_in ? ci : cr; break;
            case 2: v = re_in ? ckr : -cki; break;
            default: v = re_in ? cki : ckr; break;
        }
        return v * sB;
    };
    auto split_h = [](double v, __half& hi, __half& lo) {
        hi = __float2half_rn((float)v);
        lo = __float2half_rn((float)(v - (double)__half2float(hi)));
    };
    auto pack_bc = [&](int icw, std::vector<__half>& bh, std::vector<__half>& bl) {
        const int nch = W / icw;
        bh.assign((size_t)nch * 4 * icw * K1, __float2half(0.f));
        bl.assign((size_t)nch * 2 * icw * K1, __float2half(0.f));
        for (int c = 0; c < nch; ++c)
            for (int part = 0; part < 4; ++part)
                for (int ii = 0; ii < icw; ++ii) {
                    int i = c * icw + ii, n = part * icw + ii;
                    for (int k = 0; k < K1; ++k) {
                        __half hi, lo;
                        split_h(bc_value(part, i, k), hi, lo);
                        const int kp = kperm(k < DP ? k : k - DP, k >= DP);
                        bh[(size_t)c * 4 * icw * K1 + kmajor_off(n, kp, K1) / 2] = hi;
                        if (part < 2) bl[(size_t)c * 2 * icw * K1 + kmajor_off(n, kp, K1) / 2] = lo;
                    }
                }
    };
    // K-slabs of the wide stage kernels: for K step s (positions 16s .. 16s + 15 of the K order above),
    // rows n = q * W + i with q = 0..3 the hi values of parts 0..3 and q = 4, 5
    // the lo values of parts 0, 1; K-major with K = 16 (6W x 32 bytes a slab).
    std::vector<__half> bs((size_t)(K1 / 16) * 6 * W * 16, __float2half(0.f));
    for (int st = 0; st < K1 / 16; ++st)
        for (int q = 0; q < 6; ++q)
            for (int i = 0; i < W; ++i)
                for (int kk = 0; kk < 16; ++kk) {
                    __half hi, lo;
                    split_h(bc_value(q < 4 ? q : q - 4, i, knat(16 * st + kk, DP)), hi, lo);
                    bs[(size_t)st * 6 * W * 16 + kmajor_off(q * W + i, kk, 16) / 2] = q < 4 ? hi : lo;
                }
    std::vector<__half> bh2, bl2;
    pl->IC2 = W < 16 ? W : 16;
    pl->NCH2 = W / pl->IC2;
    pack_bc(pl->IC2, bh2, bl2);
    // G^T operand: rows n = i' (< RP, zero beyond R), K = W.
    std::vector<__half> gh((size_t)RP * W, __float2half(0.f)), gl((size_t)RP * W, __float2half(0.f));
    for (int ip = 0; ip < R; ++ip)
        for (int i = 0; i < W; ++i) {
            double v = w->G[(size_t)ip * W + i] * sG;
            __half hi = __float2half_rn((float)v);
            __half lo = __float2half_rn((float)(v - (double)__half2float(hi)));
            gh[kmajor_off(ip, i, W) / 2] = hi;
            gl[kmajor_off(ip, i, W) / 2] = lo;
        }
    std::vector<__half> g1h((size_t)128 * W, __float2half(0.f)), g1l((size_t)128 * W, __float2half(0.f));
    for (int ip = 0; ip < R; ++ip)
        for (int i = 0; i < W; ++i) {
            g1h[kmajor_off(ip, i, W) / 2] = gh[kmajor_off(ip, i, W) / 2];
            g1l[kmajor_off(ip, i, W) / 2] = gl[kmajor_off(ip, i, W) / 2];
        }
    // phase0 = phase - kzoil * zfocus (the zoil term of PSFPhase.java:560 with zoil = Zfocus),
    // padded to DP x DP with the other pupil tables
    std::vector<double> ph0((size_t)DP * DP, 0.0), kzp((size_t)DP * DP, 0.0), kxp(DP, 0.0), kyp(DP, 0.0);
    std::vector<float> pupf((size_t)DP * DP, 0.f);
    // Order of the DP x DP tables: [b / 8][(b % 8) / 2][a][b % 2] for phase0 and kz
    // (double pairs), [b / 8][(b % 8) / 4][a][b % 4] for the pupil (float quads), so
    // that 32 consecutive rows a of one column group are one contiguous warp load.
    for (int a = 0; a < D; ++a) {
        kxp[a] = p->kx[a];
        kyp[a] = p->ky[a];
        for (int b = 0; b < D; ++b) {
            const size_t i = (size_t)a * D + b;
            const size_t o2 = (((size_t)(b / 8) * 4 + (b % 8) / 2) * DP + a) * 2 + b % 2;
            const size_t o4 = (((size_t)(b / 8) * 2 + (b % 8) / 4) * DP + a) * 4 + b % 4;
            ph0[o2] = p->phase[i] - p->kzoil[i] * p->o.zfocus;
            kzp[o2] = p->kz[i];
            pupf[o4] = (float)p->pupil[i];
        }
    }

    cudaError_t e = cudaSuccess;
    auto up = [&](void** dst, const void* src, size_t bytes) {
        if (e != cudaSuccess) return;
        e = cudaMalloc(dst, bytes);
        if (e == cudaSuccess) e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    };
    up((void**)&pl->d_bc2_hi, bh2.data(), bh2.size() * 2);
    up((void**)&pl->d_bc2_lo, bl2.data(), bl2.size() * 2);
    up((void**)&pl->d_bcs, bs.data(), bs.size() * 2);
    up((void**)&pl->d_gt_hi, gh.data(), gh.size() * 2);
    up((void**)&pl->d_gt_lo, gl.data(), gl.size() * 2);
    up((void**)&pl->d_g128_hi, g1h.data(), g1h.size() * 2);
    up((void**)&pl->d_g128_lo, g1l.data(), g1l.size() * 2);
    up((void**)&pl->d_phase0, ph0.data(), ph0.size() * 8);
    up((void**)&pl->d_kz, kzp.data(), kzp.size() * 8);
    up((void**)&pl->d_pupf, pupf.data(), pupf.size() * 4);
    up((void**)&pl->d_kx, kxp.data(), kxp.size() * 8);
    up((void**)&pl->d_ky, kyp.data(), kyp.size() * 8);
    if (e != cudaSuccess) {
        err = std::string("split plan upload: ") + cudaGetErrorString(e);
        delete pl;
        return nullptr;
    }
    w->d_split = pl;
    return pl;
}

void free_split_plan(void* plan) {
    SplitPlanHost* pl = (SplitPlanHost*)plan;
    if (!pl) return;
    cudaFree(pl->d_bc2_hi);
    cudaFree(pl->d_bc2_lo);
    cudaFree(pl->d_bcs);
    cudaFree(pl->d_gt_hi);
    cudaFree(pl->d_gt_lo);
    cudaFree(pl->d_g128_hi);
    cudaFree(pl->d_g128_lo);
    cudaFree(pl->d_phase0);
    cudaFree(pl->d_kz);
    cudaFree(pl->d_pupf);
    cudaFree(pl->d_kx);
    cudaFree(pl->d_ky);
    delete pl;
}

// ------------------------------------------------------------- helpers -----
__device__ __forceinline__ uint32_t tmem_lane_addr(uint32_t base, int col) {
    const int quad = (threadIdx.x >> 5) & 3;
    return base + ((uint32_t)(quad * 32) << 16) + (uint32_t)col;
}

// N groups of 8 TMEM columns of this thread's lane, all loads in flight before
// one wait; the empty asm after the wait keeps every use of a loaded register
// behind it.
template <int N>
__device__ __forceinline__ void tmem_ld8_multi(const uint32_t (&addr)[N], float (&v)[N][8]) {
    uint32_t r[N][8];
#pragma unroll
    for (int i = 0; i < N; ++i) umma::tmem_ld8_nw(addr[i], r[i]);
    umma::tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            asm volatile("" : "+r"(r[i][j]));
            v[i][j] = __uint_as_float(r[i][j]);
        }
}

__device__ __forceinline__ void store8h(void* dst, const __half* v) {
    uint4 u;
    u.x = (uint32_t)__half_as_ushort(v[0]) | ((uint32_t)__half_as_ushort(v[1]) << 16);
    u.y = (uint32_t)__half_as_ushort(v[2]) | ((uint32_t)__half_as_ushort(v[3]) << 16);
    u.z = (uint32_t)__half_as_ushort(v[4]) | ((uint32_t)__half_as_ushort(v[5]) << 16);
    u.w = (uint32_t)__half_as_ushort(v[6]) | ((uint32_t)__half_as_ushort(v[7]) << 16);
    *(uint4*)dst = u;
}

// Two floats rounded to a packed f16 pair (a in the low half).
__device__ __forceinline__ uint32_t pack_h2(float a, float b) {
    union { __half2 h; uint32_t u; } cv;
    cv.h = __floats2half2_rn(a, b);
    return cv.u;
}

// hi + lo f16 split of two floats, as packed pairs (the same values as
// umma::split_f16 on each, with one conversion instruction per pair).
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    union { __half2 h; uint32_t u; } h, l;
    h.h = __floats2half2_rn(a, b);
    const float2 f = __half22float2(h.h);
    l.h = __floats2half2_rn(a - f.x, b - f.y);
    hi = h.u;
    lo = l.u;
}

__device__ __forceinline__ void store4w(void* dst, const uint32_t* w) { *(uint4*)dst = make_uint4(w[0], w[1], w[2], w[3]); }

// sin and cos of an FP64 phase.  The phase is reduced in FP64 by the nearest
// multiple q of pi/2 (pi/2 as a two-double sum, so r = ph - q pi/2 keeps FP64
// accuracy for any phase the model produces); r in [-pi/4, pi/4] is rounded
// to FP32 and sin r, cos r come from their Taylor polynomials of degree 9 and
// 10 (truncation below 2e-9 on that interval, under the FP32 rounding of the
// result), rotated by the quadrant q mod 4.
__device__ __forceinline__ void sincos_phase(double ph, float& s, float& c) {
    const double q = rint(ph * 0.6366197723675814);
    double r = fma(-q, 1.5707963267948966, ph);
    r = fma(-q, 6.123233995736766e-17, r);
    const float x = (float)r, x2 = x * x;
    const float sp = fmaf(x * x2, -1.f / 6 + x2 * (1.f / 120 + x2 * (-1.f / 5040 + x2 * (1.f / 362880))), x);
    const float cp = 1.f + x2 * (-0.5f + x2 * (1.f / 24 + x2 * (-1.f / 720 + x2 * (1.f / 40320 + x2 * (-1.f / 3628800)))));
    const int k = (int)q & 3;
    const float ss = (k & 1) ? cp : sp, cc = (k & 1) ? sp : cp;
    s = (k & 2) ? -ss : ss;
    c = ((k + 1) & 2) ? -cc : cc;
}

// Issue an MMA chain over K (in steps of 16) for one accumulator.
__device__ __forceinline__ void mma_chain(uint32_t tmem_d, uint32_t a_addr, uint32_t a_lbo, uint32_t a_sbo,
                                          uint32_t a_kstep, uint32_t b_addr, uint32_t b_lbo, uint32_t b_sbo,
                                          uint32_t b_kstep, int K, uint32_t idesc, bool accumulate) {
    for (int s = 0; s < K / 16; ++s) {
        uint64_t ad = umma::smem_desc(a_addr + s * a_kstep, a_lbo, a_sbo);
        uint64_t bd = umma::smem_desc(b_addr + s * b_kstep, b_lbo, b_sbo);
        umma::mma_f16(tmem_d, ad, bd, idesc, (accumulate || s > 0) ? 1u : 0u);
    }
}

__device__ __forceinline__ int tmem_cols_pow2(int c) {
    int p = 32;
    while (p < c) p <<= 1;
    return p;
}

// True when any of the g slots from s0 holds a ROI.  Every thread evaluates it
// before the first barrier, so CTAs whose slots have all retired (the pool
// drains at the end of a batch) exit at once.
__device__ __forceinline__ bool tile_live(const SplitDev& P, int s0, int g) {
    bool live = false;
    for (int k = 0; k < g; ++k) live |= P.slot_roi[s0 + k] >= 0;
    return live;
}

// The next ROI of the queue among those already on the device, or -1.  With
// every input on the device this is one atomicAdd.  While inputs are still
// arriving, one lane of the warp takes a run of indices below the available
// count for all the lanes that ask (compare-and-swap; the queue only advances,
// so the loop ends), which keeps the contention per warp, not per slot.
__device__ __forceinline__ int take_roi(const SplitDev& P, int n) {
    const int avail = min(*(volatile const int*)P.navail, n);
    if (avail >= n) {
        const int q = atomicAdd(P.queue, 1);
        return q < n ? q : -1;
    }
    const unsigned m = __activemask();
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    const int rank = __popc(m & ((1u << lane) - 1u)), cnt = __popc(m);
    int base = 0, got = 0;
    if (lane == leader) {
        int q = *(volatile int*)P.queue;
        while (q < avail) {
            const int k = min(cnt, avail - q);
            const int old = atomicCAS(P.queue, q, q + k);
            if (old == q) {
                base = q;
                got = k;
                break;
            }
            q = old;
        }
    }
    base = __shfl_sync(m, base, leader);
    got = __shfl_sync(m, got, leader);
    return rank < got ? base + rank : -1;
}

// ----------------------------------------------- persistent-kernel helpers ----
// True in every thread when any of the tiles blockIdx.x, + gridDim.x, ... (of g
// slots each) holds a ROI.  A CTA without one leaves before it allocates TMEM
// or loads constants (a draining pool's last rounds).
__device__ __forceinline__ bool cta_has_live_tile(const SplitDev& P, int ntiles, int g) {
    __shared__ int s_any;
    if (threadIdx.x == 0) {
        int any = 0;
        for (int tile = blockIdx.x; tile < ntiles && !any; tile += gridDim.x) any = tile_live(P, tile * g, g);
        s_any = any;
    }
    __syncthreads();
    return s_any != 0;
}

// Named barrier 1 over the first N threads of the CTA (the epilogue warps).
template <int N = SPLIT_THREADS>
__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, %0;" ::"n"(N) : "memory"); }
// The same barrier, returning the OR of p over its threads (the same value in every thread).
template <int N = SPLIT_THREADS>
__device__ __forceinline__ bool epi_bar_or(bool p) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred P, Q;\n\tsetp.ne.u32 P, %1, 0;\n\t"
        "bar.red.or.pred Q, 1, %2, P;\n\tselp.u32 %0, 1, 0, Q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)p), "n"(N)
        : "memory");
    return r != 0;
}

// Named barrier `id` over N threads (a warp group's own barrier), and its OR form.
template <int N>
__device__ __forceinline__ void group_bar(int id) { asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(N) : "memory"); }
template <int N>
__device__ __forceinline__ bool group_bar_or(int id, bool p) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred P, Q;\n\tsetp.ne.u32 P, %1, 0;\n\t"
        "bar.red.or.pred Q, %2, %3, P;\n\tselp.u32 %0, 1, 0, Q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)p), "r"(id), "n"(N)
        : "memory");
    return r != 0;
}

__host__ __device__ constexpr int s2_slab_bytes(int W) { return 6 * W * 32; }
// one ring step of A2 K-slabs: W = 128 streams S hi, S lo (phase A) or S_y, S_z
// (phase B); smaller windows all four arrays at once
__host__ __device__ constexpr int s2_ring_bytes(int W) { return (W > 64 ? 2 : 4) * 4096; }
constexpr int S2_NBUF = 4;

__device__ __forceinline__ void warp_arrive(uint64_t* mbar) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) umma::mbar_arrive(mbar);
}

// ------------------------------------------------------------- work units ----
// The persistent stage kernels work in units of UG = max(G1, G2) consecutive
// slots, so that a unit is made of whole pupil-DFT tiles (G1 slots) and whole
// window tiles (G2 slots).  The round-based kernels walk the units statically
// (blockIdx.x, + gridDim.x, ...).  The dataflow kernel (k_flow) runs all five
// stages at once (the four model stages and the LM step), each on its own
// CTAs: a unit's state word counts its finished stages (5 e + s: ready for
// stage s of its evaluation e; UNIT_DEAD
// once its slots have retired and the ROI queue is empty), and in every CTA one
// scheduler thread hands the units of its share that are ready for its stage to
// the CTA's warps through a ring in shared memory.
constexpr int UNIT_DEAD = -1;
// Set in a unit's state word by the scheduler that handed it out, until the
// stage releases it: a unit is never handed out twice at once.
constexpr int UNIT_CLAIMED = 1 << 30;
constexpr int URING = 4;

__host__ __device__ inline int unit_slots(int G1, int G2) { return G1 > G2 ? G1 : G2; }


__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Relaxed loads of several state words can be in flight together; a unit found
// ready is then acquired with one fence.
__device__ __forceinline__ int ld_relaxed(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Slot s takes ROI r: fresh LM state at the ROI's (clamped) start point.
__device__ __forceinline__ void slot_take(const SplitDev& P, const FitIO& F, int s, int r) {
    P.slot_roi[s] = r;
    P.slot_phase[s] = 0;
    double* tr = P.lm[s].trial;
    for (int q = 0; q < 5; ++q) tr[q] = F.init[5 * r + q];
    lm_clamp(tr, F.prm);
}

// Stage 1's scheduler prepares unit u: its idle slots take ROIs that have
// arrived.  1: the unit has a live slot; 0: not yet (inputs still arriving);
// -1: none and the queue is exhausted (the unit is marked dead).
__device__ int unit_refill(const SplitDev& P, const FitIO& F, int u) {
    const int UG = unit_slots(P.G1, P.G2);
    bool live = false;
    for (int g = 0; g < UG; ++g) {
        const int s = u * UG + g;
        if (P.slot_roi[s] < 0 && *(volatile int*)P.queue < F.n) {
            const int r = take_roi(P, F.n);
            if (r >= 0) {
                slot_take(P, F, s, r);
                atomicAdd(P.active, 1);
            }
        }
        live |= P.slot_roi[s] >= 0;
    }
    if (live) return 1;
    if (*(volatile int*)P.queue >= F.n) {
        st_release(P.ustate + u, UNIT_DEAD);
        return -1;
    }
    return 0;
}

// State word of unit u after its LM step: its next evaluation, or dead when
// no slot holds a ROI and the queue is exhausted.
__device__ int unit_after_lm(const SplitDev& P, const FitIO& F, int u, int tag) {
    const int UG = unit_slots(P.G1, P.G2);
    bool live = false;
    for (int g = 0; g < UG; ++g) live |= P.slot_roi[u * UG + g] >= 0;
    if (!live && *(volatile int*)P.queue >= F.n) return UNIT_DEAD;
    return tag + 1;
}

struct StaticUnits {
    static constexpr bool flow = false;
    int u = -1;
    // The next unit with a live slot, or -1.  Every calling thread walks the
    // same sequence.
    __device__ int next(const SplitDev& P, int& tag, bool = false) {
        const int UG = unit_slots(P.G1, P.G2), U = P.P / UG;
        for (u = u < 0 ? (int)blockIdx.x : u + (int)gridDim.x; u < U; u += gridDim.x)
            if (tile_live(P, u * UG, UG)) {
                tag = 0;
                return u;
            }
        return -1;
    }
    __device__ void fence_writes() {}
    __device__ void release(const SplitDev&, int, int) {}
    __device__ void schedule(const SplitDev&, const FitIO&) {}
};

struct UnitRing {
    int unit[URING], tag[URING];
    int released;  // units this CTA has finished (for the scheduler's bookkeeping)
    uint64_t full[URING], freed[URING];
};

struct FlowUnits {
    static constexpr bool flow = true;
    UnitRing* r;
    int stage, first, stride;  // this CTA serves units first, first + stride, ... at stage `stage`
    int q;
    // The next unit handed out, or -1 when there is none left (or a wait gave
    // up).  Called by every lane of a warp, or by one lane (single); each
    // caller group arrives once on the ring entry.
    __device__ int next(const SplitDev& P, int& tag, bool single = false) {
        const int b = q % URING;
        const uint32_t par = (uint32_t)((q / URING) & 1);
        ++q;
        int u = -1;
        if (umma::mbar_wait(&r->full[b], par, P.err)) {
            u = r->unit[b];
            tag = r->tag[b];
        }
        if (single) {
            umma::mbar_arrive(&r->freed[b]);
        } else {
            __syncwarp();
            if ((threadIdx.x & 31) == 0) umma::mbar_arrive(&r->freed[b]);
        }
        // the unit's operands, written by other CTAs, are seen by this CTA's loads and bulk copies
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        asm volatile("fence.proxy.async.global;" ::: "memory");
        return u;
    }
    // Every thread that wrote a unit's operands: its generic-proxy writes are
    // made visible to the next stage's bulk (async-proxy) copies.
    __device__ void fence_writes() { asm volatile("fence.proxy.async.global;" ::: "memory"); }
    // One thread, once every writer of the unit has passed a barrier behind
    // fence_writes: publish the unit's next state.
    __device__ void release(const SplitDev& P, int u, int v) {
        __threadfence();
        st_release(P.ustate + u, v);
        atomicAdd(&r->released, 1);
    }
    // The scheduler thread: scan this CTA's units round-robin and hand out
    // those ready for its stage; stage 1's scheduler refills idle slots first.
    // Ends (handing out -1) when all its units are dead, when an error was
    // raised, or after P.wait_limit clocks without a ready unit (then it
    // raises the error word: 2).
    __device__ void schedule(const SplitDev& P, const FitIO& F) {
        const int UG = unit_slots(P.G1, P.G2), U = P.P / UG;
        const int mine = first < U ? (U - first + stride - 1) / stride : 0;
        int qq = 0, cur = 0;
        auto push = [&](int u, int tag) {
            const int b = qq % URING;
            if (qq >= URING && !umma::mbar_wait(&r->freed[b], (uint32_t)(((qq / URING) - 1) & 1), P.err)) return false;
            r->unit[b] = u;
            r->tag[b] = tag;
            umma::mbar_arrive(&r->full[b]);
            ++qq;
            return true;
        };
        const long long start = clock64();
        long long t0 = start, idle = 0, idle_since = -1;
        constexpr int SCAN = 8;  // state words loaded together
        while (*(volatile int*)P.err == 0) {
            int found = -1, tag = 0, dead = 0;
            for (int k0 = 0; k0 < mine && found < 0; k0 += SCAN) {
                int vv[SCAN], uu[SCAN];
#pragma unroll
                for (int j = 0; j < SCAN; ++j) {
                    const int k = k0 + j, i = cur + k < mine ? cur + k : cur + k - mine;
                    uu[j] = first + i * stride;
                    vv[j] = k < mine ? ld_relaxed(P.ustate + uu[j]) : UNIT_CLAIMED;
                }
                for (int j = 0; j < SCAN && k0 + j < mine; ++j) {
                    const int v = vv[j], u = uu[j];
                    if (v < 0) {
                        ++dead;
                        continue;
                    }
                    if ((v & UNIT_CLAIMED) || v % FLOW_STAGES != stage) continue;
                    asm volatile("fence.acq_rel.gpu;" ::: "memory");  // acquire what the unit's last stage wrote
                    if (stage == 0) {
                        const int ok = unit_refill(P, F, u);
                        if (ok < 0) ++dead;
                        if (ok <= 0) continue;
                    }
                    found = u;
                    tag = v;
                    const int i = k0 + j + cur < mine ? k0 + j + cur : k0 + j + cur - mine;
                    cur = i + 1 < mine ? i + 1 : 0;
                    break;
                }
            }
            if (found >= 0) {
                if (idle_since >= 0) idle += clock64() - idle_since;
                idle_since = -1;
                t0 = clock64();
                P.ustate[found] = tag | UNIT_CLAIMED;  // only this thread reads the claim
                if (!push(found, tag)) break;
                t0 = clock64();
                continue;
            }
            if (dead == mine) break;
            // the CTA is idle once every unit handed out has been finished
            const bool drained = *(volatile int*)&r->released >= qq;
            if (idle_since < 0 && drained) idle_since = clock64();
            if (clock64() - t0 > P.wait_limit) {
                atomicExch(P.err, 2);
                break;
            }
            __nanosleep(32);
        }
        push(-1, 0);
        const long long end = clock64();
        if (idle_since >= 0) idle += end - idle_since;
        P.clk[3 * blockIdx.x] = (unsigned long long)idle;
        P.clk[3 * blockIdx.x + 1] = (unsigned long long)(end - start);
        P.clk[3 * blockIdx.x + 2] = (unsigned long long)(qq > 0 ? qq - 1 : 0);
    }
};


// ------------------------------------------------- stage 1 (persistent) -----
// One CTA per SM walks the stage-1 tiles (G1 slots x DP pupil rows a) with the
// DFT constants resident in shared memory (the K-slabs the window stage uses).
// The 512 builder threads compute the pupil field Q one K step at a time (8
// pupil columns b with their real and imaginary parts, in the K order of
// kperm) into a 4-deep ring; the MMA warp multiplies each step against the
// resident constants: hi x [parts 0-3] gives S and S_y, hi x [lo parts 0-1]
// and lo x [parts 0-1] accumulate onto S, and Q_z = i kz Q x [parts 0-1] gives
// S_z.  S, S_y and S_z need 6W columns: for W = 128 that exceeds TMEM, so a
// second pass over K rebuilds only Q_z.  The builders then move the
// accumulators to the stage-2 operand A2 (rows (slot, i), K = a).
constexpr int S1_THREADS = SPLIT_THREADS + 32;
constexpr int S1_NBQ = 4;
constexpr int S1_QB = 128 * 32;  // one Q array for one K step: 128 rows x 16 k, f16

__host__ __device__ constexpr int s1_qring_bytes(int W) { return (W > 64 ? 2 : 3) * S1_QB; }

template <int W, class UNITS>
__device__ __forceinline__ void stage1_body(const SplitDev& P, const FitIO& F, UNITS units) {
    extern __shared__ __align__(1024) char smem[];
    constexpr bool TWO = W > 64;
    constexpr int SLAB = s2_slab_bytes(W), QRING = s1_qring_bytes(W), NBQ = S1_NBQ, QB = S1_QB;
    constexpr int NCOLS = W >= 64 ? 512 : 256;
    const int K1 = P.K1, DP = P.DP, G1 = P.G1, t = threadIdx.x, warp = t >> 5, lane = t & 31;
    // W = 128 comes with K1 = 128 (64 pupil rows): 8 K steps, known here so that the
    // Q_z values of pass A stay in registers for pass B
    const int NS = TWO ? 8 : K1 / 16;
    const int T1 = unit_slots(G1, P.G2) / G1;  // stage-1 tiles per unit
    char* CS = smem;               // NS constant K-slabs
    char* QR = smem + NS * SLAB;   // ring of Q K-slabs
    __shared__ __align__(8) uint64_t cfull, qfull[NBQ], qfree[NBQ], accA, accB, tfree, fin;
    __shared__ uint32_t tmem_base;
    if (t < 32) umma::tmem_alloc(&tmem_base, NCOLS);
    if (t == 0) {
        umma::mbar_init(&cfull, 1);
        for (int b = 0; b < NBQ; ++b) { umma::mbar_init(&qfull[b], SPLIT_THREADS / 32); umma::mbar_init(&qfree[b], 1); }
        umma::mbar_init(&accA, 1);
        umma::mbar_init(&accB, 1);
        umma::mbar_init(&tfree, SPLIT_THREADS / 32);
        umma::mbar_init(&fin, 1);
        umma::mbar_fence_init();
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tbase = tmem_base;
    if (t == 0) {
        umma::mbar_expect_tx(&cfull, (uint32_t)(NS * SLAB));
        for (int s = 0; s < NS; ++s)
            umma::bulk_g2s(CS + s * SLAB, (const char*)P.bcs + (size_t)s * SLAB, SLAB, &cfull);
    }

    if (warp == SPLIT_THREADS / 32) {  // ---------------- MMA issuer (lane 0), scheduler (lane 1)
        if constexpr (UNITS::flow)
            if (lane == 1) {
                units.schedule(P, F);
                return;
            }
        if (lane != 0) return;
        bool ok = umma::mbar_wait(&cfull, 0, P.err);
        int q = 0, nwait = 0, nphase = 0;
        auto tmem_ready = [&]() {  // every MMA phase after the first waits for the epilogue before it
            if (nphase++ == 0) return true;
            const bool r = umma::mbar_wait(&tfree, (uint32_t)(nwait & 1), P.err);
            ++nwait;
            umma::fence_after_sync();
            return r;
        };
        auto steps = [&](bool pb) {
            for (int s = 0; s < NS; ++s, ++q) {
                const int buf = q % NBQ;
                if (!umma::mbar_wait(&qfull[buf], (uint32_t)((q / NBQ) & 1), P.err)) return false;
                umma::fence_after_sync();
                const uint32_t qs = umma::smem_u32(QR + buf * QRING), cb = umma::smem_u32(CS + s * SLAB);
                auto mma = [&](uint32_t a, int row0, int N, int col, bool acc) {
                    const uint64_t ad = umma::smem_desc(a, 128, 256);
                    const uint64_t bd = umma::smem_desc(cb + (uint32_t)(row0 / 8) * 256, 128, 256);
                    umma::mma_f16(tbase + col, ad, bd, umma::idesc_f16(128, N, false, false), acc ? 1u : 0u);
                };
                if (!pb) {
#pragma unroll
                    for (int r = 0; r < 4 * W; r += 256) mma(qs, r, 4 * W < 256 ? 4 * W : 256, r, s > 0);  // S, S_y
                    mma(qs, 4 * W, 2 * W, 0, true);    // + hi x lo(C)
                    mma(qs + QB, 0, 2 * W, 0, true);   // + lo x hi(C)
                    if (!TWO) mma(qs + 2 * QB, 0, 2 * W, 4 * W, s > 0);  // S_z
                } else {
                    mma(qs, 0, 2 * W, 0, s > 0);       // S_z
                }
                umma::mma_commit(&qfree[buf]);
            }
            return true;
        };
        for (int tag = 0; ok;) {
            const int unit = units.next(P, tag, true);
            if (unit < 0) break;
            for (int k = 0; k < T1 && ok; ++k) {
                const int tile = unit * T1 + k;
                if (!tile_live(P, tile * G1, G1)) continue;
                ok = tmem_ready() && steps(false);
                umma::mma_commit(&accA);
                if (TWO && ok) {
                    ok = tmem_ready() && steps(true);
                    umma::mma_commit(&accB);
                }
            }
        }
        umma::mma_commit(&fin);
        return;
    }

    // ---------------- builders / epilogue
    // build mapping: slab row brow (8 per warp, conflict-free 4-byte stores), column pair bp
    const int brow = 8 * warp + (lane & 7), bp = lane >> 3;
    const int bg = brow / DP, ba = brow % DP;
    // epilogue mapping: TMEM row (g, a) = t % 128, its warpgroup's share of the output index i
    const int row = t & 127, wg = t >> 7;
    const int g = row / DP, a = row % DP;
    const int kre = kperm(a, false), kim = kperm(a, true);
    const size_t arr = (size_t)128 * K1 * 2;
    constexpr int CW = W / 4;
    int q = 0, ntile = 0;
    bool abort = false;
    for (int tag = 0; !abort;) {
        const int unit = units.next(P, tag);
        if (unit < 0) break;
        for (int k = 0; k < T1 && !abort; ++k) {
            const int tile = unit * T1 + k;
            if (!tile_live(P, tile * G1, G1)) continue;
            const uint32_t ph = (uint32_t)(ntile & 1);
            ++ntile;
            const int bslot = tile * G1 + bg;
            const bool blive = P.slot_roi[bslot] >= 0;
            double x = 0, y = 0, z = 0;
            if (blive) {
                x = P.lm[bslot].trial[0]; y = P.lm[bslot].trial[1]; z = P.lm[bslot].trial[2];
            }
            const double kxa = P.kx[ba];
            // one K step of Q (columns b = 8 s + 2 bp + {0, 1} of row brow); the table loads of
            // the next step are issued before this step's arithmetic
            struct QTab { double2 p0, kz, ky; float2 pu; };
            auto qtab = [&](int s) {
                const size_t i2 = (((size_t)s * 4 + bp) * DP + ba) * 2;
                const size_t i4 = (((size_t)s * 2 + (bp >> 1)) * DP + ba) * 4 + (bp & 1) * 2;
                QTab q2;
                q2.p0 = *(const double2*)(P.phase0 + i2);
                q2.kz = *(const double2*)(P.kz + i2);
                q2.pu = *(const float2*)(P.pupf + i4);
                q2.ky = *(const double2*)(P.ky + 8 * s + 2 * bp);
                return q2;
            };
            // the table lines of step s on their way to L1 (the same for every tile)
            auto qpre = [&](int s) {
                const size_t i2 = (((size_t)s * 4 + bp) * DP + ba) * 2;
                const size_t i4 = (((size_t)s * 2 + (bp >> 1)) * DP + ba) * 4 + (bp & 1) * 2;
                asm volatile("prefetch.global.L1 [%0];" ::"l"(P.phase0 + i2));
                asm volatile("prefetch.global.L1 [%0];" ::"l"(P.kz + i2));
                asm volatile("prefetch.global.L1 [%0];" ::"l"(P.pupf + i4));
            };
            const uint32_t ore = kmajor_off(brow, 2 * bp, 16), oim = kmajor_off(brow, 8 + 2 * bp, 16);
            auto slot_wait = [&]() {  // ring slot for the next K step
                const int buf = q % NBQ;
                if (q >= NBQ) umma::mbar_wait(&qfree[buf], (uint32_t)((q / NBQ - 1) & 1), P.err);
                ++q;
                return QR + buf * QRING;
            };
            auto slot_done = [&](char* qs) {  // every writer fences its stores; one arrive per warp
                umma::fence_proxy_async();
                warp_arrive(&qfull[(qs - QR) / QRING]);
            };
            uint32_t zkeep[TWO ? 8 : 1][2] = {};  // pass A's Q_z of each K step (W = 128)
            auto build = [&](int s, const QTab& tb, uint32_t& zr, uint32_t& zi) {
                const double ph0[2] = {tb.p0.x, tb.p0.y}, kzr[2] = {tb.kz.x, tb.kz.y}, kyr[2] = {tb.ky.x, tb.ky.y};
                const float pu[2] = {tb.pu.x, tb.pu.y};
                float qr[2], qi[2], kzv[2];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    qr[e] = 0.f; qi[e] = 0.f; kzv[e] = 0.f;
                    if (blive && pu[e] != 0.f) {
                        float sn, cs;
                        sincos_phase(ph0[e] + kxa * x + kyr[e] * y + kzr[e] * z, sn, cs);
                        qr[e] = pu[e] * cs;
                        qi[e] = pu[e] * sn;
                        kzv[e] = (float)kzr[e];
                    }
                }
                zr = pack_h2(-kzv[0] * qi[0] * P.sc.qz, -kzv[1] * qi[1] * P.sc.qz);  // Q_z = i kz Q
                zi = pack_h2(kzv[0] * qr[0] * P.sc.qz, kzv[1] * qr[1] * P.sc.qz);
                uint32_t rh, rl, ih, il;
                split2(qr[0] * P.sc.q, qr[1] * P.sc.q, rh, rl);
                split2(qi[0] * P.sc.q, qi[1] * P.sc.q, ih, il);
                char* qs = slot_wait();
                *(uint32_t*)(qs + ore) = rh;
                *(uint32_t*)(qs + oim) = ih;
                *(uint32_t*)(qs + QB + ore) = rl;
                *(uint32_t*)(qs + QB + oim) = il;
                if (!TWO) {
                    *(uint32_t*)(qs + 2 * QB + ore) = zr;
                    *(uint32_t*)(qs + 2 * QB + oim) = zi;
                }
                slot_done(qs);
            };
            // W = 128: steps s and s + 1 together, so that four sin/cos chains are in flight
            auto build_pair = [&](int s, const QTab& ta, const QTab& tc, uint32_t (&za)[2], uint32_t (&zc)[2]) {
                float qr[4], qi[4], kzv[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const QTab& tb = e < 2 ? ta : tc;
                    const double ph0 = (e & 1) ? tb.p0.y : tb.p0.x, kzr = (e & 1) ? tb.kz.y : tb.kz.x;
                    const double kyr = (e & 1) ? tb.ky.y : tb.ky.x;
                    const float pu = (e & 1) ? tb.pu.y : tb.pu.x;
                    qr[e] = 0.f; qi[e] = 0.f; kzv[e] = 0.f;
                    if (blive && pu != 0.f) {
                        float sn, cs;
                        sincos_phase(ph0 + kxa * x + kyr * y + kzr * z, sn, cs);
                        qr[e] = pu * cs;
                        qi[e] = pu * sn;
                        kzv[e] = (float)kzr;
                    }
                }
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int e = 2 * h;
                    uint32_t(&zz)[2] = h == 0 ? za : zc;
                    zz[0] = pack_h2(-kzv[e] * qi[e] * P.sc.qz, -kzv[e + 1] * qi[e + 1] * P.sc.qz);  // Q_z = i kz Q
                    zz[1] = pack_h2(kzv[e] * qr[e] * P.sc.qz, kzv[e + 1] * qr[e + 1] * P.sc.qz);
                    uint32_t rh, rl, ih, il;
                    split2(qr[e] * P.sc.q, qr[e + 1] * P.sc.q, rh, rl);
                    split2(qi[e] * P.sc.q, qi[e + 1] * P.sc.q, ih, il);
                    char* qs = slot_wait();
                    *(uint32_t*)(qs + ore) = rh;
                    *(uint32_t*)(qs + oim) = ih;
                    *(uint32_t*)(qs + QB + ore) = rl;
                    *(uint32_t*)(qs + QB + oim) = il;
                    slot_done(qs);
                }
            };
            auto build_z = [&](int s) {  // pass B (W = 128): the kept Q_z of step s
                char* qs = slot_wait();
                *(uint32_t*)(qs + ore) = zkeep[TWO ? s : 0][0];
                *(uint32_t*)(qs + oim) = zkeep[TWO ? s : 0][1];
                slot_done(qs);
            };
            // A2 destination of this thread's TMEM row: stage-2 tile of the slot, K positions of a
            const int slot = tile * G1 + g;
            const bool live = P.slot_roi[slot] >= 0;
            const int tile2 = slot / P.G2, mrow0 = (slot % P.G2) * W;
            char* a2t = P.a2 + (size_t)tile2 * a2_tile_bytes(K1);
            // epilogue of one pass: maps at TMEM columns c0 (S), c0 + 2W (S_y), zc (S_z; < 0: none)
            auto epilogue = [&](bool sy, int zc, uint32_t phase, uint64_t* accb) {
                umma::mbar_wait(accb, phase, P.err);
                umma::fence_after_sync();
#pragma unroll 1
                for (int h = wg * CW; h < (wg + 1) * CW; h += 8) {
                    const int m = mrow0 + h;
                    if (sy) {
                        float v4[4][8];
                        const uint32_t ad[4] = {tmem_lane_addr(tbase, h), tmem_lane_addr(tbase, W + h),
                                                tmem_lane_addr(tbase, 2 * W + h), tmem_lane_addr(tbase, 3 * W + h)};
                        tmem_ld8_multi<4>(ad, v4);
                        const float *sr = v4[0], *si = v4[1], *yr = v4[2], *yi = v4[3];
                        if (live) {
                            uint32_t shr[4], slr[4], shi[4], sli[4], wyr[4], wyi[4];
#pragma unroll
                            for (int u = 0; u < 8; u += 2) {
                                split2(sr[u] * P.sc.c2, sr[u + 1] * P.sc.c2, shr[u / 2], slr[u / 2]);
                                split2(si[u] * P.sc.c2, si[u + 1] * P.sc.c2, shi[u / 2], sli[u / 2]);
                                wyr[u / 2] = pack_h2(yr[u] * P.sc.c2y, yr[u + 1] * P.sc.c2y);
                                wyi[u / 2] = pack_h2(yi[u] * P.sc.c2y, yi[u + 1] * P.sc.c2y);
                            }
                            store4w(a2t + 0 * arr + mnmajor_off(m, kre, 128), shr);
                            store4w(a2t + 1 * arr + mnmajor_off(m, kre, 128), slr);
                            store4w(a2t + 0 * arr + mnmajor_off(m, kim, 128), shi);
                            store4w(a2t + 1 * arr + mnmajor_off(m, kim, 128), sli);
                            store4w(a2t + 2 * arr + mnmajor_off(m, kre, 128), wyr);
                            store4w(a2t + 2 * arr + mnmajor_off(m, kim, 128), wyi);
                        }
                    }
                    if (zc >= 0) {
                        float v2[2][8];
                        const uint32_t ad[2] = {tmem_lane_addr(tbase, zc + h), tmem_lane_addr(tbase, zc + W + h)};
                        tmem_ld8_multi<2>(ad, v2);
                        const float *zr8 = v2[0], *zi8 = v2[1];
                        if (live) {
                            uint32_t wzr[4], wzi[4];
#pragma unroll
                            for (int u = 0; u < 8; u += 2) {
                                wzr[u / 2] = pack_h2(zr8[u] * P.sc.c2z, zr8[u + 1] * P.sc.c2z);
                                wzi[u / 2] = pack_h2(zi8[u] * P.sc.c2z, zi8[u + 1] * P.sc.c2z);
                            }
                            store4w(a2t + 3 * arr + mnmajor_off(m, kre, 128), wzr);
                            store4w(a2t + 3 * arr + mnmajor_off(m, kim, 128), wzi);
                        }
                    }
                }
                umma::fence_before_sync();
                warp_arrive(&tfree);
            };
            if constexpr (TWO) {
#pragma unroll
                for (int s = 0; s < 8; s += 2) {
                    if (s + 2 < 8) {
                        qpre(s + 2);
                        qpre(s + 3);
                    }
                    build_pair(s, qtab(s), qtab(s + 1), zkeep[s], zkeep[s + 1]);
                }
                qpre(0);  // the next tile's first pair
                qpre(1);
#pragma unroll
                for (int s = 0; s < NBQ; ++s) build_z(s);
                epilogue(true, -1, ph, &accA);
#pragma unroll
                for (int s = NBQ; s < 8; ++s) build_z(s);
                epilogue(false, 0, ph, &accB);
            } else {
                QTab cur = qtab(0);
                for (int s = 0; s < NS; ++s) {
                    QTab nxt;
                    if (s + 1 < NS) nxt = qtab(s + 1);
                    uint32_t zr, zi;
                    build(s, cur, zr, zi);
                    if (s + 1 < NS) cur = nxt;
                }
                epilogue(true, 4 * W, ph, &accA);
            }
            // (a bounded wait that gave up makes every builder leave the loop together)
            units.fence_writes();
            abort = epi_bar_or(t == 0 && *(volatile int*)P.err != 0);
        }
        if (!abort && t == 0) units.release(P, unit, tag + 1);
    }
    if (t == 0) {
        umma::mbar_wait(&fin, 0, P.err);    // every MMA of this CTA has completed
        umma::mbar_wait(&cfull, 0, P.err);  // and the constant copies have landed
    }
    epi_bar();
    if (t < 32) umma::tmem_dealloc(tbase, NCOLS);
}

template <int W>
__global__ void __launch_bounds__(S1_THREADS, 1) k_stage1p(SplitDev P, FitIO F) {
    if (!cta_has_live_tile(P, P.P / unit_slots(P.G1, P.G2), unit_slots(P.G1, P.G2))) return;
    stage1_body<W>(P, F, StaticUnits{});
}


// ------------------------------------------------- stage 2 (persistent) -----
// One CTA per SM walks the stage-2 tiles (G2 slots x W rows j) with the
// constants resident in shared memory: the K-slabs (16 columns of K1, all 6W
// rows: hi of parts 0-3, lo of parts 0-1) are loaded once per CTA, so the
// per-tile traffic is the A2 operand only, streamed in 4 KB K-slabs per array
// through an NBUF-deep ring by a producer warp.  Per K step, hi x [parts 0-3]
// produces E and Ex (N up to 256 per instruction), hi x [lo parts 0-1] and
// lo x [parts 0-1] accumulate onto E, y x [parts 0-1] and z x [parts 0-1]
// produce Ey and Ez.  The 8W accumulator columns fit TMEM for W <= 64 (one
// phase); for W = 128 phase A computes E and Ex, its epilogue stores I, lo(I)
// and I_x and keeps E in registers, and phase B reuses the columns for Ey and
// Ez.  Warps 0-15 run the epilogues (thread 0 also issues the MMAs), warp 16
// is the producer.
constexpr int S2_THREADS = SPLIT_THREADS + 32;

template <int W, class UNITS>
__device__ __forceinline__ void stage2_body(const SplitDev& P, const FitIO& F, UNITS units) {
    extern __shared__ __align__(1024) char smem[];
    constexpr bool TWO = W > 64;
    constexpr int SLAB = s2_slab_bytes(W), RING = s2_ring_bytes(W), NBUF = S2_NBUF;
    constexpr int NCOLS = W >= 64 ? 512 : 256;
    const int K1 = P.K1, G2 = P.G2, t = threadIdx.x;
    const int NS = K1 / 16, NSTEP = TWO ? 2 * NS : NS;
    const int T2 = unit_slots(P.G1, G2) / G2;  // window tiles per unit
    const uint32_t arr = 128u * K1 * 2;
    char* CS = smem;                 // NS constant K-slabs
    char* RB = smem + NS * SLAB;     // ring of A2 K-slabs
    __shared__ __align__(8) uint64_t cfull, full[NBUF], freed[NBUF], accA, accB;
    __shared__ uint32_t tmem_base;
    if (t < 32) umma::tmem_alloc(&tmem_base, NCOLS);
    if (t == 0) {
        umma::mbar_init(&cfull, 1);
        for (int b = 0; b < NBUF; ++b) { umma::mbar_init(&full[b], 1); umma::mbar_init(&freed[b], 1); }
        umma::mbar_init(&accA, 1);
        umma::mbar_init(&accB, 1);
        umma::mbar_fence_init();
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tbase = tmem_base;

    if (t >= SPLIT_THREADS) {  // ---------------- producer (lane 0), scheduler (lane 1)
        if constexpr (UNITS::flow)
            if (t == SPLIT_THREADS + 1) {
                units.schedule(P, F);
                return;
            }
        if (t != SPLIT_THREADS) return;
        umma::mbar_expect_tx(&cfull, (uint32_t)(NS * SLAB));
        for (int s = 0; s < NS; ++s)
            umma::bulk_g2s(CS + s * SLAB, (const char*)P.bcs + (size_t)s * SLAB, SLAB, &cfull);
        int q = 0;
        for (int tag = 0;;) {
            const int unit = units.next(P, tag, true);
            if (unit < 0) break;
            for (int k = 0; k < T2; ++k) {
                const int tile = unit * T2 + k;
                if (!tile_live(P, tile * G2, G2)) continue;
                const char* src = P.a2 + (size_t)tile * a2_tile_bytes(K1);
                for (int n = 0; n < NSTEP; ++n, ++q) {
                    const int buf = q % NBUF;
                    if (q >= NBUF && !umma::mbar_wait(&freed[buf], (uint32_t)((q / NBUF - 1) & 1), P.err)) return;
                    const bool pb = TWO && n >= NS;
                    const int s = pb ? n - NS : n;
                    const int a0 = pb ? 2 : 0;  // phase B streams the y and z arrays
                    constexpr int NARR = TWO ? 2 : 4;  // A2 arrays per ring step
                    umma::mbar_expect_tx(&full[buf], RING);
                    for (int j = 0; j < NARR; ++j)
                        umma::bulk_g2s(RB + buf * RING + j * 4096, src + (size_t)(a0 + j) * arr + (size_t)s * 4096, 4096,
                                       &full[buf]);
                }
            }
        }
        return;
    }

    // ---------------- epilogue warps; thread 0 issues the MMAs
    const int row = t & 127, wg = t >> 7;
    constexpr int CW = W / 4;  // indices i per warpgroup
    const size_t arr3 = (size_t)128 * W * 2;
    const uint32_t lbo_mn = (128 / 8) * 128;
    int q = 0, ph = 0;
    auto issue_steps = [&](int n0, int n1) {
        for (int n = n0; n < n1; ++n, ++q) {
            const int buf = q % NBUF;
            if (!umma::mbar_wait(&full[buf], (uint32_t)((q / NBUF) & 1), P.err)) return;
            umma::fence_after_sync();
            const uint32_t rb = umma::smem_u32(RB + buf * RING);
            const bool pb = TWO && n >= NS;
            const uint32_t cb = umma::smem_u32(CS + (pb ? n - NS : n) * SLAB);
            const bool first = (pb ? n - NS : n) == 0;
            auto mma = [&](uint32_t a, int row0, int N, int col, bool acc) {
                const uint64_t ad = umma::smem_desc(a, lbo_mn, 128);
                const uint64_t bd = umma::smem_desc(cb + (uint32_t)(row0 / 8) * 256, 128, 256);
                umma::mma_f16(tbase + col, ad, bd, umma::idesc_f16(128, N, true, false), acc ? 1u : 0u);
            };
            if (!pb) {
#pragma unroll
                for (int r = 0; r < 4 * W; r += 256) mma(rb, r, 4 * W < 256 ? 4 * W : 256, r, !first);  // E, Ex
                mma(rb, 4 * W, 2 * W, 0, true);         // + hi x lo(C)
                mma(rb + 4096, 0, 2 * W, 0, true);      // + lo x hi(C)
                if (!TWO) {
                    mma(rb + 8192, 0, 2 * W, 4 * W, !first);   // Ey
                    mma(rb + 12288, 0, 2 * W, 6 * W, !first);  // Ez
                }
            } else {
                mma(rb, 0, 2 * W, 0, !first);          // Ey
                mma(rb + 4096, 0, 2 * W, 2 * W, !first);  // Ez
            }
            umma::mma_commit(&freed[buf]);
        }
    };
    auto ipx = [](const float* er, const float* ei, const float* xr, const float* xi, int u, float cf) {
        return (er[u] * xr[u] + ei[u] * xi[u]) * cf;
    };
    if (t == 0) umma::mbar_wait(&cfull, 0, P.err);
    bool abort = false;
    for (int tag = 0; !abort;) {
        const int unit = units.next(P, tag);
        if (unit < 0) break;
        for (int k = 0; k < T2 && !abort; ++k) {
            const int tile = unit * T2 + k;
            if (!tile_live(P, tile * G2, G2)) continue;
            char* a3t = P.a3 + (size_t)tile * a3_tile_bytes(W);
            if (t == 0) {
                issue_steps(0, NS);
                umma::mma_commit(&accA);
            }
            umma::mbar_wait(&accA, (uint32_t)ph, P.err);
            umma::fence_after_sync();
            if constexpr (TWO) {
                float er[CW], ei[CW];
#pragma unroll
                for (int h = 0; h < CW; h += 8) {
                    const int i0 = wg * CW + h;
                    float v4[4][8];
                    const uint32_t ad[4] = {tmem_lane_addr(tbase, i0), tmem_lane_addr(tbase, W + i0),
                                            tmem_lane_addr(tbase, 2 * W + i0), tmem_lane_addr(tbase, 3 * W + i0)};
                    tmem_ld8_multi<4>(ad, v4);
#pragma unroll
                    for (int u = 0; u < 8; ++u) { er[h + u] = v4[0][u]; ei[h + u] = v4[1][u]; }
                    const float *xr = v4[2], *xi = v4[3];
                    uint32_t hh[4], ll[4], dx[4];
#pragma unroll
                    for (int u = 0; u < 8; u += 2) {
                        split2((er[h + u] * er[h + u] + ei[h + u] * ei[h + u]) * P.sc.cI,
                               (er[h + u + 1] * er[h + u + 1] + ei[h + u + 1] * ei[h + u + 1]) * P.sc.cI, hh[u / 2],
                               ll[u / 2]);
                        dx[u / 2] = pack_h2(ipx(er + h, ei + h, xr, xi, u, P.sc.cIx),
                                            ipx(er + h, ei + h, xr, xi, u + 1, P.sc.cIx));
                    }
                    const uint32_t off = kmajor_off(row, i0, W);
                    store4w(a3t + 0 * arr3 + off, hh);
                    store4w(a3t + 1 * arr3 + off, ll);
                    store4w(a3t + 2 * arr3 + off, dx);
                }
                umma::fence_before_sync();
                epi_bar();
                if (t == 0) {
                    umma::fence_after_sync();
                    issue_steps(NS, NSTEP);
                    umma::mma_commit(&accB);
                }
                umma::mbar_wait(&accB, (uint32_t)ph, P.err);
                umma::fence_after_sync();
#pragma unroll
                for (int h = 0; h < CW; h += 8) {
                    const int i0 = wg * CW + h;
                    float v4[4][8];
                    const uint32_t ad[4] = {tmem_lane_addr(tbase, i0), tmem_lane_addr(tbase, W + i0),
                                            tmem_lane_addr(tbase, 2 * W + i0), tmem_lane_addr(tbase, 3 * W + i0)};
                    tmem_ld8_multi<4>(ad, v4);
                    uint32_t dy[4], dz[4];
#pragma unroll
                    for (int u = 0; u < 8; u += 2) {
                        dy[u / 2] = pack_h2(ipx(er + h, ei + h, v4[0], v4[1], u, P.sc.cIy),
                                            ipx(er + h, ei + h, v4[0], v4[1], u + 1, P.sc.cIy));
                        dz[u / 2] = pack_h2(ipx(er + h, ei + h, v4[2], v4[3], u, P.sc.cIz),
                                            ipx(er + h, ei + h, v4[2], v4[3], u + 1, P.sc.cIz));
                    }
                    const uint32_t off = kmajor_off(row, i0, W);
                    store4w(a3t + 3 * arr3 + off, dy);
                    store4w(a3t + 4 * arr3 + off, dz);
                }
            } else {
#pragma unroll
                for (int h = 0; h < CW; h += 8) {
                    const int i0 = wg * CW + h;
                    float v4[4][8];
                    const uint32_t ad[4] = {tmem_lane_addr(tbase, i0), tmem_lane_addr(tbase, W + i0),
                                            tmem_lane_addr(tbase, 2 * W + i0), tmem_lane_addr(tbase, 3 * W + i0)};
                    tmem_ld8_multi<4>(ad, v4);
                    const float *er = v4[0], *ei = v4[1], *xr = v4[2], *xi = v4[3];
                    uint32_t hh[4], ll[4], dx[4], dy[4], dz[4];
#pragma unroll
                    for (int u = 0; u < 8; u += 2) {
                        split2((er[u] * er[u] + ei[u] * ei[u]) * P.sc.cI,
                               (er[u + 1] * er[u + 1] + ei[u + 1] * ei[u + 1]) * P.sc.cI, hh[u / 2], ll[u / 2]);
                        dx[u / 2] = pack_h2(ipx(er, ei, xr, xi, u, P.sc.cIx), ipx(er, ei, xr, xi, u + 1, P.sc.cIx));
                    }
                    float w4[4][8];
                    const uint32_t bd[4] = {tmem_lane_addr(tbase, 4 * W + i0), tmem_lane_addr(tbase, 5 * W + i0),
                                            tmem_lane_addr(tbase, 6 * W + i0), tmem_lane_addr(tbase, 7 * W + i0)};
                    tmem_ld8_multi<4>(bd, w4);
#pragma unroll
                    for (int u = 0; u < 8; u += 2) {
                        dy[u / 2] = pack_h2(ipx(er, ei, w4[0], w4[1], u, P.sc.cIy), ipx(er, ei, w4[0], w4[1], u + 1, P.sc.cIy));
                        dz[u / 2] = pack_h2(ipx(er, ei, w4[2], w4[3], u, P.sc.cIz), ipx(er, ei, w4[2], w4[3], u + 1, P.sc.cIz));
                    }
                    const uint32_t off = kmajor_off(row, i0, W);
                    store4w(a3t + 0 * arr3 + off, hh);
                    store4w(a3t + 1 * arr3 + off, ll);
                    store4w(a3t + 2 * arr3 + off, dx);
                    store4w(a3t + 3 * arr3 + off, dy);
                    store4w(a3t + 4 * arr3 + off, dz);
                }
            }
            // all TMEM reads of this tile done before the next tile's MMAs
            // (a bounded wait that gave up makes every epilogue thread leave the loop together)
            umma::fence_before_sync();
            units.fence_writes();
            abort = epi_bar_or(t == 0 && *(volatile int*)P.err != 0);
            if (t == 0) umma::fence_after_sync();
            ph ^= 1;
        }
        if (!abort && t == 0) units.release(P, unit, tag + 1);
    }
    epi_bar();
    if (t < 32) umma::tmem_dealloc(tbase, NCOLS);
}

template <int W>
__global__ void __launch_bounds__(S2_THREADS, 1) k_stage2p(SplitDev P, FitIO F) {
    if (!cta_has_live_tile(P, P.P / unit_slots(P.G1, P.G2), unit_slots(P.G1, P.G2))) return;
    stage2_body<W>(P, F, StaticUnits{});
}


// ------------------------------------------------- stage 3 (persistent) -----
// Blur along the first image index: J^T[(g2, j)][i'] = sum_i I[j][i] G[i'][i]
// for each window tile (G2 slots x W rows j).  One CTA per SM keeps G^T in
// shared memory; warp 16 loads a tile's five intensity arrays (A3) and issues
// its MMAs into one of two TMEM accumulators, so that the next tile's load and
// MMAs overlap this tile's epilogue (warps 0-15), which writes the row-blurred
// maps as the column-blur B operand (hi, lo; N = 4 RP rows (map, i'), K = j).
constexpr int S3_THREADS = SPLIT_THREADS + 32;
// Window tiles of the row blur in shared memory: two (a loader lane fills one
// while the MMAs read the other) for windows up to 64 in the round-based
// kernel, one otherwise (160 KB at W = 128; the dataflow kernel's stage CTAs
// keep the smaller plan).
__host__ __device__ constexpr int s3_nbuf(int W, bool flow) { return !flow && W <= 64 ? 2 : 1; }

template <class UNITS>
__device__ __forceinline__ void stage3_body(const SplitDev& P, const FitIO& F, UNITS units) {
    extern __shared__ __align__(1024) char smem[];
    const int W = P.W, RP = P.RP, G2 = P.G2, t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int T2 = unit_slots(P.G1, G2) / G2;
    const size_t arr3 = (size_t)128 * W * 2, gbytes = (size_t)RP * W * 2;
    const int NB3 = s3_nbuf(W, UNITS::flow);
    char* A3 = smem;                  // NB3 window tiles: I hi, I lo, I_x, I_y, I_z
    char* GT = A3 + NB3 * 5 * arr3;   // G^T hi, lo
    __shared__ __align__(8) uint64_t gfull, full[2], acc[2], tfree[2], fin;
    __shared__ uint32_t tmem_base;
    const int nc = tmem_cols_pow2(4 * RP);  // one accumulator
    if (t < 32) umma::tmem_alloc(&tmem_base, 2 * nc);
    if (t == 0) {
        umma::mbar_init(&gfull, 1);
        umma::mbar_init(&full[0], 1);
        umma::mbar_init(&full[1], 1);
        for (int b = 0; b < 2; ++b) {
            umma::mbar_init(&acc[b], 1);
            umma::mbar_init(&tfree[b], SPLIT_THREADS / 32);
        }
        umma::mbar_init(&fin, 1);
        umma::mbar_fence_init();
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tbase = tmem_base;

    if (warp == SPLIT_THREADS / 32) {  // ------- MMAs (lane 0), scheduler (lane 1) or A3 loader (lane 1, two buffers)
        if constexpr (UNITS::flow)
            if (lane == 1) {
                units.schedule(P, F);
                return;
            }
        if (NB3 == 2 && lane == 1) {
            // the loader: tile n goes to buffer n & 1 once the MMAs of tile n - 2 (the
            // buffer's last reader) have completed; the MMA lane walks the same tiles
            int n = 0;
            for (int tag = 0;;) {
                const int unit = units.next(P, tag, true);
                if (unit < 0) break;
                bool ok = true;
                for (int k = 0; k < T2; ++k) {
                    const int tile = unit * T2 + k;
                    if (!tile_live(P, tile * G2, G2)) continue;
                    const int b = n & 1;
                    if (n >= 2 && !umma::mbar_wait(&acc[b], (uint32_t)(((n >> 1) - 1) & 1), P.err)) { ok = false; break; }
                    umma::mbar_expect_tx(&full[b], (uint32_t)(5 * arr3));
                    const char* src = P.a3 + (size_t)tile * a3_tile_bytes(W);
                    char* dst = A3 + (size_t)b * 5 * arr3;
                    for (int q = 0; q < 5; ++q) umma::bulk_g2s(dst + q * arr3, src + q * arr3, (uint32_t)arr3, &full[b]);
                    ++n;
                }
                if (!ok) break;
            }
            // (normally the MMA lane has waited for every copy; after a wait that gave up,
            // the copies still in flight land before the CTA leaves)
            for (int q = n - 2 < 0 ? 0 : n - 2; q < n; ++q) umma::mbar_wait(&full[q & 1], (uint32_t)((q >> 1) & 1), P.err);
            return;
        }
        if (lane != 0) return;
        umma::mbar_expect_tx(&gfull, (uint32_t)(2 * gbytes));
        umma::bulk_g2s(GT, P.gt_hi, (uint32_t)gbytes, &gfull);
        umma::bulk_g2s(GT + gbytes, P.gt_lo, (uint32_t)gbytes, &gfull);
        bool ok = umma::mbar_wait(&gfull, 0, P.err);
        const uint32_t sbo = (W / 8) * 128;
        const uint32_t id = umma::idesc_f16(128, RP, false, false);
        const uint32_t ghi = umma::smem_u32(GT), glo = ghi + (uint32_t)gbytes;
        int n = 0;
        for (int tag = 0; ok;) {
            const int unit = units.next(P, tag, true);
            if (unit < 0) break;
            for (int k = 0; k < T2 && ok; ++k) {
                const int tile = unit * T2 + k;
                if (!tile_live(P, tile * G2, G2)) continue;
                const int b = n & 1;
                // accumulator b is free once the epilogue has read tile n - 2 out of it
                if (n >= 2 && !umma::mbar_wait(&tfree[b], (uint32_t)(((n >> 1) - 1) & 1), P.err)) { ok = false; break; }
                uint32_t a0;
                if (NB3 == 2) {  // the loader filled buffer b
                    if (!umma::mbar_wait(&full[b], (uint32_t)((n >> 1) & 1), P.err)) { ok = false; break; }
                    a0 = umma::smem_u32(A3 + (size_t)b * 5 * arr3);
                } else {
                    // the one A3 buffer is free once the previous tile's MMAs have completed
                    if (n >= 1 && !umma::mbar_wait(&acc[(n - 1) & 1], (uint32_t)(((n - 1) >> 1) & 1), P.err)) { ok = false; break; }
                    umma::mbar_expect_tx(&full[0], (uint32_t)(5 * arr3));
                    const char* src = P.a3 + (size_t)tile * a3_tile_bytes(W);
                    for (int q = 0; q < 5; ++q) umma::bulk_g2s(A3 + q * arr3, src + q * arr3, (uint32_t)arr3, &full[0]);
                    if (!umma::mbar_wait(&full[0], (uint32_t)(n & 1), P.err)) { ok = false; break; }
                    a0 = umma::smem_u32(A3);
                }
                umma::fence_after_sync();
                const uint32_t td = tbase + (uint32_t)(b * nc);
                mma_chain(td, a0, 128, sbo, 256, ghi, 128, sbo, 256, W, id, false);
                mma_chain(td, a0, 128, sbo, 256, glo, 128, sbo, 256, W, id, true);
                mma_chain(td, a0 + (uint32_t)arr3, 128, sbo, 256, ghi, 128, sbo, 256, W, id, true);
                for (int m = 1; m < 4; ++m)
                    mma_chain(td + m * RP, a0 + (uint32_t)((m + 1) * arr3), 128, sbo, 256, ghi, 128, sbo, 256, W, id,
                              false);
                umma::mma_commit(&acc[b]);
                ++n;
            }
        }
        umma::mma_commit(&fin);
        return;
    }

    // ---------------- epilogue: thread row (g2, j) = t % 128 -> J column k = j of
    // the slot's (map, i') rows; warpgroup = map
    const int row = t & 127, m = t >> 7;
    const int g2 = row / W, j = row % W;
    const int NT = 4 * RP;
    const size_t arrJ = (size_t)NT * W * 2;
    int n = 0;
    bool abort = false;
    for (int tag = 0; !abort;) {
        const int unit = units.next(P, tag);
        if (unit < 0) break;
        for (int k = 0; k < T2 && !abort; ++k) {
            const int tile = unit * T2 + k;
            if (!tile_live(P, tile * G2, G2)) continue;
            const int b = n & 1;
            umma::mbar_wait(&acc[b], (uint32_t)((n >> 1) & 1), P.err);
            umma::fence_after_sync();
            ++n;
            char* a4s = P.a4 + (size_t)(tile * G2 + g2) * a4_slot_bytes(W, RP);
            for (int h = 0; h < RP; h += 16) {
                float v[16];
                umma::tmem_ld16(tmem_lane_addr(tbase, b * nc + m * RP + h), v);
                for (int i8 = 0; i8 < 16; i8 += 8) {
                    const int r = m * RP + h + i8;  // n = (map, i')
                    uint32_t hh[4], ll[4];
#pragma unroll
                    for (int u = 0; u < 8; u += 2)
                        split2(v[i8 + u] * P.sc.cJ[m], v[i8 + u + 1] * P.sc.cJ[m], hh[u / 2], ll[u / 2]);
                    const uint32_t off = mnmajor_off(r, j, NT);
                    store4w(a4s + off, hh);
                    store4w(a4s + arrJ + off, ll);
                }
            }
            umma::fence_before_sync();
            warp_arrive(&tfree[b]);
            units.fence_writes();
            // (a bounded wait that gave up makes every epilogue thread leave the loop together)
            abort = epi_bar_or(t == 0 && *(volatile int*)P.err != 0);
        }
        if (!abort && t == 0) units.release(P, unit, tag + 1);
    }
    if (t == 0) umma::mbar_wait(&fin, 0, P.err);  // every MMA of this CTA has completed
    epi_bar();
    if (t < 32) umma::tmem_dealloc(tbase, 2 * nc);
}

__global__ void __launch_bounds__(S3_THREADS, 1) k_stage3(SplitDev P, FitIO F) {
    if (!cta_has_live_tile(P, P.P / unit_slots(P.G1, P.G2), unit_slots(P.G1, P.G2))) return;
    stage3_body(P, F, StaticUnits{});
}


// ----------------------------------------------------------- stage 4 -------
// Blur along the second index, transposed so that one pixel column lands in
// one TMEM lane: T^T[j'][(map, i')] = sum_j G[j'][j] J[(map, i')][j]
// (A = G padded to 128 rows, B = the slot's J with N = 4 RP).  Model-only
// evaluation: one CTA per slot writes the FP32 maps.
__global__ void __launch_bounds__(SPLIT_THREADS, 1) k_stage4(SplitDev P) {
    extern __shared__ __align__(1024) char smem[];
    const int W = P.W, RP = P.RP, R = P.R, NT = 4 * RP, t = threadIdx.x;
    const uint32_t jarr = (uint32_t)NT * W * 2, garr = 128u * W * 2;
    char* J = smem;  // hi, lo
    char* G = J + 2 * jarr;
    __shared__ __align__(8) uint64_t full, done;
    __shared__ uint32_t tmem_base;
    const int slot = blockIdx.x;
    if (P.slot_roi[slot] < 0) return;
    const int ncols = tmem_cols_pow2(NT);
    if (t < 32) umma::tmem_alloc(&tmem_base, ncols);
    if (t == 0) {
        umma::mbar_init(&full, 1);
        umma::mbar_init(&done, 1);
        umma::mbar_fence_init();
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tbase = tmem_base;
    if (t == 0) {
        umma::mbar_expect_tx(&full, 2 * jarr + 2 * garr);
        umma::bulk_g2s(J, P.a4 + (size_t)slot * a4_slot_bytes(W, RP), 2 * jarr, &full);
        umma::bulk_g2s(G, P.g128_hi, garr, &full);
        umma::bulk_g2s(G + garr, P.g128_lo, garr, &full);
        if (umma::mbar_wait(&full, 0, P.err)) {
            umma::fence_after_sync();
            const uint32_t id = umma::idesc_f16(128, NT, false, true);
            const uint32_t ghi = umma::smem_u32(G), glo = ghi + garr, jhi = umma::smem_u32(J), jlo = jhi + jarr;
            const uint32_t sbo_g = (W / 8) * 128, lbo_j = (NT / 8) * 128, kstep_j = 2 * lbo_j;
            mma_chain(tbase, ghi, 128, sbo_g, 256, jhi, lbo_j, 128, kstep_j, W, id, false);
            mma_chain(tbase, glo, 128, sbo_g, 256, jhi, lbo_j, 128, kstep_j, W, id, true);
            mma_chain(tbase, ghi, 128, sbo_g, 256, jlo, lbo_j, 128, kstep_j, W, id, true);
        }
        umma::mma_commit(&done);
    }
    umma::mbar_wait(&done, 0, P.err);
    umma::fence_after_sync();
    // thread: pixel column j' = its TMEM lane, map = its warpgroup, rows i' = 0..RP-1
    const int jp = t & 127, map = t >> 7;
    float* dst = P.tmaps + ((size_t)slot * 4 + map) * R * R;
    for (int h = 0; h < RP; h += 4) {
        float v[4];
        umma::tmem_ld4(tmem_lane_addr(tbase, map * RP + h), v);
        if (jp < R)
            for (int u = 0; u < 4 && h + u < R; ++u) dst[(size_t)(h + u) * R + jp] = v[u] * P.sc.cT[map];
    }
    umma::fence_before_sync();
    __syncthreads();
    if (t < 32) umma::tmem_dealloc(tbase, ncols);
}

// ----------------------------------------------------------- stage 5 -------
constexpr int NRED = 1 + 5 + 15 + 15;

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
    float y = v - c;
    float t2 = s + y;
    c = (t2 - s) - y;
    s = t2;
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Butterfly reduce-scatter of 32 per-lane values: after 31 shuffles lane k
// holds the warp total of value k (the plain form needs 5 shuffles per value).
__device__ __forceinline__ float warp_reduce_scatter32f(float (&v)[32], int lane) {
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) {
        const bool up = (lane & h) != 0;
#pragma unroll
        for (int i = 0; i < h; ++i) {
            const float send = up ? v[i] : v[i + h], keep = up ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, h);
        }
    }
    return v[0];
}

// A warp's totals of the 36 per-thread likelihood sums into red[0..35]: the
// likelihood and gradient (s6 - c6, the caller's compensated FP32 sums) in
// FP64, the 30 Gauss-Newton Hessian and Fisher terms by the FP32 butterfly
// (their relative rounding, about 2^-21, is far below what the LM step and
// the CRLB need), so that no per-thread FP64 array is held.
__device__ __forceinline__ void warp_sums36(const float (&s6)[6], const float (&c6)[6], const float (&sh)[30],
                                            double* red, int lane) {
    float w[32];
#pragma unroll
    for (int k = 0; k < 30; ++k) w[k] = sh[k];
    w[30] = 0.f;
    w[31] = 0.f;
    const float hk = warp_reduce_scatter32f(w, lane);
    if (lane < 30) red[6 + lane] = (double)hk;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const double x = warp_sum((double)s6[k] - (double)c6[k]);
        if (lane == k) red[k] = x;
    }
}

constexpr int NSUM = NRED + 1;  // sums per slot: NRED + the non-positive-model flag

// The FP64 LM step of one slot from its sums: start or update the damped
// Gauss-Newton iteration, propose the next trial point, or retire the ROI and
// refill the slot from the queue.
__device__ __noinline__ void lm_slot(const SplitDev& P, const FitIO& io, int slot) {
    const FitParamsDev& prm = io.prm;
    const int roi = P.slot_roi[slot];
    if (roi < 0) return;
    const double* tot = P.sums + (size_t)slot * NSUM;
    double nll = tot[NRED] != 0.0 ? INFINITY : tot[0], g[5], H[25], F[25];
    for (int q = 0; q < 5; ++q) g[q] = tot[1 + q];
    int o = 6;
    for (int q = 0; q < 5; ++q)
        for (int r2 = 0; r2 <= q; ++r2) {
            H[q * 5 + r2] = H[r2 * 5 + q] = tot[o];
            F[q * 5 + r2] = F[r2 * 5 + q] = tot[o + 15];
            ++o;
        }
    // the step works on a local copy of the slot state (written back once)
    LMState st = P.lm[slot];
    if (P.slot_phase[slot] == 0) {
        for (int q = 0; q < 5; ++q) st.th[q] = st.trial[q];
        lm_start(st, nll, g, H, F, prm);
        P.slot_phase[slot] = 1;
    } else {
        lm_update(st, nll, g, H, F, prm);
    }
    const bool more = lm_propose(st, prm);
    P.lm[slot] = st;
    if (more) return;
    // retire
    for (int q = 0; q < 5; ++q) io.out5[5 * roi + q] = st.th[q];
    if (io.nll) io.nll[roi] = st.nll;
    if (io.status) io.status[roi] = st.status;
    if (io.iters) io.iters[roi] = st.evals;
    if (io.crlb5) lm_crlb(st.F, io.crlb5 + 5 * roi);
    // refill from the queue
    const int next = take_roi(P, io.n);
    if (next >= 0) {
        slot_take(P, io, slot, next);
    } else {
        P.slot_roi[slot] = -1;
        atomicSub(P.active, 1);
    }
}

// The round-based fit's LM step: every occupied slot of the pool, one thread each.
__global__ void k_lm(SplitDev P, FitIO F) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = slot < P.P && P.slot_roi[slot] >= 0;
    const unsigned m = __ballot_sync(0xffffffffu, live);  // model evaluations: one atomic per warp
    if (P.evals && (threadIdx.x & 31) == 0 && m) atomicAdd(P.evals, (unsigned long long)__popc(m));
    if (live) lm_slot(P, F, slot);
}

// ------------------------------------------------- LM stage (dataflow) -----
// The FP64 LM steps of the dataflow kernel.  Warp k of an LM CTA owns the
// units first + (k + i warps) stride and polls their state words; when a
// unit's sums are done, lanes 0 .. UG - 1 apply the LM step to the unit's slots
// (retiring converged fits and refilling their slots) and lane 0 publishes the
// unit's next state.  One unit per warp, so the LM steps of different units
// overlap, and many units are stepped at once: the FP64 work never holds up
// the tensor-core stages.
__device__ void lm_role(const SplitDev& P, const FitIO& F, int first, int stride) {
    const int UG = unit_slots(P.G1, P.G2), U = P.P / UG;
    const int lane = threadIdx.x & 31, g = lane, lead = 0;
    const unsigned gmask = 0xffffffffu;
    const int group = (int)threadIdx.x >> 5, ngroups = (int)blockDim.x >> 5;
    __shared__ unsigned long long busy_sum, units_done;
    __shared__ int owners;
    if (threadIdx.x == 0) {
        busy_sum = 0;
        units_done = 0;
        owners = 0;
    }
    __syncthreads();
    const long long start = clock64();
    long long busy = 0, idle_since = start;
    int mine = 0, done_units = 0;
    for (int u = first + group * stride; u < U; u += ngroups * stride) ++mine;
    if (mine && g == 0) atomicAdd(&owners, 1);
    // every decision that ends a loop is taken by the group's first lane and
    // broadcast, so the lanes of a group stay together
    const unsigned long long cap = (unsigned long long)F.n * (F.prm.max_iter + 1) + 2ull * P.P;
    for (;;) {
        int ctl = 0;
        if (g == 0) ctl = *(volatile int*)P.err != 0;
        if (__shfl_sync(gmask, ctl, lead)) break;
        bool any = false;
        int dead = 0;
        for (int u = first + group * stride; u < U; u += ngroups * stride) {
            int v = 0;
            if (g == 0) v = ld_acquire(P.ustate + u);
            v = __shfl_sync(gmask, v, lead);
            if (v < 0) {
                ++dead;
                continue;
            }
            // (a unit another stage handed out carries the claim bit; this stage claims none)
            if ((v & UNIT_CLAIMED) || v % FLOW_STAGES != FLOW_STAGES - 1) continue;
            const long long b0 = clock64();
            const bool lv = g < UG && P.slot_roi[u * UG + g] >= 0;
            const unsigned lmask = __ballot_sync(gmask, lv);
            if (g == 0 && lmask) atomicAdd(P.evals, (unsigned long long)__popc(lmask));
            if (lv) lm_slot(P, F, u * UG + g);
            __syncwarp(gmask);
            // every ROI takes at most max_iter evaluations: more means the fit lost
            // track of its slots, and the whole kernel stops with an error
            int stop = 0;
            if (g == 0) stop = *(volatile unsigned long long*)P.evals > cap;
            if (__shfl_sync(gmask, stop, lead)) {
                if (g == 0) atomicExch(P.err, 3);
                break;
            }
            if (g == 0) {
                __threadfence();
                st_release(P.ustate + u, unit_after_lm(P, F, u, v));
                ++done_units;
            }
            busy += clock64() - b0;
            any = true;
        }
        if (dead == mine) break;
        if (any) {
            idle_since = clock64();
            continue;
        }
        int late = 0;
        if (g == 0) late = clock64() - idle_since > P.wait_limit;
        if (__shfl_sync(gmask, late, lead)) {
            if (g == 0) atomicExch(P.err, 2);
            break;
        }
        __nanosleep(200);
    }
    if (g == 0) {
        atomicAdd(&busy_sum, (unsigned long long)busy);
        atomicAdd(&units_done, (unsigned long long)done_units);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const long long total = clock64() - start;
        const long long used = owners ? (long long)(busy_sum / (unsigned long long)owners) : 0;
        P.clk[3 * blockIdx.x] = (unsigned long long)(total > used ? total - used : 0);
        P.clk[3 * blockIdx.x + 1] = (unsigned long long)total;
        P.clk[3 * blockIdx.x + 2] = units_done;
    }
}

// ---------------------------------- stages 4 + 5 sums (persistent) -----
// ROIs of 33 px and more (window 128).  One CTA per SM walks the occupied slots.  The column blur is computed
// transposed, T^T[j'][(map, i')] = sum_j G[j'][j] J[(map, i')][j] (A = G
// padded to 128 rows, resident in shared memory; B = the slot's J, N = 4 RP,
// streamed in K-slabs by a producer warp; three FP16 products per K step
// issued by an MMA warp into one of two TMEM buffers), so TMEM lane j' holds
// all four maps of pixel column j'.  The epilogue warps read them straight
// from TMEM and form the normalisation, likelihood, gradient, Gauss-Newton
// Hessian and Fisher sums (process/cpu/Localization.java:1125-1143 with the
// Jacobian of psi = |T|/sum|T| of PSFPhase.java:602-629): per-pixel terms in
// FP32 (a thread sums a few pixels), thread partials combined in FP64.  The
// next slot's MMAs run in the other TMEM buffer meanwhile.  The sums and a
// non-positive-model flag go to P.sums; once a unit's slots are summed, one
// lane per slot applies the FP64 LM step.
constexpr int E45_THREADS = 384;                 // 12 epilogue warps: three per TMEM lane quadrant
constexpr int S45_THREADS = E45_THREADS + 64;    // + producer warp + MMA warp
constexpr int S45_NBUF = 4;
// ROIs whose window is 128 take this kernel, smaller ones the warp-per-slot
// sums (stage45s).  The choice depends on R only, never on the batch, so a
// ROI's fit is the same bit for bit in any batch.
constexpr int S45_MIN_W = 128;

__host__ __device__ inline size_t s45_roi_bytes(int R) { return ((size_t)R * R * 4 + 127) / 128 * 128; }


template <class UNITS>
__device__ __forceinline__ void stage45_body(const SplitDev& P, const FitIO& F, UNITS units) {
    extern __shared__ __align__(1024) char smem[];
    const int W = P.W, RP = P.RP, R = P.R, NT = 4 * RP, RR = R * R, t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31, NS4 = W / 16, UG = unit_slots(P.G1, P.G2);
    const float* rois = F.rois;
    const float* scmos = F.scmos;
    if (t >= S45_THREADS) {  // (a dataflow CTA has more threads than this stage uses)
        __syncthreads();
        return;
    }
    const uint32_t garr = 128u * W * 2, kslab = 32u * NT, ringb = 2 * kslab, roib = (uint32_t)s45_roi_bytes(R);
    char* G = smem;                      // G hi, lo
    char* RG = G + 2 * garr;             // ring of J K-slabs (hi, lo)
    char* RO = RG + S45_NBUF * ringb;    // two buffers of (ROI, sCMOS variance)
    float* Tm = (float*)(RO + 4 * roib); // the slot's four FP32 maps, row stride RS
    const int RS = tm_stride(R), MS = R * RS;
    double (*red)[NRED] = (double (*)[NRED])(((uintptr_t)(Tm + 4 * MS) + 15) & ~(uintptr_t)15);  // per-warp sums
    double (*nrm4)[4] = (double (*)[4])(red + E45_THREADS / 32);  // per-warp normalisation sums
    int* bad_w = (int*)(nrm4 + E45_THREADS / 32);
    const bool vec = (R % 2) == 0;       // whole 16-byte units: ROI copies by TMA
    __shared__ __align__(8) uint64_t gfull, full[S45_NBUF], freed[S45_NBUF], acc[2], tfree[2], rfull[2], rfree[2], fin;
    __shared__ uint32_t tmem_base;
    const int ncols = tmem_cols_pow2(2 * NT);
    if (t < 32) umma::tmem_alloc(&tmem_base, ncols);
    if (t == 0) {
        umma::mbar_init(&gfull, 1);
        for (int b = 0; b < S45_NBUF; ++b) { umma::mbar_init(&full[b], 1); umma::mbar_init(&freed[b], 1); }
        for (int b = 0; b < 2; ++b) {
            umma::mbar_init(&acc[b], 1);
            umma::mbar_init(&tfree[b], E45_THREADS / 32);
            umma::mbar_init(&rfull[b], 1);
            umma::mbar_init(&rfree[b], E45_THREADS / 32);
        }
        umma::mbar_init(&fin, 1);
        umma::mbar_fence_init();
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tbase = tmem_base;

    if (warp == E45_THREADS / 32) {  // ---------------- producer (lane 0), scheduler (lane 1)
        if constexpr (UNITS::flow)
            if (lane == 1) {
                units.schedule(P, F);
                return;
            }
        if (lane != 0) return;
        umma::mbar_expect_tx(&gfull, 2 * garr);
        umma::bulk_g2s(G, P.g128_hi, garr, &gfull);
        umma::bulk_g2s(G + garr, P.g128_lo, garr, &gfull);
        int q = 0, n = 0;
        bool ok = true;
        for (int tag = 0; ok;) {
            const int unit = units.next(P, tag, true);
            if (unit < 0) break;
            for (int slot = unit * UG; slot < (unit + 1) * UG && ok; ++slot) {
                const int roi = P.slot_roi[slot];
                if (roi < 0) continue;
                const int b = n & 1;
                if (vec) {
                    if (n >= 2 && !umma::mbar_wait(&rfree[b], (uint32_t)(((n >> 1) - 1) & 1), P.err)) {
                        ok = false;
                        break;
                    }
                    char* dst = RO + b * 2 * roib;
                    umma::mbar_expect_tx(&rfull[b], (scmos ? 2u : 1u) * RR * 4);
                    umma::bulk_g2s(dst, rois + (size_t)roi * RR, RR * 4, &rfull[b]);
                    if (scmos) umma::bulk_g2s(dst + roib, scmos + (size_t)roi * RR, RR * 4, &rfull[b]);
                }
                ++n;
                const char* src = P.a4 + (size_t)slot * a4_slot_bytes(W, RP);
                for (int s = 0; s < NS4; ++s, ++q) {
                    const int buf = q % S45_NBUF;
                    if (q >= S45_NBUF && !umma::mbar_wait(&freed[buf], (uint32_t)((q / S45_NBUF - 1) & 1), P.err)) {
                        ok = false;
                        break;
                    }
                    umma::mbar_expect_tx(&full[buf], ringb);
                    umma::bulk_g2s(RG + buf * ringb, src + (size_t)s * kslab, kslab, &full[buf]);
                    umma::bulk_g2s(RG + buf * ringb + kslab, src + (size_t)NT * W * 2 + (size_t)s * kslab, kslab, &full[buf]);
                }
            }
        }
        // copies still in flight land before the CTA can exit
        umma::mbar_wait(&gfull, 0, P.err);
        for (int j = q > S45_NBUF ? q - S45_NBUF : 0; j < q; ++j)
            umma::mbar_wait(&full[j % S45_NBUF], (uint32_t)((j / S45_NBUF) & 1), P.err);
        if (vec)
            for (int m = n > 2 ? n - 2 : 0; m < n; ++m) umma::mbar_wait(&rfull[m & 1], (uint32_t)((m >> 1) & 1), P.err);
        return;
    }
    if (warp == E45_THREADS / 32 + 1) {  // ---------------- MMA issuer (lane 0)
        if (lane != 0) return;
        const uint32_t id = umma::idesc_f16(128, NT, false, true);
        const uint32_t sbo_g = (W / 8) * 128, lbo_j = (NT / 8) * 128;
        const uint32_t ghi = umma::smem_u32(G), glo = ghi + garr;
        bool ok = umma::mbar_wait(&gfull, 0, P.err);
        int q = 0, n = 0;
        for (int tag = 0; ok;) {
            const int unit = units.next(P, tag, true);
            if (unit < 0) break;
            for (int slot = unit * UG; slot < (unit + 1) * UG && ok; ++slot) {
                if (P.slot_roi[slot] < 0) continue;
                const int b = n & 1;
                if (n >= 2 && !umma::mbar_wait(&tfree[b], (uint32_t)(((n >> 1) - 1) & 1), P.err)) {
                    ok = false;
                    break;
                }
                umma::fence_after_sync();
                const uint32_t td = tbase + b * NT;
                for (int s = 0; s < NS4; ++s, ++q) {
                    const int buf = q % S45_NBUF;
                    if (!umma::mbar_wait(&full[buf], (uint32_t)((q / S45_NBUF) & 1), P.err)) { ok = false; break; }
                    umma::fence_after_sync();
                    const uint32_t jhi = umma::smem_u32(RG + buf * ringb), jlo = jhi + kslab;
                    const uint64_t gh = umma::smem_desc(ghi + s * 256, 128, sbo_g), gl = umma::smem_desc(glo + s * 256, 128, sbo_g);
                    const uint64_t bh = umma::smem_desc(jhi, lbo_j, 128), bl = umma::smem_desc(jlo, lbo_j, 128);
                    umma::mma_f16(td, gh, bh, id, s > 0 ? 1u : 0u);
                    umma::mma_f16(td, gl, bh, id, 1u);
                    umma::mma_f16(td, gh, bl, id, 1u);
                    umma::mma_commit(&freed[buf]);
                }
                umma::mma_commit(&acc[b]);
                ++n;
            }
        }
        umma::mma_commit(&fin);
        return;
    }

    // ---------------- epilogue warps.  The maps go from TMEM (lane = pixel column j') to
    // shared memory, which frees the TMEM buffer for the slot after next; the pixel sums
    // then run over all epilogue threads.
    const int jp = (warp & 3) * 32 + lane, wg = warp >> 2;
    constexpr int NWG = E45_THREADS / 128, NW = E45_THREADS / 32;
    int n = 0;
    bool abort = false;
    for (int tag = 0; !abort;) {
        const int unit = units.next(P, tag);
        if (unit < 0) break;
        for (int slot = unit * UG; slot < (unit + 1) * UG; ++slot) {
            const int roi = P.slot_roi[slot];
            if (roi < 0) continue;
            const int b = n & 1;
            const uint32_t ph = (uint32_t)((n >> 1) & 1);
            ++n;
            umma::mbar_wait(&acc[b], ph, P.err);
            umma::fence_after_sync();
            const uint32_t tb = tbase + b * NT;
            // the normalisation sums accumulate over the values this thread copies
            float ns[4] = {0, 0, 0, 0};
            for (int c0 = 4 * wg; c0 < RP; c0 += 4 * NWG) {
                uint32_t r[4][4];
#pragma unroll
                for (int m = 0; m < 4; ++m) umma::tmem_ld4_nw(tmem_lane_addr(tb, m * RP + c0), r[m]);
                umma::tmem_wait_ld();
#pragma unroll
                for (int m = 0; m < 4; ++m)
#pragma unroll
                    for (int u = 0; u < 4; ++u) asm volatile("" : "+r"(r[m][u]));
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    if (jp >= R || c0 + u >= R) continue;
                    float v[4];
#pragma unroll
                    for (int m = 0; m < 4; ++m) {
                        v[m] = __uint_as_float(r[m][u]) * P.sc.cT[m];
                        Tm[m * MS + (c0 + u) * RS + jp] = v[m];
                    }
                    const float sg = v[0] < 0 ? -1.f : 1.f;
                    ns[0] += fabsf(v[0]);
                    ns[1] += sg * v[1];
                    ns[2] += sg * v[2];
                    ns[3] += sg * v[3];
                }
            }
            umma::fence_before_sync();
            warp_arrive(&tfree[b]);
            if (vec) umma::mbar_wait(&rfull[b], ph, P.err);
            {
                const double v0 = warp_sum(ns[0]), v1 = warp_sum(ns[1]), v2 = warp_sum(ns[2]), v3 = warp_sum(ns[3]);
                if (lane == 0) { nrm4[warp][0] = v0; nrm4[warp][1] = v1; nrm4[warp][2] = v2; nrm4[warp][3] = v3; }
            }
            // the maps and norms are in; in the round-based kernel this barrier also takes the
            // vote on a bounded wait that gave up (every epilogue thread leaves the loop together)
            if (epi_bar_or<E45_THREADS>(!UNITS::flow && t == 0 && *(volatile int*)P.err != 0)) {
                abort = true;
                break;
            }
            double sum4[4] = {0, 0, 0, 0};
            for (int w = 0; w < NW; ++w)
                for (int q = 0; q < 4; ++q) sum4[q] += nrm4[w][q];
            const float S = (float)sum4[0], Dx = (float)sum4[1], Dy = (float)sum4[2], Dz = (float)sum4[3];
            const float invS = 1.f / S;
            const double* th = P.lm[slot].trial;
            const float A = (float)th[3], B = (float)th[4];
            const float* d = vec ? (const float*)(RO + b * 2 * roib) : rois + (size_t)roi * RR;
            const float* sv = !scmos ? nullptr : vec ? (const float*)(RO + b * 2 * roib + roib) : scmos + (size_t)roi * RR;
            // a thread sums about RR / 384 pixels before the FP64 combination across threads,
            // so plain FP32 partials suffice here
            float sg6[6], sh[30];
#pragma unroll
            for (int k = 0; k < 6; ++k) sg6[k] = 0.f;
#pragma unroll
            for (int k = 0; k < 30; ++k) sh[k] = 0.f;
            bool bad = false;
            // pixel k = ip R + jc of the maps' rows (stride RS), stepped without a division
            int ip = t / R, jc = t - (t / R) * R;
            const int dq = E45_THREADS / R, dr = E45_THREADS - (E45_THREADS / R) * R;
#pragma unroll 3
            for (int k = t; k < RR; k += E45_THREADS) {
                const int to = ip * RS + jc;
                ip += dq;
                jc += dr;
                if (jc >= R) {
                    jc -= R;
                    ++ip;
                }
                const float v = Tm[to], sgn = v < 0 ? -1.f : 1.f, psi = fabsf(v) * invS;
                float jv[5];
                jv[0] = A * (sgn * Tm[MS + to] - psi * Dx) * invS;
                jv[1] = A * (sgn * Tm[2 * MS + to] - psi * Dy) * invS;
                jv[2] = A * (sgn * Tm[3 * MS + to] - psi * Dz) * invS;
                jv[3] = psi;
                jv[4] = 1.f;
                const float mu = A * psi + B + (sv ? sv[k] : 0.f);
                if (!(mu > 0.f)) { bad = true; continue; }
                const float dk = d[k];
                sg6[0] += dk > 0.f ? mu - dk - dk * logf(mu / dk) : mu;
                const float wf = 1.f / mu, wgt = 1.f - dk * wf, wh = dk * wf * wf;
#pragma unroll
                for (int q = 0; q < 5; ++q) sg6[1 + q] += wgt * jv[q];
                int o = 0;
#pragma unroll
                for (int q = 0; q < 5; ++q)
#pragma unroll
                    for (int r2 = 0; r2 <= q; ++r2) {
                        sh[o] += wh * jv[q] * jv[r2];
                        sh[o + 15] += wf * jv[q] * jv[r2];
                        ++o;
                    }
            }
            if (vec) warp_arrive(&rfree[b]);  // this slot's ROI buffer is free for the slot after next
            {
                const float zero6[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                warp_sums36(sg6, zero6, sh, red[warp], lane);
            }
            const bool wbad = __any_sync(0xffffffffu, bad);
            if (lane == 0) bad_w[warp] = wbad;
            epi_bar<E45_THREADS>();
            if (t < NRED) {
                double v = 0;
                for (int w = 0; w < NW; ++w) v += red[w][t];
                P.sums[(size_t)slot * NSUM + t] = v;
            }
            if (t == NRED) {
                int any = 0;
                for (int w = 0; w < NW; ++w) any |= bad_w[w];
                P.sums[(size_t)slot * NSUM + NRED] = any ? 1.0 : 0.0;
            }
            // The dataflow kernel publishes the unit once its sums are written, behind this
            // barrier, which also takes the vote on a bounded wait that gave up.  The
            // round-based kernel needs neither: the next slot's first barrier orders the
            // sums and maps against their next writers.
            if constexpr (UNITS::flow) {
                if (epi_bar_or<E45_THREADS>(t == 0 && *(volatile int*)P.err != 0)) {
                    abort = true;
                    break;
                }
            }
        }
        if (abort) break;
        if (t == 0) units.release(P, unit, tag + 1);  // (flow: the sums were written before the last barrier)
    }
    if (t == 0) umma::mbar_wait(&fin, 0, P.err);  // every MMA of this CTA has completed
    epi_bar<E45_THREADS>();
    if (t < 32) umma::tmem_dealloc(tbase, ncols);
}

__global__ void __launch_bounds__(S45_THREADS, 1) k_stage45p(SplitDev P, FitIO F) {
    if (!cta_has_live_tile(P, P.P / unit_slots(P.G1, P.G2), unit_slots(P.G1, P.G2))) return;
    stage45_body(P, F, StaticUnits{});
}

// Likelihood sums of a unit's live slots from their maps in shared memory (slot
// g, map m at Tm + (4 g + m) R^2, row-major), all 16 epilogue warps at once:
// 16 / UG warps per slot, each thread summing strided pixels (per-pixel terms
// in FP32; the normalisation, likelihood and gradient with Kahan
// compensation), warp partials combined in FP64 in a fixed order.  Writes
// P.sums; the caller's next barrier publishes them.
template <int NTG>
__device__ __noinline__ void unit_sums(const SplitDev& P, const FitIO& F, int unit, const float* Tm,
                                       double (*red)[NRED], double (*nrm)[4], int* badw, int t, int bar_id) {
    const int warp = t >> 5, lane = t & 31, UG = unit_slots(P.G1, P.G2);
    const int wps = (NTG / 32) / UG, g = warp / wps, ws = warp - g * wps;
    const int tid = ws * 32 + lane, nts = wps * 32, R = P.R, RR = R * R;
    const int slot = unit * UG + g, roi = P.slot_roi[slot];
    const float* T0 = Tm + (size_t)g * 4 * RR;
    {
        float ns[4] = {0, 0, 0, 0}, nc = 0.f;
        if (roi >= 0)
            for (int k = tid; k < RR; k += nts) {
                const float v = T0[k], sg = v < 0 ? -1.f : 1.f;
                kahan_add(ns[0], nc, fabsf(v));
                ns[1] += sg * T0[RR + k];
                ns[2] += sg * T0[2 * RR + k];
                ns[3] += sg * T0[3 * RR + k];
            }
        const double v0 = warp_sum((double)ns[0] - (double)nc), v1 = warp_sum(ns[1]), v2 = warp_sum(ns[2]),
                     v3 = warp_sum(ns[3]);
        if (lane == 0) { nrm[warp][0] = v0; nrm[warp][1] = v1; nrm[warp][2] = v2; nrm[warp][3] = v3; }
    }
    group_bar<NTG>(bar_id);
    double s4[4] = {0, 0, 0, 0};
    for (int w = g * wps; w < (g + 1) * wps; ++w)
        for (int q = 0; q < 4; ++q) s4[q] += nrm[w][q];
    const float S = (float)s4[0], Dx = (float)s4[1], Dy = (float)s4[2], Dz = (float)s4[3];
    const float invS = 1.f / S;
    float sg6[6], cg6[6], sh[30];
#pragma unroll
    for (int k = 0; k < 6; ++k) { sg6[k] = 0.f; cg6[k] = 0.f; }
#pragma unroll
    for (int k = 0; k < 30; ++k) sh[k] = 0.f;
    bool bad = false;
    if (roi >= 0) {
        const double* th = P.lm[slot].trial;
        const float A = (float)th[3], B = (float)th[4];
        const float* d = F.rois + (size_t)roi * RR;
        const float* sv = F.scmos ? F.scmos + (size_t)roi * RR : nullptr;  // sCMOS var/gain^2 (Localization.java:1132)
        for (int k = tid; k < RR; k += nts) {
            const float v = T0[k], sgn = v < 0 ? -1.f : 1.f, psi = fabsf(v) * invS;
            float j[5];
            j[0] = A * (sgn * T0[RR + k] - psi * Dx) * invS;
            j[1] = A * (sgn * T0[2 * RR + k] - psi * Dy) * invS;
            j[2] = A * (sgn * T0[3 * RR + k] - psi * Dz) * invS;
            j[3] = psi;
            j[4] = 1.f;
            const float mu = A * psi + B + (sv ? sv[k] : 0.f);
            if (!(mu > 0.f)) { bad = true; continue; }
            const float dk = d[k];
            kahan_add(sg6[0], cg6[0], dk > 0.f ? mu - dk - dk * logf(mu / dk) : mu);
            const float wgt = 1.f - dk / mu, wf = 1.f / mu, wh = dk * wf * wf;
#pragma unroll
            for (int q = 0; q < 5; ++q) kahan_add(sg6[1 + q], cg6[1 + q], wgt * j[q]);
            int o = 0;
#pragma unroll
            for (int q = 0; q < 5; ++q)
#pragma unroll
                for (int r2 = 0; r2 <= q; ++r2) {
                    sh[o] += wh * j[q] * j[r2];
                    sh[o + 15] += wf * j[q] * j[r2];
                    ++o;
                }
        }
    }
    warp_sums36(sg6, cg6, sh, red[warp], lane);
    const bool wbad = __any_sync(0xffffffffu, bad);
    if (lane == 0) badw[warp] = wbad;
    group_bar<NTG>(bar_id);
    for (int i = t; i < UG * (NRED + 1); i += NTG) {
        const int gg = i / (NRED + 1), k = i - gg * (NRED + 1), sl = unit * UG + gg;
        if (P.slot_roi[sl] < 0) continue;
        if (k < NRED) {
            double v = 0;
            for (int w = gg * wps; w < (gg + 1) * wps; ++w) v += red[w][k];
            P.sums[(size_t)sl * NSUM + k] = v;
        } else {
            int any = 0;
            for (int w = gg * wps; w < (gg + 1) * wps; ++w) any |= badw[w];
            P.sums[(size_t)sl * NSUM + NRED] = any ? 1.0 : 0.0;
        }
    }
}

// ------------------------------ stages 4 + 5 for small ROIs (persistent) -----
// ROIs whose window is 32 or 64.  One CTA per SM walks the units: warp 16
// loads a unit's row-blurred maps J (hi, lo; all UG slots at once) into one
// of two buffers and issues the column blur of each live slot,
// T^T[j'][(map, i')] = sum_j G[j'][j] J[(map, i')][j] (A = G padded to 128
// rows, resident), into one of two TMEM accumulators.  The epilogue warps copy
// the maps to shared memory (lane = pixel column j', warpgroup = map), then
// form the likelihood sums of the unit's slots (unit_sums); the LM step
// follows in its own stage.
constexpr int S45S_THREADS = SPLIT_THREADS + 32;

// Map areas of the epilogue: two warp groups of 256 threads, each summing its
// own unit (units alternate between them, with the J buffers and TMEM
// accumulators), when there are two buffers; one group of 512 threads
// otherwise.  The choice depends on the class alone, so the round-based and
// dataflow kernels sum in the same order.
__host__ __device__ inline int s45s_groups(int nb) { return nb == 2 ? 2 : 1; }
__host__ __device__ inline size_t s45s_smem(int W, int RP, int R, int UG, int nb, int groups = 1) {
    return (size_t)2 * 128 * W * 2 + (size_t)nb * UG * a4_slot_bytes(W, RP) + (size_t)groups * UG * 4 * R * R * 4 +
           16 + (size_t)(SPLIT_THREADS / 32) * ((NRED + 4) * 8 + 4);
}
// J buffers and TMEM accumulators: two when they fit (the next unit's load and
// MMAs overlap this unit's epilogue), else one.
__host__ __device__ inline int s45s_nbuf(int W, int RP, int R, int UG) {
    return 2 * UG * 4 * RP <= 512 && s45s_smem(W, RP, R, UG, 2, s45s_groups(2)) <= 225 * 1024 ? 2 : 1;
}

// The epilogue of one group of NTG threads (tg its thread index, bar_id its
// barrier): the maps of each unit it owns from TMEM to shared memory (pixel
// column j' = TMEM lane; 4 NTG / 512 maps a thread), then the unit's sums.
template <int NTG, class UNITS>
__device__ __forceinline__ void s45s_epilogue(const SplitDev& P, const FitIO& F, UNITS& units, int NB, int grp,
                                              int tg, int bar_id, uint32_t tbase, float* Tm, double (*red)[NRED],
                                              double (*nrm)[4], int* badw, uint64_t* acc, uint64_t* tfree) {
    constexpr int NG = SPLIT_THREADS / NTG;  // groups
    const int R = P.R, RP = P.RP, NT = 4 * RP, RR = R * R, UG = unit_slots(P.G1, P.G2), nc = UG * NT;
    const int jp = tg & 127;
    int n = 0;
    bool abort = false;
    for (int tag = 0; !abort;) {
        const int unit = units.next(P, tag);
        if (unit < 0) break;
        const int b = n % NB;
        const uint32_t par = (uint32_t)((n / NB) & 1);
        ++n;
        if (NG == 2 && b != grp) continue;  // the other group's unit
        umma::mbar_wait(&acc[b], par, P.err);
        umma::fence_after_sync();
#pragma unroll
        for (int mi = 0; mi < NG; ++mi) {
            const int map = NG == 1 ? (tg >> 7) : 2 * (tg >> 7) + mi;
            const float cT = P.sc.cT[map];
            if (UG * RP == 64) {
                // the whole unit's columns of this map and lane (8 groups of 8) in flight before one wait
                uint32_t ad[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int g = q / (RP / 8), h = (q - g * (RP / 8)) * 8;
                    ad[q] = tmem_lane_addr(tbase, b * nc + g * NT + map * RP + h);
                }
                float v[8][8];
                tmem_ld8_multi<8>(ad, v);
                if (jp < R)
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int g = q / (RP / 8), h = (q - g * (RP / 8)) * 8;
                        if (P.slot_roi[unit * UG + g] < 0) continue;
                        float* dst = Tm + (size_t)(g * 4 + map) * RR;
#pragma unroll
                        for (int u = 0; u < 8; ++u)
                            if (h + u < R) dst[(h + u) * R + jp] = v[q][u] * cT;
                    }
            } else {
                for (int g = 0; g < UG; ++g) {
                    if (P.slot_roi[unit * UG + g] < 0) continue;
                    float* dst = Tm + (size_t)(g * 4 + map) * RR;
                    for (int h = 0; h < RP; h += 16) {  // 16 columns a wait
                        const uint32_t ad[2] = {tmem_lane_addr(tbase, b * nc + g * NT + map * RP + h),
                                                tmem_lane_addr(tbase, b * nc + g * NT + map * RP + h + 8)};
                        float v[2][8];
                        tmem_ld8_multi<2>(ad, v);
                        if (jp < R)
#pragma unroll
                            for (int u = 0; u < 16; ++u)
                                if (h + u < R) dst[(h + u) * R + jp] = v[u >> 3][u & 7] * cT;
                    }
                }
            }
        }
        umma::fence_before_sync();
        warp_arrive(&tfree[b]);
        // the maps are in; in the round-based kernel this barrier also takes the vote on a
        // bounded wait that gave up (every thread of the group leaves the loop together)
        if (group_bar_or<NTG>(bar_id, !UNITS::flow && tg == 0 && *(volatile int*)P.err != 0)) break;
        unit_sums<NTG>(P, F, unit, Tm, red, nrm, badw, tg, bar_id);
        // The dataflow kernel publishes the unit once its sums are written, behind this
        // barrier (with the vote); the round-based kernel needs neither: the next unit's
        // first barrier orders the sums and maps against their next writers.
        if constexpr (UNITS::flow) {
            abort = group_bar_or<NTG>(bar_id, tg == 0 && *(volatile int*)P.err != 0);
            if (!abort && tg == 0) units.release(P, unit, tag + 1);
        }
    }
}

template <class UNITS>
__device__ __forceinline__ void stage45s_body(const SplitDev& P, const FitIO& F, UNITS units) {
    extern __shared__ __align__(1024) char smem[];
    const int W = P.W, RP = P.RP, R = P.R, NT = 4 * RP, RR = R * R, t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int UG = unit_slots(P.G1, P.G2);
    const uint32_t garr = 128u * W * 2, jslot = (uint32_t)a4_slot_bytes(W, RP), jarr = jslot / 2;
    char* G = smem;                                      // G hi, lo (128 rows, rows >= R zero)
    const int NB = s45s_nbuf(W, RP, R, UG);
    const int NGRP = s45s_groups(NB);
    char* JB = G + 2 * garr;                             // NB buffers of a unit's J
    float* Tm = (float*)(JB + (size_t)NB * UG * jslot);  // per group, a unit's maps: slot g, map m at (4 g + m) R^2
    double (*red)[NRED] =
        (double (*)[NRED])(((uintptr_t)(Tm + (size_t)NGRP * UG * 4 * RR) + 15) & ~(uintptr_t)15);
    double (*nrm)[4] = (double (*)[4])(red + SPLIT_THREADS / 32);  // per-warp sums: likelihood terms, normalisation
    int* badw = (int*)(nrm + SPLIT_THREADS / 32);
    __shared__ __align__(8) uint64_t gfull, full[2], acc[2], tfree[2], fin;
    __shared__ uint32_t tmem_base;
    const int nc = UG * NT;  // TMEM columns of one unit
    const int ncols = tmem_cols_pow2(NB * nc);
    if (t < 32) umma::tmem_alloc(&tmem_base, ncols);
    if (t == 0) {
        umma::mbar_init(&gfull, 1);
        for (int b = 0; b < 2; ++b) {
            umma::mbar_init(&full[b], 1);
            umma::mbar_init(&acc[b], 1);
            umma::mbar_init(&tfree[b], SPLIT_THREADS / 32 / NGRP);  // the warps of the unit's group
        }
        umma::mbar_init(&fin, 1);
        umma::mbar_fence_init();
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tbase = tmem_base;

    if (warp == SPLIT_THREADS / 32) {  // ---------------- loads + MMAs (lane 0), scheduler (lane 1)
        if constexpr (UNITS::flow)
            if (lane == 1) {
                units.schedule(P, F);
                return;
            }
        if (lane != 0) return;
        umma::mbar_expect_tx(&gfull, 2 * garr);
        umma::bulk_g2s(G, P.g128_hi, garr, &gfull);
        umma::bulk_g2s(G + garr, P.g128_lo, garr, &gfull);
        bool ok = umma::mbar_wait(&gfull, 0, P.err);
        const uint32_t id = umma::idesc_f16(128, NT, false, true);
        const uint32_t ghi = umma::smem_u32(G), glo = ghi + garr;
        const uint32_t sbo_g = (W / 8) * 128, lbo_j = (NT / 8) * 128, kstep_j = 2 * lbo_j;
        int n = 0;
        for (int tag = 0; ok;) {
            const int unit = units.next(P, tag, true);
            if (unit < 0) break;
            const int b = n % NB, use = n / NB;
            const uint32_t par = (uint32_t)((use - 1) & 1);
            // buffer b was last used by unit n - NB: its MMAs (and so its J reads) are done
            // once acc[b] completed, and its accumulator is free once the epilogue read it
            if (use >= 1 && (!umma::mbar_wait(&acc[b], par, P.err) || !umma::mbar_wait(&tfree[b], par, P.err))) break;
            char* jb = JB + (size_t)b * UG * jslot;
            umma::mbar_expect_tx(&full[b], (uint32_t)UG * jslot);
            umma::bulk_g2s(jb, P.a4 + (size_t)unit * UG * jslot, (uint32_t)UG * jslot, &full[b]);
            if (!umma::mbar_wait(&full[b], (uint32_t)(use & 1), P.err)) break;
            umma::fence_after_sync();
            for (int g = 0; g < UG; ++g) {
                if (P.slot_roi[unit * UG + g] < 0) continue;
                const uint32_t td = tbase + (uint32_t)(b * nc + g * NT);
                const uint32_t jhi = umma::smem_u32(jb + (size_t)g * jslot), jlo = jhi + jarr;
                mma_chain(td, ghi, 128, sbo_g, 256, jhi, lbo_j, 128, kstep_j, W, id, false);
                mma_chain(td, glo, 128, sbo_g, 256, jhi, lbo_j, 128, kstep_j, W, id, true);
                mma_chain(td, ghi, 128, sbo_g, 256, jlo, lbo_j, 128, kstep_j, W, id, true);
            }
            umma::mma_commit(&acc[b]);
            ++n;
        }
        umma::mma_commit(&fin);
        return;
    }

    // ---------------- epilogue: one group of 512 threads, or two of 256
    if (NGRP == 2) {
        const int grp = t >> 8, tg = t & 255;
        s45s_epilogue<256>(P, F, units, NB, grp, tg, 2 + grp, tbase, Tm + (size_t)grp * UG * 4 * RR, red + 8 * grp,
                           nrm + 8 * grp, badw + 8 * grp, acc, tfree);
    } else {
        s45s_epilogue<SPLIT_THREADS>(P, F, units, NB, 0, t, 1, tbase, Tm, red, nrm, badw, acc, tfree);
    }
    if (t == 0) umma::mbar_wait(&fin, 0, P.err);  // every MMA of this CTA has completed
    epi_bar();
    if (t < 32) umma::tmem_dealloc(tbase, ncols);
}

__global__ void __launch_bounds__(S45S_THREADS, 1) k_stage45s(SplitDev P, FitIO F) {
    if (!cta_has_live_tile(P, P.P / unit_slots(P.G1, P.G2), unit_slots(P.G1, P.G2))) return;
    stage45s_body(P, F, StaticUnits{});
}


// ------------------------------------------------- fused stages 2 to 5 ------
// One CTA per stage-2 tile (G2 slots x W rows j).  The window DFT runs over
// 16-wide i-chunks; each chunk's intensity products go straight into the
// row-blur accumulators (stage 3, chunked over K = i) in TMEM; the finished
// row-blurred maps are rebuilt as stage-4 operands in the (now free) A2
// region; the column blur lands in shared memory as FP32 maps; and the
// likelihood sums and the FP64 LM step (stage 5) run on them in place.  Only
// the A2 tile crosses global memory.
//
// Shared memory: [A2: 4 x 128 x K1 f16 | later A4 tiles] [BC chunk buffers]
// [A3 chunk: 5 x 128 x 16 f16] [G^T hi, lo]; once the column blur is done the
// whole block holds the FP32 maps (row stride tm_stride(R)).
// TMEM: stage-2 chunk buffers at 0 (and 128), row-blur accumulators at JB,
// column-blur outputs at 0 once stage 2 is done.
__global__ void __launch_bounds__(SPLIT_THREADS, 1) k_fused25(SplitDev P, const float* rois, const float* scmos,
                                                              const double* init, int n,
                                                              FitParamsDev prm, double* out5, double* crlb5,
                                                              double* nll_out, int* st_out, int* it_out) {
    extern __shared__ __align__(1024) char smem[];
    constexpr int IC2 = 16;
    const int K1 = P.K1, W = P.W, RP = P.RP, R = P.R, G2 = P.G2, NT4 = P.NT4, NCH2 = P.NCH2;
    const int t = threadIdx.x, row = t & 127, wg = t >> 7, warp = t >> 5, lane = t & 31;
    const bool dbl = W >= 64;
    const int nbuf = dbl ? 2 : 1;
    const size_t arr2 = (size_t)128 * K1 * 2;
    const int bc_hi_b = 4 * IC2 * K1 * 2, bc_lo_b = 2 * IC2 * K1 * 2, bcb = bc_hi_b + bc_lo_b;
    const int arr3 = 128 * IC2 * 2;
    const int gtb = RP * W * 2;
    char* A2 = smem;
    char* BCB = A2 + 4 * arr2;
    char* A3 = BCB + nbuf * bcb;
    char* GT = A3 + 5 * arr3;
    float* Tm = (float*)smem;  // FP32 maps after stage 4
    const int RS = tm_stride(R), MS = R * RS;
    __shared__ __align__(8) uint64_t full_a2, bc_full[2], mma2[2], mma3, mma4;
    __shared__ uint32_t tmem_base;
    __shared__ double red[SPLIT_THREADS / 32][NRED];
    __shared__ int bad_slot[4];
    const int ncols = dbl ? 512 : 256;
    const int JB = dbl ? 256 : 128;
    if (!tile_live(P, blockIdx.x * G2, G2)) return;
    if (t < 4) bad_slot[t] = 0;
    if (t < 32) umma::tmem_alloc(&tmem_base, ncols);
    if (t == 0) {
        umma::mbar_init(&full_a2, 1);
        umma::mbar_init(&bc_full[0], 1); umma::mbar_init(&bc_full[1], 1);
        umma::mbar_init(&mma2[0], 1); umma::mbar_init(&mma2[1], 1);
        umma::mbar_init(&mma3, 1); umma::mbar_init(&mma4, 1);
        umma::mbar_fence_init();
    }
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tbase = tmem_base;
    auto load_bc = [&](int c, int buf) {
        char* dst = BCB + buf * bcb;
        umma::mbar_expect_tx(&bc_full[buf], bcb);
        umma::bulk_g2s(dst, (const char*)P.bc2_hi + (size_t)c * bc_hi_b, bc_hi_b, &bc_full[buf]);
        umma::bulk_g2s(dst + bc_hi_b, (const char*)P.bc2_lo + (size_t)c * bc_lo_b, bc_lo_b, &bc_full[buf]);
    };
    if (t == 0) {
        umma::mbar_expect_tx(&full_a2, (uint32_t)(4 * arr2 + 2 * gtb));
        const char* src = P.a2 + (size_t)blockIdx.x * a2_tile_bytes(K1);
        for (int q = 0; q < 4; ++q) umma::bulk_g2s(A2 + q * arr2, src + q * arr2, (uint32_t)arr2, &full_a2);
        umma::bulk_g2s(GT, P.gt_hi, (uint32_t)gtb, &full_a2);
        umma::bulk_g2s(GT + gtb, P.gt_lo, (uint32_t)gtb, &full_a2);
        load_bc(0, 0);
        if (dbl && NCH2 > 1) load_bc(1, 1);
    }
    const uint32_t lbo_mn = (128 / 8) * 128, kstep_mn = 2 * lbo_mn, sbo_k1 = (K1 / 8) * 128, sbo_w = (W / 8) * 128;
    const uint32_t id64 = umma::idesc_f16(128, 4 * IC2, true, false);
    const uint32_t id32 = umma::idesc_f16(128, 2 * IC2, true, false);
    const uint32_t idJ = umma::idesc_f16(128, RP, false, false);
    const uint32_t id4 = umma::idesc_f16(128, RP, true, false);
    auto bc_parity = [&](int c) { return dbl ? (uint32_t)((c >> 1) & 1) : (uint32_t)(c & 1); };
    auto issue2 = [&](int c) {
        const int buf = dbl ? (c & 1) : 0;
        if (c == 0) umma::mbar_wait(&full_a2, 0, P.err);
        umma::mbar_wait(&bc_full[buf], bc_parity(c), P.err);
        umma::fence_after_sync();
        const uint32_t bhi = umma::smem_u32(BCB + buf * bcb), blo = bhi + bc_hi_b;
        const uint32_t ahi = umma::smem_u32(A2), alo = ahi + (uint32_t)arr2, ay = ahi + 2 * (uint32_t)arr2,
                       az = ahi + 3 * (uint32_t)arr2;
        const uint32_t td = tbase + buf * 128;
        mma_chain(td, ahi, lbo_mn, 128, kstep_mn, bhi, 128, sbo_k1, 256, K1, id64, false);
        mma_chain(td, ahi, lbo_mn, 128, kstep_mn, blo, 128, sbo_k1, 256, K1, id32, true);
        mma_chain(td, alo, lbo_mn, 128, kstep_mn, bhi, 128, sbo_k1, 256, K1, id32, true);
        mma_chain(td + 64, ay, lbo_mn, 128, kstep_mn, bhi, 128, sbo_k1, 256, K1, id32, false);
        mma_chain(td + 96, az, lbo_mn, 128, kstep_mn, bhi, 128, sbo_k1, 256, K1, id32, false);
        umma::mma_commit(&mma2[buf]);
    };
    if (t == 0) issue2(0);
    for (int c = 0; c < NCH2; ++c) {
        const int buf = dbl ? (c & 1) : 0;
        if (t == 0 && dbl && c + 1 < NCH2) issue2(c + 1);
        umma::mbar_wait(&mma2[buf], bc_parity(c), P.err);
        if (c > 0) umma::mbar_wait(&mma3, (uint32_t)((c - 1) & 1), P.err);  // A3 chunk buffer free
        umma::fence_after_sync();
        {
            const uint32_t b0 = buf * 128;
            const int u0 = wg * 4;
            float er[4], ei[4], xr[4], xi[4];
            umma::tmem_ld4(tmem_lane_addr(tbase, b0 + 0 * IC2 + u0), er);
            umma::tmem_ld4(tmem_lane_addr(tbase, b0 + 1 * IC2 + u0), ei);
            umma::tmem_ld4(tmem_lane_addr(tbase, b0 + 2 * IC2 + u0), xr);
            umma::tmem_ld4(tmem_lane_addr(tbase, b0 + 3 * IC2 + u0), xi);
            __half hh[4], ll[4], dx[4], dy[4], dz[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                umma::split_f16((er[u] * er[u] + ei[u] * ei[u]) * P.sc.cI, hh[u], ll[u]);
                dx[u] = __float2half_rn((er[u] * xr[u] + ei[u] * xi[u]) * P.sc.cIx);
            }
            umma::tmem_ld4(tmem_lane_addr(tbase, b0 + 64 + u0), xr);
            umma::tmem_ld4(tmem_lane_addr(tbase, b0 + 80 + u0), xi);
#pragma unroll
            for (int u = 0; u < 4; ++u) dy[u] = __float2half_rn((er[u] * xr[u] + ei[u] * xi[u]) * P.sc.cIy);
            umma::tmem_ld4(tmem_lane_addr(tbase, b0 + 96 + u0), xr);
            umma::tmem_ld4(tmem_lane_addr(tbase, b0 + 112 + u0), xi);
#pragma unroll
            for (int u = 0; u < 4; ++u) dz[u] = __float2half_rn((er[u] * xr[u] + ei[u] * xi[u]) * P.sc.cIz);
            const uint32_t off = kmajor_off(row, u0, IC2);
            const __half* arrs[5] = {hh, ll, dx, dy, dz};
#pragma unroll
            for (int q = 0; q < 5; ++q) {
                uint2 v;
                v.x = (uint32_t)__half_as_ushort(arrs[q][0]) | ((uint32_t)__half_as_ushort(arrs[q][1]) << 16);
                v.y = (uint32_t)__half_as_ushort(arrs[q][2]) | ((uint32_t)__half_as_ushort(arrs[q][3]) << 16);
                *(uint2*)(A3 + q * arr3 + off) = v;
            }
        }
        umma::fence_before_sync();
        umma::fence_proxy_async();
        __syncthreads();
        if (t == 0) {
            umma::fence_after_sync();
            const uint32_t a3 = umma::smem_u32(A3), ghi = umma::smem_u32(GT) + (uint32_t)c * 256,
                           glo = umma::smem_u32(GT) + (uint32_t)gtb + (uint32_t)c * 256;
            const uint32_t sbo3 = (IC2 / 8) * 128;
            // one K = 16 step per chunk: J_m += A3_m G^T[:, chunk]
            umma::mma_f16(tbase + JB, umma::smem_desc(a3, 128, sbo3), umma::smem_desc(ghi, 128, sbo_w), idJ, c > 0);
            umma::mma_f16(tbase + JB, umma::smem_desc(a3, 128, sbo3), umma::smem_desc(glo, 128, sbo_w), idJ, 1);
            umma::mma_f16(tbase + JB, umma::smem_desc(a3 + arr3, 128, sbo3), umma::smem_desc(ghi, 128, sbo_w), idJ, 1);
            for (int m = 1; m < 4; ++m)
                umma::mma_f16(tbase + JB + m * RP, umma::smem_desc(a3 + (m + 1) * arr3, 128, sbo3),
                              umma::smem_desc(ghi, 128, sbo_w), idJ, c > 0);
            umma::mma_commit(&mma3);
            if (c + nbuf < NCH2) load_bc(c + nbuf, buf);
            if (!dbl && c + 1 < NCH2) issue2(c + 1);
        }
    }
    umma::mbar_wait(&mma3, (uint32_t)((NCH2 - 1) & 1), P.err);
    umma::fence_after_sync();
    // stage 3 epilogue: row-blurred maps -> stage-4 operands in the A2 region
    {
        const int g2 = row / W, j = row % W, m = wg;
        const size_t t4 = (size_t)2 * 128 * W * 2, arr4 = (size_t)128 * W * 2;
        for (int h = 0; h < RP; h += 16) {
            float v[16];
            umma::tmem_ld16(tmem_lane_addr(tbase, JB + m * RP + h), v);
            for (int i8 = 0; i8 < 16; i8 += 8) {
                const int r = m * RP + h + i8;
                char* tile = A2 + (size_t)(g2 * NT4 + r / 128) * t4;
                __half hh[8], ll[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) umma::split_f16(v[i8 + u] * P.sc.cJ[m], hh[u], ll[u]);
                const uint32_t off = mnmajor_off(r % 128, j, 128);
                store8h(tile + off, hh);
                store8h(tile + arr4 + off, ll);
            }
        }
    }
    umma::fence_before_sync();
    umma::fence_proxy_async();
    __syncthreads();
    if (t == 0) {
        umma::fence_after_sync();
        const size_t t4 = (size_t)2 * 128 * W * 2, arr4 = (size_t)128 * W * 2;
        const uint32_t ghi = umma::smem_u32(GT), glo = ghi + (uint32_t)gtb;
        for (int tt = 0; tt < G2 * NT4; ++tt) {
            const uint32_t ahi = umma::smem_u32(A2 + (size_t)tt * t4), alo = ahi + (uint32_t)arr4;
            const uint32_t td = tbase + tt * RP;
            mma_chain(td, ahi, lbo_mn, 128, kstep_mn, ghi, 128, sbo_w, 256, W, id4, false);
            mma_chain(td, ahi, lbo_mn, 128, kstep_mn, glo, 128, sbo_w, 256, W, id4, true);
            mma_chain(td, alo, lbo_mn, 128, kstep_mn, ghi, 128, sbo_w, 256, W, id4, true);
        }
        umma::mma_commit(&mma4);
    }
    umma::mbar_wait(&mma4, 0, P.err);
    umma::fence_after_sync();
    // stage 4 epilogue: FP32 maps into shared memory
    {
        const int cq = RP / 4;
        for (int tt = 0; tt < G2 * NT4; ++tt) {
            const int g2 = tt / NT4, r = (tt % NT4) * 128 + row, map = r / RP, ip = r % RP;
            for (int h = wg * cq; h < (wg + 1) * cq; h += 4) {
                float v[4];
                umma::tmem_ld4(tmem_lane_addr(tbase, tt * RP + h), v);
                if (map < 4 && ip < R && h < R) {
                    const float c = P.sc.cT[map];
                    float* dst = Tm + (size_t)(g2 * 4 + map) * MS + ip * RS + h;
                    if (h + 4 <= R)
                        *(float4*)dst = make_float4(v[0] * c, v[1] * c, v[2] * c, v[3] * c);
                    else
                        for (int u = 0; h + u < R; ++u) dst[u] = v[u] * c;
                }
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    // stage 5: per slot, 16 / G2 warps
    const int wps = (SPLIT_THREADS / 32) / G2, g2 = warp / wps, tid_s = t - g2 * wps * 32, nts = wps * 32;
    const int slot = blockIdx.x * G2 + g2;
    const int roi = P.slot_roi[slot];
    const int RR = R * R;
    const float* T0 = Tm + (size_t)g2 * 4 * MS;
    float ns[4] = {0, 0, 0, 0}, nc = 0.f;
    if (roi >= 0)
        for (int k = tid_s; k < RR; k += nts) {
            const int ip = k / R, o = ip * RS + (k - ip * R);
            const float v = T0[o], sg = v < 0 ? -1.f : 1.f;
            kahan_add(ns[0], nc, fabsf(v));
            ns[1] += sg * T0[MS + o];
            ns[2] += sg * T0[2 * MS + o];
            ns[3] += sg * T0[3 * MS + o];
        }
    {
        double v0 = warp_sum((double)ns[0] - (double)nc), v1 = warp_sum(ns[1]), v2 = warp_sum(ns[2]), v3 = warp_sum(ns[3]);
        if (lane == 0) { red[warp][0] = v0; red[warp][1] = v1; red[warp][2] = v2; red[warp][3] = v3; }
    }
    __syncthreads();
    double sum4[4] = {0, 0, 0, 0};
    for (int w = g2 * wps; w < (g2 + 1) * wps; ++w)
        for (int q = 0; q < 4; ++q) sum4[q] += red[w][q];
    __syncthreads();
    const float S = (float)sum4[0], Dx = (float)sum4[1], Dy = (float)sum4[2], Dz = (float)sum4[3];
    const float invS = 1.f / S;
    float sg6[6], cg6[6], sh[30];
#pragma unroll
    for (int k = 0; k < 6; ++k) { sg6[k] = 0.f; cg6[k] = 0.f; }
#pragma unroll
    for (int k = 0; k < 30; ++k) sh[k] = 0.f;
    bool bad = false;
    if (roi >= 0) {
        const double* th = P.lm[slot].trial;
        const float A = (float)th[3], B = (float)th[4];
        const float* d = rois + (size_t)roi * RR;
        const float* sv = scmos ? scmos + (size_t)roi * RR : nullptr;
        for (int k = tid_s; k < RR; k += nts) {
            const int ip = k / R, to = ip * RS + (k - ip * R);
            const float v = T0[to], sgn = v < 0 ? -1.f : 1.f, psi = fabsf(v) * invS;
            float jv[5];
            jv[0] = A * (sgn * T0[MS + to] - psi * Dx) * invS;
            jv[1] = A * (sgn * T0[2 * MS + to] - psi * Dy) * invS;
            jv[2] = A * (sgn * T0[3 * MS + to] - psi * Dz) * invS;
            jv[3] = psi;
            jv[4] = 1.f;
            const float mu = A * psi + B + (sv ? sv[k] : 0.f);
            if (!(mu > 0.f)) { bad = true; continue; }
            const float dk = d[k];
            kahan_add(sg6[0], cg6[0], dk > 0.f ? mu - dk - dk * logf(mu / dk) : mu);
            const float wgt = 1.f - dk / mu, wf = 1.f / mu, wh = dk * wf * wf;
#pragma unroll
            for (int q = 0; q < 5; ++q) kahan_add(sg6[1 + q], cg6[1 + q], wgt * jv[q]);
            int o = 0;
#pragma unroll
            for (int q = 0; q < 5; ++q)
#pragma unroll
                for (int r2 = 0; r2 <= q; ++r2) {
                    sh[o] += wh * jv[q] * jv[r2];
                    sh[o + 15] += wf * jv[q] * jv[r2];
                    ++o;
                }
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const double v = warp_sum((double)sg6[k] - (double)cg6[k]);
        if (lane == 0) red[warp][k] = v;
    }
#pragma unroll
    for (int k = 0; k < 30; ++k) {
        const double v = warp_sum((double)sh[k]);
        if (lane == 0) red[warp][6 + k] = v;
    }
    if (bad) bad_slot[g2] = 1;
    __syncthreads();
    if (tid_s == 0 && roi >= 0) {
        double tot[NRED];
        for (int q = 0; q < NRED; ++q) {
            double v = 0;
            for (int w = g2 * wps; w < (g2 + 1) * wps; ++w) v += red[w][q];
            tot[q] = v;
        }
        double nll = bad_slot[g2] ? INFINITY : tot[0], g[5], H[25], F[25];
        for (int q = 0; q < 5; ++q) g[q] = tot[1 + q];
        int o = 6;
        for (int q = 0; q < 5; ++q)
            for (int r2 = 0; r2 <= q; ++r2) {
                H[q * 5 + r2] = H[r2 * 5 + q] = tot[o];
                F[q * 5 + r2] = F[r2 * 5 + q] = tot[o + 15];
                ++o;
            }
        LMState& st = P.lm[slot];
        bool next_trial = false;
        if (P.slot_phase[slot] == 0) {
            for (int q = 0; q < 5; ++q) st.th[q] = st.trial[q];
            lm_start(st, nll, g, H, F, prm);
            P.slot_phase[slot] = 1;
        } else {
            lm_update(st, nll, g, H, F, prm);
        }
        next_trial = lm_propose(st, prm);
        if (!next_trial) {
            for (int q = 0; q < 5; ++q) out5[5 * roi + q] = st.th[q];
            if (nll_out) nll_out[roi] = st.nll;
            if (st_out) st_out[roi] = st.status;
            if (it_out) it_out[roi] = st.evals;
            if (crlb5) lm_crlb(st.F, crlb5 + 5 * roi);
            const int nx = take_roi(P, n);
            if (nx >= 0) {
                P.slot_roi[slot] = nx;
                P.slot_phase[slot] = 0;
                for (int q = 0; q < 5; ++q) st.trial[q] = init[5 * nx + q];
                lm_clamp(st.trial, prm);
            } else {
                P.slot_roi[slot] = -1;
                atomicSub(P.active, 1);
            }
        }
    }
    __syncthreads();
    if (t < 32) umma::tmem_dealloc(tbase, ncols);
}

// Fill the pool from the queue.  Units with a ROI are ready for stage 1 of
// their first evaluation (state 0); units without one are dead unless more
// ROIs are still to arrive.  avail: the caller's device count of ROIs on the
// device (P.navail points at it), else navail.
__global__ void k_init_slots(SplitDev P, const double* init, int n, int navail, FitParamsDev prm,
                             const int* avail = nullptr) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= P.P) return;
    if (avail) navail = *(volatile const int*)avail;
    const int m = n < navail ? n : navail;
    if (slot < m) {
        P.slot_roi[slot] = slot;
        P.slot_phase[slot] = 0;
        for (int q = 0; q < 5; ++q) P.lm[slot].trial[q] = init[5 * slot + q];
        lm_clamp(P.lm[slot].trial, prm);
    } else {
        P.slot_roi[slot] = -1;
    }
    const int UG = unit_slots(P.G1, P.G2);
    if (slot % UG == 0) P.ustate[slot / UG] = slot < m || navail < n ? 0 : UNIT_DEAD;
    if (slot == 0) {
        *P.queue = P.P < m ? P.P : m;
        *P.active = P.P < m ? P.P : m;
        *P.err = 0;
        *P.evals = 0;
        if (!avail) *P.navail = navail;
    }
}

// Idle slots (their last ROI retired while the queue had reached the ROIs on
// the device) take ROIs that have arrived since.
__global__ void k_refill(SplitDev P, const double* init, int n, FitParamsDev prm) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= P.P || P.slot_roi[slot] >= 0) return;
    const int r = take_roi(P, n);
    if (r < 0) return;
    P.slot_roi[slot] = r;
    P.slot_phase[slot] = 0;
    double* tr = P.lm[slot].trial;
    for (int q = 0; q < 5; ++q) tr[q] = init[5 * r + q];
    lm_clamp(tr, prm);
    atomicAdd(P.active, 1);
}

__global__ void k_set_int(int* p, int v) { *p = v; }

// ------------------------------------------------------- dataflow kernel ----
// The whole fit in one cooperative launch: CTAs [first[s], first[s + 1]) run
// stage s (pupil DFT, window DFT, row blur, column blur + sums, LM step) on the
// units u with u = (CTA index within the stage) mod (CTAs of the stage).  A unit
// cycles through the five stages once per evaluation; its operands pass from
// one stage to the next through global memory while they are still in L2 (the
// pool is small enough), and no stage waits for a round of the whole pool.
// Converged fits retire and their slots refill from the ROI queue in the LM
// step; the kernel ends when every unit is dead.
constexpr int FLOW_THREADS = SPLIT_THREADS + 32;

struct FlowRoles {
    int first[FLOW_STAGES + 1];
};

template <int W>
__global__ void __launch_bounds__(FLOW_THREADS, 1) k_flow(SplitDev P, FitIO F, FlowRoles roles) {
    __shared__ UnitRing ring;
    int s = 0;
    while (s < FLOW_STAGES - 1 && (int)blockIdx.x >= roles.first[s + 1]) ++s;
    FlowUnits units{&ring, s, (int)blockIdx.x - roles.first[s], roles.first[s + 1] - roles.first[s], 0};
    if (s == FLOW_STAGES - 1) {
        lm_role(P, F, units.first, units.stride);
        return;
    }
    if (threadIdx.x == 0) {  // (each stage body publishes these with its own barrier set-up)
        const int readers = s == 3 && W >= S45_MIN_W ? E45_THREADS / 32 + 2 : SPLIT_THREADS / 32 + 1;
        for (int b = 0; b < URING; ++b) {
            umma::mbar_init(&ring.full[b], 1);
            umma::mbar_init(&ring.freed[b], readers);
        }
        ring.released = 0;
    }
    if (s == 0) {
        stage1_body<W>(P, F, units);
    } else if (s == 1) {
        stage2_body<W>(P, F, units);
    } else if (s == 2) {
        stage3_body(P, F, units);
    } else {
        if constexpr (W >= S45_MIN_W) stage45_body(P, F, units);
        else stage45s_body(P, F, units);
    }
}


// ---------------------------------------------------------------- host -----
static size_t smem_stage1p(const SplitPlanHost& pl) {
    return (size_t)(pl.K1 / 16) * s2_slab_bytes(pl.W) + (size_t)S1_NBQ * s1_qring_bytes(pl.W);
}
static size_t smem_stage2p(const SplitPlanHost& pl) {
    return (size_t)(pl.K1 / 16) * s2_slab_bytes(pl.W) + (size_t)S2_NBUF * s2_ring_bytes(pl.W);
}
static size_t smem_stage3(const SplitPlanHost& pl, bool flow = false) {
    return (size_t)s3_nbuf(pl.W, flow) * 5 * 128 * pl.W * 2 + (size_t)4 * pl.RP * pl.W;
}
static size_t smem_stage4(const SplitPlanHost& pl) { return a4_slot_bytes(pl.W, pl.RP) + (size_t)2 * 128 * pl.W * 2; }
static size_t smem_stage45(const SplitPlanHost& pl) {
    return (size_t)2 * 128 * pl.W * 2 + (size_t)S45_NBUF * 2 * 32 * 4 * pl.RP + 4 * s45_roi_bytes(pl.R) +
           (size_t)4 * pl.R * tm_stride(pl.R) * 4 + 16 + (size_t)(E45_THREADS / 32) * (NRED * 8 + 4 * 8 + 4);
}
static size_t smem_stage45s(const SplitPlanHost& pl) {
    const int UG = unit_slots(pl.G1, pl.G2), nb = s45s_nbuf(pl.W, pl.RP, pl.R, UG);
    return s45s_smem(pl.W, pl.RP, pl.R, UG, nb, s45s_groups(nb));
}
static size_t smem_fused(const SplitPlanHost& pl) {
    const int nbuf = pl.W >= 64 ? 2 : 1;
    return (size_t)4 * 128 * pl.K1 * 2 + (size_t)nbuf * 12 * 16 * pl.K1 + (size_t)5 * 128 * 16 * 2 +
           (size_t)2 * pl.RP * pl.W * 2;
}
static bool fused_fits(const SplitPlanHost& pl) {
    const size_t maps = (size_t)pl.G2 * 4 * pl.R * tm_stride(pl.R) * 4;
    const size_t a4 = (size_t)pl.G2 * pl.NT4 * 2 * 128 * pl.W * 2;
    return smem_fused(pl) <= 225 * 1024 && maps <= smem_fused(pl) &&
           a4 <= (size_t)4 * 128 * pl.K1 * 2 && pl.G2 <= 4 && 4 * pl.RP + (pl.W >= 64 ? 256 : 128) <= (pl.W >= 64 ? 512 : 256);
}

// psi and d psi / d{x,y,z} of every occupied slot from its blurred maps
// (model-only evaluation through the tensor-core stages).
__global__ void k_model_out(SplitDev P, int n, double* out, double* dout) {
    const int slot = blockIdx.x, R = P.R, RR = R * R;
    if (slot >= n) return;
    __shared__ float red[4][4];
    const float* T0 = P.tmaps + (size_t)slot * 4 * RR;
    float v[4] = {0, 0, 0, 0};
    for (int k = threadIdx.x; k < RR; k += blockDim.x) {
        float t0 = T0[k], sg = t0 < 0 ? -1.f : 1.f;
        v[0] += fabsf(t0);
        v[1] += sg * T0[RR + k];
        v[2] += sg * T0[2 * RR + k];
        v[3] += sg * T0[3 * RR + k];
    }
    for (int q = 0; q < 4; ++q)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 4; ++q) red[threadIdx.x >> 5][q] = v[q];
    __syncthreads();
    float S = 0, D3[3] = {0, 0, 0};
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        S += red[w][0];
        for (int q = 0; q < 3; ++q) D3[q] += red[w][q + 1];
    }
    for (int k = threadIdx.x; k < RR; k += blockDim.x) {
        float t0 = T0[k], sg = t0 < 0 ? -1.f : 1.f, psi = fabsf(t0) / S;
        out[(size_t)slot * RR + k] = psi;
        if (dout)
            for (int q = 0; q < 3; ++q)
                dout[((size_t)slot * 3 + q) * RR + k] = (sg * T0[(q + 1) * RR + k] - psi * D3[q]) / S;
    }
}

// Slots evaluate the given (x, y, z) points (model-only use of the pool).
__global__ void k_init_points(SplitDev P, const double* xyz, int n) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= P.P) return;
    if (slot < n) {
        P.slot_roi[slot] = slot;
        for (int q = 0; q < 3; ++q) P.lm[slot].trial[q] = xyz[3 * slot + q];
        P.lm[slot].trial[3] = 1.0;
        P.lm[slot].trial[4] = 0.0;
    } else {
        P.slot_roi[slot] = -1;
    }
    if (slot == 0) *P.err = 0;
}

struct SplitPool {
    SplitPlanHost* pl = nullptr;
    SplitDev D{};
    int U = 0;  // units of UG slots
    size_t s1 = 0, s2 = 0, s3 = 0, s4 = 0, s45 = 0, sf = 0, sflow = 0;
};

template <int W>
static cudaError_t set_smem_attrs(const SplitPool& sp) {
    const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    cudaError_t e = cudaFuncSetAttribute(k_stage1p<W>, a, (int)sp.s1);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage2p<W>, a, (int)sp.s2);
    if (e == cudaSuccess && sp.sflow) e = cudaFuncSetAttribute(k_flow<W>, a, (int)sp.sflow);
    return e;
}

static cudaError_t smem_attrs(int W, const SplitPool& sp) {
    if (W == 32) return set_smem_attrs<32>(sp);
    if (W == 64) return set_smem_attrs<64>(sp);
    return set_smem_attrs<128>(sp);
}

static int unit_grid(zola_ctx* ctx, const SplitPool& sp) { return std::min(sp.U, ctx->num_sms); }

static void launch_stage1(zola_ctx* ctx, const SplitPool& sp, const FitIO& F, cudaStream_t st) {
    const int grid = unit_grid(ctx, sp);
    if (sp.D.W == 32)
        k_stage1p<32><<<grid, S1_THREADS, sp.s1, st>>>(sp.D, F);
    else if (sp.D.W == 64)
        k_stage1p<64><<<grid, S1_THREADS, sp.s1, st>>>(sp.D, F);
    else
        k_stage1p<128><<<grid, S1_THREADS, sp.s1, st>>>(sp.D, F);
}

static void launch_stage2(zola_ctx* ctx, const SplitPool& sp, const FitIO& F, cudaStream_t st) {
    const int grid = unit_grid(ctx, sp);
    if (sp.D.W == 32)
        k_stage2p<32><<<grid, S2_THREADS, sp.s2, st>>>(sp.D, F);
    else if (sp.D.W == 64)
        k_stage2p<64><<<grid, S2_THREADS, sp.s2, st>>>(sp.D, F);
    else
        k_stage2p<128><<<grid, S2_THREADS, sp.s2, st>>>(sp.D, F);
}

// Pool of slots for n ROIs: at most pmax slots (0: state up to 8 GB, at most
// 32768), in whole units; for the dataflow kernel at most max_units units.  The
// pool's device state is carved from base, or from the context's scratch when
// base is null; with need given, only the bytes it takes are reported.
static int setup_pool(zola_ctx* ctx, zola_psf* p, WindowTables* w, int n, int pmax_override, SplitPool& sp,
                      cudaStream_t st, int max_units = 0, char* base_in = nullptr, size_t* need = nullptr) {
    if (p->D > 64) {
        ctx->err = "split path: pupil disk wider than 64 rows (grid too large for this optics)";
        return ZOLA_E_UNSUPPORTED;
    }
    if (w->W < 32 || w->R > 64) {
        ctx->err = "split path supports windows W >= 32 and ROI sides up to 64";
        return ZOLA_E_UNSUPPORTED;
    }
    SplitPlanHost* pl = get_plan(p, w, ctx->err);
    if (!pl) return ZOLA_E_CUDA;
    sp.pl = pl;
    if (w->W == 128 && 2 * (p->D <= 32 ? 32 : 64) != 128) {
        ctx->err = "split path: a 128 window needs a pupil disk of more than 32 rows";
        return ZOLA_E_UNSUPPORTED;
    }
    if (w->W != 32 && w->W != 64 && w->W != 128) {
        ctx->err = "split path: window sizes 32, 64 and 128 only";
        return ZOLA_E_UNSUPPORTED;
    }
    const int UG = unit_slots(pl->G1, pl->G2);
    sp.s1 = smem_stage1p(*pl);
    sp.s2 = smem_stage2p(*pl);
    sp.s3 = smem_stage3(*pl);
    sp.s4 = smem_stage4(*pl);
    sp.s45 = pl->W >= S45_MIN_W ? smem_stage45(*pl) : smem_stage45s(*pl);
    sp.sflow = max_units > 0 ? std::max(std::max(sp.s1, sp.s2), std::max(smem_stage3(*pl, true), sp.s45)) : 0;
    const size_t lim = 225 * 1024;
    if (sp.s1 > lim || sp.s2 > lim || sp.s3 > lim || sp.s4 > lim || sp.s45 > lim || sp.sflow > lim) {
        ctx->err = "split path: shared-memory plan exceeds 225 KB";
        return ZOLA_E_UNSUPPORTED;
    }
    const size_t per_slot = a2_tile_bytes(pl->K1) / pl->G2 + a3_tile_bytes(pl->W) / pl->G2 +
                            (size_t)pl->NT4 * a4_tile_bytes(pl->W) + (size_t)4 * pl->R * pl->R * 4 + sizeof(LMState) + NSUM * 8 + 16;
    int Pmax = (int)std::min<size_t>(32768, ((size_t)8 << 30) / per_slot);  // at most 8 GB of pool state
    if (pmax_override > 0) Pmax = std::min(Pmax, pmax_override);
    if (max_units > 0) Pmax = std::min(Pmax, max_units * UG);
    Pmax = std::max(UG, Pmax / UG * UG);
    const int P = std::min(Pmax, (n + UG - 1) / UG * UG);
    sp.U = P / UG;
    auto al = [](size_t v) { return (v + 1023) / 1024 * 1024; };
    const size_t b_a2 = al((size_t)(P / pl->G2) * a2_tile_bytes(pl->K1));
    const size_t b_a3 = al((size_t)(P / pl->G2) * a3_tile_bytes(pl->W));
    const size_t b_a4 = al((size_t)P * pl->NT4 * a4_tile_bytes(pl->W));
    const size_t b_t = al((size_t)P * 4 * pl->R * pl->R * 4);
    const size_t b_lm = al((size_t)P * sizeof(LMState));
    const size_t b_sums = al((size_t)P * NSUM * 8);
    const size_t b_int = al((size_t)P * 8 + (size_t)sp.U * 4 + 64);
    const size_t b_clk = al(((size_t)3 * ctx->num_sms + 1) * 8);
    const size_t total = b_a2 + b_a3 + b_a4 + b_t + b_lm + b_sums + b_clk + b_int;
    if (need) {
        *need = total;
        return ZOLA_OK;
    }
    if (!base_in && ensure_scratch(ctx, total, ctx->err)) return ZOLA_E_CUDA;
    char* base = base_in ? base_in : (char*)ctx->scratch;
    SplitDev& D = sp.D;
    D = SplitDev{};
    D.R = pl->R; D.W = pl->W; D.D = pl->D; D.DP = pl->DP; D.K1 = pl->K1;
    D.RP = pl->RP; D.G1 = pl->G1; D.G2 = pl->G2; D.NT4 = pl->NT4; D.P = P; D.a0 = p->a0; D.N = p->N;
    D.zfocus = p->o.zfocus;
    D.gt_hi = pl->d_gt_hi; D.gt_lo = pl->d_gt_lo;
    D.g128_hi = pl->d_g128_hi; D.g128_lo = pl->d_g128_lo;
    D.bc2_hi = pl->d_bc2_hi; D.bc2_lo = pl->d_bc2_lo; D.NCH2 = pl->NCH2; D.bcs = pl->d_bcs;
    D.pupf = pl->d_pupf; D.phase0 = pl->d_phase0; D.kz = pl->d_kz; D.kx = pl->d_kx; D.ky = pl->d_ky;
    D.a2 = base; base += b_a2;
    D.a3 = base; base += b_a3;
    D.a4 = base; base += b_a4;
    D.tmaps = (float*)base; base += b_t;
    D.lm = (LMState*)base; base += b_lm;
    D.sums = (double*)base; base += b_sums;
    D.evals = (unsigned long long*)base;
    D.clk = D.evals + 1;
    base += b_clk;
    D.slot_roi = (int*)base;
    D.slot_phase = D.slot_roi + P;
    D.queue = D.slot_phase + P;
    D.active = D.queue + 1;
    D.err = D.queue + 2;
    D.navail = D.queue + 3;
    D.ustate = D.queue + 16;
    D.wait_limit = ctx->wait_limit > 0 ? ctx->wait_limit : (1ll << 31);
    D.sc = pl->sc;
    ZOLA_CUDA_CHECK(cudaMemsetAsync(D.a4, 0, b_a4, st), ctx);
    ZOLA_CUDA_CHECK(smem_attrs(pl->W, sp), ctx);
    const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    ZOLA_CUDA_CHECK(cudaFuncSetAttribute(k_stage3, a, (int)sp.s3), ctx);
    ZOLA_CUDA_CHECK(cudaFuncSetAttribute(k_stage4, a, (int)sp.s4), ctx);
    if (pl->W >= S45_MIN_W)
        ZOLA_CUDA_CHECK(cudaFuncSetAttribute(k_stage45p, a, (int)sp.s45), ctx);
    else
        ZOLA_CUDA_CHECK(cudaFuncSetAttribute(k_stage45s, a, (int)sp.s45), ctx);
    sp.sf = smem_fused(*pl);
    if (fused_fits(*pl)) ZOLA_CUDA_CHECK(cudaFuncSetAttribute(k_fused25, a, (int)sp.sf), ctx);
    return ZOLA_OK;
}

// Stages 1-3 (pupil DFT, window DFT, row blur) of every occupied slot.
static void launch_stages123(zola_ctx* ctx, const SplitPool& sp, const FitIO& F, cudaStream_t st) {
    prof_begin(ctx, 0, st);
    launch_stage1(ctx, sp, F, st);
    prof_end(ctx, st);
    prof_begin(ctx, 1, st);
    launch_stage2(ctx, sp, F, st);
    prof_end(ctx, st);
    prof_begin(ctx, 2, st);
    k_stage3<<<unit_grid(ctx, sp), S3_THREADS, sp.s3, st>>>(sp.D, F);
    prof_end(ctx, st);
    ctx->launches += 3;
}

static int read_flags(zola_ctx* ctx, const SplitDev& D, cudaStream_t st, int* active, int* err, int* queue = nullptr) {
    if (!ctx->h_flags) ZOLA_CUDA_CHECK(cudaMallocHost(&ctx->h_flags, 4 * sizeof(int)), ctx);
    ZOLA_CUDA_CHECK(cudaMemcpyAsync(ctx->h_flags, D.queue, 3 * sizeof(int), cudaMemcpyDeviceToHost, st), ctx);
    ZOLA_CUDA_CHECK(cudaStreamSynchronize(st), ctx);
    prof_collect(ctx);
    if (queue) *queue = ctx->h_flags[0];
    *active = ctx->h_flags[1];
    *err = ctx->h_flags[2];
    return ZOLA_OK;
}

int launch_model_split(zola_ctx* ctx, zola_psf* p, WindowTables* w, const double* d_xyz, int n, double* d_out,
                       double* d_dout, cudaStream_t st) {
    const FitIO none{};
    for (int done = 0; done < n;) {
        SplitPool sp;
        int rc = setup_pool(ctx, p, w, n - done, 0, sp, st);
        if (rc) return rc;
        const int m = std::min(sp.D.P, n - done);
        k_init_points<<<(sp.D.P + 127) / 128, 128, 0, st>>>(sp.D, d_xyz + 3 * (size_t)done, m);
        launch_stages123(ctx, sp, none, st);
        prof_begin(ctx, 3, st);
        k_stage4<<<sp.D.P, SPLIT_THREADS, sp.s4, st>>>(sp.D);
        prof_end(ctx, st);
        const size_t RR = (size_t)w->R * w->R;
        k_model_out<<<m, 128, 0, st>>>(sp.D, m, d_out + RR * done, d_dout ? d_dout + 3 * RR * done : nullptr);
        ctx->launches += 3;
        ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
        int active, err;
        rc = read_flags(ctx, sp.D, st, &active, &err);
        if (rc) return rc;
        if (err) { ctx->err = "split model: a bounded device wait timed out"; return ZOLA_E_TIMEOUT; }
        done += m;
    }
    return ZOLA_OK;
}

// Default shape of the dataflow kernel: two units per SM, and the SMs split
// between the stages in proportion to each stage's share of a unit's device
// time for this window size (measured on B200 with the round-based kernels).
static FlowShape default_shape(int W, int grid) {
    static const double share[3][FLOW_STAGES] = {{0.33, 0.20, 0.17, 0.25, 0.05},   // W = 32
                                                 {0.38, 0.23, 0.16, 0.19, 0.04},   // W = 64
                                                 {0.22, 0.31, 0.18, 0.26, 0.03}};  // W = 128
    const int wi = W == 32 ? 0 : W == 64 ? 1 : 2;
    FlowShape f;
    f.units = 2 * grid;
    // CTAs in proportion to the shares, at least one each, adding up to grid
    int sum = 0;
    for (int s = 0; s < FLOW_STAGES; ++s) sum += f.ctas[s] = std::max(1, (int)std::lround(share[wi][s] * grid));
    for (int s = 0; sum != grid; s = (s + 1) % FLOW_STAGES) {
        if (sum > grid && f.ctas[s] > 1) { --f.ctas[s]; --sum; }
        else if (sum < grid) { ++f.ctas[s]; ++sum; }
    }
    return f;
}

// CTAs in proportion to the busy time (time with a unit in flight) each stage
// had in a measured launch, moved half way from the current split.
static void rebalance(FlowShape& f, const unsigned long long* clk, int grid) {
    double work[FLOW_STAGES] = {}, tot = 0;
    int b = 0;
    for (int s = 0; s < FLOW_STAGES; ++s)
        for (int k = 0; k < f.ctas[s]; ++k, ++b) work[s] += (double)(clk[3 * b + 1] - std::min(clk[3 * b], clk[3 * b + 1]));
    for (int s = 0; s < FLOW_STAGES; ++s) tot += work[s];
    if (!(tot > 0)) return;
    int sum = 0;
    for (int s = 0; s < FLOW_STAGES; ++s)
        sum += f.ctas[s] = std::max(1, (int)std::lround(0.5 * f.ctas[s] + 0.5 * work[s] / tot * grid));
    for (int s = 0; sum != grid; s = (s + 1) % FLOW_STAGES) {
        if (sum > grid && f.ctas[s] > 1) { --f.ctas[s]; --sum; }
        else if (sum < grid) { ++f.ctas[s]; ++sum; }
    }
}

static std::string tune_key(const zola_psf* p, const WindowTables* w) {
    return "N" + std::to_string(p->N) + "_D" + std::to_string(p->D) + "_R" + std::to_string(w->R) + "_W" +
           std::to_string(w->W);
}

// The autotuner's cache: {"<class>": {"units": U, "ctas": [a, b, c, d, e], "ns_per_eval": t}, ...} for the
// dataflow kernel, {"<class>_pool": {"pool": P, "ns_per_eval": t}, ...} for the round-based kernels.
static void tune_save(zola_ctx* ctx) {
    if (ctx->tune_path.empty()) return;
    FILE* f = std::fopen(ctx->tune_path.c_str(), "w");
    if (!f) return;
    std::fprintf(f, "{");
    bool first = true;
    for (const auto& kv : ctx->tunes) {
        if (!kv.second.done) continue;
        const FlowShape& b = kv.second.best;
        std::fprintf(f, "%s\n  \"%s\": {\"units\": %d, \"ctas\": [%d, %d, %d, %d, %d], \"ns_per_eval\": %.3f}",
                     first ? "" : ",", kv.first.c_str(), b.units, b.ctas[0], b.ctas[1], b.ctas[2], b.ctas[3],
                     b.ctas[4], kv.second.best_ns);
        first = false;
    }
    for (const auto& kv : ctx->pool_tunes) {
        if (!kv.second.done) continue;
        std::fprintf(f, "%s\n  \"%s\": {\"pool\": %d, \"ns_per_eval\": %.3f}", first ? "" : ",", kv.first.c_str(),
                     kv.second.best, kv.second.best_ns);
        first = false;
    }
    std::fprintf(f, "\n}\n");
    std::fclose(f);
}

void tune_load(zola_ctx* ctx) {
    if (ctx->tune_path.empty()) return;
    FILE* f = std::fopen(ctx->tune_path.c_str(), "r");
    if (!f) return;
    std::string txt;
    char buf[4096];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0) txt.append(buf, k);
    std::fclose(f);
    size_t pos = 0;
    while ((pos = txt.find('"', pos)) != std::string::npos) {
        const size_t end = txt.find('"', pos + 1);
        if (end == std::string::npos) break;
        const std::string key = txt.substr(pos + 1, end - pos - 1);
        pos = end + 1;
        if (key.empty() || key[0] != 'N') continue;
        PoolTune pt;
        if (std::sscanf(txt.c_str() + pos, " : {\"pool\": %d, \"ns_per_eval\": %lf", &pt.best, &pt.best_ns) == 2) {
            if (pt.best > 0) {
                pt.done = true;
                ctx->pool_tunes[key] = pt;
            }
            continue;
        }
        FlowTune t;
        if (std::sscanf(txt.c_str() + pos, " : {\"units\": %d, \"ctas\": [%d, %d, %d, %d, %d], \"ns_per_eval\": %lf",
                        &t.best.units, &t.best.ctas[0], &t.best.ctas[1], &t.best.ctas[2], &t.best.ctas[3],
                        &t.best.ctas[4], &t.best_ns) == 7) {
            int sum = 0;
            for (int s = 0; s < FLOW_STAGES; ++s) sum += t.best.ctas[s] > 0 ? t.best.ctas[s] : -100000;
            if (sum == ctx->num_sms && t.best.units > 0) {
                t.done = true;
                ctx->tunes[key] = t;
            }
        }
    }
}

// Shape of this launch: the context's explicit setting, a tuned shape, the
// tuner's next trial (large batches of an untuned class while tuning is on),
// or the default.  *trial: the launch is to be measured for the tuner.
static FlowShape pick_shape(zola_ctx* ctx, const std::string& key, int W, int n, int UG, bool* trial) {
    const int grid = ctx->num_sms;
    *trial = false;
    FlowShape f = default_shape(W, grid);
    if (ctx->flow_ctas[0] > 0)
        for (int s = 0; s < FLOW_STAGES; ++s) f.ctas[s] = ctx->flow_ctas[s];
    if (ctx->flow_units > 0) f.units = ctx->flow_units;
    if (ctx->flow_units > 0 || ctx->flow_ctas[0] > 0) return f;
    auto it = ctx->tunes.find(key);
    if (it != ctx->tunes.end() && it->second.done) return it->second.best;
    // tuning needs a batch that keeps the pool busy for many evaluations
    if (!ctx->tune || n < 16 * 3 * grid * UG) return f;
    FlowTune& t = ctx->tunes[key];
    *trial = true;
    return t.trials == 0 ? f : t.next;
}

// After a measured launch: record it and choose the next trial.  Trials 0-4
// rebalance the CTAs per stage from the measured busy times at two units per
// SM; trials 5 and 6 try three and one and a half units per SM with the best
// split; then the best shape is kept (and written to the cache file).
static void tune_record(zola_ctx* ctx, const std::string& key, const FlowShape& used, double ns_per_eval,
                        const unsigned long long* clk) {
    FlowTune& t = ctx->tunes[key];
    if (t.trials == 0 || ns_per_eval < t.best_ns) {
        t.best = used;
        t.best_ns = ns_per_eval;
    }
    ++t.trials;
    const int grid = ctx->num_sms;
    t.next = used;
    if (t.trials < 5) {
        rebalance(t.next, clk, grid);
    } else if (t.trials == 5) {
        t.next = t.best;
        t.next.units = 3 * grid;
    } else if (t.trials == 6) {
        t.next = t.best;
        t.next.units = 3 * grid / 2;
    } else {
        t.done = true;
        tune_save(ctx);
    }
}

// Slot pools the round-based tuner tries, in this order (each capped by the
// 8 GB pool-state limit of setup_pool).
static const int POOL_TRIALS[] = {4096, 8192, 16384, 32768};
constexpr int N_POOL_TRIALS = 4;

// Pool of a round-based fit: the context's explicit setting, the tuned pool,
// the tuner's next trial (large batches of an untuned class while tuning is
// on), or 0 (automatic).  *trial: the fit is to be measured for the tuner.
static int pick_pool(zola_ctx* ctx, const std::string& key, int n, bool* trial) {
    *trial = false;
    if (ctx->split_pool_max > 0) return ctx->split_pool_max;
    auto it = ctx->pool_tunes.find(key);
    if (it != ctx->pool_tunes.end() && it->second.done) return it->second.best;
    if (!ctx->tune || n < 4 * POOL_TRIALS[N_POOL_TRIALS - 1]) return 0;
    *trial = true;
    return POOL_TRIALS[ctx->pool_tunes[key].trials];
}

static void pool_record(zola_ctx* ctx, const std::string& key, int pool, double ns_per_eval) {
    PoolTune& t = ctx->pool_tunes[key];
    if (t.trials == 0 || ns_per_eval < t.best_ns) {
        t.best = pool;
        t.best_ns = ns_per_eval;
    }
    if (++t.trials == N_POOL_TRIALS) {
        t.done = true;
        tune_save(ctx);
    }
}

static std::string pool_key(const zola_psf* p, const WindowTables* w) { return tune_key(p, w) + "_pool"; }

static int launch_fit_flow(zola_ctx* ctx, zola_psf* p, WindowTables* w, const FitIO& F, cudaStream_t st,
                           const RoiFeed* feed, const int* d_avail) {
    SplitPool sp;
    const int grid = ctx->num_sms;
    SplitPlanHost* pl = get_plan(p, w, ctx->err);
    if (!pl) return ZOLA_E_CUDA;
    const std::string key = tune_key(p, w);
    bool trial = false;
    const FlowShape shape = pick_shape(ctx, key, w->W, F.n, unit_slots(pl->G1, pl->G2), &trial);
    int rc = setup_pool(ctx, p, w, F.n, ctx->split_pool_max, sp, st, shape.units);
    if (rc) return rc;
    if (d_avail) sp.D.navail = const_cast<int*>(d_avail);  // read only
    const SplitDev& D = sp.D;
    int navail = F.n;
    if (feed && feed->n_chunks > 0) {
        ZOLA_CUDA_CHECK(cudaStreamWaitEvent(st, feed->ev[0], 0), ctx);
        navail = feed->chunk_end[0];
    }
    k_init_slots<<<(D.P + 127) / 128, 128, 0, st>>>(D, F.init, F.n, navail, F.prm, d_avail);
    ctx->launches++;
    ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
    if (feed && feed->n_chunks > 1) {
        // the ROI count on the device follows the input chunks as they land (a
        // copy per chunk, after the pool was filled), while the kernel runs
        if (!ctx->h_feed) ZOLA_CUDA_CHECK(cudaMallocHost(&ctx->h_feed, 64 * sizeof(int)), ctx);
        if (!ctx->ev_init) ZOLA_CUDA_CHECK(cudaEventCreateWithFlags(&ctx->ev_init, cudaEventDisableTiming), ctx);
        ZOLA_CUDA_CHECK(cudaStreamSynchronize(ctx->feed_stream), ctx);  // the previous call's count copies are done
        ZOLA_CUDA_CHECK(cudaEventRecord(ctx->ev_init, st), ctx);
        ZOLA_CUDA_CHECK(cudaStreamWaitEvent(ctx->feed_stream, ctx->ev_init, 0), ctx);
        for (int c = 1; c < feed->n_chunks && c < 64; ++c) {
            ctx->h_feed[c] = feed->chunk_end[c];
            ZOLA_CUDA_CHECK(cudaStreamWaitEvent(ctx->feed_stream, feed->ev[c], 0), ctx);
            ZOLA_CUDA_CHECK(cudaMemcpyAsync(D.navail, ctx->h_feed + c, sizeof(int), cudaMemcpyHostToDevice,
                                            ctx->feed_stream), ctx);
        }
    }
    FlowRoles roles;
    roles.first[0] = 0;
    for (int s = 0; s < FLOW_STAGES; ++s) roles.first[s + 1] = roles.first[s] + shape.ctas[s];
    SplitDev dv = D;
    FitIO io = F;
    void* args[] = {&dv, &io, &roles};
    const void* fn = D.W == 32 ? (const void*)k_flow<32> : D.W == 64 ? (const void*)k_flow<64> : (const void*)k_flow<128>;
    if (trial) {
        for (auto& e : ctx->tune_ev)
            if (!e) ZOLA_CUDA_CHECK(cudaEventCreate(&e), ctx);
        ZOLA_CUDA_CHECK(cudaEventRecord(ctx->tune_ev[0], st), ctx);
    }
    prof_begin(ctx, 8, st);
    cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(FLOW_THREADS), args, sp.sflow, st);
    prof_end(ctx, st);
    ctx->launches++;
    if (e != cudaSuccess) {
        ctx->err = std::string("split fit (dataflow kernel): ") + cudaGetErrorString(e);
        return ZOLA_E_CUDA;
    }
    if (trial) ZOLA_CUDA_CHECK(cudaEventRecord(ctx->tune_ev[1], st), ctx);
    int active, err;
    rc = read_flags(ctx, D, st, &active, &err);
    if (rc) return rc;
    if (err == 2) {
        ctx->err = "split fit: no unit became ready within the wait limit (inputs did not arrive)";
        return ZOLA_E_TIMEOUT;
    }
    if (err == 3) {
        ctx->err = "split fit: more model evaluations than the ROIs allow (internal error)";
        return ZOLA_E_CUDA;
    }
    if (err) {
        ctx->err = "split fit: a bounded device wait timed out";
        return ZOLA_E_TIMEOUT;
    }
    // per stage: busy fraction and device clocks per unit (bookkeeping of the last launch)
    if (!ctx->h_tune) ZOLA_CUDA_CHECK(cudaMallocHost(&ctx->h_tune, (3 * (size_t)grid + 1) * 8), ctx);
    ZOLA_CUDA_CHECK(cudaMemcpy(ctx->h_tune, D.evals, (3 * (size_t)grid + 1) * 8, cudaMemcpyDeviceToHost), ctx);
    {
        const unsigned long long* clk = ctx->h_tune + 1;
        int b = 0;
        for (int s = 0; s < FLOW_STAGES; ++s) {
            double idle = 0, tot = 0, units = 0;
            for (int k = 0; k < shape.ctas[s]; ++k, ++b) {
                idle += (double)clk[3 * b];
                tot += (double)clk[3 * b + 1];
                units += (double)clk[3 * b + 2];
            }
            ctx->flow_busy[s] = tot > 0 ? 1.0 - idle / tot : 0.0;
            ctx->flow_clk_per_unit[s] = units > 0 ? (tot - idle) / units : 0.0;
        }
        ctx->flow_evals = (double)ctx->h_tune[0];
    }
    if (trial) {
        float ms = 0;
        ZOLA_CUDA_CHECK(cudaEventElapsedTime(&ms, ctx->tune_ev[0], ctx->tune_ev[1]), ctx);
        if (ctx->h_tune[0] > 0) tune_record(ctx, key, shape, ms * 1e6 / (double)ctx->h_tune[0], ctx->h_tune + 1);
    }
    return ZOLA_OK;
}

// The shape the dataflow kernel uses for this PSF and window; true when it was tuned.
bool flow_shape(zola_ctx* ctx, zola_psf* p, WindowTables* w, FlowShape* out, double* ns_per_eval) {
    auto it = ctx->tunes.find(tune_key(p, w));
    const bool tuned = it != ctx->tunes.end() && it->second.done;
    *out = tuned ? it->second.best : default_shape(w->W, ctx->num_sms);
    if (ns_per_eval) *ns_per_eval = tuned ? it->second.best_ns : 0.0;
    return tuned;
}

// One LM round of the round-based kernels: pupil DFT, window DFT, row blur,
// column blur + sums, LM step.  Window 128: column blur and likelihood sums in
// one persistent kernel, one slot at a time over all its threads (the maps
// never leave the SM).  Smaller windows: the unit's maps go to shared memory
// and its slots are summed together.  The two sum in different orders; the
// choice depends on R alone so that a fit never depends on the batch it is in.
static void issue_round(zola_ctx* ctx, const SplitPool& sp, const FitIO& F, cudaStream_t st) {
    launch_stages123(ctx, sp, F, st);
    prof_begin(ctx, 3, st);
    if (sp.pl->W >= S45_MIN_W)
        k_stage45p<<<unit_grid(ctx, sp), S45_THREADS, sp.s45, st>>>(sp.D, F);
    else
        k_stage45s<<<unit_grid(ctx, sp), S45S_THREADS, sp.s45, st>>>(sp.D, F);
    prof_end(ctx, st);
    prof_begin(ctx, 7, st);
    k_lm<<<(sp.D.P + 127) / 128, 128, 0, st>>>(sp.D, F);
    prof_end(ctx, st);
    ctx->launches += 2;
}

// Four rounds: 20 launches whose arguments stay the same for the whole fit.
static void issue_rounds(zola_ctx* ctx, const SplitPool& sp, const FitIO& F, cudaStream_t st) {
    for (int k = 0; k < 4; ++k) issue_round(ctx, sp, F, st);
}

// The four rounds captured once per fit as a CUDA graph and replayed between
// the host's flag reads: one launch instead of 20 per block.  Not with the
// context's kernel profiling on (its events bracket single launches); if the
// capture fails the rounds are issued directly.
struct RoundGraph {
    cudaGraphExec_t exec = nullptr;
    RoundGraph() = default;
    RoundGraph(const RoundGraph&) = delete;
    RoundGraph& operator=(const RoundGraph&) = delete;
    ~RoundGraph() { if (exec) cudaGraphExecDestroy(exec); }
    void capture(zola_ctx* ctx, const SplitPool& sp, const FitIO& F, cudaStream_t st) {
        if (ctx->profile || !ctx->round_graphs) return;
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        const long long l0 = ctx->launches;
        issue_rounds(ctx, sp, F, st);
        ctx->launches = l0;
        if (cudaStreamEndCapture(st, &g) != cudaSuccess || !g) {
            cudaGetLastError();
            return;
        }
        if (cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) {
            exec = nullptr;
            cudaGetLastError();
        }
        cudaGraphDestroy(g);
    }
    void run(zola_ctx* ctx, const SplitPool& sp, const FitIO& F, cudaStream_t st) {
        if (exec && cudaGraphLaunch(exec, st) == cudaSuccess) {
            ctx->launches += 20;
            return;
        }
        issue_rounds(ctx, sp, F, st);
    }
};

int launch_fit_split(zola_ctx* ctx, zola_psf* p, WindowTables* w, const float* d_rois, const float* d_scmos,
                     const double* d_init, int n,
                     const zola_fit_params* prm, double* d_out5, double* d_crlb5, double* d_nll, int* d_status,
                     int* d_iters, cudaStream_t st, const RoiFeed* feed, const int* d_avail) {
    // the likelihood is summed in FP32 and the model is good to about 2^-22:
    // likelihood changes below 1e-3 are not resolved (lm_update)
    FitParamsDev fp{prm->zmin, prm->zmax, prm->xymax, prm->tol_xyz, prm->step_xy, prm->step_z, prm->max_iter, 1e-3};
    const FitIO F{d_rois, d_scmos, d_init, n, fp, d_out5, d_crlb5, d_nll, d_status, d_iters};
    if (ctx->split_mode == ZOLA_SPLIT_FLOW || d_avail) return launch_fit_flow(ctx, p, w, F, st, feed, d_avail);
    SplitPool sp;
    const std::string pkey = pool_key(p, w);
    bool trial = false;
    const int pool = pick_pool(ctx, pkey, n, &trial);
    trial = trial && !feed && ctx->split_mode == ZOLA_SPLIT_STAGED;
    int rc = setup_pool(ctx, p, w, n, pool, sp, st);
    if (rc) return rc;
    const SplitDev& D = sp.D;
    const int P = D.P;
    if (trial) {
        if (!ctx->tune_ev[0])
            for (auto& e : ctx->tune_ev) ZOLA_CUDA_CHECK(cudaEventCreate(&e), ctx);
        ZOLA_CUDA_CHECK(cudaEventRecord(ctx->tune_ev[0], st), ctx);
    }
    // inputs still arriving: the fit starts on the first chunk, and chunks are
    // handed to the pool as their copies complete
    int chunk = 0, navail = n, queue = 0;
    if (feed && feed->n_chunks > 0) {
        ZOLA_CUDA_CHECK(cudaStreamWaitEvent(st, feed->ev[0], 0), ctx);
        navail = feed->chunk_end[0];
    }
    auto poll_feed = [&](bool block) -> int {
        const int before = navail;
        while (feed && chunk + 1 < feed->n_chunks) {
            if (block) {
                ZOLA_CUDA_CHECK(cudaEventSynchronize(feed->ev[chunk + 1]), ctx);
                block = false;
            } else if (cudaEventQuery(feed->ev[chunk + 1]) != cudaSuccess) {
                break;
            }
            navail = feed->chunk_end[++chunk];
        }
        if (navail != before) {
            k_set_int<<<1, 1, 0, st>>>(D.navail, navail);
            ctx->launches++;
        }
        return ZOLA_OK;
    };
    k_init_slots<<<(P + 127) / 128, 128, 0, st>>>(D, d_init, n, navail, fp);
    ctx->launches++;
    ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
    const int max_rounds = (prm->max_iter + 2) * ((n + P - 1) / P + 1) + 8 + 4 * (feed ? feed->n_chunks : 0);
    int rounds = 0;
    const bool fused = ctx->split_mode == ZOLA_SPLIT_FUSED && fused_fits(*sp.pl);
    RoundGraph graph;
    if (!fused && !feed) graph.capture(ctx, sp, F, st);
    while (true) {
        if (!fused && !feed) {
            graph.run(ctx, sp, F, st);
        } else for (int k = 0; k < 4; ++k) {
            if (feed && queue < n) {  // idle slots take ROIs that arrived since
                k_refill<<<(P + 127) / 128, 128, 0, st>>>(D, d_init, n, fp);
                ctx->launches++;
            }
            if (fused) {
                prof_begin(ctx, 0, st);
                launch_stage1(ctx, sp, F, st);
                prof_end(ctx, st);
                prof_begin(ctx, 4, st);
                k_fused25<<<P / sp.pl->G2, SPLIT_THREADS, sp.sf, st>>>(D, d_rois, d_scmos, d_init, n, fp, d_out5, d_crlb5, d_nll,
                                                                      d_status, d_iters);
                prof_end(ctx, st);
                ctx->launches += 2;
                continue;
            }
            issue_round(ctx, sp, F, st);
        }
        rounds += 4;
        ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
        int active, err;
        rc = read_flags(ctx, D, st, &active, &err, &queue);
        if (rc) return rc;
        if (err) { ctx->err = "split fit: a bounded device wait timed out"; return ZOLA_E_TIMEOUT; }
        if ((rc = poll_feed(false))) return rc;
        if (active <= 0) {
            if (queue >= n) break;
            // every slot idle and the queue at the arrived ROIs: wait for the next chunk
            if (navail <= queue && (rc = poll_feed(true))) return rc;
        }
        if (rounds > max_rounds) { ctx->err = "split fit: did not drain the ROI queue"; return ZOLA_E_TIMEOUT; }
    }
    if (trial) {  // device time per model evaluation of this pool size
        unsigned long long evals = 0;
        float ms = 0;
        ZOLA_CUDA_CHECK(cudaEventRecord(ctx->tune_ev[1], st), ctx);
        ZOLA_CUDA_CHECK(cudaMemcpyAsync(&evals, D.evals, sizeof evals, cudaMemcpyDeviceToHost, st), ctx);
        ZOLA_CUDA_CHECK(cudaEventSynchronize(ctx->tune_ev[1]), ctx);
        ZOLA_CUDA_CHECK(cudaEventElapsedTime(&ms, ctx->tune_ev[0], ctx->tune_ev[1]), ctx);
        if (evals > 0) pool_record(ctx, pkey, pool, ms * 1e6 / (double)evals);
    }
    return ZOLA_OK;
}

int split_pool_choice(zola_psf* p, WindowTables* w, int* pool, double* ns_per_eval) {
    const auto it = p->ctx->pool_tunes.find(pool_key(p, w));
    const bool tuned = it != p->ctx->pool_tunes.end() && it->second.done;
    if (pool) *pool = tuned ? it->second.best : p->ctx->split_pool_max;
    if (ns_per_eval) *ns_per_eval = tuned ? it->second.best_ns : 0.0;
    return tuned ? 1 : 0;
}

// ------------------------------------------------------- mixed batches -----
// Several ROI classes (PSF, ROI side) fitted in one call: each class gets its
// own slot pool (carved from one scratch area) and its own stream, and the host
// interleaves the classes' LM rounds, so the draining tail of one class
// overlaps the others' work.  Each ROI's fit is the same bit for bit as in a
// call of its class alone (a fit does not depend on its batch).
int launch_fit_split_mixed(zola_ctx* ctx, int nc, MixedClass* mc, cudaStream_t st, const RoiFeed* feeds) {
    if (nc > ZOLA_MAX_CLASSES) {
        ctx->err = "zola_fit_batch_mixed_dev: too many classes";
        return ZOLA_E_ARG;
    }
    std::vector<SplitPool> sp(nc);
    std::vector<size_t> off(nc + 1, 0);
    std::vector<int> pool(nc, 0);
    for (int c = 0; c < nc; ++c) {
        size_t need = 0;
        bool trial = false;
        pool[c] = pick_pool(ctx, pool_key(mc[c].p, mc[c].w), 0, &trial);  // explicit, tuned or automatic
        int rc = setup_pool(ctx, mc[c].p, mc[c].w, mc[c].F.n, pool[c], sp[c], st, 0, nullptr, &need);
        if (rc) return rc;
        off[c + 1] = off[c] + (need + 4095) / 4096 * 4096;
    }
    if (ensure_scratch(ctx, off[nc], ctx->err)) return ZOLA_E_CUDA;
    if (!ctx->mix_ev[0])
        for (auto& e : ctx->mix_ev) ZOLA_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), ctx);
    if (!ctx->h_mix) ZOLA_CUDA_CHECK(cudaMallocHost(&ctx->h_mix, 4 * ZOLA_MAX_CLASSES * sizeof(int)), ctx);
    ZOLA_CUDA_CHECK(cudaEventRecord(ctx->mix_ev[ZOLA_MAX_CLASSES], st), ctx);
    // A class whose inputs are still arriving (feeds[c] with chunks) starts on its
    // first chunk; between blocks of rounds the host hands it the chunks that have
    // landed (the device count of arrived ROIs), and idle slots take them.
    struct State {
        int rounds = 0, max_rounds = 0, chunk = 0, navail = 0, queue = 0;
        bool done = false, feed = false;
    };
    std::vector<State> S(nc);
    RoundGraph graphs[ZOLA_MAX_CLASSES];
    for (int c = 0; c < nc; ++c) {
        if (!ctx->mix_stream[c]) ZOLA_CUDA_CHECK(cudaStreamCreateWithFlags(&ctx->mix_stream[c], cudaStreamNonBlocking), ctx);
        cudaStream_t cs = ctx->mix_stream[c];
        const FitIO& F = mc[c].F;
        ZOLA_CUDA_CHECK(cudaStreamWaitEvent(cs, ctx->mix_ev[ZOLA_MAX_CLASSES], 0), ctx);
        S[c].feed = feeds && feeds[c].n_chunks > 0;
        S[c].navail = F.n;
        if (S[c].feed) {
            ZOLA_CUDA_CHECK(cudaStreamWaitEvent(cs, feeds[c].ev[0], 0), ctx);  // the first chunk has landed
            S[c].navail = feeds[c].chunk_end[0];
        }
        int rc = setup_pool(ctx, mc[c].p, mc[c].w, F.n, pool[c], sp[c], cs, 0, (char*)ctx->scratch + off[c]);
        if (rc) return rc;
        const SplitDev& D = sp[c].D;
        k_init_slots<<<(D.P + 127) / 128, 128, 0, cs>>>(D, F.init, F.n, S[c].navail, F.prm);
        ctx->launches++;
        S[c].max_rounds = (F.prm.max_iter + 2) * ((F.n + D.P - 1) / D.P + 1) + 8 + (S[c].feed ? 4 * feeds[c].n_chunks : 0);
        S[c].done = F.n == 0;
        if (!S[c].done && !S[c].feed) graphs[c].capture(ctx, sp[c], F, cs);
    }
    ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
    // hand class c the chunks that have landed (block: wait for at least one)
    auto poll_feed = [&](int c, bool block) -> int {
        State& q = S[c];
        const RoiFeed& fd = feeds[c];
        const int before = q.navail;
        while (q.chunk + 1 < fd.n_chunks) {
            if (block) {
                ZOLA_CUDA_CHECK(cudaEventSynchronize(fd.ev[q.chunk + 1]), ctx);
                block = false;
            } else if (cudaEventQuery(fd.ev[q.chunk + 1]) != cudaSuccess) {
                break;
            }
            q.navail = fd.chunk_end[++q.chunk];
        }
        if (q.navail != before) {
            k_set_int<<<1, 1, 0, ctx->mix_stream[c]>>>(sp[c].D.navail, q.navail);
            ctx->launches++;
        }
        return ZOLA_OK;
    };
    for (;;) {
        bool any = false;
        for (int c = 0; c < nc; ++c) {
            if (S[c].done) continue;
            any = true;
            cudaStream_t cs = ctx->mix_stream[c];
            const SplitPool& p = sp[c];
            if (S[c].feed && S[c].queue < mc[c].F.n) {
                for (int k = 0; k < 4; ++k) {  // idle slots take ROIs that arrived since
                    k_refill<<<(p.D.P + 127) / 128, 128, 0, cs>>>(p.D, mc[c].F.init, mc[c].F.n, mc[c].F.prm);
                    ctx->launches++;
                    issue_round(ctx, p, mc[c].F, cs);
                }
            } else {
                if (S[c].feed && !graphs[c].exec) graphs[c].capture(ctx, p, mc[c].F, cs);  // every ROI taken
                graphs[c].run(ctx, p, mc[c].F, cs);
            }
            S[c].rounds += 4;
            ZOLA_CUDA_CHECK(cudaMemcpyAsync(ctx->h_mix + 4 * c, p.D.queue, 3 * sizeof(int), cudaMemcpyDeviceToHost, cs),
                            ctx);
            ZOLA_CUDA_CHECK(cudaEventRecord(ctx->mix_ev[c], cs), ctx);
        }
        if (!any) break;
        ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
        for (int c = 0; c < nc; ++c) {  // the other classes keep running while one is read back
            if (S[c].done) continue;
            ZOLA_CUDA_CHECK(cudaEventSynchronize(ctx->mix_ev[c]), ctx);
            const int queue = ctx->h_mix[4 * c], active = ctx->h_mix[4 * c + 1], err = ctx->h_mix[4 * c + 2];
            if (err) {
                ctx->err = "split fit: a bounded device wait timed out";
                return ZOLA_E_TIMEOUT;
            }
            S[c].queue = queue;
            if (S[c].feed) {
                int rc = poll_feed(c, false);
                // every slot idle and the queue at the arrived ROIs: wait for the next chunk
                if (!rc && active <= 0 && queue < mc[c].F.n && S[c].navail <= queue) rc = poll_feed(c, true);
                if (rc) return rc;
            }
            if (active <= 0 && queue >= mc[c].F.n) S[c].done = true;
            else if (S[c].rounds > S[c].max_rounds) {
                ctx->err = "split fit: did not drain the ROI queue";
                return ZOLA_E_TIMEOUT;
            }
        }
    }
    for (int c = 0; c < nc; ++c) {
        ZOLA_CUDA_CHECK(cudaEventRecord(ctx->mix_ev[c], ctx->mix_stream[c]), ctx);
        ZOLA_CUDA_CHECK(cudaStreamWaitEvent(st, ctx->mix_ev[c], 0), ctx);
    }
    return ZOLA_OK;
}

}  // namespace zola
