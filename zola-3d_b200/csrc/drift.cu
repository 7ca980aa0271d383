// 3-D drift correction (process/cpu/DriftCorrection.java:125-990, utils/SplineFit.java).
//
// The localizations are binned in time; for every window of sizeFFT voxels
// (windows overlap by half, :280-300) each bin's 3-D histogram is zero-padded
// to twice the window, Fourier transformed, multiplied by a Gaussian of width
// 3 x the mean CRLB (float-rounded as the reference, :290-320), and every pair
// of bins (t < s) is cross-correlated: IFFT(F_t conj(F_s)), centred and
// cropped to the window, summed over the windows (:700-780).  The drift of a
// pair is the centroid of the values above the 95% quantile in the 11^3
// neighbourhood of the first maximum (LocalMaxima, :1084-1200); bin 0 is the
// reference, and with more than two bins the drift of every bin comes from the
// least squares over all pairs with two passes of outlier rejection at the
// mean CRLB (:540-640).  The per-localization drift is the SplineFit of the
// bin drifts at its frame (:660-700).
//
// GPU: histograms by atomic adds, batched 3-D C2C FFTs (the hand-written
// radix-2 transform below, single precision like the reference's float
// transforms), pair products, inverse FFTs and the centring crop in chunks of
// pairs, and one CTA per pair for the peak centroid.  The circular shift the reference applies before the forward
// FFT multiplies every spectrum by the same sign pattern, which cancels in
// F_t conj(F_s), so it is left out.  The least squares and the spline run on
// the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "zola_internal.h"

namespace zola {

struct DriftDev {
    int P0, P1, P2;          // padded cube [z][y][x]: P0 = z, P1 = y, P2 = x
    int S0, S1, S2;          // window (crop) sizes z, y, x
    int bins;
    double px;               // voxel size, nm
    double minX, minY, minZ;
    int minF, maxF;
    double g0[3], g1[3];     // window bounds x, y, z (nm from the minima)
};

__global__ void k_drift_hist(DriftDev D, const double* xyz, const int* frame, int n, float2* cubes) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double x = xyz[3 * k] - D.minX, y = xyz[3 * k + 1] - D.minY, z = xyz[3 * k + 2] - D.minZ;
    if (!(x >= D.g0[0] && x < D.g1[0] && y >= D.g0[1] && y < D.g1[1] && z >= D.g0[2] && z < D.g1[2])) return;
    const int b = D.bins * (frame[k] - D.minF) / (1 + D.maxF - D.minF);
    const int xi = D.S2 / 2 + min(max((int)(fmod(x, D.S2 * D.px) / D.px), 0), D.S2 - 1);
    const int yi = D.S1 / 2 + min(max((int)(fmod(y, D.S1 * D.px) / D.px), 0), D.S1 - 1);
    const int zi = D.S0 / 2 + min(max((int)(fmod(z, D.S0 * D.px) / D.px), 0), D.S0 - 1);
    const size_t PV = (size_t)D.P0 * D.P1 * D.P2;
    atomicAdd(&cubes[(size_t)b * PV + ((size_t)zi * D.P1 + yi) * D.P2 + xi].x, 1.0f);
}

// Spectra times the float-rounded Fourier Gaussian (frequency index q -> q or q - P).
__global__ void k_drift_gauss(DriftDev D, float2* spec, double sf0, double sf1, double sf2) {
    const size_t PV = (size_t)D.P0 * D.P1 * D.P2;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < PV * D.bins; k += (size_t)gridDim.x * blockDim.x) {
        const size_t v = k % PV;
        const int c = (int)(v % D.P2), b = (int)((v / D.P2) % D.P1), a = (int)(v / ((size_t)D.P2 * D.P1));
        const double dz = a < D.P0 / 2 ? a : a - D.P0, dy = b < D.P1 / 2 ? b : b - D.P1, dx = c < D.P2 / 2 ? c : c - D.P2;
        const float g = (float)exp(-.5 * (dx * dx / sf2 + dy * dy / sf1 + dz * dz / sf0));
        spec[k].x *= g;
        spec[k].y *= g;
    }
}

// ---------------------------------------------------------------------------
// Batched complex FFT along one axis of [outer][L][inner] data (L a power of
// two, 2 .. 256): line (o, i) holds the elements (o L + k) inner + i.  A CTA
// takes TL consecutive lines into shared memory (bit-reversed), runs the
// log2(L) radix-2 decimation-in-time stages there and writes them back in
// place.  Loads and stores run along the line (inner = 1) or across lines
// (inner > 1), whichever is contiguous in memory.  Unnormalised; sign -1 is
// exp(-2 pi i j k / L) (forward), +1 the inverse.  tw[m] = exp(-2 pi i m / 256),
// m < 128, rounded from double; length L uses every (256 / L)-th entry.
constexpr int FFT_LMAX = 256, FFT_THREADS = 256;

__global__ void __launch_bounds__(FFT_THREADS) k_fft_lines(float2* data, int L, int lg, long long inner,
                                                           long long lines, int TL, const float2* tw, float sign) {
    extern __shared__ float2 sbuf[];
    const int LS = L + 1;
    const long long q0 = (long long)blockIdx.x * TL;
    const int nl = (int)min((long long)TL, lines - q0);
    auto addr = [&](int q, int k) {
        const long long line = q0 + q, o = line / inner, i = line - o * inner;
        return (o * L + k) * inner + i;
    };
    for (int e = threadIdx.x; e < nl * L; e += FFT_THREADS) {
        int q, k;
        if (inner == 1) { q = e / L; k = e - q * L; } else { k = e / nl; q = e - k * nl; }
        sbuf[q * LS + (int)(__brev((unsigned)k) >> (32 - lg))] = data[addr(q, k)];
    }
    __syncthreads();
    const int H = L / 2;
    for (int half = 1; half < L; half <<= 1) {
        const int ts = (FFT_LMAX / 2) / half;
        for (int b = threadIdx.x; b < nl * H; b += FFT_THREADS) {
            const int q = b / H, j = b - q * H, m = j & (half - 1);
            const int i0 = q * LS + 2 * (j - m) + m, i1 = i0 + half;
            float2 w = tw[m * ts];
            w.y *= -sign;
            const float2 a = sbuf[i0], c = sbuf[i1];
            const float2 t = make_float2(w.x * c.x - w.y * c.y, w.x * c.y + w.y * c.x);
            sbuf[i0] = make_float2(a.x + t.x, a.y + t.y);
            sbuf[i1] = make_float2(a.x - t.x, a.y - t.y);
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < nl * L; e += FFT_THREADS) {
        int q, k;
        if (inner == 1) { q = e / L; k = e - q * L; } else { k = e / nl; q = e - k * nl; }
        data[addr(q, k)] = sbuf[q * LS + k];
    }
}

// In-place 3-D FFTs of `batch` cubes [P0][P1][P2] (x = P2 fastest), one pass per axis.
static void fft3d(zola_ctx* ctx, float2* d, int batch, int P0, int P1, int P2, float sign, const float2* tw,
                  cudaStream_t st) {
    const int dims[3] = {P0, P1, P2};
    const long long total = (long long)batch * P0 * P1 * P2;
    long long inner = 1;
    for (int ax = 2; ax >= 0; --ax) {
        const int L = dims[ax];
        if (L > 1) {
            int lg = 0;
            while ((1 << lg) < L) ++lg;
            const long long lines = total / L;
            const int TL = (int)std::max<long long>(1, std::min<long long>(lines, 4096 / (L + 1)));  // <= 32 KB
            const size_t smem = (size_t)TL * (L + 1) * sizeof(float2);
            k_fft_lines<<<(unsigned)((lines + TL - 1) / TL), FFT_THREADS, smem, st>>>(d, L, lg, inner, lines, TL, tw,
                                                                                     sign);
            ctx->launches++;
        }
        inner *= L;
    }
}

// out[j] = F_p1 conj(F_p2) for the pairs first .. first + npair - 1.
__global__ void k_drift_pairs(DriftDev D, const float2* spec, const int* p1, const int* p2, int first, int npair,
                              float2* out) {
    const size_t PV = (size_t)D.P0 * D.P1 * D.P2;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < PV * npair; k += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(k / PV);
        const size_t v = k % PV;
        const float2 a = spec[(size_t)p1[first + j] * PV + v], b = spec[(size_t)p2[first + j] * PV + v];
        out[k] = make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
    }
}

// result[pair] += real part of the centred correlation, cropped to the window.
__global__ void k_drift_crop(DriftDev D, const float2* corr, int first, int npair, float* result) {
    const size_t PV = (size_t)D.P0 * D.P1 * D.P2, RV = (size_t)D.S0 * D.S1 * D.S2;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < RV * npair; k += (size_t)gridDim.x * blockDim.x) {
        const int j = (int)(k / RV);
        const size_t v = k % RV;
        const int c = (int)(v % D.S2), b = (int)((v / D.S2) % D.S1), a = (int)(v / ((size_t)D.S2 * D.S1));
        const int as = (a + D.S0 / 2 + D.P0 / 2) % D.P0, bs = (b + D.S1 / 2 + D.P1 / 2) % D.P1,
                  cs = (c + D.S2 / 2 + D.P2 / 2) % D.P2;
        result[(size_t)(first + j) * RV + v] += corr[(size_t)j * PV + ((size_t)as * D.P1 + bs) * D.P2 + cs].x;
    }
}

// LocalMaxima.run(0.95) per pair (one CTA): first maximum above
// Double.MIN_VALUE in scan order, the in-bounds values of the odd patch
// around it (<= 11 per axis, < size), the 95% quantile, and the centroid of
// the values above it; drift[pair] = -(centroid - size/2) along z, y, x.
constexpr int LM_THREADS = 256;
__global__ void __launch_bounds__(LM_THREADS) k_drift_peak(DriftDev D, const float* result, double* drift) {
    __shared__ float vals[2048];
    __shared__ float bv[LM_THREADS];
    __shared__ long long bi[LM_THREADS];
    __shared__ double red[4][LM_THREADS / 32];
    const int W0 = D.S0, W1 = D.S1, W2 = D.S2;
    const size_t RV = (size_t)W0 * W1 * W2;
    const float* im = result + (size_t)blockIdx.x * RV;
    float best = 0.0f;
    long long bidx = -1;
    for (size_t k = threadIdx.x; k < RV; k += LM_THREADS) {
        const float v = im[k];
        if (v > 0.0f && (bidx < 0 || v > best)) { best = v; bidx = (long long)k; }
    }
    bv[threadIdx.x] = best;
    bi[threadIdx.x] = bidx;
    __syncthreads();
    if (threadIdx.x == 0) {  // strict > in scan order = the first index among equal maxima
        float m = 0.0f;
        long long idx = -1;
        for (int t = 0; t < LM_THREADS; ++t) {
            if (bi[t] < 0) continue;
            if (idx < 0 || bv[t] > m || (bv[t] == m && bi[t] < idx)) { m = bv[t]; idx = bi[t]; }
        }
        bi[0] = idx < 0 ? 0 : idx;
    }
    __syncthreads();
    const long long mi = bi[0];
    const int a0 = (int)(mi / ((long long)W1 * W2)), b0 = (int)((mi / W2) % W1), c0 = (int)(mi % W2);
    int s0 = min(11, W0 - 1), s1 = min(11, W1 - 1), s2 = min(11, W2 - 1);
    if (s0 % 2 == 0) s0--;
    if (s1 % 2 == 0) s1--;
    if (s2 % 2 == 0) s2--;
    // a one-voxel axis (flat data; the reference throws there) keeps its single voxel
    s0 = max(s0, 1); s1 = max(s1, 1); s2 = max(s2, 1);
    const int np = s0 * s1 * s2;
    // gather in scan order (inside-the-volume entries), pad with +inf for the sort
    __shared__ int number;
    if (threadIdx.x == 0) {
        int cnt = 0;
        for (int q = 0; q < np; ++q) {
            const int i = q / (s1 * s2), ii = (q / s2) % s1, iii = q % s2;
            const int A = i + a0 - s0 / 2, B = ii + b0 - s1 / 2, C = iii + c0 - s2 / 2;
            if (A >= 0 && B >= 0 && C >= 0 && A < W0 && B < W1 && C < W2) vals[cnt++] = im[((size_t)A * W1 + B) * W2 + C];
        }
        number = cnt;
    }
    __syncthreads();
    for (int q = number + threadIdx.x; q < 2048; q += LM_THREADS) vals[q] = INFINITY;
    __syncthreads();
    for (int k = 2; k <= 2048; k <<= 1)  // bitonic sort, ascending
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < 2048; t += LM_THREADS) {
                const int p = t ^ j;
                if (p > t) {
                    const bool up = (t & k) == 0;
                    const float x = vals[t], y = vals[p];
                    if ((x > y) == up) { vals[t] = y; vals[p] = x; }
                }
            }
            __syncthreads();
        }
    const float thr = vals[(int)((number - 1) * .95)];
    double acc[4] = {0, 0, 0, 0};
    for (int q = threadIdx.x; q < np; q += LM_THREADS) {
        const int i = q / (s1 * s2), ii = (q / s2) % s1, iii = q % s2;
        const int A = i + a0 - s0 / 2, B = ii + b0 - s1 / 2, C = iii + c0 - s2 / 2;
        if (A >= 0 && B >= 0 && C >= 0 && A < W0 && B < W1 && C < W2) {
            const float v = im[((size_t)A * W1 + B) * W2 + C];
            if (v > thr) {
                acc[0] += v;
                acc[1] += (double)A * v;
                acc[2] += (double)B * v;
                acc[3] += (double)C * v;
            }
        }
    }
    for (int q = 0; q < 4; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[4] = {0, 0, 0, 0};
        for (int q = 0; q < 4; ++q)
            for (int w = 0; w < LM_THREADS / 32; ++w) t[q] += red[q][w];
        double* o = drift + 3 * (size_t)blockIdx.x;
        o[0] = -(t[1] / t[0] - W0 / 2);  // z
        o[1] = -(t[2] / t[0] - W1 / 2);  // y
        o[2] = -(t[3] / t[0] - W2 / 2);  // x
    }
}

}  // namespace zola

using namespace zola;

namespace {

// Gaussian elimination with partial pivoting; false on an exact-zero pivot
// (utils/GaussianElimination.java:107-140 with EPSILONF = 0).
bool gauss_solve(std::vector<std::vector<double>> A, std::vector<double> b, std::vector<double>& x) {
    const int N = (int)b.size();
    for (int p = 0; p < N; ++p) {
        int mx = p;
        for (int i = p + 1; i < N; ++i)
            if (std::fabs(A[i][p]) > std::fabs(A[mx][p])) mx = i;
        std::swap(A[p], A[mx]);
        std::swap(b[p], b[mx]);
        if (A[p][p] == 0) return false;
        for (int i = p + 1; i < N; ++i) {
            const double alpha = A[i][p] / A[p][p];
            b[i] -= alpha * b[p];
            for (int j = p; j < N; ++j) A[i][j] -= alpha * A[p][j];
        }
    }
    x.assign(N, 0.0);
    for (int i = N - 1; i >= 0; --i) {
        double sum = 0.0;
        for (int j = i + 1; j < N; ++j) sum += A[i][j] * x[j];
        x[i] = (b[i] - sum) / A[i][i];
    }
    return true;
}

// Polynomial through up to four knots in Newton form (value and slope).
struct Interp {
    int n = 0;
    double x[4] = {0, 0, 0, 0}, c[4] = {0, 0, 0, 0};
    void fit(const double* xs, const double* ys, int m) {
        n = m;
        for (int i = 0; i < m; ++i) { x[i] = xs[i]; c[i] = ys[i]; }
        for (int j = 1; j < m; ++j)
            for (int i = m - 1; i >= j; --i) c[i] = (c[i] - c[i - 1]) / (x[i] - x[i - j]);
    }
    double value(double t) const {
        double v = c[n - 1];
        for (int i = n - 2; i >= 0; --i) v = v * (t - x[i]) + c[i];
        return v;
    }
    double slope(double t) const {
        double v = c[n - 1], d = 0;
        for (int i = n - 2; i >= 0; --i) { d = d * (t - x[i]) + v; v = v * (t - x[i]) + c[i]; }
        return d;
    }
};

// SplineFit: cubic windows over four consecutive knots (the interpolating
// cubic; the reference solves its normal equations), knot interval id uses
// window id - 2, linear extrapolation with the end windows' slopes.
struct DriftSpline {
    std::vector<double> x, y;
    std::vector<Interp> pf;
    void fit(const std::vector<double>& xs, const std::vector<double>& ys) {
        x = xs;
        y = ys;
        for (size_t i = 0; i < x.size(); ++i)
            for (size_t ii = 1; ii < x.size() - i; ++ii)
                if (x[ii] < x[ii - 1]) { std::swap(x[ii], x[ii - 1]); std::swap(y[ii], y[ii - 1]); }
        const int L = (int)x.size();
        pf.assign(std::max(1, L + 1 - 4), Interp());
        if (L < 2) return;
        if (L < 4) { pf[0].fit(x.data(), y.data(), L); return; }
        for (int id = 0; id < L - 3; ++id) pf[id].fit(&x[id], &y[id], 4);
    }
    double eval(double X) const {
        const int L = (int)x.size();
        if (L < 2) return -1;
        if (L < 4) return pf[0].value(X);
        int id = 0;
        for (int i = 0; i < L; ++i) { id = i; if (X < x[i]) break; }
        if (X > x[L - 1]) id = L;
        if (id == 1) id = 2;
        if (id == L - 1) id = L - 2;
        if (id == 0) return pf[0].slope(x[0]) * (X - x[0]) + y[0];
        if (id == L) return pf[L - 4].slope(x[L - 1]) * (X - x[L - 1]) + y[L - 1];
        return pf[id - 2].value(X);
    }
};

}  // namespace

extern "C" int zola_drift(zola_ctx* ctx, const double* xyz_nm, const double* crlb_nm, const int* frame, int n,
                          const zola_drift_params* prm, double* bin_drift, double* loc_drift, double* pixel_nm_used) {
    if (!ctx) return ZOLA_E_ARG;
    if (!xyz_nm || !frame || !prm || !bin_drift || n < 1 || prm->bins < 1 || !(prm->pixel_nm > 0) ||
        !(prm->max_drift_um > 0)) {
        ctx->err = "zola_drift: need n >= 1, bins >= 1, pixel_nm > 0, max_drift_um > 0 and non-null buffers";
        return ZOLA_E_ARG;
    }
    cudaSetDevice(ctx->device);
    const int bin = prm->bins;
    double pixel = prm->pixel_nm;
    const double sub = prm->max_drift_um;
    int sizeFFT = (int)std::pow(2, (int)std::ceil(std::log(sub / (pixel / 1000.)) / std::log(2)));
    while (sizeFFT > 128) {  // the reference grows the voxel 1% at a time (:127-135)
        pixel *= 1.01;
        sizeFFT = (int)std::pow(2, (int)std::ceil(std::log(sub / (std::floor(pixel + 0.5) / 1000.)) / std::log(2)));
    }
    pixel = std::floor(pixel + 0.5);
    if (pixel_nm_used) *pixel_nm_used = pixel;
    // extents and mean precision (:180-260), with the reference's Double.MIN_VALUE start for the maxima
    const double DMIN = 4.9e-324, DMAX = 1.7976931348623157e308;
    double mn[3] = {DMAX, DMAX, DMAX}, mx[3] = {DMIN, DMIN, DMIN}, prec[3] = {0, 0, 0};
    int cnt[3] = {0, 0, 0}, minF = 2147483647, maxF = -2147483647 - 1;
    for (int k = 0; k < n; ++k) {
        for (int d = 0; d < 3; ++d) {
            const double v = xyz_nm[3 * k + d];
            if (v < mn[d]) mn[d] = v;
            if (v > mx[d]) mx[d] = v;
            if (crlb_nm && crlb_nm[3 * k + d] != -1) { prec[d] += crlb_nm[3 * k + d]; cnt[d]++; }
        }
        minF = std::min(minF, frame[k]);
        maxF = std::max(maxF, frame[k]);
    }
    for (int d = 0; d < 3; ++d) prec[d] = cnt[d] == 0 ? 50 : prec[d] / cnt[d];
    int ext[3], sF[3], nbw[3];
    for (int d = 0; d < 3; ++d) {
        ext[d] = std::max((int)std::ceil((mx[d] - mn[d]) / pixel), 1);
        sF[d] = std::min(sizeFFT, ext[d]);
        sF[d] = std::max(sF[d], (int)std::pow(2, std::ceil(std::log(sF[d]) / std::log(2))));
        nbw[d] = sF[d] < 2 ? 1 : (int)std::ceil((double)(ext[d] - sF[d] / 2) / (double)(sF[d] / 2));
    }
    DriftDev D{};
    D.P2 = 2 * sF[0]; D.P1 = 2 * sF[1]; D.P0 = 2 * sF[2];
    D.S2 = sF[0]; D.S1 = sF[1]; D.S0 = sF[2];
    D.bins = bin; D.px = pixel; D.minX = mn[0]; D.minY = mn[1]; D.minZ = mn[2]; D.minF = minF; D.maxF = maxF;
    const size_t PV = (size_t)D.P0 * D.P1 * D.P2, RV = (size_t)sF[0] * sF[1] * sF[2];
    const double sigma = 3 * std::max(std::max(prec[0], prec[1]), prec[2]) / pixel;
    double sfp[3];  // (1/sigma) P / (2 pi), squared, per axis x, y, z
    const int Pd[3] = {D.P2, D.P1, D.P0};
    for (int d = 0; d < 3; ++d) { const double v = (1. / sigma) * (double)Pd[d] / (M_PI * 2.); sfp[d] = v * v; }
    std::vector<int> p1, p2;
    for (int t = 0; t < bin - 1; ++t)
        for (int s = t + 1; s < bin; ++s) { p1.push_back(t); p2.push_back(s); }
    const int tot = (int)p1.size();
    // device buffers
    const size_t chunk_budget = (size_t)4 << 30;
    const int CH = tot > 0 ? (int)std::max<size_t>(1, std::min<size_t>(tot, chunk_budget / (PV * sizeof(float2)))) : 1;
    DevBuf<double> d_xyz, d_drift;
    DevBuf<int> d_frame, d_p1, d_p2;
    DevBuf<float2> d_spec, d_corr;
    DevBuf<float> d_res;
    ZOLA_CUDA_CHECK(d_xyz.alloc((size_t)3 * n), ctx);
    ZOLA_CUDA_CHECK(d_frame.alloc((size_t)n), ctx);
    ZOLA_CUDA_CHECK(d_spec.alloc(PV * bin), ctx);
    if (tot > 0) {
        ZOLA_CUDA_CHECK(d_p1.alloc((size_t)tot), ctx);
        ZOLA_CUDA_CHECK(d_p2.alloc((size_t)tot), ctx);
        ZOLA_CUDA_CHECK(d_corr.alloc(PV * CH), ctx);
        ZOLA_CUDA_CHECK(d_res.alloc(RV * tot), ctx);
        ZOLA_CUDA_CHECK(d_drift.alloc((size_t)3 * tot), ctx);
    }
    cudaStream_t st = ctx->stream;
    ZOLA_CUDA_CHECK(cudaMemcpyAsync(d_xyz.p, xyz_nm, (size_t)24 * n, cudaMemcpyHostToDevice, st), ctx);
    ZOLA_CUDA_CHECK(cudaMemcpyAsync(d_frame.p, frame, (size_t)4 * n, cudaMemcpyHostToDevice, st), ctx);
    if (tot > 0) {
        ZOLA_CUDA_CHECK(cudaMemcpyAsync(d_p1.p, p1.data(), (size_t)4 * tot, cudaMemcpyHostToDevice, st), ctx);
        ZOLA_CUDA_CHECK(cudaMemcpyAsync(d_p2.p, p2.data(), (size_t)4 * tot, cudaMemcpyHostToDevice, st), ctx);
        ZOLA_CUDA_CHECK(cudaMemsetAsync(d_res.p, 0, RV * tot * sizeof(float), st), ctx);
    }
    // twiddles exp(-2 pi i m / 256), m < 128, for every transform length
    DevBuf<float2> d_tw;
    {
        std::vector<float2> tw(FFT_LMAX / 2);
        for (int m = 0; m < FFT_LMAX / 2; ++m)
            tw[m] = make_float2((float)std::cos(2 * M_PI * m / FFT_LMAX), (float)-std::sin(2 * M_PI * m / FFT_LMAX));
        ZOLA_CUDA_CHECK(d_tw.alloc(tw.size()), ctx);
        ZOLA_CUDA_CHECK(cudaMemcpyAsync(d_tw.p, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, st),
                        ctx);
        ZOLA_CUDA_CHECK(cudaStreamSynchronize(st), ctx);  // tw is a host temporary
    }
    const int grid = ctx->num_sms * 8;
    for (int u = 0; u < nbw[0]; ++u)
        for (int uu = 0; uu < nbw[1]; ++uu)
            for (int uuu = 0; uuu < nbw[2]; ++uuu) {
                const int uv[3] = {u, uu, uuu};
                for (int d = 0; d < 3; ++d) {
                    D.g0[d] = (uv[d] / 2) * sF[d] * pixel + (uv[d] % 2) * (sF[d] / 2) * pixel;
                    D.g1[d] = (uv[d] / 2 + 1) * sF[d] * pixel + (uv[d] % 2) * (sF[d] / 2) * pixel;
                }
                ZOLA_CUDA_CHECK(cudaMemsetAsync(d_spec.p, 0, PV * bin * sizeof(float2), st), ctx);
                k_drift_hist<<<(n + 255) / 256, 256, 0, st>>>(D, d_xyz.p, d_frame.p, n, d_spec.p);
                fft3d(ctx, d_spec.p, bin, D.P0, D.P1, D.P2, -1.f, d_tw.p, st);
                k_drift_gauss<<<grid, 256, 0, st>>>(D, d_spec.p, sfp[2], sfp[1], sfp[0]);
                ctx->launches += 2;
                for (int first = 0; first < tot; first += CH) {
                    const int np = std::min(CH, tot - first);
                    k_drift_pairs<<<grid, 256, 0, st>>>(D, d_spec.p, d_p1.p, d_p2.p, first, np, d_corr.p);
                    fft3d(ctx, d_corr.p, np, D.P0, D.P1, D.P2, 1.f, d_tw.p, st);
                    k_drift_crop<<<grid, 256, 0, st>>>(D, d_corr.p, first, np, d_res.p);
                    ctx->launches += 2;
                }
                ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
            }
    std::vector<double> pd((size_t)3 * tot);
    if (tot > 0) {
        k_drift_peak<<<tot, LM_THREADS, 0, st>>>(D, d_res.p, d_drift.p);
        ctx->launches++;
        ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
        ZOLA_CUDA_CHECK(cudaMemcpyAsync(pd.data(), d_drift.p, pd.size() * 8, cudaMemcpyDeviceToHost, st), ctx);
    }
    ZOLA_CUDA_CHECK(cudaStreamSynchronize(st), ctx);
    // bin drifts: pairs with bin 0, then least squares over all pairs (:480-640)
    const double fpb = ((double)(maxF - minF)) / ((double)bin);
    std::vector<double> di(bin, 0.0), dr[3];
    for (int d = 0; d < 3; ++d) dr[d].assign(bin, 0.0);
    di[0] = (double)minF + fpb / 2.;
    std::vector<std::vector<double>> Am(tot, std::vector<double>(std::max(bin - 1, 0), 0.0));
    std::vector<double> Rm[3];
    for (int d = 0; d < 3; ++d) Rm[d].assign(tot, 0.0);
    for (int id = 0; id < tot; ++id) {
        const double drift[3] = {pd[3 * id + 2] * pixel, pd[3 * id + 1] * pixel, pd[3 * id] * pixel};  // x, y, z
        const int t = p1[id], s = p2[id];
        if (t == 0) {
            di[s] = (((double)s) / ((double)bin)) * ((double)(1. + maxF - minF)) + ((double)minF) + (fpb / 2.);
            for (int d = 0; d < 3; ++d) dr[d][s] = drift[d];
        }
        for (int d = 0; d < 3; ++d) Rm[d][id] = drift[d];
        if (t != 0) Am[id][t - 1] = -1;
        Am[id][s - 1] = 1;
    }
    if (bin > 2 && tot > bin) {
        std::vector<int> del[3];
        for (int check = 0; check < 2; ++check)
            for (int d = 0; d < 3; ++d) {
                std::vector<std::vector<double>> An;
                std::vector<double> Rn;
                for (int i = 0; i < tot; ++i) {
                    if (std::find(del[d].begin(), del[d].end(), i) != del[d].end()) continue;
                    An.push_back(Am[i]);
                    Rn.push_back(Rm[d][i]);
                }
                if ((int)An.size() < bin - 1) continue;
                const int m = bin - 1;
                std::vector<std::vector<double>> N(m, std::vector<double>(m, 0.0));
                std::vector<double> r(m, 0.0), sol;
                for (int a = 0; a < m; ++a) {
                    for (int b = 0; b < m; ++b)
                        for (size_t i = 0; i < An.size(); ++i) N[a][b] += An[i][a] * An[i][b];
                    for (size_t i = 0; i < An.size(); ++i) r[a] += An[i][a] * Rn[i];
                }
                if (!gauss_solve(N, r, sol)) continue;  // the reference logs and keeps the previous drifts
                for (size_t i = 0; i < An.size(); ++i) {
                    double fit = 0;
                    for (int a = 0; a < m; ++a) fit += An[i][a] * sol[a];
                    if (std::fabs(fit - Rn[i]) > prec[d]) del[d].push_back((int)i);
                }
                for (int a = 0; a < m; ++a) dr[d][a + 1] = sol[a];
            }
    }
    for (int b = 0; b < bin; ++b) {
        bin_drift[4 * b] = di[b];
        for (int d = 0; d < 3; ++d) bin_drift[4 * b + 1 + d] = dr[d][b];
    }
    if (loc_drift) {
        DriftSpline sp[3];
        for (int d = 0; d < 3; ++d) sp[d].fit(di, dr[d]);
        for (int k = 0; k < n; ++k)
            for (int d = 0; d < 3; ++d) loc_drift[3 * k + d] = sp[d].eval((double)frame[k]);
    }
    return ZOLA_OK;
}
