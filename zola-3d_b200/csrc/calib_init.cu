// Calibration data preparation: InitBackgroundAndPhotonNumber
// (process/InitBackgroundAndPhotonNumber.java).
//
//   photons = max((adu/gain) raw - offset adu/gain + 1, 0)            (:50-72)
//   seeds   refined to the centroid of the brightest 10% of the summed
//           patch's central half, if the move is below sizePatch/4    (:587-640)
//   stack statistics, low-voxel mask is2 = v <= mean + 3 std          (:642-705)
//   dimmest slice window (box filter +-sizeFilt), voxels of that window
//   whose 5x5x5 neighbourhood is all in is2, per-pixel mean over them,
//   order-2 polynomial surface by least squares                      (:706-900)
//   B_p = mean of the surface over the bead patch; A_p(z) = sum(patch - B_p),
//   box-filtered over +-sizeFilt slices; patches (outside: B_p)       (:110-420)
//
// The voxel passes (conversion, the four statistics, the masks, the dilated
// per-pixel means) run on the GPU with per-slice partial sums combined on the
// host in slice order; the per-bead steps and the 6 x 6 least squares are
// host code.  Image layout [slice][x][y] (first index x, as the reference's
// image[z][i][ii]).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "zola_internal.h"

namespace zola {

constexpr int CI_THREADS = 256;

__device__ inline double ci_block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0;
    for (int w = 0; w < CI_THREADS / 32; ++w) s += red[w];
    __syncthreads();
    return s;
}

// ADU -> photons (+1, clamped at 0); per-slice sum.  One CTA per slice.
__global__ void __launch_bounds__(CI_THREADS) k_ci_convert(const float* raw, int plane, double slope, double intercept,
                                                           double* im, double* sums) {
    __shared__ double red[CI_THREADS / 32];
    const size_t off = (size_t)blockIdx.x * plane;
    double s = 0;
    for (int k = threadIdx.x; k < plane; k += CI_THREADS) {
        double v = ((double)raw[off + k] * slope + intercept) + 1;
        if (v < 0) v = 0;
        im[off + k] = v;
        s += v;
    }
    s = ci_block_sum(s, red);
    if (threadIdx.x == 0) sums[blockIdx.x] = s;
}

// Per-slice statistics pass: mode 0 sum (v - m)^2; 1 sum and count of
// v <= thr; 2 sum (v - m)^2 over v <= thr; 3 sum and count of v <= thr2 (the
// is2 mask, also written out).
__global__ void __launch_bounds__(CI_THREADS) k_ci_stats(const double* im, int plane, int mode, double m, double thr,
                                                         double* sums, double* counts, unsigned char* is2) {
    __shared__ double red[CI_THREADS / 32];
    const size_t off = (size_t)blockIdx.x * plane;
    double s = 0, c = 0;
    for (int k = threadIdx.x; k < plane; k += CI_THREADS) {
        const double v = im[off + k];
        if (mode == 0) {
            s += (v - m) * (v - m);
        } else if (mode == 1) {
            if (v <= thr) { s += v; c += 1; }
        } else if (mode == 2) {
            if (v <= thr) s += (v - m) * (v - m);
        } else {
            const bool in = !(v > thr);
            is2[off + k] = in ? 1 : 0;
            if (in) { s += v; c += 1; }
        }
    }
    s = ci_block_sum(s, red);
    c = ci_block_sum(c, red);
    if (threadIdx.x == 0) {
        sums[blockIdx.x] = s;
        counts[blockIdx.x] = c;
    }
}

// Per pixel: slices z0..z1 whose 5 x 5 x 5 neighbourhood (inside the stack)
// is all in is2; count and sum of the pixel over them.
__global__ void k_ci_dilate(const double* im, const unsigned char* is2, int ns, int W, int H, int z0, int z1,
                            double* psum, int* pcount) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= W * H) return;
    const int i = k / H, ii = k % H;
    double s = 0;
    int c = 0;
    for (int z = z0; z <= z1; ++z) {
        bool ok = true;
        for (int u = -2; u <= 2 && ok; ++u)
            for (int uu = -2; uu <= 2 && ok; ++uu)
                for (int uuu = -2; uuu <= 2 && ok; ++uuu) {
                    const int zz = z + u, a = i + uu, b = ii + uuu;
                    if (zz >= 0 && zz < ns && a >= 0 && a < W && b >= 0 && b < H && !is2[((size_t)zz * W + a) * H + b])
                        ok = false;
                }
        if (ok) {
            ++c;
            s += im[((size_t)z * W + i) * H + ii];
        }
    }
    psum[k] = s;
    pcount[k] = c;
}

}  // namespace zola

using namespace zola;

namespace {

// Least squares on 1, x, x^2, y, x y, y^2 (normal equations, partial pivoting).
bool poly2_fit(const std::vector<double>& xs, const std::vector<double>& ys, const std::vector<double>& v,
               double coef[6]) {
    const int ex[6] = {0, 1, 2, 0, 1, 0}, ey[6] = {0, 0, 0, 1, 1, 2};
    double M[6][7] = {};
    for (size_t k = 0; k < v.size(); ++k) {
        double m[6];
        for (int t = 0; t < 6; ++t) m[t] = std::pow(xs[k], ex[t]) * std::pow(ys[k], ey[t]);
        for (int i = 0; i < 6; ++i) {
            for (int j = 0; j < 6; ++j) M[i][j] += m[i] * m[j];
            M[i][6] += m[i] * v[k];
        }
    }
    for (int c = 0; c < 6; ++c) {
        int piv = c;
        for (int r = c + 1; r < 6; ++r)
            if (std::fabs(M[r][c]) > std::fabs(M[piv][c])) piv = r;
        if (M[piv][c] == 0) return false;
        if (piv != c)
            for (int j = 0; j < 7; ++j) std::swap(M[c][j], M[piv][j]);
        for (int r = c + 1; r < 6; ++r) {
            const double f = M[r][c] / M[c][c];
            for (int j = c; j < 7; ++j) M[r][j] -= f * M[c][j];
        }
    }
    for (int i = 5; i >= 0; --i) {
        double s = M[i][6];
        for (int j = i + 1; j < 6; ++j) s -= M[i][j] * coef[j];
        coef[i] = s / M[i][i];
    }
    return true;
}

}  // namespace

extern "C" {

int zola_calib_init(zola_ctx* ctx, const float* raw, int nslice, int W, int H, float* xpoints, float* ypoints,
                    int nbead, int size_patch, double adu, double gain, double offset, double zstep, double* photons,
                    double* background, double* patches, double* poly_background) {
    if (!ctx) return ZOLA_E_ARG;
    if (!raw || !xpoints || !ypoints || !photons || !background || !patches || nslice < 1 || W < 1 || H < 1 ||
        nbead < 1 || size_patch < 4 || !(gain != 0) || !(zstep > 0)) {
        ctx->err = "zola_calib_init: null buffer or bad size (slices, W, H, beads >= 1, patch >= 4, gain != 0, zstep > 0)";
        return ZOLA_E_ARG;
    }
    cudaSetDevice(ctx->device);
    const int plane = W * H, sp = size_patch;
    const size_t N = (size_t)nslice * plane;
    const double slope = adu / gain, intercept = -offset * adu / gain;
    const int sizeFilt = std::max((int)(0.5 / zstep) / 2, 1);
    DevBuf<float> d_raw;
    DevBuf<double> d_im, d_s, d_c, d_psum;
    DevBuf<unsigned char> d_is2;
    DevBuf<int> d_pc;
    ZOLA_CUDA_CHECK(d_raw.alloc(N), ctx);
    ZOLA_CUDA_CHECK(d_im.alloc(N), ctx);
    ZOLA_CUDA_CHECK(d_s.alloc(nslice), ctx);
    ZOLA_CUDA_CHECK(d_c.alloc(nslice), ctx);
    ZOLA_CUDA_CHECK(d_is2.alloc(N), ctx);
    ZOLA_CUDA_CHECK(d_psum.alloc(plane), ctx);
    ZOLA_CUDA_CHECK(d_pc.alloc(plane), ctx);
    cudaStream_t st = ctx->stream;
    ZOLA_CUDA_CHECK(cudaMemcpyAsync(d_raw.p, raw, N * sizeof(float), cudaMemcpyHostToDevice, st), ctx);
    std::vector<double> hs(nslice), hc(nslice);
    auto fetch = [&](bool counts) -> int {
        ZOLA_CUDA_CHECK(cudaMemcpyAsync(hs.data(), d_s.p, nslice * 8, cudaMemcpyDeviceToHost, st), ctx);
        if (counts) ZOLA_CUDA_CHECK(cudaMemcpyAsync(hc.data(), d_c.p, nslice * 8, cudaMemcpyDeviceToHost, st), ctx);
        ZOLA_CUDA_CHECK(cudaStreamSynchronize(st), ctx);
        return ZOLA_OK;
    };
    k_ci_convert<<<nslice, CI_THREADS, 0, st>>>(d_raw.p, plane, slope, intercept, d_im.p, d_s.p);
    ctx->launches++;
    ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
    if (fetch(false)) return ZOLA_E_CUDA;
    double mean0 = 0;
    for (int z = 0; z < nslice; ++z) mean0 += hs[z];
    mean0 /= (double)N;
    k_ci_stats<<<nslice, CI_THREADS, 0, st>>>(d_im.p, plane, 0, mean0, 0, d_s.p, d_c.p, nullptr);
    if (fetch(false)) return ZOLA_E_CUDA;
    double std0 = 0;
    for (int z = 0; z < nslice; ++z) std0 += hs[z];
    std0 = std::sqrt(std0 / (double)N);
    k_ci_stats<<<nslice, CI_THREADS, 0, st>>>(d_im.p, plane, 1, 0, mean0 + 2 * std0, d_s.p, d_c.p, nullptr);
    if (fetch(true)) return ZOLA_E_CUDA;
    double mean = 0, cnt0 = 0;
    for (int z = 0; z < nslice; ++z) { mean += hs[z]; cnt0 += hc[z]; }
    if (cnt0 > 0) mean /= cnt0;
    k_ci_stats<<<nslice, CI_THREADS, 0, st>>>(d_im.p, plane, 2, mean, mean0 + 3 * std0, d_s.p, d_c.p, nullptr);
    if (fetch(false)) return ZOLA_E_CUDA;
    double sd = 0;
    for (int z = 0; z < nslice; ++z) sd += hs[z];
    if (cnt0 > 0) sd = std::sqrt(sd / cnt0);  // the reference divides by the 2-sigma count
    k_ci_stats<<<nslice, CI_THREADS, 0, st>>>(d_im.p, plane, 3, 0, mean + 3 * sd, d_s.p, d_c.p, d_is2.p);
    ctx->launches += 4;
    if (fetch(true)) return ZOLA_E_CUDA;
    std::vector<double> mstack(nslice), filt(nslice, 0.0);
    for (int z = 0; z < nslice; ++z) mstack[z] = hc[z] != 0 ? hs[z] / hc[z] : 0.0;
    int mp = 0;
    for (int z = 0; z < nslice; ++z) {
        int c = 0;
        for (int u = -sizeFilt; u <= sizeFilt; ++u)
            if (z + u >= 0 && z + u < nslice) { filt[z] += mstack[z + u]; c++; }
        if (c != 0) filt[z] /= c;
        if (filt[z] < filt[mp]) mp = z;
    }
    if (mp < sizeFilt) mp = sizeFilt;
    if (mp >= nslice - sizeFilt) mp = nslice - sizeFilt - 1;
    k_ci_dilate<<<(plane + 255) / 256, 256, 0, st>>>(d_im.p, d_is2.p, nslice, W, H, std::max(mp - sizeFilt, 0),
                                                     std::min(mp + sizeFilt, nslice - 1), d_psum.p, d_pc.p);
    ctx->launches++;
    ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
    std::vector<double> im(N), psum(plane);
    std::vector<int> pc(plane);
    ZOLA_CUDA_CHECK(cudaMemcpyAsync(im.data(), d_im.p, N * 8, cudaMemcpyDeviceToHost, st), ctx);
    ZOLA_CUDA_CHECK(cudaMemcpyAsync(psum.data(), d_psum.p, plane * 8, cudaMemcpyDeviceToHost, st), ctx);
    ZOLA_CUDA_CHECK(cudaMemcpyAsync(pc.data(), d_pc.p, plane * 4, cudaMemcpyDeviceToHost, st), ctx);
    ZOLA_CUDA_CHECK(cudaStreamSynchronize(st), ctx);
    auto at = [&](int z, int i, int ii) { return im[((size_t)z * W + i) * H + ii]; };
    // seed refinement (uses the photon image, before the background)
    for (int p = 0; p < nbead; ++p) {
        const int x0 = (int)(xpoints[p]) - sp / 2, y0 = (int)(ypoints[p]) - sp / 2;
        std::vector<double> sub((size_t)sp * sp, 0.0);
        for (int z = 0; z < nslice; ++z)
            for (int u = 0; u < sp; ++u)
                for (int uu = 0; uu < sp; ++uu)
                    if (x0 + u >= 0 && x0 + u < W && y0 + uu >= 0 && y0 + uu < H) sub[u * sp + uu] += at(z, x0 + u, y0 + uu);
        std::vector<double> v(sub);
        std::sort(v.begin(), v.end());
        const double thr = v[(int)((v.size() - 1) * .9)];
        double mx = 0, my = 0, sum = 0;
        int count = 0;
        for (int u = sp / 4; u < 3 * sp / 4; ++u)
            for (int uu = sp / 4; uu < 3 * sp / 4; ++uu)
                if (sub[u * sp + uu] > thr) {
                    mx += (x0 + u) * sub[u * sp + uu];
                    my += (y0 + uu) * sub[u * sp + uu];
                    sum += sub[u * sp + uu];
                    count++;
                }
        if (count >= 1) {
            const float fx = (float)(mx / sum), fy = (float)(my / sum);
            const float dxf = xpoints[p] - fx, dyf = ypoints[p] - fy;
            if (std::sqrt((double)(dxf * dxf)) < sp / 4) xpoints[p] = fx;
            if (std::sqrt((double)(dyf * dyf)) < sp / 4) ypoints[p] = fy;
        }
    }
    // polynomial background surface
    std::vector<double> px, py, pv;
    for (int k = 0; k < plane; ++k)
        if (pc[k] >= 1) {
            px.push_back(k / H);
            py.push_back(k % H);
            pv.push_back(psum[k] / pc[k]);
        }
    double cf[6];
    if (!poly2_fit(px, py, pv, cf)) {
        ctx->err = "zola_calib_init: singular background fit (too few low voxels)";
        return ZOLA_E_ARG;
    }
    std::vector<double> pb((size_t)plane);
    for (int i = 0; i < W; ++i)
        for (int ii = 0; ii < H; ++ii)
            pb[(size_t)i * H + ii] = cf[0] + cf[1] * i + cf[2] * std::pow((double)i, 2) + cf[3] * ii +
                                     cf[4] * i * (double)ii + cf[5] * std::pow((double)ii, 2);
    if (poly_background) std::memcpy(poly_background, pb.data(), pb.size() * 8);
    // per bead: B, filtered photon curve, patches
    for (int p = 0; p < nbead; ++p) {
        const int x0 = (int)(xpoints[p]) - sp / 2, y0 = (int)(ypoints[p]) - sp / 2;
        double b = 0, cb = 0;
        for (int u = 0; u < sp; ++u)
            for (int uu = 0; uu < sp; ++uu)
                if (x0 + u >= 0 && x0 + u < W && y0 + uu >= 0 && y0 + uu < H) { b += pb[(size_t)(x0 + u) * H + y0 + uu]; cb++; }
        if (cb >= 1) b /= cb;
        background[p] = b;
        std::vector<double> a(nslice, 0.0);
        for (int z = 0; z < nslice; ++z)
            for (int u = 0; u < sp; ++u)
                for (int uu = 0; uu < sp; ++uu)
                    if (x0 + u >= 0 && x0 + u < W && y0 + uu >= 0 && y0 + uu < H) a[z] += at(z, x0 + u, y0 + uu) - b;
        for (int z = 0; z < nslice; ++z) {
            double m = 0, c = 0;
            for (int f = -sizeFilt; f <= sizeFilt; ++f)
                if (z + f >= 0 && z + f < nslice) { m += a[z + f]; c++; }
            if (c >= 1) m /= c;
            photons[(size_t)p * nslice + z] = m;
        }
        for (int z = 0; z < nslice; ++z)
            for (int u = 0; u < sp; ++u)
                for (int uu = 0; uu < sp; ++uu)
                    patches[(((size_t)p * nslice + z) * sp + u) * sp + uu] =
                        (x0 + u >= 0 && x0 + u < W && y0 + uu >= 0 && y0 + uu < H) ? at(z, x0 + u, y0 + uu) : b;
    }
    return ZOLA_OK;
}

}  // extern "C"
