// CRLB curves and the z-centre search.
//
// zola_crlb_curve: the finite-difference Fisher matrix of an emitter at
// (0, 0, z) for a list of depths (process/cpu/CRLB.java:255-340,
// SearchPSFcenter.java:210-330): the seven FP64 models of each depth
// [f, x+h, x-h, y+h, y-h, z+h, z-h] come from one batched model launch, one
// CTA per depth reduces the 15 distinct Fisher entries over the R x R pixels,
// and the host inverts the 5 x 5 matrices.  As in the reference, the A and B
// rows perturb the already formed mean f1 = photons psi + bg, so
// dmu/dA = f1 a_step / h and dmu/dB = 1.
//
// zola_psf_center_search: SearchPSFcenter.getPosition
// (process/cpu/SearchPSFcenter.java:37-203; variant 1 follows
// process/gpu/SearchPSFcenter_.java).  A coarse scan of the lateral CRLB
// sqrt(crlb_x^2 + crlb_y^2) over depth, up to ten refinements that halve the
// step around the minimum, then the axial window of width axialRange / 2
// (sampled at the pixel size) whose summed lateral CRLB is smallest.  The
// loops keep the reference's floating-point accumulation (u += step), so the
// depths evaluated are the reference's own; every pass is one batched call.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <vector>

#include "zola_internal.h"

namespace zola {

constexpr int CF_THREADS = 256;

__global__ void __launch_bounds__(CF_THREADS) k_center_fisher(const double* psi, int RR, double photons, double bg,
                                                              double h, double ha, double* F15) {
    const double* f = psi + (size_t)blockIdx.x * 7 * RR;
    const double den = 2 * fabs(h);
    double acc[15];
#pragma unroll
    for (int o = 0; o < 15; ++o) acc[o] = 0.0;
    for (int k = threadIdx.x; k < RR; k += CF_THREADS) {
        const double f1 = f[k] * photons + bg;
        double d[5];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const double f2 = f[(size_t)(1 + 2 * q) * RR + k] * photons + bg;
            const double f0 = f[(size_t)(2 + 2 * q) * RR + k] * photons + bg;
            d[q] = (f2 - f0) / den;
        }
        d[3] = ((f1 * (photons + ha) + bg) - (f1 * (photons - ha) + bg)) / den;
        d[4] = ((f1 * photons + (bg + h)) - (f1 * photons + (bg - h))) / den;
        const double w = 1 / f1;
        int o = 0;
#pragma unroll
        for (int a = 0; a < 5; ++a)
#pragma unroll
            for (int b = a; b < 5; ++b) acc[o++] += w * d[a] * d[b];
    }
    __shared__ double red[CF_THREADS / 32][15];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 0; o < 15; ++o) {
        double v = acc[o];
        for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
        if (lane == 0) red[warp][o] = v;
    }
    __syncthreads();
    if (threadIdx.x < 15) {
        double v = 0.0;
        for (int w = 0; w < CF_THREADS / 32; ++w) v += red[w][threadIdx.x];
        F15[(size_t)blockIdx.x * 15 + threadIdx.x] = v;
    }
}

namespace {

// sqrt(diag(F^-1)) by Gauss-Jordan elimination with partial pivoting; a
// singular F gives sqrt(1 / F_ii) (DBL_MAX where F_ii = 0), the reference's
// fallback.
void crlb_from_fisher(const double* F15, double* crlb5) {
    double F[5][5], M[5][10];
    int o = 0;
    for (int a = 0; a < 5; ++a)
        for (int b = a; b < 5; ++b) { F[a][b] = F[b][a] = F15[o]; ++o; }
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 10; ++j) M[i][j] = j < 5 ? F[i][j] : (j - 5 == i ? 1.0 : 0.0);
    bool ok = true;
    for (int c = 0; c < 5 && ok; ++c) {
        int piv = c;
        for (int r = c + 1; r < 5; ++r)
            if (std::fabs(M[r][c]) > std::fabs(M[piv][c])) piv = r;
        if (M[piv][c] == 0.0) { ok = false; break; }
        if (piv != c)
            for (int j = 0; j < 10; ++j) std::swap(M[c][j], M[piv][j]);
        const double dv = M[c][c];
        for (int j = 0; j < 10; ++j) M[c][j] /= dv;
        for (int r = 0; r < 5; ++r) {
            if (r == c) continue;
            const double fct = M[r][c];
            for (int j = 0; j < 10; ++j) M[r][j] -= fct * M[c][j];
        }
    }
    for (int i = 0; i < 5; ++i) {
        if (ok) crlb5[i] = std::sqrt(M[i][5 + i]);
        else crlb5[i] = F[i][i] != 0.0 ? std::sqrt(1 / F[i][i]) : DBL_MAX;
    }
}

struct CrlbScan {
    zola_ctx* ctx;
    zola_psf* psf;
    int R;
    double photons, bg, h, ha;
    cudaStream_t st;

    // crlb5 (n x 5) of an emitter at (0, 0, z[i])
    int run(const std::vector<double>& z, std::vector<double>& crlb5) {
        const int n = (int)z.size();
        crlb5.assign((size_t)5 * n, 0.0);
        if (n == 0) return ZOLA_OK;
        const size_t RR = (size_t)R * R;
        std::vector<double> xyz((size_t)21 * n, 0.0);
        for (int i = 0; i < n; ++i) {
            double* q = &xyz[(size_t)21 * i];
            q[2] = z[i];
            q[3] = 0 + h; q[5] = z[i];
            q[6] = 0 - h; q[8] = z[i];
            q[10] = 0 + h; q[11] = z[i];
            q[13] = 0 - h; q[14] = z[i];
            q[17] = z[i] + h;
            q[20] = z[i] - h;
        }
        DevBuf<double> d_xyz, d_psi, d_F;
        ZOLA_CUDA_CHECK(d_xyz.alloc(xyz.size()), ctx);
        ZOLA_CUDA_CHECK(d_psi.alloc(7 * RR * n), ctx);
        ZOLA_CUDA_CHECK(d_F.alloc((size_t)15 * n), ctx);
        ZOLA_CUDA_CHECK(cudaMemcpyAsync(d_xyz.p, xyz.data(), xyz.size() * sizeof(double), cudaMemcpyHostToDevice, st),
                        ctx);
        WindowTables* w = get_window(psf, R, ctx->err);
        if (!w) return ZOLA_E_ARG;
        int rc = launch_model_f64(ctx, psf, w, d_xyz.p, 7 * n, d_psi.p, nullptr, st);
        if (rc) return rc;
        k_center_fisher<<<n, CF_THREADS, 0, st>>>(d_psi.p, (int)RR, photons, bg, h, ha, d_F.p);
        ctx->launches++;
        ZOLA_CUDA_CHECK(cudaGetLastError(), ctx);
        std::vector<double> F((size_t)15 * n);
        ZOLA_CUDA_CHECK(cudaMemcpyAsync(F.data(), d_F.p, F.size() * sizeof(double), cudaMemcpyDeviceToHost, st), ctx);
        ZOLA_CUDA_CHECK(cudaStreamSynchronize(st), ctx);
        for (int i = 0; i < n; ++i) crlb_from_fisher(&F[(size_t)15 * i], &crlb5[(size_t)5 * i]);
        return ZOLA_OK;
    }

    // lateral CRLB sqrt(crlb_x^2 + crlb_y^2) at each depth
    int lateral(const std::vector<double>& z, std::vector<double>& out) {
        std::vector<double> c;
        int rc = run(z, c);
        if (rc) return rc;
        out.resize(z.size());
        for (size_t i = 0; i < z.size(); ++i) out[i] = std::sqrt(c[5 * i] * c[5 * i] + c[5 * i + 1] * c[5 * i + 1]);
        return ZOLA_OK;
    }
};

// getMinPositionCRLB (SearchPSFcenter.java:173-203)
int min_position(CrlbScan& cs, double minZ, double maxZ, double stepZ, double* pos) {
    std::vector<double> zs, c;
    for (double u = minZ; u < maxZ; u += stepZ) zs.push_back(u);
    int rc = cs.lateral(zs, c);
    if (rc) return rc;
    double best = INFINITY, p = 0;
    for (size_t i = 0; i < zs.size(); ++i)
        if (best > c[i]) { best = c[i]; p = zs[i]; }
    *pos = p;
    return ZOLA_OK;
}

// getMinRangeCRLB (SearchPSFcenter.java:88-170)
int min_range(CrlbScan& cs, double minZ, double maxZ, double stepZ, double axialRange, double* pos) {
    const double ar = axialRange / 2;
    std::vector<double> zs, crlb;
    for (double u = minZ - ar / 2; u <= maxZ + ar / 2; u += stepZ) zs.push_back(u);
    int rc = cs.lateral(zs, crlb);
    if (rc) return rc;
    double best = INFINITY, p = 0;
    int nb = (int)(ar / (2 * stepZ));
    for (double u = minZ; u < maxZ; u += stepZ) {
        double s = 0;
        int nb2 = -(int)(ar / (2 * stepZ));
        for (double i = -ar / 2; i <= ar / 2; i += stepZ) {
            const int k = nb + nb2;
            if (k < 0 || k >= (int)crlb.size()) {
                cs.ctx->err = "zola_psf_center_search: the axial window runs past the sampled depths";
                return ZOLA_E_ARG;
            }
            s += crlb[k];
            nb2++;
        }
        if (best > s) { best = s; p = u; }
        nb++;
    }
    *pos = p;
    return ZOLA_OK;
}

bool check_scan_args(zola_ctx* ctx, zola_psf* psf, int R) {
    if (R < 4 || R % 2 || R > psf->N) {
        ctx->err = "model side must be even, >= 4 and <= the pupil grid";
        return false;
    }
    return true;
}

}  // namespace
}  // namespace zola

using namespace zola;

extern "C" {

int zola_crlb_curve(zola_psf* psf, int R, const double* z, int n, double photons, double background, double h,
                    double a_step, double* crlb5) {
    if (!psf) return ZOLA_E_ARG;
    zola_ctx* ctx = psf->ctx;
    if (n < 0 || (n > 0 && (!z || !crlb5))) { ctx->err = "zola_crlb_curve: bad n or null buffer"; return ZOLA_E_ARG; }
    if (!(h != 0) || !(photons > 0) || !(background >= 0)) {
        ctx->err = "zola_crlb_curve: need h != 0, photons > 0, background >= 0";
        return ZOLA_E_ARG;
    }
    if (!check_scan_args(ctx, psf, R)) return ZOLA_E_ARG;
    cudaSetDevice(ctx->device);
    CrlbScan cs{ctx, psf, R, photons, background, h, a_step, ctx->stream};
    std::vector<double> zs(z, z + n), out;
    int rc = cs.run(zs, out);
    if (rc) return rc;
    for (size_t i = 0; i < out.size(); ++i) crlb5[i] = out[i];
    return ZOLA_OK;
}

int zola_psf_center_search(zola_psf* psf, int R, double axial_range, int variant, double* z_center) {
    if (!psf) return ZOLA_E_ARG;
    zola_ctx* ctx = psf->ctx;
    if (!z_center || (variant != ZOLA_CENTER_CPU && variant != ZOLA_CENTER_GPU)) {
        ctx->err = "zola_psf_center_search: null output or unknown variant";
        return ZOLA_E_ARG;
    }
    if (!check_scan_args(ctx, psf, R)) return ZOLA_E_ARG;
    const double zfocus = psf->o.zfocus;
    *z_center = zfocus;
    if (axial_range <= 0) return ZOLA_OK;  // the reference logs and keeps Zfocus
    if (variant == ZOLA_CENTER_GPU && psf->o.n_oil == psf->o.n_wat) return ZOLA_OK;
    cudaSetDevice(ctx->device);
    const double h = variant == ZOLA_CENTER_GPU ? .0005 : .005;
    const double ha = variant == ZOLA_CENTER_GPU ? h : h * 100;
    CrlbScan cs{ctx, psf, R, 3000.0, 50.0, h, ha, ctx->stream};
    double stepZ = psf->o.xystep * 5;
    double minZ = zfocus - 2 * axial_range - std::fabs(zfocus);
    double maxZ = zfocus + std::fabs(zfocus) + 2 * axial_range;
    double position;
    int rc = min_position(cs, minZ, maxZ, stepZ, &position);
    if (rc) return rc;
    double old = INFINITY;
    for (int i = 0; i < 10; i++) {
        minZ = position - stepZ * 5;
        maxZ = position + stepZ * 5;
        stepZ = stepZ / 2;
        rc = min_position(cs, minZ, maxZ, stepZ, &position);
        if (rc) return rc;
        if (std::fabs(old - position) < 0.00001) break;
        old = position;
    }
    rc = min_range(cs, position - axial_range * 2, position + axial_range * 2, psf->o.xystep, axial_range, &position);
    if (rc) return rc;
    *z_center = position;
    return ZOLA_OK;
}

}  // extern "C"
