// Host-side optics set-up: pupil-disk geometry, Zernike phase, k-tables, the
// partial-DFT twiddles and the circular blur matrix.  Everything here runs once
// per calibration (or per ROI size) in FP64 and is uploaded to the device.
//
// Reference (paths relative to src/main/java/org/pasteur/imagej/):
//   grid, disk test, centre N/2-0.5     process/PhaseParameters.java:265-366
//   Zernike order and radial formula    utils/Zernike.java:26-79, 540-608
//   phase = sum a_i Z_i on the disk     process/cpu/ZernikePhase.java:200-224
//   kx, ky, kz, kz_oil, pupil           process/cpu/PSFPhase.java:140-220
//   resetKz (evanescent kz = 2pi sqrt|.|)  process/cpu/PSFPhase.java:417-464
//   W window and spectral Gaussian      process/cpu/PSFPhase.java:100-108, 361-378
#include <cmath>
#include <cstring>

#include "zola_internal.h"

namespace zola {

static int pow2ceil(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

int window_size(int R, int N) {
    int w = 2 * R;
    if (w > N) w = N;
    return pow2ceil(w);
}

static double fact(int n) {
    double f = 1.0;
    for (int i = 2; i <= n; ++i) f *= i;
    return f;
}

// Un-normalised Zernike radial polynomial times cos/sin(|m| theta).
static double zernike(int n, int m, double theta, double rho) {
    int am = m < 0 ? -m : m;
    double s = 0.0;
    for (int k = 0; k <= (n - am) / 2; ++k) {
        double num = ((k & 1) ? -1.0 : 1.0) * fact(n - k);
        double den = fact(k) * fact((n + am) / 2 - k) * fact((n - am) / 2 - k);
        s += (num / den) * std::pow(rho, n - 2 * k);
    }
    return m >= 0 ? s * std::cos(theta * am) : s * std::sin(theta * am);
}

int build_psf_tables(zola_psf* p, const zola_optics* o, const double* zern, int nz, std::string& err) {
    if (o->size_fft <= 1 || !(o->xystep > 0) || !(o->na > 0) || !(o->wavelength > 0) || !(o->n_oil > 0) ||
        !(o->n_wat > 0) || !(o->sigma > 0) || nz < 0 || (nz > 0 && !zern)) {
        err = "zola_psf_load: invalid optics (size_fft>1, positive xystep/na/wavelength/indices/sigma required)";
        return ZOLA_E_ARG;
    }
    int N = o->size_fft;
    if (N % 2) N--;
    N = pow2ceil(N);
    if (N > 1024) {
        err = "zola_psf_load: size_fft above 1024 is not supported";
        return ZOLA_E_ARG;
    }
    const double dx = o->xystep;
    const double ring = (o->na / o->wavelength) * (o->na / o->wavelength);
    const double c = (double)(N / 2) - 0.5;
    const double radius = std::sqrt(ring) * (N * dx);
    const double left = (o->n_wat / o->wavelength) * (o->n_wat / o->wavelength);
    const double left_oil = (o->n_oil / o->wavelength) * (o->n_oil / o->wavelength);

    int lo = N, hi = -1, K = 0;
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            double a = (i - c) / (N * dx), b = (j - c) / (N * dx);
            if (a * a + b * b <= ring) {
                lo = std::min(lo, i);
                hi = std::max(hi, i);
                ++K;
            }
        }
    if (K == 0) {
        err = "zola_psf_load: empty pupil disk (NA/wavelength too small for this grid)";
        return ZOLA_E_ARG;
    }
    const int D = hi - lo + 1, a0 = lo;
    p->N = N; p->K = K; p->D = D; p->a0 = a0;
    p->o = *o;
    p->zern.assign(zern, zern + nz);
    size_t DD = (size_t)D * D;
    p->pupil.assign(DD, 0.0); p->phase.assign(DD, 0.0); p->kz.assign(DD, 0.0); p->kzoil.assign(DD, 0.0);
    p->isim.assign(DD, 0.0); p->isimoil.assign(DD, 0.0); p->kx.assign(D, 0.0); p->ky.assign(D, 0.0);

    std::vector<int> zn(nz), zm(nz);
    for (int idx = 0, n = 0; idx < nz; ++n)
        for (int m = -n; m <= n && idx < nz; m += 2, ++idx) { zn[idx] = n; zm[idx] = m; }

    for (int a = 0; a < D; ++a) {
        p->kx[a] = ((a0 + a) - c) * (2 * M_PI) / (dx * N);
        p->ky[a] = ((a0 + a) - c) * (2 * M_PI) / (dx * N);
    }
    for (int a = 0; a < D; ++a)
        for (int b = 0; b < D; ++b) {
            int i = a0 + a, j = a0 + b;
            double u = (i - c) / (N * dx), v = (j - c) / (N * dx);
            double right = u * u + v * v;
            if (!(right <= ring)) continue;
            size_t k = (size_t)a * D + b;
            if (left > right) { p->kz[k] = 2 * M_PI * std::sqrt(left - right); p->isim[k] = 1; }
            else { p->kz[k] = o->kz_reset ? 2 * M_PI * std::sqrt(std::fabs(left - right)) : 0.0; p->isim[k] = 0; }
            if (left_oil > right) { p->kzoil[k] = 2 * M_PI * std::sqrt(left_oil - right); p->isimoil[k] = 1; }
            else { p->kzoil[k] = 0.0; p->isimoil[k] = 0; }
            double x = (i - c) / radius, y = (j - c) / radius;
            double rho = std::sqrt(x * x + y * y), th = std::atan2(y, x);
            double ph = 0.0;
            for (int z = 0; z < nz; ++z) ph += (rho < 1 ? zernike(zn[z], zm[z], th, rho) : 0.0) * zern[z];
            p->phase[k] = ph;
            if (o->with_apo) {
                p->pupil[k] = left_oil > right ? (double)(float)(1.0 / std::pow(1 - right / left_oil, .25)) : 0.0;
            } else {
                p->pupil[k] = 1.0 / std::sqrt((double)K);
            }
        }
    // upload: 6 D*D arrays + 2 D arrays
    size_t total = 6 * DD + 2 * (size_t)D;
    std::vector<double> h(total);
    double* w = h.data();
    auto put = [&](const std::vector<double>& v) { std::memcpy(w, v.data(), v.size() * sizeof(double)); w += v.size(); };
    put(p->pupil); put(p->phase); put(p->kz); put(p->kzoil); put(p->isim); put(p->isimoil); put(p->kx); put(p->ky);
    cudaError_t e = cudaMalloc(&p->d_tables, total * sizeof(double));
    if (e != cudaSuccess) { err = std::string("cudaMalloc: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
    e = cudaMemcpy(p->d_tables, h.data(), total * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { err = std::string("cudaMemcpy: ") + cudaGetErrorString(e); return ZOLA_E_CUDA; }
    PsfView& pv = p->view;
    pv.N = N; pv.D = D; pv.a0 = a0; pv.dx = dx; pv.zfocus = o->zfocus;
    pv.pupil = p->d_tables; pv.phase = pv.pupil + DD; pv.kz = pv.phase + DD; pv.kzoil = pv.kz + DD;
    pv.isim = pv.kzoil + DD; pv.isimoil = pv.isim + DD; pv.kx = pv.isimoil + DD; pv.ky = pv.kx + D;
    return ZOLA_OK;
}

// Partial-DFT twiddles and blur matrix for ROI side R.
//
// The reference computes E = IFFT_N(pupil field) and crops a W x W window
// centred on N/2 (PSFPhase.java:580-590).  Only the D disk rows / columns of the
// pupil are non-zero, so the window is E = C Q C^T with the W x D matrix
// C[w][a] = exp(+2 pi i ((a0+a+N/2)(w-W/2) mod N)/N); the constant 1/N scale
// is dropped because the PSF is normalised to sum 1 at the end.
//
// The blur is IFFT_W(FFT_W(I) g) with g(f) = exp(-f^2/(2 s^2)),
// s = W/(2 pi sigma), f the signed frequency (PSFPhase.java:361-378, 597-606):
// a circular convolution with the real even kernel
//   h(d) = (1/W) sum_f g(f) cos(2 pi f d / W),
// which is separable.  The final R x R crop reads window rows (i'-R/2) mod W,
// so G[i'][i] = h(((i'-R/2) - (i-W/2)) mod W) and blurred = G I G^T.
// R x W blur-and-crop matrix of the window: row ip is the circulant kernel
// h(d) = (1/W) sum_f g(f) cos(2 pi f d / W) of the spectral Gaussian
// g(f) = exp(-f^2 / (2 s^2)), s = W / (2 pi sigma), shifted so that output
// pixel ip sits at window pixel ip - R/2 + W/2.  With dG, also d G / d sigma
// (dg/dsigma = -g f^2 / (s^2 sigma)).
void blur_matrix(int R, int W, double sigma, std::vector<double>& G, std::vector<double>* dG) {
    std::vector<double> h(W), dh(W);
    const double s = W / (2 * M_PI * sigma);
    for (int d = 0; d < W; ++d) {
        double acc = 0.0, dacc = 0.0;
        for (int f = 0; f < W; ++f) {
            int fs = f < W / 2 ? f : f - W;
            double g = std::exp(-0.5 * (double)fs * fs / (s * s));
            long long m = ((long long)f * d) % W;
            const double cs = std::cos(2 * M_PI * (double)m / W);
            acc += g * cs;
            dacc += -g * (double)fs * fs / (s * s * sigma) * cs;
        }
        h[d] = acc / W;
        dh[d] = dacc / W;
    }
    G.resize((size_t)R * W);
    if (dG) dG->resize((size_t)R * W);
    for (int ip = 0; ip < R; ++ip)
        for (int i = 0; i < W; ++i) {
            int d = ((ip - R / 2) - (i - W / 2)) % W;
            if (d < 0) d += W;
            G[(size_t)ip * W + i] = h[d];
            if (dG) (*dG)[(size_t)ip * W + i] = dh[d];
        }
}

WindowTables* get_window(zola_psf* p, int R, std::string& err) {
    auto it = p->win.find(R);
    if (it != p->win.end()) return &it->second;
    if (R < 4 || R % 2 || R > p->N) {
        err = "ROI side must be even, >= 4 and <= the pupil grid";
        return nullptr;
    }
    WindowTables t;
    const int N = p->N, D = p->D, a0 = p->a0;
    const int W = window_size(R, N);
    t.R = R; t.W = W;
    t.C.resize((size_t)W * D * 2);
    for (int w = 0; w < W; ++w)
        for (int a = 0; a < D; ++a) {
            long long m = (long long)(a0 + a + N / 2) * (long long)(w - W / 2);
            m %= N;
            if (m < 0) m += N;
            double ang = 2.0 * M_PI * (double)m / (double)N;
            t.C[((size_t)w * D + a) * 2] = std::cos(ang);
            t.C[((size_t)w * D + a) * 2 + 1] = std::sin(ang);
        }
    blur_matrix(R, W, p->o.sigma, t.G, nullptr);
    cudaError_t e = cudaMalloc(&t.d_C, t.C.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(t.d_C, t.C.data(), t.C.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&t.d_G, t.G.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(t.d_G, t.G.data(), t.G.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        err = std::string("window tables: ") + cudaGetErrorString(e);
        return nullptr;
    }
    auto res = p->win.emplace(R, t);
    return &res.first->second;
}

}  // namespace zola
