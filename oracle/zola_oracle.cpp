// ORACLE — test infrastructure only.
//
// FP64 CPU restatement of ZOLA-3D's localization hot path, written from the
// reference's Java sources (paths relative to src/main/java/org/pasteur/imagej/).
// It is the checker for the CUDA library: only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline leg may load it.  The product never links it.
//
// PARITY UNPINNED: the reference ships no tests, golden vectors or fixtures for
// this path, and it is a Java/ImageJ plugin that cannot be built or run in this
// environment (no JVM).  This restatement is therefore pinned only by
// known-answer tests derived from the mathematics (FFT round trip, Zernike
// orthogonality, symmetric in-focus PSF, translation equivariance).
//
// What is restated, function by function:
//   geometry          process/PhaseParameters.java:265-366
//   Zernike basis     utils/Zernike.java:26-79, 540-608, 818-836
//   phase combination process/cpu/ZernikePhase.java:200-224
//   pupil tables      process/cpu/PSFPhase.java:96-269 (constructor),
//                     :417-464 (resetKz)
//   PSF model         process/cpu/PSFPhase.java:361-378 (Gaussian), :557-629
//   unitary FFT       utils/FastFourierTransform.java:628-796 (convention only:
//                     every 1-D pass divided by sqrt(n), forward exponent -i)
//   likelihood        process/cpu/Localization.java:1125-1143
//   coordinate descent process/cpu/Localization.java:491-1058
//   Fisher / CRLB     process/cpu/Localization.java:317-451
//   z-centre search   process/cpu/SearchPSFcenter.java:37-330 (and the GPU
//                     form process/gpu/SearchPSFcenter_.java)
//   detection         process/cpu/Predetection.java:63-593
//   calibration NLL   process/cpu/ZernikePhaseRetrieval.java:1519-1530, 1843-1874
//   calibration init  process/InitBackgroundAndPhotonNumber.java (+ utils/PolynomialFit.java)
//   drift correction  process/cpu/DriftCorrection.java, utils/SplineFit.java,
//                     utils/GaussianElimination.java
// plus the FP64 Levenberg-Marquardt fit of the same Poisson NLL with analytic
// x/y/z derivatives (no reference counterpart: the "FP64 oracle of the same
// fit" that the GPU fits are compared against).

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <thread>
#include <atomic>
#include <array>
#include <functional>

namespace {

typedef std::complex<double> cplx;

int pow2ceil(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

// ---------------------------------------------------------------- FFT ------
// Radix-2 in-place complex FFT with exact twiddles, unitary scaling per pass.
// sign = -1 forward, +1 inverse (FastFourierTransform.java:700-790 convention).
void fft1d(cplx* a, int n, int sign) {
    for (int i = 1, j = 0; i < n; ++i) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1;
        for (int k = 0; k < half; ++k) {
            double ang = sign * 2.0 * M_PI * (double)k / (double)len;
            cplx w(std::cos(ang), std::sin(ang));
            for (int i = 0; i < n; i += len) {
                cplx u = a[i + k];
                cplx v = a[i + k + half] * w;
                a[i + k] = u + v;
                a[i + k + half] = u - v;
            }
        }
    }
    double s = 1.0 / std::sqrt((double)n);
    for (int i = 0; i < n; ++i) a[i] *= s;
}

// 2-D unitary FFT over a row-major n x n array.
void fft2d(std::vector<cplx>& a, int n, int sign) {
    std::vector<cplx> col(n);
    for (int i = 0; i < n; ++i) fft1d(&a[(size_t)i * n], n, sign);
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < n; ++i) col[i] = a[(size_t)i * n + j];
        fft1d(col.data(), n, sign);
        for (int i = 0; i < n; ++i) a[(size_t)i * n + j] = col[i];
    }
}

// ------------------------------------------------------------- Zernike -----
double factorial(int n) {  // Zernike.java:818-836 (long table to 19, then double)
    double f = 1.0;
    for (int i = 2; i <= n; ++i) f *= i;
    return f;
}

// Un-normalised Zernike polynomial, Zernike.java:574-608.
double zernike_value(int n, int m, double theta, double rho) {
    int am = m < 0 ? -m : m;
    double som = 0.0;
    for (int k = 0; k <= (n - am) / 2; ++k) {
        double truc = ((k & 1) ? -1.0 : 1.0) * factorial(n - k);
        double trac = factorial(k) * factorial((n + am) / 2 - k) * factorial((n - am) / 2 - k);
        som += (truc / trac) * std::pow(rho, n - 2 * k);
    }
    return m >= 0 ? som * std::cos(theta * am) : som * std::sin(theta * am);
}

// Index order of Zernike.java:31-47: n = 0,1,2..., m = -n, -n+2, ..., n.
void zernike_nm(int idx, int* n_out, int* m_out) {
    int i = 0;
    for (int n = 0;; ++n)
        for (int m = -n; m <= n; m += 2) {
            if (i == idx) { *n_out = n; *m_out = m; return; }
            ++i;
        }
}

// ----------------------------------------------------------------- PSF -----
struct Psf {
    int N;                 // pupil grid (power of two, size_cpu)
    double dx, na, lambda, n_oil, n_wat, sigma, zfocus;
    int apo, kz_reset, gauss_f32;
    int K;                 // disk pixels
    std::vector<int> di, dj;
    std::vector<double> kx, ky, kz, kzoil, isim, isimoil, pupil, phase;
};

// PhaseParameters.java:300-362 + PSFPhase.java:140-220 (+ resetKz :417-464).
Psf* psf_build(int N_in, double dx, double na, double lambda, double n_oil, double n_wat,
               double sigma, int apo, double zfocus, int kz_reset, int gauss_f32,
               int nz, const double* zern) {
    Psf* p = new Psf();
    int N = N_in;
    if (N % 2) N--;
    N = pow2ceil(N);
    p->N = N; p->dx = dx; p->na = na; p->lambda = lambda; p->n_oil = n_oil; p->n_wat = n_wat;
    p->sigma = sigma; p->apo = apo; p->zfocus = zfocus; p->kz_reset = kz_reset; p->gauss_f32 = gauss_f32;
    double ringsize = (na / lambda) * (na / lambda);
    double c = (double)(N / 2) - 0.5;
    double radius = std::sqrt(ringsize) * (N * dx);
    double left = (n_wat / lambda) * (n_wat / lambda);
    double left_oil = (n_oil / lambda) * (n_oil / lambda);
    std::vector<double> zn(nz), zm(nz);
    for (int i = 0; i < N; ++i)
        for (int ii = 0; ii < N; ++ii) {
            double a = (i - c) / (N * dx), b = (ii - c) / (N * dx);
            double disk = a * a + b * b;
            if (!(disk <= ringsize)) continue;
            p->di.push_back(i); p->dj.push_back(ii);
            p->kx.push_back((i - c) * (2 * M_PI) / (dx * N));
            p->ky.push_back((ii - c) * (2 * M_PI) / (dx * N));
            double kxx = ((i - c) / (dx * N)) * ((i - c) / (dx * N));
            double kyy = ((ii - c) / (dx * N)) * ((ii - c) / (dx * N));
            double right = kxx + kyy;
            if (left > right) { p->kz.push_back(2 * M_PI * std::sqrt(left - right)); p->isim.push_back(1); }
            else { p->kz.push_back(kz_reset ? 2 * M_PI * std::sqrt(std::fabs(left - right)) : 0.0); p->isim.push_back(0); }
            if (left_oil > right) { p->kzoil.push_back(2 * M_PI * std::sqrt(left_oil - right)); p->isimoil.push_back(1); }
            else { p->kzoil.push_back(0.0); p->isimoil.push_back(0); }
            // phase: sum_i a_i Z_i, Zernike evaluated where rho < 1 (Zernike.java:553-560)
            double x = (i - c) / radius, y = (ii - c) / radius;
            double rho = std::sqrt(x * x + y * y), theta = std::atan2(y, x);
            double ph = 0.0;
            for (int z = 0; z < nz; ++z) {
                int n, m;
                zernike_nm(z, &n, &m);
                double v = rho < 1 ? zernike_value(n, m, theta, rho) : 0.0;
                ph += v * zern[z];
            }
            p->phase.push_back(ph);
        }
    p->K = (int)p->di.size();
    for (int k = 0; k < p->K; ++k) {
        if (apo) {
            double kxx = p->kx[k] / (2 * M_PI), kyy = p->ky[k] / (2 * M_PI);
            double right = kxx * kxx + kyy * kyy;
            p->pupil.push_back(left_oil > right ? (double)(float)(1.0 / std::pow(1 - right / left_oil, .25)) : 0.0);
        } else {
            p->pupil.push_back(1.0 / std::sqrt((double)p->K));
        }
    }
    return p;
}

int window_size(int R, int N) {  // PSFPhase.java:100-108
    int w = 2 * R;
    if (w > N) w = N;
    return pow2ceil(w);
}

// Separable spectral Gaussian g(f) for the W-grid blur, PSFPhase.java:361-378.
double gauss_value(const Psf* p, int W, int a, int b) {
    double sigF = (1.0 / p->sigma) * W / (M_PI * 2);
    double sigpow = sigF * sigF;
    double cc = W / 2;
    double v = std::exp(-.5 * ((a - cc) * (a - cc) + (b - cc) * (b - cc)) / sigpow);
    return p->gauss_f32 ? (double)(float)v : v;
}

// Pupil field with an optional per-pixel multiplier (used for derivatives).
// deriv: 0 none, 1 x, 2 y, 3 z (zwat).  For deriv != 0 the field is the
// derivative of the field with respect to that coordinate.
void pupil_field(const Psf* p, double x, double y, double zoil, double zwat, int deriv,
                 std::vector<cplx>& grid) {
    int N = p->N;
    grid.assign((size_t)N * N, cplx(0, 0));
    for (int k = 0; k < p->K; ++k) {
        double pp = p->kx[k] * x + p->ky[k] * y + p->phase[k];
        double q = pp + p->kz[k] * zwat - p->kzoil[k] * zoil;
        double r = pp + p->kz[k] * zwat * p->isim[k] - p->kzoil[k] * zoil * p->isimoil[k];
        cplx v;
        if (deriv == 0) v = cplx(p->pupil[k] * std::cos(q), p->pupil[k] * std::sin(r));
        else {
            double dq, dr;
            if (deriv == 1) { dq = p->kx[k]; dr = p->kx[k]; }
            else if (deriv == 2) { dq = p->ky[k]; dr = p->ky[k]; }
            else { dq = p->kz[k]; dr = p->kz[k] * p->isim[k]; }
            v = cplx(-p->pupil[k] * std::sin(q) * dq, p->pupil[k] * std::cos(r) * dr);
        }
        grid[(size_t)((p->di[k] + N / 2) % N) * N + (p->dj[k] + N / 2) % N] = v;
    }
}

// Blur of a real W x W intensity window laid out as in PSFPhase.computePSF
// (centre at W/2), returning the complex blurred window (unitary FFTs).
void blur_window(const Psf* p, int W, const std::vector<double>& I, std::vector<cplx>& out) {
    out.assign((size_t)W * W, cplx(0, 0));
    for (int i = 0; i < W; ++i)
        for (int ii = 0; ii < W; ++ii)
            out[(size_t)((i + W / 2) % W) * W + (ii + W / 2) % W] = cplx(I[(size_t)i * W + ii], 0);
    fft2d(out, W, -1);
    for (int i = 0; i < W; ++i)
        for (int ii = 0; ii < W; ++ii)
            out[(size_t)i * W + ii] *= gauss_value(p, W, (i + W / 2) % W, (ii + W / 2) % W);
    fft2d(out, W, +1);
}

// PSFPhase.computePSF (PSFPhase.java:557-629): psi[R][R], first index <-> x.
// With derivs != nullptr also the analytic derivatives d psi / d{x,y,zwat}
// (3 * R * R), obtained through the same FFT route.
void psf_model(const Psf* p, int R, double x, double y, double zoil, double zwat,
               double* psi, double* derivs) {
    int N = p->N, W = window_size(R, N);
    std::vector<cplx> E, Ed[3];
    pupil_field(p, x, y, zoil, zwat, 0, E);
    fft2d(E, N, +1);
    int nd = derivs ? 3 : 0;
    for (int d = 0; d < nd; ++d) {
        pupil_field(p, x, y, zoil, zwat, d + 1, Ed[d]);
        fft2d(Ed[d], N, +1);
    }
    std::vector<double> I((size_t)W * W), Id[3];
    for (int d = 0; d < nd; ++d) Id[d].resize((size_t)W * W);
    for (int i = 0; i < W; ++i)
        for (int ii = 0; ii < W; ++ii) {
            size_t src = (size_t)((N / 2 - W / 2 + i + N / 2) % N) * N + (N / 2 - W / 2 + ii + N / 2) % N;
            cplx e = E[src];
            I[(size_t)i * W + ii] = e.real() * e.real() + e.imag() * e.imag();
            for (int d = 0; d < nd; ++d)
                Id[d][(size_t)i * W + ii] = 2.0 * (std::conj(e) * Ed[d][src]).real();
        }
    std::vector<cplx> B, Bd[3];
    blur_window(p, W, I, B);
    for (int d = 0; d < nd; ++d) blur_window(p, W, Id[d], Bd[d]);
    double sum = 0.0;
    std::vector<double> m((size_t)R * R), dm[3];
    for (int d = 0; d < nd; ++d) dm[d].resize((size_t)R * R);
    double dsum[3] = {0, 0, 0};
    for (int i = 0; i < R; ++i)
        for (int ii = 0; ii < R; ++ii) {
            size_t src = (size_t)((W / 2 - R / 2 + i + W / 2) % W) * W + (W / 2 - R / 2 + ii + W / 2) % W;
            cplx b = B[src];
            double mag = std::sqrt(b.real() * b.real() + b.imag() * b.imag());
            m[(size_t)i * R + ii] = mag;
            sum += mag;
            for (int d = 0; d < nd; ++d) {
                // d|b| = Re(conj(b) db)/|b|; the blurred window is real up to rounding.
                double v = mag > 0 ? (std::conj(b) * Bd[d][src]).real() / mag : 0.0;
                dm[d][(size_t)i * R + ii] = v;
                dsum[d] += v;
            }
        }
    for (int k = 0; k < R * R; ++k) psi[k] = m[k] / sum;
    for (int d = 0; d < nd; ++d)
        for (int k = 0; k < R * R; ++k)
            derivs[(size_t)d * R * R + k] = (dm[d][k] - psi[k] * dsum[d]) / sum;
}

// ------------------------------------------------- coordinate descent ------
// Localization.java (single camera, single frame), with Zfocus as zoil.
struct CD {
    const Psf* p;
    int R;
    const double* d;   // patch R*R (photons), [x][y]
    const double* v = nullptr;  // sCMOS var/gain^2 patch (Localization.java:1132), or none
    double minZ, maxZ;
    int iterMax;
    double photonThreshold;
    double h = .0005, eps = .0001, maxShift;
    double tx, ty, tz, ta, tb;
    std::vector<double> psi, mu;
    int nevals = 0;

    double lik(double x, double y, double z, double a, double b) {  // :1125-1143
        psf_model(p, R, x, y, p->zfocus, z, psi.data(), nullptr);
        ++nevals;
        double l = 0;
        for (int k = 0; k < R * R; ++k) {
            double m = psi[k] * a + b + (v ? v[k] : 0.0);
            mu[k] = m;
            l += m - d[k] * std::log(m);
        }
        return l;
    }
    void clampAB() { ta = std::max(1.0, ta); tb = std::max(.01, tb); }  // testPhotonNumber
    static double newton(double l1, double l2, double l3, double h) {
        double curv = std::fabs((l3 + l1 - 2 * l2) / (h * h));
        if (curv == 0) return (l3 - l1) * (2 * h);
        return ((l3 - l1) / (2 * h)) / curv;
    }
    // minimizeX/Y/Z (:672-916): Newton step capped at maxShift, gamma 1, .1, .01.
    double minCoord(double* t, double prev, int which) {
        double save = *t;
        double l1, l3;
        double sv = *t;
        *t = sv - h; l1 = lik(tx, ty, tz, ta, tb);
        *t = sv + h; l3 = lik(tx, ty, tz, ta, tb);
        *t = sv;
        (void)which;
        double l2 = prev;
        double g = newton(l1, l2, l3, h);
        if (g > maxShift) g = maxShift;
        else if (g < -maxShift) g = -maxShift;
        for (double gamma = 1; gamma > .02; gamma /= 10) {
            *t -= gamma * g;
            double l = lik(tx, ty, tz, ta, tb);
            if (l < l2) { prev = l; break; }
            *t = save;
        }
        return prev;
    }
    // minimizeA (:919-970) and minimizeB (:974-1036): no early break.
    double minAB(double* t, double hh) {
        double save = *t;
        double sv = *t;
        *t = sv - hh; double l1 = lik(tx, ty, tz, ta, tb);
        *t = sv; double l2 = lik(tx, ty, tz, ta, tb);
        *t = sv + hh; double l3 = lik(tx, ty, tz, ta, tb);
        *t = save;
        double g = newton(l1, l2, l3, hh);
        for (double gamma = 1; gamma > .02; gamma /= 10) {
            *t -= gamma * g;
            double l = lik(tx, ty, tz, ta, tb);
            if (l < l2) { l2 = l; save = *t; }
            else *t = save;
        }
        return lik(tx, ty, tz, ta, tb);
    }
    // localize (:491-653); returns false on the photon-count break or NaN.
    int run() {
        clampAB();
        double likelihood = lik(tx, ty, tz, ta, tb);
        double oX = 1e300, oY = 1e300, oZ = 1e300;
        bool brk4 = false;
        likelihood = minAB(&ta, h * 1000); clampAB();
        likelihood = minAB(&tb, h * 10); clampAB();
        int it = 0;
        for (int i = 0; i < iterMax; ++i) {
            it = i + 1;
            likelihood = minCoord(&tz, likelihood, 2);
            if (tz < minZ) tz = minZ;
            if (tz > maxZ) tz = maxZ;
            likelihood = minCoord(&tx, likelihood, 0);
            likelihood = minCoord(&ty, likelihood, 1);
            likelihood = minAB(&ta, h * 1000); clampAB();
            likelihood = minAB(&tb, h * 10); clampAB();
            double dist = std::sqrt((tx - oX) * (tx - oX) + (ty - oY) * (ty - oY) + (tz - oZ) * (tz - oZ));
            bool breaking = false;
            if (i > 4) { breaking = !(ta > photonThreshold); if (breaking) brk4 = true; }
            if (dist < eps || breaking) break;
            if (std::isnan(likelihood)) return -1;
            oX = tx; oY = ty; oZ = tz;
        }
        (void)it;
        return brk4 ? 0 : 1;
    }
};

// Finite-difference Fisher matrix and CRLB, Localization.java:317-451,
// including its A-derivative, which differentiates mu*(a+-h)+b (mu, not psi).
// Finite-difference Fisher matrix of Localization.java:317-451 (also
// process/cpu/CRLB.java:255-340 and SearchPSFcenter.java:210-330): central
// differences of step h in x, y, z; the A and B rows perturb the already
// formed mean f1 = a psi + b, so dmu/dA = f1 * ha / h and dmu/dB = 1.
void fisher_fd(const Psf* p, int R, double x, double y, double z, double a, double b, double h, double ha,
               double F[5][5]) {
    int n = R * R;
    std::vector<double> f(n), f1(n), f0[5], f2[5], tmp(n);
    for (int q = 0; q < 5; ++q) { f0[q].resize(n); f2[q].resize(n); }
    psf_model(p, R, x, y, p->zfocus, z, f.data(), nullptr);
    for (int k = 0; k < n; ++k) f1[k] = f[k] * a + b;
    double sh[3][2][3] = {{{x + h, y, z}, {x - h, y, z}}, {{x, y + h, z}, {x, y - h, z}}, {{x, y, z + h}, {x, y, z - h}}};
    for (int q = 0; q < 3; ++q) {
        psf_model(p, R, sh[q][0][0], sh[q][0][1], p->zfocus, sh[q][0][2], tmp.data(), nullptr);
        for (int k = 0; k < n; ++k) f2[q][k] = tmp[k] * a + b;
        psf_model(p, R, sh[q][1][0], sh[q][1][1], p->zfocus, sh[q][1][2], tmp.data(), nullptr);
        for (int k = 0; k < n; ++k) f0[q][k] = tmp[k] * a + b;
    }
    for (int k = 0; k < n; ++k) {
        f0[3][k] = f1[k] * (a - ha) + b; f2[3][k] = f1[k] * (a + ha) + b;
        f0[4][k] = f1[k] * a + (b - h); f2[4][k] = f1[k] * a + (b + h);
    }
    for (int q = 0; q < 5; ++q)
        for (int qq = 0; qq < 5; ++qq) {
            double s = 0;
            for (int k = 0; k < n; ++k) {
                double d1 = (f2[q][k] - f0[q][k]) / (2 * std::fabs(h));
                double d2 = (f2[qq][k] - f0[qq][k]) / (2 * std::fabs(h));
                s += (1 / f1[k]) * d1 * d2;
            }
            F[q][qq] = s;
        }
}

// sqrt(diag(F^-1)) (Gauss-Jordan with partial pivoting); when F is singular,
// sqrt(1 / F_ii) as the reference's fallback.
void crlb_from_fisher(const double F[5][5], double* crlb, int nout) {
    double M[5][10];
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 10; ++j) M[i][j] = j < 5 ? F[i][j] : (j - 5 == i ? 1 : 0);
    bool ok = true;
    for (int c = 0; c < 5 && ok; ++c) {
        int piv = c;
        for (int r = c + 1; r < 5; ++r) if (std::fabs(M[r][c]) > std::fabs(M[piv][c])) piv = r;
        if (M[piv][c] == 0) { ok = false; break; }
        for (int j = 0; j < 10; ++j) std::swap(M[c][j], M[piv][j]);
        double dv = M[c][c];
        for (int j = 0; j < 10; ++j) M[c][j] /= dv;
        for (int r = 0; r < 5; ++r) if (r != c) {
            double fct = M[r][c];
            for (int j = 0; j < 10; ++j) M[r][j] -= fct * M[c][j];
        }
    }
    for (int i = 0; i < nout; ++i) {
        if (ok) crlb[i] = std::sqrt(M[i][5 + i]);
        else crlb[i] = F[i][i] != 0 ? std::sqrt(1 / F[i][i]) : 1.79769313486231570e308;
    }
}

void fisher_crlb_fd(const Psf* p, int R, double x, double y, double z, double a, double b,
                    double* crlb3) {
    double F[5][5];
    fisher_fd(p, R, x, y, z, a, b, .0005, .0005, F);
    crlb_from_fisher(F, crlb3, 3);
}

// ------------------------------------------------------ z-centre search ----
// process/cpu/SearchPSFcenter.java:37-203 (variant 0: h = 5 nm, A step 100 h)
// and process/gpu/SearchPSFcenter_.java (variant 1: h = 0.5 nm, A step h,
// returns zfocus at once when n_oil == n_wat).  Emitter at (0, 0, zwat = u),
// zoil = zfocus, 3000 photons, background 50; the model is the R x R field
// with R the grid size the caller loaded (SearchPSFcenter.java:31 builds it
// at the FFT size).  Loops keep the reference's floating-point accumulation.
struct CenterSearch {
    const Psf* p;
    int R;
    double h, ha;
    double crlb_xy(double z) const {
        double F[5][5], c[5];
        fisher_fd(p, R, 0, 0, z, 3000, 50, h, ha, F);
        crlb_from_fisher(F, c, 5);
        return std::sqrt(c[0] * c[0] + c[1] * c[1]);
    }
    double min_position(double minZ, double maxZ, double stepZ) const {  // :173-203
        double best = INFINITY, pos = 0;
        for (double u = minZ; u < maxZ; u += stepZ) {
            double c = crlb_xy(u);
            if (best > c) { best = c; pos = u; }
        }
        return pos;
    }
    bool min_range(double minZ, double maxZ, double stepZ, double axialRange, double* out) const {  // :88-170
        double ar = axialRange / 2;
        std::vector<double> crlb;
        for (double u = minZ - ar / 2; u <= maxZ + ar / 2; u += stepZ) crlb.push_back(crlb_xy(u));
        double best = INFINITY, pos = 0;
        int nb = (int)(ar / (2 * stepZ));
        for (double u = minZ; u < maxZ; u += stepZ) {
            double s = 0;
            int nb2 = -(int)(ar / (2 * stepZ));
            for (double i = -ar / 2; i <= ar / 2; i += stepZ) {
                int k = nb + nb2;
                if (k < 0 || k >= (int)crlb.size()) return false;
                s += crlb[k];
                nb2++;
            }
            if (best > s) { best = s; pos = u; }
            nb++;
        }
        *out = pos;
        return true;
    }
};

double center_search(const Psf* p, int R, double axialRange, int variant, int* status) {  // :37-84
    *status = 0;
    double zfocus = p->zfocus;
    if (axialRange <= 0) return zfocus;
    if (variant == 1 && p->n_oil == p->n_wat) return zfocus;
    CenterSearch cs{p, R, variant == 1 ? .0005 : .005, variant == 1 ? .0005 : .005 * 100};
    double stepZ = p->dx * 5;
    double minZ = zfocus - 2 * axialRange - std::fabs(zfocus);
    double maxZ = zfocus + std::fabs(zfocus) + 2 * axialRange;
    double position = cs.min_position(minZ, maxZ, stepZ);
    double old = INFINITY;
    for (int i = 0; i < 10; i++) {
        minZ = position - stepZ * 5;
        maxZ = position + stepZ * 5;
        stepZ = stepZ / 2;
        position = cs.min_position(minZ, maxZ, stepZ);
        if (std::fabs(old - position) < 0.00001) break;
        old = position;
    }
    double out = position;
    if (!cs.min_range(position - axialRange * 2, position + axialRange * 2, p->dx, axialRange, &out)) *status = -1;
    return out;
}

// ------------------------------------------------------------ LM fit -------
// The FP64 Levenberg-Marquardt fit shared (as an algorithm) with the GPU
// library.  theta = x, y, z (um), A (photons), B (photons/px).
struct LMParams {
    double zmin, zmax, xymax;  // box: |x|,|y| <= xymax, zmin <= z <= zmax
    int max_iter;              // model evaluations
    double tol_xyz;            // um
    double step_xy, step_z;    // per-iteration caps (um)
};

// Deviance-form Poisson NLL: sum mu - d - d ln(mu/d) (mu - d ln mu + const).
// Returns +inf if any mu <= 0.
// v (nullable): the sCMOS term var/gain^2 added to the model mean
// (process/cpu/Localization.java:1132).
double model_eval(const Psf* p, int R, const double* d, const double* th, double* g, double H[5][5],
                  std::vector<double>& psi, std::vector<double>& dpsi, const double* v = nullptr) {
    int n = R * R;
    psf_model(p, R, th[0], th[1], p->zfocus, th[2], psi.data(), dpsi.data());
    double nll = 0;
    for (int q = 0; q < 5; ++q) { g[q] = 0; for (int r = 0; r < 5; ++r) H[q][r] = 0; }
    for (int k = 0; k < n; ++k) {
        double mu = th[3] * psi[k] + th[4] + (v ? v[k] : 0.0);
        if (!(mu > 0)) return INFINITY;
        double dk = d[k];
        nll += dk > 0 ? mu - dk - dk * std::log(mu / dk) : mu;
        double j[5] = {th[3] * dpsi[k], th[3] * dpsi[n + k], th[3] * dpsi[2 * n + k], psi[k], 1.0};
        double w = 1.0 - dk / mu, w2 = dk / (mu * mu);
        for (int q = 0; q < 5; ++q) {
            g[q] += w * j[q];
            for (int r = 0; r <= q; ++r) H[q][r] += w2 * j[q] * j[r];
        }
    }
    for (int q = 0; q < 5; ++q) for (int r = q + 1; r < 5; ++r) H[q][r] = H[r][q];
    return nll;
}

// Cholesky solve of (H + lambda max(diag H, floor)) delta = -g; false if not
// positive definite.  The floors (1 um^-2 for x, y, z; 1e-10 and 1e-6 for A
// and B) keep the damping positive where a derivative vanishes by symmetry.
bool damped_solve(const double H[5][5], const double* g, double lambda, double* delta) {
    static const double floor_[5] = {1.0, 1.0, 1.0, 1e-10, 1e-6};
    double L[5][5] = {};
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = H[i][j] + (i == j ? lambda * std::max(H[i][i], floor_[i]) : 0.0);
            for (int k = 0; k < j; ++k) s -= L[i][k] * L[j][k];
            if (i == j) {
                if (!(s > 0)) return false;
                L[i][i] = std::sqrt(s);
            } else L[i][j] = s / L[j][j];
        }
    double yv[5];
    for (int i = 0; i < 5; ++i) {
        double s = -g[i];
        for (int k = 0; k < i; ++k) s -= L[i][k] * yv[k];
        yv[i] = s / L[i][i];
    }
    for (int i = 4; i >= 0; --i) {
        double s = yv[i];
        for (int k = i + 1; k < 5; ++k) s -= L[k][i] * delta[k];
        delta[i] = s / L[i][i];
    }
    return true;
}

void clamp_theta(double* th, const LMParams& P) {
    th[0] = std::min(std::max(th[0], -P.xymax), P.xymax);
    th[1] = std::min(std::max(th[1], -P.xymax), P.xymax);
    th[2] = std::min(std::max(th[2], P.zmin), P.zmax);
    th[3] = std::max(th[3], 1.0);
    th[4] = std::max(th[4], 0.01);
}

// status: 1 converged, 2 max evaluations, 3 stalled (lambda at bound), -1 NaN.
int lm_fit(const Psf* p, int R, const double* d, const double* init, const LMParams& P,
           double* out, double* nll_out, int* evals_out, double* crlb5, const double* v = nullptr) {
    int n = R * R;
    std::vector<double> psi(n), dpsi(3 * n), psi2(n), dpsi2(3 * n);
    double th[5], g[5], H[5][5];
    for (int q = 0; q < 5; ++q) th[q] = init[q];
    clamp_theta(th, P);
    double nll = model_eval(p, R, d, th, g, H, psi, dpsi, v);
    int evals = 1;
    double lambda = 1e-3;
    int status = 2;
    // converged when the undamped Gauss-Newton step from the accepted point
    // moves x, y, z by less than tol and A, B by less than 1e-4 of their values
    // (distance to the local optimum)
    auto at_optimum = [&]() {
        double d0[5];
        if (!damped_solve(H, g, 0.0, d0)) return false;
        return std::max(std::fabs(d0[0]), std::max(std::fabs(d0[1]), std::fabs(d0[2]))) < P.tol_xyz &&
               std::fabs(d0[3]) < 1e-4 * th[3] && std::fabs(d0[4]) < 1e-4 * std::max(th[4], 1.0);
    };
    if (!std::isfinite(nll)) status = -1;
    else if (at_optimum()) status = 1;
    while (status == 2 && evals < P.max_iter) {
        double delta[5];
        if (!damped_solve(H, g, lambda, delta)) {
            lambda *= 10;
            if (lambda > 1e7) { status = 3; break; }
            continue;
        }
        double sxy = std::max(std::fabs(delta[0]), std::fabs(delta[1]));
        double scale = 1.0;
        if (sxy > P.step_xy) scale = P.step_xy / sxy;
        if (std::fabs(delta[2]) * scale > P.step_z) scale = P.step_z / std::fabs(delta[2]);
        double t2[5], g2[5], H2[5][5];
        for (int q = 0; q < 5; ++q) t2[q] = th[q] + scale * delta[q];
        clamp_theta(t2, P);
        double nll2 = model_eval(p, R, d, t2, g2, H2, psi2, dpsi2, v);
        ++evals;
        if (nll2 <= nll) {
            for (int q = 0; q < 5; ++q) { th[q] = t2[q]; g[q] = g2[q]; for (int r = 0; r < 5; ++r) H[q][r] = H2[q][r]; }
            nll = nll2;
            lambda = std::max(lambda * 0.1, 1e-7);
            if (at_optimum()) status = 1;
        } else {
            lambda *= 10;
            if (lambda > 1e7) status = 3;
        }
    }
    for (int q = 0; q < 5; ++q) out[q] = th[q];
    *nll_out = nll;
    *evals_out = evals;
    if (crlb5) {  // sqrt(diag(F^-1)) from the analytic Fisher matrix at the optimum
        model_eval(p, R, d, th, g, H, psi, dpsi, v);
        double F[5][5] = {};
        for (int k = 0; k < n; ++k) {
            double mu = th[3] * psi[k] + th[4] + (v ? v[k] : 0.0);
            double j[5] = {th[3] * dpsi[k], th[3] * dpsi[n + k], th[3] * dpsi[2 * n + k], psi[k], 1.0};
            for (int q = 0; q < 5; ++q) for (int r = 0; r < 5; ++r) F[q][r] += j[q] * j[r] / mu;
        }
        for (int c = 0; c < 5; ++c) {
            double e[5] = {0, 0, 0, 0, 0}, col[5];
            e[c] = 1;
            double G[5] = {-e[0], -e[1], -e[2], -e[3], -e[4]};
            if (damped_solve(F, G, 0.0, col)) crlb5[c] = std::sqrt(col[c]);
            else crlb5[c] = NAN;
        }
    }
    return status;
}

// ----------------------------------------------------------- detection ----
// Predetection.java:63-593 (one frame).  image is [X][Y] (first index x).
struct Detector {
    const Psf* p;
    int SX, SY, R, MX, MY, nz;
    double thr, zstep;
    std::vector<double> range, varPSF, normImage;
    std::vector<std::vector<cplx>> dict;
    std::vector<std::vector<double>> libpsf;
};

void fft2d_rect(std::vector<cplx>& a, int nx, int ny, int sign) {
    std::vector<cplx> col(nx);
    for (int i = 0; i < nx; ++i) fft1d(&a[(size_t)i * ny], ny, sign);
    for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) col[i] = a[(size_t)i * ny + j];
        fft1d(col.data(), nx, sign);
        for (int i = 0; i < nx; ++i) a[(size_t)i * ny + j] = col[i];
    }
}

Detector* det_build(const Psf* p, int SX, int SY, int R, double minZ, double maxZ, double step, double thr) {
    Detector* D = new Detector();
    D->p = p; D->SX = SX; D->SY = SY; D->R = R; D->thr = thr; D->zstep = step;
    D->MX = pow2ceil(2 * SX); D->MY = pow2ceil(2 * SY);
    D->normImage.resize((size_t)SX * SY);
    for (int i = 0; i < SX; ++i)          // Predetection.java:95-116, verbatim index rules
        for (int ii = 0; ii < SY; ++ii) {
            int vx1 = R / 2, vx2 = R / 2;
            if (i < R / 2 - 1) vx1 = i + 1;
            if (i > SX - R / 2 - 2) vx2 = SY - i - 1;
            int vy1 = R / 2, vy2 = R / 2;
            if (ii < R / 2 - 1) vy1 = ii + 1;
            if (ii > SX - R / 2 - 2) vy2 = SY - ii - 2;
            D->normImage[(size_t)i * SY + ii] = (double)((vx1 + vx2) * (vy1 + vy2));
        }
    int number = (int)std::ceil((maxZ - minZ) / step);
    double z = minZ;
    for (int i = 0; i < number; ++i) { D->range.push_back(z); z += step; }
    D->nz = number;
    std::vector<double> psf((size_t)R * R);
    for (int i = 0; i < number; ++i) {
        psf_model(p, R, 0, 0, p->zfocus, D->range[i], psf.data(), nullptr);
        D->libpsf.push_back(psf);
        double mean = 0;
        for (int k = 0; k < R * R; ++k) mean += psf[k];
        mean /= (double)R * R;
        double var = 0;
        std::vector<double> pd(psf);
        for (int k = 0; k < R * R; ++k) { pd[k] -= mean; var += pd[k] * pd[k]; }
        var /= (double)(R * R);
        D->varPSF.push_back(var);
        std::vector<cplx> g((size_t)D->MX * D->MY, cplx(0, 0));
        for (int u = 0; u < R; ++u)
            for (int uu = 0; uu < R; ++uu) {
                int x = (u - R / 2 + D->MX / 2 + D->MX / 2) % D->MX;
                int y = (uu - R / 2 + D->MY / 2 + D->MY / 2) % D->MY;
                g[(size_t)x * D->MY + y] = cplx(pd[(size_t)u * R + uu], 0);
            }
        fft2d_rect(g, D->MX, D->MY, -1);
        D->dict.push_back(g);
    }
    return D;
}

double top_of_parabola(double xa, double ya, double xb, double yb, double xc, double yc) {
    double a = (yc - ya) / ((xc - xa) * (xc - xb)) - (yb - ya) / ((xb - xa) * (xc - xb));
    double b = ((yb - ya) / (xb - xa)) - a * (xb + xa);
    return -b / (2 * a);
}

// Candidate rows: score, r, i, j, topZ, topX, topY (Predetection.java:520-540).
void det_frame(const Detector* D, const double* image, std::vector<std::array<double, 7>>& out) {
    int SX = D->SX, SY = D->SY, R = D->R, MX = D->MX, MY = D->MY;
    std::vector<double> full((size_t)SX * SY);
    std::vector<cplx> X((size_t)MX * MY, cplx(0, 0));
    for (int i = 0; i < SX; ++i)
        for (int ii = 0; ii < SY; ++ii) {
            full[(size_t)i * SY + ii] = (double)(float)image[(size_t)i * SY + ii];
            int x = (i - SX / 2 + MX / 2 + MX / 2) % MX;
            int y = (ii - SY / 2 + MY / 2 + MY / 2) % MY;
            X[(size_t)x * MY + y] = cplx(image[(size_t)i * SY + ii], 0);
        }
    fft2d_rect(X, MX, MY, -1);
    // running sums (Predetection.java:337-405)
    std::vector<double> s1((size_t)SX * SY), s2((size_t)SX * SY), t1((size_t)SX * SY), t2((size_t)SX * SY);
    auto F = [&](int i, int j) { return full[(size_t)i * SY + j]; };
    for (int i = 0; i < SX; ++i) {
        double a = 0, b = 0;
        for (int t = 0; t < R / 2 + 1; ++t) if (t < SY) { a += F(i, t); b += F(i, t) * F(i, t); }
        s1[(size_t)i * SY] = a; s2[(size_t)i * SY] = b;
        for (int ii = 1; ii < SY; ++ii) {
            double v = s1[(size_t)i * SY + ii - 1];
            if (ii - R / 2 >= 0) v -= F(i, ii - R / 2);
            if (ii + R / 2 < SY) v += F(i, ii + R / 2);
            s1[(size_t)i * SY + ii] = v;
            double w = s2[(size_t)i * SY + ii - 1];
            if (ii - R / 2 >= 0) w -= F(i, ii - R / 2) * F(i, ii - R / 2);
            if (ii + R / 2 < SY) w += F(i, ii + R / 2) * F(i, ii + R / 2);
            s2[(size_t)i * SY + ii] = w;
        }
    }
    std::vector<double> var((size_t)SX * SY);
    for (int ii = 0; ii < SY; ++ii) {
        double a = 0, b = 0;
        for (int t = 0; t < R / 2 + 1; ++t) if (t < SX) { a += s1[(size_t)t * SY + ii]; b += s2[(size_t)t * SY + ii]; }
        t1[ii] = a; t2[ii] = b;
        for (int i = 1; i < SX; ++i) {
            double v = t1[(size_t)(i - 1) * SY + ii];
            if (i - R / 2 >= 0) v -= s1[(size_t)(i - R / 2) * SY + ii];
            if (i + R / 2 < SX) v += s1[(size_t)(i + R / 2) * SY + ii];
            t1[(size_t)i * SY + ii] = v;
            double w = t2[(size_t)(i - 1) * SY + ii];
            if (i - R / 2 >= 0) w -= s2[(size_t)(i - R / 2) * SY + ii];
            if (i + R / 2 < SX) w += s2[(size_t)(i + R / 2) * SY + ii];
            t2[(size_t)i * SY + ii] = w;
        }
        for (int i = 0; i < SX; ++i) {
            double nrm = D->normImage[(size_t)i * SY + ii];
            double mean = t1[(size_t)i * SY + ii] / nrm;
            var[(size_t)i * SY + ii] = (t2[(size_t)i * SY + ii] / nrm) - mean * mean;
        }
    }
    // correlation maps
    int nz = D->nz;
    std::vector<double> res((size_t)nz * SX * SY, 0.0);
    std::vector<cplx> P((size_t)MX * MY);
    for (int r = 0; r < nz; ++r) {
        const std::vector<cplx>& Dz = D->dict[r];
        for (size_t k = 0; k < P.size(); ++k)
            P[k] = cplx(X[k].imag() * Dz[k].imag() + X[k].real() * Dz[k].real(),
                        X[k].imag() * Dz[k].real() - X[k].real() * Dz[k].imag());
        fft2d_rect(P, MX, MY, +1);
        for (int ii = 0; ii < SX; ++ii)
            for (int iii = 0; iii < SY; ++iii) {
                int x = (ii - SX / 2 + MX / 2 + MX / 2) % MX;
                int y = (iii - SY / 2 + MY / 2 + MY / 2) % MY;
                double v = var[(size_t)ii * SY + iii];
                double s = std::sqrt(D->varPSF[r] * v);
                double o;
                if (s > 0) o = P[(size_t)x * MY + y].real() / s;
                else if (D->varPSF[r] <= 0) o = -1;
                else o = -2;  // v <= 0 (or NaN product)
                res[((size_t)r * SX + ii) * SY + iii] = o;
            }
    }
    // local maxima (getVectMaxPosition, Predetection.java:480-560)
    int dec = 3, lo = std::max(dec, R / 2);
    std::vector<double> tmp((size_t)SX * SY, 0.0);
    auto RC = [&](int r, int i, int j) { return res[((size_t)r * SX + i) * SY + j]; };
    out.clear();
    for (int r = 0; r < nz; ++r) {
        for (int i = lo; i < SX - lo; ++i)
            for (int j = lo; j < SY - lo; ++j)
                if (RC(r, i, j) > 0) {
                    double t = -INFINITY;
                    for (int a = -dec; a <= dec; ++a) t = std::max(RC(r, i, j + a), t);
                    tmp[(size_t)i * SY + j] = t;
                }
        for (int j = lo; j < SY - lo; ++j)
            for (int i = lo; i < SX - lo; ++i) {
                double v = RC(r, i, j);
                if (!(v > D->thr)) continue;
                if (v != tmp[(size_t)i * SY + j]) continue;
                double mx = -INFINITY;
                for (int a = -dec; a <= dec; ++a) mx = std::max(tmp[(size_t)(i + a) * SY + j], mx);
                if (mx != v) continue;
                double tz = 0, tx = 0, ty = 0;
                if (r > 1 && r < nz - 1) tz = top_of_parabola(-D->zstep, RC(r - 1, i, j), 0, v, D->zstep, RC(r + 1, i, j));
                if (i > 1 && i < SX - 1) tx = top_of_parabola(-D->p->dx, RC(r, i - 1, j), 0, v, D->p->dx, RC(r, i + 1, j));
                if (j > 1 && j < SY - 1) ty = top_of_parabola(-D->p->dx, RC(r, i, j - 1), 0, v, D->p->dx, RC(r, i, j + 1));
                out.push_back({v, (double)r, (double)i, (double)j, tz, tx, ty});
            }
    }
    std::stable_sort(out.begin(), out.end(), [](const std::array<double, 7>& a, const std::array<double, 7>& b) { return a[0] > b[0]; });
}

}  // namespace

// ================================================================ C ABI ====
extern "C" {

void* orc_psf_create(int N, double dx, double na, double lambda, double n_oil, double n_wat,
                     double sigma, int apo, double zfocus, int kz_reset, int gauss_f32,
                     int nz, const double* zern) {
    return psf_build(N, dx, na, lambda, n_oil, n_wat, sigma, apo, zfocus, kz_reset, gauss_f32, nz, zern);
}
void orc_psf_destroy(void* h) { delete (Psf*)h; }
int orc_psf_info(void* h, int* N, int* K) { Psf* p = (Psf*)h; *N = p->N; *K = p->K; return 0; }
int orc_psf_tables(void* h, double* kx, double* ky, double* kz, double* kzoil, double* pupil, double* phase) {
    Psf* p = (Psf*)h;
    for (int k = 0; k < p->K; ++k) {
        kx[k] = p->kx[k]; ky[k] = p->ky[k]; kz[k] = p->kz[k]; kzoil[k] = p->kzoil[k];
        pupil[k] = p->pupil[k]; phase[k] = p->phase[k];
    }
    return 0;
}
int orc_window_size(int R, int N) { return window_size(R, N); }

// n models at (x, y, z) with zoil = zfocus; out n*R*R (+ derivs n*3*R*R).
void orc_psf_model(void* h, int R, int n, const double* xyz, double* out, double* derivs) {
    const Psf* p = (const Psf*)h;
    for (int i = 0; i < n; ++i)
        psf_model(p, R, xyz[3 * i], xyz[3 * i + 1], p->zfocus, xyz[3 * i + 2], out + (size_t)i * R * R,
                  derivs ? derivs + (size_t)i * 3 * R * R : nullptr);
}

// Explicit zoil/zwat form (calibration uses zoil = slice depth, zwat = 0).
void orc_psf_model_oil(void* h, int R, double x, double y, double zoil, double zwat, double* out) {
    psf_model((const Psf*)h, R, x, y, zoil, zwat, out, nullptr);
}

}

static void parallel_for(int n, int threads, const std::function<void(int)>& f) {
    if (threads <= 1) { for (int i = 0; i < n; ++i) f(i); return; }
    std::atomic<int> next(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&]() { for (int i; (i = next.fetch_add(1)) < n;) f(i); });
    for (auto& th : pool) th.join();
}

extern "C" {

// Reference coordinate-descent localisation (+ finite-difference CRLB) of n
// patches.  init: n*5 (A, B, x, y, z) in the order Localization.init takes.
// out: n*5 (x, y, z, A, B); crlb: n*3 (um); status: 1 ok, 0 photon break, -1 NaN.
// eps is the stopping distance of the x/y/z move per sweep (the reference's
// 1e-4 um, Localization.java:31); orc_localize_cd_eps takes another one.
void orc_localize_cd_eps(void* h, int R, int n, const double* patches, const double* init,
                         double minZ, double maxZ, int iterMax, double photonThr, double eps,
                         double* out, double* crlb, int* status, int* evals, int threads) {
    const Psf* p = (const Psf*)h;
    parallel_for(n, threads, [&](int i) {
        CD cd;
        cd.eps = eps;
        cd.p = p; cd.R = R; cd.d = patches + (size_t)i * R * R;
        cd.minZ = minZ; cd.maxZ = maxZ; cd.iterMax = iterMax; cd.photonThreshold = photonThr;
        cd.maxShift = p->dx / 2.;
        cd.psi.resize(R * R); cd.mu.resize(R * R);
        cd.ta = init[5 * i]; cd.tb = init[5 * i + 1]; cd.tx = init[5 * i + 2]; cd.ty = init[5 * i + 3]; cd.tz = init[5 * i + 4];
        int st = cd.run();
        out[5 * i] = cd.tx; out[5 * i + 1] = cd.ty; out[5 * i + 2] = cd.tz; out[5 * i + 3] = cd.ta; out[5 * i + 4] = cd.tb;
        if (crlb) fisher_crlb_fd(p, R, cd.tx, cd.ty, cd.tz, cd.ta, cd.tb, crlb + 3 * i);
        status[i] = st;
        if (evals) evals[i] = cd.nevals;
    });
}

void orc_localize_cd(void* h, int R, int n, const double* patches, const double* init,
                     double minZ, double maxZ, int iterMax, double photonThr,
                     double* out, double* crlb, int* status, int* evals, int threads) {
    orc_localize_cd_eps(h, R, n, patches, init, minZ, maxZ, iterMax, photonThr, 1e-4, out, crlb, status, evals,
                        threads);
}

// FP64 LM fit of n patches.  init/out: n*5 (x, y, z, A, B).  params:
// zmin, zmax, xymax, tol_xyz, step_xy, step_z; max_iter evaluations.
void orc_fit_lm(void* h, int R, int n, const double* patches, const double* init, const double* params,
                int max_iter, double* out, double* nll, int* status, int* evals, double* crlb5, int threads) {
    const Psf* p = (const Psf*)h;
    LMParams P{params[0], params[1], params[2], max_iter, params[3], params[4], params[5]};
    parallel_for(n, threads, [&](int i) {
        status[i] = lm_fit(p, R, patches + (size_t)i * R * R, init + 5 * i, P, out + 5 * i, nll + i,
                           evals + i, crlb5 ? crlb5 + 5 * i : nullptr);
    });
}

// The same fits with a per-ROI sCMOS term (n x R x R, added to the mean).
void orc_fit_lm_scmos(void* h, int R, int n, const double* patches, const double* scmos, const double* init,
                      const double* params, int max_iter, double* out, double* nll, int* status, int* evals,
                      double* crlb5, int threads) {
    const Psf* p = (const Psf*)h;
    LMParams P{params[0], params[1], params[2], max_iter, params[3], params[4], params[5]};
    parallel_for(n, threads, [&](int i) {
        status[i] = lm_fit(p, R, patches + (size_t)i * R * R, init + 5 * i, P, out + 5 * i, nll + i, evals + i,
                           crlb5 ? crlb5 + 5 * i : nullptr, scmos + (size_t)i * R * R);
    });
}

// Deviance-form NLL and its analytic gradient / Gauss-Newton Hessian at theta.
double orc_nll_grad(void* h, int R, const double* patch, const double* th, double* g, double* H25) {
    const Psf* p = (const Psf*)h;
    std::vector<double> psi(R * R), dpsi(3 * R * R);
    double H[5][5];
    double v = model_eval(p, R, patch, th, g, H, psi, dpsi);
    for (int q = 0; q < 5; ++q) for (int r = 0; r < 5; ++r) H25[5 * q + r] = H[q][r];
    return v;
}

double orc_center_search(void* h, int R, double axial_range, int variant, int* status) {
    return center_search((Psf*)h, R, axial_range, variant, status);
}
void orc_crlb_curve(void* h, int R, int n, const double* z, double photons, double bg, double step, double a_step,
                    double* crlb5) {
    for (int i = 0; i < n; ++i) {
        double F[5][5];
        fisher_fd((Psf*)h, R, 0, 0, z[i], photons, bg, step, a_step, F);
        crlb_from_fisher(F, crlb5 + 5 * i, 5);
    }
}
void orc_crlb_fd(void* h, int R, const double* th, double* crlb3) {
    const Psf* p = (const Psf*)h;
    fisher_crlb_fd(p, R, th[0], th[1], th[2], th[3], th[4], crlb3);
}

void* orc_det_create(void* h, int SX, int SY, int R, double minZ, double maxZ, double step, double thr) {
    return det_build((const Psf*)h, SX, SY, R, minZ, maxZ, step, thr);
}
void orc_det_destroy(void* d) { delete (Detector*)d; }
int orc_det_nslices(void* d) { return ((Detector*)d)->nz; }
void orc_det_library(void* d, double* range, double* psfs) {
    Detector* D = (Detector*)d;
    for (int i = 0; i < D->nz; ++i) {
        range[i] = D->range[i];
        std::memcpy(psfs + (size_t)i * D->R * D->R, D->libpsf[i].data(), sizeof(double) * D->R * D->R);
    }
}
// Detect on nframes frames [f][X][Y]; out rows of 7 doubles, capacity cap per
// frame; counts[f] = number of candidates (may exceed cap: then truncated).
void orc_detect(void* d, int nframes, const double* frames, int cap, double* out, int* counts, int threads) {
    Detector* D = (Detector*)d;
    parallel_for(nframes, threads, [&](int f) {
        std::vector<std::array<double, 7>> rows;
        det_frame(D, frames + (size_t)f * D->SX * D->SY, rows);
        counts[f] = (int)rows.size();
        for (int k = 0; k < (int)rows.size() && k < cap; ++k)
            for (int c = 0; c < 7; ++c) out[((size_t)f * cap + k) * 7 + c] = rows[k][c];
    });
}

// Frame pipeline (LocalizationThread.run, LocalizationPipeline.java:720-990)
// with the reference coordinate-descent fit (iterMax 20, z clamp minZ-0.3 ..
// maxZ+0.3) and finite-difference CRLB.  det uses the resetKz library PSF,
// psf the fit PSF.  Rows: frame, x_nm, y_nm, z_nm, A, B, chi2, crlbx, crlby,
// crlbz (nm), in processing order per frame.
}  // extern "C"

namespace {

// LocalizationPipeline frame loop.  det_frames feed the detection, fit_frames
// the patches; vmap (SX x SY, nullable) is the sCMOS var/gain^2 map: getAandB
// then uses patch - v (:1168-1211), the fit and the model add v, and the
// Fisher matrix leaves it out (Localization.java:317-451).
//
// lmp (nullable): fit each candidate with the FP64 LM (lm_fit, the oracle of
// the library's own fit) instead of the reference coordinate descent, on the
// patch rounded to float as the library stages it; a fit is then used unless
// its model went non-positive.  Rows hold ncol values: 10, or 12 with the
// candidate's index in its frame's sorted candidate list and the LM status
// (1 converged, 2 evaluation cap, 3 stalled) last.
int localize_frames_impl(Detector* D, const Psf* p, int nframes, const double* det_frames, const double* fit_frames,
                         const double* vmap, double minZ, double maxZ, double photonThr, double maxSNR, int rows_cap,
                         double* rows, int threads, const LMParams* lmp = nullptr, int ncol = 10) {
    const int SX = D->SX, SY = D->SY, R = D->R, h = R / 2;
    std::vector<std::vector<std::array<double, 12>>> per(nframes);
    parallel_for(nframes, threads, [&](int f) {
        const double* img = fit_frames + (size_t)f * SX * SY;
        std::vector<std::array<double, 7>> v;
        det_frame(D, det_frames + (size_t)f * SX * SY, v);
        std::vector<char> mask((size_t)SX * SY, 0);
        std::vector<double> patch((size_t)R * R), psi((size_t)R * R), sv((size_t)R * R, 0.0);
        int pointer = 0;
        while (true) {
            int sel = -1;
            for (int i = pointer; i < (int)v.size(); ++i) {
                int ci = (int)std::lround(v[i][2]), cj = (int)std::lround(v[i][3]);
                if (mask[(size_t)ci * SY + cj]) continue;
                if (ci > R / 2 + 1 && cj > R / 2 + 1 && ci < SX - R / 2 - 1 && cj < SY - R / 2 - 1) { sel = i; pointer = i + 1; break; }
            }
            if (sel < 0) break;
            int r = (int)std::lround(v[sel][1]), ci = (int)std::lround(v[sel][2]), cj = (int)std::lround(v[sel][3]);
            bool treated = false;
            for (int a = 0; a < R && !treated; ++a)
                for (int b = 0; b < R; ++b) {
                    if (mask[(size_t)(ci - h + a) * SY + (cj - h + b)]) { treated = true; break; }
                    patch[(size_t)a * R + b] = img[(size_t)(ci - h + a) * SY + (cj - h + b)];
                    if (vmap) sv[(size_t)a * R + b] = vmap[(size_t)(ci - h + a) * SY + (cj - h + b)];
                }
            if (treated) continue;
            const std::vector<double>& lp = D->libpsf[r];  // getAandB (LocalizationPipeline.java:1119-1162)
            double maxp = -INFINITY, maxi = -INFINITY;
            for (int k = 0; k < R * R; ++k) { maxi = std::max(maxi, lp[k]); maxp = std::max(maxp, patch[k] - sv[k]); }
            double thr = maxi * 0.1, A = 0, B = 0, ca = 0, cb = 0;
            for (int k = 0; k < R * R; ++k) {
                if (lp[k] < thr) { B += patch[k] - sv[k]; cb++; } else { A += patch[k] - sv[k]; ca++; }
            }
            B = cb != 0 ? B / cb : 0;
            A -= ca * B;
            bool part = false;
            if (maxp / B > maxSNR && B > 0) {
                CD cd;
                cd.p = p; cd.R = R; cd.d = patch.data(); cd.v = vmap ? sv.data() : nullptr;
                cd.minZ = minZ - .3; cd.maxZ = maxZ + .3; cd.iterMax = 20; cd.photonThreshold = photonThr;
                cd.maxShift = p->dx / 2.;
                cd.psi.resize(R * R); cd.mu.resize(R * R);
                cd.ta = A; cd.tb = B; cd.tx = -v[sel][5]; cd.ty = -v[sel][6]; cd.tz = D->range[r] + v[sel][4];
                int st, lm_status = 0;
                if (lmp) {
                    std::vector<double> pf((size_t)R * R), vf;
                    for (int k = 0; k < R * R; ++k) pf[k] = (double)(float)patch[k];
                    if (vmap) {
                        vf.resize((size_t)R * R);
                        for (int k = 0; k < R * R; ++k) vf[k] = (double)(float)sv[k];
                    }
                    const double init[5] = {cd.tx, cd.ty, cd.tz, cd.ta, cd.tb};
                    double o[5], nll;
                    int ev;
                    lm_status = lm_fit(p, R, pf.data(), init, *lmp, o, &nll, &ev, nullptr, vmap ? vf.data() : nullptr);
                    st = lm_status != -1;
                    cd.tx = o[0]; cd.ty = o[1]; cd.tz = o[2]; cd.ta = o[3]; cd.tb = o[4];
                } else {
                    st = cd.run();
                }
                if (st == 1) {
                    psf_model(p, R, cd.tx, cd.ty, p->zfocus, cd.tz, psi.data(), nullptr);
                    double mthr = 0;
                    for (int k = 0; k < R * R; ++k) mthr = std::max(mthr, psi[k] * cd.ta + cd.tb + sv[k] - cd.tb);
                    mthr *= .2;
                    if (cd.ta > photonThr && std::fabs(cd.tx) < 10 * p->dx && std::fabs(cd.ty) < 10 * p->dx) {
                        int px = (int)(ci - (cd.tx / p->dx)), py = (int)(cj - (cd.ty / p->dx));
                        if (px >= 0 && px < SX && py >= 0 && py < SY && !mask[(size_t)px * SY + py] && cd.tz > minZ && cd.tz < maxZ) {
                            double chi = 0;
                            for (int k = 0; k < R * R; ++k) {
                                double mu = psi[k] * cd.ta + cd.tb + sv[k];
                                chi += (patch[k] - mu) * (patch[k] - mu) / mu;
                            }
                            chi /= (double)(R * R);
                            double cr[3];
                            fisher_crlb_fd(p, R, cd.tx, cd.ty, cd.tz, cd.ta, cd.tb, cr);
                            per[f].push_back({(double)f, 1000 * (ci * p->dx - cd.tx), 1000 * (cj * p->dx - cd.ty), 1000 * cd.tz,
                                              cd.ta, cd.tb, chi, 1000 * cr[0], 1000 * cr[1], 1000 * cr[2],
                                              (double)sel, (double)lm_status});
                            for (int a = 0; a < R; ++a)
                                for (int b = 0; b < R; ++b)
                                    if (psi[(size_t)a * R + b] * cd.ta + cd.tb + sv[(size_t)a * R + b] - cd.tb > mthr)
                                        mask[(size_t)(ci - h + a) * SY + (cj - h + b)] = 1;
                            part = true;
                        }
                    }
                }
            }
            if (!part)
                for (int a = 0; a < R; ++a)
                    for (int b = 0; b < R; ++b)
                        if (patch[(size_t)a * R + b] > maxp * .5) mask[(size_t)(ci - h + a) * SY + (cj - h + b)] = 1;
        }
    });
    int n = 0;
    for (int f = 0; f < nframes; ++f)
        for (auto& row : per[f]) {
            if (n < rows_cap)
                for (int c = 0; c < ncol; ++c) rows[(size_t)n * ncol + c] = row[c];
            ++n;
        }
    return n;
}

}  // namespace

extern "C" {

int orc_localize_frames(void* dh, void* ph, int nframes, const double* frames, double minZ, double maxZ,
                        double photonThr, double maxSNR, int rows_cap, double* rows, int threads) {
    return localize_frames_impl((Detector*)dh, (const Psf*)ph, nframes, frames, frames, nullptr, minZ, maxZ,
                                photonThr, maxSNR, rows_cap, rows, threads);
}

// The same frame loop with every candidate fitted by the FP64 LM of the
// library's fit (lm_fit): the oracle of zola_localize_frames.  params: max_iter
// evaluations and tol_xyz (um); the fit box and step caps as the library sets
// them (z in [minZ - 0.3, maxZ + 0.3], |x|, |y| <= 10 dx + 1e-3, steps dx and
// 2 dx).  Rows of 12: the 10 columns above, the candidate index and the LM status.
int orc_localize_frames_lm(void* dh, void* ph, int nframes, const double* frames, double minZ, double maxZ,
                           double photonThr, double maxSNR, int max_iter, double tol_xyz, int rows_cap, double* rows,
                           int threads) {
    const Psf* p = (const Psf*)ph;
    const LMParams P{minZ - 0.3, maxZ + 0.3, 10 * p->dx + 1e-3, max_iter, tol_xyz, p->dx, 2 * p->dx};
    return localize_frames_impl((Detector*)dh, p, nframes, frames, frames, nullptr, minZ, maxZ, photonThr, maxSNR,
                                rows_cap, rows, threads, &P, 12);
}

// sCMOS form (LocalizationPipeline.java:588-640): detection on
// (ADU - offset)/gain + vargain[0][0] clamped at 0, fits on
// (ADU - offset)/gain + vargain, vargain = variance / gain^2.
int orc_localize_frames_scmos(void* dh, void* ph, int nframes, const double* adu, const double* offset,
                              const double* gain, const double* variance, double minZ, double maxZ, double photonThr,
                              double maxSNR, int rows_cap, double* rows, int threads) {
    Detector* D = (Detector*)dh;
    const size_t SS = (size_t)D->SX * D->SY;
    std::vector<double> vg(SS), det(SS * nframes), fit(SS * nframes);
    for (size_t k = 0; k < SS; ++k) vg[k] = variance[k] / (gain[k] * gain[k]);
    for (int f = 0; f < nframes; ++f)
        for (size_t k = 0; k < SS; ++k) {
            const double c = (adu[(size_t)f * SS + k] - offset[k]) / gain[k];
            double dv = c + vg[0];
            det[(size_t)f * SS + k] = dv < 0 ? 0 : dv;
            fit[(size_t)f * SS + k] = c + vg[k];
        }
    return localize_frames_impl(D, (const Psf*)ph, nframes, det.data(), fit.data(), vg.data(), minZ, maxZ, photonThr,
                                maxSNR, rows_cap, rows, threads);
}

// Calibration stack NLL (ZernikePhaseRetrieval.java:1843-1874) for one bead:
// slices s at zoil = dz[s] + bz, zwat = 0; mu = A*psi + B clamped at 1e-8;
// NLL = sum mu - d ln mu.  Registration x/y/z enter as the kx, ky, kz_oil
// phase modes (ZernikePhaseRetrieval.java:93-95), i.e. as the coordinates.
double orc_calib_nll(void* h, int R, int nslice, const double* dz, const double* stack,
                     double bx, double by, double bz, double A, double B) {
    const Psf* p = (const Psf*)h;
    std::vector<double> psi(R * R);
    double nll = 0;
    for (int s = 0; s < nslice; ++s) {
        psf_model(p, R, bx, by, dz[s] + bz, 0.0, psi.data(), nullptr);
        for (int k = 0; k < R * R; ++k) {
            double mu = psi[k] * A + B;
            if (mu <= 0) mu = 0.00000001;
            nll += mu - stack[(size_t)s * R * R + k] * std::log(mu);
        }
    }
    return nll;
}


// Calibration stack NLL of one bead with the reference's full photometry
// (ZernikePhaseRetrieval.java:1843-1874, background :1519-1530):
//   mu = psi (A0_s + a_s) + sum_k c_k m_k(i, ii),  m = 1, i, i^2, ii, i ii, ii^2
// (PolynomialBackground, order 2, exponent digits of 0..8 in base 3), mu <= 0
// -> 1e-8; psi at (x, y, zoil = dz_s + z, zwat = 0) with blur width sigma.
double orc_calib_nll_full(void* h, int R, int nslice, const double* dz, const double* stack, const double* A0,
                          double sigma, double x, double y, double z, const double* a, const double* c) {
    Psf q = *(const Psf*)h;
    q.sigma = sigma;
    std::vector<double> psi(R * R);
    double nll = 0;
    for (int s = 0; s < nslice; ++s) {
        psf_model(&q, R, x, y, dz[s] + z, 0.0, psi.data(), nullptr);
        const double At = (A0 ? A0[s] : 0.0) + a[s];
        for (int i = 0; i < R; ++i)
            for (int ii = 0; ii < R; ++ii) {
                const double bg = c[0] + c[1] * i + c[2] * (double)i * i + c[3] * ii + c[4] * (double)i * ii +
                                  c[5] * (double)ii * ii;
                double mu = psi[i * R + ii] * At + bg;
                if (mu <= 0) mu = 0.00000001;
                nll += mu - stack[((size_t)s * R + i) * R + ii] * std::log(mu);
            }
    }
    return nll;
}

}  // extern "C"

namespace {

// Least squares of values v at (x, y) on the order-2 basis 1, x, x^2, y, xy, y^2
// by normal equations and Gaussian elimination (utils/PolynomialFit.java:80-140,
// 544-600); returns false when singular.
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
        for (int r = c + 1; r < 6; ++r) if (std::fabs(M[r][c]) > std::fabs(M[piv][c])) piv = r;
        if (M[piv][c] == 0) return false;
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

// InitBackgroundAndPhotonNumber (process/InitBackgroundAndPhotonNumber.java):
// ADU -> photons + 1 (:50-72), seed refinement (:587-640), the stack's
// polynomial background from low, dilated voxels around the dimmest slices
// (:642-900), per-bead background B, per-slice photons A (box-filtered over
// +-sizeFilt slices) and the bead patches (:110-420).  Image [slice][x][y].
int orc_calib_init(const double* raw, int ns, int W, int H, float* xp, float* yp, int nb, int sp, double adu,
                   double gain, double offset, double zstep, double* A, double* B, double* patches, double* poly) {
    const size_t N = (size_t)ns * W * H;
    std::vector<double> im(N);
    const double slope = adu / gain, intercept = -offset * adu / gain;
    for (size_t k = 0; k < N; ++k) {
        double v = (raw[k] * slope + intercept) + 1;
        im[k] = v < 0 ? 0 : v;
    }
    auto at = [&](int z, int i, int ii) { return im[((size_t)z * W + i) * H + ii]; };
    const int sizeFilt = std::max((int)(0.5 / zstep) / 2, 1);
    // refinePoints
    for (int p = 0; p < nb; ++p) {
        const int x0 = (int)(xp[p]) - sp / 2, y0 = (int)(yp[p]) - sp / 2;
        std::vector<double> sub((size_t)sp * sp, 0.0);
        for (int z = 0; z < ns; ++z)
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
            const float dxf = xp[p] - fx, dyf = yp[p] - fy;
            if (std::sqrt((double)(dxf * dxf)) < sp / 4) xp[p] = fx;
            if (std::sqrt((double)(dyf * dyf)) < sp / 4) yp[p] = fy;
        }
    }
    // computeBackground
    double mean0 = 0, std0 = 0;
    for (size_t k = 0; k < N; ++k) mean0 += im[k];
    mean0 /= (double)(int)N;
    for (size_t k = 0; k < N; ++k) std0 += (im[k] - mean0) * (im[k] - mean0);
    std0 /= (double)(int)N;
    std0 = std::sqrt(std0);
    double mean = 0, sd = 0;
    int cnt0 = 0;
    for (size_t k = 0; k < N; ++k)
        if (im[k] <= mean0 + 2 * std0) { mean += im[k]; cnt0++; }
    if (cnt0 > 0) mean /= cnt0;
    for (size_t k = 0; k < N; ++k)
        if (im[k] <= mean0 + 3 * std0) sd += (im[k] - mean) * (im[k] - mean);
    if (cnt0 > 0) { sd /= cnt0; sd = std::sqrt(sd); }
    std::vector<char> is2(N);
    for (size_t k = 0; k < N; ++k) is2[k] = im[k] > mean + 3 * sd ? 0 : 1;
    std::vector<double> mstack(ns, 0.0), filt(ns, 0.0);
    for (int z = 0; z < ns; ++z) {
        int c = 0;
        for (int i = 0; i < W; ++i)
            for (int ii = 0; ii < H; ++ii)
                if (is2[((size_t)z * W + i) * H + ii]) { mstack[z] += at(z, i, ii); c++; }
        if (c != 0) mstack[z] /= c;
    }
    int mp = 0;
    for (int z = 0; z < ns; ++z) {
        int c = 0;
        for (int u = -sizeFilt; u <= sizeFilt; ++u)
            if (z + u >= 0 && z + u < ns) { filt[z] += mstack[z + u]; c++; }
        if (c != 0) filt[z] /= c;
        if (filt[z] < filt[mp]) mp = z;
    }
    const int nn = sizeFilt;
    if (mp < nn) mp = nn;
    if (mp >= ns - nn) mp = ns - nn - 1;
    std::vector<double> px, py, pv;
    for (int i = 0; i < W; ++i)
        for (int ii = 0; ii < H; ++ii) {
            int count = 0;
            double m = 0;
            for (int z = 0; z < ns; ++z) {
                bool ok = !(z < mp - nn) && !(z > mp + nn);
                if (ok) {
                    for (int u = -2; u <= 2 && ok; ++u)
                        for (int uu = -2; uu <= 2 && ok; ++uu)
                            for (int uuu = -2; uuu <= 2 && ok; ++uuu)
                                if (z + u >= 0 && z + u < ns && i + uu >= 0 && i + uu < W && ii + uuu >= 0 &&
                                    ii + uuu < H && !is2[((size_t)(z + u) * W + i + uu) * H + ii + uuu])
                                    ok = false;
                }
                if (ok) { count++; m += at(z, i, ii); }
            }
            if (count >= 1) {
                px.push_back(i);
                py.push_back(ii);
                pv.push_back(m / count);
            }
        }
    double cf[6];
    if (!poly2_fit(px, py, pv, cf)) return -1;
    std::vector<double> pb((size_t)W * H);
    for (int i = 0; i < W; ++i)
        for (int ii = 0; ii < H; ++ii)
            pb[(size_t)i * H + ii] = cf[0] + cf[1] * i + cf[2] * std::pow((double)i, 2) + cf[3] * ii +
                                     cf[4] * i * (double)ii + cf[5] * std::pow((double)ii, 2);
    if (poly) std::memcpy(poly, pb.data(), pb.size() * 8);
    // B per bead, A per slice (box filtered), patches
    for (int p = 0; p < nb; ++p) {
        const int x0 = (int)(xp[p]) - sp / 2, y0 = (int)(yp[p]) - sp / 2;
        double b = 0, cb = 0;
        for (int u = 0; u < sp; ++u)
            for (int uu = 0; uu < sp; ++uu)
                if (x0 + u >= 0 && x0 + u < W && y0 + uu >= 0 && y0 + uu < H) { b += pb[(size_t)(x0 + u) * H + y0 + uu]; cb++; }
        if (cb >= 1) b /= cb;
        B[p] = b;
        std::vector<double> a(ns, 0.0);
        for (int z = 0; z < ns; ++z)
            for (int u = 0; u < sp; ++u)
                for (int uu = 0; uu < sp; ++uu)
                    if (x0 + u >= 0 && x0 + u < W && y0 + uu >= 0 && y0 + uu < H) a[z] += at(z, x0 + u, y0 + uu) - b;
        for (int z = 0; z < ns; ++z) {
            double m = 0, c = 0;
            for (int f = -sizeFilt; f <= sizeFilt; ++f)
                if (z + f >= 0 && z + f < ns) { m += a[z + f]; c++; }
            if (c >= 1) m /= c;
            A[(size_t)p * ns + z] = m;
        }
        for (int z = 0; z < ns; ++z)
            for (int u = 0; u < sp; ++u)
                for (int uu = 0; uu < sp; ++uu)
                    patches[(((size_t)p * ns + z) * sp + u) * sp + uu] =
                        (x0 + u >= 0 && x0 + u < W && y0 + uu >= 0 && y0 + uu < H) ? at(z, x0 + u, y0 + uu) : b;
    }
    return 0;
}


}  // extern "C"

namespace {

// In-place 3D FFT of a P0 x P1 x P2 complex cube (index [a][b][c]), 1-D passes
// along each axis (sign -1 forward, +1 inverse; unitary per pass).
void fft3d(std::vector<cplx>& v, int P0, int P1, int P2, int sign) {
    std::vector<cplx> line(std::max(P0, std::max(P1, P2)));
    for (int a = 0; a < P0; ++a)
        for (int b = 0; b < P1; ++b) fft1d(&v[((size_t)a * P1 + b) * P2], P2, sign);
    for (int a = 0; a < P0; ++a)
        for (int c = 0; c < P2; ++c) {
            for (int b = 0; b < P1; ++b) line[b] = v[((size_t)a * P1 + b) * P2 + c];
            fft1d(line.data(), P1, sign);
            for (int b = 0; b < P1; ++b) v[((size_t)a * P1 + b) * P2 + c] = line[b];
        }
    for (int b = 0; b < P1; ++b)
        for (int c = 0; c < P2; ++c) {
            for (int a = 0; a < P0; ++a) line[a] = v[((size_t)a * P1 + b) * P2 + c];
            fft1d(line.data(), P0, sign);
            for (int a = 0; a < P0; ++a) v[((size_t)a * P1 + b) * P2 + c] = line[a];
        }
}

// utils/GaussianElimination.java:107-140 (partial pivoting; exact-zero pivot = singular).
bool gauss_solve(std::vector<std::vector<double>> A, std::vector<double> b, std::vector<double>& x) {
    const int N = (int)b.size();
    for (int p = 0; p < N; ++p) {
        int mx = p;
        for (int i = p + 1; i < N; ++i) if (std::fabs(A[i][p]) > std::fabs(A[mx][p])) mx = i;
        std::swap(A[p], A[mx]);
        std::swap(b[p], b[mx]);
        if (std::fabs(A[p][p]) <= 0) return false;
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

// Interpolating polynomial through up to 4 points (utils/SplineFit.java's
// PolynomialFit windows), value and first derivative by Newton divided
// differences.
struct Cubic {
    int n = 0;
    double x[4], c[4];
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

// SplineFit (utils/SplineFit.java:24-75, 88-150, 195-250): cubic windows of 4
// consecutive knots, linear extrapolation with the end windows' slopes.
struct Spline {
    std::vector<double> x, y;
    std::vector<Cubic> pf;
    void fit(const std::vector<double>& xs, const std::vector<double>& ys) {
        x = xs; y = ys;
        for (size_t i = 0; i < x.size(); ++i)  // bubble sort as the reference
            for (size_t ii = 1; ii < x.size() - i; ++ii)
                if (x[ii] < x[ii - 1]) { std::swap(x[ii], x[ii - 1]); std::swap(y[ii], y[ii - 1]); }
        const int L = (int)x.size();
        pf.assign(std::max(1, L + 1 - 4), Cubic());
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

// LocalMaxima.run(threshold) (process/cpu/DriftCorrection.java:1084-1200) on a
// W0 x W1 x W2 float volume: centroid of the values above the threshold
// quantile in the 11^3 patch around the first maximum; returns the drift
// (-(c - size/2)) along the three indices.
void local_maxima(const std::vector<float>& im, int W0, int W1, int W2, double thr, double d[3]) {
    int s0 = std::min(11, W0 - 1), s1 = std::min(11, W1 - 1), s2 = std::min(11, W2 - 1);
    if (s0 % 2 == 0) s0--;
    if (s1 % 2 == 0) s1--;
    if (s2 % 2 == 0) s2--;
    s0 = std::max(s0, 1); s1 = std::max(s1, 1); s2 = std::max(s2, 1);  // one-voxel axes (the reference throws)
    double mx = 4.9e-324;  // Double.MIN_VALUE
    int a0 = 0, b0 = 0, c0 = 0;
    for (int i = 0; i < W0; ++i)
        for (int ii = 0; ii < W1; ++ii)
            for (int iii = 0; iii < W2; ++iii)
                if (mx < im[((size_t)i * W1 + ii) * W2 + iii]) { mx = im[((size_t)i * W1 + ii) * W2 + iii]; a0 = i; b0 = ii; c0 = iii; }
    std::vector<float> v;
    auto inb = [&](int i, int ii, int iii) {
        return i + a0 - s0 / 2 >= 0 && ii + b0 - s1 / 2 >= 0 && iii + c0 - s2 / 2 >= 0 && i + a0 - s0 / 2 < W0 &&
               ii + b0 - s1 / 2 < W1 && iii + c0 - s2 / 2 < W2;
    };
    auto val = [&](int i, int ii, int iii) {
        return im[((size_t)(i + a0 - s0 / 2) * W1 + (ii + b0 - s1 / 2)) * W2 + (iii + c0 - s2 / 2)];
    };
    for (int i = 0; i < s0; ++i)
        for (int ii = 0; ii < s1; ++ii)
            for (int iii = 0; iii < s2; ++iii)
                if (inb(i, ii, iii)) v.push_back(val(i, ii, iii));
    std::sort(v.begin(), v.end());
    const float t = v[(int)((v.size() - 1) * thr)];
    double x = 0, y = 0, z = 0, sum = 0;
    for (int i = 0; i < s0; ++i)
        for (int ii = 0; ii < s1; ++ii)
            for (int iii = 0; iii < s2; ++iii)
                if (inb(i, ii, iii) && val(i, ii, iii) > t) {
                    const double w = val(i, ii, iii);
                    sum += w;
                    x += (i + a0 - s0 / 2) * w;
                    y += (ii + b0 - s1 / 2) * w;
                    z += (iii + c0 - s2 / 2) * w;
                }
    x /= sum; y /= sum; z /= sum;
    d[0] = -(x - W0 / 2);
    d[1] = -(y - W1 / 2);
    d[2] = -(z - W2 / 2);
}

}  // namespace

extern "C" {

// DriftCorrection (process/cpu/DriftCorrection.java:125-410, 418-990): 3-D
// histograms of the localizations per time bin in half-overlapping windows of
// sizeFFT voxels (zero-padded to twice that), Gaussian-filtered in Fourier
// space, all-pairs cross-correlations summed over the windows, sub-voxel peak
// centroids, least-squares drift per bin relative to bin 0 with two passes of
// outlier rejection at the mean CRLB, and the SplineFit of the bin drifts at
// every localization's frame.  xyz / crlb in nm (crlb -1: unknown).
// bin_out: bins x 4 (frame index, dx, dy, dz nm); loc_out: n x 3.
int orc_drift(const double* xyz, const double* crlb, const int* frame, int n, double pixel_nm, int bin,
              double sub_um, double* bin_out, double* loc_out, double* px_used) {
    if (n < 1 || bin < 1) return -1;
    int sizeFFT = (int)std::pow(2, (int)std::ceil(std::log(sub_um / (pixel_nm / 1000.)) / std::log(2)));
    while (sizeFFT > 128) {
        pixel_nm *= 1.01;
        sizeFFT = (int)std::pow(2, (int)std::ceil(std::log(sub_um / (std::floor(pixel_nm + 0.5) / 1000.)) / std::log(2)));
    }
    pixel_nm = std::floor(pixel_nm + 0.5);
    if (px_used) *px_used = pixel_nm;
    const double DMIN = 4.9e-324, DMAX = 1.7976931348623157e308;
    double minX = DMAX, maxX = DMIN, minY = DMAX, maxY = DMIN, minZ = DMAX, maxZ = DMIN;
    int minF = 2147483647, maxF = -2147483647 - 1;
    double px = 0, py = 0, pz = 0;
    int cx = 0, cy = 0, cz = 0;
    for (int k = 0; k < n; ++k) {
        const double x = xyz[3 * k], y = xyz[3 * k + 1], z = xyz[3 * k + 2];
        const int f = frame[k];
        if (x < minX) minX = x;
        if (y < minY) minY = y;
        if (x > maxX) maxX = x;
        if (y > maxY) maxY = y;
        if (z < minZ) minZ = z;
        if (z > maxZ) maxZ = z;
        if (f < minF) minF = f;
        if (f > maxF) maxF = f;
        if (crlb) {
            if (crlb[3 * k] != -1) { px += crlb[3 * k]; cx++; }
            if (crlb[3 * k + 1] != -1) { py += crlb[3 * k + 1]; cy++; }
            if (crlb[3 * k + 2] != -1) { pz += crlb[3 * k + 2]; cz++; }
        }
    }
    px = cx == 0 ? 50 : px / cx;
    py = cy == 0 ? 50 : py / cy;
    pz = cz == 0 ? 50 : pz / cz;
    int width = std::max((int)std::ceil((maxX - minX) / pixel_nm), 1);
    int height = std::max((int)std::ceil((maxY - minY) / pixel_nm), 1);
    int depth = std::max((int)std::ceil((maxZ - minZ) / pixel_nm), 1);
    int sF[3] = {std::min(sizeFFT, width), std::min(sizeFFT, height), std::min(sizeFFT, depth)};
    for (int d = 0; d < 3; ++d) sF[d] = std::max(sF[d], (int)std::pow(2, std::ceil(std::log(sF[d]) / std::log(2))));
    const int ext[3] = {width, height, depth};
    int nb[3];
    for (int d = 0; d < 3; ++d)  // a one-voxel extent gives one window (the reference divides by zero there)
        nb[d] = sF[d] < 2 ? 1 : (int)std::ceil((double)(ext[d] - sF[d] / 2) / (double)(sF[d] / 2));
    const int P[3] = {2 * sF[0], 2 * sF[1], 2 * sF[2]};  // x, y, z
    const size_t PV = (size_t)P[0] * P[1] * P[2];
    // Fourier Gaussian, cube index [z][y][x], float-rounded (:290-320)
    const double sigma = 3 * std::max(std::max(px, py), pz) / pixel_nm;
    double sf2[3];
    for (int d = 0; d < 3; ++d) { const double v = (1. / sigma) * (double)P[d] / (M_PI * 2.); sf2[d] = v * v; }
    std::vector<float> gauss(PV);
    for (int xx = 0; xx < P[0]; ++xx)
        for (int yy = 0; yy < P[1]; ++yy)
            for (int zz = 0; zz < P[2]; ++zz) {
                const int xs = (xx + P[0] / 2) % P[0], ys = (yy + P[1] / 2) % P[1], zs = (zz + P[2] / 2) % P[2];
                const double dx = (xx - P[0] / 2.) * (xx - P[0] / 2.), dy = (yy - P[1] / 2.) * (yy - P[1] / 2.),
                             dz = (zz - P[2] / 2.) * (zz - P[2] / 2.);
                gauss[((size_t)zs * P[1] + ys) * P[0] + xs] = (float)std::exp(-.5 * (dx / sf2[0] + dy / sf2[1] + dz / sf2[2]));
            }
    std::vector<int> pos1, pos2;
    for (int t = 0; t < bin - 1; ++t)
        for (int s = t + 1; s < bin; ++s) { pos1.push_back(t); pos2.push_back(s); }
    const int tot = (int)pos1.size();
    const size_t RV = (size_t)sF[0] * sF[1] * sF[2];
    std::vector<float> result((size_t)tot * RV, 0.0f);
    std::vector<std::vector<cplx>> spec(bin, std::vector<cplx>(PV));
    std::vector<cplx> prod(PV), tmp(PV);
    for (int u = 0; u < nb[0]; ++u)
        for (int uu = 0; uu < nb[1]; ++uu)
            for (int uuu = 0; uuu < nb[2]; ++uuu) {
                const int uv[3] = {u, uu, uuu};
                double g0[3], g1[3];
                for (int d = 0; d < 3; ++d) {
                    g0[d] = (uv[d] / 2) * sF[d] * pixel_nm + (uv[d] % 2) * (sF[d] / 2) * pixel_nm;
                    g1[d] = (uv[d] / 2 + 1) * sF[d] * pixel_nm + (uv[d] % 2) * (sF[d] / 2) * pixel_nm;
                }
                std::vector<std::vector<double>> img(bin, std::vector<double>(PV, 0.0));
                for (int k = 0; k < n; ++k) {
                    const double x = xyz[3 * k] - minX, y = xyz[3 * k + 1] - minY, z = xyz[3 * k + 2] - minZ;
                    if (!(x >= g0[0] && x < g1[0] && y >= g0[1] && y < g1[1] && z >= g0[2] && z < g1[2])) continue;
                    const int idBin = bin * (frame[k] - minF) / (1 + maxF - minF);
                    const int xi = sF[0] / 2 + std::min(std::max((int)(std::fmod(x, sF[0] * pixel_nm) / pixel_nm), 0), sF[0] - 1);
                    const int yi = sF[1] / 2 + std::min(std::max((int)(std::fmod(y, sF[1] * pixel_nm) / pixel_nm), 0), sF[1] - 1);
                    const int zi = sF[2] / 2 + std::min(std::max((int)(std::fmod(z, sF[2] * pixel_nm) / pixel_nm), 0), sF[2] - 1);
                    img[idBin][((size_t)zi * P[1] + yi) * P[0] + xi] += 1;
                }
                for (int b = 0; b < bin; ++b) {  // Init: shift3D, FFT, Gaussian
                    for (int a = 0; a < P[2]; ++a)
                        for (int bb = 0; bb < P[1]; ++bb)
                            for (int c = 0; c < P[0]; ++c)
                                spec[b][((size_t)a * P[1] + bb) * P[0] + c] =
                                    cplx(img[b][((size_t)((a + P[2] / 2) % P[2]) * P[1] + (bb + P[1] / 2) % P[1]) * P[0] +
                                                (c + P[0] / 2) % P[0]], 0.0);
                    fft3d(spec[b], P[2], P[1], P[0], -1);
                    for (size_t k = 0; k < PV; ++k) spec[b][k] *= (double)gauss[k];
                }
                for (int id = 0; id < tot; ++id) {  // Process: F1 conj(F2), IFFT, shift3D, crop
                    const auto& F1 = spec[pos1[id]];
                    const auto& F2 = spec[pos2[id]];
                    for (size_t k = 0; k < PV; ++k) prod[k] = F1[k] * std::conj(F2[k]);
                    fft3d(prod, P[2], P[1], P[0], +1);
                    for (int a = 0; a < sF[2]; ++a)
                        for (int bb = 0; bb < sF[1]; ++bb)
                            for (int c = 0; c < sF[0]; ++c) {
                                const int as = (a + sF[2] / 2 + P[2] / 2) % P[2], bs = (bb + sF[1] / 2 + P[1] / 2) % P[1],
                                          cs = (c + sF[0] / 2 + P[0] / 2) % P[0];
                                result[(size_t)id * RV + ((size_t)a * sF[1] + bb) * sF[0] + c] +=
                                    (float)prod[((size_t)as * P[1] + bs) * P[0] + cs].real();
                            }
                }
            }
    const double fpb = ((double)(maxF - minF)) / ((double)bin);
    std::vector<double> di(bin, 0.0), dr[3];
    for (int d = 0; d < 3; ++d) dr[d].assign(bin, 0.0);
    di[0] = (double)minF + fpb / 2.;
    std::vector<std::vector<double>> Am(tot, std::vector<double>(std::max(bin - 1, 0), 0.0));
    std::vector<double> Rm[3];
    for (int d = 0; d < 3; ++d) Rm[d].assign(tot, 0.0);
    for (int id = 0; id < tot; ++id) {
        std::vector<float> vol(result.begin() + (size_t)id * RV, result.begin() + (size_t)(id + 1) * RV);
        double lm[3];  // along z, y, x indices
        local_maxima(vol, sF[2], sF[1], sF[0], .95, lm);
        const double drift[3] = {lm[2] * pixel_nm, lm[1] * pixel_nm, lm[0] * pixel_nm};
        const int t = pos1[id], s = pos2[id];
        if (t == 0) {
            di[s] = (((double)s) / ((double)bin)) * ((double)(1. + maxF - minF)) + ((double)minF) + (fpb / 2.);
            for (int d = 0; d < 3; ++d) dr[d][s] = drift[d];
        }
        for (int d = 0; d < 3; ++d) Rm[d][id] = drift[d];
        if (t != 0) Am[id][t - 1] = -1;
        Am[id][s - 1] = 1;
    }
    const double thr[3] = {px, py, pz};
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
                if (!gauss_solve(N, r, sol)) continue;
                for (size_t i = 0; i < An.size(); ++i) {
                    double fit = 0;
                    for (int a = 0; a < m; ++a) fit += An[i][a] * sol[a];
                    if (std::fabs(fit - Rn[i]) > thr[d]) del[d].push_back((int)i);
                }
                for (int a = 0; a < m; ++a) dr[d][a + 1] = sol[a];
            }
    }
    for (int b = 0; b < bin; ++b) {
        bin_out[4 * b] = di[b];
        for (int d = 0; d < 3; ++d) bin_out[4 * b + 1 + d] = dr[d][b];
    }
    if (loc_out) {
        Spline sp[3];
        for (int d = 0; d < 3; ++d) sp[d].fit(di, dr[d]);
        for (int k = 0; k < n; ++k)
            for (int d = 0; d < 3; ++d) loc_out[3 * k + d] = sp[d].eval((double)frame[k]);
    }
    return 0;
}

}  // extern "C"
