// Levenberg-Marquardt state machine for the 5-parameter Poisson MLE
// (theta = x, y, z in um; A photons; B photons/px), in FP64.
//
// The reference fits by cyclic finite-difference Newton steps per coordinate
// (process/cpu/Localization.java:491-1058).  This library fits the same Poisson
// likelihood (Localization.java:1125-1143) with a damped Gauss-Newton step on
// analytic gradients; both reach the same optimum (the coordinate descent stops
// once the x/y/z move per sweep is below 0.1 nm).  The FP64 and split-precision
// kernels share this code, so they differ only in how the model is computed.
//
// Per evaluation the kernels supply, at the trial point:
//   nll = sum mu - d - d ln(mu/d)  (mu for d = 0), +inf if any mu <= 0
//   g   = sum (1 - d/mu) J,   H = sum d/mu^2 J J^T,   F = sum J J^T / mu
// with J = dmu/dtheta = (A dpsi/dx, A dpsi/dy, A dpsi/dz, psi, 1).
#pragma once

#include "zola_internal.h"

namespace zola {

struct LMState {
    double th[5];      // accepted point
    double g[5];
    double H[25];
    double F[25];      // Fisher matrix at the accepted point (for the CRLB)
    double nll;
    double lambda;
    double trial[5];   // proposed point
    double step;       // max |trial - th| over x, y, z
    double pred;       // decrease of the likelihood the quadratic model predicts for the trial step
    int evals;
    int status;        // 2 running, 1 converged, 3 stalled, -1 NaN / non-positive model
};

__host__ __device__ inline void lm_clamp(double* t, const FitParamsDev& P) {
    t[0] = fmin(fmax(t[0], -P.xymax), P.xymax);
    t[1] = fmin(fmax(t[1], -P.xymax), P.xymax);
    t[2] = fmin(fmax(t[2], P.zmin), P.zmax);
    t[3] = fmax(t[3], 1.0);
    t[4] = fmax(t[4], 0.01);
}

// Damping floors (units 1/um^2 for x, y, z; 1/photon^2 for A and B): the
// Marquardt term lambda * max(H_ii, floor_i) stays positive where a
// derivative vanishes by symmetry (e.g. d mu / dz at x = y = z = 0 for an
// odd aberration), so the damped system can always be solved.
__host__ __device__ inline double lm_floor(int i) {
    return i < 3 ? 1.0 : (i == 3 ? 1e-10 : 1e-6);
}

// Cholesky solve of (H + lambda max(diag H, floor)) delta = -g.
__host__ __device__ inline bool lm_solve(const double* H, const double* g, double lambda, double* delta) {
    double L[5][5];
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) L[i][j] = 0.0;
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j <= i; ++j) {
            double s = H[i * 5 + j] + (i == j ? lambda * fmax(H[i * 5 + i], lm_floor(i)) : 0.0);
            for (int k = 0; k < j; ++k) s -= L[i][k] * L[j][k];
            if (i == j) {
                if (!(s > 0.0)) return false;
                L[i][i] = sqrt(s);
            } else {
                L[i][j] = s / L[j][j];
            }
        }
    double y[5];
    for (int i = 0; i < 5; ++i) {
        double s = -g[i];
        for (int k = 0; k < i; ++k) s -= L[i][k] * y[k];
        y[i] = s / L[i][i];
    }
    for (int i = 4; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < 5; ++k) s -= L[k][i] * delta[k];
        delta[i] = s / L[i][i];
    }
    return true;
}

// Convergence test at an accepted point: the undamped Gauss-Newton step
// -H^-1 g (the distance to the optimum of the local quadratic model) moves
// x, y and z by less than tol and A, B by less than 1e-4 of their values.
// Damped steps shrink with lambda on flat likelihoods, so their size alone is
// not a distance to the optimum.
__host__ __device__ inline bool lm_at_optimum(const LMState& s, const FitParamsDev& P) {
    double d[5];
    if (!lm_solve(s.H, s.g, 0.0, d)) return false;
    return fmax(fabs(d[0]), fmax(fabs(d[1]), fabs(d[2]))) < P.tol_xyz && fabs(d[3]) < 1e-4 * s.th[3] &&
           fabs(d[4]) < 1e-4 * fmax(s.th[4], 1.0);
}

// First evaluation result at the (clamped) initial point.
__host__ __device__ inline void lm_start(LMState& s, double nll, const double* g, const double* H, const double* F,
                                         const FitParamsDev& P) {
    s.nll = nll;
    for (int q = 0; q < 5; ++q) s.g[q] = g[q];
    for (int q = 0; q < 25; ++q) { s.H[q] = H[q]; s.F[q] = F[q]; }
    s.evals = 1;
    s.lambda = 1e-3;
    s.status = isfinite(nll) ? 2 : -1;
    if (s.status == 2 && lm_at_optimum(s, P)) s.status = 1;
}

// Propose the next trial point.  Returns false when the fit is finished.
__host__ __device__ inline bool lm_propose(LMState& s, const FitParamsDev& P) {
    while (s.status == 2 && s.evals < P.max_iter) {
        double d[5];
        if (!lm_solve(s.H, s.g, s.lambda, d)) {
            s.lambda *= 10.0;
            if (s.lambda > 1e7) s.status = 3;
            continue;
        }
        double sxy = fmax(fabs(d[0]), fabs(d[1]));
        double scale = 1.0;
        if (sxy > P.step_xy) scale = P.step_xy / sxy;
        if (fabs(d[2]) * scale > P.step_z) scale = P.step_z / fabs(d[2]);
        for (int q = 0; q < 5; ++q) s.trial[q] = s.th[q] + scale * d[q];
        lm_clamp(s.trial, P);
        s.step = fmax(fabs(s.trial[0] - s.th[0]), fmax(fabs(s.trial[1] - s.th[1]), fabs(s.trial[2] - s.th[2])));
        double dl[5], hd = 0, gd = 0;
        for (int q = 0; q < 5; ++q) dl[q] = s.trial[q] - s.th[q];
        for (int q = 0; q < 5; ++q) {
            gd += s.g[q] * dl[q];
            for (int r = 0; r < 5; ++r) hd += dl[q] * s.H[q * 5 + r] * dl[r];
        }
        s.pred = -(gd + 0.5 * hd);
        return true;
    }
    if (s.status == 2) s.status = 2;  // max evaluations reached: stays "max iter"
    return false;
}

// Accept or reject the evaluated trial point.  Near the optimum of a flat
// likelihood (a faint or defocused emitter) the decrease of the last steps is
// below the rounding of a likelihood summed in FP32.  So when the quadratic
// model predicts a decrease of at most P.accept_nll, the step is accepted
// unless the likelihood rose by more than that; the next Gauss-Newton step
// from the accepted point decides convergence.  (P.accept_nll = 0: a step is
// accepted only when the likelihood did not rise.)
__host__ __device__ inline void lm_update(LMState& s, double nll, const double* g, const double* H, const double* F,
                                          const FitParamsDev& P) {
    s.evals += 1;
    if (nll <= s.nll || (s.pred <= P.accept_nll && nll <= s.nll + P.accept_nll)) {
        for (int q = 0; q < 5; ++q) { s.th[q] = s.trial[q]; s.g[q] = g[q]; }
        for (int q = 0; q < 25; ++q) { s.H[q] = H[q]; s.F[q] = F[q]; }
        s.nll = nll;
        s.lambda = fmax(s.lambda * 0.1, 1e-7);
        if (lm_at_optimum(s, P)) s.status = 1;
    } else {
        s.lambda *= 10.0;
        if (s.lambda > 1e7) s.status = 3;
    }
}

// CRLB = sqrt(diag(F^-1)) for all five parameters (NaN if F is singular).
__host__ __device__ inline void lm_crlb(const double* F, double* crlb) {
    for (int c = 0; c < 5; ++c) {
        double rhs[5] = {0, 0, 0, 0, 0}, col[5];
        rhs[c] = -1.0;  // lm_solve solves A x = -rhs
        if (lm_solve(F, rhs, 0.0, col)) crlb[c] = sqrt(col[c]);
        else crlb[c] = NAN;
    }
}

}  // namespace zola
