// rWW analytical feedback inhibition control (FIC), host and device.
//
// Reference: src/ext/models/rww.cpp:73-146 (prep_params) and
// src/ext/models/rww_fic.cpp:62-231 (analytical_fic_het, gsl_fsolve).  For each
// simulation and node j: the steady-state inhibitory current I_I solves
//     F(x) = I0_I + J_N,j S_E_ss - w_II gamma_I_s tau_I_s phi_I(x) - x = 0,   x in [0, 2]
// (phi_I(x) = (a_I x - b_I) / (1 - exp(-d_I (a_I x - b_I)))), then
//     S_I_ss = phi_I(I_I) tau_I_s gamma_I_s,
//     K_EE[j][k] = G SC[k][j] J_N,j (+ w_p,j J_N,j on the diagonal),
//     wIE_j = -(1 / S_I_ss) (I_E_ss - I_ext - I0_E - sum_k K_EE[j][k] S_E_ss).
// A root-finding failure or a negative wIE in any node marks the simulation
// unstable and sets wIE = 1 in all its nodes.
#pragma once
#include <cmath>
#include "engine.h"

namespace cbnm {

// Brent's method (Brent 1973) with the iteration of GSL 2.7's brent fsolver
// (gsl_root_fsolver_brent, the solver the reference calls in rww_fic.cpp:62-102)
// step for step: the same interpolation / bisection switch, tolerance
// 0.5 * DBL_EPSILON * |b| and bracket update, so that FIC parity holds.  Each
// iteration reports the bracket; the caller stops when |hi-lo| < 1e-3 *
// min(|lo|,|hi|) (0 if the bracket holds 0), at most 100 iterations, -1 on failure.
template <class F>
__host__ __device__ inline double brent_root(F f, double x_lo, double x_hi) {
    const double eps = 2.2204460492503131e-16;
    double a = x_lo, b = x_hi, fa = f(a), fb = f(b);
    if ((fa < 0.0 && fb < 0.0) || (fa > 0.0 && fb > 0.0)) return -1;
    double c = b, fc = fb, d = b - a, e = b - a, root = 0.5 * (x_lo + x_hi);
    for (int iter = 1; iter <= 100; ++iter) {
        bool lin = false;
        if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) { lin = true; c = a; fc = fa; d = b - a; e = b - a; }
        if (fabs(fc) < fabs(fb)) { lin = true; a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
        const double tol = 0.5 * eps * fabs(b), m = 0.5 * (c - b);
        double lo, hi;
        if (fb == 0) {
            root = b; lo = b; hi = b;
        } else if (fabs(m) <= tol) {
            root = b; lo = (b < c) ? b : c; hi = (b < c) ? c : b;
        } else {
            if (fabs(e) < tol || fabs(fa) <= fabs(fb)) {
                d = m; e = m;
            } else {
                double p, q, r, s = fb / fa;
                if (lin) { p = 2 * m * s; q = 1 - s; }
                else {
                    q = fa / fc; r = fb / fc;
                    p = s * (2 * m * q * (q - r) - (b - a) * (r - 1));
                    q = (q - 1) * (r - 1) * (s - 1);
                }
                if (p > 0) q = -q; else p = -p;
                const double t1 = 3 * m * q - fabs(tol * q), t2 = fabs(e * q);
                if (2 * p < ((t1 < t2) ? t1 : t2)) { e = d; d = p / q; }
                else { d = m; e = m; }
            }
            a = b; fa = fb;
            if (fabs(d) > tol) b += d; else b += (m > 0 ? +tol : -tol);
            fb = f(b);
            root = b;
            double cc = c;
            if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) cc = a;
            if (b < cc) { lo = b; hi = cc; } else { lo = cc; hi = b; }
        }
        const double alo = fabs(lo), ahi = fabs(hi);
        const double min_abs = ((lo > 0 && hi > 0) || (lo < 0 && hi < 0)) ? ((alo < ahi) ? alo : ahi) : 0.0;
        if (fabs(hi - lo) < 0.001 * min_abs) return root;
    }
    return -1;
}

// wIE of node j, or a negative value when the node fails (no root / wIE < 0).
// sc: the simulation's SC [k][j] (row = source); w_p_j, J_N_j: its regional params.
__host__ __device__ inline double rww_fic_node(const double *sc, int n, int j, double G, double w_p_j, double J_N_j,
                                              const RWWK &m) {
    const double I0_I = m.I_0 * m.w_I, I0_E = m.I_0 * m.w_E;
    const double a_I = 615, b_I = 177, d_I = 0.087;  // rww.cpp:19-21
    const double w_EE_j = w_p_j * J_N_j;
    auto phi_I = [&](double II) { return ((a_I * II) - b_I) / (1 - exp(-1 * d_I * ((a_I * II) - b_I))); };
    auto F = [&](double x) { return I0_I + J_N_j * m.S_E_ss - m.w_II * m.gamma_I_s * m.tau_I_s * phi_I(x) - x; };
    const double I_I = brent_root(F, 0.0, 2.0);
    if (I_I == -1) return -1.0;
    const double r_I = phi_I(I_I);
    const double S_I_ss = r_I * m.tau_I_s * m.gamma_I_s;
    double dot = 0.0;
    for (int k = 0; k < n; ++k) {
        double kee = (sc[(size_t)k * n + j] * G) * J_N_j;  // K_EE[j][k], SC transposed
        if (k == j) kee = kee + w_EE_j;
        dot += kee * m.S_E_ss;
    }
    const double w = (-1 / S_I_ss) * (m.I_E_ss - m.I_ext - I0_E - dot);
    return (w < 0) ? -1.0 : w;
}

}  // namespace cbnm
