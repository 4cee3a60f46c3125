// Tangent-linear (forward-mode) steps along the global coupling G: the node
// state s and its derivative ds = ds/dG advance together.  The value part is
// the model's own FP32 step (models.cuh), so a tangent run produces the same
// state and BOLD as the plain FP32 run; the derivative part is the step
// differentiated by hand (rWW: rww.cpp:194-232; WC: wc.cpp:51-80;
// Balloon-Windkessel: bw.cu:4-15):
//
//   rWW  dI_E = w_p J_N dS_E + J_N (in + G din) - wIE dS_I,  dI_I = J_N dS_E - w_II dS_I
//        dr   = r'(a I - b) a dI,  r(x) = x / (1 - e^{-d x}),  r' = (D - d x e) / D^2 (D = 1 - e, e = e^{-d x};
//               1/2 + d x / 6 near 0)
//        dS_E += dt gamma_E ((1 - S_E) dr_E - r_E dS_E) - dt / tau_E dS_E,  dS_I += dt gamma_I dr_I - dt / tau_I dS_I
//   WC   dz_E = c_EE dE - c_IE dI + in + G din,  dz_I = c_EI dE - c_II dI
//        dsig = a sig (1 - sig) dz
//        dE  += dt itau_E (-dE - sig_E dE + (1 - E) dsig_E),  dI likewise
//   both: the derivative of a state clamped to 0 or 1 in this step is 0.
// din is the coupling of the derivatives, sum_k SC[k][j] dx_k(t - d_kj); the
// noise does not depend on G.
#pragma once
#include "engine.h"
#include "models.cuh"

namespace cbnm {

template <class M>
struct Tangent {  // no tangent for this model
    static constexpr bool OK = false;
    static constexpr int NT = 1;
    static constexpr int CONN_T = 0;
    __device__ static void step(float *, float *, float *, const float *, const float *, float, float, float, float,
                                const ModelK &) {}
};

__device__ __forceinline__ float rate_deriv_f(float x, float df) {
    const float u = df * x;
    if (fabsf(u) < 1e-2f) return 0.5f + u * (1.0f / 6.0f);
    const float e = expf(-u), den = -expm1f(-u);
    return (den - u * e) / (den * den);
}

template <>
struct Tangent<RWWm<float>> {
    static constexpr bool OK = true;
    static constexpr int NT = 2;   // tangents of S_E, S_I
    static constexpr int CONN_T = 0;
    using M = RWWm<float>;
    __device__ static void step(float *s, float *ds, float *iv, const float *g, const float *r, float in, float din,
                                float n0, float n1, const ModelK &K) {
        const RWWK &m = K.rww;
        const float SE = s[4], SI = s[5], dSE = ds[0], dSI = ds[1];
        const float IE = float(m.w_E__I_0) + r[0] * r[1] * SE + in * g[0] * r[1] - r[2] * SI;
        const float II = float(m.w_I__I_0) + r[1] * SE - float(m.w_II) * SI;
        const float xE = float(m.a_E) * IE - float(m.b_E), xI = float(m.a_I) * II - float(m.b_I);
        const float rE = rate_of<float>(xE, m.d_E), rI = rate_of<float>(xI, m.d_I);
        const float dIE = r[0] * r[1] * dSE + r[1] * (in + g[0] * din) - r[2] * dSI;
        const float dII = r[1] * dSE - float(m.w_II) * dSI;
        const float drE = rate_deriv_f(xE, float(m.d_E)) * float(m.a_E) * dIE;
        const float drI = rate_deriv_f(xI, float(m.d_I)) * float(m.a_I) * dII;
        const float nE = dSE + float(m.dt_gamma_E) * ((1.0f - SE) * drE - rE * dSE) - float(m.dt_itau_E) * dSE;
        const float nI = dSI + float(m.dt_gamma_I) * drI - float(m.dt_itau_I) * dSI;
        M::step(s, iv, g, r, in, n0, n1, K);
        ds[0] = (s[4] > 0.0f && s[4] < 1.0f) ? nE : 0.0f;
        ds[1] = (s[5] > 0.0f && s[5] < 1.0f) ? nI : 0.0f;
    }
};

template <>
struct Tangent<WCm<float>> {
    static constexpr bool OK = true;
    static constexpr int NT = 2;   // tangents of E, I
    static constexpr int CONN_T = 0;
    using M = WCm<float>;
    __device__ static void step(float *s, float *ds, float *iv, const float *g, const float *r, float in, float din,
                                float n0, float n1, const ModelK &K) {
        const WCK &m = K.wc;
        const float E = s[0], I = s[1], dE = ds[0], dI = ds[1];
        const float sE = 1.0f / (1.0f + expf(-float(m.a_E) * (r[0] * E - r[1] * I + g[0] * in + r[4] - float(m.mu_E))));
        const float sI = 1.0f / (1.0f + expf(-float(m.a_I) * (r[2] * E - r[3] * I + r[5] - float(m.mu_I))));
        const float dsE = float(m.a_E) * sE * (1.0f - sE) * (r[0] * dE - r[1] * dI + in + g[0] * din);
        const float dsI = float(m.a_I) * sI * (1.0f - sI) * (r[2] * dE - r[3] * dI);
        const float nE = dE + float(m.dt) * float(m.itau_E) * (-dE - sE * dE + (1.0f - E) * dsE);
        const float nI = dI + float(m.dt) * float(m.itau_I) * (-dI - sI * dI + (1.0f - I) * dsI);
        M::step(s, iv, g, r, in, n0, n1, K);
        ds[0] = (s[0] > 0.0f && s[0] < 1.0f) ? nE : 0.0f;
        ds[1] = (s[1] > 0.0f && s[1] < 1.0f) ? nI : 0.0f;
    }
};

// Tangent of the FP64 Balloon-Windkessel step (bw.cu:4-15; q uses the updated nu):
//   dx' = dx + dt (dz - kappa dx - y df),  df' = df + dt dx'  (f advances with the new x),
//   dnu' = dnu + dt/tau (df - (1/alpha) nu^(1/alpha - 1) dnu),
//   dq' = dq + dt/tau ([1 - E + E ln(1 - rho) / f] / rho df - (1/alpha - 1) nu'^(1/alpha - 2) q dnu'
//         - nu'^(1/alpha - 1) dq),  E = (1 - rho)^(1/f),
// then the value step itself.  Powers by exp2 / log2 (the derivative path needs
// no more than double precision's last few bits).
__device__ __forceinline__ void bw_tangent64(double x, double f, double nu, double q, double &dx, double &df, double &dnu,
                                             double &dq, double dz, const BWFast &c) {
    const double ct = c.dt_itau;
    const double a1 = c.ialpha - 1.0;
    const double dx1 = dx + c.dt * (dz - c.kappa * dx - c.y * df);
    const double df1 = df + c.dt * dx1;
    const double nua = exp2(c.ialpha * log2(nu));                  // nu^(1/alpha)
    const double nu1 = nu + ct * (f - nua);
    const double dnu1 = dnu + ct * (df - c.ialpha * nua / nu * dnu);
    const double nu1a1 = exp2(a1 * log2(nu1));                     // nu'^(1/alpha - 1)
    const double E = exp2(c.log2_omr / f);                         // (1 - rho)^(1/f)
    const double dq1 = dq + ct * ((1.0 - E + E * c.ln_omr / f) * c.irho * df - a1 * nu1a1 / nu1 * q * dnu1 - nu1a1 * dq);
    dx = dx1;
    df = df1;
    dnu = dnu1;
    dq = dq1;
}

}  // namespace cbnm
