// Node models of the per-simulation integrator, written once for both state
// precisions R = double (reference arithmetic) and R = float (FP32 mode).
//
// With R = double every expression keeps the reference's operation order
// (src/ext/models/<model>.cpp h_step); the file that instantiates it is
// compiled with --fmad=false, so results match the reference's double build.
// With R = float the constants are rounded to float once and the rate
// functions of rWW / rWWEx use expm1 (x / (1 - e^{-dx}) loses all its digits to
// cancellation near x = 0 in single precision).
//
// State layout per model: s[NS] state variables (type S) in the reference's
// order, iv[NI] intermediates (type R), r[NR] regional parameters (type P),
// CONN = the state that couples, BOLDV = the one that drives the
// Balloon-Windkessel model.  S = P = R except for Kuramoto, whose phase, initial
// phase, frequency and noise scale stay double in FP32 mode (only the coupling
// sum of sines is FP32): the phase itself drives the BOLD model and is wrapped
// by fmod(., 2 pi), so a float phase (ulp 4.8e-7 near 2 pi) or a float
// frequency (a drift of omega t 6e-8) moves wraps across samples, and the BOLD
// input by 2 pi there.
#pragma once
#include "engine.h"

namespace cbnm {

// x / (1 - exp(-d x)): rWW / rWWEx firing rate (rww.cpp:202-203, rwwex.cpp:62)
template <class R>
__device__ __forceinline__ R rate_of(R x, double d);
template <>
__device__ __forceinline__ double rate_of<double>(double x, double d) {
    return x / (1 - exp(-d * x));
}
template <>
__device__ __forceinline__ float rate_of<float>(float x, double d) {
    const float df = (float)d;
    const float y = -df * x;
    return (y == 0.0f) ? 1.0f / df : x / -expm1f(y);
}

template <class R>
struct RWWm {
    using S = R;
    using P = R;
    static constexpr int NS = 6, NI = 4, NN = 2, NG = 1, NR = 4, CONN = 4, BOLDV = 4;
    static constexpr bool OSC = false, POSTBW = true;
    __device__ static void init(S *s, R *, const R *, const P *) {
        s[0] = s[1] = s[2] = s[3] = R(0);
        s[4] = R(0.001); s[5] = R(0.001);
    }
    __device__ static void restart(S *s, R *, const P *) { s[4] = R(0.001); s[5] = R(0.001); }
    __device__ static void step(S *s, R *iv, const R *g, const P *r, R in, R n0, R n1, const ModelK &K) {  // rww.cpp:194-232
        const RWWK &m = K.rww;
        s[0] = R(m.w_E__I_0) + r[0] * r[1] * s[4] + in * g[0] * r[1] - r[2] * s[5];
        s[1] = R(m.w_I__I_0) + r[1] * s[4] - R(m.w_II) * s[5];
        iv[0] = R(m.a_E) * s[0] - R(m.b_E);
        iv[1] = R(m.a_I) * s[1] - R(m.b_I);
        s[2] = rate_of<R>(iv[0], m.d_E);
        s[3] = rate_of<R>(iv[1], m.d_I);
        iv[2] = n0 * r[3] * R(m.sqrt_dt) + R(m.dt_gamma_E) * ((R(1) - s[4]) * s[2]) - R(m.dt_itau_E) * s[4];
        iv[3] = n1 * r[3] * R(m.sqrt_dt) + R(m.dt_gamma_I) * s[3] - R(m.dt_itau_I) * s[5];
        s[4] += iv[2];
        s[5] += iv[3];
        s[4] = fmax(R(0), fmin(R(1), s[4]));
        s[5] = fmax(R(0), fmin(R(1), s[5]));
    }
};

template <class R>
struct WCm {
    using S = R;
    using P = R;
    static constexpr int NS = 2, NI = 4, NN = 2, NG = 1, NR = 8, CONN = 0, BOLDV = 0;
    static constexpr bool OSC = false, POSTBW = false;
    __device__ static void init(S *s, R *, const R *, const P *) { s[0] = R(0.001); s[1] = R(0.001); }
    __device__ static void restart(S *s, R *, const P *) { s[0] = R(0.001); s[1] = R(0.001); }
    __device__ static void step(S *s, R *iv, const R *g, const P *r, R in, R n0, R n1, const ModelK &K) {  // wc.cpp:51-80
        const WCK &m = K.wc;
        iv[0] = R(1) / (R(1) + exp(-R(m.a_E) * (r[0] * s[0] - r[1] * s[1] + g[0] * in + r[4] - R(m.mu_E))));
        iv[1] = R(1) / (R(1) + exp(-R(m.a_I) * (r[2] * s[0] - r[3] * s[1] + r[5] - R(m.mu_I))));
        iv[2] = (-s[0] + (R(1) - s[0]) * iv[0]) * R(m.itau_E);
        iv[3] = (-s[1] + (R(1) - s[1]) * iv[1]) * R(m.itau_I);
        s[0] += R(m.dt) * iv[2] + R(m.sqrt_dt) * n0 * r[6];
        s[1] += R(m.dt) * iv[3] + R(m.sqrt_dt) * n1 * r[7];
        s[0] = fmax(R(0), fmin(R(1), s[0]));
        s[1] = fmax(R(0), fmin(R(1), s[1]));
    }
};

template <class R>
struct JRm {
    using S = R;
    using P = R;
    static constexpr int NS = 8, NI = 9, NN = 1, NG = 1, NR = 6, CONN = 7, BOLDV = 6;
    static constexpr bool OSC = false, POSTBW = false;
    __device__ static void init(S *s, R *, const R *, const P *) {
        for (int i = 0; i < 8; ++i) s[i] = R(0);
    }
    __device__ static void restart(S *s, R *, const P *) { for (int i = 0; i < 8; ++i) s[i] = R(0); }
    __device__ static void step(S *s, R *iv, const R *g, const P *r, R in, R n0, R, const ModelK &K) {  // jr.cpp:80-133
        const JRK &m = K.jr;
        iv[0] = R(2) * R(m.nu_max) / (R(1) + exp(R(m.r) * (R(m.v0) - (s[1] - s[2]))));
        iv[1] = R(2) * R(m.nu_max) / (R(1) + exp(R(m.r) * (R(m.v0) - (r[1] * r[0] * s[0]))));
        iv[2] = R(2) * R(m.nu_max) / (R(1) + exp(R(m.r) * (R(m.v0) - (r[3] * r[0] * s[0]))));
        iv[3] = s[3];
        iv[4] = s[4];
        iv[5] = s[5];
        iv[6] = R(m.A) * R(m.a) * iv[0] - R(2) * R(m.a) * s[3] - R(m.a_sq) * s[0];
        iv[7] = R(m.A) * R(m.a) * (R(m.mu) + r[2] * r[0] * iv[1] + g[0] * in) - R(2) * R(m.a) * s[4] - R(m.a_sq) * s[1];
        iv[8] = R(m.B) * R(m.b) * (r[4] * r[0] * iv[2]) - R(2) * R(m.b) * s[5] - R(m.b_sq) * s[2];
        s[0] += R(m.dt) * iv[3];
        s[1] += R(m.dt) * iv[4];
        s[2] += R(m.dt) * iv[5];
        s[3] += R(m.dt) * iv[6] + R(m.sqrt_dt) * n0 * r[5];
        s[4] += R(m.dt) * iv[7];
        s[5] += R(m.dt) * iv[8];
        s[6] = s[1] - s[2];
        s[7] = R(m.cmin) + (R(m.cmax) - R(m.cmin)) / (R(1) + exp(R(m.r) * (R(m.midpoint) - (s[6]))));
    }
};

template <class R>
struct Kuramotom {
    using S = double;
    using P = double;
    static constexpr int NS = 1, NI = 1, NN = 1, NG = 1, NR = 3, CONN = 0, BOLDV = 0;
    static constexpr bool OSC = true, POSTBW = false;
    __device__ static void init(S *s, R *, const R *, const P *r) { s[0] = S(r[0]); }
    __device__ static void restart(S *s, R *, const P *r) { s[0] = S(r[0]); }
    __device__ static void step(S *s, R *iv, const R *g, const P *r, R in, R n0, R, const ModelK &K) {  // kuramoto.cpp:48-61
        const KurK &m = K.kur;
        const S w = r[1] + S(g[0] * in);  // instantaneous frequency, in double
        iv[0] = R(w);
        s[0] = s[0] + m.dt * w + m.sqrt_dt * S(n0) * r[2];
        s[0] = fmod(s[0], m.twopi);
    }
};

template <class R>
struct RWWExm {
    using S = R;
    using P = R;
    static constexpr int NS = 3, NI = 2, NN = 1, NG = 1, NR = 3, CONN = 2, BOLDV = 2;
    static constexpr bool OSC = false, POSTBW = false;
    __device__ static void init(S *s, R *, const R *, const P *) { s[0] = s[1] = R(0); s[2] = R(0.001); }
    __device__ static void restart(S *s, R *, const P *) { s[2] = R(0.001); }
    __device__ static void step(S *s, R *iv, const R *g, const P *r, R in, R n0, R, const ModelK &K) {  // rwwex.cpp:48-73
        const RWWExK &m = K.rwwex;
        s[0] = r[0] * R(m.J_N) * s[2] + g[0] * R(m.J_N) * in + r[1];
        iv[0] = R(m.a) * s[0] - R(m.b);
        s[1] = rate_of<R>(iv[0], m.d);
        iv[1] = R(m.dt_gamma) * ((R(1) - s[2]) * s[1]) - R(m.dt_itau) * s[2] + n0 * R(m.sqrt_dt) * r[2];
        s[2] += iv[1];
        s[2] = fmax(R(0), fmin(R(1), s[2]));
    }
};

}  // namespace cbnm
