// FP64 integrator: the reference-precision path (the "plain" GPU method).
//
// One CTA per simulation, one thread per node, everything in FP64, so that its
// output matches the reference's double build on the same noise.  This file is
// compiled with --fmad=false: every multiply and add rounds separately, in the
// same order as the reference's C++ (src/ext/models/<model>.cpp h_step,
// src/ext/models/bw.cpp:24-35), so the only differences left are the last-ulp
// differences between CUDA's and glibc's exp/pow/sin.
//
// Time loop: src/ext/bnm.cu:117-505 (GPU) and src/ext/bnm.cpp:69-522 (CPU);
// coupling: bnm.cu:48-101; numerical FIC: src/ext/models/rww.cpp:233-298.
#include <cstdint>
#include "engine.h"

namespace cbnm {
namespace {

// ---------------------------------------------------------------- models (FP64)
struct RWW {
    static constexpr int NS = 6, NI = 7, NN = 2, NG = 1, NR = 4, CONN = 4, BOLDV = 4;
    static constexpr bool OSC = false, POSTBW = true;
    __device__ static void init(double *s, double *iv, const double *, const double *, const IntegrateArgs &a) {
        s[0] = s[1] = s[2] = s[3] = 0.0;
        s[4] = 0.001; s[5] = 0.001; iv[4] = 0.0; iv[5] = a.init_delta; iv[6] = 0.0;
    }
    __device__ static void restart(double *s, double *iv, const double *) { s[4] = 0.001; s[5] = 0.001; iv[4] = 0.0; }
    __device__ static void step(double *s, double *iv, const double *g, const double *r, double in, double n0, double n1,
                                const ModelK &K) {  // rww.cpp:194-232
        const RWWK &m = K.rww;
        s[0] = m.w_E__I_0 + r[0] * r[1] * s[4] + in * g[0] * r[1] - r[2] * s[5];
        s[1] = m.w_I__I_0 + r[1] * s[4] - m.w_II * s[5];
        iv[0] = m.a_E * s[0] - m.b_E;
        iv[1] = m.a_I * s[1] - m.b_I;
        s[2] = iv[0] / (1 - exp(-m.d_E * iv[0]));
        s[3] = iv[1] / (1 - exp(-m.d_I * iv[1]));
        iv[2] = n0 * r[3] * m.sqrt_dt + m.dt_gamma_E * ((1 - s[4]) * s[2]) - m.dt_itau_E * s[4];
        iv[3] = n1 * r[3] * m.sqrt_dt + m.dt_gamma_I * s[3] - m.dt_itau_I * s[5];
        s[4] += iv[2];
        s[5] += iv[3];
        s[4] = fmax(0.0, fmin(1.0, s[4]));
        s[5] = fmax(0.0, fmin(1.0, s[5]));
    }
};

struct WC {
    static constexpr int NS = 2, NI = 4, NN = 2, NG = 1, NR = 8, CONN = 0, BOLDV = 0;
    static constexpr bool OSC = false, POSTBW = false;
    __device__ static void init(double *s, double *, const double *, const double *, const IntegrateArgs &) { s[0] = 0.001; s[1] = 0.001; }
    __device__ static void restart(double *s, double *, const double *) { s[0] = 0.001; s[1] = 0.001; }
    __device__ static void step(double *s, double *iv, const double *g, const double *r, double in, double n0, double n1,
                                const ModelK &K) {  // wc.cpp:51-80
        const WCK &m = K.wc;
        iv[0] = 1.0 / (1.0 + exp(-m.a_E * (r[0] * s[0] - r[1] * s[1] + g[0] * in + r[4] - m.mu_E)));
        iv[1] = 1.0 / (1.0 + exp(-m.a_I * (r[2] * s[0] - r[3] * s[1] + r[5] - m.mu_I)));
        iv[2] = (-s[0] + (1.0 - s[0]) * iv[0]) * m.itau_E;
        iv[3] = (-s[1] + (1.0 - s[1]) * iv[1]) * m.itau_I;
        s[0] += m.dt * iv[2] + m.sqrt_dt * n0 * r[6];
        s[1] += m.dt * iv[3] + m.sqrt_dt * n1 * r[7];
        s[0] = fmax(0.0, fmin(1.0, s[0]));
        s[1] = fmax(0.0, fmin(1.0, s[1]));
    }
};

struct JR {
    static constexpr int NS = 8, NI = 9, NN = 1, NG = 1, NR = 6, CONN = 7, BOLDV = 6;
    static constexpr bool OSC = false, POSTBW = false;
    __device__ static void init(double *s, double *, const double *, const double *, const IntegrateArgs &) {
        for (int i = 0; i < 8; ++i) s[i] = 0.0;
    }
    __device__ static void restart(double *s, double *, const double *) { for (int i = 0; i < 8; ++i) s[i] = 0.0; }
    __device__ static void step(double *s, double *iv, const double *g, const double *r, double in, double n0, double,
                                const ModelK &K) {  // jr.cpp:80-133
        const JRK &m = K.jr;
        iv[0] = 2.0 * m.nu_max / (1.0 + exp(m.r * (m.v0 - (s[1] - s[2]))));
        iv[1] = 2.0 * m.nu_max / (1.0 + exp(m.r * (m.v0 - (r[1] * r[0] * s[0]))));
        iv[2] = 2.0 * m.nu_max / (1.0 + exp(m.r * (m.v0 - (r[3] * r[0] * s[0]))));
        iv[3] = s[3];
        iv[4] = s[4];
        iv[5] = s[5];
        iv[6] = m.A * m.a * iv[0] - 2.0 * m.a * s[3] - (m.a_sq) * s[0];
        iv[7] = m.A * m.a * (m.mu + r[2] * r[0] * iv[1] + g[0] * in) - 2.0 * m.a * s[4] - (m.a_sq) * s[1];
        iv[8] = m.B * m.b * (r[4] * r[0] * iv[2]) - 2.0 * m.b * s[5] - (m.b_sq) * s[2];
        s[0] += m.dt * iv[3];
        s[1] += m.dt * iv[4];
        s[2] += m.dt * iv[5];
        s[3] += m.dt * iv[6] + m.sqrt_dt * n0 * r[5];
        s[4] += m.dt * iv[7];
        s[5] += m.dt * iv[8];
        s[6] = s[1] - s[2];
        s[7] = m.cmin + (m.cmax - m.cmin) / (1.0 + exp(m.r * (m.midpoint - (s[6]))));
    }
};

struct Kuramoto {
    static constexpr int NS = 1, NI = 1, NN = 1, NG = 1, NR = 3, CONN = 0, BOLDV = 0;
    static constexpr bool OSC = true, POSTBW = false;
    __device__ static void init(double *s, double *, const double *, const double *r, const IntegrateArgs &) { s[0] = r[0]; }
    __device__ static void restart(double *s, double *, const double *r) { s[0] = r[0]; }
    __device__ static void step(double *s, double *iv, const double *g, const double *r, double in, double n0, double,
                                const ModelK &K) {  // kuramoto.cpp:48-61
        const KurK &m = K.kur;
        iv[0] = r[1] + g[0] * in;
        s[0] = s[0] + m.dt * iv[0] + m.sqrt_dt * n0 * r[2];
        s[0] = fmod(s[0], m.twopi);
    }
};

struct RWWEx {
    static constexpr int NS = 3, NI = 2, NN = 1, NG = 1, NR = 3, CONN = 2, BOLDV = 2;
    static constexpr bool OSC = false, POSTBW = false;
    __device__ static void init(double *s, double *, const double *, const double *, const IntegrateArgs &) {
        s[0] = s[1] = 0.0; s[2] = 0.001;
    }
    __device__ static void restart(double *s, double *, const double *) { s[2] = 0.001; }
    __device__ static void step(double *s, double *iv, const double *g, const double *r, double in, double n0, double,
                                const ModelK &K) {  // rwwex.cpp:48-73
        const RWWExK &m = K.rwwex;
        s[0] = r[0] * m.J_N * s[2] + g[0] * m.J_N * in + r[1];
        iv[0] = m.a * s[0] - m.b;
        s[1] = iv[0] / (1 - exp(-m.d * iv[0]));
        iv[1] = m.dt_gamma * ((1 - s[2]) * s[1]) - m.dt_itau * s[2] + n0 * m.sqrt_dt * r[2];
        s[2] += iv[1];
        s[2] = fmax(0.0, fmin(1.0, s[2]));
    }
};

// BW Euler step, bw.cu:4-15 (the q update uses the already-updated nu)
__device__ __forceinline__ void bw_step(double &x, double &f, double &nu, double &q, double n_state, const BWConst &c) {
    x = x + c.dt * (n_state - c.kappa * x - c.y * (f - 1.0));
    double tmp_f = f + c.dt * x;
    nu = nu + c.dt_itau * (f - pow(nu, c.ialpha));
    q = q + c.dt_itau * (f * (1.0 - pow(c.oneminrho, (1.0 / f))) / c.rho - pow(nu, c.ialpha) * q / nu);
    f = tmp_f;
}

// ---------------------------------------------------------------- kernel
template <class M, bool DELAY>
__global__ void __launch_bounds__(1024) k_integrate_fp64(const IntegrateArgs a) {
    const int sim = a.sim_begin + blockIdx.x;
    const int j = threadIdx.x;
    const int n = a.nodes;
    const bool act = j < n;
    extern __shared__ double x1[];  // conn-state of every node, previous step (no delay)
    __shared__ int s_trial, s_adjust, s_failed;

    const double *SC = a.sc + (size_t)a.sc_idx[sim] * n * n;
    double g[M::NG], r[M::NR], s[M::NS], iv[M::NI], ssum[M::NS];
#pragma unroll
    for (int i = 0; i < M::NG; ++i) g[i] = a.gparams[(size_t)i * a.n_sims + sim];
    const size_t rstride = (size_t)a.n_sims * n;
#pragma unroll
    for (int i = 0; i < M::NR; ++i) r[i] = act ? a.rparams[i * rstride + (size_t)sim * n + j] : 0.0;
#pragma unroll
    for (int i = 0; i < M::NI; ++i) iv[i] = 0.0;
#pragma unroll
    for (int i = 0; i < M::NS; ++i) { s[i] = 0.0; ssum[i] = 0.0; }
    M::init(s, iv, g, r, a);
    if (j == 0) { s_trial = 0; s_adjust = (a.do_fic && a.max_fic_trials > 0) ? 1 : 0; s_failed = 0; }

    double bx = 0.0, bf = 1.0, bnu = 1.0, bq = 1.0;
    // ring buffer (delay) or shared immediate history
    int D = 0, buff = 0;
    double *hist = nullptr;
    const int *dly = nullptr;
    if (DELAY) {
        D = a.max_delay[sim];
        hist = a.hist + a.hist_off[sim];
        dly = a.delay + (size_t)a.delay_idx[sim] * n * n;
        buff = D - 1;
    }
    auto reset_conn = [&]() {
        if (!act) return;
        if (DELAY) { for (int b = 0; b < D; ++b) hist[(size_t)b * n + j] = s[M::CONN]; }
        else x1[j] = s[M::CONN];
    };
    reset_conn();

    double *bold = a.bold + (size_t)sim * a.bold_len * n;
    const size_t ext = a.states_ts ? (size_t)n * a.states_len : (size_t)n;
    int bw_i = 0, bold_i = 0, states_i = 0, repeat = 0;
    int sh_j = act ? a.sh_nodes[j] : 0;
    while (bw_i < a.bw_it) {
        const int sh_ts = a.sh_ts[(bw_i % a.noise_bw_it) + repeat * a.noise_bw_it];
        for (int inner = 0; inner < a.inner_it; ++inner) {
            __syncthreads();  // conn-states of the previous step are visible
            double in = 0.0;
            if (act) {
                if (DELAY) {
                    const double xj = hist[(size_t)buff * n + j];
                    for (int k = 0; k < n; ++k) {
                        int kb = buff + __ldg(&dly[(size_t)k * n + j]);
                        if (kb >= D) kb -= D;
                        const double xk = hist[(size_t)kb * n + k];
                        if (M::OSC) in += __ldg(&SC[(size_t)k * n + j]) * sin(xk - xj);
                        else in += __ldg(&SC[(size_t)k * n + j]) * xk;
                    }
                } else {
                    const double xj = x1[j];
                    for (int k = 0; k < n; ++k) {
                        if (M::OSC) in += __ldg(&SC[(size_t)k * n + j]) * sin(x1[k] - xj);
                        else in += __ldg(&SC[(size_t)k * n + j]) * x1[k];
                    }
                }
                const long long ni = ((long long)sh_ts * a.inner_it + inner) * n * M::NN + (long long)sh_j * M::NN;
                const double n0 = a.noise[ni];
                const double n1 = (M::NN > 1) ? a.noise[ni + 1] : 0.0;
                M::step(s, iv, g, r, in, n0, n1, a.K);
            }
            __syncthreads();  // every read of the previous conn-states is done
            if (act) {
                if (DELAY) hist[(size_t)buff * n + j] = s[M::CONN];
                else x1[j] = s[M::CONN];
            }
            if (DELAY) buff = (buff + D - 1) % D;
        }
        if (act) bw_step(bx, bf, bnu, bq, s[M::BOLDV], a.bw);
        if ((bw_i + 1) % a.bold_tr_iters == 0) {  // bnm.cpp:316-335
            if (act)
                bold[(size_t)bold_i * n + j] =
                    a.bw.V_0 * (a.bw.k1 * (1 - bq) + a.bw.k2 * (1 - bq / bnu) + a.bw.k3 * (1 - bnu));
            bold_i++;
        }
        if (a.ext_out && (bw_i + 1) % a.states_sampling_iters == 0) {  // bnm.cpp:337-355
            if (act) {
                if (a.states_ts) {
#pragma unroll
                    for (int v = 0; v < M::NS; ++v)
                        a.states[((size_t)v * a.n_sims + sim) * ext + (size_t)states_i * n + j] = s[v];
                } else if (states_i >= a.n_states_samples_remove) {
#pragma unroll
                    for (int v = 0; v < M::NS; ++v) ssum[v] += s[v];
                }
            }
            states_i++;
        }
        if ((bw_i + 1) % a.noise_bw_it == 0 && bw_i + 1 < a.bw_it) {
            repeat++;
            sh_j = act ? a.sh_nodes[(size_t)repeat * n + j] : 0;
        }
        bool restart = false;
        if constexpr (M::POSTBW) {  // numerical FIC, rww.cpp:233-298
            const int t = bw_i + 1;
            if (s_adjust) {  // block-uniform: only changed by thread 0 between barriers
                if (act && t >= a.I_start && t <= a.I_end) iv[4] += s[0];
                if (t == a.I_end) {
                    const int trial = s_trial;
                    int need = 0;
                    if (act) {
                        iv[4] /= a.I_dur;
                        iv[6] = iv[4] - a.K.rww.b_a_ratio_E;
                        if (fabs(iv[6] + 0.026) > 0.005) {
                            need = 1;
                            if (trial < a.max_fic_trials) {
                                if (iv[6] < -0.026) {
                                    r[2] -= iv[5];
                                    iv[5] -= 0.001;
                                    iv[5] = fmax(iv[5], 0.001);
                                } else {
                                    r[2] += iv[5];
                                }
                            }
                        }
                    }
                    const int any = __syncthreads_or(need);
                    if (any) {
                        if (trial < a.max_fic_trials) {
                            restart = true;
                            if (j == 0) s_trial = trial + 1;
                        } else if (j == 0) {
                            s_adjust = 0;
                            s_failed = 1;
                        }
                    } else if (j == 0) {
                        s_adjust = 0;
                    }
                    __syncthreads();
                }
            }
        }
        bw_i++;
        if (restart) {  // bnm.cpp:386-434
            if (act) M::restart(s, iv, r);
            bx = 0.0; bf = 1.0; bnu = 1.0; bq = 1.0;
            __syncthreads();
            reset_conn();
            bold_i = 0; states_i = 0; bw_i = 0; repeat = 0;
            buff = D - 1;
            sh_j = act ? a.sh_nodes[j] : 0;
        }
    }
    if constexpr (M::POSTBW) {
        if (a.do_fic) {  // rww.cpp:300-314 post_integration
            if (act) a.rparams_out[2 * rstride + (size_t)sim * n + j] = r[2];
            if (j == 0) {
                a.gints[sim] = s_trial;
                a.gbools[(size_t)a.n_sims + sim] = (unsigned char)s_failed;
            }
        }
    }
    if (act && a.ext_out && !a.states_ts) {
        const int pts = states_i - a.n_states_samples_remove;
#pragma unroll
        for (int v = 0; v < M::NS; ++v) a.states[((size_t)v * a.n_sims + sim) * ext + j] = ssum[v] / pts;
    }
}

template <class M>
cudaError_t launch_model(const IntegrateArgs &a, cudaStream_t st) {
    const int threads = ((a.nodes + 31) / 32) * 32;
    const size_t smem = a.has_delay ? 0 : sizeof(double) * a.nodes;
    if (a.has_delay) k_integrate_fp64<M, true><<<a.n_sims - a.sim_begin, threads, smem, st>>>(a);
    else k_integrate_fp64<M, false><<<a.n_sims - a.sim_begin, threads, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_integrate_fp64(int model, const IntegrateArgs &a, cudaStream_t st) {
    switch (model) {
        case MODEL_RWW: return launch_model<RWW>(a, st);
        case MODEL_WC: return launch_model<WC>(a, st);
        case MODEL_JR: return launch_model<JR>(a, st);
        case MODEL_KURAMOTO: return launch_model<Kuramoto>(a, st);
        case MODEL_RWWEX: return launch_model<RWWEx>(a, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace cbnm
