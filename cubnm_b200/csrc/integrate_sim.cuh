// Per-simulation integrator: one CTA per simulation, one thread per node.
//
// The time loop of src/ext/bnm.cu:117-505 (GPU) / src/ext/bnm.cpp:69-522 (CPU)
// with the node state in R (double: reference arithmetic; float: FP32 mode) and
// the Balloon-Windkessel state always in double.  Coupling, bnm.cu:48-101:
//     in_j = sum_k SC[k][j] * x_k            (x_k(t - d_kj) with delays; Kuramoto: sin(x_k - x_j))
// read from the previous step's conn-states in shared memory (no delay) or from
// the simulation's ring buffer in global memory (delay; the buffer index moves
// backwards, bnm.cu:28-46).  Numerical FIC (rww.cpp:233-298) restarts the whole
// simulation from t = 0 with adjusted wIE, as the CPU path does.
#pragma once
#include <cstdint>
#include "engine.h"
#include "models.cuh"

namespace cbnm {

// BW Euler step, bw.cu:4-15 (the q update uses the already-updated nu)
__device__ __forceinline__ void bw_step(double &x, double &f, double &nu, double &q, double n_state, const BWConst &c) {
    x = x + c.dt * (n_state - c.kappa * x - c.y * (f - 1.0));
    double tmp_f = f + c.dt * x;
    nu = nu + c.dt_itau * (f - pow(nu, c.ialpha));
    q = q + c.dt_itau * (f * (1.0 - pow(c.oneminrho, (1.0 / f))) / c.rho - pow(nu, c.ialpha) * q / nu);
    f = tmp_f;
}

// The arrays of IntegrateArgs in precision R (SC, noise) or in the model's
// state type (delay ring buffers).
template <class R>
struct SimArrays;
template <>
struct SimArrays<double> {
    __device__ static const double *sc(const IntegrateArgs &a) { return a.sc; }
    __device__ static const double *noise(const IntegrateArgs &a) { return a.noise; }
    __device__ static double *hist(const IntegrateArgs &a) { return a.hist; }
    using Ell = int4;  // {weight lo, weight hi, ring-buffer offset, 0}
    __device__ static const int4 *ell(const IntegrateArgs &a) { return a.ell_pk64; }
    __device__ static double ell_w(const int4 v) { return __hiloint2double(v.y, v.x); }
    __device__ static int ell_off(const int4 v) { return v.z; }
};
template <>
struct SimArrays<float> {
    __device__ static const float *sc(const IntegrateArgs &a) { return a.sc_f32; }
    __device__ static const float *noise(const IntegrateArgs &a) { return a.noise_f32; }
    __device__ static float *hist(const IntegrateArgs &a) { return a.hist_f32; }
    using Ell = int2;  // {ring-buffer offset, weight bits}
    __device__ static const int2 *ell(const IntegrateArgs &a) { return a.ell_pk32; }
    __device__ static float ell_w(const int2 v) { return __int_as_float(v.y); }
    __device__ static int ell_off(const int2 v) { return v.x; }
};

// FP32 coupling input of node j, sum_k SC[k][j] x[k] (x in shared memory, 16-byte
// aligned): four independent partial sums over k = 0,1,2,3 mod 4 (float4 reads
// of x), so the FMA chain is a quarter as long; combined as (s0 + s1) + (s2 + s3).
// The FP64 path keeps the reference's sequential order instead.
__device__ __forceinline__ float coupling_f32(const float *__restrict__ SC, const float *x, int n, int j) {
    float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
    const float4 *x4 = reinterpret_cast<const float4 *>(x);
    int k = 0;
    for (; k + 3 < n; k += 4) {
        const float4 v = x4[k >> 2];
        s0 += __ldg(&SC[(size_t)k * n + j]) * v.x;
        s1 += __ldg(&SC[(size_t)(k + 1) * n + j]) * v.y;
        s2 += __ldg(&SC[(size_t)(k + 2) * n + j]) * v.z;
        s3 += __ldg(&SC[(size_t)(k + 3) * n + j]) * v.w;
    }
    for (; k < n; ++k) s0 += __ldg(&SC[(size_t)k * n + j]) * x[k];
    return (s0 + s1) + (s2 + s3);
}

// MAXT = the block size bound: 1024 (at most 64 registers a thread), or 512 (up
// to 128 registers, no spills) for delayed networks of 129-512 nodes.
template <class M, bool DELAY, class R, bool SPARSE, int MAXT>
__global__ void __launch_bounds__(MAXT) k_integrate_sim(const IntegrateArgs a) {
    const int sim = a.sim_begin + blockIdx.x;
    const int j = threadIdx.x;
    const int n = a.nodes;
    const bool act = j < n;
    using S = typename M::S;  // state type (R, or double for the Kuramoto phase)
    using P = typename M::P;  // regional-parameter type
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S *x1 = reinterpret_cast<S *>(smem_raw);  // conn-state of every node, previous step (no delay)
    __shared__ int s_trial, s_adjust, s_failed;

    const int sc_i = a.sc_idx[sim];
    const R *SC = SimArrays<R>::sc(a) + (size_t)sc_i * n * n;
    // sparse coupling: the nonzero sources of node j (ascending k), then zero-weight padding
    using EA = SimArrays<R>;
    const int EK = SPARSE ? a.ell_k : 0;
    const typename EA::Ell *pk = nullptr;
    if (SPARSE && act) {
        const int table = DELAY ? a.delay_idx[sim] : 0;
        pk = EA::ell(a) + ((size_t)sc_i * a.ell_tables + table) * EK * n + j;
    }
    const R *noise = SimArrays<R>::noise(a);
    R g[M::NG], iv[M::NI];
    P r[M::NR];
    S s[M::NS];
    double ssum[M::NS];
#pragma unroll
    for (int i = 0; i < M::NG; ++i) g[i] = (R)a.gparams[(size_t)i * a.n_sims + sim];
    const size_t rstride = (size_t)a.n_sims * n;
#pragma unroll
    for (int i = 0; i < M::NR; ++i) r[i] = act ? (P)a.rparams[i * rstride + (size_t)sim * n + j] : P(0);
#pragma unroll
    for (int i = 0; i < M::NI; ++i) iv[i] = R(0);
#pragma unroll
    for (int i = 0; i < M::NS; ++i) { s[i] = S(0); ssum[i] = 0.0; }
    M::init(s, iv, g, r);
    // numerical FIC bookkeeping (rww.cpp:233-298), in double for both precisions
    double fic_sum = 0.0, fic_delta = a.init_delta;
    if (j == 0) { s_trial = 0; s_adjust = (a.do_fic && a.max_fic_trials > 0) ? 1 : 0; s_failed = 0; }

    double bx = 0.0, bf = 1.0, bnu = 1.0, bq = 1.0;
    int D = 0, buff = 0;
    S *hist = nullptr;
    const int *dly = nullptr;
    if (DELAY) {
        D = a.max_delay[sim];
        hist = SimArrays<S>::hist(a) + a.hist_off[sim];
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
            R in = R(0);
            if (act) {
                if (SPARSE && DELAY) {
                    // ((buff + d) mod D) * n + k as buff * n + (d * n + k), wrapped once
                    // (buff < D and d <= D); the host keeps 2 * D * n below 2^31.
                    const int hbase = buff * n, hwrap = D * n;
                    const S xj = hist[hbase + j];
                    // eight entries unrolled: eight ring-buffer loads in flight (1,103 ->
                    // 1,344 sims x sim-s / s at 400 nodes with delays, 343 -> 364 at 1,000)
#pragma unroll 8
                    for (int q = 0; q < EK; ++q) {
                        const auto v = __ldg(pk + (size_t)q * n);
                        int h = hbase + EA::ell_off(v);
                        if (h >= hwrap) h -= hwrap;
                        const S xk = hist[h];
                        if (M::OSC) in += EA::ell_w(v) * sin(R(xk - xj));
                        else in += EA::ell_w(v) * R(xk);
                    }
                } else if (SPARSE) {
                    const S xj = x1[j];
#pragma unroll 4
                    for (int q = 0; q < EK; ++q) {
                        const auto v = __ldg(pk + (size_t)q * n);
                        const S xk = x1[EA::ell_off(v)];
                        if (M::OSC) in += EA::ell_w(v) * sin(R(xk - xj));
                        else in += EA::ell_w(v) * R(xk);
                    }
                } else if (DELAY) {
                    const S xj = hist[(size_t)buff * n + j];
                    for (int k = 0; k < n; ++k) {
                        int kb = buff + __ldg(&dly[(size_t)k * n + j]);
                        if (kb >= D) kb -= D;
                        const S xk = hist[(size_t)kb * n + k];
                        if (M::OSC) in += __ldg(&SC[(size_t)k * n + j]) * sin(R(xk - xj));
                        else in += __ldg(&SC[(size_t)k * n + j]) * R(xk);
                    }
                } else if constexpr (sizeof(R) == 4 && sizeof(S) == 4 && !M::OSC) {
                    in = coupling_f32(SC, x1, n, j);
                } else {
                    const S xj = x1[j];
                    for (int k = 0; k < n; ++k) {
                        if (M::OSC) in += __ldg(&SC[(size_t)k * n + j]) * sin(R(x1[k] - xj));
                        else in += __ldg(&SC[(size_t)k * n + j]) * R(x1[k]);
                    }
                }
                const long long ni = ((long long)sh_ts * a.inner_it + inner) * n * M::NN + (long long)sh_j * M::NN;
                const R n0 = noise[ni];
                const R n1 = (M::NN > 1) ? noise[ni + 1] : R(0);
                M::step(s, iv, g, r, in, n0, n1, a.K);
            }
            __syncthreads();  // every read of the previous conn-states is done
            if (act) {
                if (DELAY) hist[(size_t)buff * n + j] = s[M::CONN];
                else x1[j] = s[M::CONN];
            }
            if (DELAY) buff = (buff + D - 1) % D;
        }
        if (act) bw_step(bx, bf, bnu, bq, (double)s[M::BOLDV], a.bw);
        if ((bw_i + 1) % a.bold_tr_iters == 0) {  // bnm.cpp:316-335
            // the truncated iteration counts (bw_it, bold_tr_iters) can give one more
            // sample than bold_len for some TR / bw_dt; that sample has no slot
            if (act && bold_i < a.bold_len)
                bold[(size_t)bold_i * n + j] =
                    a.bw.V_0 * (a.bw.k1 * (1 - bq) + a.bw.k2 * (1 - bq / bnu) + a.bw.k3 * (1 - bnu));
            bold_i++;
        }
        if (a.ext_out && (bw_i + 1) % a.states_sampling_iters == 0) {  // bnm.cpp:337-355
            if (act) {
                if (a.states_ts) {
                    if (states_i < a.states_len)
#pragma unroll
                        for (int v = 0; v < M::NS; ++v)
                            a.states[((size_t)v * a.n_sims + sim) * ext + (size_t)states_i * n + j] = (double)s[v];
                } else if (states_i >= a.n_states_samples_remove) {
#pragma unroll
                    for (int v = 0; v < M::NS; ++v) ssum[v] += (double)s[v];
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
                if (act && t >= a.I_start && t <= a.I_end) fic_sum += (double)s[0];
                if (t == a.I_end) {
                    const int trial = s_trial;
                    int need = 0;
                    if (act) {
                        fic_sum /= a.I_dur;
                        const double diff = fic_sum - a.K.rww.b_a_ratio_E;
                        if (fabs(diff + 0.026) > 0.005) {
                            need = 1;
                            if (trial < a.max_fic_trials) {
                                if (diff < -0.026) {
                                    r[2] = (P)((double)r[2] - fic_delta);
                                    fic_delta -= 0.001;
                                    fic_delta = fmax(fic_delta, 0.001);
                                } else {
                                    r[2] = (P)((double)r[2] + fic_delta);
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
            fic_sum = 0.0;
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
            if (act) a.rparams_out[2 * rstride + (size_t)sim * n + j] = (double)r[2];
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

template <class M, class R, int MAXT, bool DELAY>
cudaError_t launch_sim_variant(const IntegrateArgs &a, int grid, int threads, size_t smem, cudaStream_t st) {
    if (a.ell_k > 0) k_integrate_sim<M, DELAY, R, true, MAXT><<<grid, threads, smem, st>>>(a);
    else k_integrate_sim<M, DELAY, R, false, MAXT><<<grid, threads, smem, st>>>(a);
    return cudaGetLastError();
}

// UNCAP: with delays at 129-512 nodes, launch the 512-thread-bound variant.  Its
// extra registers cost CTAs per SM; measured on one B200 (FP32 unless noted,
// 8 s, 20% density, 6 m/s) it gains with delays: rWW 200 nodes FP64 1.59x, rWW
// 400 1.40x, rWW 512 1.47x, WC 300 1.50x, JR 160 1.64x, rWW 400 FP64 1.01x; but
// rWWEx 200 0.85x (its capped variant does not spill), and without delays
// 0.77-0.88x (rWW 200 and 256 nodes, FP32 and FP64), so those keep the cap
// (as does Kuramoto, not measured).
template <class M, class R, bool UNCAP>
cudaError_t launch_sim_kernel(const IntegrateArgs &a, cudaStream_t st) {
    const int threads = ((a.nodes + 31) / 32) * 32;
    const size_t smem = a.has_delay ? 0 : sizeof(typename M::S) * a.nodes;
    const int grid = a.n_sims - a.sim_begin;
    if (!a.has_delay) return launch_sim_variant<M, R, 1024, false>(a, grid, threads, smem, st);
    if constexpr (UNCAP) {
        if (threads > 128 && threads <= 512) return launch_sim_variant<M, R, 512, true>(a, grid, threads, smem, st);
    }
    return launch_sim_variant<M, R, 1024, true>(a, grid, threads, smem, st);
}

template <class R>
cudaError_t launch_sim_model(int model, const IntegrateArgs &a, cudaStream_t st) {
    switch (model) {
        case MODEL_RWW: return launch_sim_kernel<RWWm<R>, R, true>(a, st);
        case MODEL_WC: return launch_sim_kernel<WCm<R>, R, true>(a, st);
        case MODEL_JR: return launch_sim_kernel<JRm<R>, R, true>(a, st);
        case MODEL_KURAMOTO: return launch_sim_kernel<Kuramotom<R>, R, false>(a, st);  // not measured
        case MODEL_RWWEX: return launch_sim_kernel<RWWExm<R>, R, false>(a, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace cbnm
