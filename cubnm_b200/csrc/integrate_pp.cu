// Two-tile tensor-core integrator for rWW (precision "fp32"), the fast path of
// the benchmark workload: shared-SC batches without delays, <= 128 nodes.
//
// The time loop is the reference's (src/ext/bnm.cu:117-505: Euler-Maruyama
// node update, coupling bnm.cu:48-77, Balloon-Windkessel bnm.cu:357-371, BOLD at
// TR, time-averaged or sampled states), organised so that the tensor core and
// the CUDA cores work at the same time:
//
//  * A CTA integrates 64 simulations that share one SC as two halves of 32
//    (h = 0, 1).  Each step of a half is a coupling GEMM
//        D_h[j][s] = sum_k SC[k][j] x_k^s        (M = 128 node lanes, N = 32, K = KP)
//    on tcgen05 in BF16x3 (A = SC^T hi / lo in TMEM, B = x hi / lo in shared
//    memory) followed by the elementwise update of its 32 x n node states.
//    The halves alternate: while the update threads step half 0, the tensor
//    core runs the GEMM of half 1, and the reverse, so the GEMM phase no longer
//    adds to the step time.
//  * Warps 0-15 update: warp w owns TMEM lane quarter w % 4 (node j = lane of
//    that quarter) and simulations 8 (w / 4) .. 8 (w / 4) + 7 of both halves, as
//    four packed FP32x2 pairs per half.  Warp 16 issues the MMAs: it waits on an
//    mbarrier that the 512 update threads arrive on once they have written the
//    half's B operand, issues the 21 MMAs into that half's accumulator and
//    commits them to a second mbarrier that the update threads wait on.
//  * The node state (S_E, S_I of 16 simulations) lives in registers; the model
//    parameters of all 64 simulations live in TMEM (5 columns per simulation),
//    read per pair each step; the FP64 Balloon-Windkessel state (x, f, nu, q)
//    lives in a per-CTA global scratch that stays in L2 (2 KB per node for the 64
//    simulations), updated once per bw step for one simulation pair per inner
//    step (after the halves' updates, while the next GEMMs run), staggered
//    between warpgroups so that their loads spread over the bw step.  The time-averaged states are
//    accumulated in shared memory (FP32) and written once per simulation.
//  * Every wait is bounded (about 2 s); on timeout the CTA records a status,
//    leaves its loops, frees its TMEM and returns.
//
// TMEM columns: [0, 64) accumulators (half h at 32 h) | [64, 64 + KP) SC^T hi
// then lo (two BF16 per column, K chunk kk at +8 kk) | [64 + KP, 64 + KP + 320)
// parameters, param q of half h for simulation s at 64 + KP + (5 h + q) 32 + s.
// SMEM: B operands [h][hi, lo] (MN-major, no swizzle, 8-row x 16-byte core
// matrices: element (k, s) at (k/8) LBO + (s/8) 128 + (k%8) 16 + (s%8) 2, LBO =
// 512 B), then z[16][512] (the Balloon-Windkessel inputs of the last bw step,
// one column per thread), then the FP32 state sums [NOUT][64][n] when they fit.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cuda/atomic>
#include "engine.h"
#include "tc_common.cuh"

namespace cbnm {
namespace {

constexpr int PP_TN = 32;                      // simulations per half (MMA N)
constexpr int PP_SIMS = 2 * PP_TN;             // simulations per work item
constexpr int PP_UPD = 512;                    // update threads (4 warpgroups)
constexpr int PP_THREADS = PP_UPD + 32;        // + the MMA-issuing warp
constexpr int PP_SPT = 8;                      // simulations per thread per half
constexpr int PP_PAIRS = 2 * PP_SPT / 2;       // simulation pairs per thread (both halves)
constexpr uint32_t PP_LBO = (PP_TN / 8) * 128;
constexpr int PP_COL_A = 2 * PP_TN;            // SC^T after the two accumulators

struct PPSmem {
    uint64_t mbar_mma[2];   // GEMM of half h complete (one commit per step)
    uint64_t mbar_x[2];     // B operand of half h written (PP_UPD arrivals per step)
    uint32_t tmem_base;
    int abort;
    unsigned int arrived[2];  // warp-specialised form: warps of half h done writing its B operand this step
};

__host__ __device__ constexpr size_t pp_b_bytes(int KP) { return (size_t)KP * PP_TN * 2; }
__host__ __device__ constexpr size_t pp_z_bytes() { return sizeof(float) * 2 * PP_SPT * PP_UPD; }
__host__ __device__ constexpr size_t pp_sacc_bytes(int nout, int n) { return sizeof(float) * (size_t)nout * PP_SIMS * n; }

// States of one simulation pair at a sample step: the time series, or the sums
// of the kept samples (shared-memory FP32 sums when they fit, else the output
// array).  Out of line: it runs once per sample, and inlined it would hold
// registers across the whole time loop.
template <int NOUT>
__device__ __noinline__ void pp_states_out(const IntegrateArgs &a, const int *wd, float *sacc, int use_sacc,
                                           const float2 *o, int slot0, int j, int states_i) {
    const int n = a.nodes;
    const size_t ext = a.states_ts ? (size_t)n * a.states_len : (size_t)n;
    for (int u = 0; u < 2; ++u) {
        const int slot = slot0 + u;
        const int sim = wd[1 + slot];
        for (int v = 0; v < NOUT; ++v) {
            const float ov = u ? o[v].y : o[v].x;
            if (a.states_ts) {
                if (sim >= 0 && states_i < a.states_len)
                    a.states[((size_t)v * a.n_sims + sim) * ext + (size_t)states_i * n + j] = ov;
            } else if (states_i >= a.n_states_samples_remove) {
                if (use_sacc) sacc[((size_t)v * PP_SIMS + slot) * n + j] += ov;
                else if (sim >= 0) a.states[((size_t)v * a.n_sims + sim) * ext + j] += ov;
            }
        }
    }
}

// WS = false: warps 0-15 update both halves, warp 16 issues the MMAs (544 threads).
// WS = true: warps 0-15 update half 0 and warps 16-31 half 1 (1024 threads), so the
// two halves' updates can run at the same time; the last warp of a half to finish
// writing its B operand issues that half's MMAs (counted in shared memory).
template <class M, bool WS>
__device__ __forceinline__ void pp_body(const IntegrateArgs &a, const int *work, int n_work, int KP, int use_sacc) {
    static_assert(M::PAIR && M::NP <= 5, "parameters of 64 simulations must fit beside the SC in TMEM");
    constexpr int NUPD = WS ? 1024 : PP_UPD;      // update threads
    constexpr int NH = WS ? 1 : 2;                // halves a thread updates
    constexpr int NPAIR = NH * PP_SPT / 2;        // simulation pairs a thread updates
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const int n = a.nodes;
    const size_t bb = pp_b_bytes(KP);
    float *zbuf = reinterpret_cast<float *>(smem_raw + 4 * bb);
    float *sacc = zbuf + NH * PP_SPT * NUPD;
    PPSmem *sm = reinterpret_cast<PPSmem *>(reinterpret_cast<uint8_t *>(sacc) +
                                            (use_sacc ? pp_sacc_bytes(M::NOUT, n) : 0));

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const bool issuer_warp = !WS && warp == PP_UPD / 32;
    const int h_own = WS ? (warp >> 4) : 0;  // the half of a warp-specialised thread
    const int quarter = warp & 3;
    const int g = (warp >> 2) & 3;           // simulations 8 g .. 8 g + 7 of each half
    const int j = quarter * 32 + lane;       // node = TMEM lane
    const bool act = !issuer_warp && j < n;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm->tmem_base)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int h = 0; h < 2; ++h) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&sm->mbar_mma[h])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&sm->mbar_x[h])), "r"(PP_UPD));
            sm->arrived[h] = 0u;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        sm->abort = 0;
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = sm->tmem_base;
    const uint32_t t_lane = tmem + ((uint32_t)(quarter * 32) << 16);
    const int col_p = PP_COL_A + KP;
    const int half_k = KP / 2;
    uint32_t ph_mma[2] = {0u, 0u}, ph_x[2] = {0u, 0u};
    int sc_loaded = -1;

    // constants read from the parameter space where they are used (precomputed on the host)
    const typename M::K &K = *reinterpret_cast<const typename M::K *>(a.k32);
    const BW64 &bw = a.bwf;
    const size_t rstride = (size_t)a.n_sims * n;
    const size_t ext = a.states_ts ? (size_t)n * a.states_len : (size_t)n;
    const int steps = a.bw_it * a.inner_it;
    // this CTA's Balloon-Windkessel scratch: [h][g][pr][x, f, nu, q][node] of simulation pairs
    double2 *bws = reinterpret_cast<double2 *>(a.bw_scratch) + (size_t)blockIdx.x * (2 * 4 * 4 * 4) * n;

    for (int w = blockIdx.x; w < n_work; w += gridDim.x) {
        const int *wd = work + (size_t)w * (1 + PP_SIMS);
        const int sc_idx = wd[0];
        const bool live[2] = {wd[1] >= 0, wd[1 + PP_TN] >= 0};
        float2 s2[NH][PP_SPT / 2][M::NS];   // node state of the thread's pairs

        if (!issuer_warp) {
            // ---- parameters -> TMEM; initial state; SC^T when the SC changes
#pragma unroll
            for (int hh = 0; hh < NH; ++hh) {
                const int h = WS ? h_own : hh;
                uint32_t pw[M::NP][PP_SPT];
#pragma unroll
                for (int pr = 0; pr < PP_SPT / 2; ++pr) {
                    float pa[2][M::NP], sa[2][M::NS];
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const int sim = wd[1 + h * PP_TN + g * PP_SPT + 2 * pr + u];
                        M::init(sa[u]);
#pragma unroll
                        for (int q = 0; q < M::NP; ++q) pa[u][q] = 0.0f;
                        if (act && sim >= 0) {
                            double rr[8];
                            for (int q = 0; q < 8; ++q)
                                rr[q] = q < a.n_regional ? a.rparams[(size_t)q * rstride + (size_t)sim * n + j] : 0.0;
                            M::params(pa[u], a.gparams[sim], rr, K);
                        }
                    }
                    float2 p2[M::NP];
#pragma unroll
                    for (int q = 0; q < M::NP; ++q) p2[q] = make_float2(pa[0][q], pa[1][q]);
                    PairStep<M>::params(p2);
#pragma unroll
                    for (int q = 0; q < M::NP; ++q) {
                        pw[q][2 * pr] = __float_as_uint(p2[q].x);
                        pw[q][2 * pr + 1] = __float_as_uint(p2[q].y);
                    }
#pragma unroll
                    for (int q = 0; q < M::NS; ++q) s2[hh][pr][q] = make_float2(sa[0][q], sa[1][q]);
                }
#pragma unroll
                for (int q = 0; q < M::NP; ++q) tmem_st8_nowait(t_lane + col_p + (h * M::NP + q) * PP_TN + g * PP_SPT, pw[q]);
            }
            tmem_wait_st();
            if (sc_loaded != sc_idx && g == 0 && h_own == 0) {  // warpgroup 0 writes SC^T (each warp its lane quarter)
                const float *SC = a.sc_f32 + (size_t)sc_idx * n * n;
                for (int c0 = 0; c0 < half_k; c0 += 8) {
                    uint32_t hw[8], lw[8];
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const int k = 2 * (c0 + c);
                        const float v0 = (act && k < n) ? SC[(size_t)k * n + j] : 0.0f;
                        const float v1 = (act && k + 1 < n) ? SC[(size_t)(k + 1) * n + j] : 0.0f;
                        split_bf16x2(v0, v1, hw[c], lw[c]);
                    }
                    tmem_st8(t_lane + PP_COL_A + c0, hw);
                    tmem_st8(t_lane + PP_COL_A + half_k + c0, lw);
                }
            }
            // Balloon-Windkessel state x = 0, f = nu = q = 1 for the thread's pairs
            if (act) {
#pragma unroll
                for (int p = 0; p < NPAIR; ++p) {
                    double2 *b = bws + (size_t)(((WS ? h_own : (p >> 2))) * 16 + g * 4 + (p & 3)) * 4 * n + j;
                    b[0] = make_double2(0.0, 0.0);
                    b[n] = make_double2(1.0, 1.0);
                    b[2 * n] = make_double2(1.0, 1.0);
                    b[3 * n] = make_double2(1.0, 1.0);
                }
            }
            if (a.ext_out && !a.states_ts && act) {  // state sums start at zero
#pragma unroll
                for (int hh = 0; hh < NH; ++hh)
                    for (int i = 0; i < PP_SPT; ++i) {
                        const int h = WS ? h_own : hh;
                        const int slot = h * PP_TN + g * PP_SPT + i;
                        const int sim = wd[1 + slot];
                        for (int v = 0; v < M::NOUT; ++v) {
                            if (use_sacc) sacc[((size_t)v * PP_SIMS + slot) * n + j] = 0.0f;
                            else if (sim >= 0) a.states[((size_t)v * a.n_sims + sim) * ext + j] = 0.0;
                        }
                    }
            }
        }
        // B operand of half h: rows of padded nodes are zero
        auto write_x = [&](int hh) {
            if (j >= KP) return;
            const int h = WS ? h_own : hh;
            uint32_t hw[PP_SPT / 2], lw[PP_SPT / 2];
#pragma unroll
            for (int pr = 0; pr < PP_SPT / 2; ++pr) {
                const float2 x = act ? s2[hh][pr][M::CV] : make_float2(0.0f, 0.0f);
                split_bf16x2(x.x, x.y, hw[pr], lw[pr]);
            }
            const int s0 = g * PP_SPT;
            const uint32_t off = (j >> 3) * PP_LBO + (s0 >> 3) * 128 + (j & 7) * 16;
            *reinterpret_cast<uint4 *>(smem_raw + (2 * h) * bb + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            *reinterpret_cast<uint4 *>(smem_raw + (2 * h + 1) * bb + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        };
        // the 21 MMAs of one step of half h (BF16x3, 3 per K chunk of 16), committed to mbar_mma[h]
        auto issue = [&](int h) {
            const uint32_t idesc = instr_desc(PP_TN);
            const uint32_t bh = smem_u32(smem_raw + (2 * h) * bb), bl = smem_u32(smem_raw + (2 * h + 1) * bb);
            const uint32_t d = tmem + h * PP_TN;
            for (int kk = 0; kk < KP / 16; ++kk) {
                const uint32_t tah = tmem + PP_COL_A + kk * 8, tal = tah + half_k;
                const uint64_t dbh = smem_desc(bh + kk * 2 * PP_LBO, PP_LBO, 128);
                const uint64_t dbl = smem_desc(bl + kk * 2 * PP_LBO, PP_LBO, 128);
                mma_bf16_ts(d, tah, dbh, idesc, kk > 0 ? 1u : 0u);
                mma_bf16_ts(d, tah, dbl, idesc, 1u);
                mma_bf16_ts(d, tal, dbh, idesc, 1u);
            }
            mma_commit(smem_u32(&sm->mbar_mma[h]));
        };
        // B operand of half h written: the last of its 16 warps issues the half's GEMM
        auto arrive_ws = [&](int h) {
            fence_proxy_async();
            fence_before();
            __syncwarp();
            if (lane == 0) {
                cuda::atomic_ref<unsigned int, cuda::thread_scope_block> cnt(sm->arrived[h]);
                if (cnt.fetch_add(1u, cuda::memory_order_acq_rel) == 15u) {
                    cnt.store(0u, cuda::memory_order_relaxed);
                    fence_after();
                    issue(h);
                }
            }
            __syncwarp();
        };
        if (!issuer_warp) {
#pragma unroll
            for (int hh = 0; hh < NH; ++hh) write_x(hh);
            fence_proxy_async();
        }
        fence_before();
        __syncthreads();
        fence_after();
        sc_loaded = sc_idx;
        if (WS && live[h_own] && tid == h_own * 512) issue(h_own);  // step 0 of each half

        if (issuer_warp) {
            // ---- MMA issue: GEMM k of half h once its B operand is written
            if (lane == 0) {
                bool stop = false;
                for (int k = 0; k < steps && !stop; ++k) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        if (!live[h]) continue;
                        if (k > 0) {
                            const bool ok = mbar_wait(smem_u32(&sm->mbar_x[h]), ph_x[h]);
                            ph_x[h] ^= 1u;
                            if (!ok) {
                                sm->abort = 1;
                                atomicExch(a.status, 1);
                            }
                            if (*(volatile int *)&sm->abort) { stop = true; break; }
                        }
                        fence_after();
                        issue(h);
                    }
                }
            }
        } else {
            // ---- update threads
            int bold_i = 0, states_i = 0, repeat = 0;
            int sh_j = act ? a.sh_nodes[j] : 0;
            const long long nstride = (long long)n * M::NN;
            const float *nrow = a.noise_f32 + (long long)a.sh_ts[0] * a.inner_it * nstride + (long long)sh_j * M::NN;
            float nz0 = act ? __ldg(nrow) : 0.0f;
            float nz1 = (act && M::NN > 1) ? __ldg(nrow + 1) : 0.0f;
            bool aborted = false, pend = false, pend_tr = false;
            int pend_bi = 0;
            double2 bwx[4];  // Balloon-Windkessel state of the pair being updated
            const int stagger = (2 * g + (WS ? 5 * h_own : 0)) % a.inner_it;
            auto half_of = [&](int p) { return WS ? h_own : (p >> 2); };
            auto bw_ptr = [&](int p) { return bws + (size_t)(half_of(p) * 16 + g * 4 + (p & 3)) * 4 * n + j; };
            auto bw_load = [&](int p) {
                if (!act || !live[half_of(p)]) return;
                const double2 *b = bw_ptr(p);
#pragma unroll
                for (int c = 0; c < 4; ++c) bwx[c] = __ldcg(b + (size_t)c * n);
            };
            // one bw step of pair p (inputs: z of the previous bw step), BOLD at TR
            auto bw_do = [&](int p) {
                if (!act || !live[half_of(p)]) return;
                double x[2] = {bwx[0].x, bwx[0].y}, f[2] = {bwx[1].x, bwx[1].y};
                double nu[2] = {bwx[2].x, bwx[2].y}, q[2] = {bwx[3].x, bwx[3].y};
                const float z0 = zbuf[(2 * p) * NUPD + tid], z1 = zbuf[(2 * p + 1) * NUPD + tid];
                bw_step64_contracted(x[0], f[0], nu[0], q[0], (double)z0, bw);
                bw_step64_contracted(x[1], f[1], nu[1], q[1], (double)z1, bw);
                double2 *b = bw_ptr(p);
                __stcg(b, make_double2(x[0], x[1]));
                __stcg(b + n, make_double2(f[0], f[1]));
                __stcg(b + 2 * n, make_double2(nu[0], nu[1]));
                __stcg(b + 3 * n, make_double2(q[0], q[1]));
                if (pend_tr && pend_bi < a.bold_len) {  // no slot for a sample past bold_len
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const int sim = wd[1 + half_of(p) * PP_TN + g * PP_SPT + 2 * (p & 3) + u];
                        if (sim >= 0)
                            a.bold[(size_t)sim * a.bold_len * n + (size_t)pend_bi * n + j] =
                                bold64(q[u], nu[u], bw);
                    }
                }
            };
            for (int bw_i = 0; bw_i < a.bw_it && !aborted; ++bw_i) {
                const bool sample = a.ext_out && ((bw_i + 1) % a.states_sampling_iters == 0);
                int nx_repeat = repeat, nx_shj = sh_j;
                if ((bw_i + 1) % a.noise_bw_it == 0 && bw_i + 1 < a.bw_it) {
                    nx_repeat = repeat + 1;
                    nx_shj = act ? __ldg(&a.sh_nodes[(size_t)nx_repeat * n + j]) : 0;
                }
                const int nx_ts =
                    (bw_i + 1 < a.bw_it) ? __ldg(&a.sh_ts[((bw_i + 1) % a.noise_bw_it) + nx_repeat * a.noise_bw_it]) : 0;
                for (int inner = 0; inner < a.inner_it; ++inner) {
                    const bool last_step = (bw_i == a.bw_it - 1) && (inner == a.inner_it - 1);
                    const bool out_now = sample && (inner == a.inner_it - 1);
                    const float n0 = nz0, n1 = nz1;
                    if (act) {  // the next step's noise
                        const float *nr = (inner + 1 < a.inner_it) ? nrow + (inner + 1) * nstride
                                                                   : a.noise_f32 + (long long)nx_ts * a.inner_it * nstride +
                                                                         (long long)nx_shj * M::NN;
                        nz0 = __ldg(nr);
                        if (M::NN > 1) nz1 = __ldg(nr + 1);
                    }
#pragma unroll
                    for (int hh = 0; hh < NH; ++hh) {
                        const int h = WS ? h_own : hh;
                        if (!live[h]) continue;
                        const bool ok = mbar_wait(smem_u32(&sm->mbar_mma[h]), ph_mma[h]);
                        ph_mma[h] ^= 1u;
                        if (!ok) {
                            sm->abort = 1;
                            atomicExch(a.status, 1);
                        }
                        if (*(volatile int *)&sm->abort) { aborted = true; break; }
                        fence_after();
                        // coupling sums and parameters of one pair at a time, then its step
#pragma unroll
                        for (int pr = 0; pr < PP_SPT / 2; ++pr) {
                            uint32_t acc[2], pw[M::NP][2];
                            tmem_ld2(t_lane + h * PP_TN + g * PP_SPT + 2 * pr, acc);
#pragma unroll
                            for (int q = 0; q < M::NP; ++q)
                                tmem_ld2(t_lane + col_p + (h * M::NP + q) * PP_TN + g * PP_SPT + 2 * pr, pw[q]);
                            tmem_wait_ld();
                            if (act) {
                                float2 p2[M::NP], o[M::NOUT];
#pragma unroll
                                for (int q = 0; q < M::NP; ++q)
                                    p2[q] = make_float2(__uint_as_float(pw[q][0]), __uint_as_float(pw[q][1]));
                                PairStep<M>::step(s2[hh][pr], p2, make_float2(__uint_as_float(acc[0]), __uint_as_float(acc[1])),
                                                  n0, n1, K, o);
                                if (out_now)
                                    pp_states_out<M::NOUT>(a, wd, sacc, use_sacc, o, h * PP_TN + g * PP_SPT + 2 * pr, j,
                                                           states_i);
                            }
                        }
                        if (!last_step) {
                            write_x(hh);
                            if constexpr (WS) {
                                arrive_ws(h);
                            } else {
                                fence_proxy_async();
                                fence_before();
                                mbar_arrive(smem_u32(&sm->mbar_x[h]));
                            }
                        }
                    }
                    if (aborted) break;
                    // Balloon-Windkessel work of the previous bw step: pair p at inner step
                    // (p + stagger) mod inner_it, the stagger differing between warpgroups so
                    // that their L2 loads of the state spread over the bw step
                    if (pend) {
                        const int it = a.inner_it;
                        for (int p = ((inner - stagger) % it + it) % it; p < NPAIR; p += it) {
                            bw_load(p);
                            bw_do(p);
                        }
                    }
                }
                if (aborted) break;
                // this bw step's Balloon-Windkessel inputs; the updates run during the next bw step
#pragma unroll
                for (int hh = 0; hh < NH; ++hh)
#pragma unroll
                    for (int pr = 0; pr < PP_SPT / 2; ++pr) {
                        zbuf[(hh * PP_SPT + 2 * pr) * NUPD + tid] = s2[hh][pr][M::BV].x;
                        zbuf[(hh * PP_SPT + 2 * pr + 1) * NUPD + tid] = s2[hh][pr][M::BV].y;
                    }
                pend = true;
                pend_tr = ((bw_i + 1) % a.bold_tr_iters == 0);
                pend_bi = bold_i;
                if (pend_tr) bold_i++;
                if (sample) states_i++;
                repeat = nx_repeat;
                sh_j = nx_shj;
                nrow = a.noise_f32 + (long long)nx_ts * a.inner_it * nstride + (long long)sh_j * M::NN;
            }
            if (pend && !aborted) {  // the last bw step
                for (int p = 0; p < NPAIR; ++p) {
                    bw_load(p);
                    bw_do(p);
                }
            }
            if (a.ext_out && !a.states_ts && act && !aborted) {
                const int pts = states_i - a.n_states_samples_remove;
#pragma unroll
                for (int hh = 0; hh < NH; ++hh)
                    for (int i = 0; i < PP_SPT; ++i) {
                        const int h = WS ? h_own : hh;
                        const int slot = h * PP_TN + g * PP_SPT + i;
                        const int sim = wd[1 + slot];
                        if (sim < 0) continue;
                        for (int v = 0; v < M::NOUT; ++v) {
                            double *dst = a.states + ((size_t)v * a.n_sims + sim) * ext + j;
                            if (use_sacc) *dst = (double)sacc[((size_t)v * PP_SIMS + slot) * n + j] / pts;
                            else *dst /= pts;
                        }
                    }
            }
        }
        fence_before();
        __syncthreads();
        fence_after();
        if (sm->abort) break;
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

// 544 threads: the register file allows 96 registers a thread (warps are allocated
// registers in groups of four, so 17 warps are charged as 20).
template <class M>
__global__ void __launch_bounds__(PP_THREADS, 1)
    k_integrate_pp(const __grid_constant__ IntegrateArgs a, const int *work, int n_work, int KP, int use_sacc) {
    pp_body<M, false>(a, work, n_work, KP, use_sacc);
}

template <class M>
__global__ void __launch_bounds__(1024, 1)
    k_integrate_pp_ws(const __grid_constant__ IntegrateArgs a, const int *work, int n_work, int KP, int use_sacc) {
    pp_body<M, true>(a, work, n_work, KP, use_sacc);
}

template <class M>
size_t pp_smem(int KP, int n, int *use_sacc) {
    const size_t base = 4 * pp_b_bytes(KP) + pp_z_bytes() + sizeof(PPSmem) + 64;
    const size_t with = base + pp_sacc_bytes(M::NOUT, n);
    *use_sacc = with <= 227 * 1024 ? 1 : 0;
    return *use_sacc ? with : base;
}

template <class M>
cudaError_t launch_pp(const IntegrateArgs &a, cudaStream_t st) {
    const int KP = ((a.nodes + 15) / 16) * 16;
    int use_sacc = 0;
    const size_t smem = pp_smem<M>(KP, a.nodes, &use_sacc);
    const int grid = std::min(a.n_tiles, a.pp_grid);
    if (a.pp_ws) {
        cudaError_t e = allow_dynamic_smem(k_integrate_pp_ws<M>);
        if (e != cudaSuccess) return e;
        k_integrate_pp_ws<M><<<grid, 1024, smem, st>>>(a, a.tiles, a.n_tiles, KP, use_sacc);
    } else {
        cudaError_t e = allow_dynamic_smem(k_integrate_pp<M>);
        if (e != cudaSuccess) return e;
        k_integrate_pp<M><<<grid, PP_THREADS, smem, st>>>(a, a.tiles, a.n_tiles, KP, use_sacc);
    }
    return cudaGetLastError();
}

}  // namespace

bool pp_supported(int model, int nodes, bool has_delay) {
    if (has_delay || nodes < 1 || nodes > TM) return false;
    const int KP = ((nodes + 15) / 16) * 16;
    if (PP_COL_A + KP + 2 * 5 * PP_TN > 512) return false;
    return model == MODEL_RWW;
}

size_t pp_bw_scratch_bytes(int nodes, int grid) { return sizeof(double2) * (size_t)grid * 2 * 4 * 4 * 4 * nodes; }

cudaError_t launch_integrate_pp(int model, const IntegrateArgs &a, cudaStream_t st, int *launches) {
    if (launches) ++*launches;
    if (model == MODEL_RWW) return launch_pp<RWW32>(a, st);
    return cudaErrorNotSupported;
}

}  // namespace cbnm
