// FP32 / tensor-core integrator (the fast path, precision "fp32").
//
// The same time loop as the FP64 kernel (reference: src/ext/bnm.cu:117-505),
// reorganised for B200:
//
//  * A CTA integrates a tile of TN simulations that share one SC (TN = 16 with
//    two CTAs per SM, or 32 with one).  Node j of the tile lives on TMEM lane j
//    (M = 128 lanes, nodes <= 128); each thread owns one node and SPT
//    simulations (4 in the 16-wide tile, 8 in the 32-wide one); warpgroup g
//    owns simulations [SPT g, SPT g + SPT) of the tile.
//  * Coupling (bnm.cu:48-77) is a GEMM every step:
//        D[j][s] = sum_k SC[k][j] * x_k^s
//    issued as tcgen05.mma kind::f16 with A = SC^T held in TMEM (BF16, written
//    once per SC) and B = x in shared memory (BF16, MN-major, rewritten every
//    step), in BF16x3 split precision: D = A_hi B_hi + A_hi B_lo + A_lo B_hi,
//    FP32 accumulation in TMEM.  The three passes are issued by three threads
//    (lane 0 of warps 0..2) into three accumulator sets that the readers add:
//    one thread issuing all 21 MMAs of a step was itself a bottleneck (the
//    three-issuer form measured 8% faster; a fourth issuer no further gain, as
//    the tensor pipe then bounds the GEMM).  Keeping A in TMEM leaves only the 16-column x
//    slice to be read from shared memory per MMA.  Elementwise model updates run
//    in FP32 registers.
//  * The Balloon-Windkessel state (bnm.cu:357-371) stays FP64 and lives in TMEM
//    (8 x 32-bit words per simulation).  The update of bw step m runs during the
//    GEMMs of bw step m+1 (one simulation pair per inner step), from the inputs
//    saved at the end of step m, so the FP64 work overlaps the tensor core.
//  * Every wait on the MMA barrier is bounded; on timeout the CTA records a
//    status, leaves its loop, frees its TMEM and returns.
//
// TMEM columns: [0, NACC TN) accumulator sets | [NACC TN, NACC TN + KP) SC^T hi then lo, two BF16
// per column, K chunk kk at +8kk | [COLS - 8 TN, COLS) Balloon-Windkessel state.
// SMEM B operand (MN-major, no swizzle, 8-row x 16-byte core matrices):
//   element (k, n) at (k/8)*LBO_B + (n/8)*128 + (k%8)*16 + (n%8)*2,
//   LBO_B = TN/8 * 128 B (K-direction core-matrix stride), SBO = 128 B.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cuda_bf16.h>
#include "engine.h"
#include "tc_common.cuh"

namespace cbnm {
namespace {

constexpr int COL_ACC = 0;           // accumulator columns start here

// Tile geometry: TN simulations per tile (MMA N), SPT simulations per thread,
// TN/SPT warpgroups per CTA.
template <int TN_, int SPT_, int NACC_>
struct Tile {
    static constexpr int TN = TN_;
    static constexpr int SPT = SPT_;
    static constexpr int NACC = NACC_;   // independent accumulator sets the GEMM round-robins over
    static constexpr int NWG = TN / SPT;
    static constexpr int NTHREADS = NWG * 128;
    static constexpr int TMEM_COLS = TN >= 32 ? 512 : 256;   // one CTA an SM at 32 wide, two at 16
    static constexpr int CTAS_PER_SM = 512 / TMEM_COLS;
    static constexpr uint32_t LBO_B = (TN / 8) * 128;
    // threads that issue the step's GEMM: 1 (all MMAs, round-robin over the NACC sets)
    // or NACC (thread p of warp p issues pass p of BF16x3 into accumulator set p)
    static constexpr int ISSUERS = (NACC == 3) ? 3 : 1;
};

struct Smem {
    uint64_t mbar;
    uint32_t tmem_base;
    int abort;
    int sc_loaded;
};

// ---------------------------------------------------------------- kernel
template <class M, class T>
__global__ void __launch_bounds__(T::NTHREADS, T::CTAS_PER_SM) k_integrate_tc(const IntegrateArgs a, const int *tiles,
                                                                              int n_tiles, int KP) {
    constexpr int TN = T::TN, TMEM_COLS = T::TMEM_COLS;
    constexpr uint32_t LBO_B = T::LBO_B;
    constexpr int NACC = T::NACC;
    constexpr int SPT = T::SPT;
    constexpr int COL_A = TN * NACC;                   // A_hi at COL_A, A_lo at COL_A + KP/2 (bf16 pairs)
    constexpr int COL_BWT = TMEM_COLS - TN * 8;        // Balloon-Windkessel state at the top
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *B_hi = smem_raw;
    uint8_t *B_lo = B_hi + KP * TN * 2;
    Smem *sm = reinterpret_cast<Smem *>(B_lo + KP * TN * 2);
    // time-averaged states: FP32 sums [NOUT][TN][n] in shared memory, written once per simulation
    float *sacc = reinterpret_cast<float *>(B_lo + KP * TN * 2 + ((sizeof(Smem) + 15) & ~(size_t)15));
    const bool use_sacc = a.ext_out && !a.states_ts;

    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int quarter = warp & 3;          // TMEM lane quarter
    const int wg = warp >> 2;              // warpgroup: simulations [wg*SPT, wg*SPT+SPT)
    const int j = quarter * 32 + (tid & 31);  // node = TMEM lane
    const int n = a.nodes;
    const bool act = j < n;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm->tmem_base)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        // one arrival per issuing thread (ISSUERS of them commit each step)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&sm->mbar)), "r"(T::ISSUERS));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        sm->abort = 0;
        sm->sc_loaded = -1;
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = sm->tmem_base;
    const uint32_t t_lane = tmem + ((uint32_t)(quarter * 32) << 16);
    const uint32_t mbar = smem_u32(&sm->mbar);
    uint32_t phase = 0;
    const uint32_t idesc = instr_desc(TN);
    const typename M::K K = M::make(a.K);
    const BW64 &bw = a.bwf;
    const size_t rstride = (size_t)a.n_sims * n;
    const size_t ext = a.states_ts ? (size_t)n * a.states_len : (size_t)n;
    const int half = KP / 2;

    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int *td = tiles + (size_t)tile * (TN + 1);
        const int sc_idx = td[0];
        constexpr int NPR = SPT / 2;
        int sims[SPT];
        float2 p2[NPR][M::NP];   // parameters of simulation pair (2 pr, 2 pr + 1) of node j
        float2 s2[NPR][M::NS];   // state of that pair
#pragma unroll
        for (int pr = 0; pr < NPR; ++pr) {
            float pa[2][M::NP], sa[2][M::NS];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int i = 2 * pr + u;
                sims[i] = td[1 + wg * SPT + i];
                M::init(sa[u]);
#pragma unroll
                for (int q = 0; q < M::NP; ++q) pa[u][q] = 0.0f;
                if (act && sims[i] >= 0) {  // parameters of (node j, simulation)
                    double rr[8];
                    for (int q = 0; q < 8; ++q)
                        rr[q] = q < a.n_regional ? a.rparams[(size_t)q * rstride + (size_t)sims[i] * n + j] : 0.0;
                    M::params(pa[u], a.gparams[sims[i]], rr, K);
                }
            }
#pragma unroll
            for (int q = 0; q < M::NP; ++q) p2[pr][q] = make_float2(pa[0][q], pa[1][q]);
#pragma unroll
            for (int q = 0; q < M::NS; ++q) s2[pr][q] = make_float2(sa[0][q], sa[1][q]);
            PairStep<M>::params(p2[pr]);
        }
        if (use_sacc && act) {  // states sums start at zero
            for (int i = 0; i < SPT; ++i)
                for (int v = 0; v < M::NOUT; ++v) sacc[((size_t)v * TN + wg * SPT + i) * n + j] = 0.0f;
        }
        {  // Balloon-Windkessel state in TMEM: x = 0, f = nu = q = 1
            uint32_t w[8];
            const double init[4] = {0.0, 1.0, 1.0, 1.0};
            for (int q = 0; q < 4; ++q) {
                w[2 * q] = (uint32_t)__double2loint(init[q]);
                w[2 * q + 1] = (uint32_t)__double2hiint(init[q]);
            }
            for (int i = 0; i < SPT; ++i) tmem_st8(t_lane + COL_BWT + (wg * SPT + i) * 8, w);
        }
        // A operand = SC^T in TMEM (row j = target node on lane j; K = source node,
        // two BF16 per 32-bit column), split hi / lo.  Rewritten only when the SC changes;
        // warpgroup 0 writes it (each warp its own lane quarter).
        if (sm->sc_loaded != sc_idx && wg == 0) {
            const float *SC = a.sc_f32 + (size_t)sc_idx * n * n;
            for (int c0 = 0; c0 < half; c0 += 8) {
                uint32_t hw[8], lw[8];
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int k = 2 * (c0 + c);
                    const float v0 = (act && k < n) ? SC[(size_t)k * n + j] : 0.0f;
                    const float v1 = (act && k + 1 < n) ? SC[(size_t)(k + 1) * n + j] : 0.0f;
                    split_bf16x2(v0, v1, hw[c], lw[c]);
                }
                if (c0 + 8 <= half) {
                    tmem_st8(t_lane + COL_A + c0, hw);
                    tmem_st8(t_lane + COL_A + half + c0, lw);
                }
            }
        }
        // B operand rows of padded nodes are zero; live rows get the initial state
        auto write_x = [&]() {
            if (j >= KP) return;
            uint32_t hw[SPT / 2], lw[SPT / 2];
#pragma unroll
            for (int pr = 0; pr < SPT / 2; ++pr) {
                const float2 x = act ? s2[pr][M::CV] : make_float2(0.0f, 0.0f);
                split_bf16x2(x.x, x.y, hw[pr], lw[pr]);
            }
            // simulations n = wg*SPT .. wg*SPT+SPT-1 of the tile
            const int n0 = wg * SPT;
            const uint32_t off = (j >> 3) * LBO_B + (n0 >> 3) * 128 + (j & 7) * 16 + (n0 & 7) * 2;
            if constexpr (SPT == 8) {
                *reinterpret_cast<uint4 *>(B_hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                *reinterpret_cast<uint4 *>(B_lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
            } else {
                *reinterpret_cast<uint2 *>(B_hi + off) = make_uint2(hw[0], hw[1]);
                *reinterpret_cast<uint2 *>(B_lo + off) = make_uint2(lw[0], lw[1]);
            }
        };
        write_x();
        if (tid == 0) sm->sc_loaded = sc_idx;

        // Balloon-Windkessel of one bw step for simulation pair `pr`, inputs z0, z1
        // (the BOLD state at the end of that bw step), BOLD written when `tr`.
        auto bw_pair = [&](int pr, float z0, float z1, bool tr, int bi) {
            uint32_t w[16];
            const uint32_t col = t_lane + COL_BWT + (wg * SPT + 2 * pr) * 8;
            tmem_ld16(col, w);
            double x[2], f[2], nu[2], q[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                x[u] = __hiloint2double((int)w[8 * u + 1], (int)w[8 * u + 0]);
                f[u] = __hiloint2double((int)w[8 * u + 3], (int)w[8 * u + 2]);
                nu[u] = __hiloint2double((int)w[8 * u + 5], (int)w[8 * u + 4]);
                q[u] = __hiloint2double((int)w[8 * u + 7], (int)w[8 * u + 6]);
            }
            if (act) bw_step64x2(x, f, nu, q, (double)z0, (double)z1, bw);
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                w[8 * u + 0] = (uint32_t)__double2loint(x[u]); w[8 * u + 1] = (uint32_t)__double2hiint(x[u]);
                w[8 * u + 2] = (uint32_t)__double2loint(f[u]); w[8 * u + 3] = (uint32_t)__double2hiint(f[u]);
                w[8 * u + 4] = (uint32_t)__double2loint(nu[u]); w[8 * u + 5] = (uint32_t)__double2hiint(nu[u]);
                w[8 * u + 6] = (uint32_t)__double2loint(q[u]); w[8 * u + 7] = (uint32_t)__double2hiint(q[u]);
                const int sim = sims[2 * pr + u];
                if (tr && act && sim >= 0 && bi < a.bold_len)  // no slot for a sample past bold_len
                    a.bold[(size_t)sim * a.bold_len * n + (size_t)bi * n + j] = bold64(q[u], nu[u], bw);
            }
            tmem_st16(col, w);
        };
        // pending Balloon-Windkessel work of the previous bw step: its inputs and BOLD flag
        float zp[SPT];
        bool pend = false, pend_tr = false;
        int pend_bi = 0;
#pragma unroll
        for (int i = 0; i < SPT; ++i) zp[i] = 0.0f;

        fence_before();
        __syncthreads();

        int bold_i = 0, states_i = 0, repeat = 0;
        int sh_j = act ? a.sh_nodes[j] : 0;
        bool aborted = false;  // only set right after a barrier, so block-uniform
        // noise of the next step is loaded one step ahead (its address does not depend on the GEMM)
        const long long nstride = (long long)n * M::NN;
        const float *nrow = a.noise_f32 + (long long)a.sh_ts[0] * a.inner_it * nstride + (long long)sh_j * M::NN;
        float nz0 = act ? __ldg(nrow) : 0.0f;
        float nz1 = (act && M::NN > 1) ? __ldg(nrow + 1) : 0.0f;
        for (int bw_i = 0; bw_i < a.bw_it; ++bw_i) {
            const bool sample = a.ext_out && ((bw_i + 1) % a.states_sampling_iters == 0);
            // shuffled noise row of the next bw step (for the prefetch at the last inner step)
            int nx_repeat = repeat, nx_shj = sh_j;
            if ((bw_i + 1) % a.noise_bw_it == 0 && bw_i + 1 < a.bw_it) {
                nx_repeat = repeat + 1;
                nx_shj = act ? __ldg(&a.sh_nodes[(size_t)nx_repeat * n + j]) : 0;
            }
            const int nx_ts = (bw_i + 1 < a.bw_it) ? __ldg(&a.sh_ts[((bw_i + 1) % a.noise_bw_it) + nx_repeat * a.noise_bw_it]) : 0;
            for (int inner = 0; inner < a.inner_it; ++inner) {
                // (1) x written by every thread -> visible to the tensor core
                fence_proxy_async();
                fence_before();
                __syncthreads();
                if (sm->abort) { aborted = true; break; }
                // (2) the BF16x3 coupling GEMM (A from TMEM, B from SMEM)
                if constexpr (T::ISSUERS == 3) {
                    // three issuing threads in three warps, one BF16x3 pass each, into
                    // accumulator sets 0..2; each commits its own MMAs to the barrier
                    if ((tid & 31) == 0 && warp < 3) {
                        fence_after();
                        const int pass = warp;
                        const uint32_t bh = smem_u32(B_hi), bl = smem_u32(B_lo);
                        const uint32_t d = tmem + COL_ACC + pass * TN;
                        const int nk = KP / 16;
                        for (int kk = 0; kk < nk; ++kk) {
                            const uint32_t ta = tmem + COL_A + (pass == 2 ? half : 0) + kk * 8;
                            const uint64_t db = smem_desc((pass == 1 ? bl : bh) + kk * 2 * LBO_B, LBO_B, 128);
                            mma_bf16_ts(d, ta, db, idesc, kk > 0 ? 1u : 0u);
                        }
                        mma_commit(mbar);
                    }
                } else if (tid == 0) {
                    fence_after();
                    const uint32_t bh = smem_u32(B_hi), bl = smem_u32(B_lo);
                    const int nk = KP / 16;
                    // consecutive MMAs go to different accumulator sets so they do not
                    // wait on each other's read-modify-write of the same TMEM columns
                    int issued = 0;
                    for (int kk = 0; kk < nk; ++kk) {
                        const uint32_t tah = tmem + COL_A + kk * 8, tal = tmem + COL_A + half + kk * 8;
                        const uint64_t dbh = smem_desc(bh + kk * 2 * LBO_B, LBO_B, 128);
                        const uint64_t dbl = smem_desc(bl + kk * 2 * LBO_B, LBO_B, 128);
#pragma unroll
                        for (int pass = 0; pass < 3; ++pass, ++issued) {
                            const int set = issued % NACC;
                            const uint32_t d = tmem + COL_ACC + set * TN;
                            const uint32_t accumulate = issued >= NACC ? 1u : 0u;
                            if (pass == 0) mma_bf16_ts(d, tah, dbh, idesc, accumulate);
                            else if (pass == 1) mma_bf16_ts(d, tah, dbl, idesc, accumulate);
                            else mma_bf16_ts(d, tal, dbh, idesc, accumulate);
                        }
                    }
                    mma_commit(mbar);
                }
                // (2b) while the tensor core works: the previous bw step's Balloon-Windkessel
                // update, one simulation pair per inner step
                if (pend) {
#pragma unroll
                    for (int pr = 0; pr < SPT / 2; ++pr)
                        if (pr % a.inner_it == inner) bw_pair(pr, zp[2 * pr], zp[2 * pr + 1], pend_tr, pend_bi);
                    if (inner == a.inner_it - 1 || inner == SPT / 2 - 1) pend = false;
                }
                // (3) wait for the GEMM, read this thread's 8 coupling sums
                const bool ok = mbar_wait(mbar, phase);
                phase ^= 1u;
                if (!ok) {
                    sm->abort = 1;
                    atomicExch(a.status, 1);
                }
                fence_after();
                uint32_t acc[SPT];
                tmem_ld<SPT>(t_lane + COL_ACC + wg * SPT, acc);
#pragma unroll
                for (int set = 1; set < NACC; ++set) {
                    uint32_t more[SPT];
                    tmem_ld<SPT>(t_lane + COL_ACC + set * TN + wg * SPT, more);
#pragma unroll
                    for (int i = 0; i < SPT; ++i) acc[i] = __float_as_uint(__uint_as_float(acc[i]) + __uint_as_float(more[i]));
                }
                // (4) elementwise update of the 8 simulations of node j
                const float n0 = nz0, n1 = nz1;
                if (act) {  // prefetch the next step's noise
                    const float *nr = (inner + 1 < a.inner_it) ? nrow + (inner + 1) * nstride
                                                               : a.noise_f32 + (long long)nx_ts * a.inner_it * nstride +
                                                                     (long long)nx_shj * M::NN;
                    nz0 = __ldg(nr);
                    if (M::NN > 1) nz1 = __ldg(nr + 1);
                }
                if (act) {
                    const bool last = sample && (inner == a.inner_it - 1);
#pragma unroll
                    for (int pr = 0; pr < SPT / 2; ++pr) {
                        float2 o[M::NOUT];
                        PairStep<M>::step(s2[pr], p2[pr],
                                          make_float2(__uint_as_float(acc[2 * pr]), __uint_as_float(acc[2 * pr + 1])),
                                          n0, n1, K, o);
                        if (last) {
#pragma unroll
                            for (int u = 0; u < 2; ++u) {
                                const int sim = sims[2 * pr + u];
                                if (sim < 0) continue;
                                for (int v = 0; v < M::NOUT; ++v) {
                                    const float ov = u ? o[v].y : o[v].x;
                                    if (a.states_ts) {
                                        if (states_i < a.states_len)
                                            a.states[((size_t)v * a.n_sims + sim) * ext + (size_t)states_i * n + j] = ov;
                                    }
                                    else if (states_i >= a.n_states_samples_remove)
                                        sacc[((size_t)v * TN + wg * SPT + 2 * pr + u) * n + j] += ov;
                                }
                            }
                        }
                    }
                }
                write_x();
            }
            if (aborted) break;
            // this bw step's Balloon-Windkessel inputs; the update itself runs during the
            // next bw step's GEMMs
            const bool tr = ((bw_i + 1) % a.bold_tr_iters == 0);
#pragma unroll
            for (int pr = 0; pr < SPT / 2; ++pr) {
                zp[2 * pr] = s2[pr][M::BV].x;
                zp[2 * pr + 1] = s2[pr][M::BV].y;
            }
            pend = true;
            pend_tr = tr;
            pend_bi = bold_i;
            if (tr) bold_i++;
            if (sample) states_i++;
            repeat = nx_repeat;
            sh_j = nx_shj;
            nrow = a.noise_f32 + (long long)nx_ts * a.inner_it * nstride + (long long)sh_j * M::NN;
        }
        if (pend && !aborted) {  // the last bw step
#pragma unroll
            for (int pr = 0; pr < SPT / 2; ++pr) bw_pair(pr, zp[2 * pr], zp[2 * pr + 1], pend_tr, pend_bi);
        }
        if (use_sacc && act && !aborted) {
            const int pts = states_i - a.n_states_samples_remove;
            for (int i = 0; i < SPT; ++i)
                if (sims[i] >= 0)
                    for (int v = 0; v < M::NOUT; ++v)
                        a.states[((size_t)v * a.n_sims + sims[i]) * ext + j] =
                            (double)sacc[((size_t)v * TN + wg * SPT + i) * n + j] / pts;
        }
        fence_before();
        __syncthreads();
        if (sm->abort) break;
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

using Tile16 = Tile<16, 8, 1>;   // 2 warpgroups x 8 simulations, two CTAs per SM
using Tile32 = Tile<32, 8, 3>;   // 4 warpgroups x 8 simulations, one CTA per SM, 3 GEMM issuers

template <class T>
size_t smem_bytes(int KP) { return (size_t)2 * KP * T::TN * 2 + sizeof(Smem) + 64; }
// the time-averaged state sums [NOUT][TN][nodes] (FP32)
template <class M, class T>
size_t sacc_bytes(int nodes) { return sizeof(float) * (size_t)M::NOUT * T::TN * nodes + 16; }

template <class M, class T>
cudaError_t launch_tc(const IntegrateArgs &a, const int *tiles, int n_tiles, cudaStream_t st) {
    const int KP = ((a.nodes + 15) / 16) * 16;
    // shared memory large enough that no more CTAs than TMEM holds land on one SM
    const size_t floor = T::CTAS_PER_SM == 2 ? 80 * 1024 : 120 * 1024;
    const size_t smem = std::max<size_t>(smem_bytes<T>(KP) + sacc_bytes<M, T>(a.nodes), floor);
    cudaError_t e = allow_dynamic_smem(k_integrate_tc<M, T>);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::min(n_tiles, T::CTAS_PER_SM * sms);
    k_integrate_tc<M, T><<<grid, T::NTHREADS, smem, st>>>(a, tiles, n_tiles, KP);
    return cudaGetLastError();
}

template <class M>
cudaError_t launch_model(const IntegrateArgs &a, cudaStream_t st) {
    if (a.tile_width == 32) return launch_tc<M, Tile32>(a, a.tiles, a.n_tiles, st);
    if (a.tile_width == 16) return launch_tc<M, Tile16>(a, a.tiles, a.n_tiles, st);
    return cudaErrorInvalidValue;
}

// TMEM columns used: accumulator sets (NACC TN) + SC^T hi/lo (KP) + Balloon-Windkessel state (8 TN)
template <class T>
constexpr bool tmem_fits(int KP) { return T::NACC * T::TN + KP + 8 * T::TN <= T::TMEM_COLS; }

}  // namespace

// Tile width: 32 simulations (one CTA per SM, one 32-wide GEMM per step: the
// tensor core's cost is per instruction at these widths, so the wider GEMM
// halves it per simulation; measured 145k vs 140k sims*s/s for the 16-wide,
// two-CTA form on the 100-node workload).  CBNM_FP32_TILE=16 selects the
// 16-wide form where SC^T fits beside its state (nodes <= 112).
int fp32_tile_for(int nodes) {
    const char *e = std::getenv("CBNM_FP32_TILE");
    const int KP = ((nodes + 15) / 16) * 16;
    if (e && std::atoi(e) == 16 && tmem_fits<Tile16>(KP)) return 16;
    return 32;
}

bool fp32_supported(int model, int nodes, bool has_delay) {
    if (has_delay || nodes > TM || nodes < 1) return false;
    if (!tmem_fits<Tile32>(((nodes + 15) / 16) * 16)) return false;
    return model == MODEL_RWW || model == MODEL_WC || model == MODEL_JR || model == MODEL_RWWEX;
}

cudaError_t launch_integrate_fp32(int model, const IntegrateArgs &a, cudaStream_t st, int *launches) {
    if (launches) ++*launches;
    switch (model) {
        case MODEL_RWW: return launch_model<RWW32>(a, st);
        case MODEL_WC: return launch_model<WC32>(a, st);
        case MODEL_JR: return launch_model<JR32>(a, st);
        case MODEL_RWWEX: return launch_model<RWWEx32>(a, st);
        default: break;
    }
    return cudaErrorNotSupported;
}

}  // namespace cbnm
