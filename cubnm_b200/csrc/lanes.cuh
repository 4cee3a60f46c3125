// FP32 integrator with the simulations on the lanes, for the networks the
// tensor-core tiles do not take: conduction delays (any node count) and more than
// 128 nodes.  The time loop is the reference's (src/ext/bnm.cu:117-505); the
// delayed coupling is bnm.cu:48-77 with the ring-buffer index of bnm.cu:28-46.
//
// The per-simulation kernel (integrate_sim.cuh, the reference's one CTA per
// simulation and one thread per node) gathers x_k(t - d_kj) from the
// simulation's own ring buffer: each 4-byte value costs a 32-byte sector, and
// every simulation re-reads the SC / delay entries.  Here 16 simulations that
// share one SC and one delay table are integrated together, simulation s on
// lane s of a half-warp:
//
//  * thread (node row r = tid / 16, simulation s = tid % 16) updates nodes
//    j = r, r + NT/16, r + 2 NT/16, ... (MN of them) of simulation s, state in
//    registers;
//  * the ring buffer of the group is [slot][node][16 simulations] (FP32), so the
//    16 lanes that need x_k(t - d_kj) of their own simulation read 64 contiguous
//    bytes, and the packed ELLPACK entry {d n + k, weight} of (j, q) is the same
//    address for the half-warp;
//  * the buffer has max_delay + 1 slots: step t reads slots buff + d (d >= 1) and
//    writes slot buff, which no read of step t touches, so one barrier per step
//    orders the writes of step t before the reads of step t + 1.  Without delays
//    the coupling reads the previous step (d = 1, two slots);
//  * parameters are an FP32 copy laid out [node][param][16]; the FP64
//    Balloon-Windkessel state is in global memory [node][4][16] (updated once per
//    bw step, series form of tc_common.cuh); noise is shared by all simulations.
// The coupling sum runs over the nonzeros in ascending source order from zero, as
// the per-simulation kernel's, so the node states are the same as that kernel's.
// A gather is two dependent loads (the entry, then x_k(t - d_kj), which for
// networks whose ring buffers outgrow L2 comes from HBM), so the kernel is bound
// by the loads in flight: a thread interleaves the gathers of LC of its rows
// (nonzero q outer, row inner, unrolled to LN_GATHER_MLP gathers) and loads the
// entries of nonzero q + 1 while those of q are in flight.  Registers are the
// limit (64 a thread at 1,024 threads): the noise shuffle of a row is read per
// step through L1 instead of being held per row.
#pragma once
#include <algorithm>
#include <type_traits>
#include "engine.h"
#include "integrate_sim.cuh"
#include "tangent.cuh"
#include "tc_common.cuh"

namespace cbnm {
namespace lanes {

constexpr int LN_SIMS = 16;   // simulations per group (a half-warp)
constexpr int LN_GATHER_ROWS = 4;  // node rows of a thread whose coupling gathers are issued together
constexpr int LN_GATHER_MLP = 8;   // coupling gathers of a thread in flight (rows x nonzeros unrolled)

template <bool TAN>
__device__ __forceinline__ typename std::conditional<TAN, float2, float>::type hval(float x, float dx) {
    if constexpr (TAN) return make_float2(x, dx);
    else return x;
}

// States of node j of simulation sim after a sample step: the time series, or
// the running sums of the kept samples.  Out of line: it runs once per sample.
template <int NS>
__device__ __noinline__ void lanes_states_out(const IntegrateArgs &a, const float *st, int sim, int j, int states_i) {
    const int n = a.nodes;
    const size_t ext = a.states_ts ? (size_t)n * a.states_len : (size_t)n;
    for (int v = 0; v < NS; ++v) {
        if (a.states_ts) {
            if (states_i < a.states_len) a.states[((size_t)v * a.n_sims + sim) * ext + (size_t)states_i * n + j] = (double)st[v];
        } else if (states_i >= a.n_states_samples_remove) {
            a.states[((size_t)v * a.n_sims + sim) * ext + j] += (double)st[v];
        }
    }
}

// TAN: also the tangent along G (tangent.cuh): ring buffer of (x, dx/dG) pairs,
// the Balloon-Windkessel tangent beside its state, dBOLD/dG to a.tan_bold.
template <class M, int NT, int MN, int DMODE, bool TAN>
__device__ __forceinline__ void lanes_group(const IntegrateArgs &a, int gi,
                                            typename std::conditional<TAN, float2, float>::type *hist, double *bws) {
    static_assert(!M::OSC, "phase models run on the per-simulation kernel (numerical FIC too, by the host)");
    using TG = Tangent<M>;
    constexpr int NTG = TAN ? TG::NT : 1;
    constexpr int BWW = TAN ? 8 : 4;  // doubles of Balloon-Windkessel scratch per (node, simulation)
    using H = typename std::conditional<TAN, float2, float>::type;
    constexpr int ROW = NT / LN_SIMS;  // node rows per CTA
    constexpr int LC = MN < LN_GATHER_ROWS ? MN : LN_GATHER_ROWS;   // rows whose gathers interleave
    // gathers in flight: LN_GATHER_MLP with 8 or more rows a thread; 4 with fewer, where
    // more (with the prefetched entries) spilled under the 64-register limit
    constexpr int MLP = MN >= 8 ? LN_GATHER_MLP : 4;
    constexpr int QU = LC >= MLP ? 1 : MLP / LC;                      // nonzeros unrolled per row
    using R = float;
    const int tid = threadIdx.x;
    const int s = tid & (LN_SIMS - 1);
    const int r0 = tid >> 4;
    const int n = a.nodes;
    const int EK = a.ell_k;
    const size_t rstride = (size_t)a.n_sims * n;
    const size_t ext = a.states_ts ? (size_t)n * a.states_len : (size_t)n;
    const BW64 &bw = a.bwf;
    // DMODE 0: no delays, 1: delays, 2: as the run says (a.has_delay); without delays
    // the coupling reads the previous step, one slot back
    const bool delayed = DMODE == 1 || (DMODE == 2 && a.has_delay);
    const int *gd = a.ln_groups + (size_t)gi * (3 + LN_SIMS);
    const int sc_i = gd[0], table = gd[1], D = gd[2];   // D: the group's largest delay (1 without delays)
    const int sim = gd[3 + s];
    const bool live = sim >= 0;
    const float *par = a.ln_params + (size_t)gi * n * M::NR * LN_SIMS;
    const int2 *ell = a.ell_pk32 + (size_t)(sc_i * a.ell_tables + table) * EK * n;
    R g[M::NG], iv[M::NI], st[MN][M::NS], dst[MN][NTG];
#pragma unroll
    for (int i = 0; i < M::NG; ++i) g[i] = live ? (R)a.gparams[(size_t)i * a.n_sims + sim] : R(0);
#pragma unroll
    for (int i = 0; i < M::NI; ++i) iv[i] = R(0);
    const int slots = D + 1, hw = slots * n;
#pragma unroll
    for (int m = 0; m < MN; ++m) {
        const int j = r0 + ROW * m;
#pragma unroll
        for (int v = 0; v < M::NS; ++v) st[m][v] = R(0);
#pragma unroll
        for (int v = 0; v < NTG; ++v) dst[m][v] = R(0);
        if (j >= n) continue;
        R r[M::NR];
#pragma unroll
        for (int q = 0; q < M::NR; ++q) r[q] = par[((size_t)j * M::NR + q) * LN_SIMS + s];
        M::init(st[m], iv, g, r);
        for (int b = 0; b < slots; ++b) hist[((size_t)b * n + j) * LN_SIMS + s] = hval<TAN>(st[m][M::CONN], 0.0f);
        double *bj = bws + (size_t)j * BWW * LN_SIMS + s;
        bj[0] = 0.0;
        bj[LN_SIMS] = 1.0;
        bj[2 * LN_SIMS] = 1.0;
        bj[3 * LN_SIMS] = 1.0;
        if (TAN)
            for (int c = 4; c < 8; ++c) bj[c * LN_SIMS] = 0.0;
        if (live && a.ext_out && !a.states_ts)
            for (int v = 0; v < M::NS; ++v) a.states[((size_t)v * a.n_sims + sim) * ext + j] = 0.0;
    }
    __syncthreads();

    int buff = D, bold_i = 0, states_i = 0, repeat = 0;
    // the node shuffle of the current noise repeat (its row of a.sh_nodes), read per
    // row and step through L1 rather than held in MN registers
    const int *shn = a.sh_nodes;
    double *bold = a.bold + (size_t)(live ? sim : 0) * a.bold_len * n;
    for (int bw_i = 0; bw_i < a.bw_it; ++bw_i) {
        const int sh_ts = a.sh_ts[(bw_i % a.noise_bw_it) + repeat * a.noise_bw_it];
        const bool sample = a.ext_out && (bw_i + 1) % a.states_sampling_iters == 0;  // bnm.cpp:337-355
        for (int inner = 0; inner < a.inner_it; ++inner) {
            const int hbase = buff * n;
            const bool out_now = sample && live && inner == a.inner_it - 1;
            // rows in chunks of LC: the gathers of a chunk's rows interleave (q outer,
            // row inner), so LC independent ring-buffer loads are in flight where one
            // row alone would wait on each in turn; each row still sums its nonzeros
            // in ascending order from zero
#pragma unroll
            for (int m0 = 0; m0 < MN; m0 += LC) {
                R in[LC], din[LC];
#pragma unroll
                for (int c = 0; c < LC; ++c) in[c] = din[c] = R(0);
                // coupling: sum over the nonzeros of column j of SC[k][j] x_k(t - d_kj)
                // the ELLPACK entries of nonzero q + 1 load while the gathers of q are
                // in flight (one iteration ahead), so the two dependent loads of a
                // gather overlap across iterations
                int2 ecur[LC];
#pragma unroll
                for (int c = 0; c < LC; ++c) {
                    const int j = r0 + ROW * (m0 + c);
                    ecur[c] = (j < n && EK > 0) ? __ldg(ell + j) : make_int2(0, 0);
                }
#pragma unroll QU
                for (int q = 0; q < EK; ++q) {
                    int2 enext[LC];
#pragma unroll
                    for (int c = 0; c < LC; ++c) {
                        const int j = r0 + ROW * (m0 + c);
                        enext[c] = (j < n && q + 1 < EK) ? __ldg(ell + (size_t)(q + 1) * n + j) : make_int2(0, 0);
                    }
#pragma unroll
                    for (int c = 0; c < LC; ++c) {
                        const int j = r0 + ROW * (m0 + c);
                        if (j >= n) continue;
                        const int2 e = ecur[c];
                        int h = hbase + e.x + (delayed ? 0 : n);
                        if (h >= hw) h -= hw;
                        const H xk = hist[(size_t)h * LN_SIMS + s];
                        if constexpr (TAN) {
                            in[c] += __int_as_float(e.y) * xk.x;
                            din[c] += __int_as_float(e.y) * xk.y;
                        } else {
                            in[c] += __int_as_float(e.y) * xk;
                        }
                    }
#pragma unroll
                    for (int c = 0; c < LC; ++c) ecur[c] = enext[c];
                }
#pragma unroll
                for (int c = 0; c < LC; ++c) {
                    const int m = m0 + c;
                    const int j = r0 + ROW * m;
                    if (j >= n) continue;
                    const long long ni =
                        ((long long)sh_ts * a.inner_it + inner) * n * M::NN + (long long)__ldg(shn + j) * M::NN;
                    const R n0 = __ldg(a.noise_f32 + ni);
                    const R n1 = (M::NN > 1) ? __ldg(a.noise_f32 + ni + 1) : R(0);
                    R r[M::NR];
#pragma unroll
                    for (int q = 0; q < M::NR; ++q) r[q] = __ldg(par + ((size_t)j * M::NR + q) * LN_SIMS + s);
                    if constexpr (TAN) TG::step(st[m], dst[m], iv, g, r, in[c], din[c], n0, n1, a.K);
                    else M::step(st[m], iv, g, r, in[c], n0, n1, a.K);
                    if (out_now) lanes_states_out<M::NS>(a, st[m], sim, j, states_i);
                }
            }
#pragma unroll
            for (int m = 0; m < MN; ++m) {
                const int j = r0 + ROW * m;
                if (j < n) hist[((size_t)hbase + j) * LN_SIMS + s] = hval<TAN>(st[m][M::CONN], dst[m][TAN ? TG::CONN_T : 0]);
            }
            __syncthreads();  // this step's slot is written before the next step reads it
            buff = buff ? buff - 1 : D;
        }
        // Balloon-Windkessel (bw.cu:4-15), BOLD at TR (bnm.cpp:316-335)
        const bool tr = (bw_i + 1) % a.bold_tr_iters == 0;
#pragma unroll
        for (int m = 0; m < MN; ++m) {
            const int j = r0 + ROW * m;
            if (j >= n || !live) continue;
            double *bj = bws + (size_t)j * BWW * LN_SIMS + s;
            double x = bj[0], f = bj[LN_SIMS], nu = bj[2 * LN_SIMS], q = bj[3 * LN_SIMS];
            if constexpr (TAN) {
                double dx = bj[4 * LN_SIMS], df = bj[5 * LN_SIMS], dnu = bj[6 * LN_SIMS], dq = bj[7 * LN_SIMS];
                bw_tangent64(x, f, nu, q, dx, df, dnu, dq, (double)dst[m][TG::CONN_T], bw);
                bj[4 * LN_SIMS] = dx;
                bj[5 * LN_SIMS] = df;
                bj[6 * LN_SIMS] = dnu;
                bj[7 * LN_SIMS] = dq;
                bw_step64(x, f, nu, q, (double)st[m][M::BOLDV], bw);
                if (tr && bold_i < a.bold_len)  // dBOLD = V0 (-k1 dq - k2 (dq / nu - q dnu / nu^2) - k3 dnu)
                    a.tan_bold[(size_t)sim * a.bold_len * n + (size_t)bold_i * n + j] =
                        -bw.V0k1 * dq - bw.V0k2 * (dq / nu - q * dnu / (nu * nu)) - bw.V0k3 * dnu;
            } else {
                bw_step64(x, f, nu, q, (double)st[m][M::BOLDV], bw);
            }
            bj[0] = x;
            bj[LN_SIMS] = f;
            bj[2 * LN_SIMS] = nu;
            bj[3 * LN_SIMS] = q;
            if (tr && bold_i < a.bold_len)  // no slot for a sample past bold_len
                bold[(size_t)bold_i * n + j] = bold64(q, nu, bw);
        }
        if (tr) bold_i++;
        if (sample) states_i++;
        if ((bw_i + 1) % a.noise_bw_it == 0 && bw_i + 1 < a.bw_it) {
            repeat++;
            shn = a.sh_nodes + (size_t)repeat * n;
        }
    }
    if (live && a.ext_out && !a.states_ts) {
        const int pts = states_i - a.n_states_samples_remove;
#pragma unroll
        for (int m = 0; m < MN; ++m) {
            const int j = r0 + ROW * m;
            if (j >= n) continue;
            for (int v = 0; v < M::NS; ++v) a.states[((size_t)v * a.n_sims + sim) * ext + j] /= pts;
        }
    }
    __syncthreads();  // the next group reuses the ring buffer and the Balloon-Windkessel scratch
}

// One run: CTA b integrates groups b, b + grid, ... of the run.
template <class M, int NT, int MN, bool DELAY, bool TAN>
__global__ void __launch_bounds__(NT, 1024 / NT) k_integrate_lanes(const __grid_constant__ IntegrateArgs a) {
    using H = typename std::conditional<TAN, float2, float>::type;
    H *hist = reinterpret_cast<H *>(a.ln_hist + (size_t)blockIdx.x * a.ln_hist_per_cta);
    double *bws = a.ln_bw + (size_t)blockIdx.x * a.nodes * (TAN ? 8 : 4) * LN_SIMS;
    for (int gi = blockIdx.x; gi < a.ln_n_groups; gi += gridDim.x)
        lanes_group<M, NT, MN, DELAY ? 1 : 0, TAN>(a, gi, hist, bws);
}

// Several runs in one launch (the groups of an uneven batch): a work queue of
// (run, group) items, longest first, taken by persistent CTAs from an atomic
// counter; the run's arguments are copied into shared memory per item.  The
// ring-buffer and Balloon-Windkessel scratch are per CTA, sized for the largest run.
template <class M, int NT, int MN>
__global__ void __launch_bounds__(NT, 1024 / NT)
    k_integrate_lanes_multi(const IntegrateArgs *runs, const int2 *items, int n_items, int *counter, float *hist,
                            long long hist_per_cta, double *bw, long long bw_per_cta) {
    __shared__ IntegrateArgs sa;
    __shared__ int s_item;
    float *h = hist + (size_t)blockIdx.x * hist_per_cta;
    double *b = bw + (size_t)blockIdx.x * bw_per_cta;
    while (true) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const int2 w = items[it];
        const int *src = reinterpret_cast<const int *>(runs + w.x);
        int *dst = reinterpret_cast<int *>(&sa);
        for (int k = threadIdx.x; k < (int)(sizeof(IntegrateArgs) / sizeof(int)); k += blockDim.x) dst[k] = src[k];
        __syncthreads();
        lanes_group<M, NT, MN, 2, false>(sa, w.y, h, b);
        __syncthreads();  // the next item reuses the scratch and the shared arguments
    }
}

// Parameters of every group in the lane layout: out[g][j][q][s] = (float)
// regional[q][sim(g, s)][j] (zero for empty lanes).
template <int NR>
__global__ void k_lanes_params(const IntegrateArgs a, float *out) {
    constexpr int nr = NR;
    const int g = blockIdx.x;
    const int n = a.nodes;
    const int *gd = a.ln_groups + (size_t)g * (3 + LN_SIMS);
    const size_t rstride = (size_t)a.n_sims * n;
    for (int e = threadIdx.x; e < n * nr * LN_SIMS; e += blockDim.x) {
        const int s = e % LN_SIMS, q = (e / LN_SIMS) % nr, j = e / (LN_SIMS * nr);
        const int sim = gd[3 + s];
        out[(size_t)g * n * nr * LN_SIMS + e] = sim >= 0 ? (float)a.rparams[q * rstride + (size_t)sim * n + j] : 0.0f;
    }
}

// Launch of the (model, rows, tangent) instantiation for this run.
template <class M, int NT, int MN, bool TAN>
cudaError_t launch_mn(const IntegrateArgs &a, cudaStream_t st) {
    const int grid = std::min(a.ln_n_groups, a.ln_grid);
    if (a.has_delay) k_integrate_lanes<M, NT, MN, true, TAN><<<grid, NT, 0, st>>>(a);
    else k_integrate_lanes<M, NT, MN, false, TAN><<<grid, NT, 0, st>>>(a);
    return cudaGetLastError();
}

template <class M>
cudaError_t launch_params(const IntegrateArgs &a, cudaStream_t st) {
    k_lanes_params<M::NR><<<a.ln_n_groups, 256, 0, st>>>(a, a.ln_params);
    return cudaGetLastError();
}

template <class M, bool TAN>
cudaError_t launch_model(const IntegrateArgs &a, cudaStream_t st) {
    k_lanes_params<M::NR><<<a.ln_n_groups, 256, 0, st>>>(a, a.ln_params);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (a.ln_threads == 512) {  // 32 node rows a CTA, two CTAs an SM: networks of <= 128 nodes
        switch (lanes_rows(a.nodes, 512)) {
            case 1: return launch_mn<M, 512, 1, TAN>(a, st);
            case 2: return launch_mn<M, 512, 2, TAN>(a, st);
            case 4: return launch_mn<M, 512, 4, TAN>(a, st);
        }
        return cudaErrorInvalidValue;
    }
    switch (lanes_rows(a.nodes, 1024)) {
        case 1: return launch_mn<M, 1024, 1, TAN>(a, st);
        case 2: return launch_mn<M, 1024, 2, TAN>(a, st);
        case 4: return launch_mn<M, 1024, 4, TAN>(a, st);
        case 8:
            if constexpr (M::NS <= 6) return launch_mn<M, 1024, 8, TAN>(a, st);
            break;
        case 16:
            if constexpr (M::NS <= 6) return launch_mn<M, 1024, 16, TAN>(a, st);
            break;
    }
    return cudaErrorInvalidValue;
}

template <class M>
cudaError_t launch_multi(const IntegrateArgs *runs, const int2 *items, int n_items, int *counter, int mn, int grid,
                         float *hist, long long hist_per_cta, double *bw, long long bw_per_cta, cudaStream_t st) {
#define CBNM_LANES_MULTI(MNV) \
    k_integrate_lanes_multi<M, 1024, MNV><<<grid, 1024, 0, st>>>(runs, items, n_items, counter, hist, hist_per_cta, bw, bw_per_cta)
    switch (mn) {
        case 1: CBNM_LANES_MULTI(1); break;
        case 2: CBNM_LANES_MULTI(2); break;
        case 4: CBNM_LANES_MULTI(4); break;
        case 8:
            if constexpr (M::NS <= 6) { CBNM_LANES_MULTI(8); break; }
            return cudaErrorInvalidValue;
        case 16:
            if constexpr (M::NS <= 6) { CBNM_LANES_MULTI(16); break; }
            return cudaErrorInvalidValue;
        default: return cudaErrorInvalidValue;
    }
#undef CBNM_LANES_MULTI
    return cudaGetLastError();
}

}  // namespace lanes
}  // namespace cbnm
