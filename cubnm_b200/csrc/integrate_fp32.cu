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

namespace cbnm {
namespace {

constexpr int TM = 128;              // node lanes (MMA M)
constexpr int COL_ACC = 0;           // accumulator columns start here
constexpr int COL_BW = 32;           // TN x 8 words of Balloon-Windkessel state start here

// Tile geometry: TN simulations per tile (MMA N), SPT simulations per thread,
// TN/SPT warpgroups per CTA.
template <int TN_, int SPT_, int NACC_>
struct Tile {
    static constexpr int TN = TN_;
    static constexpr int SPT = SPT_;
    static constexpr int NACC = NACC_;   // independent accumulator sets the GEMM round-robins over
    static constexpr int NWG = TN / SPT;
    static constexpr int NTHREADS = NWG * 128;
    static constexpr int TMEM_COLS = (COL_BW + TN * 8 <= 256) ? 256 : 512;
    static constexpr int CTAS_PER_SM = 512 / TMEM_COLS;
    static constexpr uint32_t LBO_B = (TN / 8) * 128;
    // threads that issue the step's GEMM: 1 (all MMAs, round-robin over the NACC sets)
    // or NACC (thread p of warp p issues pass p of BF16x3 into accumulator set p)
    static constexpr int ISSUERS = (NACC == 3) ? 3 : 1;
};
constexpr long long WAIT_LIMIT_CYCLES = 4000000000LL;  // about 2 s at 1.9 GHz

struct Smem {
    uint64_t mbar;
    uint32_t tmem_base;
    int abort;
    int sc_loaded;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);  // version 1, no swizzle
}

// kind::f16 instruction descriptor: D F32, A/B BF16, A K-major, B MN-major, N, M.
__host__ __device__ constexpr uint32_t instr_desc(int TN) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (0u << 15) | (1u << 16) | ((uint32_t)(TN >> 3) << 17) |
           ((uint32_t)(TM >> 4) << 24);
}

// A from TMEM (row m on lane m, two BF16 per 32-bit column), B from SMEM.
__device__ __forceinline__ void mma_bf16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

// Bounded wait on the MMA barrier: each try_wait sleeps the warp until the
// phase completes or the hint (ns) expires, so waiting warps do not spin.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
    uint32_t ok = 0;
    asm volatile(
        "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(phase), "r"(1000000u)
        : "memory");
    if (ok) return true;
    const long long t0 = clock64();
    while (true) {
        asm volatile(
            "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, P;\n\t}\n"
            : "=r"(ok)
            : "r"(mbar), "r"(phase), "r"(1000000u)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > WAIT_LIMIT_CYCLES) return false;
    }
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
        : "r"(taddr)
        : "memory");
}

template <int W>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&r)[W]) {
    static_assert(W == 8, "accumulator reads are 8 columns wide");
    tmem_ld8(taddr, r);
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};\n\t"
        "tcgen05.wait::st.sync.aligned;\n" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
        : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};\n\t"
        "tcgen05.wait::st.sync.aligned;\n" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

// split v = hi + lo (+ residual below 2^-16 |v|), two values at once: packed hi and lo pairs
__device__ __forceinline__ void split_bf16x2(float v0, float v1, uint32_t &hi, uint32_t &lo) {
    __nv_bfloat162 h = __floats2bfloat162_rn(v0, v1);
    const float2 hf = __bfloat1622float2(h);
    __nv_bfloat162 l = __floats2bfloat162_rn(v0 - hf.x, v1 - hf.y);
    hi = *reinterpret_cast<uint32_t *>(&h);
    lo = *reinterpret_cast<uint32_t *>(&l);
}

// ---------------------------------------------------------------- models (FP32)
// rate r = x / (1 - exp(-d x)).  Near the removable singularity x = 0 the
// direct form loses ~1e-7/|y| relative (y = d x); below |y| = 1e-3 the series
// (1/d)(1 + y/2) is used instead (truncation y^2/12 < 1e-7).
__device__ __forceinline__ float rate_fn(float x, float d, float inv_d) {
    const float y = d * x;
    const float big = __fdividef(x, 1.0f - __expf(-y));
    const float small = inv_d * fmaf(0.5f, y, 1.0f);
    return fabsf(y) < 1e-3f ? small : big;
}

// ---- packed FP32x2 helpers (two simulations per instruction, sm_100 FFMA2 / FADD2 / FMUL2)
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// rate r = x / (1 - exp(-d x)) for a pair; ml2d = -d log2(e).  Near x = 0 the series
// (1/d)(1 + y/2) (y = d x) replaces the direct form (see rate_fn).
__device__ __forceinline__ float2 rate2(float2 x, float d, float id, float ml2d) {
    const float2 t = __fmul2_rn(x, f2(ml2d));
    const float2 e = make_float2(ex2_approx(t.x), ex2_approx(t.y));
    const float2 den = __ffma2_rn(e, f2(-1.0f), f2(1.0f));
    const float2 big = __fmul2_rn(x, make_float2(rcp_approx(den.x), rcp_approx(den.y)));
    const float2 y = __fmul2_rn(x, f2(d));
    const float2 small = __fmul2_rn(__ffma2_rn(y, f2(0.5f), f2(1.0f)), f2(id));
    return make_float2(fabsf(y.x) < 1e-3f ? small.x : big.x, fabsf(y.y) < 1e-3f ? small.y : big.y);
}

struct RWW32 {  // rww.cpp:194-232 in FP32
    static constexpr int NP = 5, NS = 2, NN = 2, NOUT = 6, CV = 0, BV = 0;
    struct K { float wEI0, wII0, aE, bE, dE, idE, aI, bI, dI, idI, wII, dgE, ditE, dgI, ditI, sqdt, ml2dE, ml2dI; };
    __device__ static K make(const ModelK &m) {
        const RWWK &r = m.rww;
        K k;
        k.ml2dE = (float)(-r.d_E * 1.4426950408889634); k.ml2dI = (float)(-r.d_I * 1.4426950408889634);
        k.wEI0 = (float)r.w_E__I_0; k.wII0 = (float)r.w_I__I_0; k.aE = (float)r.a_E; k.bE = (float)r.b_E;
        k.dE = (float)r.d_E; k.idE = (float)(1.0 / r.d_E); k.aI = (float)r.a_I; k.bI = (float)r.b_I;
        k.dI = (float)r.d_I; k.idI = (float)(1.0 / r.d_I); k.wII = (float)r.w_II; k.dgE = (float)r.dt_gamma_E;
        k.ditE = (float)r.dt_itau_E; k.dgI = (float)r.dt_gamma_I; k.ditI = (float)r.dt_itau_I;
        k.sqdt = (float)r.sqrt_dt;
        return k;
    }
    // params: w_p*J_N, G*J_N, J_N, wIE, sigma*sqrt(dt)
    __device__ static void params(float *p, double G, const double *r, const K &k) {
        p[0] = (float)(r[0] * r[1]); p[1] = (float)(G * r[1]); p[2] = (float)r[1]; p[3] = (float)r[2];
        p[4] = (float)r[3] * k.sqdt;
    }
    __device__ static void init(float *s) { s[0] = 0.001f; s[1] = 0.001f; }
    // One Euler step for a pair of simulations, state / params packed as float2 so that
    // every multiply-add is one FFMA2 (p[3] holds -wIE in this form, see pair_params):
    //   I_E = wEI0 + w_p J_N S_E + G J_N in - wIE S_I,  I_I = wII0 + J_N S_E - wII S_I,
    //   S_E += sigma sqrt(dt) n0 + dt gamma_E (1 - S_E) r_E - dt/tau_E S_E   (clamped to [0, 1]),
    //   S_I += sigma sqrt(dt) n1 + dt gamma_I r_I - dt/tau_I S_I            (clamped to [0, 1]).
    // Both simulations share the node's noise.
    static constexpr bool PAIR = true;
    __device__ static void pair_params(float2 *p) { p[3] = make_float2(-p[3].x, -p[3].y); }
    __device__ static void step2(float2 *s, const float2 *p, float2 in, float n0, float n1, const K &k, float2 *o) {
        const float2 sE = s[0], sI = s[1];
        float2 IE = __ffma2_rn(p[0], sE, f2(k.wEI0));
        IE = __ffma2_rn(p[1], in, IE);
        IE = __ffma2_rn(p[3], sI, IE);
        float2 II = __ffma2_rn(p[2], sE, f2(k.wII0));
        II = __ffma2_rn(f2(-k.wII), sI, II);
        const float2 rE = rate2(__ffma2_rn(f2(k.aE), IE, f2(-k.bE)), k.dE, k.idE, k.ml2dE);
        const float2 rI = rate2(__ffma2_rn(f2(k.aI), II, f2(-k.bI)), k.dI, k.idI, k.ml2dI);
        float2 dE = __fmul2_rn(f2(n0), p[4]);
        dE = __ffma2_rn(f2(k.dgE), __fmul2_rn(__ffma2_rn(sE, f2(-1.0f), f2(1.0f)), rE), dE);
        dE = __ffma2_rn(f2(-k.ditE), sE, dE);
        float2 dI = __ffma2_rn(f2(k.dgI), rI, __fmul2_rn(f2(n1), p[4]));
        dI = __ffma2_rn(f2(-k.ditI), sI, dI);
        const float2 nE = __fadd2_rn(sE, dE), nI = __fadd2_rn(sI, dI);
        s[0] = make_float2(__saturatef(nE.x), __saturatef(nE.y));
        s[1] = make_float2(__saturatef(nI.x), __saturatef(nI.y));
        o[0] = IE; o[1] = II; o[2] = rE; o[3] = rI; o[4] = s[0]; o[5] = s[1];
    }
};

// Pair form for models without a packed step: two scalar steps.
template <class M, bool = M::PAIR>
struct PairStep {
    __device__ static void params(float2 *) {}
    __device__ static void step(float2 *s, const float2 *p, float2 in, float n0, float n1, const typename M::K &k,
                                float2 *o) {
        float sa[M::NS], sb[M::NS], pa[M::NP], pb[M::NP], oa[M::NOUT], ob[M::NOUT];
#pragma unroll
        for (int q = 0; q < M::NS; ++q) { sa[q] = s[q].x; sb[q] = s[q].y; }
#pragma unroll
        for (int q = 0; q < M::NP; ++q) { pa[q] = p[q].x; pb[q] = p[q].y; }
        M::step(sa, pa, in.x, n0, n1, k, oa);
        M::step(sb, pb, in.y, n0, n1, k, ob);
#pragma unroll
        for (int q = 0; q < M::NS; ++q) s[q] = make_float2(sa[q], sb[q]);
#pragma unroll
        for (int q = 0; q < M::NOUT; ++q) o[q] = make_float2(oa[q], ob[q]);
    }
};
template <class M>
struct PairStep<M, true> {
    __device__ static void params(float2 *p) { M::pair_params(p); }
    __device__ static void step(float2 *s, const float2 *p, float2 in, float n0, float n1, const typename M::K &k,
                                float2 *o) {
        M::step2(s, p, in, n0, n1, k, o);
    }
};

struct WC32 {  // wc.cpp:51-80 in FP32
    static constexpr bool PAIR = false;
    static constexpr int NP = 9, NS = 2, NN = 2, NOUT = 2, CV = 0, BV = 0;
    struct K { float dt, sqdt, itE, itI, aE, aI, muE, muI; };
    __device__ static K make(const ModelK &m) {
        const WCK &w = m.wc;
        return K{(float)w.dt, (float)w.sqrt_dt, (float)w.itau_E, (float)w.itau_I, (float)w.a_E, (float)w.a_I,
                 (float)w.mu_E, (float)w.mu_I};
    }
    __device__ static void params(float *p, double G, const double *r, const K &k) {
        p[0] = (float)r[0]; p[1] = (float)r[1]; p[2] = (float)r[2]; p[3] = (float)r[3];
        p[4] = (float)r[4]; p[5] = (float)r[5]; p[6] = (float)r[6] * k.sqdt; p[7] = (float)r[7] * k.sqdt;
        p[8] = (float)G;
    }
    __device__ static void init(float *s) { s[0] = 0.001f; s[1] = 0.001f; }
    __device__ static void step(float *s, const float *p, float in, float n0, float n1, const K &k, float *o) {
        const float SE = __fdividef(1.0f, 1.0f + __expf(-k.aE * (p[0] * s[0] - p[1] * s[1] + p[8] * in + p[4] - k.muE)));
        const float SI = __fdividef(1.0f, 1.0f + __expf(-k.aI * (p[2] * s[0] - p[3] * s[1] + p[5] - k.muI)));
        const float Ed = (-s[0] + (1.0f - s[0]) * SE) * k.itE;
        const float Id = (-s[1] + (1.0f - s[1]) * SI) * k.itI;
        s[0] = __saturatef(s[0] + (k.dt * Ed + n0 * p[6]));
        s[1] = __saturatef(s[1] + (k.dt * Id + n1 * p[7]));
        o[0] = s[0]; o[1] = s[1];
    }
};

struct RWWEx32 {  // rwwex.cpp:48-73 in FP32
    static constexpr bool PAIR = false;
    static constexpr int NP = 4, NS = 1, NN = 1, NOUT = 3, CV = 0, BV = 0;
    struct K { float JN, a, b, d, id, dit, dg, sqdt; };
    __device__ static K make(const ModelK &m) {
        const RWWExK &w = m.rwwex;
        return K{(float)w.J_N, (float)w.a, (float)w.b, (float)w.d, (float)(1.0 / w.d), (float)w.dt_itau,
                 (float)w.dt_gamma, (float)w.sqrt_dt};
    }
    __device__ static void params(float *p, double G, const double *r, const K &k) {
        p[0] = (float)(r[0] * k.JN); p[1] = (float)(G * k.JN); p[2] = (float)r[1]; p[3] = (float)r[2] * k.sqdt;
    }
    __device__ static void init(float *s) { s[0] = 0.001f; }
    __device__ static void step(float *s, const float *p, float in, float n0, float, const K &k, float *o) {
        const float x = p[0] * s[0] + p[1] * in + p[2];
        const float r = rate_fn(k.a * x - k.b, k.d, k.id);
        s[0] = __saturatef(s[0] + (k.dg * ((1.0f - s[0]) * r) - k.dit * s[0] + n0 * p[3]));
        o[0] = x; o[1] = r; o[2] = s[0];
    }
};

struct JR32 {  // jr.cpp:80-133 in FP32
    static constexpr bool PAIR = false;
    static constexpr int NP = 7, NS = 8, NN = 1, NOUT = 8, CV = 7, BV = 6;
    struct K { float dt, sqdt, A, B, a, b, v0, numax2, r, mu, cmin, cmax, mid, asq, bsq; };
    __device__ static K make(const ModelK &m) {
        const JRK &j = m.jr;
        return K{(float)j.dt, (float)j.sqrt_dt, (float)j.A, (float)j.B, (float)j.a, (float)j.b, (float)j.v0,
                 (float)(2.0 * j.nu_max), (float)j.r, (float)j.mu, (float)j.cmin, (float)j.cmax, (float)j.midpoint,
                 (float)j.a_sq, (float)j.b_sq};
    }
    // a_1 J, a_2 J, a_3 J, a_4 J, sigma sqrt(dt), G, unused
    __device__ static void params(float *p, double G, const double *r, const K &k) {
        p[0] = (float)(r[1] * r[0]); p[1] = (float)(r[2] * r[0]); p[2] = (float)(r[3] * r[0]);
        p[3] = (float)(r[4] * r[0]); p[4] = (float)r[5] * k.sqdt; p[5] = (float)G; p[6] = 0.0f;
    }
    __device__ static void init(float *s) { for (int i = 0; i < 8; ++i) s[i] = 0.0f; }
    __device__ static void step(float *s, const float *p, float in, float n0, float, const K &k, float *o) {
        const float s12 = __fdividef(k.numax2, 1.0f + __expf(k.r * (k.v0 - (s[1] - s[2]))));
        const float s01 = __fdividef(k.numax2, 1.0f + __expf(k.r * (k.v0 - p[0] * s[0])));
        const float s03 = __fdividef(k.numax2, 1.0f + __expf(k.r * (k.v0 - p[2] * s[0])));
        const float d3 = k.A * k.a * s12 - 2.0f * k.a * s[3] - k.asq * s[0];
        const float d4 = k.A * k.a * (k.mu + p[1] * s01 + p[5] * in) - 2.0f * k.a * s[4] - k.asq * s[1];
        const float d5 = k.B * k.b * (p[3] * s03) - 2.0f * k.b * s[5] - k.bsq * s[2];
        s[0] += k.dt * s[3];
        s[1] += k.dt * s[4];
        s[2] += k.dt * s[5];
        s[3] += k.dt * d3 + n0 * p[4];
        s[4] += k.dt * d4;
        s[5] += k.dt * d5;
        s[6] = s[1] - s[2];
        s[7] = k.cmin + __fdividef(k.cmax - k.cmin, 1.0f + __expf(k.r * (k.mid - s[6])));
        for (int i = 0; i < 8; ++i) o[i] = s[i];
    }
};

// Balloon-Windkessel step in FP64 (bw.cu:4-15).
// The powers nu^(1/alpha) and (1-rho)^(1/f) and two divisions dominate its
// cost.  In the range the haemodynamic state lives in (|nu-1|, |f-1| <= 1/8):
//   nu^a       = sum_{k<=12} C(a,k) d^k, d = nu - 1 (binomial series; the
//                coefficients C(a,k) are computed once on the host; error <= 3 ulp)
//   (1-rho)^(1/f) = (1-rho) exp(ln(1-rho) (1-f)/f), exp by its Taylor series to
//                y^10/10!, |y| <= 0.06 (first omitted term < 1e-18)
//   1/x        = float reciprocal refined by two Newton steps (<= 1 ulp)
// Outside that range the general exp2 / log2 forms and IEEE division are used.
constexpr int BINOM_TERMS = 12;
struct BW64 {
    double dt, kappa, y, dt_itau, ialpha, irho, log2_omr, ln_omr, omr, V0k1, V0k2, V0k3;
    double binom[BINOM_TERMS + 1];
};

__device__ __forceinline__ double rcp_fast(double x) {
    double r = (double)__frcp_rn((float)x);
    r = r * fma(-x, r, 2.0);
    return r * fma(-x, r, 2.0);
}

__device__ __forceinline__ double exp_tiny(double y) {  // sum_{k<=10} y^k / k!
    double p = 1.0 / 3628800.0;
    p = fma(p, y, 1.0 / 362880.0);
    p = fma(p, y, 1.0 / 40320.0);
    p = fma(p, y, 1.0 / 5040.0);
    p = fma(p, y, 1.0 / 720.0);
    p = fma(p, y, 1.0 / 120.0);
    p = fma(p, y, 1.0 / 24.0);
    p = fma(p, y, 1.0 / 6.0);
    p = fma(p, y, 0.5);
    p = fma(p, y, 1.0);
    return fma(p, y, 1.0);
}

__device__ __forceinline__ double pow_nu(double nu, const BW64 &c) {  // nu^(1/alpha)
    const double d = nu - 1.0;
    if (fabs(d) <= 0.125) {
        double p = c.binom[BINOM_TERMS];
#pragma unroll
        for (int k = BINOM_TERMS - 1; k >= 0; --k) p = fma(p, d, c.binom[k]);
        return p;
    }
    return exp2(c.ialpha * log2(nu));
}

__device__ __forceinline__ double pow_omr(double f, double inv_f, const BW64 &c) {  // (1-rho)^(1/f)
    if (fabs(f - 1.0) <= 0.125) return c.omr * exp_tiny(c.ln_omr * ((1.0 - f) * inv_f));
    return exp2(c.log2_omr / f);
}

__device__ __forceinline__ void bw_step64(double &x, double &f, double &nu, double &q, double z, const BW64 &c) {
    x = x + c.dt * (z - c.kappa * x - c.y * (f - 1.0));
    const double tmp_f = f + c.dt * x;
    const double inv_f = rcp_fast(f);
    nu = nu + c.dt_itau * (f - pow_nu(nu, c));
    q = q + c.dt_itau * (f * (1.0 - pow_omr(f, inv_f, c)) * c.irho - pow_nu(nu, c) * q * rcp_fast(nu));
    f = tmp_f;
}

__device__ __forceinline__ void bw_step64x2(double (&x)[2], double (&f)[2], double (&nu)[2], double (&q)[2],
                                            double z0, double z1, const BW64 &c) {
    const double z[2] = {z0, z1};
#pragma unroll
    for (int u = 0; u < 2; ++u) bw_step64(x[u], f[u], nu[u], q[u], z[u], c);
}

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
    BW64 bw;
    bw.dt = a.bw.dt; bw.kappa = a.bw.kappa; bw.y = a.bw.y; bw.dt_itau = a.bw.dt_itau; bw.ialpha = a.bw.ialpha;
    bw.irho = 1.0 / a.bw.rho; bw.log2_omr = log2(a.bw.oneminrho); bw.ln_omr = log(a.bw.oneminrho);
    bw.omr = a.bw.oneminrho;
#pragma unroll
    for (int k = 0; k <= BINOM_TERMS; ++k) bw.binom[k] = a.bw_binom[k];
    bw.V0k1 = a.bw.V_0 * a.bw.k1; bw.V0k2 = a.bw.V_0 * a.bw.k2; bw.V0k3 = a.bw.V_0 * a.bw.k3;
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
        if (a.ext_out && !a.states_ts && act) {  // states sums start at zero
            for (int i = 0; i < SPT; ++i)
                if (sims[i] >= 0)
                    for (int v = 0; v < M::NOUT; ++v) a.states[((size_t)v * a.n_sims + sims[i]) * ext + j] = 0.0;
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
                    a.bold[(size_t)sim * a.bold_len * n + (size_t)bi * n + j] =
                        bw.V0k1 * (1 - q[u]) + bw.V0k2 * (1 - q[u] / nu[u]) + bw.V0k3 * (1 - nu[u]);
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
                                    const double ov = u ? o[v].y : o[v].x;
                                    if (a.states_ts) {
                                        if (states_i < a.states_len)
                                            a.states[((size_t)v * a.n_sims + sim) * ext + (size_t)states_i * n + j] = ov;
                                    }
                                    else if (states_i >= a.n_states_samples_remove)
                                        a.states[((size_t)v * a.n_sims + sim) * ext + j] += ov;
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
        if (a.ext_out && !a.states_ts && act && !aborted) {
            const int pts = states_i - a.n_states_samples_remove;
            for (int i = 0; i < SPT; ++i)
                if (sims[i] >= 0)
                    for (int v = 0; v < M::NOUT; ++v) a.states[((size_t)v * a.n_sims + sims[i]) * ext + j] /= pts;
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

template <class M, class T>
cudaError_t launch_tc(const IntegrateArgs &a, const int *tiles, int n_tiles, cudaStream_t st) {
    const int KP = ((a.nodes + 15) / 16) * 16;
    // shared memory large enough that no more CTAs than TMEM holds land on one SM
    const size_t floor = T::CTAS_PER_SM == 2 ? 80 * 1024 : 120 * 1024;
    const size_t smem = std::max<size_t>(smem_bytes<T>(KP), floor);
    cudaError_t e = cudaFuncSetAttribute(k_integrate_tc<M, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
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
