// Device helpers shared by the tensor-core integrators (integrate_fp32.cu,
// integrate_pp.cu): tcgen05 / mbarrier wrappers written as inline PTX, the FP32
// model steps and the FP64 Balloon-Windkessel step.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include "engine.h"

namespace cbnm {
namespace {

constexpr int TM = 128;                                // node lanes (MMA M)
constexpr long long WAIT_LIMIT_CYCLES = 4000000000LL;  // about 2 s at 1.9 GHz

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

__device__ __forceinline__ void tmem_ld2(uint32_t taddr, uint32_t (&r)[2]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];\n" : "=r"(r[0]), "=r"(r[1]) : "r"(taddr) : "memory");
}
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, uint32_t (&r)[4]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr)
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_st8_nowait(uint32_t taddr, const uint32_t (&r)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};\n" ::"r"(taddr), "r"(r[0]),
                 "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(mbar) : "memory");
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
    __host__ __device__ static K make(const ModelK &m) {
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
using BW64 = BWFast;
static_assert(sizeof(BWFast::binom) == sizeof(double) * (BINOM_TERMS + 1), "binomial terms");

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

// Every multiply-add below is spelled out (fma / __dmul_rn / __dadd_rn), so the
// compiler's contraction choices, which can differ between the kernels this is
// inlined into, never change a bit of the result: the same inputs give the same
// BOLD in every integrator that uses it.
__device__ __forceinline__ void bw_step64(double &x, double &f, double &nu, double &q, double z, const BW64 &c) {
    double t = fma(-c.kappa, x, z);
    t = fma(-c.y, __dsub_rn(f, 1.0), t);
    x = fma(c.dt, t, x);
    const double tmp_f = fma(c.dt, x, f);
    const double inv_f = rcp_fast(f);
    nu = fma(c.dt_itau, __dsub_rn(f, pow_nu(nu, c)), nu);
    const double in = __dmul_rn(__dmul_rn(f, __dsub_rn(1.0, pow_omr(f, inv_f, c))), c.irho);
    const double out = __dmul_rn(__dmul_rn(pow_nu(nu, c), q), rcp_fast(nu));
    q = fma(c.dt_itau, __dsub_rn(in, out), q);
    f = tmp_f;
}

// BOLD = V0 (k1 (1 - q) + k2 (1 - q / nu) + k3 (1 - nu))  (bnm.cpp:316-335)
__device__ __forceinline__ double bold64(double q, double nu, const BW64 &c) {
    double b = __dmul_rn(c.V0k1, __dsub_rn(1.0, q));
    b = fma(c.V0k2, __dsub_rn(1.0, __ddiv_rn(q, nu)), b);
    return fma(c.V0k3, __dsub_rn(1.0, nu), b);
}

__device__ __forceinline__ void bw_step64x2(double (&x)[2], double (&f)[2], double (&nu)[2], double (&q)[2],
                                            double z0, double z1, const BW64 &c) {
    const double z[2] = {z0, z1};
#pragma unroll
    for (int u = 0; u < 2; ++u) bw_step64(x[u], f[u], nu[u], q[u], z[u], c);
}

// The same step with the multiply-adds left to the compiler.  The two-tile
// kernel runs at its 96-register limit, where this form spills less; its
// results may differ from bw_step64 in the last bits.
__device__ __forceinline__ void bw_step64_contracted(double &x, double &f, double &nu, double &q, double z,
                                                     const BW64 &c) {
    x = x + c.dt * (z - c.kappa * x - c.y * (f - 1.0));
    const double tmp_f = f + c.dt * x;
    const double inv_f = rcp_fast(f);
    nu = nu + c.dt_itau * (f - pow_nu(nu, c));
    q = q + c.dt_itau * (f * (1.0 - pow_omr(f, inv_f, c)) * c.irho - pow_nu(nu, c) * q * rcp_fast(nu));
    f = tmp_f;
}

}  // namespace
}  // namespace cbnm
