// FP32 / tensor-core integrator (the fast path, precision "fp32").
//
// The same time loop as the FP64 kernel (reference: src/ext/bnm.cu:117-505),
// reorganised for B200:
//
//  * A CTA integrates a tile of TN = 16 simulations that share one SC.  Node j
//    of the tile lives on TMEM lane j (M = 128 lanes, nodes <= 128); each
//    thread owns one node and SPT = 8 simulations.
//  * Coupling (bnm.cu:48-77) is a GEMM every step:
//        D[j][s] = sum_k SC[k][j] * x_k^s
//    issued as tcgen05.mma kind::f16 with A = SC^T (BF16, K-major, constant
//    for the tile) and B = x (BF16, MN-major, rewritten every step), in
//    BF16x3 split precision: D = A_hi B_hi + A_hi B_lo + A_lo B_hi, FP32
//    accumulation in TMEM.  Elementwise model updates run in FP32 registers.
//  * The Balloon-Windkessel state (bnm.cu:357-371) stays FP64 and lives in TMEM
//    (8 x 32-bit words per simulation), loaded and stored once per bw step.
//  * Two CTAs per SM: while one waits for its MMA the other runs its update.
//  * Every wait on the MMA barrier is bounded; on timeout the CTA records a
//    status, leaves its loop, frees its TMEM and returns.
//
// SMEM operand layouts (no swizzle, "canonical" 8-row x 16-byte core matrices):
//   A (K-major): element (row r, k) at (k/8)*LBO_A + (r/8)*128 + (r%8)*16 + (k%8)*2,
//                LBO_A = 128/8 * 128 = 2048 B, SBO_A = 128 B
//   B (MN-major): element (k, n) at (k/8)*LBO_B + (n/8)*128 + (k%8)*16 + (n%8)*2,
//                LBO_B = TN/8 * 128 = 256 B, SBO_B = 128 B
#include <algorithm>
#include <cstdint>
#include <cuda_bf16.h>
#include "engine.h"

namespace cbnm {
namespace {

constexpr int TN = 16;               // simulations per tile (MMA N)
constexpr int TM = 128;              // node lanes (MMA M)
constexpr int NWG = 2;               // warpgroups per CTA
constexpr int SPT = TN / NWG;        // simulations per thread
constexpr int NTHREADS = NWG * 128;
constexpr int TMEM_COLS = 256;
constexpr int COL_ACC = 0;           // TN accumulator columns
constexpr int COL_BW = 32;           // TN x 8 words of Balloon-Windkessel state
constexpr uint32_t LBO_A = (TM / 8) * 128;
constexpr uint32_t LBO_B = (TN / 8) * 128;
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
__host__ __device__ constexpr uint32_t instr_desc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (0u << 15) | (1u << 16) | ((uint32_t)(TN >> 3) << 17) |
           ((uint32_t)(TM >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
    const long long t0 = clock64();
    uint32_t ok = 0;
    while (true) {
        asm volatile(
            "{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, P;\n\t}\n"
            : "=r"(ok)
            : "r"(mbar), "r"(phase)
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

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};\n\t"
        "tcgen05.wait::st.sync.aligned;\n" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
        : "memory");
}

__device__ __forceinline__ uint16_t bf16_bits(float v) {
    __nv_bfloat16 h = __float2bfloat16_rn(v);
    return *reinterpret_cast<uint16_t *>(&h);
}
__device__ __forceinline__ float bf16_val(uint16_t b) {
    __nv_bfloat16 h = *reinterpret_cast<__nv_bfloat16 *>(&b);
    return __bfloat162float(h);
}
// split v = hi + lo (+ residual below 2^-16 |v|)
__device__ __forceinline__ void split_bf16(float v, uint16_t &hi, uint16_t &lo) {
    hi = bf16_bits(v);
    lo = bf16_bits(v - bf16_val(hi));
}

// ---------------------------------------------------------------- models (FP32)
// rate r = x / (1 - exp(-d x)), with the removable singularity at x = 0 taken
// by its series (1/d)(1 + y/2 + y^2/12 - y^4/720), y = d x, when |y| < 0.1.
__device__ __forceinline__ float rate_fn(float x, float d, float inv_d) {
    const float y = d * x;
    const float big = __fdividef(x, 1.0f - __expf(-y));
    const float y2 = y * y;
    const float small = inv_d * (1.0f + 0.5f * y + y2 * (1.0f / 12.0f) - y2 * y2 * (1.0f / 720.0f));
    return fabsf(y) < 0.1f ? small : big;
}

struct RWW32 {  // rww.cpp:194-232 in FP32
    static constexpr int NP = 5, NS = 2, NN = 2, NOUT = 6;
    struct K { float wEI0, wII0, aE, bE, dE, idE, aI, bI, dI, idI, wII, dgE, ditE, dgI, ditI, sqdt; };
    __device__ static K make(const ModelK &m) {
        const RWWK &r = m.rww;
        K k;
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
    __device__ static float conn(const float *s) { return s[0]; }
    __device__ static float bold_in(const float *s) { return s[0]; }
    __device__ static void step(float *s, const float *p, float in, float n0, float n1, const K &k, float *o) {
        const float IE = k.wEI0 + p[0] * s[0] + p[1] * in - p[3] * s[1];
        const float II = k.wII0 + p[2] * s[0] - k.wII * s[1];
        const float rE = rate_fn(k.aE * IE - k.bE, k.dE, k.idE);
        const float rI = rate_fn(k.aI * II - k.bI, k.dI, k.idI);
        float sE = s[0] + (n0 * p[4] + k.dgE * ((1.0f - s[0]) * rE) - k.ditE * s[0]);
        float sI = s[1] + (n1 * p[4] + k.dgI * rI - k.ditI * s[1]);
        s[0] = fminf(fmaxf(sE, 0.0f), 1.0f);
        s[1] = fminf(fmaxf(sI, 0.0f), 1.0f);
        o[0] = IE; o[1] = II; o[2] = rE; o[3] = rI; o[4] = s[0]; o[5] = s[1];
    }
};

struct WC32 {  // wc.cpp:51-80 in FP32
    static constexpr int NP = 9, NS = 2, NN = 2, NOUT = 2;
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
    __device__ static float conn(const float *s) { return s[0]; }
    __device__ static float bold_in(const float *s) { return s[0]; }
    __device__ static void step(float *s, const float *p, float in, float n0, float n1, const K &k, float *o) {
        const float SE = __fdividef(1.0f, 1.0f + __expf(-k.aE * (p[0] * s[0] - p[1] * s[1] + p[8] * in + p[4] - k.muE)));
        const float SI = __fdividef(1.0f, 1.0f + __expf(-k.aI * (p[2] * s[0] - p[3] * s[1] + p[5] - k.muI)));
        const float Ed = (-s[0] + (1.0f - s[0]) * SE) * k.itE;
        const float Id = (-s[1] + (1.0f - s[1]) * SI) * k.itI;
        s[0] = fminf(fmaxf(s[0] + (k.dt * Ed + n0 * p[6]), 0.0f), 1.0f);
        s[1] = fminf(fmaxf(s[1] + (k.dt * Id + n1 * p[7]), 0.0f), 1.0f);
        o[0] = s[0]; o[1] = s[1];
    }
};

struct RWWEx32 {  // rwwex.cpp:48-73 in FP32
    static constexpr int NP = 4, NS = 1, NN = 1, NOUT = 3;
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
    __device__ static float conn(const float *s) { return s[0]; }
    __device__ static float bold_in(const float *s) { return s[0]; }
    __device__ static void step(float *s, const float *p, float in, float n0, float, const K &k, float *o) {
        const float x = p[0] * s[0] + p[1] * in + p[2];
        const float r = rate_fn(k.a * x - k.b, k.d, k.id);
        const float S = s[0] + (k.dg * ((1.0f - s[0]) * r) - k.dit * s[0] + n0 * p[3]);
        s[0] = fminf(fmaxf(S, 0.0f), 1.0f);
        o[0] = x; o[1] = r; o[2] = s[0];
    }
};

struct JR32 {  // jr.cpp:80-133 in FP32
    static constexpr int NP = 7, NS = 8, NN = 1, NOUT = 8;
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
    __device__ static float conn(const float *s) { return s[7]; }
    __device__ static float bold_in(const float *s) { return s[6]; }
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

// Balloon-Windkessel step in FP64 (bw.cu:4-15); x^y as exp2(y log2 x).
struct BW64 { double dt, kappa, y, dt_itau, ialpha, irho, log2_omr, V0k1, V0k2, V0k3; };
__device__ __forceinline__ void bw_step64(double &x, double &f, double &nu, double &q, double z, const BW64 &c) {
    x = x + c.dt * (z - c.kappa * x - c.y * (f - 1.0));
    const double tmp_f = f + c.dt * x;
    nu = nu + c.dt_itau * (f - exp2(c.ialpha * log2(nu)));
    const double pf = exp2(c.log2_omr / f);
    q = q + c.dt_itau * (f * (1.0 - pf) * c.irho - exp2(c.ialpha * log2(nu)) * q / nu);
    f = tmp_f;
}

// ---------------------------------------------------------------- kernel
template <class M>
__global__ void __launch_bounds__(NTHREADS, 2) k_integrate_tc(const IntegrateArgs a, const int *tiles, int n_tiles,
                                                               int KP) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *A_hi = smem_raw;
    uint8_t *A_lo = A_hi + TM * KP * 2;
    uint8_t *B_hi = A_lo + TM * KP * 2;
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
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&sm->mbar)), "r"(1));
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
    const uint32_t idesc = instr_desc();
    const typename M::K K = M::make(a.K);
    BW64 bw;
    bw.dt = a.bw.dt; bw.kappa = a.bw.kappa; bw.y = a.bw.y; bw.dt_itau = a.bw.dt_itau; bw.ialpha = a.bw.ialpha;
    bw.irho = 1.0 / a.bw.rho; bw.log2_omr = log2(a.bw.oneminrho);
    bw.V0k1 = a.bw.V_0 * a.bw.k1; bw.V0k2 = a.bw.V_0 * a.bw.k2; bw.V0k3 = a.bw.V_0 * a.bw.k3;
    const size_t rstride = (size_t)a.n_sims * n;
    const size_t ext = a.states_ts ? (size_t)n * a.states_len : (size_t)n;

    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int *td = tiles + (size_t)tile * (TN + 1);
        const int sc_idx = td[0];
        int sims[SPT];
        float p[SPT][M::NP];
        float s[SPT][M::NS];
#pragma unroll
        for (int i = 0; i < SPT; ++i) {
            sims[i] = td[1 + wg * SPT + i];
            M::init(s[i]);
#pragma unroll
            for (int q = 0; q < M::NP; ++q) p[i][q] = 0.0f;
            if (act && sims[i] >= 0) {  // parameters of (node j, simulation)
                double rr[8];
                for (int q = 0; q < 8; ++q)
                    rr[q] = q < a.n_regional ? a.rparams[(size_t)q * rstride + (size_t)sims[i] * n + j] : 0.0;
                M::params(p[i], a.gparams[sims[i]], rr, K);
            }
        }
        // states sums start at zero
        if (a.ext_out && !a.states_ts && act) {
            for (int i = 0; i < SPT; ++i)
                if (sims[i] >= 0)
                    for (int v = 0; v < M::NOUT; ++v) a.states[((size_t)v * a.n_sims + sims[i]) * ext + j] = 0.0;
        }
        // Balloon-Windkessel state in TMEM: x = 0, f = nu = q = 1
        {
            uint32_t w[8];
            const double init[4] = {0.0, 1.0, 1.0, 1.0};
            for (int q = 0; q < 4; ++q) {
                w[2 * q] = (uint32_t)__double2loint(init[q]);
                w[2 * q + 1] = (uint32_t)__double2hiint(init[q]);
            }
            for (int i = 0; i < SPT; ++i) tmem_st8(t_lane + COL_BW + (wg * SPT + i) * 8, w);
        }
        // A operand: SC^T split into BF16 hi / lo (only when the SC changes)
        if (sm->sc_loaded != sc_idx) {
            const float *SC = a.sc_f32 + (size_t)sc_idx * n * n;
            for (int e = tid; e < TM * KP; e += NTHREADS) {
                const int r = e / KP, k = e % KP;  // r = target node, k = source node
                const float v = (r < n && k < n) ? SC[(size_t)k * n + r] : 0.0f;
                uint16_t hi, lo;
                split_bf16(v, hi, lo);
                const uint32_t off = (k >> 3) * LBO_A + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
                *reinterpret_cast<uint16_t *>(A_hi + off) = hi;
                *reinterpret_cast<uint16_t *>(A_lo + off) = lo;
            }
        }
        // B operand rows of padded nodes are zero; live rows get the initial state
        auto write_x = [&]() {
            if (j >= KP) return;
            uint32_t hw[4], lw[4];
#pragma unroll
            for (int i = 0; i < SPT; i += 2) {
                uint16_t h0, l0, h1, l1;
                const float x0 = act ? M::conn(s[i]) : 0.0f, x1 = act ? M::conn(s[i + 1]) : 0.0f;
                split_bf16(x0, h0, l0);
                split_bf16(x1, h1, l1);
                hw[i / 2] = (uint32_t)h0 | ((uint32_t)h1 << 16);
                lw[i / 2] = (uint32_t)l0 | ((uint32_t)l1 << 16);
            }
            const uint32_t off = (j >> 3) * LBO_B + wg * 128 + (j & 7) * 16;  // n = wg*8 .. wg*8+7
            *reinterpret_cast<uint4 *>(B_hi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            *reinterpret_cast<uint4 *>(B_lo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        };
        write_x();
        __syncthreads();
        if (tid == 0) sm->sc_loaded = sc_idx;

        int bold_i = 0, states_i = 0, repeat = 0;
        int sh_j = act ? a.sh_nodes[j] : 0;
        bool aborted = false;  // only set right after a barrier, so block-uniform
        for (int bw_i = 0; bw_i < a.bw_it; ++bw_i) {
            const int sh_ts = a.sh_ts[(bw_i % a.noise_bw_it) + repeat * a.noise_bw_it];
            const bool sample = a.ext_out && ((bw_i + 1) % a.states_sampling_iters == 0);
            for (int inner = 0; inner < a.inner_it; ++inner) {
                // (1) x written by every thread -> visible to the tensor core
                fence_proxy_async();
                fence_before();
                __syncthreads();
                if (sm->abort) { aborted = true; break; }
                // (2) one thread issues the BF16x3 coupling GEMM
                if (tid == 0) {
                    fence_after();
                    const uint32_t ah = smem_u32(A_hi), al = smem_u32(A_lo);
                    const uint32_t bh = smem_u32(B_hi), bl = smem_u32(B_lo);
                    const int nk = KP / 16;
                    for (int kk = 0; kk < nk; ++kk) {
                        const uint64_t dah = smem_desc(ah + kk * 2 * LBO_A, LBO_A, 128);
                        const uint64_t dal = smem_desc(al + kk * 2 * LBO_A, LBO_A, 128);
                        const uint64_t dbh = smem_desc(bh + kk * 2 * LBO_B, LBO_B, 128);
                        const uint64_t dbl = smem_desc(bl + kk * 2 * LBO_B, LBO_B, 128);
                        mma_bf16(tmem + COL_ACC, dah, dbh, idesc, kk > 0 ? 1u : 0u);
                        mma_bf16(tmem + COL_ACC, dah, dbl, idesc, 1u);
                        mma_bf16(tmem + COL_ACC, dal, dbh, idesc, 1u);
                    }
                    mma_commit(mbar);
                }
                // (3) wait for the GEMM, read this thread's 8 coupling sums
                const bool ok = mbar_wait(mbar, phase);
                phase ^= 1u;
                if (!ok) {
                    sm->abort = 1;
                    atomicExch(a.status, 1);
                }
                fence_after();
                uint32_t acc[8];
                tmem_ld8(t_lane + COL_ACC + wg * SPT, acc);
                // (4) elementwise update of the 8 simulations of node j
                if (act) {
                    const long long ni = ((long long)sh_ts * a.inner_it + inner) * n * M::NN + (long long)sh_j * M::NN;
                    const float n0 = a.noise_f32[ni];
                    const float n1 = (M::NN > 1) ? a.noise_f32[ni + 1] : 0.0f;
                    const bool last = sample && (inner == a.inner_it - 1);
#pragma unroll
                    for (int i = 0; i < SPT; ++i) {
                        float o[M::NOUT];
                        M::step(s[i], p[i], __uint_as_float(acc[i]), n0, n1, K, o);
                        if (last && sims[i] >= 0) {
                            if (a.states_ts) {
                                for (int v = 0; v < M::NOUT; ++v)
                                    a.states[((size_t)v * a.n_sims + sims[i]) * ext + (size_t)states_i * n + j] = o[v];
                            } else if (states_i >= a.n_states_samples_remove) {
                                for (int v = 0; v < M::NOUT; ++v)
                                    a.states[((size_t)v * a.n_sims + sims[i]) * ext + j] += (double)o[v];
                            }
                        }
                    }
                }
                write_x();
            }
            if (aborted) break;
            // Balloon-Windkessel, FP64, state in TMEM
            const bool tr = ((bw_i + 1) % a.bold_tr_iters == 0);
#pragma unroll 1
            for (int i = 0; i < SPT; ++i) {
                uint32_t w[8];
                const uint32_t col = t_lane + COL_BW + (wg * SPT + i) * 8;
                tmem_ld8(col, w);
                double x = __hiloint2double((int)w[1], (int)w[0]);
                double f = __hiloint2double((int)w[3], (int)w[2]);
                double nu = __hiloint2double((int)w[5], (int)w[4]);
                double q = __hiloint2double((int)w[7], (int)w[6]);
                if (act) bw_step64(x, f, nu, q, (double)M::bold_in(s[i]), bw);
                w[0] = (uint32_t)__double2loint(x); w[1] = (uint32_t)__double2hiint(x);
                w[2] = (uint32_t)__double2loint(f); w[3] = (uint32_t)__double2hiint(f);
                w[4] = (uint32_t)__double2loint(nu); w[5] = (uint32_t)__double2hiint(nu);
                w[6] = (uint32_t)__double2loint(q); w[7] = (uint32_t)__double2hiint(q);
                tmem_st8(col, w);
                if (tr && act && sims[i] >= 0)
                    a.bold[(size_t)sims[i] * a.bold_len * n + (size_t)bold_i * n + j] =
                        bw.V0k1 * (1 - q) + bw.V0k2 * (1 - q / nu) + bw.V0k3 * (1 - nu);
            }
            if (tr) bold_i++;
            if (sample) states_i++;
            if ((bw_i + 1) % a.noise_bw_it == 0 && bw_i + 1 < a.bw_it) {
                repeat++;
                sh_j = act ? a.sh_nodes[(size_t)repeat * n + j] : 0;
            }
        }
        if (a.ext_out && !a.states_ts && act && !aborted) {
            const int pts = states_i - a.n_states_samples_remove;
            for (int i = 0; i < SPT; ++i)
                if (sims[i] >= 0)
                    for (int v = 0; v < M::NOUT; ++v) a.states[((size_t)v * a.n_sims + sims[i]) * ext + j] /= pts;
        }
        __syncthreads();
        if (sm->abort) break;
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

size_t smem_bytes(int KP) { return (size_t)2 * TM * KP * 2 + (size_t)2 * KP * TN * 2 + sizeof(Smem) + 64; }

template <class M>
cudaError_t launch_tc(const IntegrateArgs &a, const int *tiles, int n_tiles, cudaStream_t st) {
    const int KP = ((a.nodes + 15) / 16) * 16;
    const size_t smem = std::max<size_t>(smem_bytes(KP), 80 * 1024);  // at most 2 CTAs per SM (TMEM: 2 x 256 columns)
    cudaError_t e = cudaFuncSetAttribute(k_integrate_tc<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::min(n_tiles, 2 * sms);
    k_integrate_tc<M><<<grid, NTHREADS, smem, st>>>(a, tiles, n_tiles, KP);
    return cudaGetLastError();
}

}  // namespace

bool fp32_supported(int model, int nodes, bool has_delay) {
    if (has_delay || nodes > TM || nodes < 1) return false;
    return model == MODEL_RWW || model == MODEL_WC || model == MODEL_JR || model == MODEL_RWWEX;
}

int fp32_tile_sims() { return TN; }

cudaError_t launch_integrate_fp32(int model, const IntegrateArgs &a, cudaStream_t st, int *launches) {
    if (launches) ++*launches;
    switch (model) {
        case MODEL_RWW: return launch_tc<RWW32>(a, a.tiles, a.n_tiles, st);
        case MODEL_WC: return launch_tc<WC32>(a, a.tiles, a.n_tiles, st);
        case MODEL_JR: return launch_tc<JR32>(a, a.tiles, a.n_tiles, st);
        case MODEL_RWWEX: return launch_tc<RWWEx32>(a, a.tiles, a.n_tiles, st);
        default: break;
    }
    return cudaErrorNotSupported;
}

}  // namespace cbnm
