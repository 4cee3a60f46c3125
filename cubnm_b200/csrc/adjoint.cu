// Adjoint (reverse-mode) gradient of an FP32 rWW batch with the noise held fixed.
//
// Forward (k_adj_forward): the FP32 per-simulation rWW time loop of
// integrate_sim.cuh (same expressions, same coupling order, so the same BOLD),
// plus a checkpoint of (S_E, S_I) and the FP64 Balloon-Windkessel state
// (x, f, nu, q) at the start of every segment of seg_bw Balloon-Windkessel
// steps (seg_bw * inner_it integration steps).
//
// Backward (k_adj_backward): segments in reverse.  Each segment is recomputed
// from its checkpoint, storing the pre-step S_E, S_I and coupling input of every
// step and the pre-step Balloon-Windkessel state of every millisecond in a
// scratch; then the steps are run backwards.  With lambda the adjoint of each
// state, per integration step of node j (reference step: rww.cpp:194-232):
//   u_E = S_E + sigma sqrt(dt) n0 + dt g_E (1 - S_E) r_E - dt/t_E S_E  (clamped: lambda passes only inside [0, 1])
//   u_I = S_I + sigma sqrt(dt) n1 + dt g_I r_I - dt/t_I S_I
//   r(x) = x / (1 - e^{-d x}),  r'(x) = ((1 - e) - d x e) / (1 - e)^2,  e = e^{-d x}
//   I_E = wEI0 + w_p J_N S_E + G J_N in_j - wIE S_I,   I_I = wII0 + J_N S_E - wII S_I
//   in_j = sum_k SC[k][j] S_E,k  =>  lambda_S_E,k += sum_j SC[k][j] lambda_in,j  (a transposed product:
//   node k reads SC^T row k, coalesced across the warp; both products use the
//   four-accumulator FP32 sum of integrate_sim.cuh)
// and per millisecond the reverse of the Balloon-Windkessel Euler step
// (bw.cu:4-15; the f update uses the new x, the q update the new nu) with the
// BOLD sample (bnm.cpp:316-320) adding dL/dBOLD * dBOLD/d(q, nu).
// Parameter gradients (G per simulation; w_p, J_N, wIE, sigma per node) are
// accumulated in FP64 by the thread of each node; G is summed over nodes at
// the end.  Adjoint states are FP32 like the forward state, Balloon-Windkessel
// adjoints FP64 like its state.
#include "integrate_sim.cuh"

namespace cbnm {
namespace {

using M = RWWm<float>;

__device__ __forceinline__ int noise_ts(const IntegrateArgs &a, int bw_i, int &repeat) {
    repeat = bw_i / a.noise_bw_it;
    return a.sh_ts[(bw_i % a.noise_bw_it) + repeat * a.noise_bw_it];
}

// d r / d x for r(x) = x / (1 - e^{-d x}); series near 0 where the closed form cancels
__device__ __forceinline__ float rate_deriv(float x, double d) {
    const float df = (float)d, u = df * x;
    if (fabsf(u) < 1e-2f) return 0.5f + u * (1.0f / 6.0f);
    const float e = expf(-u), den = -expm1f(-u);
    return (den - u * e) / (den * den);
}

__device__ double block_sum_d(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        red[32] = t;
    }
    __syncthreads();
    return red[32];
}

struct Params {
    float g[M::NG];
    float r[M::NR];
};

__device__ __forceinline__ Params load_params(const IntegrateArgs &a, int sim, int j, bool act) {
    Params P;
    P.g[0] = (float)a.gparams[sim];
    const size_t rstride = (size_t)a.n_sims * a.nodes;
#pragma unroll
    for (int i = 0; i < M::NR; ++i) P.r[i] = act ? (float)a.rparams[i * rstride + (size_t)sim * a.nodes + j] : 0.0f;
    return P;
}

// One integration step of node j (the coupling input already formed), exactly as
// k_integrate_sim<RWWm<float>, false, float, ...>.
__device__ __forceinline__ void fwd_step(float *s, const Params &P, float in, const IntegrateArgs &a, int sh_ts,
                                         int inner, int sh_j) {
    const long long ni = ((long long)sh_ts * a.inner_it + inner) * a.nodes * M::NN + (long long)sh_j * M::NN;
    const float n0 = a.noise_f32[ni], n1 = a.noise_f32[ni + 1];
    float iv[M::NI];
    M::step(s, iv, P.g, P.r, in, n0, n1, a.K);
}

__global__ void __launch_bounds__(1024) k_adj_forward(const AdjArgs A) {
    const IntegrateArgs &a = A.ia;
    const int sim = A.sim_begin + blockIdx.x;
    const int j = threadIdx.x, n = a.nodes;
    const bool act = j < n;
    extern __shared__ __align__(16) float x1[];
    const float *SC = a.sc_f32 + (size_t)a.sc_idx[sim] * n * n;
    const Params P = load_params(a, sim, j, act);
    float s[M::NS];
#pragma unroll
    for (int i = 0; i < M::NS; ++i) s[i] = 0.0f;
    float iv0[M::NI];
    M::init(s, iv0, P.g, P.r);
    double bx = 0.0, bf = 1.0, bnu = 1.0, bq = 1.0;
    if (act) x1[j] = s[M::CONN];
    double *bold = a.bold + (size_t)sim * a.bold_len * n;
    int bold_i = 0;
    for (int bw_i = 0; bw_i < a.bw_it; ++bw_i) {
        if (bw_i % A.seg_bw == 0 && act) {
            const size_t c = (size_t)sim * A.n_seg + bw_i / A.seg_bw;
            A.ck_s[(c * 2 + 0) * n + j] = s[4];
            A.ck_s[(c * 2 + 1) * n + j] = s[5];
            A.ck_bw[(c * 4 + 0) * n + j] = bx;
            A.ck_bw[(c * 4 + 1) * n + j] = bf;
            A.ck_bw[(c * 4 + 2) * n + j] = bnu;
            A.ck_bw[(c * 4 + 3) * n + j] = bq;
        }
        int repeat;
        const int sh_ts = noise_ts(a, bw_i, repeat);
        const int sh_j = act ? a.sh_nodes[(size_t)repeat * n + j] : 0;
        for (int inner = 0; inner < a.inner_it; ++inner) {
            __syncthreads();
            float in = 0.0f;
            if (act) {
                in = coupling_f32(SC, x1, n, j);
                fwd_step(s, P, in, a, sh_ts, inner, sh_j);
            }
            __syncthreads();
            if (act) x1[j] = s[M::CONN];
        }
        if (act) bw_step(bx, bf, bnu, bq, (double)s[M::BOLDV], a.bw);
        if ((bw_i + 1) % a.bold_tr_iters == 0) {
            if (act && bold_i < a.bold_len)  // no slot for a sample past bold_len
                bold[(size_t)bold_i * n + j] =
                    a.bw.V_0 * (a.bw.k1 * (1 - bq) + a.bw.k2 * (1 - bq / bnu) + a.bw.k3 * (1 - bnu));
            bold_i++;
        }
    }
}

__global__ void __launch_bounds__(1024) k_adj_backward(const AdjArgs A) {
    const IntegrateArgs &a = A.ia;
    const int sim = A.sim_begin + blockIdx.x;
    const int j = threadIdx.x, n = a.nodes;
    const bool act = j < n;
    extern __shared__ __align__(16) float sh[];
    float *x1 = sh;                          // S_E of every node (forward recompute)
    float *lin = sh + ((n + 3) & ~3);        // adjoint of every node's coupling input (16-byte aligned)
    __shared__ double red[33];
    const float *SC = a.sc_f32 + (size_t)a.sc_idx[sim] * n * n;
    const float *SCT = A.sct_f32 + (size_t)a.sc_idx[sim] * n * n;
    const Params P = load_params(a, sim, j, act);
    const RWWK &m = a.K.rww;
    const BWConst &c = a.bw;
    const float w_p = P.r[0], J_N = P.r[1], wIE = P.r[2], sig = P.r[3], G = P.g[0];
    const int steps_seg = A.seg_bw * a.inner_it;
    float *scr_s = A.scr_s + (size_t)blockIdx.x * steps_seg * 3 * n;
    float *scr_z = A.scr_z + (size_t)blockIdx.x * A.seg_bw * n;
    double *scr_bw = A.scr_bw + (size_t)blockIdx.x * A.seg_bw * 4 * n;
    const double *dbold = A.dbold + (size_t)sim * a.bold_len * n;

    float lE = 0.0f, lI = 0.0f;                        // adjoints of S_E, S_I
    double lx = 0.0, lf = 0.0, lnu = 0.0, lq = 0.0;    // adjoints of the Balloon-Windkessel state
    double gG = 0.0, gWp = 0.0, gJ = 0.0, gWIE = 0.0, gSig = 0.0;
    const double a_pow = c.ialpha, ln1mr = log(c.oneminrho);
    const float sqdt = (float)m.sqrt_dt;

    for (int seg = A.n_seg - 1; seg >= 0; --seg) {
        const int bw0 = seg * A.seg_bw;
        const int nb = min(A.seg_bw, a.bw_it - bw0);
        // ---- recompute the segment from its checkpoint
        float s[M::NS];
#pragma unroll
        for (int i = 0; i < M::NS; ++i) s[i] = 0.0f;
        double bx = 0.0, bf = 1.0, bnu = 1.0, bq = 1.0;
        if (act) {
            const size_t ck = (size_t)sim * A.n_seg + seg;
            s[4] = A.ck_s[(ck * 2 + 0) * n + j];
            s[5] = A.ck_s[(ck * 2 + 1) * n + j];
            bx = A.ck_bw[(ck * 4 + 0) * n + j];
            bf = A.ck_bw[(ck * 4 + 1) * n + j];
            bnu = A.ck_bw[(ck * 4 + 2) * n + j];
            bq = A.ck_bw[(ck * 4 + 3) * n + j];
        }
        __syncthreads();
        if (act) x1[j] = s[M::CONN];
        for (int b = 0; b < nb; ++b) {
            const int bw_i = bw0 + b;
            int repeat;
            const int sh_ts = noise_ts(a, bw_i, repeat);
            const int sh_j = act ? a.sh_nodes[(size_t)repeat * n + j] : 0;
            if (act) {
                scr_bw[((size_t)b * 4 + 0) * n + j] = bx;
                scr_bw[((size_t)b * 4 + 1) * n + j] = bf;
                scr_bw[((size_t)b * 4 + 2) * n + j] = bnu;
                scr_bw[((size_t)b * 4 + 3) * n + j] = bq;
            }
            for (int inner = 0; inner < a.inner_it; ++inner) {
                __syncthreads();
                float in = 0.0f;
                if (act) {
                    in = coupling_f32(SC, x1, n, j);
                    const size_t t = (size_t)b * a.inner_it + inner;
                    scr_s[(t * 3 + 0) * n + j] = s[4];
                    scr_s[(t * 3 + 1) * n + j] = s[5];
                    scr_s[(t * 3 + 2) * n + j] = in;
                    fwd_step(s, P, in, a, sh_ts, inner, sh_j);
                }
                __syncthreads();
                if (act) x1[j] = s[M::CONN];
            }
            if (act) {
                scr_z[(size_t)b * n + j] = s[M::BOLDV];
                bw_step(bx, bf, bnu, bq, (double)s[M::BOLDV], c);
            }
        }
        // ---- reverse through the segment
        for (int b = nb - 1; b >= 0; --b) {
            const int bw_i = bw0 + b;
            int repeat;
            const int sh_ts = noise_ts(a, bw_i, repeat);
            const int sh_j = act ? a.sh_nodes[(size_t)repeat * n + j] : 0;
            if (act) {
                const double x0 = scr_bw[((size_t)b * 4 + 0) * n + j], f0 = scr_bw[((size_t)b * 4 + 1) * n + j];
                const double nu0 = scr_bw[((size_t)b * 4 + 2) * n + j], q0 = scr_bw[((size_t)b * 4 + 3) * n + j];
                const double z = (double)scr_z[(size_t)b * n + j];
                double x1b = x0, f1b = f0, nu1 = nu0, q1 = q0;
                bw_step(x1b, f1b, nu1, q1, z, c);
                const int vol = (bw_i + 1) / a.bold_tr_iters - 1;
                if ((bw_i + 1) % a.bold_tr_iters == 0 && vol < a.bold_len) {  // BOLD = V0 (k1 (1-q) + k2 (1-q/nu) + k3 (1-nu))
                    const double gb = dbold[(size_t)vol * n + j];
                    lq += gb * c.V_0 * (-c.k1 - c.k2 / nu1);
                    lnu += gb * c.V_0 * (c.k2 * q1 / (nu1 * nu1) - c.k3);
                }
                // reverse of the Balloon-Windkessel step
                const double ct = c.dt_itau;
                const double A1 = pow(nu1, a_pow) / nu1;                         // nu1^(a-1)
                const double E = pow(c.oneminrho, 1.0 / f0);
                const double dq_dq0 = 1.0 - ct * A1;
                const double dq_dnu1 = -ct * q0 * (a_pow - 1.0) * A1 / nu1;
                const double dq_df0 = ct / c.rho * ((1.0 - E) + E * ln1mr / f0);
                const double lq0 = lq * dq_dq0;
                const double lnu1 = lnu + lq * dq_dnu1;
                double lf0 = lq * dq_df0;
                const double lnu0 = lnu1 * (1.0 - ct * a_pow * pow(nu0, a_pow - 1.0));
                lf0 += lnu1 * ct;
                lf0 += lf;
                const double lx1 = lx + lf * c.dt;
                const double lx0 = lx1 * (1.0 - c.dt * c.kappa);
                lf0 += lx1 * (-c.dt * c.y);
                const double lz = lx1 * c.dt;
                lx = lx0; lf = lf0; lnu = lnu0; lq = lq0;
                lE += (float)lz;
            }
            for (int inner = a.inner_it - 1; inner >= 0; --inner) {
                float lin_j = 0.0f, SE = 0.0f, SI = 0.0f, in = 0.0f;
                if (act) {
                    const size_t t = (size_t)b * a.inner_it + inner;
                    SE = scr_s[(t * 3 + 0) * n + j];
                    SI = scr_s[(t * 3 + 1) * n + j];
                    in = scr_s[(t * 3 + 2) * n + j];
                    const long long ni = ((long long)sh_ts * a.inner_it + inner) * n * M::NN + (long long)sh_j * M::NN;
                    const float n0 = a.noise_f32[ni], n1 = a.noise_f32[ni + 1];
                    // forward pieces, as RWWm<float>::step
                    const float IE = (float)m.w_E__I_0 + w_p * J_N * SE + in * G * J_N - wIE * SI;
                    const float II = (float)m.w_I__I_0 + J_N * SE - (float)m.w_II * SI;
                    const float xE = (float)m.a_E * IE - (float)m.b_E;
                    const float xI = (float)m.a_I * II - (float)m.b_I;
                    const float rE = rate_of<float>(xE, m.d_E);
                    const float rI = rate_of<float>(xI, m.d_I);
                    const float uE = SE + (n0 * sig * sqdt + (float)m.dt_gamma_E * ((1.0f - SE) * rE) -
                                           (float)m.dt_itau_E * SE);
                    const float uI = SI + (n1 * sig * sqdt + (float)m.dt_gamma_I * rI - (float)m.dt_itau_I * SI);
                    const float luE = (uE >= 0.0f && uE <= 1.0f) ? lE : 0.0f;
                    const float luI = (uI >= 0.0f && uI <= 1.0f) ? lI : 0.0f;
                    const float lrE = luE * (float)m.dt_gamma_E * (1.0f - SE);
                    const float lrI = luI * (float)m.dt_gamma_I;
                    float lSE = luE * (1.0f - (float)m.dt_gamma_E * rE - (float)m.dt_itau_E);
                    float lSI = luI * (1.0f - (float)m.dt_itau_I);
                    const float lIE = lrE * rate_deriv(xE, m.d_E) * (float)m.a_E;
                    const float lII = lrI * rate_deriv(xI, m.d_I) * (float)m.a_I;
                    lSE += lIE * w_p * J_N + lII * J_N;
                    lSI += -lIE * wIE - lII * (float)m.w_II;
                    lin_j = lIE * G * J_N;
                    gWp += (double)(lIE * J_N * SE);
                    gJ += (double)(lIE * (w_p * SE + G * in) + lII * SE);
                    gG += (double)(lIE * J_N * in);
                    gWIE += (double)(-lIE * SI);
                    gSig += (double)((luE * n0 + luI * n1) * sqdt);
                    lE = lSE;
                    lI = lSI;
                    lin[j] = lin_j;
                }
                __syncthreads();
                if (act) {  // lambda_S_E,j += sum_k SC[j][k] lambda_in,k
                    lE += coupling_f32(SCT, lin, n, j);
                }
                __syncthreads();
            }
        }
    }
    const double gG_all = block_sum_d(act ? gG : 0.0, red);
    if (j == 0) A.grad_g[sim] = gG_all;
    if (act) {
        const size_t rs = (size_t)a.n_sims * n, o = (size_t)sim * n + j;
        A.grad_r[0 * rs + o] = gWp;
        A.grad_r[1 * rs + o] = gJ;
        A.grad_r[2 * rs + o] = gWIE;
        A.grad_r[3 * rs + o] = gSig;
    }
}

__global__ void k_transpose_sc(const double *sc, float *scf, float *sct, int n_scs, int n) {
    const size_t nn = (size_t)n * n, total = nn * n_scs;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t s = e / nn, r = e % nn;
        const int row = (int)(r / n), col = (int)(r % n);
        const float v = (float)sc[e];
        scf[e] = v;
        sct[s * nn + (size_t)col * n + row] = v;
    }
}

}  // namespace

cudaError_t launch_adjoint_forward(const AdjArgs &a, cudaStream_t st) {
    const int threads = ((a.ia.nodes + 31) / 32) * 32;
    k_adj_forward<<<a.sim_count, threads, sizeof(float) * a.ia.nodes, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_backward(const AdjArgs &a, cudaStream_t st) {
    const int threads = ((a.ia.nodes + 31) / 32) * 32;
    k_adj_backward<<<a.sim_count, threads, sizeof(float) * 2 * ((a.ia.nodes + 3) & ~3), st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_transpose_sc(const double *sc, float *sc_f32, float *sct_f32, int n_scs, int nodes, cudaStream_t st) {
    k_transpose_sc<<<592, 256, 0, st>>>(sc, sc_f32, sct_f32, n_scs, nodes);
    return cudaGetLastError();
}

}  // namespace cbnm
