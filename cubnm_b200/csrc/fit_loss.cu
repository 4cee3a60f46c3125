// Loss of the gradient fit and its gradient with respect to BOLD (FP64):
//   L = (1 - r(FC_sim, FC_emp)) + W1(FCD_sim values, FCD_emp values)
// FC and FCD as the reference computes them (src/ext/fc.cu:77-239; windows
// src/ext/utils.cpp:21-52; pair order np.tril_indices(n, -1)); r = Pearson
// correlation of the FC lower triangles; W1 = the 1-D Wasserstein distance of
// the FCD value distributions by the midpoint rule on the simulated quantiles,
// mean_i |sort(fcd)_i - q_i| with q_i = sorted_emp[floor((i + 1/2) m2 / m)]
// (the index in integer arithmetic, ((2i + 1) m2) / (2m)).
//
// Forward, per simulation s (one CTA per (s, window) for the FCs, one CTA per s
// for the rest):
//   X^w = columns of the window's BOLD centred and divided by their root sum of
//   squares sigma^w; FC^w_ij = sum_t X^w_ti X^w_tj (w = 0: static FC over
//   volumes [n_vols_remove, T)); FCD_ab = Pearson r of FC^a, FC^b over pairs.
// Backward (the chain rule of each step, written out):
//   dL/dFC_p   = -(e_p / (|s| |e|) - r s_p / |s|^2)   (s, e: centred FC vectors)
//   dL/dFCD_k  = sign(sort_i - q_i) / m at the rank i of k
//   dL/dFC^a_p = (1 / |u_a|) (sum_b g_ab Z_b[p] - (sum_b g_ab c_ab) Z_a[p])
//                (Z: centred, unit-norm window-FC vectors; c_ab = FCD_ab; g_ab = dL/dFCD_ab, symmetric)
//   dL/dx_ti   = (1 / sigma_i) (sum_j g_ij X_j[t] - X_i[t] sum_j g_ij FC_ij)   per window, summed
// The last step runs window after window in one CTA per simulation, so the
// overlapping windows add into dL/dBOLD without atomics.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>
#include "engine.h"

namespace cbnm {
namespace {

constexpr int FL_THREADS = 256;

__device__ __forceinline__ size_t tri(int i, int j) {  // lower-triangle index of (i, j), i > j
    return (size_t)i * (i - 1) / 2 + j;
}

__device__ double fl_block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        red[32] = t;
    }
    __syncthreads();
    return red[32];
}

// Volume range [r0, r1) of window w (0 = static FC).
__device__ __forceinline__ void window_range(const FitLossArgs &a, int w, int &r0, int &r1) {
    if (w == 0) { r0 = a.n_vols_remove; r1 = a.bold_len; }
    else { r0 = a.w_start[w - 1]; r1 = a.w_end[w - 1] + 1; }
}

// FC of one (simulation, window): node means / sigmas to stats, FC to fc or wfc.
__global__ void __launch_bounds__(FL_THREADS) k_fl_fc(const FitLossArgs a) {
    const int ls = blockIdx.x, sim = a.sim_begin + ls, w = blockIdx.y, n = a.nodes;
    int r0, r1;
    window_range(a, w, r0, r1);
    const int T = r1 - r0;
    const double *x = a.bold + (size_t)sim * a.bold_len * n + (size_t)r0 * n;
    double *st = a.stats + ((size_t)ls * (a.n_windows + 1) + w) * 2 * n;  // [mean n][sigma n]
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double m = 0.0;
        for (int t = 0; t < T; ++t) m += x[(size_t)t * n + j];
        m /= T;
        double q = 0.0;
        for (int t = 0; t < T; ++t) {
            const double d = x[(size_t)t * n + j] - m;
            q += d * d;
        }
        st[j] = m;
        st[n + j] = sqrt(q);
    }
    __syncthreads();
    double *out = (w == 0) ? a.fc + (size_t)ls * a.n_pairs : a.wfc + ((size_t)ls * a.n_windows + (w - 1)) * a.n_pairs;
    for (size_t p = threadIdx.x; p < (size_t)a.n_pairs; p += blockDim.x) {
        int i = (int)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
        while ((size_t)i * (i - 1) / 2 > p) --i;
        while ((size_t)(i + 1) * i / 2 <= p) ++i;
        const int j = (int)(p - (size_t)i * (i - 1) / 2);
        const double mi = st[i], mj = st[j];
        double c = 0.0;
        for (int t = 0; t < T; ++t) c += (x[(size_t)t * n + i] - mi) * (x[(size_t)t * n + j] - mj);
        out[p] = c / (st[n + i] * st[n + j]);
    }
}

// Per simulation: window-FC statistics, FCD, the two loss terms and their
// gradients with respect to FC (g_fc) and FCD (g_fcd).
__global__ void __launch_bounds__(FL_THREADS) k_fl_loss(const FitLossArgs a, int m_pow2) {
    extern __shared__ double sh[];
    __shared__ double red[33];
    const int ls = blockIdx.x, sim = a.sim_begin + ls;
    const int W = a.n_windows, P = a.n_pairs, M = a.n_window_pairs;
    const double *fc = a.fc + (size_t)ls * P;
    // ---- FC term: r = <s, e> / (|s| |e|), e = emp_fc - mean (precomputed, |e| = emp_norm)
    double sum = 0.0;
    for (int p = threadIdx.x; p < P; p += blockDim.x) sum += fc[p];
    const double mean = fl_block_sum(sum, red) / P;
    double se = 0.0, ss = 0.0;
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        const double s = fc[p] - mean;
        se += s * a.emp_c[p];
        ss += s * s;
    }
    se = fl_block_sum(se, red);
    ss = fl_block_sum(ss, red);
    const double ns = sqrt(ss), r = se / (ns * a.emp_norm);
    if (threadIdx.x == 0) a.loss_fc[sim] = 1.0 - r;
    if (a.want_grad) {
        double *g = a.g_fc + (size_t)ls * P;
        for (int p = threadIdx.x; p < P; p += blockDim.x)
            g[p] = -(a.emp_c[p] / (ns * a.emp_norm) - r * (fc[p] - mean) / ss);
    }
    if (W < 2) {
        if (threadIdx.x == 0) a.loss_fcd[sim] = 0.0;
        return;
    }
    // ---- window-FC means and root sums of squares
    const double *wfc = a.wfc + (size_t)ls * W * P;
    double *wst = a.wstat + (size_t)ls * W * 2;
    for (int w = 0; w < W; ++w) {
        const double *v = wfc + (size_t)w * P;
        double s = 0.0;
        for (int p = threadIdx.x; p < P; p += blockDim.x) s += v[p];
        const double m = fl_block_sum(s, red) / P;
        double q = 0.0;
        for (int p = threadIdx.x; p < P; p += blockDim.x) {
            const double d = v[p] - m;
            q += d * d;
        }
        q = fl_block_sum(q, red);
        if (threadIdx.x == 0) { wst[2 * w] = m; wst[2 * w + 1] = sqrt(q); }
    }
    __syncthreads();
    // ---- FCD (window pairs in (a > b) row order) into shared memory: values, then indices
    double *val = sh;
    int *idx = reinterpret_cast<int *>(sh + m_pow2);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double *fcd_out = a.fcd + (size_t)ls * M;
    for (int k = warp; k < M; k += nwarps) {
        int wa = (int)((1.0 + sqrt(1.0 + 8.0 * k)) * 0.5);
        while (wa * (wa - 1) / 2 > k) --wa;
        while ((wa + 1) * wa / 2 <= k) ++wa;
        const int wb = k - wa * (wa - 1) / 2;
        const double *x = wfc + (size_t)wa * P, *y = wfc + (size_t)wb * P;
        const double mx = wst[2 * wa], my = wst[2 * wb];
        double c = 0.0;
        for (int p = lane; p < P; p += 32) c += (x[p] - mx) * (y[p] - my);
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0) {
            c /= wst[2 * wa + 1] * wst[2 * wb + 1];
            val[k] = c;
            idx[k] = k;
            fcd_out[k] = c;
        }
    }
    for (int k = M + threadIdx.x; k < m_pow2; k += blockDim.x) { val[k] = INFINITY; idx[k] = k; }
    __syncthreads();
    // ---- bitonic sort of (value, index) ascending (ties by index)
    for (int size = 2; size <= m_pow2; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < m_pow2 / 2; t += blockDim.x) {
                const int lo = 2 * stride * (t / stride) + (t % stride), hi = lo + stride;
                const bool up = ((lo & size) == 0);
                const double vl = val[lo], vh = val[hi];
                const int il = idx[lo], ih = idx[hi];
                const bool gt = (vl > vh) || (vl == vh && il > ih);
                if (gt == up) { val[lo] = vh; val[hi] = vl; idx[lo] = ih; idx[hi] = il; }
            }
            __syncthreads();
        }
    // ---- W1 and dL/dFCD
    double w1 = 0.0;
    for (int i = threadIdx.x; i < M; i += blockDim.x) {
        const double d = val[i] - a.emp_q[i];
        w1 += fabs(d);
        if (a.want_grad) a.g_fcd[(size_t)ls * M + idx[i]] = (d > 0.0 ? 1.0 : (d < 0.0 ? -1.0 : 0.0)) / M;
    }
    w1 = fl_block_sum(w1, red);
    if (threadIdx.x == 0) a.loss_fcd[sim] = w1 / M;
}

// dL/dFC^a for window a of simulation ls (grid: simulations x windows).
__global__ void __launch_bounds__(FL_THREADS) k_fl_gwfc(const FitLossArgs a) {
    const int ls = blockIdx.x, wa = blockIdx.y, W = a.n_windows, P = a.n_pairs;
    const double *wfc = a.wfc + (size_t)ls * W * P;
    const double *wst = a.wstat + (size_t)ls * W * 2;
    const double *g = a.g_fcd + (size_t)ls * a.n_window_pairs;
    const double *fcd = a.fcd + (size_t)ls * a.n_window_pairs;
    __shared__ double gb[1024];   // g_ab / |u_b| for every b (0 at b = a)
    __shared__ double hsum;
    if (threadIdx.x == 0) {
        double h = 0.0;
        for (int b = 0; b < W; ++b) {
            if (b == wa) { gb[b] = 0.0; continue; }
            const size_t k = wa > b ? tri(wa, b) : tri(b, wa);
            gb[b] = g[k] / wst[2 * b + 1];
            h += g[k] * fcd[k];
        }
        hsum = h;
    }
    __syncthreads();
    const double ma = wst[2 * wa], na = wst[2 * wa + 1];
    double *out = a.g_wfc + ((size_t)ls * W + wa) * P;
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        double acc = 0.0;
        for (int b = 0; b < W; ++b) acc += gb[b] * (wfc[(size_t)b * P + p] - wst[2 * b]);
        out[p] = (acc - hsum * (wfc[(size_t)wa * P + p] - ma) / na) / na;
    }
}

// dL/dBOLD of simulation ls: every window's FC gradient pulled back to its volumes.
__global__ void __launch_bounds__(FL_THREADS) k_fl_gbold(const FitLossArgs a) {
    extern __shared__ double hrow[];   // [n]: sum_j g_ij FC_ij of the current window
    const int ls = blockIdx.x, sim = a.sim_begin + ls, n = a.nodes, P = a.n_pairs;
    const double *x = a.bold + (size_t)sim * a.bold_len * n;
    double *dx = a.dbold + (size_t)sim * a.bold_len * n;
    for (size_t e = threadIdx.x; e < (size_t)a.bold_len * n; e += blockDim.x) dx[e] = 0.0;
    __syncthreads();
    const int nw = a.n_windows >= 2 ? a.n_windows : 0;  // with fewer than two windows there is no FCD term
    for (int w = 0; w <= nw; ++w) {
        int r0, r1;
        window_range(a, w, r0, r1);
        const int T = r1 - r0;
        const double *st = a.stats + ((size_t)ls * (a.n_windows + 1) + w) * 2 * n;
        const double *g = (w == 0) ? a.g_fc + (size_t)ls * P : a.g_wfc + ((size_t)ls * a.n_windows + (w - 1)) * P;
        const double *c = (w == 0) ? a.fc + (size_t)ls * P : a.wfc + ((size_t)ls * a.n_windows + (w - 1)) * P;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            double h = 0.0;
            for (int j = 0; j < n; ++j) {
                if (j == i) continue;
                const size_t k = i > j ? tri(i, j) : tri(j, i);
                h += g[k] * c[k];
            }
            hrow[i] = h;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < T * n; e += blockDim.x) {
            const int t = e / n, i = e % n;
            const double *xt = x + (size_t)(r0 + t) * n;
            double acc = 0.0;
            for (int j = 0; j < n; ++j) {
                if (j == i) continue;
                const size_t k = i > j ? tri(i, j) : tri(j, i);
                acc += g[k] * (xt[j] - st[j]) / st[n + j];
            }
            const double xi = (xt[i] - st[i]) / st[n + i];
            dx[(size_t)(r0 + t) * n + i] += (acc - xi * hrow[i]) / st[n + i];
        }
        __syncthreads();
    }
}

}  // namespace

size_t fit_loss_sort_smem(int n_window_pairs) {
    int m2 = 1;
    while (m2 < n_window_pairs) m2 <<= 1;
    return (sizeof(double) + sizeof(int)) * (size_t)m2;
}

cudaError_t launch_fit_loss(const FitLossArgs &a, cudaStream_t st, int *launches) {
    if (a.n_windows > 1024) return cudaErrorInvalidValue;
    k_fl_fc<<<dim3(a.sim_count, 1 + a.n_windows), FL_THREADS, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int m2 = 1;
    while (m2 < std::max(1, a.n_window_pairs)) m2 <<= 1;
    const size_t smem = fit_loss_sort_smem(std::max(1, a.n_window_pairs));
    e = allow_dynamic_smem(k_fl_loss);
    if (e != cudaSuccess) return e;
    k_fl_loss<<<a.sim_count, FL_THREADS, smem, st>>>(a, m2);
    e = cudaGetLastError();
    if (launches) *launches += 2;
    if (e != cudaSuccess || !a.want_grad) return e;
    if (a.n_windows >= 2) {
        k_fl_gwfc<<<dim3(a.sim_count, a.n_windows), FL_THREADS, 0, st>>>(a);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (launches) ++*launches;
    }
    k_fl_gbold<<<a.sim_count, FL_THREADS, sizeof(double) * a.nodes, st>>>(a);
    if (launches) ++*launches;
    return cudaGetLastError();
}

}  // namespace cbnm
