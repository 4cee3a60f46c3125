// Goodness-of-fit reductions (reference: src/cubnm/sim/base.py:1084-1207,
// src/cubnm/utils.py:306-507).
//
// k_fc_gof: one CTA per simulation, three terms from one pass over its FC row:
//   +fc_corr  Pearson r(sim_fc, emp_fc) (scipy.stats.pearsonr; utils.py:416-507
//             computes it as z-score with ddof=1 and a dot product over n-1)
//   -fc_diff  |mean(sim_fc) - mean(emp_fc)|               (base.py:1165-1168)
//   -fc_normec ||sim_fc - emp_fc|| / (2 sqrt(n_pairs))     (base.py:1169-1173)
// k_fcd_ks: one CTA per simulation; the simulated FCD row is sorted in shared
//   memory (bitonic), then every element x of the pooled sample gets
//   F_sim(x) = #(sim <= x)/m1 and F_emp(x) = #(emp <= x)/m2 by binary search
//   (searchsorted side='right'), and the statistic is max |F_sim - F_emp| --
//   the same quantities scipy.stats.ks_2samp forms, so the value is bit-equal.
#include <cfloat>
#include "engine.h"

namespace cbnm {
namespace {

constexpr int GOF_THREADS = 256;

__device__ double bsum(double v, double *red) {
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

__device__ double bmax(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, red[w]);
        red[32] = t;
    }
    __syncthreads();
    return red[32];
}

__global__ void __launch_bounds__(GOF_THREADS) k_fc_gof(const GofArgs a) {
    __shared__ double red[33];
    const int sim = blockIdx.x;
    const int P = a.n_pairs;
    const double *x = a.sim_fc + (size_t)sim * P;
    double s = 0.0;
    for (int p = threadIdx.x; p < P; p += blockDim.x) s += x[p];
    const double mx = bsum(s, red) / P;
    double sxx = 0.0, sxy = 0.0, sd2 = 0.0;
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        const double dx = x[p] - mx, dy = a.emp_fc[p] - a.emp_fc_mean, d = x[p] - a.emp_fc[p];
        sxx += dx * dx;
        sxy += dx * dy;
        sd2 += d * d;
    }
    sxx = bsum(sxx, red);
    sxy = bsum(sxy, red);
    sd2 = bsum(sd2, red);
    if (threadIdx.x == 0) {
        if (a.fc_corr) a.fc_corr[sim] = sxy / (sqrt(sxx) * a.emp_fc_ssd);
        if (a.fc_diff) a.fc_diff[sim] = fabs(mx - a.emp_fc_mean);
        if (a.fc_normec) a.fc_normec[sim] = sqrt(sd2) / (2 * sqrt((double)P));
    }
}

__device__ __forceinline__ int count_le(const double *v, int m, double x) {  // searchsorted(v, x, 'right')
    int lo = 0, hi = m;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (x < v[mid]) hi = mid; else lo = mid + 1;
    }
    return lo;
}

__global__ void __launch_bounds__(GOF_THREADS) k_fcd_ks(const GofArgs a, int m1p) {
    extern __shared__ double srt[];  // [m1p] power-of-two padded with +inf
    __shared__ double red[33];
    const int sim = blockIdx.x;
    const int m1 = a.n_wp, m2 = a.n_emp_fcd;
    const double *x = a.sim_fcd + (size_t)sim * m1;
    for (int i = threadIdx.x; i < m1p; i += blockDim.x) srt[i] = (i < m1) ? x[i] : DBL_MAX;
    __syncthreads();
    // bitonic sort, ascending (NaN-free input assumed; NaN handled by the caller)
    for (int k = 2; k <= m1p; k <<= 1) {
        for (int jj = k >> 1; jj > 0; jj >>= 1) {
            for (int i = threadIdx.x; i < m1p; i += blockDim.x) {
                const int l = i ^ jj;
                if (l > i) {
                    const double u = srt[i], v = srt[l];
                    const bool up = (i & k) == 0;
                    if ((u > v) == up) { srt[i] = v; srt[l] = u; }
                }
            }
            __syncthreads();
        }
    }
    double dmax = 0.0;
    for (int i = threadIdx.x; i < m1 + m2; i += blockDim.x) {
        const double v = (i < m1) ? srt[i] : a.emp_fcd_sorted[i - m1];
        const double c1 = (double)count_le(srt, m1, v) / m1;
        const double c2 = (double)count_le(a.emp_fcd_sorted, m2, v) / m2;
        dmax = fmax(dmax, fabs(c1 - c2));
    }
    dmax = bmax(dmax, red);
    if (threadIdx.x == 0) a.fcd_ks[sim] = dmax;
}

}  // namespace

size_t gof_ks_smem_limit() { return 160 * 1024; }

cudaError_t launch_gof(const GofArgs &a, cudaStream_t st, int *launches) {
    cudaError_t e = cudaSuccess;
    if (a.n_sims <= 0) return e;
    if (a.sim_fc && (a.fc_corr || a.fc_diff || a.fc_normec)) {
        k_fc_gof<<<a.n_sims, GOF_THREADS, 0, st>>>(a);
        if (launches) ++*launches;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (a.sim_fcd && a.fcd_ks) {
        int m1p = 1;
        while (m1p < a.n_wp) m1p <<= 1;
        const size_t smem = sizeof(double) * (size_t)m1p;
        if (smem > gof_ks_smem_limit()) return cudaErrorInvalidValue;
        e = allow_dynamic_smem(k_fcd_ks);
        if (e != cudaSuccess) return e;
        k_fcd_ks<<<a.n_sims, GOF_THREADS, smem, st>>>(a, m1p);
        if (launches) ++*launches;
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace cbnm
