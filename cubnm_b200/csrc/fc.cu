// FC and FCD of simulated BOLD (reference: src/ext/fc.cu:4-239, src/ext/fc.cpp:1-91).
//
// k_fc: one CTA per (simulation, window); window 0 is the static FC over
//   volumes [n_vols_remove, bold_len), windows 1..W are the sliding windows.
//   The CTA stages the window's BOLD rows in shared memory, centres every node
//   column on its mean (two-pass mean and sqrt(sum of squares), as fc.cu does)
//   and then every thread forms Pearson r of node pairs:
//       r_ij = sum_t xc_ti * xc_tj / (ssd_i * ssd_j)
//   Static FC goes to the output, window FCs to a scratch array.
// k_fcd: one CTA per simulation: mean / ssd of every window-FC vector, then the
//   Pearson r of every pair of window-FC vectors (the FCD lower triangle).
// Window FCs are kept in scratch only for a chunk of simulations at a time
// (see session.cpp), so scratch stays bounded for any batch size.
#include "engine.h"

namespace cbnm {
namespace {

constexpr int FC_THREADS = 256;

// Deterministic block sum of one double per thread.
__device__ double block_sum(double v, double *red) {
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

__global__ void __launch_bounds__(FC_THREADS) k_fc(const FcArgs a, int staged) {
    extern __shared__ double sm[];
    const int sim = a.sim_begin + blockIdx.x;
    const int w = blockIdx.y;  // 0: static FC, 1..W: windows
    const int n = a.nodes;
    int r0, r1;
    if (w == 0) { r0 = a.n_vols_remove; r1 = a.bold_len; }
    else { r0 = a.w_start[w - 1]; r1 = a.w_end[w - 1] + 1; }
    const int T = r1 - r0;
    const double *bold = a.bold + (size_t)sim * a.bold_len * n + (size_t)r0 * n;
    double *mean = sm;          // [n]
    double *ssd = sm + n;       // [n]
    double *xc = sm + 2 * n;    // [T][n] centred window (when staged)
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double s = 0.0;
        for (int t = 0; t < T; ++t) s += bold[(size_t)t * n + j];
        s /= T;
        double q = 0.0;
        for (int t = 0; t < T; ++t) {
            const double d = bold[(size_t)t * n + j] - s;
            q += d * d;
        }
        mean[j] = s;
        ssd[j] = sqrt(q);
    }
    __syncthreads();
    if (staged) {
        for (int e = threadIdx.x; e < T * n; e += blockDim.x) xc[e] = bold[e] - mean[e % n];
        __syncthreads();
    }
    double *out = (w == 0) ? a.fc + (size_t)sim * a.n_pairs
                           : a.wfc + ((size_t)(sim - a.sim_begin) * a.n_windows + (w - 1)) * a.n_pairs;
    for (int p = threadIdx.x; p < a.n_pairs; p += blockDim.x) {
        const int i = a.pair_i[p], jj = a.pair_j[p];
        double cov = 0.0;
        if (staged) {
            for (int t = 0; t < T; ++t) cov += xc[t * n + i] * xc[t * n + jj];
        } else {
            const double mi = mean[i], mj = mean[jj];
            for (int t = 0; t < T; ++t) cov += (bold[(size_t)t * n + i] - mi) * (bold[(size_t)t * n + jj] - mj);
        }
        out[p] = cov / (ssd[i] * ssd[jj]);
    }
}

__global__ void __launch_bounds__(FC_THREADS) k_fcd(const FcArgs a) {
    __shared__ double red[33];
    __shared__ double wmean[1024], wssd[1024];
    const int sim = a.sim_begin + blockIdx.x;
    const int W = a.n_windows, P = a.n_pairs;
    const double *wfc = a.wfc + (size_t)(sim - a.sim_begin) * W * P;
    for (int w = 0; w < W; ++w) {
        const double *v = wfc + (size_t)w * P;
        double s = 0.0;
        for (int p = threadIdx.x; p < P; p += blockDim.x) s += v[p];
        const double m = block_sum(s, red) / P;
        double q = 0.0;
        for (int p = threadIdx.x; p < P; p += blockDim.x) {
            const double d = v[p] - m;
            q += d * d;
        }
        const double ss = sqrt(block_sum(q, red));
        if (threadIdx.x == 0) { wmean[w] = m; wssd[w] = ss; }
    }
    __syncthreads();
    // one warp per window pair, pairs in (wi > wj) row order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double *out = a.fcd + (size_t)sim * a.n_window_pairs;
    for (int wp = warp; wp < a.n_window_pairs; wp += nwarps) {
        // invert wp = wi*(wi-1)/2 + wj
        int wi = (int)((1.0 + sqrt(1.0 + 8.0 * wp)) * 0.5);
        while (wi * (wi - 1) / 2 > wp) --wi;
        while ((wi + 1) * wi / 2 <= wp) ++wi;
        const int wj = wp - wi * (wi - 1) / 2;
        const double *x = wfc + (size_t)wi * P, *y = wfc + (size_t)wj * P;
        const double mx = wmean[wi], my = wmean[wj];
        double c = 0.0;
        for (int p = lane; p < P; p += 32) c += (x[p] - mx) * (y[p] - my);
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0) out[wp] = c / (wssd[wi] * wssd[wj]);
    }
}

}  // namespace

cudaError_t launch_fc(const FcArgs &a, cudaStream_t st, int *launches) {
    // stage the largest window in shared memory when it fits
    const int maxT = a.max_T;
    size_t smem = sizeof(double) * (size_t)(2 * a.nodes + maxT * a.nodes);
    int staged = 1;
    if (smem > 200 * 1024) { staged = 0; smem = sizeof(double) * 2 * a.nodes; }
    cudaError_t e = allow_dynamic_smem(k_fc);
    if (e != cudaSuccess) return e;
    dim3 grid(a.sim_count, 1 + ((a.n_windows > 0) ? a.n_windows : 0));
    k_fc<<<grid, FC_THREADS, smem, st>>>(a, staged);
    if (launches) ++*launches;
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((a.n_windows > 0)) {
        if (a.n_windows > 1024) return cudaErrorInvalidValue;
        k_fcd<<<a.sim_count, FC_THREADS, 0, st>>>(a);
        if (launches) ++*launches;
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_fcd_only(const FcArgs &a, cudaStream_t st, int *launches) {
    if (a.n_windows > 1024) return cudaErrorInvalidValue;
    k_fcd<<<a.sim_count, FC_THREADS, 0, st>>>(a);
    if (launches) ++*launches;
    return cudaGetLastError();
}

}  // namespace cbnm
