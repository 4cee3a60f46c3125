// FC and FCD of device-resident BOLD with no device allocation.
//
// A variant of the k_fc / k_fcd pair in fc.cu for callers that must not
// allocate device memory: a host that has handed all free device memory to
// its own pooling allocator (where cudaMalloc fails or fragments the pool), or
// a fitting loop that keeps integration batches running on other streams
// (cudaFree synchronises the whole device and would stall them).  Everything
// the kernels need that fc.cu keeps in session buffers is either computed in
// the kernel or held in one fixed, file-scope device array:
//
//  * node pair p -> (i, j) and window w -> volume range are closed forms of
//    the call's scalars (the same enumeration as the session's host tables:
//    lower triangle in row order, src/ext/bnm.cu:809-835; windows as
//    src/ext/utils.cpp:21-52), so no index tables are uploaded;
//  * the window FCs of a chunk of simulations live in g_wfc_scratch
//    (NOALLOC_SCRATCH_BYTES).  The host loops over chunks that fit, in stream
//    order on the caller's stream.
//
// Nothing in the scratch has to start at zero: k_fc_scratch writes every
// window-FC entry that k_fcd_scratch later reads, earlier on the same stream.
// The scratch is one array per device, so two calls whose kernels overlap on
// the same device (different streams, or different host threads) race on it.
// The arithmetic, and its order, is that of fc.cu, so results are bit-identical.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include "engine.h"

namespace cbnm {
namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_MAX_WINDOWS = 1024;
constexpr int NA_MAX_DEVICES = 64;

static __device__ __align__(256) double g_wfc_scratch[NOALLOC_SCRATCH_BYTES / sizeof(double)];

struct NoAllocArgs {
    int nodes, bold_len, n_vols_remove, n_pairs, n_windows, n_window_pairs;
    int exc_inter;               // pairs within each hemisphere only
    int win_first, win_step, win_half;  // window w is centred on win_first + w * win_step
    int sim_begin;
    const double *bold;          // [n_sims][bold_len*nodes]
    double *fc;                  // [n_sims][n_pairs]
    double *fcd;                 // [n_sims][n_window_pairs]
    double *wfc;                 // scratch [chunk][n_windows][n_pairs]
};

// Row r and column c of entry q of a strictly lower triangle in row order
// (q = r (r - 1) / 2 + c, c < r).
__device__ __forceinline__ void tri_index(int q, int &r, int &c) {
    r = (int)((1.0 + sqrt(1.0 + 8.0 * (double)q)) * 0.5);
    while (r * (r - 1) / 2 > q) --r;
    while ((r + 1) * r / 2 <= q) ++r;
    c = q - r * (r - 1) / 2;
}

// FC entry p -> node pair (i, j), i > j.  With exc_inter the pairs are the
// left-hemisphere triangle (nodes [0, n/2)) followed by the right one.
__device__ __forceinline__ void pair_of(const NoAllocArgs &a, int p, int &i, int &j) {
    if (!a.exc_inter) { tri_index(p, i, j); return; }
    const int rh = a.nodes / 2, left = rh * (rh - 1) / 2;
    if (p < left) { tri_index(p, i, j); return; }
    tri_index(p - left, i, j);
    i += rh;
    j += rh;
}

__device__ double block_sum_na(double v, double *red) {
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

// One CTA per (simulation, window); window 0 is the static FC.
__global__ void __launch_bounds__(NA_THREADS) k_fc_scratch(const NoAllocArgs a, int staged) {
    extern __shared__ double sm[];
    const int sim = a.sim_begin + blockIdx.x;
    const int w = blockIdx.y;
    const int n = a.nodes;
    int r0, r1;
    if (w == 0) {
        r0 = a.n_vols_remove;
        r1 = a.bold_len;
    } else {
        const int ctr = a.win_first + (w - 1) * a.win_step;
        r0 = max(0, ctr - a.win_half);
        r1 = min(a.bold_len - 1, ctr + a.win_half) + 1;
    }
    const int T = r1 - r0;
    const double *bold = a.bold + (size_t)sim * a.bold_len * n + (size_t)r0 * n;
    double *mean = sm;
    double *ssd = sm + n;
    double *xc = sm + 2 * n;
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
                           : a.wfc + ((size_t)blockIdx.x * a.n_windows + (w - 1)) * a.n_pairs;
    for (int p = threadIdx.x; p < a.n_pairs; p += blockDim.x) {
        int i, jj;
        pair_of(a, p, i, jj);
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

// One CTA per simulation: Pearson r of every pair of its window-FC vectors.
__global__ void __launch_bounds__(NA_THREADS) k_fcd_scratch(const NoAllocArgs a) {
    __shared__ double red[33];
    __shared__ double wmean[NA_MAX_WINDOWS], wssd[NA_MAX_WINDOWS];
    const int sim = a.sim_begin + blockIdx.x;
    const int W = a.n_windows, P = a.n_pairs;
    const double *wfc = a.wfc + (size_t)blockIdx.x * W * P;
    for (int w = 0; w < W; ++w) {
        const double *v = wfc + (size_t)w * P;
        double s = 0.0;
        for (int p = threadIdx.x; p < P; p += blockDim.x) s += v[p];
        const double m = block_sum_na(s, red) / P;
        double q = 0.0;
        for (int p = threadIdx.x; p < P; p += blockDim.x) {
            const double d = v[p] - m;
            q += d * d;
        }
        const double ss = sqrt(block_sum_na(q, red));
        if (threadIdx.x == 0) { wmean[w] = m; wssd[w] = ss; }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double *out = a.fcd + (size_t)sim * a.n_window_pairs;
    for (int wp = warp; wp < a.n_window_pairs; wp += nwarps) {
        int wi, wj;
        tri_index(wp, wi, wj);
        const double *x = wfc + (size_t)wi * P, *y = wfc + (size_t)wj * P;
        const double mx = wmean[wi], my = wmean[wj];
        double c = 0.0;
        for (int p = lane; p < P; p += 32) c += (x[p] - mx) * (y[p] - my);
        for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
        if (lane == 0) out[wp] = c / (wssd[wi] * wssd[wj]);
    }
}

int fail(char *msg, size_t cap, int code, const char *text) {
    std::snprintf(msg, cap, "%s", text);
    return code;
}

int fail_cuda(char *msg, size_t cap, cudaError_t e) {
    std::snprintf(msg, cap, "CUDA Error: %s", cudaGetErrorString(e));
    return 4;  // CBNM_ERR_CUDA
}

}  // namespace

int fc_fcd_noalloc(const double *bold, int n_sims, int bold_len, int nodes, int n_vols_remove, int window_size,
                   int window_step, int drop_edges, int exc_inter, double *fc, double *fcd, cudaStream_t st,
                   char *msg, size_t cap) {
    // status codes of the C ABI: 1 argument, 3 configuration, 4 CUDA
    if (!bold || !fc) return fail(msg, cap, 1, "bold and fc must be device pointers");
    if (n_sims < 1 || nodes < 2 || bold_len < 1 || n_vols_remove < 0)
        return fail(msg, cap, 1, "n_sims >= 1, nodes >= 2, bold_len >= 1 and n_vols_remove >= 0 are required");
    const int corr_len = bold_len - n_vols_remove;
    if (corr_len < 2) return fail(msg, cap, 3, "fewer than 2 BOLD volumes left for FC after n_vols_remove");
    if (exc_inter && nodes % 2 != 0)
        return fail(msg, cap, 3, "exc_interhemispheric is set but number of nodes is not even");
    NoAllocArgs a;
    a.nodes = nodes; a.bold_len = bold_len; a.n_vols_remove = n_vols_remove; a.exc_inter = exc_inter ? 1 : 0;
    a.n_pairs = nodes * (nodes - 1) / 2 - (a.exc_inter ? (nodes / 2) * (nodes / 2) : 0);
    // two nodes with exc_interhemispheric leave no pair (one node per hemisphere)
    if (a.n_pairs < 1) return fail(msg, cap, 3, "no node pairs for FC (exc_interhemispheric with 2 nodes)");
    a.n_windows = 0; a.n_window_pairs = 0; a.win_first = 0; a.win_step = 1; a.win_half = 0; a.sim_begin = 0;
    a.bold = bold; a.fc = fc; a.fcd = fcd; a.wfc = nullptr;
    int max_T = corr_len;
    if (fcd) {  // utils.cpp:21-52
        if (window_step <= 0) return fail(msg, cap, 3, "window_step must be positive");
        if (window_size < 0) return fail(msg, cap, 3, "window_size must not be negative");
        const int half = window_size / 2;
        const int first = (drop_edges ? half : 0) + n_vols_remove;
        const int last = (drop_edges ? corr_len - 1 - half : corr_len - 1) + n_vols_remove;
        a.n_windows = (last >= first) ? (last - first) / window_step + 1 : 0;
        if (a.n_windows == 0) return fail(msg, cap, 3, "Number of dynamic FC windows is 0");
        if (a.n_windows > NA_MAX_WINDOWS) return fail(msg, cap, 1, "at most 1024 dynamic FC windows are supported");
        a.n_window_pairs = a.n_windows * (a.n_windows - 1) / 2;
        a.win_first = first; a.win_step = window_step; a.win_half = half;
        max_T = std::max(max_T, 2 * half + 1);
    }
    const size_t per_sim = sizeof(double) * (size_t)a.n_windows * a.n_pairs;
    int chunk = n_sims;
    if (fcd) {
        if (per_sim > NOALLOC_SCRATCH_BYTES) {
            std::snprintf(msg, cap,
                          "the window FCs of one simulation need %zu bytes (%d windows x %d pairs), more than the "
                          "%zu-byte scratch of cbnm_fc_fcd_noalloc",
                          per_sim, a.n_windows, a.n_pairs, (size_t)NOALLOC_SCRATCH_BYTES);
            return 1;
        }
        chunk = (int)std::min<size_t>((size_t)n_sims, NOALLOC_SCRATCH_BYTES / per_sim);
        // the scratch address, looked up once per device with that device current
        static std::mutex mu;
        static void *addr[NA_MAX_DEVICES] = {};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return fail_cuda(msg, cap, e);
        if (dev < 0 || dev >= NA_MAX_DEVICES) return fail(msg, cap, 1, "device ordinal beyond 63");
        {
            std::lock_guard<std::mutex> lock(mu);
            if (!addr[dev]) {
                void *p = nullptr;
                e = cudaGetSymbolAddress((void **)&p, g_wfc_scratch);
                if (e != cudaSuccess) return fail_cuda(msg, cap, e);
                addr[dev] = p;
            }
            a.wfc = (double *)addr[dev];
        }
    }
    size_t smem = sizeof(double) * (size_t)(2 * nodes + (size_t)max_T * nodes);
    int staged = 1;
    if (smem > 200 * 1024) { staged = 0; smem = sizeof(double) * 2 * nodes; }
    cudaError_t e = allow_dynamic_smem(k_fc_scratch);
    if (e != cudaSuccess) return fail_cuda(msg, cap, e);
    for (int s0 = 0; s0 < n_sims; s0 += chunk) {
        const int cnt = std::min(chunk, n_sims - s0);
        a.sim_begin = s0;
        k_fc_scratch<<<dim3(cnt, 1 + a.n_windows), NA_THREADS, smem, st>>>(a, staged);
        e = cudaGetLastError();
        if (e != cudaSuccess) return fail_cuda(msg, cap, e);
        if (fcd) {
            k_fcd_scratch<<<cnt, NA_THREADS, 0, st>>>(a);
            e = cudaGetLastError();
            if (e != cudaSuccess) return fail_cuda(msg, cap, e);
        }
    }
    msg[0] = 0;
    return 0;
}

}  // namespace cbnm
