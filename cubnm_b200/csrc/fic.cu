// rWW analytical FIC on the GPU: one CTA per simulation, one thread per node
// (strided when nodes > blockDim), FP64, the arithmetic of fic.cuh.  Replaces
// the reference's host loop over simulations and nodes (rww.cpp:73-146), which
// is serial work of O(sims x nodes x (nodes + Brent iterations)) before every run.
#include "fic.cuh"

namespace cbnm {
namespace {

__global__ void __launch_bounds__(1024) k_rww_fic(const FicArgs a) {
    const int sim = blockIdx.x;
    const int n = a.nodes;
    const size_t stride = (size_t)a.n_sims * n;
    const double *sc = a.sc + (size_t)a.sc_idx[sim] * n * n;
    const double G = a.gparams[sim];
    int bad = 0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const double w_p = a.regional[0 * stride + (size_t)sim * n + j];
        const double J_N = a.regional[1 * stride + (size_t)sim * n + j];
        const double w = rww_fic_node(sc, n, j, G, w_p, J_N, a.K);
        if (w < 0) bad = 1;
        a.regional[2 * stride + (size_t)sim * n + j] = w;
    }
    bad = __syncthreads_or(bad);
    if (bad)
        for (int j = threadIdx.x; j < n; j += blockDim.x) a.regional[2 * stride + (size_t)sim * n + j] = 1.0;
    if (threadIdx.x == 0) a.unstable[sim] = (unsigned char)bad;
}

}  // namespace

cudaError_t launch_rww_fic(const FicArgs &a, cudaStream_t st) {
    const int threads = std::min(1024, ((a.nodes + 31) / 32) * 32);
    k_rww_fic<<<a.n_sims, threads, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace cbnm
