// FP32 lane kernel: the forward integrator (see lanes.cuh for the design).
#include "lanes.cuh"

namespace cbnm {

// Node rows per thread (a power of two) for a node count: threads / 16 nodes per row.
int lanes_rows(int nodes, int threads) {
    int mn = 1;
    while (mn * (threads / 16) < nodes) mn *= 2;
    return mn;
}

bool lanes_tangent_supported(int model) { return model == MODEL_RWW || model == MODEL_WC; }

bool lanes_supported(int model, int nodes, bool numerical_fic) {
    if (nodes < 1 || nodes > 16 * 64 || numerical_fic) return false;
    if (model == MODEL_JR) return lanes_rows(nodes, 1024) <= 4;  // 8 state variables a node in registers
    return model == MODEL_RWW || model == MODEL_WC || model == MODEL_RWWEX;
}

cudaError_t launch_integrate_lanes_tan(int model, const IntegrateArgs &a, cudaStream_t st);  // integrate_lanes_tan.cu

cudaError_t launch_integrate_lanes_params(int model, const IntegrateArgs &a, cudaStream_t st) {
    switch (model) {
        case MODEL_RWW: return lanes::launch_params<RWWm<float>>(a, st);
        case MODEL_WC: return lanes::launch_params<WCm<float>>(a, st);
        case MODEL_JR: return lanes::launch_params<JRm<float>>(a, st);
        case MODEL_RWWEX: return lanes::launch_params<RWWExm<float>>(a, st);
    }
    return cudaErrorNotSupported;
}

cudaError_t launch_integrate_lanes_multi(int model, const IntegrateArgs *runs, const int2 *items, int n_items,
                                         int *counter, int mn, int grid, float *hist, long long hist_per_cta,
                                         double *bw, long long bw_per_cta, cudaStream_t st) {
    switch (model) {
        case MODEL_RWW:
            return lanes::launch_multi<RWWm<float>>(runs, items, n_items, counter, mn, grid, hist, hist_per_cta, bw,
                                                    bw_per_cta, st);
        case MODEL_WC:
            return lanes::launch_multi<WCm<float>>(runs, items, n_items, counter, mn, grid, hist, hist_per_cta, bw,
                                                   bw_per_cta, st);
        case MODEL_JR:
            return lanes::launch_multi<JRm<float>>(runs, items, n_items, counter, mn, grid, hist, hist_per_cta, bw,
                                                   bw_per_cta, st);
        case MODEL_RWWEX:
            return lanes::launch_multi<RWWExm<float>>(runs, items, n_items, counter, mn, grid, hist, hist_per_cta, bw,
                                                      bw_per_cta, st);
    }
    return cudaErrorNotSupported;
}

cudaError_t launch_integrate_lanes(int model, const IntegrateArgs &a, cudaStream_t st) {
    if (a.tan_bold) return launch_integrate_lanes_tan(model, a, st);
    switch (model) {
        case MODEL_RWW: return lanes::launch_model<RWWm<float>, false>(a, st);
        case MODEL_WC: return lanes::launch_model<WCm<float>, false>(a, st);
        case MODEL_JR: return lanes::launch_model<JRm<float>, false>(a, st);
        case MODEL_RWWEX: return lanes::launch_model<RWWExm<float>, false>(a, st);
    }
    return cudaErrorNotSupported;
}

}  // namespace cbnm
