// FP32 lane kernel with the tangent along G (forward-mode dBOLD/dG), rWW and WC
// (see lanes.cuh and tangent.cuh).
#include "lanes.cuh"

namespace cbnm {

cudaError_t launch_integrate_lanes_tan(int model, const IntegrateArgs &a, cudaStream_t st) {
    switch (model) {
        case MODEL_RWW: return lanes::launch_model<RWWm<float>, true>(a, st);
        case MODEL_WC: return lanes::launch_model<WCm<float>, true>(a, st);
    }
    return cudaErrorNotSupported;
}

}  // namespace cbnm
