// FP32 per-simulation integrator: the FP32-mode kernel for what the
// tensor-core tile kernel (integrate_fp32.cu) does not take -- conduction
// delays, numerical FIC, Kuramoto, more than 128 nodes.
//
// The per-simulation kernel of integrate_sim.cuh with R = float: node state,
// parameters, SC, noise and delay ring buffers in FP32 (half the bytes of the
// FP64 path for the gather-bound delayed coupling, MUFU exp instead of the
// FP64 software exp), Balloon-Windkessel state and BOLD in FP64.  Compiled with
// FMA contraction.
#include "integrate_sim.cuh"

namespace cbnm {

cudaError_t launch_integrate_simt32(int model, const IntegrateArgs &a, cudaStream_t st) {
    return launch_sim_model<float>(model, a, st);
}

}  // namespace cbnm
