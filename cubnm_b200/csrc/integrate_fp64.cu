// FP64 integrator: the reference-precision path (the "plain" GPU method).
//
// The per-simulation kernel of integrate_sim.cuh with R = double: one CTA per
// simulation, one thread per node, everything in FP64, so that its output
// matches the reference's double build on the same noise.  This file is
// compiled with --fmad=false: every multiply and add rounds separately, in the
// same order as the reference's C++ (src/ext/models/<model>.cpp h_step,
// src/ext/models/bw.cpp:24-35), so the only differences left are the last-ulp
// differences between CUDA's and glibc's exp/pow/sin.
//
// Time loop: src/ext/bnm.cu:117-505 (GPU) and src/ext/bnm.cpp:69-522 (CPU);
// coupling: bnm.cu:48-101; numerical FIC: src/ext/models/rww.cpp:233-298.
#include "integrate_sim.cuh"

namespace cbnm {

cudaError_t launch_integrate_fp64(int model, const IntegrateArgs &a, cudaStream_t st) {
    return launch_sim_model<double>(model, a, st);
}

}  // namespace cbnm
