// Noise segment generated on the GPU ("noise": "philox" in model_config).
//
// The reference draws the noise segment on the host, serially, from
// std::mt19937 + std::normal_distribution (src/ext/bnm.cu:1240-1245): ~6e7
// normals at 100 nodes and a 30-s segment.  This mode instead fills the same
// array in parallel from Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011):
// counter i = (i, 0, 0, 0), key = (seed, 0); the four 32-bit words give two
// 53-bit uniforms u1, u2 in (0, 1), and Box-Muller turns them into the normals
//     z[2i] = sqrt(-2 ln u1) cos(2 pi u2),   z[2i+1] = sqrt(-2 ln u1) sin(2 pi u2).
// The values differ from the reference's stream (no parity with its outputs);
// they are reproducible for a seed and independent of the launch shape.
#include "engine.h"

namespace cbnm {
namespace {

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(M0, c[0]), lo0 = M0 * c[0];
        const uint32_t hi1 = __umulhi(M1, c[2]), lo1 = M1 * c[2];
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += W0; k1 += W1;
    }
}

__global__ void k_philox_normals(uint32_t seed, double *out, float *out32, size_t count) {
    const size_t n_ctr = (count + 1) / 2;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n_ctr; i += (size_t)gridDim.x * blockDim.x) {
        uint32_t c[4] = {(uint32_t)i, 0u, 0u, 0u};
        philox4x32_10(c, seed, 0u);
        const uint64_t a = ((((uint64_t)c[0]) << 32) | c[1]) >> 11;
        const uint64_t b = ((((uint64_t)c[2]) << 32) | c[3]) >> 11;
        const double u1 = ((double)a + 0.5) * 0x1.0p-53, u2 = ((double)b + 0.5) * 0x1.0p-53;
        const double r = sqrt(-2.0 * log(u1));
        double s, co;
        sincospi(2.0 * u2, &s, &co);
        const double z0 = r * co, z1 = r * s;
        out[2 * i] = z0;
        if (out32) out32[2 * i] = (float)z0;
        if (2 * i + 1 < count) {
            out[2 * i + 1] = z1;
            if (out32) out32[2 * i + 1] = (float)z1;
        }
    }
}

}  // namespace

cudaError_t launch_philox_normals(uint32_t seed, double *out, float *out32, size_t count, cudaStream_t st) {
    k_philox_normals<<<148 * 8, 256, 0, st>>>(seed, out, out32, count);
    return cudaGetLastError();
}

}  // namespace cbnm
