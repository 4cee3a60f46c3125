// Measured FP32 throughput of this GPU, the denominator of the integrator's
// FP32 roofline: chains of independent fused multiply-adds, scalar (FFMA) and
// packed two-wide (FFMA2), timed with CUDA events; two flops per FMA lane.
#include <algorithm>
#include "engine.h"

namespace cbnm {
namespace {

constexpr int PK_THREADS = 256;
constexpr int PK_CHAINS = 8;

__global__ void __launch_bounds__(PK_THREADS) k_peak_ffma(float *sink, int iters, float a, float b) {
    float x[PK_CHAINS];
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) x[c] = threadIdx.x * 1e-3f + c;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int c = 0; c < PK_CHAINS; ++c) x[c] = fmaf(x[c], a, b);
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) s += x[c];
    if (s == 1234.5f) sink[blockIdx.x] = s;  // keeps the chains alive
}

__global__ void __launch_bounds__(PK_THREADS) k_peak_ffma2(float *sink, int iters, float a, float b) {
    float2 x[PK_CHAINS];
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) x[c] = make_float2(threadIdx.x * 1e-3f + c, c * 0.5f);
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int c = 0; c < PK_CHAINS; ++c) x[c] = __ffma2_rn(x[c], a2, b2);
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) s += x[c].x + x[c].y;
    if (s == 1234.5f) sink[blockIdx.x] = s;
}

}  // namespace

cudaError_t measure_fp32_peak(double *ffma_tflops, double *ffma2_tflops) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = sms * 8, iters = 1 << 16;
    float *sink = nullptr;
    if ((e = cudaMalloc(&sink, sizeof(float) * grid)) != cudaSuccess) return e;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    double best1 = 0.0, best2 = 0.0;
    for (int rep = 0; rep < 3; ++rep) {
        float ms = 0.0f;
        cudaEventRecord(t0);
        k_peak_ffma<<<grid, PK_THREADS>>>(sink, iters, 0.9999f, 1e-4f);
        cudaEventRecord(t1);
        cudaEventSynchronize(t1);
        cudaEventElapsedTime(&ms, t0, t1);
        best1 = std::max(best1, 2.0 * PK_CHAINS * (double)iters * grid * PK_THREADS / (ms * 1e-3) / 1e12);
        cudaEventRecord(t0);
        k_peak_ffma2<<<grid, PK_THREADS>>>(sink, iters, 0.9999f, 1e-4f);
        cudaEventRecord(t1);
        cudaEventSynchronize(t1);
        cudaEventElapsedTime(&ms, t0, t1);
        best2 = std::max(best2, 4.0 * PK_CHAINS * (double)iters * grid * PK_THREADS / (ms * 1e-3) / 1e12);
    }
    e = cudaGetLastError();
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(sink);
    *ffma_tflops = best1;
    *ffma2_tflops = best2;
    return e;
}

}  // namespace cbnm
