// FC and window FCs as tensor-core Gram products (FP32 mode).
//
// Pearson r over a window's volumes is the Gram product of the normalised
// columns (reference: src/ext/fc.cu:77-239, fc.cpp:1-91):
//     FC_ij = sum_t Z_ti Z_tj,   Z_ti = (x_ti - mean_i) / sqrt(sum_t (x_ti - mean_i)^2)
// The means and root sums of squares are FP64 (as the reference computes them),
// Z is split into BF16 hi + lo and the product runs on tcgen05 in BF16x3
// (hi hi + hi lo + lo hi, FP32 accumulation; |error| about 1e-5, against the
// mixed-precision bound |dFC| <= 2e-3).  One CTA per (simulation, window, pair
// of 128-node blocks bi >= bj): A = Z_I^T in TMEM (node m on lane m, two volumes
// per 32-bit column, hi then lo), B = Z_J in shared memory (MN-major, no swizzle,
// element (k, j) at (k/8) 2048 + (j/8) 128 + (k%8) 16 + (j%8) 2), D (128 x 128
// FP32) in TMEM, read back by the four warps (one lane quarter each) and written
// to the pair order of the output (np.tril_indices(n, -1), or the intra-hemisphere
// order) through a node-pair index table.  Volumes run in chunks of 256.  The
// FCD is the same construction one level up (k_fcd_tc): the Gram product of the
// normalised window-FC vectors over the node pairs, for up to 128 windows.
#include <algorithm>
#include <cuda_bf16.h>
#include "engine.h"
#include "tc_common.cuh"

namespace cbnm {
namespace {

constexpr int FT_THREADS = 128;
constexpr int FT_N = 128;                       // nodes per block (MMA M and N)
constexpr int FT_KC = 256;                      // volumes per chunk (multiple of 16)
constexpr uint32_t FT_LBO = (FT_N / 8) * 128;   // K-direction core-matrix stride of B
constexpr int FT_COL_A = FT_N;                  // TMEM: D [0, 128), A hi [128, 256), A lo [256, 384)
// FCD: the accumulator restarts every FT_FLUSH chunks (1,024 node pairs, a chain of
// at most 192 FP32 additions) and each group's sums are added into FP64 partials;
// one accumulation over the 499,500 pairs of 1,000 nodes had drifted by ~1e-3.
constexpr int FT_FLUSH = 4;

struct FtSmem {
    uint64_t mbar;
    uint32_t tmem_base;
};

__device__ __forceinline__ uint16_t bf16_bits(float v) {
    __nv_bfloat16 b = __float2bfloat16_rn(v);
    return *reinterpret_cast<uint16_t *>(&b);
}

__global__ void __launch_bounds__(FT_THREADS, 1) k_fc_tc(const FcArgs a, const int *pidx, int nblk) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *Bh = smem_raw, *Bl = smem_raw + (size_t)FT_KC * FT_N * 2;
    FtSmem *sm = reinterpret_cast<FtSmem *>(smem_raw + (size_t)2 * FT_KC * FT_N * 2);
    const int ls = blockIdx.x, sim = a.sim_begin + ls, w = blockIdx.y, n = a.nodes;
    // block pair (bi >= bj) of blockIdx.z in row order
    int bi = 0;
    while ((bi + 1) * (bi + 2) / 2 <= (int)blockIdx.z) ++bi;
    const int bj = blockIdx.z - bi * (bi + 1) / 2;
    (void)nblk;
    const int tid = threadIdx.x, warp = tid >> 5;
    int r0, r1;
    if (w == 0) { r0 = a.n_vols_remove; r1 = a.bold_len; }
    else { r0 = a.w_start[w - 1]; r1 = a.w_end[w - 1] + 1; }
    const int T = r1 - r0, K = ((T + 15) / 16) * 16;
    const double *x = a.bold + (size_t)sim * a.bold_len * n + (size_t)r0 * n;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm->tmem_base)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&sm->mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = sm->tmem_base;
    const uint32_t t_lane = tmem + ((uint32_t)(warp * 32) << 16);

    // column statistics (FP64, two passes) of node i = bi*128 + tid (A) and j = bj*128 + tid (B)
    const int ni = bi * FT_N + tid, nj = bj * FT_N + tid;
    double mi = 0.0, si = 1.0, mj = 0.0, sj = 1.0;
    if (ni < n) {
        double s = 0.0;
        for (int t = 0; t < T; ++t) s += x[(size_t)t * n + ni];
        mi = s / T;
        double q = 0.0;
        for (int t = 0; t < T; ++t) {
            const double d = x[(size_t)t * n + ni] - mi;
            q += d * d;
        }
        si = sqrt(q);
    }
    if (nj < n) {
        double s = 0.0;
        for (int t = 0; t < T; ++t) s += x[(size_t)t * n + nj];
        mj = s / T;
        double q = 0.0;
        for (int t = 0; t < T; ++t) {
            const double d = x[(size_t)t * n + nj] - mj;
            q += d * d;
        }
        sj = sqrt(q);
    }
    const uint32_t idesc = instr_desc(FT_N);
    uint32_t phase = 0;
    bool ok = true;
    for (int kc0 = 0; kc0 < K; kc0 += FT_KC) {
        const int kc = min(FT_KC, K - kc0);
        // A = Z_I^T: lane tid, volume pairs into 32-bit columns, hi then lo
        for (int c0 = 0; c0 < kc / 2; c0 += 8) {
            uint32_t hw[8], lw[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                float v[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int t = kc0 + 2 * (c0 + c) + u;
                    v[u] = (ni < n && t < T) ? (float)((x[(size_t)t * n + ni] - mi) / si) : 0.0f;
                }
                split_bf16x2(v[0], v[1], hw[c], lw[c]);
            }
            tmem_st8(t_lane + FT_COL_A + c0, hw);
            tmem_st8(t_lane + FT_COL_A + FT_KC / 2 + c0, lw);
        }
        // B = Z_J in shared memory, column tid
        for (int k = 0; k < kc; ++k) {
            const int t = kc0 + k;
            const float v = (nj < n && t < T) ? (float)((x[(size_t)t * n + nj] - mj) / sj) : 0.0f;
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            const float lo = v - __bfloat162float(h);
            const uint32_t off = (k >> 3) * FT_LBO + (tid >> 3) * 128 + (k & 7) * 16 + (tid & 7) * 2;
            *reinterpret_cast<uint16_t *>(Bh + off) = *reinterpret_cast<const uint16_t *>(&h);
            *reinterpret_cast<uint16_t *>(Bl + off) = bf16_bits(lo);
        }
        fence_proxy_async();
        fence_before();
        __syncthreads();
        if (tid == 0) {
            fence_after();
            const uint32_t bh = smem_u32(Bh), bl = smem_u32(Bl);
            for (int kk = 0; kk < kc / 16; ++kk) {
                const uint32_t tah = tmem + FT_COL_A + kk * 8, tal = tah + FT_KC / 2;
                const uint64_t dbh = smem_desc(bh + kk * 2 * FT_LBO, FT_LBO, 128);
                const uint64_t dbl = smem_desc(bl + kk * 2 * FT_LBO, FT_LBO, 128);
                mma_bf16_ts(tmem, tah, dbh, idesc, (kc0 % (FT_FLUSH * FT_KC) > 0 || kk > 0) ? 1u : 0u);
                mma_bf16_ts(tmem, tah, dbl, idesc, 1u);
                mma_bf16_ts(tmem, tal, dbh, idesc, 1u);
            }
            mma_commit(smem_u32(&sm->mbar));
        }
        // every thread waits for the chunk's MMAs (they read A and B) before the next chunk overwrites them
        ok = mbar_wait(smem_u32(&sm->mbar), phase) && ok;
        phase ^= 1u;
        fence_after();
        ok = __syncthreads_and(ok) != 0;  // the same decision in every thread
        if (!ok) break;
    }
    if (!ok) atomicExch(a.status_fc, 1);
    // D: lane quarter of this warp, 16 columns at a time -> output pairs (i > j)
    double *out = (w == 0) ? a.fc + (size_t)sim * a.n_pairs : a.wfc + ((size_t)ls * a.n_windows + (w - 1)) * a.n_pairs;
    if (ok) {
        for (int c0 = 0; c0 < FT_N; c0 += 16) {
            uint32_t r[16];
            tmem_ld16(t_lane + c0, r);
#pragma unroll
            for (int c = 0; c < 16; ++c) {
                const int j = bj * FT_N + c0 + c;
                if (ni < n && j < n && ni > j) {
                    const int p = pidx[(size_t)ni * n + j];
                    if (p >= 0) out[p] = (double)__uint_as_float(r[c]);
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

// Mean and root sum of squares (FP64, two passes) of every window-FC vector of a
// simulation: one warp per window.
__global__ void __launch_bounds__(256) k_wfc_stats(const FcArgs a) {
    const int ls = blockIdx.x, W = a.n_windows, P = a.n_pairs;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int w = warp; w < W; w += blockDim.x >> 5) {
        const double *v = a.wfc + ((size_t)ls * W + w) * P;
        double s = 0.0;
        for (int p = lane; p < P; p += 32) s += v[p];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        const double m = s / P;
        double q = 0.0;
        for (int p = lane; p < P; p += 32) {
            const double d = v[p] - m;
            q += d * d;
        }
        for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
        if (lane == 0) {
            a.wstat[((size_t)ls * W + w) * 2] = m;
            a.wstat[((size_t)ls * W + w) * 2 + 1] = sqrt(q);
        }
    }
}

// FCD of one simulation as the Gram product of its normalised window-FC vectors,
//     FCD_ab = sum_p Zw_ap Zw_bp,   Zw_ap = (FC^a_p - mean_a) / sqrt(sum_p (FC^a_p - mean_a)^2),
// with the pairs p as the K dimension (chunks of 256): A = Zw (window on lane, two
// pairs per 32-bit column, hi then lo) in TMEM, B = Zw^T (MN-major, window columns)
// in shared memory, BF16x3, D (windows x windows, N = windows padded to 16) in
// TMEM; at most 128 windows.
__global__ void __launch_bounds__(FT_THREADS, 1) k_fcd_tc(const FcArgs a, int NW) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    const uint32_t lbo = (uint32_t)(NW / 8) * 128;   // K-direction core-matrix stride of B
    uint8_t *Bh = smem_raw, *Bl = smem_raw + (size_t)FT_KC * NW * 2;
    const int ls = blockIdx.x, sim = a.sim_begin + ls, W = a.n_windows, P = a.n_pairs;
    double *part = reinterpret_cast<double *>(smem_raw + (size_t)2 * FT_KC * NW * 2);  // FCD lower triangle
    const int WP = W * (W - 1) / 2;
    FtSmem *sm = reinterpret_cast<FtSmem *>(part + ((WP + 1) & ~1));
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm->tmem_base)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&sm->mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int k = tid; k < WP; k += blockDim.x) part[k] = 0.0;
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = sm->tmem_base;
    const uint32_t t_lane = tmem + ((uint32_t)(warp * 32) << 16);
    const bool live = tid < W;
    const double *v = a.wfc + ((size_t)ls * W + (live ? tid : 0)) * P;
    const double m = live ? a.wstat[((size_t)ls * W + tid) * 2] : 0.0;
    const double ss = live ? a.wstat[((size_t)ls * W + tid) * 2 + 1] : 1.0;
    const uint32_t idesc = instr_desc(NW);
    const int K = ((P + 15) / 16) * 16;
    uint32_t phase = 0;
    bool ok = true;
    for (int kc0 = 0; kc0 < K; kc0 += FT_KC) {
        const int kc = min(FT_KC, K - kc0);
        for (int c0 = 0; c0 < kc / 2; c0 += 8) {
            uint32_t hw[8], lw[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                float z[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int p = kc0 + 2 * (c0 + c) + u;
                    z[u] = (live && p < P) ? (float)((v[p] - m) / ss) : 0.0f;
                }
                split_bf16x2(z[0], z[1], hw[c], lw[c]);
                // the same values, as B's column tid (rows 2 (c0 + c) and 2 (c0 + c) + 1)
                if (tid < NW) {
#pragma unroll
                    for (int u = 0; u < 2; ++u) {
                        const int k = 2 * (c0 + c) + u;
                        const uint32_t off = (k >> 3) * lbo + (tid >> 3) * 128 + (k & 7) * 16 + (tid & 7) * 2;
                        const __nv_bfloat16 h = __float2bfloat16_rn(z[u]);
                        *reinterpret_cast<uint16_t *>(Bh + off) = *reinterpret_cast<const uint16_t *>(&h);
                        *reinterpret_cast<uint16_t *>(Bl + off) = bf16_bits(z[u] - __bfloat162float(h));
                    }
                }
            }
            tmem_st8(t_lane + FT_COL_A + c0, hw);
            tmem_st8(t_lane + FT_COL_A + FT_KC / 2 + c0, lw);
        }
        fence_proxy_async();
        fence_before();
        __syncthreads();
        if (tid == 0) {
            fence_after();
            const uint32_t bh = smem_u32(Bh), bl = smem_u32(Bl);
            for (int kk = 0; kk < kc / 16; ++kk) {
                const uint32_t tah = tmem + FT_COL_A + kk * 8, tal = tah + FT_KC / 2;
                const uint64_t dbh = smem_desc(bh + kk * 2 * lbo, lbo, 128);
                const uint64_t dbl = smem_desc(bl + kk * 2 * lbo, lbo, 128);
                mma_bf16_ts(tmem, tah, dbh, idesc, (kc0 % (FT_FLUSH * FT_KC) > 0 || kk > 0) ? 1u : 0u);
                mma_bf16_ts(tmem, tah, dbl, idesc, 1u);
                mma_bf16_ts(tmem, tal, dbh, idesc, 1u);
            }
            mma_commit(smem_u32(&sm->mbar));
        }
        ok = mbar_wait(smem_u32(&sm->mbar), phase) && ok;
        phase ^= 1u;
        fence_after();
        ok = __syncthreads_and(ok) != 0;
        if (!ok) break;
        if ((kc0 / FT_KC) % FT_FLUSH == FT_FLUSH - 1 || kc0 + FT_KC >= K) {  // the group's sums into FP64
            for (int c0 = 0; c0 < NW; c0 += 16) {
                uint32_t r[16];
                tmem_ld16(t_lane + c0, r);
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const int wb = c0 + c;
                    if (live && wb < tid) part[tid * (tid - 1) / 2 + wb] += (double)__uint_as_float(r[c]);
                }
            }
        }
    }
    if (!ok) atomicExch(a.status_fc, 1);
    double *out = a.fcd + (size_t)sim * a.n_window_pairs;
    __syncthreads();
    if (ok)
        for (int k = tid; k < WP; k += blockDim.x) out[k] = part[k];
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}

}  // namespace

// FC (and window FCs when a.n_windows > 0) of a chunk on the tensor cores, then the
// FCD: on the tensor cores too for at most 128 windows, else on fc.cu's FP64 kernel.
cudaError_t launch_fc_tc(const FcArgs &a, const int *pidx, cudaStream_t st, int *launches) {
    const int nblk = (a.nodes + FT_N - 1) / FT_N;
    const size_t smem = (size_t)2 * FT_KC * FT_N * 2 + sizeof(FtSmem) + 64;
    cudaError_t e = allow_dynamic_smem(k_fc_tc);
    if (e != cudaSuccess) return e;
    dim3 grid(a.sim_count, 1 + a.n_windows, nblk * (nblk + 1) / 2);
    k_fc_tc<<<grid, FT_THREADS, smem, st>>>(a, pidx, nblk);
    if (launches) ++*launches;
    e = cudaGetLastError();
    if (e != cudaSuccess || a.n_windows == 0) return e;
    if (a.n_windows > FT_N || a.n_windows < 2) return launch_fcd_only(a, st, launches);
    k_wfc_stats<<<a.sim_count, 256, 0, st>>>(a);
    if (launches) ++*launches;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int NW = ((a.n_windows + 15) / 16) * 16;
    const int WP = a.n_windows * (a.n_windows - 1) / 2;
    const size_t fsmem = (size_t)2 * FT_KC * NW * 2 + sizeof(double) * ((WP + 1) & ~1) + sizeof(FtSmem) + 64;
    e = allow_dynamic_smem(k_fcd_tc);
    if (e != cudaSuccess) return e;
    k_fcd_tc<<<a.sim_count, FT_THREADS, fsmem, st>>>(a, NW);
    if (launches) ++*launches;
    return cudaGetLastError();
}

}  // namespace cbnm
