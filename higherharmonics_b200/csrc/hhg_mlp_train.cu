// hhg_mlp_train.cu -- training of the step-size proposer on the tensor cores.
//
// Every GEMM of the forward and backward pass is a 128-row tile on the
// 5th-generation tensor cores: operands staged by the CTA's threads into
// shared memory in the canonical K-major layout without swizzle (8-row x
// 16-byte core matrices), one elected thread issues tcgen05.mma (kind::f16,
// BF16 inputs, FP32 accumulation in tensor memory) for each K = 16 slice,
// tcgen05.commit arrives on an mbarrier, and each warp reads its 32
// accumulator rows back with tcgen05.ld.  All waits are bounded; on a
// timeout the kernel raises an error flag, waits (bounded) for the MMAs it
// issued, frees its tensor memory and returns.
//
//   forward     Z_l = H_{l-1} W_l^T + b_l,  H_l = SiLU(Z_l)        (M = rows, N = 64)
//   output      y = H_3 w_4 + b_4, loss = mean (y - T)^2           (CUDA cores, 64 -> 1)
//   data grad   dH_{l-1} = dZ_l W_l,  dZ_{l-1} = dH_{l-1} SiLU'(Z_{l-1})  (N = 64 or 16)
//   weight grad dW_l = dZ_l^T H_{l-1} over a 64-row chunk, M padded to 128
//   Adam on FP32 master weights, then BF16 copies [n][k] and [k][n].
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hhg_gpu.h"
#include "hhg_device.cuh"

namespace {

using bf16 = __nv_bfloat16;
constexpr int kH = hhg::kMlpH;          // 64
constexpr int kIn = hhg::kMlpIn;        // 8
constexpr int kInPad = hhg::kMlpInPad;  // 16
constexpr int kRows = 128;              // rows per tile (M)
constexpr int kChunk = 64;              // batch rows per weight-gradient tile (K)
constexpr long long kSpin = 1ll << 24;  // bounded mbarrier polls

// FP32 master parameters on the device (the first layer's inputs padded to 16)
constexpr int kOffW1 = 0;                      // [64][16]
constexpr int kOffB1 = kOffW1 + kH * kInPad;   // [64]
constexpr int kOffW2 = kOffB1 + kH;            // [64][64]
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;            // [64][64]
constexpr int kOffB3 = kOffW3 + kH * kH;
constexpr int kOffW4 = kOffB3 + kH;            // [64]
constexpr int kOffB4 = kOffW4 + kH;            // [1]
constexpr int kNMaster = kOffB4 + 1;
// the ABI layout of hhg_mlp::params (first layer unpadded)
constexpr int aW1 = 0, aB1 = aW1 + kH * kIn, aW2 = aB1 + kH, aB2 = aW2 + kH * kH, aW3 = aB2 + kH,
              aB3 = aW3 + kH * kH, aW4 = aB3 + kH, aB4 = aW4 + kH;
static_assert(aB4 + 1 == HHG_MLP_N_PARAMS, "hhg_mlp parameter layout");

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier primitives (PTX ISA 8.7, sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major, no swizzle: start, leading byte
// offset (between the two 8-element K chunks of a K = 16 slice), stride byte
// offset (between 8-row groups), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: D f32, A/B bf16, both K-major, M = 128, N.
__host__ __device__ constexpr uint32_t umma_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(mbar)), "r"(count) : "memory");
}

// Bounded wait for phase `parity`; true when it completed.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity) {
    const uint32_t a = smem_u32(mbar);
    for (long long it = 0; it < kSpin; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, int ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(dst_smem)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 32 consecutive FP32 columns starting at taddr (one warp).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Byte offset of element (row, k) in a canonical K-major no-swizzle tile with
// `rows` rows: core matrix (row / 8, k / 8) at ((k / 8) * rows / 8 + row / 8) *
// 128, row (row % 8) at 16 B, element (k % 8) at 2 B.  LBO (next K chunk) =
// rows * 16, SBO (next row group) = 128.
__device__ __forceinline__ uint32_t kmaj_off(int row, int k, int rows) {
    return (uint32_t)((((k >> 3) * (rows >> 3) + (row >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1));
}

// Run the K/16 MMAs of one tile (A: kRows x K, B: N x K, both canonical) into
// TMEM and wait.  Thread 0 issues; all threads wait.  Returns false on timeout.
__device__ __forceinline__ bool umma_tile(const unsigned char *sA, const unsigned char *sB, int K, int N,
                                          uint32_t taddr, uint64_t *mbar, int *err) {
    // generic-proxy smem writes -> visible to the tensor-core (async) proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
        const uint32_t idesc = umma_idesc(N);
        for (int ks = 0; ks < K / 16; ++ks) {
            // K slice ks = chunks 2ks, 2ks+1
            const uint64_t da = umma_desc(a0 + (uint32_t)(2 * ks) * (kRows * 16), kRows * 16, 128);
            const uint64_t db = umma_desc(b0 + (uint32_t)(2 * ks) * (N * 16), N * 16, 128);
            umma_f16(taddr, da, db, idesc, ks > 0 ? 1u : 0u);
        }
        umma_commit(mbar);
    }
    const bool ok = mbar_wait(mbar, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
    return ok;
}

// CTA prologue / epilogue: mbarrier + TMEM (warp 0 allocates `ncols`).
struct TileCtx {
    uint64_t mbar;
    uint32_t taddr;
};

__device__ __forceinline__ void tile_begin(TileCtx *c, int ncols) {
    if (threadIdx.x == 0) mbar_init(&c->mbar, 1);
    if (threadIdx.x < 32) tmem_alloc(&c->taddr, ncols);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tile_end(TileCtx *c, int ncols, bool ok) {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (!ok) {
        // the MMAs may still be in flight: one more bounded wait before freeing
        mbar_wait(&c->mbar, 0);
    }
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tmem_dealloc(c->taddr, ncols);
    }
}

__device__ __forceinline__ float silu_f(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu_f(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// ---------------------------------------------------------------------------
// Kernels (128 threads = 4 warps; warp w owns TMEM lanes / rows 32w..32w+31)
// ---------------------------------------------------------------------------

// Records -> standardised BF16 inputs X [n x 16] and FP32 targets.
struct Norm {
    float mu[kIn], isig[kIn];
    float out_mu, out_isig;
};
__global__ void mlp_prepare_kernel(const float *rec, int stride, long long n, const Norm nm, bf16 *X,
                                   float *T) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *r = rec + i * stride;
#pragma unroll
    for (int c = 0; c < kInPad; ++c)
        X[i * kInPad + c] = __float2bfloat16_rn(c < kIn ? (r[c] - nm.mu[c]) * nm.isig[c] : 0.0f);
    T[i] = (r[kIn] - nm.out_mu) * nm.out_isig;
}

// Z = Hin W^T + b, Hout = SiLU(Z): one 128-row tile per CTA.
template <int K>
__global__ void __launch_bounds__(128) mlp_forward_kernel(const bf16 *Hin, const bf16 *W,
                                                          const float *b, float *Z, bf16 *Hout,
                                                          long long n, int *err) {
    __shared__ __align__(128) unsigned char sA[kRows * K * 2];
    __shared__ __align__(128) unsigned char sB[kH * K * 2];
    __shared__ TileCtx tc;
    const long long r0 = (long long)blockIdx.x * kRows;
    for (int idx = threadIdx.x; idx < kRows * K; idx += blockDim.x) {
        const int row = idx / K, k = idx % K;
        const long long g = r0 + row;
        const bf16 v = g < n ? Hin[g * K + k] : __float2bfloat16_rn(0.0f);
        *reinterpret_cast<bf16 *>(sA + kmaj_off(row, k, kRows)) = v;
    }
    for (int idx = threadIdx.x; idx < kH * K; idx += blockDim.x) {
        const int row = idx / K, k = idx % K;
        *reinterpret_cast<bf16 *>(sB + kmaj_off(row, k, kH)) = W[row * K + k];
    }
    tile_begin(&tc, kH);
    const bool ok = umma_tile(sA, sB, K, kH, tc.taddr, &tc.mbar, err);
    if (ok) {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const long long g = r0 + 32 * w + lane;
        for (int half = 0; half < 2; ++half) {
            float v[32];
            tmem_ld32(tc.taddr + ((uint32_t)(32 * w) << 16) + 32 * half, v);
            if (g < n) {
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    const int col = 32 * half + c;
                    const float z = v[c] + b[col];
                    Z[g * kH + col] = z;
                    Hout[g * kH + col] = __float2bfloat16_rn(silu_f(z));
                }
            }
        }
    }
    tile_end(&tc, kH, ok);
}

// Output layer, loss and its gradient (CUDA cores): y = H3 w4 + b4 with w4
// rounded to BF16 as in inference (targets standardised), loss = mean (y -
// T)^2, dZ3 = (2 (y - T) / n) w4 * SiLU'(Z3) stored as BF16 for the
// tensor-core backward; dw4, db4 accumulated in FP32.  loss receives
// loss_scale * the batch loss.
__global__ void mlp_output_kernel(const bf16 *H3, const float *Z3, const float *P, const float *T,
                                  long long n, bf16 *dZ3, float *G, float *loss, float loss_scale) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    __shared__ float s_w4[kH];
    __shared__ float s_dw[kH];
    __shared__ float s_db, s_loss;
    for (int c = threadIdx.x; c < kH; c += blockDim.x) {
        s_dw[c] = 0.0f;
        s_w4[c] = __bfloat162float(__float2bfloat16_rn(P[kOffW4 + c]));
    }
    if (threadIdx.x == 0) s_db = s_loss = 0.0f;
    __syncthreads();
    if (i < n) {
        float y = P[kOffB4];
        for (int c = 0; c < kH; ++c) y += __bfloat162float(H3[i * kH + c]) * s_w4[c];
        const float d = y - T[i];
        const float gy = 2.0f * d / (float)n;
        atomicAdd(&s_loss, d * d / (float)n);
        atomicAdd(&s_db, gy);
        for (int c = 0; c < kH; ++c) {
            atomicAdd(&s_dw[c], gy * __bfloat162float(H3[i * kH + c]));
            dZ3[i * kH + c] = __float2bfloat16_rn(gy * s_w4[c] * dsilu_f(Z3[i * kH + c]));
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < kH; c += blockDim.x) atomicAdd(&G[kOffW4 + c], s_dw[c]);
    if (threadIdx.x == 0) {
        atomicAdd(&G[kOffB4], s_db);
        if (loss) atomicAdd(loss, s_loss * loss_scale);
    }
}

// Prediction head of the training forward: de-standardised y.
__global__ void mlp_head_kernel(const bf16 *H3, const float *P, long long n, float out_mu,
                                float out_sigma, float *y_out) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float y = P[kOffB4];
    for (int c = 0; c < kH; ++c)
        y += __bfloat162float(H3[i * kH + c]) * __bfloat162float(__float2bfloat16_rn(P[kOffW4 + c]));
    y_out[i] = y * out_sigma + out_mu;
}

// Batch gather: rows perm[0..n) of the prepared inputs and targets.
__global__ void mlp_gather_kernel(const bf16 *X, const float *T, const int *perm, long long n,
                                  bf16 *Xb, float *Tb) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long r = perm[i];
    const uint4 *src = reinterpret_cast<const uint4 *>(X + r * kInPad);
    uint4 *dst = reinterpret_cast<uint4 *>(Xb + i * kInPad);
    dst[0] = src[0];
    dst[1] = src[1];
    Tb[i] = T[r];
}

// Warp-level inference of the integration kernel on raw feature records.
__global__ void __launch_bounds__(hhg::kBlockThreads) mlp_infer_kernel(const hhg::MlpPacked *net,
                                                                       const float *rec, int stride,
                                                                       long long n, float *out) {
    extern __shared__ __align__(16) unsigned char dyn[];
    bf16 *stage = reinterpret_cast<bf16 *>(dyn);
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long i = (blockIdx.x * (long long)hhg::kWarpsPerBlock + wib) * 32 + lane;
    float f[kIn];
#pragma unroll
    for (int c = 0; c < kIn; ++c) f[c] = i < n ? rec[i * stride + c] : 0.0f;
    const float T = hhg::mlp_warp_infer(net, f, stage + wib * hhg::kMlpWarpStage);
    if (i < n) out[i] = T;
}

// dH = dZ W (W stored [64][K] as W^T [K][64] for this GEMM), then
// dZprev = dH * SiLU'(Zprev) as BF16 (the first layer has no predecessor).
template <int K>
__global__ void __launch_bounds__(128) mlp_backward_data_kernel(const bf16 *dZ, const bf16 *WT,
                                                                const float *Zprev, bf16 *dZprev,
                                                                long long n, int *err) {
    __shared__ __align__(128) unsigned char sA[kRows * kH * 2];
    __shared__ __align__(128) unsigned char sB[K * kH * 2];
    __shared__ TileCtx tc;
    const long long r0 = (long long)blockIdx.x * kRows;
    for (int idx = threadIdx.x; idx < kRows * kH; idx += blockDim.x) {
        const int row = idx / kH, k = idx % kH;
        const long long g = r0 + row;
        *reinterpret_cast<bf16 *>(sA + kmaj_off(row, k, kRows)) =
            g < n ? dZ[g * kH + k] : __float2bfloat16_rn(0.0f);
    }
    for (int idx = threadIdx.x; idx < K * kH; idx += blockDim.x) {
        const int row = idx / kH, k = idx % kH;
        *reinterpret_cast<bf16 *>(sB + kmaj_off(row, k, K)) = WT[row * kH + k];
    }
    constexpr int cols = K < 32 ? 32 : K;
    tile_begin(&tc, cols);
    const bool ok = umma_tile(sA, sB, kH, K, tc.taddr, &tc.mbar, err);
    if (ok) {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const long long g = r0 + 32 * w + lane;
        for (int half = 0; half < (K + 31) / 32; ++half) {
            float v[32];
            tmem_ld32(tc.taddr + ((uint32_t)(32 * w) << 16) + 32 * half, v);
            if (g < n) {
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    const int col = 32 * half + c;
                    if (col < K) dZprev[g * K + col] = __float2bfloat16_rn(v[c] * dsilu_f(Zprev[g * K + col]));
                }
            }
        }
    }
    tile_end(&tc, cols, ok);
}

// dW [64 x K] += dZ^T Hin over one 64-row chunk: A = dZ^T (64 rows, padded to
// 128 with zeros), B = Hin^T (K rows), K-dimension = batch rows.
template <int K>
__global__ void __launch_bounds__(128) mlp_backward_weight_kernel(const bf16 *dZ, const bf16 *Hin,
                                                                  long long n, float *dW,
                                                                  float *db, int *err) {
    __shared__ __align__(128) unsigned char sA[kRows * kChunk * 2];
    __shared__ __align__(128) unsigned char sB[K * kChunk * 2];
    __shared__ TileCtx tc;
    const long long c0 = (long long)blockIdx.x * kChunk;
    for (int idx = threadIdx.x; idx < kRows * kChunk; idx += blockDim.x) {
        const int row = idx / kChunk, kk = idx % kChunk;  // row = output unit, kk = batch row
        const long long g = c0 + kk;
        const bf16 v = (row < kH && g < n) ? dZ[g * kH + row] : __float2bfloat16_rn(0.0f);
        *reinterpret_cast<bf16 *>(sA + kmaj_off(row, kk, kRows)) = v;
    }
    for (int idx = threadIdx.x; idx < K * kChunk; idx += blockDim.x) {
        const int row = idx / kChunk, kk = idx % kChunk;  // row = input unit
        const long long g = c0 + kk;
        *reinterpret_cast<bf16 *>(sB + kmaj_off(row, kk, K)) =
            g < n ? Hin[g * K + row] : __float2bfloat16_rn(0.0f);
    }
    // bias gradient: column sums of dZ over the chunk
    if (threadIdx.x < kH) {
        float acc = 0.0f;
        for (int kk = 0; kk < kChunk; ++kk) {
            const long long g = c0 + kk;
            if (g < n) acc += __bfloat162float(dZ[g * kH + threadIdx.x]);
        }
        atomicAdd(&db[threadIdx.x], acc);
    }
    constexpr int cols = K < 32 ? 32 : K;
    tile_begin(&tc, cols);
    const bool ok = umma_tile(sA, sB, kChunk, K, tc.taddr, &tc.mbar, err);
    if (ok) {
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int row = 32 * w + lane;
        for (int half = 0; half < (K + 31) / 32; ++half) {
            float v[32];
            tmem_ld32(tc.taddr + ((uint32_t)(32 * w) << 16) + 32 * half, v);
            if (row < kH) {
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    const int col = 32 * half + c;
                    if (col < K) atomicAdd(&dW[row * K + col], v[c]);
                }
            }
        }
    }
    tile_end(&tc, cols, ok);
}

// Adam on the FP32 master parameters, then the BF16 copies.
__global__ void adam_kernel(float *p, const float *g, float *m, float *v, int n, float lr, float b1,
                            float b2, float eps, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    m[i] = b1 * m[i] + (1.0f - b1) * gi;
    v[i] = b2 * v[i] + (1.0f - b2) * gi * gi;
    p[i] -= lr * (m[i] / bc1) / (sqrtf(v[i] / bc2) + eps);
}

// Master weights -> BF16 W [64][K] and W^T [K][64] of the three hidden
// layers (one thread per element of all three).
__global__ void to_bf16_kernel(const float *P, bf16 *W1, bf16 *W2, bf16 *W2T, bf16 *W3, bf16 *W3T) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kH * kInPad) {
        W1[i] = __float2bfloat16_rn(P[kOffW1 + i]);
        return;
    }
    i -= kH * kInPad;
    if (i < kH * kH) {
        const bf16 v = __float2bfloat16_rn(P[kOffW2 + i]);
        W2[i] = v;
        W2T[(i % kH) * kH + i / kH] = v;
        return;
    }
    i -= kH * kH;
    if (i < kH * kH) {
        const bf16 v = __float2bfloat16_rn(P[kOffW3 + i]);
        W3[i] = v;
        W3T[(i % kH) * kH + i / kH] = v;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
namespace hhg {
// hhg_mlp (ABI) -> the packed BF16 device network of the integration kernel.
void pack_mlp(const hhg_mlp &net, MlpPacked *out) {
    std::memset(out, 0, sizeof *out);
    const float *p = net.params;
    for (int o = 0; o < kH; ++o) {
        for (int i = 0; i < kIn; ++i) out->w1[o][i] = __float2bfloat16_rn(p[aW1 + o * kIn + i]);
        for (int i = kIn; i < kInPad; ++i) out->w1[o][i] = __float2bfloat16_rn(0.0f);
        for (int i = 0; i < kH; ++i) {
            out->w2[o][i] = __float2bfloat16_rn(p[aW2 + o * kH + i]);
            out->w3[o][i] = __float2bfloat16_rn(p[aW3 + o * kH + i]);
        }
        out->b1[o] = p[aB1 + o];
        out->b2[o] = p[aB2 + o];
        out->b3[o] = p[aB3 + o];
    }
    for (int r = 0; r < kMlpOutPad; ++r)
        for (int i = 0; i < kH; ++i) out->w4[r][i] = __float2bfloat16_rn(r == 0 ? p[aW4 + i] : 0.0f);
    out->b4 = p[aB4];
    out->out_mu = net.out_mu;
    out->out_sigma = net.out_sigma;
    out->level_margin = net.level_margin;
    for (int c = 0; c < kIn; ++c) {
        out->in_mu[c] = net.in_mu[c];
        out->in_isig[c] = net.in_isig[c];
    }
}
}  // namespace hhg

namespace {
void abi_to_master(const float *a, float *m) {
    std::memset(m, 0, sizeof(float) * kNMaster);
    for (int o = 0; o < kH; ++o)
        for (int i = 0; i < kIn; ++i) m[kOffW1 + o * kInPad + i] = a[aW1 + o * kIn + i];
    std::memcpy(m + kOffB1, a + aB1, sizeof(float) * kH);
    std::memcpy(m + kOffW2, a + aW2, sizeof(float) * (kH * kH + kH + kH * kH + kH + kH + 1));
}

void master_to_abi(const float *m, float *a) {
    for (int o = 0; o < kH; ++o)
        for (int i = 0; i < kIn; ++i) a[aW1 + o * kIn + i] = m[kOffW1 + o * kInPad + i];
    std::memcpy(a + aB1, m + kOffB1, sizeof(float) * kH);
    std::memcpy(a + aW2, m + kOffW2, sizeof(float) * (kH * kH + kH + kH * kH + kH + kH + 1));
}

Norm make_norm(const hhg_mlp &net) {
    Norm nm{};
    for (int c = 0; c < kIn; ++c) {
        nm.mu[c] = net.in_mu[c];
        nm.isig[c] = net.in_isig[c];
    }
    nm.out_mu = net.out_mu;
    nm.out_isig = 1.0f / net.out_sigma;
    return nm;
}

uint64_t splitmix64(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Device buffers of one training / evaluation session (freed on scope exit).
struct Session {
    std::vector<void *> bufs;
    cudaError_t err = cudaSuccess;
    template <typename T>
    T *alloc(size_t n) {
        void *p = nullptr;
        if (err == cudaSuccess) err = cudaMalloc(&p, n * sizeof(T) + 16);
        if (err != cudaSuccess) return nullptr;
        bufs.push_back(p);
        return static_cast<T *>(p);
    }
    ~Session() {
        for (void *p : bufs) cudaFree(p);
    }
};

// Forward + (optionally) backward buffers for up to `rows` rows.
struct Net {
    float *P = nullptr, *G = nullptr, *m = nullptr, *v = nullptr;
    bf16 *W1 = nullptr, *W2 = nullptr, *W2T = nullptr, *W3 = nullptr, *W3T = nullptr;
    float *Z1 = nullptr, *Z2 = nullptr, *Z3 = nullptr, *Tb = nullptr;
    bf16 *Xb = nullptr, *H1 = nullptr, *H2 = nullptr, *H3 = nullptr;
    bf16 *dZ1 = nullptr, *dZ2 = nullptr, *dZ3 = nullptr;
    int *err = nullptr;
    long long rows = 0;
    bool init(Session &S, long long r, bool optimiser) {
        rows = (r + kRows - 1) / kRows * kRows;
        P = S.alloc<float>(kNMaster);
        G = S.alloc<float>(kNMaster);
        if (optimiser) {
            m = S.alloc<float>(kNMaster);
            v = S.alloc<float>(kNMaster);
        }
        W1 = S.alloc<bf16>(kH * kInPad);
        W2 = S.alloc<bf16>(kH * kH);
        W2T = S.alloc<bf16>(kH * kH);
        W3 = S.alloc<bf16>(kH * kH);
        W3T = S.alloc<bf16>(kH * kH);
        Xb = S.alloc<bf16>(rows * kInPad);
        Tb = S.alloc<float>(rows);
        Z1 = S.alloc<float>(rows * kH);
        Z2 = S.alloc<float>(rows * kH);
        Z3 = S.alloc<float>(rows * kH);
        H1 = S.alloc<bf16>(rows * kH);
        H2 = S.alloc<bf16>(rows * kH);
        H3 = S.alloc<bf16>(rows * kH);
        dZ1 = S.alloc<bf16>(rows * kH);
        dZ2 = S.alloc<bf16>(rows * kH);
        dZ3 = S.alloc<bf16>(rows * kH);
        err = S.alloc<int>(1);
        return S.err == cudaSuccess;
    }
    void weights_bf16(cudaStream_t s) const {
        const int n = kH * kInPad + 2 * kH * kH;
        to_bf16_kernel<<<(n + 255) / 256, 256, 0, s>>>(P, W1, W2, W2T, W3, W3T);
    }
    void forward(long long n, cudaStream_t s) const {
        const unsigned tiles = (unsigned)((n + kRows - 1) / kRows);
        mlp_forward_kernel<kInPad><<<tiles, 128, 0, s>>>(Xb, W1, P + kOffB1, Z1, H1, n, err);
        mlp_forward_kernel<kH><<<tiles, 128, 0, s>>>(H1, W2, P + kOffB2, Z2, H2, n, err);
        mlp_forward_kernel<kH><<<tiles, 128, 0, s>>>(H2, W3, P + kOffB3, Z3, H3, n, err);
    }
    void backward(long long n, float *loss, float loss_scale, cudaStream_t s) const {
        const unsigned tiles = (unsigned)((n + kRows - 1) / kRows);
        const unsigned chunks = (unsigned)((n + kChunk - 1) / kChunk);
        cudaMemsetAsync(G, 0, sizeof(float) * kNMaster, s);
        mlp_output_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(H3, Z3, P, Tb, n, dZ3, G, loss,
                                                                      loss_scale);
        mlp_backward_weight_kernel<kH><<<chunks, 128, 0, s>>>(dZ3, H2, n, G + kOffW3, G + kOffB3, err);
        mlp_backward_data_kernel<kH><<<tiles, 128, 0, s>>>(dZ3, W3T, Z2, dZ2, n, err);
        mlp_backward_weight_kernel<kH><<<chunks, 128, 0, s>>>(dZ2, H1, n, G + kOffW2, G + kOffB2, err);
        mlp_backward_data_kernel<kH><<<tiles, 128, 0, s>>>(dZ2, W2T, Z1, dZ1, n, err);
        mlp_backward_weight_kernel<kInPad><<<chunks, 128, 0, s>>>(dZ1, Xb, n, G + kOffW1, G + kOffB1, err);
    }
};

hhg_status fail(hhg_status st, const char *what, cudaError_t e, std::string *msg) {
    if (msg) *msg = std::string(what) + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
    return st;
}

bool check_net(const hhg_mlp *net) {
    if (!net || !(net->out_sigma > 0.0f) || !std::isfinite(net->out_sigma)) return false;
    for (int c = 0; c < kIn; ++c)
        if (!std::isfinite(net->in_mu[c]) || !std::isfinite(net->in_isig[c])) return false;
    return true;
}
}  // namespace

// Internal entry points used by the C ABI (hhg_gpu.cu owns the context).
namespace hhg {
hhg_status mlp_train_impl(cudaStream_t s, const float *records, int64_t n, const hhg_train_opts &o,
                          hhg_mlp *net, float *epoch_loss, double *train_ms, std::string *msg) {
    if (!records || !net || n < kRows) return fail(HHG_BAD_CONFIG, "need at least 128 records and a network", cudaSuccess, msg);
    if (!check_net(net)) return fail(HHG_BAD_CONFIG, "network standardisation not set (hhg_mlp_init)", cudaSuccess, msg);
    if (o.epochs < 1 || o.batch < kRows || o.batch % kRows != 0 || !(o.lr > 0.0f))
        return fail(HHG_BAD_CONFIG, "epochs >= 1, batch a multiple of 128, lr > 0", cudaSuccess, msg);
    if (n > (int64_t)1 << 30) return fail(HHG_BAD_CONFIG, "at most 2^30 records", cudaSuccess, msg);
    const long long B = std::min<long long>(o.batch, n / kRows * kRows);
    const long long nb = n / B;
    Session S;
    Net W;
    if (!W.init(S, B, true)) return fail(HHG_CUDA_ERROR, "alloc training buffers", S.err, msg);
    float *d_rec = S.alloc<float>((size_t)n * HHG_HIST_FIELDS);
    bf16 *X = S.alloc<bf16>((size_t)n * kInPad);
    float *T = S.alloc<float>(n);
    int *perm = S.alloc<int>(n);
    float *d_loss = S.alloc<float>(o.epochs);
    if (S.err != cudaSuccess) return fail(HHG_CUDA_ERROR, "alloc training data", S.err, msg);
    std::vector<float> master(kNMaster);
    abi_to_master(net->params, master.data());
    cudaError_t e;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventRecord(ev0, s);
    cudaMemcpyAsync(d_rec, records, sizeof(float) * n * HHG_HIST_FIELDS, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(W.P, master.data(), sizeof(float) * kNMaster, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(W.m, 0, sizeof(float) * kNMaster, s);
    cudaMemsetAsync(W.v, 0, sizeof(float) * kNMaster, s);
    cudaMemsetAsync(W.err, 0, sizeof(int), s);
    cudaMemsetAsync(d_loss, 0, sizeof(float) * o.epochs, s);
    mlp_prepare_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_rec, HHG_HIST_FIELDS, n, make_norm(*net), X, T);
    W.weights_bf16(s);
    std::vector<int> hp(n);
    for (long long i = 0; i < n; ++i) hp[i] = (int)i;
    uint64_t rng = o.seed;
    const double total = (double)o.epochs * nb;
    long long step = 0;
    for (int ep = 0; ep < o.epochs; ++ep) {
        for (long long i = n - 1; i > 0; --i) std::swap(hp[i], hp[splitmix64(rng) % (uint64_t)(i + 1)]);
        if ((e = cudaMemcpyAsync(perm, hp.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return fail(HHG_CUDA_ERROR, "upload batch order", e, msg);
        for (long long b = 0; b < nb; ++b, ++step) {
            mlp_gather_kernel<<<(unsigned)((B + 255) / 256), 256, 0, s>>>(X, T, perm + b * B, B, W.Xb, W.Tb);
            W.forward(B, s);
            W.backward(B, d_loss + ep, 1.0f / (float)nb, s);
            const double t = (double)(step + 1);
            const double lr = o.lr_final + 0.5 * (o.lr - o.lr_final) * (1.0 + std::cos(M_PI * step / total));
            adam_kernel<<<(kNMaster + 255) / 256, 256, 0, s>>>(
                W.P, W.G, W.m, W.v, kNMaster, (float)lr, o.beta1, o.beta2, o.eps,
                (float)(1.0 - std::pow((double)o.beta1, t)), (float)(1.0 - std::pow((double)o.beta2, t)));
            W.weights_bf16(s);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(HHG_CUDA_ERROR, "training launch", e, msg);
    }
    cudaEventRecord(ev1, s);
    int h_err = 0;
    std::vector<float> h_loss(o.epochs);
    cudaMemcpyAsync(master.data(), W.P, sizeof(float) * kNMaster, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&h_err, W.err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h_loss.data(), d_loss, sizeof(float) * o.epochs, cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(HHG_CUDA_ERROR, "training", e, msg);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (h_err) return fail(HHG_CUDA_ERROR, "tensor-core completion wait timed out", cudaSuccess, msg);
    for (float v : master)
        if (!std::isfinite(v)) return fail(HHG_NONFINITE, "training diverged (non-finite weights)", cudaSuccess, msg);
    master_to_abi(master.data(), net->params);
    if (epoch_loss) std::memcpy(epoch_loss, h_loss.data(), sizeof(float) * o.epochs);
    if (train_ms) *train_ms = ms;
    return HHG_OK;
}

hhg_status mlp_gradients_impl(cudaStream_t s, const float *records, int64_t n, const hhg_mlp *net,
                              float *grad_out, float *loss_out, std::string *msg) {
    if (!records || !net || !grad_out || n < 1 || n > (int64_t)1 << 20)
        return fail(HHG_BAD_CONFIG, "1 <= n_records <= 2^20, network and output required", cudaSuccess, msg);
    if (!check_net(net)) return fail(HHG_BAD_CONFIG, "network standardisation not set", cudaSuccess, msg);
    Session S;
    Net W;
    if (!W.init(S, n, false)) return fail(HHG_CUDA_ERROR, "alloc buffers", S.err, msg);
    float *d_rec = S.alloc<float>((size_t)n * HHG_HIST_FIELDS);
    float *d_loss = S.alloc<float>(1);
    if (S.err != cudaSuccess) return fail(HHG_CUDA_ERROR, "alloc records", S.err, msg);
    std::vector<float> master(kNMaster);
    abi_to_master(net->params, master.data());
    cudaMemcpyAsync(d_rec, records, sizeof(float) * n * HHG_HIST_FIELDS, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(W.P, master.data(), sizeof(float) * kNMaster, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(W.err, 0, sizeof(int), s);
    cudaMemsetAsync(d_loss, 0, sizeof(float), s);
    mlp_prepare_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_rec, HHG_HIST_FIELDS, n, make_norm(*net), W.Xb, W.Tb);
    W.weights_bf16(s);
    W.forward(n, s);
    W.backward(n, d_loss, 1.0f, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(HHG_CUDA_ERROR, "gradient launch", e, msg);
    int h_err = 0;
    float h_loss = 0.0f;
    cudaMemcpyAsync(master.data(), W.G, sizeof(float) * kNMaster, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&h_err, W.err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&h_loss, d_loss, sizeof(float), cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(HHG_CUDA_ERROR, "gradients", e, msg);
    if (h_err) return fail(HHG_CUDA_ERROR, "tensor-core completion wait timed out", cudaSuccess, msg);
    master_to_abi(master.data(), grad_out);
    if (loss_out) *loss_out = h_loss;
    return HHG_OK;
}

hhg_status mlp_predict_impl(cudaStream_t s, const float *records, int64_t n, const hhg_mlp *net,
                            int path, float *out, std::string *msg) {
    if (!records || !net || !out || n < 1 || n > (int64_t)1 << 24 || (path != 0 && path != 1))
        return fail(HHG_BAD_CONFIG, "1 <= n_records <= 2^24, path 0 or 1", cudaSuccess, msg);
    if (!check_net(net)) return fail(HHG_BAD_CONFIG, "network standardisation not set", cudaSuccess, msg);
    Session S;
    float *d_rec = S.alloc<float>((size_t)n * HHG_HIST_FIELDS);
    float *d_out = S.alloc<float>(n);
    if (S.err != cudaSuccess) return fail(HHG_CUDA_ERROR, "alloc records", S.err, msg);
    cudaMemcpyAsync(d_rec, records, sizeof(float) * n * HHG_HIST_FIELDS, cudaMemcpyHostToDevice, s);
    int h_err = 0;
    Net W;
    if (path == 0) {
        MlpPacked *d_net = S.alloc<MlpPacked>(1);
        if (S.err != cudaSuccess) return fail(HHG_CUDA_ERROR, "alloc network", S.err, msg);
        MlpPacked h;
        pack_mlp(*net, &h);
        cudaMemcpyAsync(d_net, &h, sizeof h, cudaMemcpyHostToDevice, s);
        const long long rows_per_cta = 32LL * kWarpsPerBlock;
        mlp_infer_kernel<<<(unsigned)((n + rows_per_cta - 1) / rows_per_cta), kBlockThreads, mlp_smem_bytes(), s>>>(
            d_net, d_rec, HHG_HIST_FIELDS, n, d_out);
        // the packed copy must outlive the kernel: synchronise before the session frees it
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return fail(HHG_CUDA_ERROR, "inference", e, msg);
    } else {
        if (!W.init(S, n, false)) return fail(HHG_CUDA_ERROR, "alloc buffers", S.err, msg);
        std::vector<float> master(kNMaster);
        abi_to_master(net->params, master.data());
        cudaMemcpyAsync(W.P, master.data(), sizeof(float) * kNMaster, cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(W.err, 0, sizeof(int), s);
        mlp_prepare_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_rec, HHG_HIST_FIELDS, n, make_norm(*net), W.Xb, W.Tb);
        W.weights_bf16(s);
        W.forward(n, s);
        mlp_head_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(W.H3, W.P, n, net->out_mu, net->out_sigma, d_out);
        cudaMemcpyAsync(&h_err, W.err, sizeof(int), cudaMemcpyDeviceToHost, s);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(HHG_CUDA_ERROR, "predict launch", e, msg);
    cudaMemcpyAsync(out, d_out, sizeof(float) * n, cudaMemcpyDeviceToHost, s);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(HHG_CUDA_ERROR, "predict", e, msg);
    if (h_err) return fail(HHG_CUDA_ERROR, "tensor-core completion wait timed out", cudaSuccess, msg);
    return HHG_OK;
}
}  // namespace hhg

extern "C" {

void hhg_default_train_opts(hhg_train_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->epochs = 30;
    o->batch = 4096;
    o->lr = 2e-3f;
    o->beta1 = 0.9f;
    o->beta2 = 0.999f;
    o->eps = 1e-8f;
    o->lr_final = 1e-4f;
    o->seed = 1;
}

hhg_status hhg_mlp_init(uint64_t seed, const float *records, int64_t n, hhg_mlp *net) {
    if (!net) return HHG_BAD_CONFIG;
    std::memset(net, 0, sizeof *net);
    uint64_t s = seed;
    auto uni = [&](float bound) {
        const double u = (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
        return (float)((2.0 * u - 1.0) * bound);
    };
    float *p = net->params;
    const float b_in = 1.0f / std::sqrt((float)kIn), b_h = 1.0f / std::sqrt((float)kH);
    for (int i = 0; i < kH * kIn; ++i) p[aW1 + i] = uni(b_in);
    for (int i = 0; i < kH; ++i) p[aB1 + i] = uni(b_in);
    for (int i = 0; i < kH * kH; ++i) p[aW2 + i] = uni(b_h);
    for (int i = 0; i < kH; ++i) p[aB2 + i] = uni(b_h);
    for (int i = 0; i < kH * kH; ++i) p[aW3 + i] = uni(b_h);
    for (int i = 0; i < kH; ++i) p[aB3 + i] = uni(b_h);
    for (int i = 0; i < kH; ++i) p[aW4 + i] = uni(b_h);
    p[aB4] = 0.0f;
    for (int c = 0; c < kIn; ++c) {
        net->in_mu[c] = 0.0f;
        net->in_isig[c] = 1.0f;
    }
    net->out_mu = 0.0f;
    net->out_sigma = 1.0f;
    net->level_margin = -0.5f;
    if (records && n > 1) {
        double sum[kIn + 1] = {}, sq[kIn + 1] = {};
        for (int64_t r = 0; r < n; ++r)
            for (int c = 0; c <= kIn; ++c) {
                const double v = records[r * HHG_HIST_FIELDS + c];
                sum[c] += v;
                sq[c] += v * v;
            }
        for (int c = 0; c <= kIn; ++c) {
            const double mu = sum[c] / n;
            const double var = std::max(sq[c] / n - mu * mu, 0.0);
            const double sd = std::sqrt(var);
            if (c < kIn) {
                net->in_mu[c] = (float)mu;
                net->in_isig[c] = sd > 1e-12 ? (float)(1.0 / sd) : 1.0f;
            } else {
                net->out_mu = (float)mu;
                net->out_sigma = (float)std::max(sd, 1e-3);
            }
        }
    }
    return HHG_OK;
}

}  // extern "C"
