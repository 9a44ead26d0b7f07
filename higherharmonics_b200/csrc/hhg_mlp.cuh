// hhg_mlp.cuh -- the learned step-size proposer: features, the packed network
// layout shared by training and inference, and the warp-level inference used
// inside the integration kernel.
//
// Network: 4 linear layers 8 -> 64 -> 64 -> 64 -> 1, SiLU after the first
// three, BF16 weights and activations, FP32 accumulation.  Inputs (per
// k-point, at the start of a measurement interval): kx/pi, ky/pi, A(t), E(t) =
// -dA/dt, the Bloch vector S, log2(h_prev / interval); output: the level T =
// log2(interval / h*) of the largest step the embedded RKF78 error would
// accept.  Inputs are standardised with (mu, 1/sigma) fitted on the training
// set; the output is de-standardised with (out_mu, out_sigma).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace hhg {

constexpr int kMlpIn = 8;
constexpr int kMlpInPad = 16;
constexpr int kMlpH = 64;
constexpr int kMlpOutPad = 8;  // the output layer as an n8 tile (row 0 real)

// Packed device network (one contiguous global buffer).
struct MlpPacked {
    __nv_bfloat16 w1[kMlpH][kMlpInPad];   // [out][in], in padded with zeros
    __nv_bfloat16 w2[kMlpH][kMlpH];
    __nv_bfloat16 w3[kMlpH][kMlpH];
    __nv_bfloat16 w4[kMlpOutPad][kMlpH];  // row 0 = output weights, rows 1..7 zero
    float b1[kMlpH], b2[kMlpH], b3[kMlpH];
    float b4;
    float out_mu, out_sigma;
    float level_margin;  // the warp steps at level max ceil(T + level_margin)
    float in_mu[kMlpIn], in_isig[kMlpIn];
};

// E(t) = -dA/dt of the pulse (zero outside the window).
__device__ __forceinline__ double laser_field(const PulseDev &p, double t) {
    if (t <= p.t_begin || t >= p.t_end) return 0.0;
    double sc, cc;
    sincos(t + p.phase, &sc, &cc);
    if (p.kind == PULSE_CONTINUOUS) return -p.amplitude * cc;
    if (p.kind == PULSE_GAUSS) {
        const double x = t - p.gauss_c;
        const double env = exp(-(x * x) / p.gauss_2s2), denv = -2.0 * x / p.gauss_2s2 * env;
        return -p.amplitude * (denv * sc + env * cc);
    }
    if (p.kind == PULSE_SPLINE) {
        double d;
        spline_value(p, t, &d);
        return -p.amplitude * d;
    }
    double se, ce;
    sincos(p.inv_n_cycles * (t - p.t_begin), &se, &ce);
    const double env = 0.5 * (1. - ce), denv = 0.5 * p.inv_n_cycles * se;
    return -p.amplitude * (denv * sc + env * cc);
}

__device__ __forceinline__ void mlp_features(const double *row, double A, double E, const double *S,
                                             double log2_hrel, float *f) {
    const double ipi = 0.31830988618379067154;
    f[0] = float(row[0] * ipi);
    f[1] = float(row[1] * ipi);
    f[2] = float(A);
    f[3] = float(E);
    f[4] = float(S[0]);
    f[5] = float(S[1]);
    f[6] = float(S[2]);
    f[7] = float(log2_hrel);
}

// Warp-level inference reads the packed network from global memory (it is
// 18 KB and shared by every warp, so it stays in L1/L2); only the per-warp
// feature tile needs shared memory: 32 rows of kLdIn bf16 (16 features
// padded to 24 so the A-fragment loads of the eight row groups hit distinct
// banks).  A shared-memory copy per CTA would take ~23 KB from every
// 2-warp CTA's share of L1 for the whole run, while the network is
// consulted on a small fraction of the intervals.
constexpr int kLdIn = 24;

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// SiLU of two pre-activations, returned as the packed BF16 pair the next
// layer's A fragment takes: x sigmoid(x) = h + h tanh(h), h = x / 2, in BF16x2
// arithmetic with the hardware tanh (one MUFU operation per pair instead of an
// exponential and a reciprocal per element).  The training forward pass
// evaluates the same function in FP32 before rounding to BF16.
__device__ __forceinline__ uint32_t silu_bf16x2(float lo, float hi) {
    const __nv_bfloat162 x = __floats2bfloat162_rn(lo, hi);
    const __nv_bfloat162 h = __hmul2(x, __float2bfloat162_rn(0.5f));
    const uint32_t hu = *reinterpret_cast<const uint32_t *>(&h);
    uint32_t tu;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(tu) : "r"(hu));
    const __nv_bfloat162 y = __hfma2(h, *reinterpret_cast<const __nv_bfloat162 *>(&tu), h);
    return *reinterpret_cast<const uint32_t *>(&y);
}

// D = A (16x16 bf16) * B (16x8 bf16) + C, FP32 accumulate (warp-wide).
__device__ __forceinline__ void mma_bf16_16816(float *d, const uint32_t *a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ldg_b32(const __nv_bfloat16 *p) {
    return __ldg(reinterpret_cast<const unsigned int *>(p));
}

// One hidden layer for one 16-row m-tile: acc[nt][4] = A W^T + b over eight
// n8 tiles, SiLU, repacked in place as the next layer's A fragments
// out[kc][4] (the m16n8 accumulators of two adjacent n-tiles form the
// m16n8k16 A operand).  W is [64][LD] bf16 in global memory; lane (g, tig)
// loads its B fragment W[8 nt + g][16 kc + 2 tig] and [... + 8] as 32-bit
// words.
template <int KC, int LD>
__device__ __forceinline__ void mlp_hidden(const uint32_t (&a)[KC][4], const __nv_bfloat16 *w,
                                           const float *b, uint32_t (&out)[4][4], int g, int tig) {
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        acc[nt][0] = acc[nt][2] = __ldg(b + 8 * nt + 2 * tig);
        acc[nt][1] = acc[nt][3] = __ldg(b + 8 * nt + 2 * tig + 1);
    }
#pragma unroll
    for (int kc = 0; kc < KC; ++kc) {
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const __nv_bfloat16 *wr = w + (8 * nt + g) * LD + 16 * kc + 2 * tig;
            mma_bf16_16816(acc[nt], a[kc], ldg_b32(wr), ldg_b32(wr + 8));
        }
    }
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
        const float *c0 = acc[2 * kc], *c1 = acc[2 * kc + 1];
        out[kc][0] = silu_bf16x2(c0[0], c0[1]);
        out[kc][1] = silu_bf16x2(c0[2], c0[3]);
        out[kc][2] = silu_bf16x2(c1[0], c1[1]);
        out[kc][3] = silu_bf16x2(c1[2], c1[3]);
    }
}

// Warp-level inference: every lane passes its 8 raw features and receives the
// predicted level T for its own row.  `stage` is a 32 x kLdIn bf16 scratch
// area of this warp in shared memory.  The two 16-row m-tiles run one after
// the other to keep the register footprint small.
__device__ __forceinline__ float mlp_warp_infer(const MlpPacked *__restrict__ W, const float *feat,
                                                __nv_bfloat16 *stage) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, tig = lane & 3;
    __nv_bfloat16 *my = stage + lane * kLdIn;
#pragma unroll
    for (int c = 0; c < kMlpIn; ++c)
        my[c] = __float2bfloat16_rn((feat[c] - __ldg(W->in_mu + c)) * __ldg(W->in_isig + c));
#pragma unroll
    for (int c = kMlpIn; c < kMlpInPad; ++c) my[c] = __float2bfloat16_rn(0.0f);
    __syncwarp();
    float y_mine = 0.0f;
#pragma unroll 1
    for (int mt = 0; mt < 2; ++mt) {
        uint32_t a1[1][4];
        const __nv_bfloat16 *r0 = stage + (16 * mt + g) * kLdIn + 2 * tig;
        const __nv_bfloat16 *r1 = stage + (16 * mt + g + 8) * kLdIn + 2 * tig;
        a1[0][0] = *reinterpret_cast<const uint32_t *>(r0);
        a1[0][1] = *reinterpret_cast<const uint32_t *>(r1);
        a1[0][2] = *reinterpret_cast<const uint32_t *>(r0 + 8);
        a1[0][3] = *reinterpret_cast<const uint32_t *>(r1 + 8);
        uint32_t h1[4][4], h2[4][4];
        mlp_hidden<1, kMlpInPad>(a1, &W->w1[0][0], W->b1, h1, g, tig);
        mlp_hidden<4, kMlpH>(h1, &W->w2[0][0], W->b2, h2, g, tig);
        mlp_hidden<4, kMlpH>(h2, &W->w3[0][0], W->b3, h1, g, tig);
        float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int kc = 0; kc < 4; ++kc) {
            const __nv_bfloat16 *wr = &W->w4[g][0] + 16 * kc + 2 * tig;
            mma_bf16_16816(o, h1[kc], ldg_b32(wr), ldg_b32(wr + 8));
        }
        // row r of this m-tile, column 0: lane 4 (r mod 8), register 0 (r < 8) or 2
        const int r = lane & 15;
        const float v0 = __shfl_sync(0xffffffffu, o[0], 4 * (r & 7));
        const float v2 = __shfl_sync(0xffffffffu, o[2], 4 * (r & 7));
        if ((lane >> 4) == mt) y_mine = r < 8 ? v0 : v2;
    }
    __syncwarp();
    return (y_mine + __ldg(&W->b4)) * __ldg(&W->out_sigma) + __ldg(&W->out_mu);
}

// The integration kernel's call: not inlined, so the inference's registers
// are those of a function call made on a small fraction of the intervals and
// the stepping loop keeps its own allocation.
static __device__ __noinline__ float mlp_warp_infer_call(const MlpPacked *__restrict__ W,
                                                         const float *feat, __nv_bfloat16 *stage) {
    return mlp_warp_infer(W, feat, stage);
}

// Dynamic shared memory of a CTA of `warps` warps running the inference.
__host__ __device__ constexpr int mlp_stage_bytes(int warps) { return warps * 32 * kLdIn * 2; }

}  // namespace hhg
