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

__device__ __forceinline__ float2 mlp_k_features(const double *row) {
    const double ipi = 0.31830988618379067154;
    return make_float2(float(row[0] * ipi), float(row[1] * ipi));
}

__device__ __forceinline__ void mlp_features(float2 kf, double A, double E, const double *S,
                                             double log2_hrel, float *f) {
    f[0] = kf.x;
    f[1] = kf.y;
    f[2] = float(A);
    f[3] = float(E);
    f[4] = float(S[0]);
    f[5] = float(S[1]);
    f[6] = float(S[2]);
    f[7] = float(log2_hrel);
}

// Warp-level inference reads the packed network from global memory (it is
// 18 KB and shared by every warp, so it stays in L1/L2; a shared-memory copy
// per CTA would take ~23 KB from every 2-warp CTA's share of L1 for the whole
// run, while the network is consulted on a small fraction of the
// intervals).  The warp's activations live in a per-warp shared-memory tile
// of 32 rows x kLdH bf16: the features in columns 0..15 (8 inputs, zero
// padded), each layer's output over its input.  The row stride of 72
// elements (36 words) puts the eight row groups of an A-fragment load on
// distinct banks.
constexpr int kLdH = 72;
constexpr int kMlpWarpStage = 32 * kLdH;  // bf16 elements per warp

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

// A fragment (16 x 16 bf16, row-major) of m-tile mt, k-chunk kc from the
// warp's activation tile H: lane (g, tig) holds rows g and g + 8, columns
// 16 kc + 2 tig (+1) and the same + 8.
__device__ __forceinline__ void mlp_load_a(const __nv_bfloat16 *H, int mt, int kc, int g, int tig,
                                           uint32_t (&a)[4]) {
    const __nv_bfloat16 *r0 = H + (16 * mt + g) * kLdH + 16 * kc + 2 * tig;
    const __nv_bfloat16 *r1 = r0 + 8 * kLdH;
    a[0] = *reinterpret_cast<const uint32_t *>(r0);
    a[1] = *reinterpret_cast<const uint32_t *>(r1);
    a[2] = *reinterpret_cast<const uint32_t *>(r0 + 8);
    a[3] = *reinterpret_cast<const uint32_t *>(r1 + 8);
}

// One hidden layer over both 16-row m-tiles, in place on H: the layer's
// input (KC k-chunks) is read into registers first, then every n8 tile of
// the 64 outputs is accumulated from bias + A W^T (FP32), passed through
// SiLU and stored back as bf16 pairs (C-fragment rows g and g + 8, columns
// 8 nt + 2 tig, +1; exactly the next layer's A-fragment positions).  The
// n-tile loop is not unrolled, so at most 2 x 4 accumulators and one B
// fragment are live beside the input: the inference runs inside the
// stepping loop without displacing its registers.  W is [64][LD] bf16 in
// global memory; lane (g, tig) loads W[8 nt + g][16 kc + 2 tig] and
// [... + 8] as 32-bit words.
template <int KC, int LD>
__device__ __forceinline__ void mlp_layer(__nv_bfloat16 *H, const __nv_bfloat16 *w, const float *b,
                                          int g, int tig) {
    uint32_t a[2][KC][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int kc = 0; kc < KC; ++kc) mlp_load_a(H, mt, kc, g, tig, a[mt][kc]);
    __syncwarp();
#pragma unroll 1
    for (int nt = 0; nt < 8; ++nt) {
        const float b0 = __ldg(b + 8 * nt + 2 * tig), b1 = __ldg(b + 8 * nt + 2 * tig + 1);
        float acc[2][4] = {{b0, b1, b0, b1}, {b0, b1, b0, b1}};
#pragma unroll
        for (int kc = 0; kc < KC; ++kc) {
            const __nv_bfloat16 *wr = w + (8 * nt + g) * LD + 16 * kc + 2 * tig;
            const uint32_t w0 = ldg_b32(wr), w1 = ldg_b32(wr + 8);
            mma_bf16_16816(acc[0], a[0][kc], w0, w1);
            mma_bf16_16816(acc[1], a[1][kc], w0, w1);
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            __nv_bfloat16 *o = H + (16 * mt + g) * kLdH + 8 * nt + 2 * tig;
            *reinterpret_cast<uint32_t *>(o) = silu_bf16x2(acc[mt][0], acc[mt][1]);
            *reinterpret_cast<uint32_t *>(o + 8 * kLdH) = silu_bf16x2(acc[mt][2], acc[mt][3]);
        }
    }
    __syncwarp();
}

// Warp-level inference: every lane passes its 8 raw features and receives the
// predicted level T for its own row.  H is this warp's kMlpWarpStage-element
// activation tile in shared memory.
__device__ __forceinline__ float mlp_warp_infer(const MlpPacked *__restrict__ W, const float *feat,
                                                __nv_bfloat16 *H) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, tig = lane & 3;
    __nv_bfloat16 *my = H + lane * kLdH;
#pragma unroll
    for (int c = 0; c < kMlpIn; c += 2)
        *reinterpret_cast<uint32_t *>(my + c) =
            pack_bf16x2((feat[c] - __ldg(W->in_mu + c)) * __ldg(W->in_isig + c),
                        (feat[c + 1] - __ldg(W->in_mu + c + 1)) * __ldg(W->in_isig + c + 1));
#pragma unroll
    for (int c = kMlpIn; c < kMlpInPad; c += 2) *reinterpret_cast<uint32_t *>(my + c) = 0u;
    __syncwarp();
    mlp_layer<1, kMlpInPad>(H, &W->w1[0][0], W->b1, g, tig);
    mlp_layer<4, kMlpH>(H, &W->w2[0][0], W->b2, g, tig);
    mlp_layer<4, kMlpH>(H, &W->w3[0][0], W->b3, g, tig);
    // output layer: one n8 tile (row 0 of w4 real), both m-tiles
    float o[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
        const __nv_bfloat16 *wr = &W->w4[g][0] + 16 * kc + 2 * tig;
        const uint32_t w0 = ldg_b32(wr), w1 = ldg_b32(wr + 8);
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            uint32_t a[4];
            mlp_load_a(H, mt, kc, g, tig, a);
            mma_bf16_16816(o[mt], a, w0, w1);
        }
    }
    __syncwarp();  // H may be rewritten by the next consult
    // row r of m-tile mt, column 0: lane 4 (r mod 8), register 0 (r < 8) or 2
    const int r = lane & 15, src = 4 * (r & 7);
    const float v00 = __shfl_sync(0xffffffffu, o[0][0], src), v02 = __shfl_sync(0xffffffffu, o[0][2], src);
    const float v10 = __shfl_sync(0xffffffffu, o[1][0], src), v12 = __shfl_sync(0xffffffffu, o[1][2], src);
    const float y = (lane < 16) ? (r < 8 ? v00 : v02) : (r < 8 ? v10 : v12);
    return (y + __ldg(&W->b4)) * __ldg(&W->out_sigma) + __ldg(&W->out_mu);
}

// Dynamic shared memory of a CTA of `warps` warps running the inference.
__host__ __device__ constexpr int mlp_stage_bytes(int warps) { return warps * kMlpWarpStage * 2; }


}  // namespace hhg
