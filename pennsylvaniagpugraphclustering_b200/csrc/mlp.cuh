// mlp.cuh -- the learned move filter's network: 8 features -> 32 -> 32 -> 1
// logit, BF16 weights, FP32 accumulation.  The reference has no learned
// filter; this is a project addition that only decides which vertices a sweep
// evaluates (gains stay exact).
//
// Inference runs on the tensor cores, one warp per 32 vertices as two 16-row
// tiles: layer 1 is one m16n8k16 BF16 MMA per 8 hidden units (the 8 features
// padded to K = 16 with zeros), its FP32 accumulators (+ bias, ReLU) are
// rounded to BF16 and reused in registers as the A operand of layer 2 (the
// m16n8 accumulator layout of two adjacent n-blocks is the m16k16 A layout),
// layer 2 is 2 x 4 MMAs, and layer 3 (32 -> 1) is a quad reduction in FP32.
//
// Arithmetic (shared with the trainer and the CPU oracle): inputs, W1, W2 and
// the layer-1 activations are rounded to BF16 (nearest even); layer-2
// activations stay FP32 and meet BF16-rounded W3; biases are FP32.
#pragma once
#include <cuda_bf16.h>
#include "common.cuh"

namespace pggc {

constexpr int MLP_IN = 8, MLP_H = 32;
constexpr int MLP_O_W1 = 0, MLP_O_B1 = 256, MLP_O_W2 = 288, MLP_O_B2 = 1312, MLP_O_W3 = 1344, MLP_O_B3 = 1376;
constexpr int MLP_PARAMS = 1377;

// BF16 copy of the network in the layout the fragments are loaded from
struct MlpDev {
    __nv_bfloat16 w1[MLP_H * MLP_IN];  // [out][in]
    __nv_bfloat16 w2[MLP_H * MLP_H];   // [out][in]
    float w3[MLP_H];                   // BF16-rounded, stored as FP32
    float b1[MLP_H], b2[MLP_H];
    float b3;
};

__device__ __forceinline__ u32 pack_bf16x2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<u32*>(&v);
}
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ void mma_bf16_16816(float (&c)[4], const u32 (&a)[4], u32 b0, u32 b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Per-lane register copy of the network (g = lane / 4, t = lane % 4).
struct MlpRegs {
    u32 w1[4];           // n-block j: W1[8j+g][2t..2t+1]
    u32 w2[4][2][2];     // n-block j, k-chunk kk: W2[8j+g][16kk+2t..], W2[8j+g][16kk+8+2t..]
    float b1[4][2], b2[4][2], w3[4][2];
    float b3;
};

__device__ __forceinline__ void mlp_load(const MlpDev* m, MlpRegs& r) {
    const int l = threadIdx.x & 31, g = l >> 2, t = l & 3;
    const u32* w1 = reinterpret_cast<const u32*>(m->w1);
    const u32* w2 = reinterpret_cast<const u32*>(m->w2);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int row = 8 * j + g;
        r.w1[j] = w1[(row * MLP_IN + 2 * t) >> 1];
#pragma unroll
        for (int kk = 0; kk < 2; kk++) {
            r.w2[j][kk][0] = w2[(row * MLP_H + 16 * kk + 2 * t) >> 1];
            r.w2[j][kk][1] = w2[(row * MLP_H + 16 * kk + 8 + 2 * t) >> 1];
        }
        const int c = 8 * j + 2 * t;
        r.b1[j][0] = m->b1[c];
        r.b1[j][1] = m->b1[c + 1];
        r.b2[j][0] = m->b2[c];
        r.b2[j][1] = m->b2[c + 1];
        r.w3[j][0] = m->w3[c];
        r.w3[j][1] = m->w3[c + 1];
    }
    r.b3 = m->b3;
}

// Logits of one 16-row tile.  xs: FP32 features, row stride `xs_stride`
// floats (row r at xs + r * xs_stride).  Must be called by all 32 lanes; lane
// (g, t) returns the logits of rows g (lg0) and g + 8 (lg1), identical across t.
__device__ __forceinline__ void mlp_tile(const MlpRegs& r, const float* xs, int xs_stride, float& lg0, float& lg1) {
    const int l = threadIdx.x & 31, g = l >> 2, t = l & 3;
    u32 a[4];
    a[0] = pack_bf16x2(xs[g * xs_stride + 2 * t], xs[g * xs_stride + 2 * t + 1]);
    a[1] = pack_bf16x2(xs[(g + 8) * xs_stride + 2 * t], xs[(g + 8) * xs_stride + 2 * t + 1]);
    a[2] = 0u;
    a[3] = 0u;
    float h1[4][4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        h1[j][0] = h1[j][1] = h1[j][2] = h1[j][3] = 0.f;
        mma_bf16_16816(h1[j], a, r.w1[j], 0u);
        h1[j][0] = fmaxf(h1[j][0] + r.b1[j][0], 0.f);
        h1[j][1] = fmaxf(h1[j][1] + r.b1[j][1], 0.f);
        h1[j][2] = fmaxf(h1[j][2] + r.b1[j][0], 0.f);
        h1[j][3] = fmaxf(h1[j][3] + r.b1[j][1], 0.f);
    }
    u32 a2[2][4];
#pragma unroll
    for (int kk = 0; kk < 2; kk++) {
        a2[kk][0] = pack_bf16x2(h1[2 * kk][0], h1[2 * kk][1]);
        a2[kk][1] = pack_bf16x2(h1[2 * kk][2], h1[2 * kk][3]);
        a2[kk][2] = pack_bf16x2(h1[2 * kk + 1][0], h1[2 * kk + 1][1]);
        a2[kk][3] = pack_bf16x2(h1[2 * kk + 1][2], h1[2 * kk + 1][3]);
    }
    float p0 = 0.f, p1 = 0.f;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        mma_bf16_16816(c, a2[0], r.w2[j][0][0], r.w2[j][0][1]);
        mma_bf16_16816(c, a2[1], r.w2[j][1][0], r.w2[j][1][1]);
        const float h00 = fmaxf(c[0] + r.b2[j][0], 0.f), h01 = fmaxf(c[1] + r.b2[j][1], 0.f);
        const float h10 = fmaxf(c[2] + r.b2[j][0], 0.f), h11 = fmaxf(c[3] + r.b2[j][1], 0.f);
        p0 = p0 + h00 * r.w3[j][0];
        p0 = p0 + h01 * r.w3[j][1];
        p1 = p1 + h10 * r.w3[j][0];
        p1 = p1 + h11 * r.w3[j][1];
    }
    p0 = p0 + __shfl_xor_sync(FULL, p0, 1);
    p0 = p0 + __shfl_xor_sync(FULL, p0, 2);
    p1 = p1 + __shfl_xor_sync(FULL, p1, 1);
    p1 = p1 + __shfl_xor_sync(FULL, p1, 2);
    lg0 = p0 + r.b3;
    lg1 = p1 + r.b3;
}

// Logits of 32 rows held in shared memory xs[32][xs_stride] (one warp); the
// result for row `lane` is returned to that lane.  `scratch` is 32 floats of
// this warp's shared memory.
__device__ __forceinline__ float mlp_warp32(const MlpRegs& r, const float* xs, int xs_stride, float* scratch) {
    const int l = threadIdx.x & 31, g = l >> 2, t = l & 3;
    float a0, a1, b0, b1;
    mlp_tile(r, xs, xs_stride, a0, a1);
    mlp_tile(r, xs + 16 * xs_stride, xs_stride, b0, b1);
    if (t == 0) {
        scratch[g] = a0;
        scratch[g + 8] = a1;
        scratch[g + 16] = b0;
        scratch[g + 24] = b1;
    }
    __syncwarp();
    float v = scratch[l];
    __syncwarp();
    return v;
}

}  // namespace pggc
