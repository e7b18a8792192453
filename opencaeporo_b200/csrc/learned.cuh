// learned.cuh -- the learned initialiser's network on the tensor cores:
// an MLP (nin -> 64 -> 64 -> nout, SiLU) with BF16 weights and activations
// and FP32 accumulation, evaluated and differentiated warp by warp with
// mma.sync.m16n8k16 (BF16 x BF16 -> FP32). No counterpart in the reference.
//
// Operands live in shared memory; every tile product names its operands by
// strides, so the transposed products of the backward pass need no copies:
// A(m, k) = A[m * sm + k * sk], B(n, k) = B[n * sn + k * sk].
//
// Parameter vector (FP32, MLP_NPARAM floats), row-major [out][in] weights,
// inputs and outputs zero-padded to 16:
//   W1[64][16] b1[64] W2[64][64] b2[64] W3[16][64] b3[16]
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace ocpf {

constexpr int MLP_H      = 64;  // hidden width
constexpr int MLP_IO     = 16;  // padded input / output width
constexpr int MLP_OFF_W1 = 0;
constexpr int MLP_OFF_B1 = MLP_OFF_W1 + MLP_H * MLP_IO;
constexpr int MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;
constexpr int MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H;
constexpr int MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;
constexpr int MLP_OFF_B3 = MLP_OFF_W3 + MLP_IO * MLP_H;
constexpr int MLP_NPARAM = MLP_OFF_B3 + MLP_IO;  // 6288

using bf16 = __nv_bfloat16;

// Weights of one CTA in shared memory (BF16) with FP32 biases.
struct MlpSmemW {
    bf16  w1[MLP_H * MLP_IO];
    bf16  w2[MLP_H * MLP_H];
    bf16  w3[MLP_IO * MLP_H];
    float b1[MLP_H], b2[MLP_H], b3[MLP_IO];
};

__device__ __forceinline__ void mlp_load_weights(MlpSmemW& w, const float* __restrict__ p)
{
    for (int i = threadIdx.x; i < MLP_H * MLP_IO; i += blockDim.x) w.w1[i] = __float2bfloat16(p[MLP_OFF_W1 + i]);
    for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) w.w2[i] = __float2bfloat16(p[MLP_OFF_W2 + i]);
    for (int i = threadIdx.x; i < MLP_IO * MLP_H; i += blockDim.x) w.w3[i] = __float2bfloat16(p[MLP_OFF_W3 + i]);
    for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
        w.b1[i] = p[MLP_OFF_B1 + i];
        w.b2[i] = p[MLP_OFF_B2 + i];
    }
    for (int i = threadIdx.x; i < MLP_IO; i += blockDim.x) w.b3[i] = p[MLP_OFF_B3 + i];
}

__device__ __forceinline__ uint32_t pack_bf16(bf16 lo, bf16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// D = A B + C for one 16x8 tile, K = 16 (PTX mma.m16n8k16, row.col).
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Fragment loads for mma.m16n8k16 (16-bit types): lane = 4 g + t holds
//   A: (g, 2t..2t+1), (g+8, 2t..2t+1), (g, 2t+8..2t+9), (g+8, 2t+8..2t+9)
//   B: (k = 2t..2t+1, n = g), (k = 2t+8..2t+9, n = g)
//   C: (g, 2t..2t+1), (g+8, 2t..2t+1)
__device__ __forceinline__ void load_a(const bf16* A, int sm, int sk, int m0, int k0, uint32_t (&a)[4])
{
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    const bf16* r0 = A + (m0 + g) * sm;
    const bf16* r1 = A + (m0 + g + 8) * sm;
    const int   k  = k0 + 2 * t;
    a[0] = pack_bf16(r0[k * sk], r0[(k + 1) * sk]);
    a[1] = pack_bf16(r1[k * sk], r1[(k + 1) * sk]);
    a[2] = pack_bf16(r0[(k + 8) * sk], r0[(k + 9) * sk]);
    a[3] = pack_bf16(r1[(k + 8) * sk], r1[(k + 9) * sk]);
}

__device__ __forceinline__ void load_b(const bf16* B, int sn, int sk, int n0, int k0, uint32_t (&b)[2])
{
    const int   g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    const bf16* r = B + (n0 + g) * sn;
    const int   k = k0 + 2 * t;
    b[0] = pack_bf16(r[k * sk], r[(k + 1) * sk]);
    b[1] = pack_bf16(r[(k + 8) * sk], r[(k + 9) * sk]);
}

// One 16x8 output tile of A (16 x K) times B (K x 8), K = 16 * ksteps.
__device__ __forceinline__ void tile_mm(float (&c)[4], const bf16* A, int sm, int sak, int m0, const bf16* B,
                                        int sn, int sbk, int n0, int ksteps)
{
    c[0] = c[1] = c[2] = c[3] = 0.f;
    for (int s = 0; s < ksteps; s++) {
        uint32_t a[4], b[2];
        load_a(A, sm, sak, m0, 16 * s, a);
        load_b(B, sn, sbk, n0, 16 * s, b);
        mma_bf16(c, a, b);
    }
}

__device__ __forceinline__ float silu(float v) { return v / (1.f + __expf(-v)); }
__device__ __forceinline__ float silu_grad(float v)
{
    const float s = 1.f / (1.f + __expf(-v));
    return s * (1.f + v * (1.f - s));
}

// Forward pass of the 16 samples m0..m0+15 held by one warp: xs [.][16]
// (sample-major BF16 inputs, padded) -> out [16][16] FP32 (the warp's rows,
// row-major, nout used). With a1/a2 non-null the FP32 pre-activations of the
// two hidden layers are kept ([.][64] sample-major) and h1/h2 receive the
// BF16 activations; otherwise h1/h2 are the warp's scratch.
__device__ __forceinline__ void mlp_forward_warp(const MlpSmemW& w, const bf16* xs, int m0, bf16* h1, bf16* h2,
                                                 float* a1, float* a2, float* out)
{
    const int g = (threadIdx.x & 31) >> 2, t = threadIdx.x & 3;
    // layer 1: [16 x 16] x [16 x 64]
    for (int nt = 0; nt < MLP_H / 8; nt++) {
        float c[4];
        tile_mm(c, xs, MLP_IO, 1, m0, w.w1, MLP_IO, 1, 8 * nt, 1);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int   r = m0 + g + (e >> 1) * 8, col = 8 * nt + 2 * t + (e & 1);
            const float v = c[e] + w.b1[col];
            if (a1) a1[r * MLP_H + col] = v;
            h1[r * MLP_H + col] = __float2bfloat16(silu(v));
        }
    }
    __syncwarp();
    // layer 2: [16 x 64] x [64 x 64]
    for (int nt = 0; nt < MLP_H / 8; nt++) {
        float c[4];
        tile_mm(c, h1, MLP_H, 1, m0, w.w2, MLP_H, 1, 8 * nt, MLP_H / 16);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int   r = m0 + g + (e >> 1) * 8, col = 8 * nt + 2 * t + (e & 1);
            const float v = c[e] + w.b2[col];
            if (a2) a2[r * MLP_H + col] = v;
            h2[r * MLP_H + col] = __float2bfloat16(silu(v));
        }
    }
    __syncwarp();
    // layer 3: [16 x 64] x [64 x 16]
    for (int nt = 0; nt < MLP_IO / 8; nt++) {
        float c[4];
        tile_mm(c, h2, MLP_H, 1, m0, w.w3, MLP_H, 1, 8 * nt, MLP_H / 16);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int r = g + (e >> 1) * 8, col = 8 * nt + 2 * t + (e & 1);
            out[r * MLP_IO + col] = c[e] + w.b3[col];
        }
    }
    __syncwarp();
}

}  // namespace ocpf
