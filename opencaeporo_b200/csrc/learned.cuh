// learned.cuh -- the learned initialiser's network: an MLP
// (nin -> 64 -> 64 -> nout, SiLU) with BF16 weights and activations and FP32
// accumulation. This header holds its parameter layout and the scalar
// pieces; the tensor-core kernels are in learned_tc.cuh (evaluation) and
// learned.cu (training). No counterpart in the reference.
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

__device__ __forceinline__ uint32_t pack_bf16(bf16 lo, bf16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ float silu(float v) { return v / (1.f + __expf(-v)); }
__device__ __forceinline__ float silu_grad(float v)
{
    const float s = 1.f / (1.f + __expf(-v));
    return s * (1.f + v * (1.f - s));
}

}  // namespace ocpf
