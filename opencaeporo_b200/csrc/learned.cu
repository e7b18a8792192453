// learned.cu -- training and evaluation kernels of the learned initialiser's
// MLP (learned.cuh) and their C entry points. No counterpart in the
// reference.
//
// Loss over a batch of n samples (outputs o, targets t, lnK weight w_s):
//   L = 1/n sum_s [ softplus(o_0) - t_0 o_0                    (stability logit)
//                   + lam w_s / (nout-1) sum_{i>=1} (o_i - t_i)^2 ]   (ln K)
// One CTA takes 64 samples (4 warps x 16): forward, loss gradient and the
// backward pass through both hidden layers on the tensor cores, then the
// weight gradients as 64-sample tile products, added into the FP32
// gradient with atomics.
#include <cuda_runtime.h>

#include "learned.cuh"
#include "learned_tc.cuh"
#include "ocp_flash.h"

namespace ocpf {
namespace {

constexpr int TS  = 64;  // samples per CTA
constexpr int NTH = 128;

struct GradSmem {
    MlpSmemW w;
    bf16     xs[TS * MLP_IO];
    bf16     h1[TS * MLP_H], h2[TS * MLP_H];
    float    a1[TS * MLP_H], a2[TS * MLP_H];
    float    out[TS * MLP_IO];
    bf16     d3[TS * MLP_IO];
    bf16     d2[TS * MLP_H], d1[TS * MLP_H];
};

__device__ __forceinline__ void load_inputs(bf16* xs, const float* __restrict__ x, int nin, int64_t n, int64_t base)
{
    for (int i = threadIdx.x; i < TS * MLP_IO; i += blockDim.x) {
        const int     s = i / MLP_IO, f = i % MLP_IO;
        const int64_t g = base + s;
        const float   v = (f < nin && g < n) ? x[(int64_t)f * n + g] : 0.f;
        xs[i]           = __float2bfloat16(v);
    }
}

__global__ void __launch_bounds__(NTH) k_mlp_grad(int nin, int nout, int64_t n, const float* __restrict__ p,
                                                  const float* __restrict__ x, const float* __restrict__ tgt,
                                                  const float* __restrict__ wmask, float lam,
                                                  float* __restrict__ grad, float* __restrict__ loss)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem&     sm   = *reinterpret_cast<GradSmem*>(smem_raw);
    const int64_t base = (int64_t)blockIdx.x * TS;
    const int     warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int     g = lane >> 2, t = lane & 3;
    const int     m0 = 16 * warp;
    mlp_load_weights(sm.w, p);
    load_inputs(sm.xs, x, nin, n, base);
    __syncthreads();

    // forward (the warp's 16 samples)
    mlp_forward_warp(sm.w, sm.xs, m0, sm.h1, sm.h2, sm.a1, sm.a2, sm.out + m0 * MLP_IO);

    // loss and dL/d(out): lane r < 16 takes sample m0 + r
    float bce = 0.f, mse = 0.f;
    if (lane < 16) {
        const int     r  = m0 + lane;
        const int64_t s  = base + r;
        const bool    in = s < n;
        const float*  o  = sm.out + r * MLP_IO;
        float         d[MLP_IO];
#pragma unroll
        for (int j = 0; j < MLP_IO; j++) d[j] = 0.f;
        if (in) {
            const float inv = 1.f / (float)n;
            const float z   = o[0];
            const float y   = tgt[s];
            bce             = fmaxf(z, 0.f) + log1pf(__expf(-fabsf(z))) - y * z;
            d[0]            = (1.f / (1.f + __expf(-z)) - y) * inv;
            const float w   = wmask[s] * lam / (float)(nout - 1);
            for (int j = 1; j < nout; j++) {
                const float e = o[j] - tgt[(int64_t)j * n + s];
                mse += wmask[s] * e * e / (float)(nout - 1);
                d[j] = 2.f * w * e * inv;
            }
        }
#pragma unroll
        for (int j = 0; j < MLP_IO; j++) sm.d3[r * MLP_IO + j] = __float2bfloat16(d[j]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        bce += __shfl_xor_sync(0xffffffffu, bce, o);
        mse += __shfl_xor_sync(0xffffffffu, mse, o);
    }
    if (lane == 0) {
        atomicAdd(&loss[0], bce);
        atomicAdd(&loss[1], mse);
    }
    __syncwarp();

    // backward through layer 3: dh2 = d3 W3, d2 = dh2 * silu'(a2)
    for (int nt = 0; nt < MLP_H / 8; nt++) {
        float c[4];
        tile_mm(c, sm.d3, MLP_IO, 1, m0, sm.w.w3, 1, MLP_H, 8 * nt, 1);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int r = m0 + g + (e >> 1) * 8, col = 8 * nt + 2 * t + (e & 1);
            sm.d2[r * MLP_H + col] = __float2bfloat16(c[e] * silu_grad(sm.a2[r * MLP_H + col]));
        }
    }
    __syncwarp();
    // through layer 2: dh1 = d2 W2, d1 = dh1 * silu'(a1)
    for (int nt = 0; nt < MLP_H / 8; nt++) {
        float c[4];
        tile_mm(c, sm.d2, MLP_H, 1, m0, sm.w.w2, 1, MLP_H, 8 * nt, MLP_H / 16);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int r = m0 + g + (e >> 1) * 8, col = 8 * nt + 2 * t + (e & 1);
            sm.d1[r * MLP_H + col] = __float2bfloat16(c[e] * silu_grad(sm.a1[r * MLP_H + col]));
        }
    }
    __syncthreads();

    // weight gradients over the CTA's 64 samples (K = 64): 48 tiles of 16x8
    //   dW1[o1][i] = sum_s d1[s][o1] xs[s][i]   (4 x 2 tiles)
    //   dW2[o2][o1] = sum_s d2[s][o2] h1[s][o1] (4 x 8 tiles)
    //   dW3[j][o2] = sum_s d3[s][j] h2[s][o2]   (1 x 8 tiles)
    for (int tile = warp; tile < 48; tile += NTH / 32) {
        float c[4];
        int   off, ld, mt, nt;
        if (tile < 8) {
            mt = tile >> 1, nt = tile & 1, off = MLP_OFF_W1, ld = MLP_IO;
            tile_mm(c, sm.d1, 1, MLP_H, 16 * mt, sm.xs, 1, MLP_IO, 8 * nt, TS / 16);
        } else if (tile < 40) {
            mt = (tile - 8) >> 3, nt = (tile - 8) & 7, off = MLP_OFF_W2, ld = MLP_H;
            tile_mm(c, sm.d2, 1, MLP_H, 16 * mt, sm.h1, 1, MLP_H, 8 * nt, TS / 16);
        } else {
            mt = 0, nt = tile - 40, off = MLP_OFF_W3, ld = MLP_H;
            tile_mm(c, sm.d3, 1, MLP_IO, 0, sm.h2, 1, MLP_H, 8 * nt, TS / 16);
        }
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int row = 16 * mt + g + (e >> 1) * 8, col = 8 * nt + 2 * t + (e & 1);
            atomicAdd(&grad[off + row * ld + col], c[e]);
        }
    }
    // bias gradients
    for (int k = threadIdx.x; k < 2 * MLP_H + MLP_IO; k += blockDim.x) {
        float s = 0.f;
        if (k < MLP_H) {
            for (int r = 0; r < TS; r++) s += __bfloat162float(sm.d1[r * MLP_H + k]);
            atomicAdd(&grad[MLP_OFF_B1 + k], s);
        } else if (k < 2 * MLP_H) {
            for (int r = 0; r < TS; r++) s += __bfloat162float(sm.d2[r * MLP_H + k - MLP_H]);
            atomicAdd(&grad[MLP_OFF_B2 + k - MLP_H], s);
        } else {
            for (int r = 0; r < TS; r++) s += __bfloat162float(sm.d3[r * MLP_IO + k - 2 * MLP_H]);
            atomicAdd(&grad[MLP_OFF_B3 + k - 2 * MLP_H], s);
        }
    }
}

// Forward pass for evaluation on the tcgen05 tensor cores (learned_tc.cuh):
// 128 samples per CTA tile, grid-stride over the tiles.
__global__ void __launch_bounds__(MLP_TC_ROWS) k_mlp_forward(int nin, int nout, int64_t n, const float* __restrict__ p,
                                                             const float* __restrict__ x, float* __restrict__ y)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    MlpTc net(*reinterpret_cast<MlpTcSmem*>(smem_raw));
    net.begin(p);
    for (int64_t base = (int64_t)blockIdx.x * MLP_TC_ROWS; base < n; base += (int64_t)gridDim.x * MLP_TC_ROWS) {
        const int64_t s = base + threadIdx.x;
        float         f[MLP_IO], o[MLP_IO];
#pragma unroll
        for (int j = 0; j < MLP_IO; j++) f[j] = (j < nin && s < n) ? x[(int64_t)j * n + s] : 0.f;
        net.forward(f, o);
        if (s < n)
            for (int j = 0; j < nout; j++) y[(int64_t)j * n + s] = o[j];
    }
    net.end();
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected) on the FP32 master
// parameters; zeroes the gradient it consumed.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ gr, float* __restrict__ m, float* __restrict__ v,
                       float lr, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_NPARAM) return;
    const float g  = gr[i];
    const float mi = 0.9f * m[i] + 0.1f * g;
    const float vi = 0.999f * v[i] + 0.001f * g * g;
    m[i]           = mi;
    v[i]           = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
    gr[i] = 0.f;
}

bool io_ok(int nin, int nout) { return nin >= 1 && nin <= MLP_IO && nout >= 2 && nout <= MLP_IO; }

}  // namespace
}  // namespace ocpf

using namespace ocpf;

extern "C" int ocpf_mlp_param_count(void) { return MLP_NPARAM; }

extern "C" int ocpf_mlp_forward(int nin, int nout, int64_t n, const float* params, const float* x, float* y,
                                void* stream)
{
    if (!io_ok(nin, nout) || n < 0 || !params || (n > 0 && (!x || !y))) return OCPF_EINVAL;
    if (n == 0) return OCPF_OK;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return OCPF_ECUDA;
    const int64_t tiles  = (n + MLP_TC_ROWS - 1) / MLP_TC_ROWS;
    const int64_t blocks = tiles < (int64_t)sms * 8 ? tiles : (int64_t)sms * 8;
    const size_t  sm     = sizeof(MlpTcSmem);
    if (cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
        return OCPF_ECUDA;
    k_mlp_forward<<<(unsigned)blocks, MLP_TC_ROWS, sm, (cudaStream_t)stream>>>(nin, nout, n, params, x, y);
    return cudaGetLastError() == cudaSuccess ? OCPF_OK : OCPF_ECUDA;
}

extern "C" int ocpf_mlp_grad(int nin, int nout, int64_t n, const float* params, const float* x, const float* target,
                             const float* wmask, float lnk_weight, float* grad, float* loss, void* stream)
{
    if (!io_ok(nin, nout) || n < 0 || !params || !grad || !loss) return OCPF_EINVAL;
    if (n > 0 && (!x || !target || !wmask)) return OCPF_EINVAL;
    if (n == 0) return OCPF_OK;
    const int64_t blocks = (n + TS - 1) / TS;
    if (blocks > 0x7fffffffLL) return OCPF_EINVAL;
    const size_t sm = sizeof(GradSmem);
    if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
        return OCPF_ECUDA;
    k_mlp_grad<<<(unsigned)blocks, NTH, sm, (cudaStream_t)stream>>>(nin, nout, n, params, x, target, wmask,
                                                                    lnk_weight, grad, loss);
    return cudaGetLastError() == cudaSuccess ? OCPF_OK : OCPF_ECUDA;
}

extern "C" int ocpf_mlp_adam(float* params, float* grad, float* m, float* v, int step, float lr, void* stream)
{
    if (!params || !grad || !m || !v || step < 1) return OCPF_EINVAL;
    const float c1 = 1.f - powf(0.9f, (float)step);
    const float c2 = 1.f - powf(0.999f, (float)step);
    k_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, grad, m, v, lr, c1, c2);
    return cudaGetLastError() == cudaSuccess ? OCPF_OK : OCPF_ECUDA;
}
