// learned.cu -- training and evaluation kernels of the learned initialiser's
// MLP (learned.cuh) on the tcgen05 tensor cores (learned_tc.cuh), and their
// C entry points. No counterpart in the reference.
//
// Loss over a batch of n samples (outputs o, targets t, lnK weight w_s):
//   L = 1/n sum_s [ softplus(o_0) - t_0 o_0                    (stability logit)
//                   + lam w_s / (nout-1) sum_{i>=1} (o_i - t_i)^2 ]   (ln K)
// Training: one CTA of 128 threads takes 128 samples, thread t sample t.
// The forward pass, the backward pass through both hidden layers and the
// weight gradients are tcgen05.mma GEMMs with FP32 accumulators in tensor
// memory; the per-CTA gradient sums are added into the FP32 gradient with
// atomics.
#include <cuda_runtime.h>

#include "learned.cuh"
#include "learned_tc.cuh"
#include "ocp_flash.h"

namespace ocpf {
namespace {

// Shared memory of the training kernel. Activations are stored sample-major
// in the core-matrix layout of learned_tc.cuh, several per buffer, so that
// one buffer serves as a K-major operand of the forward and backward GEMMs
// (sample x feature, K = features) and as an MN-major operand of the
// weight-gradient GEMMs (feature x sample, K = samples):
//   q: x (features 0-15) | d2 (16-79) | d3 (80-95) | 1 (96) | 0 (97-111)
//   p: d1 (0-63) | h1 (64-127)
//   r: h2 (0-63) | 1 (64) | 0 (65-127)
// Weight-gradient GEMMs (M = 128 feature rows of p or r, N = features of q,
// K = the tile's 128 samples):
//   G1 = p^T q[0:112]: rows 0-63 x cols 0-15 = dW1, rows 0-63 x col 96 = db1,
//                      rows 64-127 x cols 16-79 = dW2^T
//   G2 = r^T q[16:96]: rows 0-63 x cols 64-79 = dW3^T, row 64 = (db2, db3)
// The other products of the two GEMMs are not used.
constexpr int QF = 112, PF = 128, RF = 128;  // features per sample of q, p, r

struct GradTcSmem {
    alignas(128) unsigned char w1[MLP_H * MLP_IO * 2];   // W1 [o1][i]   (N 64, K 16)
    alignas(128) unsigned char w2[MLP_H * MLP_H * 2];    // W2 [o2][o1]  (N 64, K 64)
    alignas(128) unsigned char w3[MLP_IO * MLP_H * 2];   // W3 [j][o2]   (N 16, K 64)
    alignas(128) unsigned char w3t[MLP_H * MLP_IO * 2];  // W3^T [o2][j] (N 64, K 16)
    alignas(128) unsigned char w2t[MLP_H * MLP_H * 2];   // W2^T [o1][o2] (N 64, K 64)
    alignas(128) unsigned char q[MLP_TC_ROWS * QF * 2];
    alignas(128) unsigned char p[MLP_TC_ROWS * PF * 2];
    alignas(128) unsigned char r[MLP_TC_ROWS * RF * 2];
    float    b1[MLP_H], b2[MLP_H], b3[MLP_IO];
    uint64_t mbar;
    uint32_t tmem;
};

// TMEM columns of the training kernel's accumulators (256 allocated)
constexpr uint32_t T_A1 = 0, T_A2 = 64, T_O = 128, T_DH2 = 192, T_DH1 = 64, T_G1 = 0, T_G2 = 128;
constexpr uint32_t T_COLS = 256;

__device__ __forceinline__ void st_bf16(unsigned char* buf, int row, int f, int kc, float v)
{
    *reinterpret_cast<bf16*>(buf + core_off(row, f, kc)) = __float2bfloat16(v);
}

// 8 BF16 values of features f..f+7 (f a multiple of 8) of one row
__device__ __forceinline__ void st_bf16x8(unsigned char* buf, int row, int f, int kc, const float* v)
{
    uint32_t w[4];
#pragma unroll
    for (int e = 0; e < 4; e++) w[e] = pack_bf16(__float2bfloat16(v[2 * e]), __float2bfloat16(v[2 * e + 1]));
    *reinterpret_cast<uint4*>(buf + core_off(row, f, kc)) = make_uint4(w[0], w[1], w[2], w[3]);
}

// K-major operand: features f0.. of a buffer with kc chunks per row
__device__ __forceinline__ TcOperand kmaj(const unsigned char* buf, int f0, int kc)
{
    return TcOperand{smem_u32(buf) + 16u * (uint32_t)f0, 128u, 128u * kc, 256u};
}
// MN-major operand: features f0.. (M or N) by samples (K) of a buffer
__device__ __forceinline__ TcOperand mnmaj(const unsigned char* buf, int f0, int kc)
{
    return TcOperand{smem_u32(buf) + 16u * (uint32_t)f0, 128u * kc, 128u, 256u * kc};
}

__device__ bool tc_step(GradTcSmem& sm, uint32_t& phase)
{
    const bool done = mbar_wait(&sm.mbar, phase);
    phase ^= 1u;
    tc_fence_after();
    return done;
}

// this thread's TMEM lane, columns c0..c0+16*nq-1 (nq <= 4)
__device__ __forceinline__ void tc_row(const GradTcSmem& sm, uint32_t c0, int nq, float* v)
{
    const uint32_t taddr = sm.tmem + ((uint32_t)(threadIdx.x & ~31) << 16) + c0;
    for (int q = 0; q < nq; q++) {
        float t[16];
        tc_ld16(taddr + 16u * q, t);
#pragma unroll
        for (int i = 0; i < 16; i++) v[16 * q + i] = t[i];
    }
}

__device__ __forceinline__ void tc_publish()
{
    tc_fence_before();
    fence_async_smem();
    __syncthreads();
}

__global__ void __launch_bounds__(MLP_TC_ROWS) k_mlp_grad(int nin, int nout, int64_t n, const float* __restrict__ prm,
                                                          const float* __restrict__ x, const float* __restrict__ tgt,
                                                          const float* __restrict__ wmask, float lam,
                                                          float* __restrict__ grad, float* __restrict__ loss)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    GradTcSmem& sm = *reinterpret_cast<GradTcSmem*>(smem_raw);
    const int   t  = threadIdx.x, lane = t & 31;
    if (t < 32) {
        __syncwarp();
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem)),
                     "r"(T_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sm.mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = t; i < MLP_H * MLP_IO; i += blockDim.x) {
        const int a = i / MLP_IO, b = i % MLP_IO;  // W1[a][b]
        st_bf16(sm.w1, a, b, MLP_IO / 8, prm[MLP_OFF_W1 + i]);
    }
    for (int i = t; i < MLP_H * MLP_H; i += blockDim.x) {
        const int a = i / MLP_H, b = i % MLP_H;  // W2[a][b]
        st_bf16(sm.w2, a, b, MLP_H / 8, prm[MLP_OFF_W2 + i]);
        st_bf16(sm.w2t, b, a, MLP_H / 8, prm[MLP_OFF_W2 + i]);
    }
    for (int i = t; i < MLP_IO * MLP_H; i += blockDim.x) {
        const int a = i / MLP_H, b = i % MLP_H;  // W3[a][b]
        st_bf16(sm.w3, a, b, MLP_H / 8, prm[MLP_OFF_W3 + i]);
        st_bf16(sm.w3t, b, a, MLP_IO / 8, prm[MLP_OFF_W3 + i]);
    }
    for (int i = t; i < MLP_H; i += blockDim.x) {
        sm.b1[i] = prm[MLP_OFF_B1 + i];
        sm.b2[i] = prm[MLP_OFF_B2 + i];
    }
    for (int i = t; i < MLP_IO; i += blockDim.x) sm.b3[i] = prm[MLP_OFF_B3 + i];

    // this thread's sample: x, the ones columns and the zero padding
    const int64_t s     = (int64_t)blockIdx.x * MLP_TC_ROWS + t;
    const bool    valid = s < n;
    {
        float v[8];
        for (int c = 0; c < 2; c++) {
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const int f = 8 * c + e;
                v[e]        = (valid && f < nin) ? x[(int64_t)f * n + s] : 0.f;
            }
            st_bf16x8(sm.q, t, 8 * c, QF / 8, v);
        }
#pragma unroll
        for (int e = 0; e < 8; e++) v[e] = 0.f;
        for (int f = 96; f < QF; f += 8) {
            v[0] = (f == 96 && valid) ? 1.f : 0.f;
            st_bf16x8(sm.q, t, f, QF / 8, v);
        }
        for (int f = 64; f < RF; f += 8) {
            v[0] = (f == 64 && valid) ? 1.f : 0.f;
            st_bf16x8(sm.r, t, f, RF / 8, v);
        }
    }
    tc_publish();
    tc_fence_after();

    uint32_t  phase = 0;
    bool      good  = true;
    const uint32_t T = sm.tmem;
    float     v[64], a[64];

    // F1: a1 = x W1^T
    if (t == 0) {
        tc_fence_after();
        tc_gemm(T + T_A1, kmaj(sm.q, 0, QF / 8), kmaj(sm.w1, 0, MLP_IO / 8), 1, umma_idesc_bf16(MLP_H));
        tc_commit(&sm.mbar);
    }
    good = __syncthreads_and(tc_step(sm, phase));
    if (good) {  // h1 = silu(a1 + b1)
        tc_row(sm, T_A1, 4, v);
        for (int c = 0; c < 8; c++) {
            float h[8];
#pragma unroll
            for (int e = 0; e < 8; e++) h[e] = silu(v[8 * c + e] + sm.b1[8 * c + e]);
            st_bf16x8(sm.p, t, 64 + 8 * c, PF / 8, h);
        }
        tc_publish();
        // F2: a2 = h1 W2^T
        if (t == 0) {
            tc_fence_after();
            tc_gemm(T + T_A2, kmaj(sm.p, 64, PF / 8), kmaj(sm.w2, 0, MLP_H / 8), MLP_H / 16, umma_idesc_bf16(MLP_H));
            tc_commit(&sm.mbar);
        }
        good = tc_step(sm, phase);
    }
    good = __syncthreads_and(good);
    if (good) {  // h2 = silu(a2 + b2)
        tc_row(sm, T_A2, 4, v);
        for (int c = 0; c < 8; c++) {
            float h[8];
#pragma unroll
            for (int e = 0; e < 8; e++) h[e] = silu(v[8 * c + e] + sm.b2[8 * c + e]);
            st_bf16x8(sm.r, t, 8 * c, RF / 8, h);
        }
        tc_publish();
        // F3: o = h2 W3^T
        if (t == 0) {
            tc_fence_after();
            tc_gemm(T + T_O, kmaj(sm.r, 0, RF / 8), kmaj(sm.w3, 0, MLP_H / 8), MLP_H / 16, umma_idesc_bf16(MLP_IO));
            tc_commit(&sm.mbar);
        }
        good = tc_step(sm, phase);
    }
    good = __syncthreads_and(good);
    float bce = 0.f, mse = 0.f;
    if (good) {  // loss and d3 = dL/do
        float o[16], d[16];
        tc_row(sm, T_O, 1, o);
#pragma unroll
        for (int j = 0; j < MLP_IO; j++) d[j] = 0.f;
        if (valid) {
            const float inv = 1.f / (float)n;
            const float z   = o[0] + sm.b3[0];
            const float y   = tgt[s];
            bce             = fmaxf(z, 0.f) + log1pf(__expf(-fabsf(z))) - y * z;
            d[0]            = (1.f / (1.f + __expf(-z)) - y) * inv;
            const float w   = wmask[s] * lam / (float)(nout - 1);
            for (int j = 1; j < nout; j++) {
                const float e = o[j] + sm.b3[j] - tgt[(int64_t)j * n + s];
                mse += wmask[s] * e * e / (float)(nout - 1);
                d[j] = 2.f * w * e * inv;
            }
        }
        st_bf16x8(sm.q, t, 80, QF / 8, d);
        st_bf16x8(sm.q, t, 88, QF / 8, d + 8);
        tc_publish();
        // B1: dh2 = d3 W3
        if (t == 0) {
            tc_fence_after();
            tc_gemm(T + T_DH2, kmaj(sm.q, 80, QF / 8), kmaj(sm.w3t, 0, MLP_IO / 8), 1, umma_idesc_bf16(MLP_H));
            tc_commit(&sm.mbar);
        }
        good = tc_step(sm, phase);
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
    good = __syncthreads_and(good);
    if (good) {  // d2 = dh2 * silu'(a2 + b2)
        tc_row(sm, T_DH2, 4, v);
        tc_row(sm, T_A2, 4, a);
        for (int c = 0; c < 8; c++) {
            float h[8];
#pragma unroll
            for (int e = 0; e < 8; e++) h[e] = v[8 * c + e] * silu_grad(a[8 * c + e] + sm.b2[8 * c + e]);
            st_bf16x8(sm.q, t, 16 + 8 * c, QF / 8, h);
        }
        tc_publish();
        // B2: dh1 = d2 W2 (into a2's columns, read above)
        if (t == 0) {
            tc_fence_after();
            tc_gemm(T + T_DH1, kmaj(sm.q, 16, QF / 8), kmaj(sm.w2t, 0, MLP_H / 8), MLP_H / 16, umma_idesc_bf16(MLP_H));
            tc_commit(&sm.mbar);
        }
        good = tc_step(sm, phase);
    }
    good = __syncthreads_and(good);
    if (good) {  // d1 = dh1 * silu'(a1 + b1)
        tc_row(sm, T_DH1, 4, v);
        tc_row(sm, T_A1, 4, a);
        for (int c = 0; c < 8; c++) {
            float h[8];
#pragma unroll
            for (int e = 0; e < 8; e++) h[e] = v[8 * c + e] * silu_grad(a[8 * c + e] + sm.b1[8 * c + e]);
            st_bf16x8(sm.p, t, 8 * c, PF / 8, h);
        }
        tc_publish();
        // G1 = p^T q[0:112], G2 = r^T q[16:96]: the tile's 128 samples as K
        if (t == 0) {
            tc_fence_after();
            tc_gemm(T + T_G1, mnmaj(sm.p, 0, PF / 8), mnmaj(sm.q, 0, QF / 8), MLP_TC_ROWS / 16,
                    umma_idesc_bf16(QF, true, true));
            tc_gemm(T + T_G2, mnmaj(sm.r, 0, RF / 8), mnmaj(sm.q, 16, QF / 8), MLP_TC_ROWS / 16,
                    umma_idesc_bf16(80, true, true));
            tc_commit(&sm.mbar);
        }
        good = tc_step(sm, phase);
    }
    good = __syncthreads_and(good);
    if (good) {
        // G1 row t: t < 64 -> dW1[t][0:16] and db1[t]; t >= 64 -> dW2[0:64][t - 64]
        if (t < 64) {
            tc_row(sm, T_G1, 1, v);
            tc_row(sm, T_G1 + 96, 1, a);
            for (int i = 0; i < MLP_IO; i++) atomicAdd(&grad[MLP_OFF_W1 + t * MLP_IO + i], v[i]);
            atomicAdd(&grad[MLP_OFF_B1 + t], a[0]);
        } else {
            tc_row(sm, T_G1 + 16, 4, v);
            for (int o2 = 0; o2 < MLP_H; o2++) atomicAdd(&grad[MLP_OFF_W2 + o2 * MLP_H + (t - 64)], v[o2]);
        }
        // G2 row t: t < 64 -> dW3[0:16][t]; t == 64 -> db2, db3
        tc_row(sm, T_G2, 4, v);
        tc_row(sm, T_G2 + 64, 1, a);
        if (t < 64) {
            for (int j = 0; j < MLP_IO; j++) atomicAdd(&grad[MLP_OFF_W3 + j * MLP_H + t], a[j]);
        } else if (t == 64) {
            for (int o2 = 0; o2 < MLP_H; o2++) atomicAdd(&grad[MLP_OFF_B2 + o2], v[o2]);
            for (int j = 0; j < MLP_IO; j++) atomicAdd(&grad[MLP_OFF_B3 + j], a[j]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (t < 32) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(T), "r"(T_COLS));
    }
    if (!good && t == 0) loss[0] = __int_as_float(0x7fc00000);  // the tensor-core pipeline did not answer
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
    const int64_t blocks = (n + MLP_TC_ROWS - 1) / MLP_TC_ROWS;
    if (blocks > 0x7fffffffLL) return OCPF_EINVAL;
    const size_t sm = sizeof(GradTcSmem);
    if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
        return OCPF_ECUDA;
    k_mlp_grad<<<(unsigned)blocks, MLP_TC_ROWS, sm, (cudaStream_t)stream>>>(nin, nout, n, params, x, target, wmask,
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
