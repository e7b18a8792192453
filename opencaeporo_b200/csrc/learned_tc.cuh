// learned_tc.cuh -- the learned initialiser's forward pass on Blackwell's
// fifth-generation tensor cores (tcgen05): one CTA of 128 threads evaluates
// the MLP of learned.cuh (nin -> 64 -> 64 -> nout, SiLU, BF16 operands, FP32
// accumulation) for a tile of 128 samples, one sample per thread. No
// counterpart in the reference.
//
// Per tile:
//   * every thread writes its sample's 16 BF16 features into shared memory
//     (the A operand of layer 1);
//   * thread 0 issues the layer's tcgen05.mma (M = 128 samples, N = 64 or 16
//     outputs, K = 16 per instruction) with both operands read from shared
//     memory through matrix descriptors and the FP32 accumulator in tensor
//     memory (TMEM), then tcgen05.commit arrives on an mbarrier;
//   * every warp reads its 32 TMEM lanes (= its 32 samples) back with
//     tcgen05.ld, adds the bias, applies SiLU and writes the BF16 activations
//     as the next layer's A operand.
// The weights are staged once per CTA. The three layers share 64 TMEM
// columns (a layer's accumulator is read before the next layer's MMA is
// issued), so eight CTAs fit an SM's 512 columns.
//
// Shared-memory operand layout: K-major without swizzle, in 8-row x 16-byte
// core matrices. Row r's K elements 8c..8c+7 sit at byte
//   ((r / 8) * KC + c) * 128 + (r % 8) * 16,       KC = K / 8,
// so the descriptor's leading-dimension byte offset (between the two core
// matrices of one K = 16 step) is 128 and its stride byte offset (between
// 8-row groups) is KC * 128; the k-th K step starts 256 k bytes further.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

#include "learned.cuh"

namespace ocpf {

constexpr int MLP_TC_ROWS = 128;  // samples per tile = threads per CTA
constexpr int MLP_TC_COLS = 64;   // TMEM columns held by a CTA

struct MlpTcSmem {
    alignas(128) unsigned char w1[MLP_H * MLP_IO * 2];   // B of layer 1: 64 x 16
    alignas(128) unsigned char w2[MLP_H * MLP_H * 2];    // B of layer 2: 64 x 64
    alignas(128) unsigned char w3[MLP_IO * MLP_H * 2];   // B of layer 3: 16 x 64
    alignas(128) unsigned char xs[MLP_TC_ROWS * MLP_IO * 2];  // A of layer 1
    alignas(128) unsigned char h[MLP_TC_ROWS * MLP_H * 2];    // A of layers 2 and 3
    float    b1[MLP_H], b2[MLP_H], b3[MLP_IO];
    uint64_t mbar;
    uint32_t tmem;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of (row, K element) in the core-matrix layout above
__device__ __forceinline__ uint32_t core_off(int row, int k, int kc)
{
    return (uint32_t)(((row >> 3) * kc + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (SWIZZLE_NONE, K-major), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, M = 128; A and
// B K-major unless a_mn / b_mn (MN-major: bits 15 and 16).
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n, bool a_mn = false, bool b_mn = false)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(MLP_TC_ROWS >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

// An operand as the MMAs read it: start address, the descriptor's leading
// and stride byte offsets, and the advance of the start per K = 16 step.
struct TcOperand {
    uint32_t start, lbo, sbo, kstep;
};

// D (at TMEM address dtmem) = A B^T over `ksteps` K = 16 steps; issued by
// the calling thread.
__device__ __forceinline__ void tc_gemm(uint32_t dtmem, const TcOperand& A, const TcOperand& B, int ksteps,
                                        uint32_t idesc)
{
    for (int k = 0; k < ksteps; k++)
        tc_mma(dtmem, umma_desc(A.start + A.kstep * k, A.lbo, A.sbo), umma_desc(B.start + B.kstep * k, B.lbo, B.sbo),
               idesc, k > 0 ? 1u : 0u);
}

__device__ __forceinline__ void tc_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    __syncwarp();
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Waits for the mbarrier phase with the given parity; false when it has not
// completed after `limit` polls (each poll may suspend the thread briefly).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = (1u << 22))
{
    const uint32_t a = smem_u32(bar);
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// The CTA's network: weights staged once, TMEM held from begin() to end().
// Every member is called by all 128 threads of the CTA.
struct MlpTc {
    MlpTcSmem& s;
    uint32_t   phase = 0;
    bool       ok    = true;  // false once a wait has run out (every later tile is skipped)

    __device__ explicit MlpTc(MlpTcSmem& sm) : s(sm) {}

    __device__ void begin(const float* __restrict__ p)
    {
        const int t = threadIdx.x;
        if (t < 32) {
            __syncwarp();
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                         "r"((uint32_t)MLP_TC_COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
        if (t == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s.mbar)));
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        for (int i = t; i < MLP_H * MLP_IO; i += blockDim.x)
            *reinterpret_cast<bf16*>(s.w1 + core_off(i / MLP_IO, i % MLP_IO, MLP_IO / 8)) =
                __float2bfloat16(p[MLP_OFF_W1 + i]);
        for (int i = t; i < MLP_H * MLP_H; i += blockDim.x)
            *reinterpret_cast<bf16*>(s.w2 + core_off(i / MLP_H, i % MLP_H, MLP_H / 8)) =
                __float2bfloat16(p[MLP_OFF_W2 + i]);
        for (int i = t; i < MLP_IO * MLP_H; i += blockDim.x)
            *reinterpret_cast<bf16*>(s.w3 + core_off(i / MLP_H, i % MLP_H, MLP_H / 8)) =
                __float2bfloat16(p[MLP_OFF_W3 + i]);
        for (int i = t; i < MLP_H; i += blockDim.x) {
            s.b1[i] = p[MLP_OFF_B1 + i];
            s.b2[i] = p[MLP_OFF_B2 + i];
        }
        for (int i = t; i < MLP_IO; i += blockDim.x) s.b3[i] = p[MLP_OFF_B3 + i];
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }

    // Issues one layer (thread 0) and waits for its accumulator.
    __device__ bool layer(uint32_t a_base, int a_kc, uint32_t b_base, int b_kc, int ksteps, int n)
    {
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t idesc = umma_idesc_bf16(n);
            for (int k = 0; k < ksteps; k++)
                tc_mma(s.tmem, umma_desc(a_base + 256u * k, 128u, 128u * a_kc),
                       umma_desc(b_base + 256u * k, 128u, 128u * b_kc), idesc, k > 0 ? 1u : 0u);
            tc_commit(&s.mbar);
        }
        const bool done = mbar_wait(&s.mbar, phase);
        phase ^= 1u;
        tc_fence_after();
        return done;
    }

    // Layer output of this thread's sample: columns 0..63 + bias, SiLU, BF16
    // into the A operand of the next layer.
    __device__ void hidden_out(const float* bias)
    {
        const int      r     = threadIdx.x;
        const uint32_t taddr = s.tmem + ((uint32_t)(r & ~31) << 16);
#pragma unroll
        for (int q = 0; q < MLP_H / 16; q++) {
            float v[16];
            tc_ld16(taddr + 16u * q, v);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                uint32_t w[4];
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int c = 16 * q + 8 * h + 2 * e;
                    w[e] = pack_bf16(__float2bfloat16(silu(v[8 * h + 2 * e] + bias[c])),
                                     __float2bfloat16(silu(v[8 * h + 2 * e + 1] + bias[c + 1])));
                }
                *reinterpret_cast<uint4*>(s.h + core_off(r, 16 * q + 8 * h, MLP_H / 8)) =
                    make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
        tc_fence_before();
        fence_async_smem();
        __syncthreads();
    }

    // One tile: this thread's 16 features in, its 16 outputs (nout used)
    // out; NaN outputs when the tensor-core pipeline did not answer.
    __device__ void forward(const float (&f)[MLP_IO], float (&o)[MLP_IO])
    {
        const int r = threadIdx.x;
        if (ok) {
            uint32_t w[8];
#pragma unroll
            for (int e = 0; e < 8; e++) w[e] = pack_bf16(__float2bfloat16(f[2 * e]), __float2bfloat16(f[2 * e + 1]));
            *reinterpret_cast<uint4*>(s.xs + core_off(r, 0, MLP_IO / 8)) = make_uint4(w[0], w[1], w[2], w[3]);
            *reinterpret_cast<uint4*>(s.xs + core_off(r, 8, MLP_IO / 8)) = make_uint4(w[4], w[5], w[6], w[7]);
            fence_async_smem();
        }
        // previous tile's TMEM reads are done before this tile's MMA overwrites them
        tc_fence_before();
        __syncthreads();
        bool good = ok;
        if (good) good = layer(smem_u32(s.xs), MLP_IO / 8, smem_u32(s.w1), MLP_IO / 8, 1, MLP_H);
        good = __syncthreads_and(good);
        if (good) {
            hidden_out(s.b1);
            good = layer(smem_u32(s.h), MLP_H / 8, smem_u32(s.w2), MLP_H / 8, MLP_H / 16, MLP_H);
        }
        good = __syncthreads_and(good);
        if (good) {
            hidden_out(s.b2);
            good = layer(smem_u32(s.h), MLP_H / 8, smem_u32(s.w3), MLP_H / 8, MLP_H / 16, MLP_IO);
        }
        good = __syncthreads_and(good);
        if (good) {
            float v[16];
            tc_ld16(s.tmem + ((uint32_t)(r & ~31) << 16), v);
#pragma unroll
            for (int j = 0; j < MLP_IO; j++) o[j] = v[j] + s.b3[j];
        } else {
#pragma unroll
            for (int j = 0; j < MLP_IO; j++) o[j] = __int_as_float(0x7fc00000);
        }
        ok = good;
    }

    __device__ void end()
    {
        tc_fence_before();
        __syncthreads();
        if (threadIdx.x < 32) {
            __syncwarp();
            tc_fence_after();
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem),
                         "r"((uint32_t)MLP_TC_COLS));
        }
    }
};

}  // namespace ocpf
