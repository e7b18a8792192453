// flash_plain_nc9.cu -- the plain FP64 FIM flash kernel for 9 hydrocarbon
// components (one translation unit per component count keeps builds parallel).
#include "flash_fim.cuh"

namespace ocpf {

// One thread per cell, 128 cells per block: the hardware block scheduler
// balances the very uneven per-cell iteration counts across the SMs.
__global__ void __launch_bounds__(128) k_flash_fim_plain_nc9(const __grid_constant__ FluidConst F,
                                                             int64_t count, int64_t stride,
                                                             const ocpf_fim_in in, const ocpf_skip sk,
                                                             const ocpf_fim_out out, const FlashTail tail)
{
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= count) return;
    FimCell<9> c(F);
    c.run(n, stride, in, sk, out, tail);
}

// The same for FlashFIMn / InitFlashFIMn (the FIMn tail in a kernel of its own).
__global__ void __launch_bounds__(128) k_flash_fimn_plain_nc9(const __grid_constant__ FluidConst F,
                                                              int64_t count, int64_t stride,
                                                              const ocpf_fim_in in, const ocpf_skip sk,
                                                              const ocpf_fim_out out, const FlashTail tail)
{
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= count) return;
    FimCell<9> c(F);
    c.template run<true>(n, stride, in, sk, out, tail);
}

cudaError_t launch_plain_nc9(const FluidConst& F, int64_t count, int64_t stride, const ocpf_fim_in& in,
                              const ocpf_skip& sk, const ocpf_fim_out& out, const FlashTail& tail,
                              unsigned blocks, int bs, cudaStream_t st)
{
    if (tail.mode & FM_FIMN)
        k_flash_fimn_plain_nc9<<<blocks, bs, 0, st>>>(F, count, stride, in, sk, out, tail);
    else
        k_flash_fim_plain_nc9<<<blocks, bs, 0, st>>>(F, count, stride, in, sk, out, tail);
    return cudaGetLastError();
}

}  // namespace ocpf
