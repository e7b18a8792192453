// flash_plain_inst.cuh -- the plain FP64 FIM flash kernels for one component
// count. Included once per translation unit flash_plain_ncN.cu with OCPF_NC
// defined (one unit per component count keeps the builds parallel).
#ifndef OCPF_NC
#error "define OCPF_NC (the component count) before including flash_plain_inst.cuh"
#endif

#include "flash_fim.cuh"

#define OCPF_CAT2(a, b) a##b
#define OCPF_CAT(a, b) OCPF_CAT2(a, b)

namespace ocpf {

// One thread per cell, 128 cells per block: the hardware block scheduler
// balances the very uneven per-cell iteration counts across the SMs.
__global__ void __launch_bounds__(128) OCPF_CAT(k_flash_fim_plain_nc, OCPF_NC)(
    const __grid_constant__ FluidConst F, int64_t count, int64_t stride, const ocpf_fim_in in, const ocpf_skip sk,
    const ocpf_fim_out out, const FlashTail tail)
{
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= count) return;
    FimCell<OCPF_NC> c(F);
    c.run(n, stride, in, sk, out, tail);
}

// The same for FlashFIMn / InitFlashFIMn (the FIMn tail in a kernel of its own).
__global__ void __launch_bounds__(128) OCPF_CAT(k_flash_fimn_plain_nc, OCPF_NC)(
    const __grid_constant__ FluidConst F, int64_t count, int64_t stride, const ocpf_fim_in in, const ocpf_skip sk,
    const ocpf_fim_out out, const FlashTail tail)
{
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= count) return;
    FimCell<OCPF_NC> c(F);
    c.template run<true>(n, stride, in, sk, out, tail);
}

cudaError_t OCPF_CAT(launch_plain_nc, OCPF_NC)(const FluidConst& F, int64_t count, int64_t stride,
                                               const ocpf_fim_in& in, const ocpf_skip& sk, const ocpf_fim_out& out,
                                               const FlashTail& tail, unsigned blocks, int bs, cudaStream_t st)
{
    if (tail.mode & FM_FIMN)
        OCPF_CAT(k_flash_fimn_plain_nc, OCPF_NC)<<<blocks, bs, 0, st>>>(F, count, stride, in, sk, out, tail);
    else
        OCPF_CAT(k_flash_fim_plain_nc, OCPF_NC)<<<blocks, bs, 0, st>>>(F, count, stride, in, sk, out, tail);
    return cudaGetLastError();
}

}  // namespace ocpf
