// flash_batched_nc6.cu -- the batched (persistent equilibrium + finalize)
// FIM flash kernels for 6 hydrocarbon components.
#include "flash_batched.cuh"

namespace ocpf {

__global__ void __launch_bounds__(128) k_eq_batched_nc6(const __grid_constant__ FluidConst F, int64_t count,
                                                         int64_t stride, const ocpf_fim_in in,
                                                         const ocpf_skip sk, const EqBuf eb,
                                                         unsigned long long* queue)
{
    eq_persistent_body<6>(F, count, stride, in, sk, eb, queue);
}

__global__ void __launch_bounds__(128) k_finalize_nc6(const __grid_constant__ FluidConst F, int64_t count,
                                                       int64_t stride, const ocpf_fim_in in,
                                                       const ocpf_skip sk, const EqBuf eb,
                                                       const ocpf_fim_out out)
{
    finalize_body<6>(F, count, stride, in, sk, eb, out);
}

cudaError_t launch_batched_nc6(const FluidConst& F, int64_t count, int64_t stride, const ocpf_fim_in& in,
                                const ocpf_skip& sk, const ocpf_fim_out& out, const EqBuf& eb,
                                unsigned long long* queue, int eq_blocks, cudaStream_t st)
{
    if (eq_blocks <= 0) {
        int per_sm = 0, dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_eq_batched_nc6, 128, 0);
        eq_blocks = sms * (per_sm > 0 ? per_sm : 1);
    }
    const int64_t need = (count + 127) / 128;
    if (eq_blocks > need) eq_blocks = (int)need;
    cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st);
    k_eq_batched_nc6<<<eq_blocks, 128, 0, st>>>(F, count, stride, in, sk, eb, queue);
    const unsigned fb = (unsigned)((count + 127) / 128);
    k_finalize_nc6<<<fb, 128, 0, st>>>(F, count, stride, in, sk, eb, out);
    return cudaGetLastError();
}

}  // namespace ocpf
