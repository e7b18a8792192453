// flash_multi_d.cu -- multi-region kernels of the last steps: the split's
// restarts (one warp or one thread per cell) and finalize (flash_multi.cuh).
#include "flash_multi.cuh"

namespace ocpf {

#define KM __global__ void __launch_bounds__(128)
KM kpm_slow(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M)
{
    OCPF_MULTI_ITEMS(MF, M, (slow_body<NC_>(F_, A_, L_SLOW)));
}
KM kpm_slow_thread(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M)
{
    OCPF_MULTI_ITEMS(MF, M, (slow_thread_body<NC_>(F_, A_, L_SLOW)));
}
KM kpm_finalize(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M)
{
    OCPF_MULTI_ITEMS(MF, M, (phased_finalize_body<NC_>(F_, A_)));
}
KM kpm_finalize_fimn(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M)
{
    OCPF_MULTI_ITEMS(MF, M, (phased_finalize_body<NC_, true>(F_, A_)));
}
#undef KM

cudaError_t multi_step_d(int s, const MultiFluid& MF, const MultiArgs& M, unsigned grid, int block, size_t smem,
                         cudaStream_t st, int, int, int, bool)
{
    switch (s) {
        case MS_SLOW: kpm_slow<<<grid, block, smem, st>>>(MF, M); break;
        case MS_SLOW_THREAD: kpm_slow_thread<<<grid, block, smem, st>>>(MF, M); break;
        case MS_FINALIZE: kpm_finalize<<<grid, block, smem, st>>>(MF, M); break;
        case MS_FINALIZE_FIMN: kpm_finalize_fimn<<<grid, block, smem, st>>>(MF, M); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int multi_occupancy_d(int)
{
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, (const void*)kpm_finalize, 128, 0);
    return n > 0 ? n : 1;
}

}  // namespace ocpf
