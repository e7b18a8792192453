// flash_multi_b.cu -- multi-region kernels of the strict stability test:
// FP64 and FP32 substitution, verdict, Newton (flash_multi.cuh).
#include "flash_multi.cuh"

namespace ocpf {

#define KM __global__ void __launch_bounds__(128)
KM kpm_sta_ssm(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int list)
{
    OCPF_MULTI_PERSIST(MF, M, (sta_ssm_body<NC_>(F_, A_, list)));
}
KM kpm_sta_ssm32(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int k)
{
    OCPF_MULTI_PERSIST(MF, M, (sta_ssm32_body<NC_>(F_, A_, k)));
}
KM kpm_sta_verdict(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int k, int list,
                   int nrlist, bool from32)
{
    OCPF_MULTI_ITEMS(MF, M, (sta_verdict_body<NC_>(F_, A_, k, list, nrlist, from32)));
}
KM kpm_sta_nr(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int k, int list,
              int fallback)
{
    OCPF_MULTI_PERSIST(MF, M, (sta_nr_body<NC_>(F_, A_, k, list, fallback)));
}
#undef KM

cudaError_t multi_step_b(int s, const MultiFluid& MF, const MultiArgs& M, unsigned grid, int block, size_t smem,
                         cudaStream_t st, int i0, int i1, int i2, bool b0)
{
    switch (s) {
        case MS_STA_SSM: kpm_sta_ssm<<<grid, block, smem, st>>>(MF, M, i0); break;
        case MS_STA_SSM32: kpm_sta_ssm32<<<grid, block, smem, st>>>(MF, M, i0); break;
        case MS_STA_VERDICT: kpm_sta_verdict<<<grid, block, smem, st>>>(MF, M, i0, i1, i2, b0); break;
        case MS_STA_NR: kpm_sta_nr<<<grid, block, smem, st>>>(MF, M, i0, i1, i2); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int multi_occupancy_b(int s)
{
    const void* k = s == MS_STA_SSM32 ? (const void*)kpm_sta_ssm32
                  : s == MS_STA_NR    ? (const void*)kpm_sta_nr
                  : s == MS_STA_SSM   ? (const void*)kpm_sta_ssm
                                      : (const void*)kpm_sta_verdict;
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, 128, 0);
    return n > 0 ? n : 1;
}

}  // namespace ocpf
