// flash_multi_c.cu -- multi-region kernels of the split's rounds: set-up,
// substitution, Newton start, Newton (flash_multi.cuh).
#include "flash_multi.cuh"

namespace ocpf {

#define KM __global__ void __launch_bounds__(128)
KM kpm_sp_prep(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int r)
{
    OCPF_MULTI_ITEMS(MF, M, (sp_prep_body<NC_>(F_, A_, r)));
}
KM kpm_sp_ssm(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int r)
{
    OCPF_MULTI_PERSIST(MF, M, (sp_ssm_body<NC_>(F_, A_, r)));
}
KM kpm_sp_nrinit(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int r)
{
    OCPF_MULTI_ITEMS(MF, M, (sp_nrinit_body<NC_>(F_, A_, r)));
}
KM kpm_sp_nr(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int r)
{
    OCPF_MULTI_PERSIST(MF, M, (sp_nr_body<NC_>(F_, A_, r)));
}
#undef KM

cudaError_t multi_step_c(int s, const MultiFluid& MF, const MultiArgs& M, unsigned grid, int block, size_t smem,
                         cudaStream_t st, int i0, int, int, bool)
{
    switch (s) {
        case MS_SP_PREP: kpm_sp_prep<<<grid, block, smem, st>>>(MF, M, i0); break;
        case MS_SP_SSM: kpm_sp_ssm<<<grid, block, smem, st>>>(MF, M, i0); break;
        case MS_SP_NRINIT: kpm_sp_nrinit<<<grid, block, smem, st>>>(MF, M, i0); break;
        case MS_SP_NR: kpm_sp_nr<<<grid, block, smem, st>>>(MF, M, i0); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int multi_occupancy_c(int s)
{
    const void* k = s == MS_SP_SSM ? (const void*)kpm_sp_ssm
                  : s == MS_SP_NR  ? (const void*)kpm_sp_nr
                                   : (const void*)kpm_sp_prep;
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, 128, 0);
    return n > 0 ? n : 1;
}

}  // namespace ocpf
