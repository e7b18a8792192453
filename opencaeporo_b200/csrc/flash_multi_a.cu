// flash_multi_a.cu -- multi-region kernels of the sequence's first steps:
// init, the relaxed stability rounds, the strict rounds' set-up and the
// learned initialiser (flash_multi.cuh).
#include "flash_multi.cuh"

namespace ocpf {

#define KM __global__ void __launch_bounds__(128)
KM kpm_init(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M)
{
    OCPF_MULTI_ITEMS(MF, M, (init_body<NC_>(F_, A_)));
}
KM kpm_s01_prep(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int k)
{
    OCPF_MULTI_ITEMS(MF, M, (s01_prep_body<NC_>(F_, A_, k)));
}
KM kpm_s01_ssm(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int k)
{
    OCPF_MULTI_PERSIST(MF, M, (s01_ssm_body<NC_>(F_, A_, k)));
}
KM kpm_s01_end(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int k)
{
    OCPF_MULTI_ITEMS(MF, M, (s01_end_body<NC_>(F_, A_, k)));
}
KM kpm_sta_prep(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M, int k)
{
    OCPF_MULTI_ITEMS(MF, M, (sta_prep_body<NC_>(F_, A_, k)));
}
// Only the regions whose context holds a trained network (PH_LEARN) run it;
// the others have no parameters to read. The test is block-uniform, as the
// body's barriers need.
KM kpm_learn(const __grid_constant__ MultiFluid MF, const __grid_constant__ MultiArgs M)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (!(M.a[blockIdx.x % (uint32_t)M.n].opts & PH_LEARN) || !M.a[blockIdx.x % (uint32_t)M.n].mlp) return;
    OCPF_MULTI_ITEMS(MF, M, (learn_body<NC_>(F_, A_, *reinterpret_cast<LearnSmem*>(smem_raw))));
}
#undef KM

cudaError_t multi_step_a(int s, const MultiFluid& MF, const MultiArgs& M, unsigned grid, int block, size_t smem,
                         cudaStream_t st, int i0, int, int, bool)
{
    switch (s) {
        case MS_INIT: kpm_init<<<grid, block, smem, st>>>(MF, M); break;
        case MS_S01_PREP: kpm_s01_prep<<<grid, block, smem, st>>>(MF, M, i0); break;
        case MS_S01_SSM: kpm_s01_ssm<<<grid, block, smem, st>>>(MF, M, i0); break;
        case MS_S01_END: kpm_s01_end<<<grid, block, smem, st>>>(MF, M, i0); break;
        case MS_STA_PREP: kpm_sta_prep<<<grid, block, smem, st>>>(MF, M, i0); break;
        case MS_LEARN: {
            static bool attr = false;
            if (!attr) {
                cudaFuncSetAttribute(kpm_learn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(LearnSmem));
                attr = true;
            }
            kpm_learn<<<grid, block, smem, st>>>(MF, M);
            break;
        }
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int multi_occupancy_a(int s)
{
    const void* k = s == MS_S01_SSM ? (const void*)kpm_s01_ssm : (const void*)kpm_init;
    int         n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, 128, 0);
    return n > 0 ? n : 1;
}

}  // namespace ocpf
