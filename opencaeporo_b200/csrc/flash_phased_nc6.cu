// flash_phased_nc6.cu -- the batched (phase-by-phase) FIM flash kernels
// for 6 hydrocarbon components and their launch sequence.
#include "flash_phased_kernels.cuh"

namespace ocpf {

#define K128 __global__ void __launch_bounds__(128)
K128 kp_init_6(const __grid_constant__ FluidConst F, const PhasedArgs a) { init_body<6>(F, a); }
K128 kp_s01_prep_6(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { s01_prep_body<6>(F, a, k); }
K128 kp_s01_ssm_6(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { s01_ssm_body<6>(F, a, k); }
K128 kp_s01_end_6(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { s01_end_body<6>(F, a, k); }
K128 kp_sta_prep_6(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { sta_prep_body<6>(F, a, k); }
K128 kp_sta_ssm_6(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { sta_ssm_body<6>(F, a, k); }
K128 kp_sta_verdict_6(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { sta_verdict_body<6>(F, a, k); }
K128 kp_sta_nr_6(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { sta_nr_body<6>(F, a, k); }
K128 kp_sp_prep_6(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_prep_body<6>(F, a, r); }
K128 kp_sp_ssm_6(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_ssm_body<6>(F, a, r); }
K128 kp_sp_nrinit_6(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_nrinit_body<6>(F, a, r); }
K128 kp_sp_nr_6(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_nr_body<6>(F, a, r); }
K128 kp_slow_6(const __grid_constant__ FluidConst F, const PhasedArgs a) { slow_body<6>(F, a); }
K128 kp_finalize_6(const __grid_constant__ FluidConst F, const PhasedArgs a) { phased_finalize_body<6>(F, a); }
#undef K128

static int persistent_grid(const void* k, int sms)
{
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 128, 0);
    return sms * (per_sm > 0 ? per_sm : 1);
}

cudaError_t launch_phased_nc6(const FluidConst& F, const PhasedArgs& a, cudaStream_t st)
{
    static int g_s01 = 0, g_sta = 0, g_sp = 0, sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g_s01 = persistent_grid((const void*)kp_s01_ssm_6, sms);
        g_sta = persistent_grid((const void*)kp_sta_ssm_6, sms);
        g_sp  = persistent_grid((const void*)kp_sp_ssm_6, sms);
    }
    const int64_t need  = (a.count + 127) / 128;
    const int     gcell = (int)(need < (int64_t)sms * 8 ? need : (int64_t)sms * 8);
    const int     gp    = gcell;  // thread-per-item kernels over lists
    cudaMemsetAsync(a.L.ctr, 0, sizeof(uint32_t) * 2 * L_COUNT, st);
    kp_init_6<<<gcell, 128, 0, st>>>(F, a);
    for (int k = 0; k < 2; k++) {
        kp_s01_prep_6<<<gp, 128, 0, st>>>(F, a, k);
        kp_s01_ssm_6<<<g_s01, 128, 0, st>>>(F, a, k);
        kp_s01_end_6<<<gp, 128, 0, st>>>(F, a, k);
    }
    for (int k = 0; k < 4; k++) {
        kp_sta_prep_6<<<gp, 128, 0, st>>>(F, a, k);
        kp_sta_ssm_6<<<g_sta, 128, 0, st>>>(F, a, k);
        kp_sta_verdict_6<<<gp, 128, 0, st>>>(F, a, k);
        kp_sta_nr_6<<<gp, 128, 0, st>>>(F, a, k);
    }
    for (int r = 0; r < SPLIT_ROUNDS; r++) {
        kp_sp_prep_6<<<gp, 128, 0, st>>>(F, a, r);
        kp_sp_ssm_6<<<g_sp, 128, 0, st>>>(F, a, r);
        kp_sp_nrinit_6<<<gp, 128, 0, st>>>(F, a, r);
        kp_sp_nr_6<<<gp, 128, 0, st>>>(F, a, r);
    }
    kp_slow_6<<<gp, 128, 0, st>>>(F, a);
    kp_finalize_6<<<gcell, 128, 0, st>>>(F, a);
    return cudaGetLastError();
}

int phased_state_doubles_nc6() { return SF<6>::COUNT; }

}  // namespace ocpf
