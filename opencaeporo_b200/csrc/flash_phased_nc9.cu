// flash_phased_nc9.cu -- the batched (phase-by-phase) FIM flash kernels
// for 9 hydrocarbon components and their launch sequence.
#include <algorithm>

#include "flash_learned.cuh"
#include "flash_mixed.cuh"
#include "flash_phased_kernels.cuh"

namespace ocpf {

#define K128 __global__ void __launch_bounds__(128)
K128 kp_init_9(const __grid_constant__ FluidConst F, const PhasedArgs a) { init_body<9>(F, a); }
K128 kp_s01_prep_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { s01_prep_body<9>(F, a, k); }
K128 kp_s01_ssm_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { s01_ssm_body<9>(F, a, k); }
K128 kp_s01_end_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { s01_end_body<9>(F, a, k); }
K128 kp_sta_prep_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { sta_prep_body<9>(F, a, k); }
K128 kp_sta_ssm_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int list) { sta_ssm_body<9>(F, a, list); }
K128 kp_sta_ssm32_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { sta_ssm32_body<9>(F, a, k); }
K128 kp_sta_verdict_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int k, int list, int nrlist, bool from32)
{
    sta_verdict_body<9>(F, a, k, list, nrlist, from32);
}
K128 kp_sta_nr_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int k, int list, int fallback)
{
    sta_nr_body<9>(F, a, k, list, fallback);
}
K128 kp_sp_prep_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_prep_body<9>(F, a, r); }
K128 kp_sp_ssm_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_ssm_body<9>(F, a, r); }
K128 kp_sp_nrinit_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_nrinit_body<9>(F, a, r); }
K128 kp_sp_nr_9(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_nr_body<9>(F, a, r); }
K128 kp_slow_9(const __grid_constant__ FluidConst F, const PhasedArgs a) { slow_body<9>(F, a); }
__global__ void __launch_bounds__(128) kp_learn_9(const __grid_constant__ FluidConst F, const PhasedArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    learn_body<9>(F, a, *reinterpret_cast<LearnSmem*>(smem_raw));
}
K128 kp_finalize_9(const __grid_constant__ FluidConst F, const PhasedArgs a) { phased_finalize_body<9>(F, a); }
K128 kp_finalize_fimn_9(const __grid_constant__ FluidConst F, const PhasedArgs a) { phased_finalize_body<9, true>(F, a); }
#undef K128

static int persistent_grid(const void* k, int sms)
{
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 128, 0);
    return sms * (per_sm > 0 ? per_sm : 1);
}

// One split round: set-up, successive substitution, Newton start, Newton.
static void split_round_9(const FluidConst& F, const PhasedArgs& a, cudaStream_t st, int r, int gp, int gs,
                            int gnr)
{
    kp_sp_prep_9<<<gp, 128, 0, st>>>(F, a, r);
    kp_sp_ssm_9<<<gs, 128, 0, st>>>(F, a, r);
    kp_sp_nrinit_9<<<gp, 128, 0, st>>>(F, a, r);
    kp_sp_nr_9<<<gnr, 128, 0, st>>>(F, a, r);
}

cudaError_t launch_phased_nc9(const FluidConst& F, const PhasedArgs& a, cudaStream_t st)
{
    static int g_s01 = 0, g_sta = 0, g_sp = 0, g_sta32 = 0, g_spnr = 0, g_stnr = 0, sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g_s01 = persistent_grid((const void*)kp_s01_ssm_9, sms);
        g_sta = persistent_grid((const void*)kp_sta_ssm_9, sms);
        g_sp  = persistent_grid((const void*)kp_sp_ssm_9, sms);
        g_sta32 = persistent_grid((const void*)kp_sta_ssm32_9, sms);
        g_spnr  = persistent_grid((const void*)kp_sp_nr_9, sms);
        g_stnr  = persistent_grid((const void*)kp_sta_nr_9, sms);
        cudaFuncSetAttribute(kp_learn_9, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(LearnSmem));
    }
    const int64_t need  = (a.count + 127) / 128;
    const int     gcell = (int)(need < (int64_t)sms * 8 ? need : (int64_t)sms * 8);
    const int     gp    = gcell;  // thread-per-item kernels over lists
    const bool    mixed = (a.opts & PH_MIXED) != 0;
    cudaMemsetAsync(a.L.ctr, 0, sizeof(uint32_t) * 2 * L_COUNT, st);
    kp_init_9<<<gcell, 128, 0, st>>>(F, a);
    if (a.opts & PH_LEARN) {
        // learned initialiser: predicted-unstable fresh cells split first
        const int gl = (int)std::min<int64_t>((a.count + 63) / 64, (int64_t)sms * 4);
        kp_learn_9<<<gl, 128, sizeof(LearnSmem), st>>>(F, a);
        split_round_9(F, a, st, LEARN_ROUND, gp, g_sp, g_spnr);
    }
    for (int k = 0; k < 2; k++) {
        kp_s01_prep_9<<<gp, 128, 0, st>>>(F, a, k);
        kp_s01_ssm_9<<<g_s01, 128, 0, st>>>(F, a, k);
        kp_s01_end_9<<<gp, 128, 0, st>>>(F, a, k);
    }
    for (int k = 0; k < 4; k++) {
        kp_sta_prep_9<<<gp, 128, 0, st>>>(F, a, k);
        if (mixed) {
            // FP32 substitution, FP64 end point and Newton; trials whose
            // Newton fails continue in FP64, then Newton again
            kp_sta_ssm32_9<<<g_sta32, 128, 0, st>>>(F, a, k);
            kp_sta_verdict_9<<<gp, 128, 0, st>>>(F, a, k, L_STA_0 + k, L_NRSTA_0 + k, true);
            kp_sta_nr_9<<<g_stnr, 128, 0, st>>>(F, a, k, L_NRSTA_0 + k, L_STC_0 + k);
            kp_sta_ssm_9<<<g_sta, 128, 0, st>>>(F, a, L_STC_0 + k);
            kp_sta_verdict_9<<<gp, 128, 0, st>>>(F, a, k, L_STC_0 + k, L_NRSTC_0 + k, false);
            kp_sta_nr_9<<<g_stnr, 128, 0, st>>>(F, a, k, L_NRSTC_0 + k, -1);
        } else {
            kp_sta_ssm_9<<<g_sta, 128, 0, st>>>(F, a, L_STA_0 + k);
            kp_sta_verdict_9<<<gp, 128, 0, st>>>(F, a, k, L_STA_0 + k, L_NRSTA_0 + k, false);
            kp_sta_nr_9<<<g_stnr, 128, 0, st>>>(F, a, k, L_NRSTA_0 + k, -1);
        }
    }
    for (int r = 0; r < SPLIT_ROUNDS; r++)
        split_round_9(F, a, st, r, gp, g_sp, g_spnr);
    kp_slow_9<<<gp, 128, 0, st>>>(F, a);
    if (a.tail.mode & FM_FIMN)
        kp_finalize_fimn_9<<<gcell, 128, 0, st>>>(F, a);
    else
        kp_finalize_9<<<gcell, 128, 0, st>>>(F, a);
    return cudaGetLastError();
}

int phased_state_doubles_nc9() { return SF<9>::COUNT; }

}  // namespace ocpf
