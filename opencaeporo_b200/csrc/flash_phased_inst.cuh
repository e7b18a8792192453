// flash_phased_inst.cuh -- the batched (phase-by-phase) FIM flash kernels for
// one component count and their launch sequence. Included once per
// translation unit flash_phased_ncN.cu with OCPF_NC defined (one unit per
// component count keeps the builds parallel); every kernel is named
// kp_<step>_<NC>.
#ifndef OCPF_NC
#error "define OCPF_NC (the component count) before including flash_phased_inst.cuh"
#endif

#include <algorithm>

#include "flash_learned.cuh"
#include "flash_mixed.cuh"
#include "flash_phased_kernels.cuh"

#define OCPF_CAT2(a, b) a##b
#define OCPF_CAT(a, b) OCPF_CAT2(a, b)
#define KP(step) OCPF_CAT(kp_##step##_, OCPF_NC)

namespace ocpf {

constexpr int kNC = OCPF_NC;

#define K128 __global__ void __launch_bounds__(128)
K128 KP(init)(const __grid_constant__ FluidConst F, const PhasedArgs a) { init_body<kNC>(F, a); }
K128 KP(s01_prep)(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { s01_prep_body<kNC>(F, a, k); }
K128 KP(s01_ssm)(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { s01_ssm_body<kNC>(F, a, k); }
K128 KP(s01_end)(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { s01_end_body<kNC>(F, a, k); }
K128 KP(sta_prep)(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { sta_prep_body<kNC>(F, a, k); }
K128 KP(sta_ssm)(const __grid_constant__ FluidConst F, const PhasedArgs a, int list) { sta_ssm_body<kNC>(F, a, list); }
K128 KP(sta_ssm32)(const __grid_constant__ FluidConst F, const PhasedArgs a, int k) { sta_ssm32_body<kNC>(F, a, k); }
K128 KP(sta_verdict)(const __grid_constant__ FluidConst F, const PhasedArgs a, int k, int list, int nrlist,
                     bool from32)
{
    sta_verdict_body<kNC>(F, a, k, list, nrlist, from32);
}
K128 KP(sta_nr)(const __grid_constant__ FluidConst F, const PhasedArgs a, int k, int list, int fallback)
{
    sta_nr_body<kNC>(F, a, k, list, fallback);
}
K128 KP(sp_prep)(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_prep_body<kNC>(F, a, r); }
K128 KP(sp_ssm)(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_ssm_body<kNC>(F, a, r); }
K128 KP(sp_nrinit)(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_nrinit_body<kNC>(F, a, r); }
K128 KP(sp_nr)(const __grid_constant__ FluidConst F, const PhasedArgs a, int r) { sp_nr_body<kNC>(F, a, r); }
K128 KP(slow)(const __grid_constant__ FluidConst F, const PhasedArgs a, int list) { slow_body<kNC>(F, a, list); }
K128 KP(slow_thread)(const __grid_constant__ FluidConst F, const PhasedArgs a, int list)
{
    slow_thread_body<kNC>(F, a, list);
}
K128 KP(learn)(const __grid_constant__ FluidConst F, const PhasedArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    learn_body<kNC>(F, a, *reinterpret_cast<LearnSmem*>(smem_raw));
}
K128 KP(finalize)(const __grid_constant__ FluidConst F, const PhasedArgs a) { phased_finalize_body<kNC>(F, a); }
K128 KP(finalize_fimn)(const __grid_constant__ FluidConst F, const PhasedArgs a)
{
    phased_finalize_body<kNC, true>(F, a);
}
#undef K128

namespace {

// Resident blocks per SM of a persistent kernel at 128 threads (what its
// registers allow), scaled by the tuned percentage.
int OCPF_CAT(persistent_grid_, OCPF_NC)(const void* k, int sms, int pct)
{
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 128, 0);
    per_sm = per_sm > 0 ? per_sm : 1;
    const int use = std::max(1, (per_sm * pct + 99) / 100);
    return sms * use;
}

// One split round: set-up, successive substitution, Newton start, Newton.
void OCPF_CAT(split_round_, OCPF_NC)(const FluidConst& F, const PhasedArgs& a, cudaStream_t st, int r, int gp,
                                    int bp, int gs, int gnr)
{
    KP(sp_prep)<<<gp, bp, 0, st>>>(F, a, r);
    KP(sp_ssm)<<<gs, 128, 0, st>>>(F, a, r);
    KP(sp_nrinit)<<<gp, bp, 0, st>>>(F, a, r);
    KP(sp_nr)<<<gnr, 128, 0, st>>>(F, a, r);
}

}  // namespace

// The launch sequence of one batched flash (the schedule of flash_phased.cuh)
// with the context's launch shape. marks (may be null): two events recorded
// on the stream just before and just after the split-restart kernel, so that
// a caller can time the sequence's parts. With PH_EARLY in a.opts, the
// split round and restarts of the cells that strict trial k >= 1 finds
// unstable run on side->s[k] (on `st` itself when side is null), forked
// after trial k and joined before the finalize; trial 0's (most of the
// split work) stay in round 0 on `st` after the last trial, so that its
// persistent kernels do not hold the SMs while trials 1-3 run.
cudaError_t OCPF_CAT(launch_phased_nc, OCPF_NC)(const FluidConst& F, const PhasedArgs& a, const LaunchTune& t,
                                                cudaStream_t st, const cudaEvent_t* marks, const SideStreams* side)
{
    static int sms = 0, occ_s01 = 0, occ_sta = 0, occ_sp = 0, occ_sta32 = 0, occ_spnr = 0, occ_stnr = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        occ_s01   = OCPF_CAT(persistent_grid_, OCPF_NC)((const void*)KP(s01_ssm), 1, 100);
        occ_sta   = OCPF_CAT(persistent_grid_, OCPF_NC)((const void*)KP(sta_ssm), 1, 100);
        occ_sp    = OCPF_CAT(persistent_grid_, OCPF_NC)((const void*)KP(sp_ssm), 1, 100);
        occ_sta32 = OCPF_CAT(persistent_grid_, OCPF_NC)((const void*)KP(sta_ssm32), 1, 100);
        occ_spnr  = OCPF_CAT(persistent_grid_, OCPF_NC)((const void*)KP(sp_nr), 1, 100);
        occ_stnr  = OCPF_CAT(persistent_grid_, OCPF_NC)((const void*)KP(sta_nr), 1, 100);
        cudaFuncSetAttribute(KP(learn), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(LearnSmem));
    }
    const int  pct  = t.persist_pct > 0 && t.persist_pct <= 100 ? t.persist_pct : 100;
    auto       grid = [&](int occ) { return sms * std::max(1, (occ * pct + 99) / 100); };
    const int  g_s01 = grid(occ_s01), g_sta = grid(occ_sta), g_sp = grid(occ_sp), g_sta32 = grid(occ_sta32),
              g_spnr = grid(occ_spnr), g_stnr = grid(occ_stnr);
    const int     bp    = (t.block == 64) ? 64 : 128;  // thread-per-item kernels
    const int64_t need  = (a.count + bp - 1) / bp;
    const int     gcell = (int)(need < (int64_t)sms * 8 * (128 / bp) ? need : (int64_t)sms * 8 * (128 / bp));
    const int     gp    = gcell;
    const bool    mixed = (a.opts & PH_MIXED) != 0;
    cudaMemsetAsync(a.L.ctr, 0, sizeof(uint32_t) * 2 * L_COUNT, st);
    KP(init)<<<gcell, bp, 0, st>>>(F, a);
    const bool defer = (a.opts & PH_DEFER) != 0;
    if (a.opts & PH_LEARN) {
        // learned initialiser: predicted-unstable fresh cells split first
        // (with PH_DEFER their split waits until trial 1 has run, below)
        const int gl = (int)std::min<int64_t>((a.count + LEARN_TILE - 1) / LEARN_TILE, (int64_t)sms * 4);
        KP(learn)<<<gl, 128, sizeof(LearnSmem), st>>>(F, a);
        if (!defer) OCPF_CAT(split_round_, OCPF_NC)(F, a, st, LEARN_ROUND, gp, bp, g_sp, g_spnr);
    }
    for (int k = 0; k < 2; k++) {
        KP(s01_prep)<<<gp, bp, 0, st>>>(F, a, k);
        KP(s01_ssm)<<<g_s01, 128, 0, st>>>(F, a, k);
        KP(s01_end)<<<gp, bp, 0, st>>>(F, a, k);
    }
    // strict stability trial k of the pass whose arguments are A (its lists:
    // the main set, or with A.sdup the deferred fallback pass's own set)
    auto trial = [&](const PhasedArgs& A, cudaStream_t s, int k) {
        const bool d  = A.sdup != 0;
        const int  sa = stab_list(L_STA_0 + k, d), na = stab_list(L_NRSTA_0 + k, d);
        const int  sc = stab_list(L_STC_0 + k, d), nc = stab_list(L_NRSTC_0 + k, d);
        KP(sta_prep)<<<gp, bp, 0, s>>>(F, A, k);
        if (mixed) {
            // FP32 substitution, FP64 end point and Newton; trials whose
            // Newton fails continue in FP64, then Newton again
            KP(sta_ssm32)<<<g_sta32, 128, 0, s>>>(F, A, k);
            KP(sta_verdict)<<<gp, bp, 0, s>>>(F, A, k, sa, na, true);
            KP(sta_nr)<<<g_stnr, 128, 0, s>>>(F, A, k, na, sc);
            KP(sta_ssm)<<<g_sta, 128, 0, s>>>(F, A, sc);
            KP(sta_verdict)<<<gp, bp, 0, s>>>(F, A, k, sc, nc, false);
            KP(sta_nr)<<<g_stnr, 128, 0, s>>>(F, A, k, nc, -1);
        } else {
            KP(sta_ssm)<<<g_sta, 128, 0, s>>>(F, A, sa);
            KP(sta_verdict)<<<gp, bp, 0, s>>>(F, A, k, sa, na, false);
            KP(sta_nr)<<<g_stnr, 128, 0, s>>>(F, A, k, na, -1);
        }
    };
    for (int k = 0; k < 4; k++) {
        trial(a, st, k);
        if ((a.opts & PH_EARLY) && k > 0) {
            // trial k's unstable cells: split and restarts beside the later trials
            cudaStream_t ss = st;
            if (side) {
                ss = side->s[k];
                cudaEventRecord(side->fork[k], st);
                cudaStreamWaitEvent(ss, side->fork[k], 0);
            }
            OCPF_CAT(split_round_, OCPF_NC)(F, a, ss, TRIAL_ROUND0 + k, gp, bp, g_sp, g_spnr);
            if (t.slow_threads)
                KP(slow_thread)<<<gp, bp, 0, ss>>>(F, a, L_SLOW_T0 + k);
            else
                KP(slow)<<<gp, 128, 0, ss>>>(F, a, L_SLOW_T0 + k);
            if (side) cudaEventRecord(side->join[k], ss);
        }
        if (defer && k == 1) {
            // the learned round, off the path of trials 0 and 1 (whose
            // restart chains are the call's longest), on side stream 0 at the
            // default priority; then the strict test of the cells whose
            // learned split it did not keep, on lists of their own, all four
            // trials; their unstable cells join split round 0
            cudaStream_t ss = st;
            if (side) {
                ss = side->s[0];
                cudaEventRecord(side->fork[0], st);
                cudaStreamWaitEvent(ss, side->fork[0], 0);
            }
            OCPF_CAT(split_round_, OCPF_NC)(F, a, ss, LEARN_ROUND, gp, bp, g_sp, g_spnr);
            PhasedArgs b = a;
            b.sdup       = 1;
            b.opts &= ~(PH_EARLY | PH_DEFER);
            for (int kk = 0; kk < 4; kk++) trial(b, ss, kk);
            if (side) cudaEventRecord(side->join[0], ss);
        }
    }
    if (defer && side) cudaStreamWaitEvent(st, side->join[0], 0);
    for (int r = 0; r < SPLIT_ROUNDS; r++) OCPF_CAT(split_round_, OCPF_NC)(F, a, st, r, gp, bp, g_sp, g_spnr);
    if (marks) cudaEventRecord(marks[0], st);
    if (t.slow_threads)
        KP(slow_thread)<<<gp, bp, 0, st>>>(F, a, L_SLOW);
    else
        KP(slow)<<<gp, 128, 0, st>>>(F, a, L_SLOW);
    if (marks) cudaEventRecord(marks[1], st);
    if ((a.opts & PH_EARLY) && side)
        for (int k = 1; k < 4; k++) cudaStreamWaitEvent(st, side->join[k], 0);
    if (a.tail.mode & FM_FIMN)
        KP(finalize_fimn)<<<gcell, bp, 0, st>>>(F, a);
    else
        KP(finalize)<<<gcell, bp, 0, st>>>(F, a);
    return cudaGetLastError();
}

int OCPF_CAT(phased_state_doubles_nc, OCPF_NC)() { return SF<kNC>::COUNT; }

}  // namespace ocpf

#undef KP
