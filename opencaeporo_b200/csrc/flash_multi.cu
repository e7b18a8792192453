// flash_multi.cu -- the launch sequence of the multi-region batched flash
// (flash_multi.cuh): the schedule of flash_phased.cuh with every step one
// kernel over all regions.
#include <algorithm>

#include "flash_multi.cuh"

namespace ocpf {

namespace {

cudaError_t step(int s, const MultiFluid& MF, const MultiArgs& M, unsigned grid, int block, size_t smem,
                 cudaStream_t st, int i0 = 0, int i1 = 0, int i2 = 0, bool b0 = false)
{
    if (grid == 0) return cudaSuccess;
    if (s <= MS_LEARN) return multi_step_a(s, MF, M, grid, block, smem, st, i0, i1, i2, b0);
    if (s <= MS_STA_NR) return multi_step_b(s, MF, M, grid, block, smem, st, i0, i1, i2, b0);
    if (s <= MS_SP_NR) return multi_step_c(s, MF, M, grid, block, smem, st, i0, i1, i2, b0);
    return multi_step_d(s, MF, M, grid, block, smem, st, i0, i1, i2, b0);
}

int occupancy(int s)
{
    if (s <= MS_LEARN) return multi_occupancy_a(s);
    if (s <= MS_STA_NR) return multi_occupancy_b(s);
    if (s <= MS_SP_NR) return multi_occupancy_c(s);
    return multi_occupancy_d(s);
}

}  // namespace

cudaError_t launch_phased_multi(const MultiFluid& MF, const MultiArgs& M, const LaunchTune& t, cudaStream_t st)
{
    static int sms = 0, o_s01 = 0, o_sta = 0, o_sta32 = 0, o_stnr = 0, o_sp = 0, o_spnr = 0;
    if (M.n < 1 || M.n > MULTI_MAX) return cudaErrorInvalidValue;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        o_s01   = occupancy(MS_S01_SSM);
        o_sta   = occupancy(MS_STA_SSM);
        o_sta32 = occupancy(MS_STA_SSM32);
        o_stnr  = occupancy(MS_STA_NR);
        o_sp    = occupancy(MS_SP_SSM);
        o_spnr  = occupancy(MS_SP_NR);
    }
    const int n   = M.n;
    const int pct = t.persist_pct > 0 && t.persist_pct <= 100 ? t.persist_pct : 100;
    auto pgrid = [&](int occ) { return (unsigned)(sms * std::max(1, (occ * pct + 99) / 100)); };
    const unsigned g_s01 = pgrid(o_s01), g_sta = pgrid(o_sta), g_sta32 = pgrid(o_sta32), g_stnr = pgrid(o_stnr),
                   g_sp = pgrid(o_sp), g_spnr = pgrid(o_spnr);
    int64_t maxc  = 0;
    bool    learn = false;
    for (int r = 0; r < n; r++) {
        maxc = std::max(maxc, M.a[r].count);
        learn |= (M.a[r].opts & PH_LEARN) != 0;
    }
    // thread-per-item kernels: every region gets the blocks its largest
    // batch would get alone, so the grid is n times that
    const int     bp   = (t.block == 64) ? 64 : 128;
    const int64_t capb = (int64_t)sms * 8 * (128 / bp);
    const unsigned gp  = (unsigned)(n * std::min<int64_t>((maxc + bp - 1) / bp, capb));
    const unsigned gw  = (unsigned)(n * std::min<int64_t>((maxc + 127) / 128, (int64_t)sms * 8));
    const bool mixed = (M.a[0].opts & PH_MIXED) != 0;
    for (int r = 0; r < n; r++) cudaMemsetAsync(M.a[r].L.ctr, 0, sizeof(uint32_t) * 2 * L_COUNT, st);
    auto split_round = [&](int r) {
        step(MS_SP_PREP, MF, M, gp, bp, 0, st, r);
        step(MS_SP_SSM, MF, M, g_sp, 128, 0, st, r);
        step(MS_SP_NRINIT, MF, M, gp, bp, 0, st, r);
        step(MS_SP_NR, MF, M, g_spnr, 128, 0, st, r);
    };
    step(MS_INIT, MF, M, gp, bp, 0, st);
    if (learn) {
        const unsigned gl = (unsigned)(n * std::min<int64_t>((maxc + LEARN_TILE - 1) / LEARN_TILE, (int64_t)sms * 4));
        step(MS_LEARN, MF, M, gl, 128, sizeof(LearnSmem), st);
        split_round(LEARN_ROUND);
    }
    for (int k = 0; k < 2; k++) {
        step(MS_S01_PREP, MF, M, gp, bp, 0, st, k);
        step(MS_S01_SSM, MF, M, g_s01, 128, 0, st, k);
        step(MS_S01_END, MF, M, gp, bp, 0, st, k);
    }
    for (int k = 0; k < 4; k++) {
        step(MS_STA_PREP, MF, M, gp, bp, 0, st, k);
        if (mixed) {
            step(MS_STA_SSM32, MF, M, g_sta32, 128, 0, st, k);
            step(MS_STA_VERDICT, MF, M, gp, bp, 0, st, k, L_STA_0 + k, L_NRSTA_0 + k, true);
            step(MS_STA_NR, MF, M, g_stnr, 128, 0, st, k, L_NRSTA_0 + k, L_STC_0 + k);
            step(MS_STA_SSM, MF, M, g_sta, 128, 0, st, L_STC_0 + k);
            step(MS_STA_VERDICT, MF, M, gp, bp, 0, st, k, L_STC_0 + k, L_NRSTC_0 + k, false);
            step(MS_STA_NR, MF, M, g_stnr, 128, 0, st, k, L_NRSTC_0 + k, -1);
        } else {
            step(MS_STA_SSM, MF, M, g_sta, 128, 0, st, L_STA_0 + k);
            step(MS_STA_VERDICT, MF, M, gp, bp, 0, st, k, L_STA_0 + k, L_NRSTA_0 + k, false);
            step(MS_STA_NR, MF, M, g_stnr, 128, 0, st, k, L_NRSTA_0 + k, -1);
        }
    }
    for (int r = 0; r < SPLIT_ROUNDS; r++) split_round(r);
    if (t.slow_threads)
        step(MS_SLOW_THREAD, MF, M, gp, bp, 0, st);
    else
        step(MS_SLOW, MF, M, gw, 128, 0, st);
    step((M.a[0].tail.mode & FM_FIMN) ? MS_FINALIZE_FIMN : MS_FINALIZE, MF, M, gp, bp, 0, st);
    return cudaGetLastError();
}

}  // namespace ocpf
