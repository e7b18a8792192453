// flash_phased.cuh -- the batched form of the FIM flash, organised by phase.
//
// A one-thread-per-cell flash runs at ~20 % SIMT efficiency: the cells of a
// warp need 2 to 400+ fugacity evaluations, take different branches, and the
// fully inlined flash overflows the instruction cache. Here the flash of a
// batch is a fixed sequence of small kernels; cells move between them through
// device-side lists (appended with atomics, so each kernel sees only the
// cells that need it):
//
//   init          every cell: inputs, flash type, fugacity of z; route
//   S01 round k   relaxed stability trial k (StableSSM01), k = 0, 1:
//                 prep -> persistent SSM -> end-of-trial logic
//   strict round k (StableSSM trial k + StableNR), k = 0..3:
//                 prep -> persistent SSM -> verdict -> Newton
//   split         (SplitSSM2 + SplitNR, first try):
//                 prep -> persistent SSM -> Newton start -> persistent Newton
//   restarts      cells whose split restarts: the rest of PhaseSplit, one
//                 warp per cell (flash_warp.cuh)
//   finalize      every cell: properties, derivatives, copy-out
//
// The persistent SSM kernels are where the time goes. Their loop body is one
// fugacity evaluation plus an O(NC) update, the same for every lane; a lane
// whose trial ends stores it and loads the next prepared item. Everything
// irregular (trial set-up, Newton steps, routing) runs in the one-thread-per-
// item kernels around them.
//
// Every cell takes exactly the reference's steps in the reference's order
// (src/MixtureComp.cpp:1279-2166); only the schedule across cells changes.
#pragma once

#include "flash_fim.cuh"

namespace ocpf {

// ------------------------------------------------------------ cell state
// Per-cell state kept across the phase kernels, structure of arrays with
// field stride `cap`. Double fields first (ids below), then int fields.
template <int NC>
struct SF {  // double field ids
    enum : int {
        ePEC = 0, nu0, nu1, Aj0, Aj1, Bj0, Bj1, Zj0, Zj1,
        x0, x1 = x0 + NC, n0 = x1 + NC, n1 = n0 + NC,          // finalize reads up to here
        Yt = n1 + NC, SeSSM, rtSSMSTA, rtNRSTA, rtSSMSP, rtNRSP, SeSP, Stol, eNR, eNR0, Asta, Bsta, Zsta,
        phiZ, Y = phiZ + NC, phiS = Y + NC, Ks = phiS + NC, phi0 = Ks + NC, phi1 = phi0 + NC,
        di = phi1 + NC, sA = di + NC, Bi = sA + NC,
        lnY = Bi + NC, lndi = lnY + NC,  // mixed form: FP32 stability trial in log form
        COUNT = lndi + NC
    };
};
// int fields
enum : int { IF_META = 0, IF_STATUS, IF_IT0, IF_IT1, IF_IT2, IF_IT3, IF_IT4, IF_MAXIT, IF_GUARD, IF_COUNT };

// meta bits
constexpr uint32_t M_NP_MASK   = 0xF;     // hydrocarbon phase count
constexpr int      M_FTYPE_SH  = 4;       // 2 bits
constexpr uint32_t M_FLAGSKIP  = 1u << 8;
constexpr uint32_t M_C_SSMSTA  = 1u << 9;   // convergence flags of the four solvers
constexpr uint32_t M_C_NRSTA   = 1u << 10;
constexpr uint32_t M_C_SSMSP   = 1u << 11;
constexpr uint32_t M_C_NRSP    = 1u << 12;
constexpr uint32_t M_RESTART   = 1u << 13;  // next split SSM is a restart
constexpr uint32_t M_STAB_RES  = 1u << 14;  // last stability verdict: stable
constexpr uint32_t M_NRFLAG    = 1u << 15;  // flag of the last StableNR
constexpr uint32_t M_SPPHASE   = 1u << 16;  // split loop: after a restart
constexpr uint32_t M_LEARNED   = 1u << 17;  // split started from the learned initialiser's K
constexpr uint32_t M_STC       = 1u << 18;  // mixed form: stability trial continued in FP64

template <int NC>
constexpr int state_doubles() { return SF<NC>::COUNT; }
inline size_t state_bytes_per_cell(int nc_doubles) { return 8 * (size_t)nc_doubles + 4 * (size_t)IF_COUNT; }

struct StateBuf {
    double*  d;  // [COUNT][cap]
    int32_t* i;  // [IF_COUNT][cap]
    int64_t  cap;
    __device__ __forceinline__ double& D(int f, int64_t c) const { return d[(int64_t)f * cap + c]; }
    __device__ __forceinline__ int32_t& I(int f, int64_t c) const { return i[(int64_t)f * cap + c]; }
};

// ------------------------------------------------------------------ lists
// Split round 0 is PhaseSplit's first try; the cells that restart go on to
// the warp-per-cell path (L_SLOW). Round LEARN_ROUND is the learned
// initialiser's split of fresh cells (before any stability test), whose
// failures fall back to the stability test.
enum ListId : int {
    L_S01_0 = 0, L_S01_1,
    L_STA_0, L_STA_1, L_STA_2, L_STA_3,
    L_NRSTA_0, L_NRSTA_1, L_NRSTA_2, L_NRSTA_3,
    L_SP_0, L_SP_LEARN, L_SP_T0, L_SP_T1, L_SP_T2, L_SP_T3,
    L_SPNR_0, L_SPNR_LEARN, L_SPNR_T0, L_SPNR_T1, L_SPNR_T2, L_SPNR_T3,
    L_SLOW, L_SLOW_T0, L_SLOW_T1, L_SLOW_T2, L_SLOW_T3,
    L_FRESH,  // fresh cells awaiting the learned initialiser
    // mixed form: stability trials whose Newton polish failed from the FP32
    // end point, continued by FP64 substitution, and their Newton step
    L_STC_0, L_STC_1, L_STC_2, L_STC_3,
    L_NRSTC_0, L_NRSTC_1, L_NRSTC_2, L_NRSTC_3,
    // with PH_DEFER: the strict test of the cells whose learned split was
    // not kept runs as a pass of its own, on a duplicate of the 16
    // stability lists above (stab_list)
    L_SDUP_0, L_SDUP_LAST = L_SDUP_0 + 15,
    L_COUNT
};
// A restart runs 200 or 400 substitution steps on one cell: on the
// thread-per-cell kernels that is a single busy lane per warp, so every
// restart takes the warp-per-cell path.
constexpr int SPLIT_ROUNDS = 1;
constexpr int LEARN_ROUND  = SPLIT_ROUNDS;
// With PH_EARLY, the fresh cells that strict stability trial k >= 1 finds
// unstable split in round TRIAL_ROUND0 + k (lists L_SP_Tk, L_SPNR_Tk) and
// restart from L_SLOW_Tk, on a side stream forked after trial k, while the
// later trials and round 0 run: these few cells, whose stability was the
// hardest to decide and whose restart chains are the longest, start their
// split as soon as their own trial has decided. The work of each cell, and
// its arithmetic, are the same in either schedule.
constexpr int TRIAL_ROUND0 = LEARN_ROUND + 1;
static_assert(L_SP_0 + LEARN_ROUND == L_SP_LEARN && L_SPNR_0 + LEARN_ROUND == L_SPNR_LEARN, "list order");
static_assert(L_SP_0 + TRIAL_ROUND0 == L_SP_T0 && L_SPNR_0 + TRIAL_ROUND0 == L_SPNR_T0 && L_SLOW + 1 == L_SLOW_T0,
              "list order");

struct Lists {
    int32_t*  items;  // [L_COUNT][cap]
    uint32_t* ctr;    // [L_COUNT][2]: length, consumer head
    int64_t   cap;
    __device__ __forceinline__ void push(int id, int32_t cell) const
    {
        const uint32_t at         = atomicAdd(&ctr[2 * id], 1u);
        items[(int64_t)id * cap + at] = cell;
    }
    __device__ __forceinline__ uint32_t len(int id) const { return *(volatile uint32_t*)&ctr[2 * id]; }
    __device__ __forceinline__ int32_t item(int id, uint32_t k) const { return items[(int64_t)id * cap + k]; }
    // next item for a persistent consumer, or -1
    __device__ __forceinline__ int32_t take(int id, uint32_t n) const
    {
        const uint32_t k = atomicAdd(&ctr[2 * id + 1], 1u);
        return k < n ? item(id, k) : -1;
    }
};

// Launch shape of a batched sequence, chosen per context by the autotuner
// (ocpf_autotune): threads per block of the thread-per-item kernels (64 or
// 128; every kernel is built for at most 128), the resident blocks per SM
// of the persistent kernels as a percentage of what their registers allow,
// and the restart path: one warp per cell (0) or one thread per cell (1).
// Block size and persistent grid change only which thread takes which
// cell, never a cell's arithmetic.
struct LaunchTune {
    int32_t block;
    int32_t persist_pct;
    int32_t slow_threads;
    int32_t pad;
};
constexpr LaunchTune kDefaultTune{128, 100, 0, 0};

// PhasedArgs::opts bits
constexpr uint32_t PH_MIXED = 1u;  // FP32 successive substitution (flash_mixed.cuh)
constexpr uint32_t PH_LEARN = 2u;  // learned initialiser for fresh cells (flash_learned.cuh)
constexpr uint32_t PH_EARLY = 4u;  // split each strict trial's unstable cells on its own side stream
constexpr uint32_t PH_DEFER = 8u;  // learned round after trial 1, beside the main sequence (PH_EARLY)

// Stability list `id` (L_STA_k, L_NRSTA_k, L_STC_k or L_NRSTC_k) of the main
// pass, or with `dup` of the deferred learned round's fallback pass.
__host__ __device__ constexpr int stab_list(int id, bool dup)
{
    return !dup ? id : (id < L_STC_0 ? L_SDUP_0 + (id - L_STA_0) : L_SDUP_0 + 8 + (id - L_STC_0));
}
static_assert(L_NRSTA_3 == L_STA_0 + 7 && L_NRSTC_3 == L_STC_0 + 7, "stability lists in two runs of eight");

// The side streams of the PH_EARLY schedule: trial k's split round and
// restarts run on s[k], after fork[k] is recorded on the call's stream; the
// call's stream waits for join[k] before the finalize.
struct SideStreams {
    cudaStream_t s[4];
    cudaEvent_t  fork[4], join[4];
};

struct PhasedArgs {
    int64_t      count, stride;
    uint32_t     opts;
    // Block partition of a launch shared by several regions (flash_multi):
    // this region's blocks are those with blockIdx.x % vparts == vpart, and
    // its grid-stride loops see block blockIdx.x / vparts of a grid of
    // gridDim.x / vparts. vparts <= 1: the whole launch is this region's.
    int32_t      vpart, vparts;
    // the pass's stability lists: 0 the main set, 1 the duplicate set of the
    // deferred learned round's fallback pass (stab_list)
    int32_t      sdup, pad_sdup;
    const float* mlp;  // learned initialiser parameters (PH_LEARN)
    FlashTail    tail; // entry point (FlashFIM, FlashIMPEC, InitFlash*) and its extra arrays
    ocpf_fim_in  in;
    ocpf_skip    sk;
    ocpf_fim_out out;
    StateBuf     S;
    Lists        L;
};

// The region's block index and block count within its launch (PhasedArgs::vpart).
__device__ __forceinline__ uint32_t vblock(const PhasedArgs& a)
{
    return a.vparts > 1 ? blockIdx.x / (uint32_t)a.vparts : blockIdx.x;
}
__device__ __forceinline__ uint32_t vgrid(const PhasedArgs& a)
{
    return a.vparts > 1 ? gridDim.x / (uint32_t)a.vparts : gridDim.x;
}

// z of cell c, bit for bit as FimCell::load_inputs forms it: Ni / Nh
// (InitPTN), or in the initialisation the given mole fractions (InitPTZ).
// Returns Nh (1 in the initialisation, where the tail sets it).
template <int NC>
__device__ __forceinline__ double load_z(const PhasedArgs& a, int64_t c, double* z)
{
    const int64_t N = a.stride;
    if (a.tail.mode & FM_INIT) {
#pragma unroll
        for (int i = 0; i < NC; i++) z[i] = a.in.Ni[(int64_t)i * N + c];
        return 1;
    }
    double Ni[NC], Nh = 0;
#pragma unroll
    for (int i = 0; i < NC; i++) {
        Ni[i] = a.in.Ni[(int64_t)i * N + c];
        Nh += fabs(Ni[i]);
    }
#pragma unroll
    for (int i = 0; i < NC; i++) z[i] = Ni[i] / Nh;
    return Nh;
}

// lNP of cell c: the last step's hydrocarbon phase count (none in the
// initialisation).
__device__ __forceinline__ int last_hc_np(const PhasedArgs& a, int64_t c)
{
    if (a.tail.mode & FM_INIT) return 0;
    const uint32_t lastNP = a.in.lastNP[c];
    return lastNP > 0 ? (int)lastNP - 1 : 0;
}

// Reads P, T and z of cell c into a CellFlash and computes Ai, Bi.
template <int NC>
__device__ __forceinline__ void load_ptz(CellFlash<NC>& f, const PhasedArgs& a, int64_t c)
{
    f.P  = a.in.P[c];
    f.T  = a.in.T[c] + CONV5;
    f.Nh = load_z<NC>(a, c, f.zi);
    f.cal_ai_bi();
}

// Bookkeeping of one cell that the thread-per-item kernels load and store.
template <int NC>
__device__ __forceinline__ void load_book(CellFlash<NC>& f, const StateBuf& S, int64_t c, uint32_t& meta)
{
    using F_ = SF<NC>;
    meta             = (uint32_t)S.I(IF_META, c);
    f.NP             = (int)(meta & M_NP_MASK);
    f.ftype          = (int)((meta >> M_FTYPE_SH) & 3);
    f.flagSkip       = (meta & M_FLAGSKIP) != 0;
    f.ssmsta_conflag = (meta & M_C_SSMSTA) != 0;
    f.nrsta_conflag  = (meta & M_C_NRSTA) != 0;
    f.ssmsp_conflag  = (meta & M_C_SSMSP) != 0;
    f.nrsp_conflag   = (meta & M_C_NRSP) != 0;
    f.status         = (uint16_t)S.I(IF_STATUS, c);
    f.it_ssmsta      = S.I(IF_IT0, c);
    f.it_nrsta       = S.I(IF_IT1, c);
    f.it_ssmsp       = S.I(IF_IT2, c);
    f.it_nrsp        = S.I(IF_IT3, c);
    f.it_rr          = S.I(IF_IT4, c);
    f.ssmsta_realTol = S.D(F_::rtSSMSTA, c);
    f.nrsta_realTol  = S.D(F_::rtNRSTA, c);
    f.ssmsp_realTol  = S.D(F_::rtSSMSP, c);
    f.nrsp_realTol   = S.D(F_::rtNRSP, c);
    f.Yt             = S.D(F_::Yt, c);
}

template <int NC>
__device__ __forceinline__ void store_book(const CellFlash<NC>& f, const StateBuf& S, int64_t c, uint32_t meta)
{
    using F_ = SF<NC>;
    meta &= ~(M_NP_MASK | M_FLAGSKIP | M_C_SSMSTA | M_C_NRSTA | M_C_SSMSP | M_C_NRSP | (3u << M_FTYPE_SH));
    meta |= (uint32_t)f.NP | ((uint32_t)f.ftype << M_FTYPE_SH) | (f.flagSkip ? M_FLAGSKIP : 0u) |
            (f.ssmsta_conflag ? M_C_SSMSTA : 0u) | (f.nrsta_conflag ? M_C_NRSTA : 0u) |
            (f.ssmsp_conflag ? M_C_SSMSP : 0u) | (f.nrsp_conflag ? M_C_NRSP : 0u);
    S.I(IF_META, c)         = (int32_t)meta;
    S.I(IF_STATUS, c)       = f.status;
    S.I(IF_IT0, c)          = f.it_ssmsta;
    S.I(IF_IT1, c)          = f.it_nrsta;
    S.I(IF_IT2, c)          = f.it_ssmsp;
    S.I(IF_IT3, c)          = f.it_nrsp;
    S.I(IF_IT4, c)          = f.it_rr;
    S.D(F_::rtSSMSTA, c)    = f.ssmsta_realTol;
    S.D(F_::rtNRSTA, c)     = f.nrsta_realTol;
    S.D(F_::rtSSMSP, c)     = f.ssmsp_realTol;
    S.D(F_::rtNRSP, c)      = f.nrsp_realTol;
    S.D(F_::Yt, c)          = f.Yt;
}

// Equilibrium of a single-phase cell for the finalize kernel: nu0 = 1 with
// x0 = z and the mixture a, b, Z of phase 0. init stores x0 = z for every
// cell; only kernels that overwrote x0 (the split) pass write_x = true and
// must have f.zi loaded.
template <int NC>
__device__ __forceinline__ void store_single_phase(const CellFlash<NC>& f, const StateBuf& S, int64_t c,
                                                   bool write_x = false)
{
    using F_        = SF<NC>;
    S.D(F_::nu0, c) = 1.0;
    if (write_x) {
#pragma unroll
        for (int i = 0; i < NC; i++) S.D(F_::x0 + i, c) = f.zi[i];
    }
}

template <int NC>
__device__ __forceinline__ void store_split(const CellFlash<NC>& f, const StateBuf& S, int64_t c)
{
    using F_        = SF<NC>;
    S.D(F_::nu0, c) = f.nu[0];
    S.D(F_::nu1, c) = f.nu[1];
    S.D(F_::Aj0, c) = f.Aj[0];
    S.D(F_::Aj1, c) = f.Aj[1];
    S.D(F_::Bj0, c) = f.Bj[0];
    S.D(F_::Bj1, c) = f.Bj[1];
    S.D(F_::Zj0, c) = f.Zj[0];
    S.D(F_::Zj1, c) = f.Zj[1];
#pragma unroll
    for (int i = 0; i < NC; i++) {
        S.D(F_::x0 + i, c)   = f.x[0][i];
        S.D(F_::x1 + i, c)   = f.x[1][i];
        S.D(F_::n0 + i, c)   = f.n[0][i];
        S.D(F_::n1 + i, c)   = f.n[1][i];
        S.D(F_::phi0 + i, c) = f.phi[0][i];
        S.D(F_::phi1 + i, c) = f.phi[1][i];
    }
}

template <int NC>
__device__ __forceinline__ void load_split(CellFlash<NC>& f, const StateBuf& S, int64_t c)
{
    using F_ = SF<NC>;
    f.nu[0]  = S.D(F_::nu0, c);
    f.nu[1]  = S.D(F_::nu1, c);
    f.Aj[0]  = S.D(F_::Aj0, c);
    f.Aj[1]  = S.D(F_::Aj1, c);
    f.Bj[0]  = S.D(F_::Bj0, c);
    f.Bj[1]  = S.D(F_::Bj1, c);
    f.Zj[0]  = S.D(F_::Zj0, c);
    f.Zj[1]  = S.D(F_::Zj1, c);
#pragma unroll
    for (int i = 0; i < NC; i++) {
        f.x[0][i]   = S.D(F_::x0 + i, c);
        f.x[1][i]   = S.D(F_::x1 + i, c);
        f.n[0][i]   = S.D(F_::n0 + i, c);
        f.n[1][i]   = S.D(F_::n1 + i, c);
        f.phi[0][i] = S.D(F_::phi0 + i, c);
        f.phi[1][i] = S.D(F_::phi1 + i, c);
        f.fug[0][i] = f.phi[0][i] * f.x[0][i] * f.P;
        f.fug[1][i] = f.phi[1][i] * f.x[1][i] * f.P;
        f.Ks[i]     = S.D(F_::Ks + i, c);
    }
}

// PhaseEquilibrium's ePEC and the final flagSkip of a finished cell
// (src/MixtureComp.cpp:1297-1316, 1339-1345).
template <int NC>
__device__ __forceinline__ void finish_epec(CellFlash<NC>& f)
{
    if (f.ftype == 1) {
        f.ePEC = 0.0;
        return;
    }
    if (f.ftype == 0 && f.NP > 1) f.flagSkip = false;
    if (f.ftype == 0 && f.NP == 1)
        f.ePEC = f.nrsta_conflag ? f.nrsta_realTol : (f.ssmsta_conflag ? f.ssmsta_realTol : 1e8);
    else
        f.ePEC = f.nrsp_conflag ? f.nrsp_realTol : (f.ssmsp_conflag ? f.ssmsp_realTol : 1e8);
}

}  // namespace ocpf
