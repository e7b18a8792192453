// flash_phased_kernels.cuh -- bodies of the phase kernels of the batched
// FIM flash (see flash_phased.cuh for the schedule).
#pragma once

#include "flash_phased.cuh"
#include "flash_warp.cuh"

namespace ocpf {

// Thread-per-item kernels walk their list with a grid-stride loop: the grid
// is fixed at launch (the list length is only known on the device).
#define OCPF_FOR_ITEMS(A, LIST, c)                                                                   \
    for (uint32_t _k = vblock(A) * blockDim.x + threadIdx.x, _n = (A).L.len(LIST); _k < _n;        \
         _k += vgrid(A) * blockDim.x)                                                                \
        if (const int64_t c = (A).L.item(LIST, _k); true)

// ------------------------------------------------------------------ init
// FlashFIM up to PhaseEquilibrium's first fork (src/MixtureComp.cpp:494-515,
// 1279-1293, 1319-1337): inputs, flash type, Ai/Bi, and the mixture (and for
// ftype 0 the fugacity coefficients) of z. Routes the cell to the relaxed or
// strict stability test, to the split, or finishes it (ftype 1).
template <int NC>
__device__ void init_body(const FluidConst& F, const PhasedArgs& a)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    for (int64_t c = vblock(a) * (int64_t)blockDim.x + threadIdx.x; c < a.count;
         c += (int64_t)vgrid(a) * blockDim.x) {
        FimCell<NC> f(F);
        f.load_inputs(c, a.stride, a.in, a.sk, a.tail);
        f.cal_ai_bi();
        uint32_t meta = 0;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            S.D(F_::sA + i, c) = f.sA[i];
            S.D(F_::Bi + i, c) = f.Bi[i];
        }
        S.I(IF_GUARD, c) = 0;
        store_single_phase(f, S, c, true);  // x0 = z until a split replaces it
        if (f.ftype == 0 || f.ftype == 1) {
            f.flagSkip = true;
            f.NP       = 1;
            double phiz[NC];
            f.fug_phi(f.zi, phiz, nullptr, f.Aj[0], f.Bj[0], f.Zj[0]);
            S.D(F_::Aj0, c) = f.Aj[0];
            S.D(F_::Bj0, c) = f.Bj[0];
            S.D(F_::Zj0, c) = f.Zj[0];
            if (f.ftype == 1) {
                finish_epec(f);
                S.D(F_::ePEC, c) = f.ePEC;
                store_single_phase(f, S, c);
            } else {
#pragma unroll
                for (int i = 0; i < NC; i++) S.D(F_::phiZ + i, c) = phiz[i];
                a.L.push(f.lNP == 0 ? ((a.opts & PH_LEARN) ? L_FRESH : L_STA_0) : L_S01_0, (int32_t)c);
            }
        } else {
            f.flagSkip = false;
            f.NP       = 2;
            f.Yt       = 1.01;
            a.L.push(L_SP_0, (int32_t)c);
        }
        store_book(f, S, c, meta);
    }
}

// ------------------------------------------------------ strict stability
// Trial k set-up of StableSSM (src/MixtureComp.cpp:1514-1524): Y = z / Kw_k,
// normalised, and d_i = phi_z,i z_i.
template <int NC>
__device__ void sta_prep_body(const FluidConst& F, const PhasedArgs& a, int k)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    OCPF_FOR_ITEMS(a, stab_list(L_STA_0 + k, a.sdup != 0), c)
    {
        CellFlash<NC> f(F);
        load_ptz(f, a, c);
        f.cal_kwilson();
        double Yt = 0, Y[NC];
#pragma unroll
        for (int i = 0; i < NC; i++) {
            Y[i] = f.zi[i] / f.kw(k, i);
            Yt += Y[i];
        }
        const double r = 1 / Yt;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            S.D(F_::Y + i, c)  = Y[i] * r;
            S.D(F_::di + i, c) = S.D(F_::phiZ + i, c) * f.zi[i];
        }
        S.D(F_::Yt, c) = Yt;
        if (a.opts & PH_MIXED) {  // the FP32 trial's start in log form
#pragma unroll
            for (int i = 0; i < NC; i++) {
                S.D(F_::lnY + i, c)  = log(Y[i] * r);
                S.D(F_::lndi + i, c) = log(S.D(F_::di + i, c));
            }
        }
        S.I(IF_MAXIT, c) = F.ssmsta_maxit;
    }
}

// The successive substitution of one StableSSM trial (src/MixtureComp.cpp:
// 1525-1564) on a persistent grid. Per lane: Y (next composition), d, the
// mixture terms, Yt and the iteration count. Each loop turn is one fugacity
// evaluation and an O(NC) update for every active lane.
template <int NC>
__device__ void sta_ssm_body(const FluidConst& F, const PhasedArgs& a, int list)
{
    using F_ = SF<NC>;
    const StateBuf& S     = a.S;
    const uint32_t  n     = a.L.len(list);
    double          Y[NC], di[NC], sA[NC], Bi[NC];
    double          P = 0, Yt = 0;
    int             iter = 0, maxit = 0;
    bool            first = true;
    int64_t         c     = a.L.take(list, n);
    auto load = [&]() {
        P     = a.in.P[c];
        Yt    = S.D(F_::Yt, c);
        maxit = S.I(IF_MAXIT, c);  // the cap, or what an FP32 start left of it
#pragma unroll
        for (int i = 0; i < NC; i++) {
            Y[i]  = S.D(F_::Y + i, c);
            di[i] = S.D(F_::di + i, c);
            sA[i] = S.D(F_::sA + i, c);
            Bi[i] = S.D(F_::Bi + i, c);
        }
        iter  = 0;
        first = true;
    };
    if (c >= 0) load();
    while (__any_sync(0xffffffffu, c >= 0)) {
        if (c >= 0) {
            double phi[NC], aj, bj, zj;
            fug_phi<NC>(F, sA, Bi, P, Y, phi, nullptr, aj, bj, zj);
            double Se = 0;
#pragma unroll
            for (int i = 0; i < NC; i++) Se += sq(log((phi[i] * Y[i] * P) / (di[i] * P) * Yt));
            bool done;
            if (first) {
                first = false;
                done  = !(Se > F.ssmsta_tol2);
            } else {
                iter++;
                done = (iter > maxit) || !(Se > F.ssmsta_tol2);
                if (iter > maxit) S.I(IF_STATUS, c) |= ST_SSMSTA_CAP;
            }
            if (done) {
                S.D(F_::SeSSM, c) = Se;
                S.D(F_::Yt, c)    = Yt;
                S.D(F_::Asta, c)  = aj;
                S.D(F_::Bsta, c)  = bj;
                S.D(F_::Zsta, c)  = zj;
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    S.D(F_::Y + i, c)    = Y[i];
                    S.D(F_::phiS + i, c) = phi[i];
                }
                S.I(IF_IT0, c) += iter;
                c = a.L.take(list, n);
                if (c >= 0) load();
            } else {
                Yt = 0;
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    Y[i] = di[i] / phi[i];
                    Yt += Y[i];
                }
                const double r = 1 / Yt;
#pragma unroll
                for (int i = 0; i < NC; i++) Y[i] *= r;
            }
        }
    }
}

// The verdict of StableSSM trial k (src/MixtureComp.cpp:1567-1578) once
// StableNR is done: unstable -> split; stable -> next trial or finished.
template <int NC>
__device__ __forceinline__ void sta_decide(CellFlash<NC>& f, const PhasedArgs& a, int64_t c, uint32_t meta,
                                           int k, bool flag)
{
    using F_ = SF<NC>;
    const StateBuf& S  = a.S;
    const double    Se = S.D(F_::SeSSM, c);
    if (flag && f.Yt > 1 + f.F.ssmsta_eyt) {
        f.ssmsta_conflag = true;
        f.ssmsta_realTol = sqrt(Se);
        f.NP             = 2;
        store_book(f, S, c, meta & ~(M_RESTART | M_SPPHASE));
        a.L.push((a.opts & PH_EARLY) && k > 0 ? L_SP_T0 + k : L_SP_0, (int32_t)c);
    } else if (k < 3) {
        store_book(f, S, c, meta);
        a.L.push(stab_list(L_STA_0 + k + 1, a.sdup != 0), (int32_t)c);
    } else {
        f.ssmsta_realTol = sqrt(Se);
        finish_epec(f);
        S.D(F_::ePEC, c) = f.ePEC;
        store_single_phase(f, S, c);
        store_book(f, S, c, meta);
    }
}

// Start of StableNR (src/MixtureComp.cpp:1592-1598): residual of the
// trial's end point; converged cells get their verdict here, the rest go to
// the Newton kernel.
template <int NC>
__device__ void sta_verdict_body(const FluidConst& F, const PhasedArgs& a, int k, int list, int nrlist, bool from32)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    OCPF_FOR_ITEMS(a, list, c)
    {
        CellFlash<NC> f(F);
        uint32_t      meta;
        load_book(f, S, c, meta);
        const double P = a.in.P[c];
        if (from32) {
            // the FP32 trial's end point in FP64: Y (normalised), Yt, and
            // the trial phase's phi, a, b, Z
            double Y[NC], phi[NC], s = 0;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                f.sA[i] = S.D(F_::sA + i, c);
                f.Bi[i] = S.D(F_::Bi + i, c);
                Y[i]    = exp(S.D(F_::lnY + i, c));
                s += Y[i];
            }
            f.P = P;
            double aj, bj, zj;
#pragma unroll
            for (int i = 0; i < NC; i++) Y[i] /= s;
            f.fug_phi(Y, phi, nullptr, aj, bj, zj);
            S.D(F_::Asta, c) = aj;
            S.D(F_::Bsta, c) = bj;
            S.D(F_::Zsta, c) = zj;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                S.D(F_::Y + i, c)    = Y[i];
                S.D(F_::phiS + i, c) = phi[i];
            }
        }
        double Se = 0;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            const double fz = S.D(F_::di + i, c) * P;
            const double fs = S.D(F_::phiS + i, c) * S.D(F_::Y + i, c) * P;
            Se += sq(log(fz / (fs * f.Yt)));
        }
        if (from32) S.D(F_::SeSSM, c) = Se;
        Se = sqrt(Se);
        if (Se > F.nrsta_tol) {
            a.L.push(nrlist, (int32_t)c);
        } else {
            f.nrsta_conflag = true;
            f.nrsta_realTol = Se;
            sta_decide(f, a, c, meta, k, true);
        }
    }
}

// StableNR iterations (src/MixtureComp.cpp:1600-1635), one thread per cell.
template <int NC>
__device__ void sta_nr_body(const FluidConst& F, const PhasedArgs& a, int k, int list, int fallback)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    const uint32_t  n = a.L.len(list);
    CellFlash<NC>   f(F);
    uint32_t        meta = 0;
    double          fugId[NC], Y[NC], fugSta[NC], res[NC];
    double          Asta = 0, Bsta = 0, Zsta = 0, Se = 0;
    int             iter = 0;
    int64_t         c    = a.L.take(list, n);
    auto load = [&]() {
        load_book(f, S, c, meta);
        f.P = a.in.P[c];
#pragma unroll
        for (int i = 0; i < NC; i++) {
            f.sA[i]   = S.D(F_::sA + i, c);
            f.Bi[i]   = S.D(F_::Bi + i, c);
            fugId[i]  = S.D(F_::di + i, c) * f.P;
            Y[i]      = S.D(F_::Y + i, c);
            fugSta[i] = S.D(F_::phiS + i, c) * Y[i] * f.P;
            res[i]    = log(fugId[i] / (fugSta[i] * f.Yt));
        }
        Asta = S.D(F_::Asta, c), Bsta = S.D(F_::Bsta, c), Zsta = S.D(F_::Zsta, c);
        Se   = 0;
#pragma unroll
        for (int i = 0; i < NC; i++) Se += res[i] * res[i];
        Se   = sqrt(Se);
        iter = 0;
    };
    // the end of StableNR for the lane's cell: verdict, or (mixed form) the
    // FP64 continuation of a trial whose Newton step failed from FP32
    auto finish = [&](bool flag) {
        f.it_nrsta += iter;
        if (!flag && fallback >= 0) {
            f.status &= (uint16_t)~ST_NRSTA_FAIL;
            f.Yt = S.D(F_::Yt, c);
            store_book(f, S, c, meta | M_STC);
            a.L.push(fallback, (int32_t)c);
        } else {
            f.nrsta_conflag = flag;
            f.nrsta_realTol = Se;
            sta_decide(f, a, c, meta & ~M_STC, k, flag);
        }
        c = a.L.take(list, n);
        if (c >= 0) load();
    };
    if (c >= 0) load();
    // StableNR iterations (src/MixtureComp.cpp:1600-1635) on a persistent
    // grid: one Newton step per loop turn for every active lane
    while (__any_sync(0xffffffffu, c >= 0)) {
        if (c >= 0) {
            if (!(Se > F.nrsta_tol)) {
                finish(true);
                continue;
            }
            f.sta_nr_update(Y, f.Yt, res, Asta, Bsta, Zsta);
            f.fug_phi(Y, nullptr, fugSta, Asta, Bsta, Zsta);
            Se = 0;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                res[i] = log(fugId[i] / (fugSta[i] * f.Yt));
                Se += res[i] * res[i];
            }
            Se = sqrt(Se);
            iter++;
            if (iter > F.nrsta_maxit) {
                f.status |= ST_NRSTA_FAIL;
                finish(false);
            } else if (!(Se > F.nrsta_tol)) {
                finish(true);
            }
        }
    }
}

// --------------------------------------------------------- relaxed stability
// StableSSM01 trial k set-up (src/MixtureComp.cpp:1413-1421): K = Kw_k.
template <int NC>
__device__ void s01_prep_body(const FluidConst& F, const PhasedArgs& a, int k)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    OCPF_FOR_ITEMS(a, L_S01_0 + k, c)
    {
        CellFlash<NC> f(F);
        load_ptz(f, a, c);
        f.cal_kwilson();
#pragma unroll
        for (int i = 0; i < NC; i++) S.D(F_::Ks + i, c) = f.kw(k, i);
    }
}

// The iterations of one StableSSM01 trial (src/MixtureComp.cpp:1421-1466) on
// a persistent grid: per turn, Y from K, the step test, one fugacity
// evaluation, and the K update with its two convergence tests.
template <int NC>
__device__ void s01_ssm_body(const FluidConst& F, const PhasedArgs& a, int k)
{
    using F_ = SF<NC>;
    const StateBuf& S    = a.S;
    const int       list = L_S01_0 + k;
    const uint32_t  n    = a.L.len(list);
    double          z[NC], ks[NC], dY_[NC], fid[NC], sA[NC], Bi[NC], Y[NC];
    double          P = 0, Yt = 0, Se = 0, Sk = 0;
    int             iter = 0;
    int64_t         c    = a.L.take(list, n);
    auto load = [&]() {
        P = a.in.P[c];
        load_z<NC>(a, c, z);
#pragma unroll
        for (int i = 0; i < NC; i++) {
            ks[i]  = S.D(F_::Ks + i, c);
            sA[i]  = S.D(F_::sA + i, c);
            Bi[i]  = S.D(F_::Bi + i, c);
            fid[i] = S.D(F_::phiZ + i, c) * z[i] * P;
            dY_[i] = 0;
        }
        iter = 0;
    };
    auto finish = [&](bool flag) {
        S.D(F_::SeSSM, c) = Se;
        S.D(F_::SeSP, c)  = Sk;  // StableSSM01's Sk
        S.D(F_::Yt, c)    = Yt;
        S.I(IF_IT0, c) += iter;
        S.I(IF_GUARD, c) = flag ? 1 : 0;  // the trial's convergence flag
        c                = a.L.take(list, n);
        if (c >= 0) load();
    };
    if (c >= 0) load();
    while (__any_sync(0xffffffffu, c >= 0)) {
        bool need = false;
        if (c >= 0) {
            Yt = 0;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                Y[i] = z[i] * ks[i];
                Yt += Y[i];
            }
            const double r = 1 / Yt;
#pragma unroll
            for (int i = 0; i < NC; i++) Y[i] *= r;
            bool conv = false;
            if (iter > 0) {
                double dY = 0;
#pragma unroll
                for (int i = 0; i < NC; i++) dY += sq(Y[i] - dY_[i]);
                conv = dY < 1e-6;  // dYtol, include/MixtureComp.hpp:34
            }
            if (conv)
                finish(true);
            else
                need = true;
        }
        if (need) {
            double fs[NC], aj, bj, zj;
            fug_phi<NC>(F, sA, Bi, P, Y, nullptr, fs, aj, bj, zj);
            Se = 0;
            Sk = 0;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                const double d = fid[i] / (fs[i] * Yt);
                ks[i] *= d;
                Se += sq(d - 1);
                Sk += sq(log(ks[i]));
            }
            iter++;
            if (Se < F.ssmsta_tol2 || Sk < 1e-4) {  // Ktol, include/MixtureComp.hpp:33
                finish(true);
            } else if (iter > F.ssmsta_maxit) {
                S.I(IF_STATUS, c) |= ST_SSMSTA_CAP;
                finish(false);
            } else {
#pragma unroll
                for (int i = 0; i < NC; i++) dY_[i] = Y[i];
            }
        }
    }
}

// End of StableSSM01 trial k (src/MixtureComp.cpp:1475-1489) and, after the
// last trial or an unstable one, PhaseStable's fall-back to the strict test
// when the verdict contradicts the last phase count (:1373-1383).
template <int NC>
__device__ void s01_end_body(const FluidConst& F, const PhasedArgs& a, int k)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    OCPF_FOR_ITEMS(a, L_S01_0 + k, c)
    {
        CellFlash<NC> f(F);
        uint32_t      meta;
        load_book(f, S, c, meta);
        const bool   flag = S.I(IF_GUARD, c) != 0;
        const double Se   = S.D(F_::SeSSM, c);
        const double Sk   = S.D(F_::SeSP, c);
        S.I(IF_GUARD, c)  = 0;
        if (flag && f.Yt > 1 - 0.1 && Sk > 1) f.flagSkip = false;
        int verdict;  // 0 unstable, 1 stable, -1 next trial
        if (flag && f.Yt > 1 + F.ssmsta_eyt) {
            f.ssmsta_conflag = true;
            f.ssmsta_realTol = sqrt(Se);
            verdict          = 0;
        } else if (k < 1) {
            verdict = -1;
        } else {
            f.ssmsta_realTol = sqrt(Se);
            verdict          = 1;
        }
        if (verdict < 0) {
            store_book(f, S, c, meta);
            a.L.push(L_S01_1, (int32_t)c);
            continue;
        }
        // lNP of the cell (the last phase count, water excluded)
        const int lNP   = last_hc_np(a, c);
        const int tmpNP = f.NP + (verdict ? 0 : 1);
        if (tmpNP != lNP) {
            f.flagSkip = false;
            store_book(f, S, c, meta);
            a.L.push(L_STA_0, (int32_t)c);
        } else if (verdict == 0) {
            f.NP = 2;
            store_book(f, S, c, meta & ~(M_RESTART | M_SPPHASE));
            a.L.push(L_SP_0, (int32_t)c);
        } else {
            finish_epec(f);
            S.D(F_::ePEC, c) = f.ePEC;
            store_single_phase(f, S, c);
            store_book(f, S, c, meta);
        }
    }
}

// ----------------------------------------------------------------- split
// SplitSSM2 set-up (src/MixtureComp.cpp:1849-1879): initial K (last step's
// K, or Wilson's) or the restart's, and the tolerance and iteration cap.
template <int NC>
__device__ void sp_prep_body(const FluidConst& F, const PhasedArgs& a, int r)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    OCPF_FOR_ITEMS(a, L_SP_0 + r, c)
    {
        CellFlash<NC> f(F);
        uint32_t      meta;
        load_book(f, S, c, meta);
        const bool restart = (meta & M_RESTART) != 0;
        if (!restart) {
            f.ssmsp_conflag = false;  // PhaseSplit, :1745-1749
            f.nrsp_conflag  = false;
            const int lNP = last_hc_np(a, c);
            if (lNP == 2) {
                const int64_t N = a.stride;
#pragma unroll
                for (int i = 0; i < NC; i++)
                    S.D(F_::Ks + i, c) = a.in.xij[(int64_t)i * N + c] / a.in.xij[(int64_t)(i + NC + 1) * N + c];
            } else {
                load_ptz(f, a, c);
                f.cal_kwilson();
#pragma unroll
                for (int i = 0; i < NC; i++) S.D(F_::Ks + i, c) = f.Kw0[i];
            }
        }
        f.ssmsp_conflag = true;
        double Stol     = F.ssmsp_tol2;
        int    maxIt    = F.ssmsp_maxit;
        if (restart) {
            Stol *= 1e-1;
            maxIt *= 2;
        }
        if (f.Yt < 1.1) {
            Stol *= 1e-1;
            maxIt *= 2;
        }
        S.D(F_::Stol, c)  = Stol;
        S.I(IF_MAXIT, c)  = maxIt;
        store_book(f, S, c, meta);
    }
}

// SplitSSM2's iterations (src/MixtureComp.cpp:1881-1902) on a persistent
// grid: per turn, Rachford-Rice, the phase compositions, the fugacities of
// both phases, and the K update.
template <int NC>
__device__ void sp_ssm_body(const FluidConst& F, const PhasedArgs& a, int r)
{
    using F_ = SF<NC>;
    const StateBuf& S    = a.S;
    const int       list = L_SP_0 + r;
    const uint32_t  n    = a.L.len(list);
    CellFlash<NC>   f(F);  // holds z, K, x, phi, nu, Aj/Bj/Zj, sA, Bi
    double          Stol = 0;
    int             maxIt = 0, iter = 0;
    int64_t         c     = a.L.take(list, n);
    auto load = [&]() {
        f.P = a.in.P[c];
        load_z<NC>(a, c, f.zi);
#pragma unroll
        for (int i = 0; i < NC; i++) {
            f.Ks[i] = S.D(F_::Ks + i, c);
            f.sA[i] = S.D(F_::sA + i, c);
            f.Bi[i] = S.D(F_::Bi + i, c);
        }
        Stol     = S.D(F_::Stol, c);
        maxIt    = S.I(IF_MAXIT, c);
        iter     = 0;
        f.it_rr  = 0;
        f.NP     = 2;
    };
    if (c >= 0) load();
    while (__any_sync(0xffffffffu, c >= 0)) {
        if (c >= 0) {
            f.rachford_rice2();
#pragma unroll
            for (int i = 0; i < NC; i++) {
                const double tmp = 1 + f.nu[0] * (f.Ks[i] - 1);
                f.x[1][i]        = f.zi[i] / tmp;
                f.x[0][i]        = f.Ks[i] * f.x[1][i];
            }
            double fug0[NC], fug1[NC];
            fug_phi<NC>(F, f.sA, f.Bi, f.P, f.x[0], f.phi[0], fug0, f.Aj[0], f.Bj[0], f.Zj[0]);
            fug_phi<NC>(F, f.sA, f.Bi, f.P, f.x[1], f.phi[1], fug1, f.Aj[1], f.Bj[1], f.Zj[1]);
            double Se = 0;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                Se = __dadd_rn(Se, sq(fug1[i] / fug0[i] - 1));
                f.Ks[i] = f.phi[1][i] / f.phi[0][i];
            }
            iter++;
            const bool cap = iter > maxIt;
            if (cap || !(Se > Stol)) {
                if (cap) S.I(IF_META, c) &= ~(int32_t)M_C_SSMSP;
                S.D(F_::SeSP, c) = Se;
                S.I(IF_IT2, c) += iter;
                S.I(IF_IT4, c) += f.it_rr;
#pragma unroll
                for (int i = 0; i < NC; i++) S.D(F_::Ks + i, c) = f.Ks[i];
                store_split(f, S, c);
                c = a.L.take(list, n);
                if (c >= 0) load();
            }
        }
    }
}

// End of the learned initialiser's split (no reference counterpart). The
// split is kept when SplitNR converged to its tolerance with two phases
// (CheckSplit's accept branch, src/MixtureComp.cpp:1790-1797) whose
// compositions each sum to one, that differ (sum ln^2 K > 1e-4,
// StableSSM01's trivial-solution bound) and whose Gibbs energy is below the
// feed's: sum_i z_i (ln f_i - ln f_i(z)) < 0, so the feed is unstable and the
// stability test would send it to a split. Otherwise the cell returns, as a
// fresh single-phase cell, to the strict stability test.
template <int NC>
__device__ __forceinline__ void learned_after_nr(CellFlash<NC>& f, const PhasedArgs& a, int64_t c, uint32_t meta)
{
    using F_ = SF<NC>;
    const StateBuf& S     = a.S;
    const double    nuMax = f.nu[0] < f.nu[1] ? f.nu[1] : f.nu[0];
    double          eX = 0, tk = 0, dg = 0, s0 = 0, s1 = 0;
#pragma unroll
    for (int i = 0; i < NC; i++) {
        eX += sq(f.x[0][i] - f.x[1][i]);
        tk += sq(log(f.x[0][i] / f.x[1][i]));
        dg += f.zi[i] * log(f.fug[0][i] / (S.D(F_::phiZ + i, c) * f.zi[i] * f.P));
        s0 += f.x[0][i];
        s1 += f.x[1][i];
    }
    // converged to the tolerance (not SplitNR's small-step exit), both
    // compositions summing to one (no phase-1 moles folded by |n / nu|)
    const bool keep = f.nrsp_conflag && f.nrsp_realTol < f.F.nrsp_tol && fabs(s0 - 1) < 1e-10 &&
                      fabs(s1 - 1) < 1e-10 && f.NP == 2 && nuMax < 1 && 1 - nuMax >= 1e-3 && isfinite(eX) &&
                      tk > 1e-4 && dg < 0;
    if (keep) {
        f.check_split();
        if (!f.ssmsp_conflag) f.status |= ST_SSMSP_FAIL;
        finish_epec(f);
        S.D(F_::ePEC, c) = f.ePEC;
        store_split(f, S, c);
        store_book(f, S, c, meta);
        return;
    }
    // fall back: the fresh single-phase state init left (x0 = z, the
    // mixture of z), then the strict stability test
    f.NP            = 1;
    f.nu[0]         = 1;
    f.ssmsp_conflag = false;
    f.nrsp_conflag  = false;
    f.status &= (uint16_t) ~(ST_SINGULAR | ST_COLLAPSED | ST_SSMSP_FAIL | ST_NRSP_FAIL);
    double t[NC];
    f.mix_ab(f.zi, t, f.Aj[0], f.Bj[0]);
    f.Zj[0]          = sol_eos(f.Aj[0], f.Bj[0]);
    S.D(F_::Aj0, c)  = f.Aj[0];
    S.D(F_::Bj0, c)  = f.Bj[0];
    S.D(F_::Zj0, c)  = f.Zj[0];
    S.I(IF_GUARD, c) = 0;
    store_single_phase(f, S, c, true);
    store_book(f, S, c, meta & ~(M_LEARNED | M_RESTART | M_SPPHASE));
    a.L.push(stab_list(L_STA_0, (a.opts & PH_DEFER) != 0), (int32_t)c);
}

// End of PhaseSplit once SplitNR is done (src/MixtureComp.cpp:1750-1758,
// 1784-1836): accept, restart the SSM, or collapse to one phase.
template <int NC>
__device__ __forceinline__ void sp_after_nr(CellFlash<NC>& f, const PhasedArgs& a, int64_t c, uint32_t meta,
                                            int r, double eNR, int iter)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    f.nrsp_realTol    = eNR;
    if (eNR < f.F.nrsp_tol) f.nrsp_conflag = true;
    f.it_nrsp += iter;
    if (r == LEARN_ROUND) {
        learned_after_nr(f, a, c, meta);
        return;
    }
    bool restart = false;
    if (!(meta & M_SPPHASE)) {
        if (!f.nrsp_conflag) {
            restart = true;
            meta |= M_SPPHASE | M_RESTART;
            S.I(IF_GUARD, c) = 1;
        }
    } else if (!f.check_split()) {
        // collapsed: the final check below is a no-op
    } else if (f.ssmsp_conflag || f.nrsp_conflag) {
        // loop ends
    } else {
        const int g      = S.I(IF_GUARD, c) + 1;
        S.I(IF_GUARD, c) = g;
        if (g > SPLIT_RESTART_CAP)
            f.status |= ST_SPLIT_CAP;
        else
            restart = true;
    }
    if (restart) {
        store_split(f, S, c);
        store_book(f, S, c, meta);
        const int slow = r >= TRIAL_ROUND0 ? L_SLOW_T0 + (r - TRIAL_ROUND0) : L_SLOW;
        a.L.push(r + 1 < SPLIT_ROUNDS ? L_SP_0 + r + 1 : slow, (int32_t)c);
        return;
    }
    f.check_split();
    if (!f.ssmsp_conflag) f.status |= ST_SSMSP_FAIL;
    if (!f.nrsp_conflag) f.status |= ST_NRSP_FAIL;
    finish_epec(f);
    S.D(F_::ePEC, c) = f.ePEC;
    if (f.NP == 1) {
        S.D(F_::Aj0, c) = f.Aj[0];
        S.D(F_::Bj0, c) = f.Bj[0];
        S.D(F_::Zj0, c) = f.Zj[0];
        store_single_phase(f, S, c, true);
    } else {
        store_split(f, S, c);
    }
    store_book(f, S, c, meta);
}

// Loads a split cell into a CellFlash for the thread-per-item kernels.
template <int NC>
__device__ __forceinline__ void load_split_cell(CellFlash<NC>& f, const PhasedArgs& a, int64_t c, uint32_t& meta)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    load_book(f, S, c, meta);
    f.P      = a.in.P[c];
    f.Nh     = load_z<NC>(a, c, f.zi);
#pragma unroll
    for (int i = 0; i < NC; i++) {
        f.sA[i] = S.D(F_::sA + i, c);
        f.Bi[i] = S.D(F_::Bi + i, c);
    }
    load_split(f, S, c);
}

// Start of SplitNR (src/MixtureComp.cpp:2059-2069): n = nu x and the
// residual; converged cells finish PhaseSplit here, the rest go to Newton.
template <int NC>
__device__ void sp_nrinit_body(const FluidConst& F, const PhasedArgs& a, int r)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    OCPF_FOR_ITEMS(a, L_SP_0 + r, c)
    {
        CellFlash<NC> f(F);
        uint32_t      meta;
        load_split_cell(f, a, c, meta);
        f.ssmsp_realTol = sqrt(S.D(F_::SeSP, c));
        f.nrsp_conflag  = false;
        double eNR      = 0;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            f.n[0][i] = f.nu[0] * f.x[0][i];
            f.n[1][i] = f.nu[1] * f.x[1][i];
            const double res = log(f.fug[1][i] / f.fug[0][i]);
            eNR += res * res;
        }
        eNR = sqrt(eNR);
        if (eNR > F.nrsp_tol) {
            S.D(F_::eNR0, c) = eNR;
            store_split(f, S, c);
            store_book(f, S, c, meta);
            a.L.push(L_SPNR_0 + r, (int32_t)c);
        } else {
            sp_after_nr(f, a, c, meta, r, eNR, 0);
        }
    }
}

// SplitNR iterations (src/MixtureComp.cpp:2071-2152) on a persistent grid:
// each loop turn is one Newton step (Jacobian, solve, fugacities, residual)
// for every active lane; a lane whose cell ends its Newton loop finishes it
// (sp_after_nr) and takes the next cell, so lanes stay busy however
// unequal the cells' step counts are.
template <int NC>
__device__ void sp_nr_body(const FluidConst& F, const PhasedArgs& a, int r)
{
    using F_ = SF<NC>;
    const StateBuf& S    = a.S;
    const int       list = L_SPNR_0 + r;
    const uint32_t  n    = a.L.len(list);
    CellFlash<NC>   f(F);
    uint32_t        meta = 0;
    double          res[NC];
    double          eNR0 = 0, eNR = 0;
    int             iter = 0;
    int64_t         c    = a.L.take(list, n);
    auto load = [&]() {
        load_split_cell(f, a, c, meta);
        eNR0 = S.D(F_::eNR0, c);
        eNR  = eNR0;
        iter = 0;
#pragma unroll
        for (int i = 0; i < NC; i++) res[i] = log(f.fug[1][i] / f.fug[0][i]);
    };
    if (c >= 0) load();
    while (__any_sync(0xffffffffu, c >= 0)) {
        if (c >= 0) {
            bool done = !(eNR > F.nrsp_tol);
            if (!done) {
                const double en = f.sp_nr_update(res);
                f.fug_phi_all();
                eNR = 0;
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    res[i] = log(f.fug[1][i] / f.fug[0][i]);
                    eNR += res[i] * res[i];
                }
                eNR = sqrt(eNR);
                iter++;
                if (eNR > eNR0 || iter > F.nrsp_maxit) {
                    done = true;
                } else if (en / (2 * NC) < 1e-8) {
                    f.nrsp_conflag = true;
                    done           = true;
                } else {
                    done = !(eNR > F.nrsp_tol);
                }
            }
            if (done) {
                sp_after_nr(f, a, c, meta, r, eNR, iter);
                c = a.L.take(list, n);
                if (c >= 0) load();
            }
        }
    }
}

// PhaseSplit's restart loop (src/MixtureComp.cpp:1750-1758) for the cells
// whose first split did not converge (rare: a few hundred per million
// states, some needing tens of thousands of steps), one warp per cell
// (flash_warp.cuh); lane 0 stores the result.
template <int NC>
__device__ void slow_body(const FluidConst& F, const PhasedArgs& a, int list = L_SLOW)
{
    using F_ = SF<NC>;
    const StateBuf& S    = a.S;
    const uint32_t  n    = a.L.len(list);
    const uint32_t  nw   = (vgrid(a) * blockDim.x) >> 5;
    const bool      lead = (threadIdx.x & 31) == 0;
    for (uint32_t k = (vblock(a) * blockDim.x + threadIdx.x) >> 5; k < n; k += nw) {
        const int64_t c = a.L.item(list, k);
        CellFlash<NC> f(F);
        uint32_t      meta;
        load_split_cell(f, a, c, meta);
        f.T = a.in.T[c] + CONV5;
        f.cal_kwilson();
        WarpSplit<NC> w(f);
        int           guard = S.I(IF_GUARD, c);
        while (true) {
            w.split_ssm2(true);
            w.split_nr();
            if (!f.check_split()) break;
            if (f.ssmsp_conflag || f.nrsp_conflag) break;
            if (++guard > SPLIT_RESTART_CAP) {
                f.status |= ST_SPLIT_CAP;
                break;
            }
        }
        f.check_split();
        if (!f.ssmsp_conflag) f.status |= ST_SSMSP_FAIL;
        if (!f.nrsp_conflag) f.status |= ST_NRSP_FAIL;
        finish_epec(f);
        if (lead) {
            S.D(F_::ePEC, c) = f.ePEC;
            if (f.NP == 1) {
                S.D(F_::Aj0, c) = f.Aj[0];
                S.D(F_::Bj0, c) = f.Bj[0];
                S.D(F_::Zj0, c) = f.Zj[0];
                store_single_phase(f, S, c, true);
            } else {
                store_split(f, S, c);
            }
            store_book(f, S, c, meta);
        }
    }
}

// The restart loop of slow_body with one thread per cell (CellFlash's own
// SplitSSM2 / SplitNR, as in the plain form): 32 cells per warp instead of
// one, each on a longer dependent chain. The autotuner's alternative for
// batches with many restarting cells.
template <int NC>
__device__ void slow_thread_body(const FluidConst& F, const PhasedArgs& a, int list = L_SLOW)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    OCPF_FOR_ITEMS(a, list, c)
    {
        CellFlash<NC> f(F);
        uint32_t      meta;
        load_split_cell(f, a, c, meta);
        f.T = a.in.T[c] + CONV5;
        f.cal_kwilson();
        int guard = S.I(IF_GUARD, c);
        while (true) {
            f.split_ssm2(true);
            f.split_nr();
            if (!f.check_split()) break;
            if (f.ssmsp_conflag || f.nrsp_conflag) break;
            if (++guard > SPLIT_RESTART_CAP) {
                f.status |= ST_SPLIT_CAP;
                break;
            }
        }
        f.check_split();
        if (!f.ssmsp_conflag) f.status |= ST_SSMSP_FAIL;
        if (!f.nrsp_conflag) f.status |= ST_NRSP_FAIL;
        finish_epec(f);
        S.D(F_::ePEC, c) = f.ePEC;
        if (f.NP == 1) {
            S.D(F_::Aj0, c) = f.Aj[0];
            S.D(F_::Bj0, c) = f.Bj[0];
            S.D(F_::Zj0, c) = f.Zj[0];
            store_single_phase(f, S, c, true);
        } else {
            store_split(f, S, c);
        }
        store_book(f, S, c, meta);
    }
}

// --------------------------------------------------------------- finalize
template <int NC, bool FIMN = false>
__device__ void phased_finalize_body(const FluidConst& F, const PhasedArgs& a)
{
    using F_ = SF<NC>;
    const StateBuf& S = a.S;
    for (int64_t c = vblock(a) * (int64_t)blockDim.x + threadIdx.x; c < a.count;
         c += (int64_t)vgrid(a) * blockDim.x) {
        FimCell<NC> f(F);
        f.load_inputs(c, a.stride, a.in, a.sk, a.tail);
        uint32_t meta;
        load_book(f, S, c, meta);
#pragma unroll
        for (int i = 0; i < NC; i++) {
            f.sA[i] = S.D(F_::sA + i, c);
            f.Bi[i] = S.D(F_::Bi + i, c);
        }
        f.ePEC  = S.D(F_::ePEC, c);
        f.nu[0] = S.D(F_::nu0, c);
        f.nu[1] = S.D(F_::nu1, c);
        f.Aj[0] = S.D(F_::Aj0, c);
        f.Aj[1] = S.D(F_::Aj1, c);
        f.Bj[0] = S.D(F_::Bj0, c);
        f.Bj[1] = S.D(F_::Bj1, c);
        f.Zj[0] = S.D(F_::Zj0, c);
        f.Zj[1] = S.D(F_::Zj1, c);
#pragma unroll
        for (int i = 0; i < NC; i++) {
            f.x[0][i] = S.D(F_::x0 + i, c);
            f.x[1][i] = S.D(F_::x1 + i, c);
            f.n[0][i] = S.D(F_::n0 + i, c);
            f.n[1][i] = S.D(F_::n1 + i, c);
        }
        if (FIMN && f.NP == 2) {
            // FlashFIMn's residual reads the fugacities of the split
#pragma unroll
            for (int i = 0; i < NC; i++) {
                f.phi[0][i] = S.D(F_::phi0 + i, c);
                f.phi[1][i] = S.D(F_::phi1 + i, c);
            }
        }
        f.template finalize<FIMN>(c, a.stride, a.sk, a.out, a.tail);
    }
}

}  // namespace ocpf
