/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Batch harness around the reference's own MixtureComp (compiled from the
 * reference sources by oracle/Makefile into oracle/_ref/libocpref.so). For each
 * cell it makes exactly the calls IsoT_FIM::CalFlash makes
 * (src/OCPFluidMethod.cpp:1108-1120): MixtureComp::FlashFIM followed by the
 * copy-out of IsoT_FIM::PassFlashValue (src/OCPFluidMethod.cpp:1122-1187);
 * likewise FlashIMPEC, InitFlashFIM / InitFlashIMPEC and, after the flash,
 * IsoT_FIM::CalKrPc with FlowUnit_ODGW01 (src/FlowUnit.cpp).
 * Nothing of the reference is copied here; its headers are included and its
 * objects linked. The access specifiers are opened only to read the
 * iteration counters, the flash type, the hydrocarbon phase count and the
 * SkipStaAnaly cache, which the reference keeps private.
 */
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#define private public
#define protected public
#include "DenseMat.hpp"
#include "FlowUnit.hpp"
#include "MixtureComp.hpp"
#include "OptionalFeatures.hpp"
#include "ParamReservoir.hpp"
#undef private
#undef protected

#include "oracle_api.h"

namespace {

std::string num(double v)
{
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.17g", v);
    return buf;
}

std::string num(int v) { return std::to_string(v); }

// Builds the ParamReservoir that MixtureComp(const ParamReservoir&, 0)
// consumes (src/MixtureComp.cpp:28-165, include/MixtureComp.hpp:155-167).
void make_param(const orc_fluid& f, ParamReservoir& rs)
{
    const int nc          = f.nc;
    ComponentParam& cp    = rs.comsParam;
    cp.numCom             = nc;
    cp.numPhase           = 2;
    auto set = [nc](Type_A_r<std::vector<OCP_DBL>>& dst, const double* src) {
        dst.activity = OCP_TRUE;
        dst.data.assign(1, std::vector<OCP_DBL>(src, src + nc));
    };
    cp.Cname.clear();
    for (int i = 0; i < nc; i++) cp.Cname.push_back("C" + std::to_string(i + 1));
    set(cp.Tc, f.Tc);
    set(cp.Pc, f.Pc);
    set(cp.Vc, f.Vc);
    set(cp.MW, f.MW);
    set(cp.Acf, f.Acf);
    set(cp.OmegaA, f.OmegaA);
    set(cp.OmegaB, f.OmegaB);
    set(cp.Vshift, f.Vshift);
    cp.LBCcoef.assign(f.LBCcoef, f.LBCcoef + 5);
    // lower triangle, as the BIC keyword gives it (src/MixtureComp.cpp:118-129)
    std::vector<OCP_DBL> low;
    for (int i = 1; i < nc; i++)
        for (int j = 0; j < i; j++) low.push_back(f.BIC[i * nc + j]);
    cp.BIC.assign(1, low);
    cp.SSMparamSTA = {num(f.ssmsta_maxit), num(f.ssmsta_tol), num(f.ssmsta_eyt)};
    cp.NRparamSTA  = {num(f.nrsta_maxit), num(f.nrsta_tol)};
    cp.SSMparamSP  = {num(f.ssmsp_maxit), num(f.ssmsp_tol)};
    cp.NRparamSP   = {num(f.nrsp_maxit), num(f.nrsp_tol)};
    cp.RRparam     = {num(f.rr_maxit), num(f.rr_tol)};
    cp.miscible    = OCP_FALSE;
    rs.PVTW_T.data.assign(1, std::vector<std::vector<OCP_DBL>>(5));
    for (int k = 0; k < 5; k++) rs.PVTW_T.data[0][k] = {f.pvtw[k]};
    rs.density.activity = OCP_TRUE; // std_RhoW = RHOW_STD, overwritten below
}

// The per-bulk SkipStaAnaly cache of cells [lo, lo + cnt) in and out of the
// flash object's own copy (src/AcceleratePVT.cpp).
void skip_in(const orc_fluid& f, const orc_batch& b, SkipStaAnaly& sk, int64_t lo, int64_t cnt)
{
    if (!f.use_skip) return;
    for (int64_t c = 0; c < cnt; c++) {
        const int64_t n = lo + c;
        sk.flag[c]      = b.skip_flag[n] ? OCP_TRUE : OCP_FALSE;
        sk.minEigen[c]  = b.skip_minEig[n];
        sk.P[c]         = b.skip_P[n];
        sk.T[c]         = b.skip_T[n];
        for (int i = 0; i < f.nc; i++) sk.zi[c * f.nc + i] = b.skip_z[n * f.nc + i];
    }
}

void skip_out(const orc_fluid& f, const orc_batch& b, const SkipStaAnaly& sk, int64_t lo, int64_t cnt)
{
    if (!f.use_skip) return;
    for (int64_t c = 0; c < cnt; c++) {
        const int64_t n  = lo + c;
        b.skip_flag[n]   = sk.flag[c] ? 1 : 0;
        b.skip_minEig[n] = sk.minEigen[c];
        b.skip_P[n]      = sk.P[c];
        b.skip_T[n]      = sk.T[c];
        for (int i = 0; i < f.nc; i++) b.skip_z[n * f.nc + i] = sk.zi[c * f.nc + i];
    }
}

// Copy-out of IsoT_FIM::PassFlashValue (src/OCPFluidMethod.cpp:1122-1187)
// for cell n, plus nj.
void copy_fim(const MixtureComp& mc, const orc_batch& b, int numCom, int64_t n)
{
    const int np     = 3;
    const int ncol   = numCom + 1;
    const int maxLen = ncol * ncol * np;
    int       pn = 0, len = 0;
    for (int j = 0; j < np; j++) {
        b.S[n * np + j]          = mc.GetS(j);
        const int ex             = mc.GetPhaseExist(j) ? 1 : 0;
        b.phaseExist[n * np + j] = ex;
        if (ex) {
            pn++;
            b.rho[n * np + j]  = mc.GetRho(j);
            b.xi[n * np + j]   = mc.GetXi(j);
            b.mu[n * np + j]   = mc.GetMu(j);
            b.rhoP[n * np + j] = mc.GetRhoP(j);
            b.xiP[n * np + j]  = mc.GetXiP(j);
            b.muP[n * np + j]  = mc.GetMuP(j);
            b.nj[n * np + j]   = mc.GetNj(j);
            for (int i = 0; i < numCom; i++) {
                const int64_t o = (n * np + j) * numCom + i;
                b.xij[o]        = mc.GetXij(j, i);
                b.rhox[o]       = mc.GetRhoX(j, i);
                b.xix[o]        = mc.GetXiX(j, i);
                b.mux[o]        = mc.GetMuX(j, i);
            }
        }
        b.pSderExist[n * np + j] = mc.GetPSderExist(j) ? 1 : 0;
        b.pVnumCom[n * np + j]   = static_cast<int32_t>(mc.GetPVnumCom(j));
        if (b.pSderExist[n * np + j]) len++;
        len += b.pVnumCom[n * np + j];
    }
    b.phaseNum[n] = pn;
    b.Nt[n]       = mc.GetNt();
    b.vf[n]       = mc.GetVf();
    b.vfP[n]      = mc.GetVfP();
    for (int i = 0; i < numCom; i++) b.vfi[n * numCom + i] = mc.GetVfi(i);
    b.bRowSizedSdP[n]              = len;
    const std::vector<OCP_DBL>& dd = mc.GetDXsDXp();
    std::copy(dd.begin(), dd.begin() + len * ncol, b.dSec_dPri + n * maxLen);
}

// Copy-out of IsoT_IMPEC::PassFlashValue (src/OCPFluidMethod.cpp:275-305)
// for cell n, the phase volumes into vjout.
void copy_impec(const MixtureComp& mc, const orc_batch& b, double* vjout, int numCom, int64_t n)
{
    const int np = 3;
    int       pn = 0;
    for (int j = 0; j < np; j++) {
        b.S[n * np + j]          = mc.GetS(j);
        const int ex             = mc.GetPhaseExist(j) ? 1 : 0;
        b.phaseExist[n * np + j] = ex;
        if (ex) {
            pn++;
            for (int i = 0; i < numCom; i++) b.xij[(n * np + j) * numCom + i] = mc.GetXij(j, i);
            vjout[n * np + j] = mc.GetVj(j);
            b.rho[n * np + j] = mc.GetRho(j);
            b.xi[n * np + j]  = mc.GetXi(j);
            b.mu[n * np + j]  = mc.GetMu(j);
        }
    }
    b.phaseNum[n] = pn;
    b.Nt[n]       = mc.GetNt();
    b.vf[n]       = mc.GetVf();
    b.vfP[n]      = mc.GetVfP();
    for (int i = 0; i < numCom; i++) b.vfi[n * numCom + i] = mc.GetVfi(i);
}

// Runs cells [lo, hi) of a batch on one flash object of its own: for each
// cell `call(mc, n, c)` makes the reference's flash call (c: the cell's bulk
// id within the object) and `copy(mc, n)` its copy-out; the diagnostics
// (ePEC, flash type, hydrocarbon phase count, iteration counts) follow.
template <class Call, class Copy>
void run_cells(const orc_fluid& f, const orc_batch& b, int64_t lo, int64_t hi, double* secs, Call call, Copy copy)
{
    const int64_t cnt = hi - lo;
    if (cnt <= 0) {
        *secs = 0;
        return;
    }
    ParamReservoir rs;
    make_param(f, rs);
    MixtureComp mc(rs, 0);
    mc.std_RhoW = f.std_rho_w;
    OptionalFeatures of;
    of.skipStaAnaly.SetUseSkip(f.use_skip ? OCP_TRUE : OCP_FALSE);
    mc.SetupOptionalFeatures(of, static_cast<OCP_USI>(cnt));
    SkipStaAnaly& sk = of.skipStaAnaly;
    skip_in(f, b, sk, lo, cnt);
    auto t0 = std::chrono::steady_clock::now();
    for (int64_t c = 0; c < cnt; c++) {
        const int64_t n      = lo + c;
        const OCP_ULL it0[5] = {mc.itersSSMSTA, mc.itersNRSTA, mc.itersSSMSP, mc.itersNRSP, mc.itersRR};
        call(mc, n, static_cast<OCP_USI>(c));
        copy(mc, n);
        b.ePEC[n]          = mc.GetErrorPEC();
        b.ftype[n]         = static_cast<int32_t>(mc.ftype);
        b.NPhc[n]          = static_cast<int32_t>(mc.NP);
        b.iters[n * 5 + 0] = static_cast<int32_t>(mc.itersSSMSTA - it0[0]);
        b.iters[n * 5 + 1] = static_cast<int32_t>(mc.itersNRSTA - it0[1]);
        b.iters[n * 5 + 2] = static_cast<int32_t>(mc.itersSSMSP - it0[2]);
        b.iters[n * 5 + 3] = static_cast<int32_t>(mc.itersNRSP - it0[3]);
        b.iters[n * 5 + 4] = static_cast<int32_t>(mc.itersRR - it0[4]);
    }
    auto t1 = std::chrono::steady_clock::now();
    *secs   = std::chrono::duration<double>(t1 - t0).count();
    skip_out(f, b, sk, lo, cnt);
}

// FlashFIM over cells [lo, hi): the calls of IsoT_FIM::CalFlash
// (src/OCPFluidMethod.cpp:1108-1120).
void run_chunk(const orc_fluid& f, const orc_batch& b, int64_t lo, int64_t hi, double* secs)
{
    const int           numCom = f.nc + 1, np = 3;
    std::vector<double> Sin(np), xin(np * numCom), Nin(numCom);
    run_cells(
        f, b, lo, hi, secs,
        [&](MixtureComp& mc, int64_t n, OCP_USI c) {
            std::copy(b.S_in + n * np, b.S_in + (n + 1) * np, Sin.begin());
            std::copy(b.xij_in + n * np * numCom, b.xij_in + (n + 1) * np * numCom, xin.begin());
            std::copy(b.Ni + n * numCom, b.Ni + (n + 1) * numCom, Nin.begin());
            mc.FlashFIM(b.P[n], b.T[n], Nin.data(), Sin.data(), static_cast<USI>(b.lastNP[n]), xin.data(), c);
        },
        [&](const MixtureComp& mc, int64_t n) { copy_fim(mc, b, numCom, n); });
}

// FlashIMPEC over cells [lo, hi): the calls of IsoT_IMPEC::CalFlash
// (src/OCPFluidMethod.cpp:264-273).
void run_chunk_impec(const orc_fluid& f, const orc_batch& b, double* vjout, int64_t lo, int64_t hi, double* secs)
{
    const int           numCom = f.nc + 1, np = 3;
    std::vector<double> xin(np * numCom), Nin(numCom);
    run_cells(
        f, b, lo, hi, secs,
        [&](MixtureComp& mc, int64_t n, OCP_USI c) {
            std::copy(b.xij_in + n * np * numCom, b.xij_in + (n + 1) * np * numCom, xin.begin());
            std::copy(b.Ni + n * numCom, b.Ni + (n + 1) * numCom, Nin.begin());
            mc.FlashIMPEC(b.P[n], b.T[n], Nin.data(), static_cast<USI>(b.lastNP[n]), xin.data(), c);
        },
        [&](const MixtureComp& mc, int64_t n) { copy_impec(mc, b, vjout, numCom, n); });
}

// InitFlashFIM or InitFlashIMPEC over cells [lo, hi): the calls of
// IsoT_FIM::InitFlash (src/OCPFluidMethod.cpp:1095-1106) or
// IsoT_IMPEC::InitFlash (:251-262). b.Ni holds the mole fractions z, S_in
// the initial saturations; Ni receives the flash object's Ni afterwards.
void run_chunk_init(const orc_fluid& f, const orc_batch& b, const double* Vpore, int impec, double* Niout,
                    double* vjout, int64_t lo, int64_t hi, double* secs)
{
    const int           numCom = f.nc + 1, np = 3;
    std::vector<double> Sin(np), zin(numCom);
    run_cells(
        f, b, lo, hi, secs,
        [&](MixtureComp& mc, int64_t n, OCP_USI c) {
            std::copy(b.S_in + n * np, b.S_in + (n + 1) * np, Sin.begin());
            std::copy(b.Ni + n * numCom, b.Ni + (n + 1) * numCom, zin.begin());
            const OCP_DBL Pbb = 0;  // unused by MixtureComp
            if (impec)
                mc.InitFlashIMPEC(b.P[n], Pbb, b.T[n], Sin.data(), Vpore[n], zin.data(), c);
            else
                mc.InitFlashFIM(b.P[n], Pbb, b.T[n], Sin.data(), Vpore[n], zin.data(), c);
            for (int i = 0; i < numCom; i++) Niout[n * numCom + i] = mc.GetNi(i);
        },
        [&](const MixtureComp& mc, int64_t n) {
            if (impec)
                copy_impec(mc, b, vjout, numCom, n);
            else
                copy_fim(mc, b, numCom, n);
        });
}

// Copy-out of IsoT_FIMn::PassFlashValue (src/OCPFluidMethod.cpp:3179-3196)
// for cell n: the FIM copy-out, then the first bRowSizedSdP entries of the
// flash's res into res [n * 3 * (numCom + 1)] and resPc.
void copy_fimn(const MixtureComp& mc, const orc_batch& b, double* res, double* resPc, int numCom, int64_t n)
{
    copy_fim(mc, b, numCom, n);
    const int                   len = b.bRowSizedSdP[n];
    const std::vector<OCP_DBL>& r   = mc.GetRes();
    std::copy(r.begin(), r.begin() + len, res + n * 3 * (numCom + 1));
    resPc[n] = mc.GetResPc();
}

// FlashFIMn over cells [lo, hi): the calls of IsoT_FIMn::CalFlash
// (src/OCPFluidMethod.cpp:3152-3177). The flash reads its njin and
// phaseExistin arguments only to count input phases for a branch it never
// takes (src/MixtureComp.cpp:586-592); they are passed as zeros and the
// saturation-based flags.
void run_chunk_fimn(const orc_fluid& f, const orc_batch& b, double* res, double* resPc, int64_t lo, int64_t hi,
                    double* secs)
{
    const int           numCom = f.nc + 1, np = 3;
    std::vector<double> Sin(np), xin(np * numCom), Nin(numCom), njin(np, 0.0);
    std::vector<USI>    ex(np, 0);
    run_cells(
        f, b, lo, hi, secs,
        [&](MixtureComp& mc, int64_t n, OCP_USI c) {
            std::copy(b.S_in + n * np, b.S_in + (n + 1) * np, Sin.begin());
            std::copy(b.xij_in + n * np * numCom, b.xij_in + (n + 1) * np * numCom, xin.begin());
            std::copy(b.Ni + n * numCom, b.Ni + (n + 1) * numCom, Nin.begin());
            for (int j = 0; j < np; j++) ex[j] = (j == np - 1 || Sin[j] > 0) ? 1 : 0;
            mc.FlashFIMn(b.P[n], b.T[n], Nin.data(), Sin.data(), xin.data(), njin.data(), ex.data(),
                         static_cast<USI>(b.lastNP[n]), c);
        },
        [&](const MixtureComp& mc, int64_t n) { copy_fimn(mc, b, res, resPc, numCom, n); });
}

// InitFlashFIMn over cells [lo, hi): the calls of IsoT_FIMn::InitFlash
// (src/OCPFluidMethod.cpp:3129-3150), inputs as run_chunk_init.
void run_chunk_init_fimn(const orc_fluid& f, const orc_batch& b, const double* Vpore, double* Niout, double* res,
                         double* resPc, int64_t lo, int64_t hi, double* secs)
{
    const int           numCom = f.nc + 1, np = 3;
    std::vector<double> Sin(np), zin(numCom);
    run_cells(
        f, b, lo, hi, secs,
        [&](MixtureComp& mc, int64_t n, OCP_USI c) {
            std::copy(b.S_in + n * np, b.S_in + (n + 1) * np, Sin.begin());
            std::copy(b.Ni + n * numCom, b.Ni + (n + 1) * numCom, zin.begin());
            const OCP_DBL Pbb = 0;  // unused by MixtureComp
            mc.InitFlashFIMn(b.P[n], Pbb, b.T[n], Sin.data(), Vpore[n], zin.data(), c);
            for (int i = 0; i < numCom; i++) Niout[n * numCom + i] = mc.GetNi(i);
        },
        [&](const MixtureComp& mc, int64_t n) { copy_fimn(mc, b, res, resPc, numCom, n); });
}

// Runs `chunk(lo, hi, &secs)` over nthreads host threads with the
// reference's console output muted; *seconds: the slowest thread's loop.
template <class Chunk>
int run_threads(int64_t n, int nthreads, double* seconds, Chunk chunk)
{
    if (nthreads < 1) nthreads = 1;
    if (n <= 0) {
        if (seconds) *seconds = 0;
        return 0;
    }
    if (nthreads > n) nthreads = static_cast<int>(n);
    // The reference prints from its constructor and from CheckSplit; mute it.
    std::ios::iostate st = std::cout.rdstate();
    std::cout.setstate(std::ios::failbit);
    std::vector<double>      secs(nthreads, 0.0);
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) {
        const int64_t lo = n * t / nthreads, hi = n * (t + 1) / nthreads;
        th.emplace_back([&chunk, lo, hi, &secs, t]() { chunk(lo, hi, &secs[t]); });
    }
    for (auto& x : th) x.join();
    std::cout.clear(st);
    if (seconds) *seconds = *std::max_element(secs.begin(), secs.end());
    return 0;
}

} // namespace

extern "C" int orc_flash_fim_batch(const orc_fluid* fluid, const orc_batch* batch, int nthreads, double* seconds)
{
    if (!fluid || !batch || fluid->nc < 2 || fluid->nc > ORC_MAX_NC) return 1;
    return run_threads(batch->n, nthreads, seconds, [fluid, batch](int64_t lo, int64_t hi, double* s) {
        run_chunk(*fluid, *batch, lo, hi, s);
    });
}

extern "C" int orc_flash_impec_batch(const orc_fluid* fluid, const orc_batch* batch, double* vj, int nthreads,
                                     double* seconds)
{
    if (!fluid || !batch || !vj || fluid->nc < 2 || fluid->nc > ORC_MAX_NC) return 1;
    return run_threads(batch->n, nthreads, seconds, [fluid, batch, vj](int64_t lo, int64_t hi, double* s) {
        run_chunk_impec(*fluid, *batch, vj, lo, hi, s);
    });
}

extern "C" int orc_init_flash_batch(const orc_fluid* fluid, const orc_batch* batch, const double* Vpore, int impec,
                                    double* Ni, double* vj, int nthreads, double* seconds)
{
    if (!fluid || !batch || !Vpore || !Ni || fluid->nc < 2 || fluid->nc > ORC_MAX_NC) return 1;
    if (impec && !vj) return 1;
    return run_threads(batch->n, nthreads, seconds,
                       [fluid, batch, Vpore, impec, Ni, vj](int64_t lo, int64_t hi, double* s) {
                           run_chunk_init(*fluid, *batch, Vpore, impec, Ni, vj, lo, hi, s);
                       });
}

// IsoT_FIM::CalKrPc (src/OCPFluidMethod.cpp:1189-1199) or, without
// derivatives, IsoT_IMPEC::CalKrPc, over cells [lo, hi) with one
// FlowUnit_ODGW01 per saturation region of this thread (the tables keep a
// search position, so threads do not share them).
static void run_chunk_krpc(int nreg, const orc_satfunc* reg, const orc_krpc_batch* b, int64_t lo, int64_t hi,
                           double* secs)
{
    ParamReservoir rs;
    auto cols = [](const double* rows, int nrow) {
        std::vector<std::vector<OCP_DBL>> c(4, std::vector<OCP_DBL>(nrow));
        for (int r = 0; r < nrow; r++)
            for (int k = 0; k < 4; k++) c[k][r] = rows[r * 4 + k];
        return c;
    };
    for (int i = 0; i < nreg; i++) {
        rs.SWOF_T.data.push_back(cols(reg[i].swof, reg[i].nrow_swof));
        rs.SGOF_T.data.push_back(cols(reg[i].sgof, reg[i].nrow_sgof));
    }
    std::vector<FlowUnit_ODGW01*> fu;
    for (int i = 0; i < nreg; i++) fu.push_back(new FlowUnit_ODGW01(rs, static_cast<USI>(i)));
    auto t0 = std::chrono::steady_clock::now();
    for (int64_t n = lo; n < hi; n++) {
        const int r = b->satnum ? b->satnum[n] : 0;
        if (b->deriv)
            fu[r]->CalKrPcDeriv(b->S + 3 * n, b->kr + 3 * n, b->Pc + 3 * n, b->dKr_dS + 9 * n, b->dPcj_dS + 9 * n,
                                static_cast<OCP_USI>(n));
        else
            fu[r]->CalKrPc(b->S + 3 * n, b->kr + 3 * n, b->Pc + 3 * n, static_cast<OCP_USI>(n));
        for (int j = 0; j < 3; j++) b->Pj[3 * n + j] = b->P[n] + b->Pc[3 * n + j];
    }
    auto t1 = std::chrono::steady_clock::now();
    *secs   = std::chrono::duration<double>(t1 - t0).count();
    for (auto* f : fu) delete f;
}

extern "C" int orc_krpc(int nreg, const orc_satfunc* reg, const orc_krpc_batch* b, int nthreads, double* seconds)
{
    if (nreg < 1 || !reg || !b || !b->P || !b->S || !b->kr || !b->Pc || !b->Pj) return 1;
    if (b->deriv && (!b->dKr_dS || !b->dPcj_dS)) return 1;
    for (int i = 0; i < nreg; i++)
        if (!reg[i].swof || !reg[i].sgof || reg[i].nrow_swof < 2 || reg[i].nrow_sgof < 2) return 1;
    if (b->satnum)
        for (int64_t n = 0; n < b->n; n++)
            if (b->satnum[n] < 0 || b->satnum[n] >= nreg) return 1;
    return run_threads(b->n, nthreads, seconds, [nreg, reg, b](int64_t lo, int64_t hi, double* s) {
        run_chunk_krpc(nreg, reg, b, lo, hi, s);
    });
}

// The same over FlowUnit_ODGW02 units built from SWFN / SGFN / SOF3 tables
// (src/FlowUnit.cpp:522-535), one per region and thread.
static void run_chunk_krpc_sof3(int nreg, const orc_satfunc3* reg, const orc_krpc_batch* b, int64_t lo,
                                int64_t hi, double* secs)
{
    ParamReservoir rs;
    auto cols = [](const double* rows, int nrow) {
        std::vector<std::vector<OCP_DBL>> c(3, std::vector<OCP_DBL>(nrow));
        for (int r = 0; r < nrow; r++)
            for (int k = 0; k < 3; k++) c[k][r] = rows[r * 3 + k];
        return c;
    };
    for (int i = 0; i < nreg; i++) {
        rs.SWFN_T.data.push_back(cols(reg[i].swfn, reg[i].nrow_swfn));
        rs.SGFN_T.data.push_back(cols(reg[i].sgfn, reg[i].nrow_sgfn));
        rs.SOF3_T.data.push_back(cols(reg[i].sof3, reg[i].nrow_sof3));
    }
    std::vector<FlowUnit_ODGW02*> fu;
    for (int i = 0; i < nreg; i++) fu.push_back(new FlowUnit_ODGW02(rs, static_cast<USI>(i)));
    auto t0 = std::chrono::steady_clock::now();
    for (int64_t n = lo; n < hi; n++) {
        const int r = b->satnum ? b->satnum[n] : 0;
        if (b->deriv)
            fu[r]->CalKrPcDeriv(b->S + 3 * n, b->kr + 3 * n, b->Pc + 3 * n, b->dKr_dS + 9 * n, b->dPcj_dS + 9 * n,
                                static_cast<OCP_USI>(n));
        else
            fu[r]->CalKrPc(b->S + 3 * n, b->kr + 3 * n, b->Pc + 3 * n, static_cast<OCP_USI>(n));
        for (int j = 0; j < 3; j++) b->Pj[3 * n + j] = b->P[n] + b->Pc[3 * n + j];
    }
    auto t1 = std::chrono::steady_clock::now();
    *secs   = std::chrono::duration<double>(t1 - t0).count();
    for (auto* f : fu) delete f;
}

extern "C" int orc_krpc_sof3(int nreg, const orc_satfunc3* reg, const orc_krpc_batch* b, int nthreads,
                             double* seconds)
{
    if (nreg < 1 || !reg || !b || !b->P || !b->S || !b->kr || !b->Pc || !b->Pj) return 1;
    if (b->deriv && (!b->dKr_dS || !b->dPcj_dS)) return 1;
    for (int i = 0; i < nreg; i++)
        if (!reg[i].swfn || !reg[i].sgfn || !reg[i].sof3 || reg[i].nrow_swfn < 2 || reg[i].nrow_sgfn < 2 ||
            reg[i].nrow_sof3 < 2)
            return 1;
    if (b->satnum)
        for (int64_t n = 0; n < b->n; n++)
            if (b->satnum[n] < 0 || b->satnum[n] >= nreg) return 1;
    return run_threads(b->n, nthreads, seconds, [nreg, reg, b](int64_t lo, int64_t hi, double* s) {
        run_chunk_krpc_sof3(nreg, reg, b, lo, hi, s);
    });
}

// The reference's own dense product of the FIM assembly (DaABpbC,
// src/DenseMat.cpp:75-94): C = A B + C, row-major, A m x k, B k x n.
extern "C" void orc_daabpbc(int m, int n, int k, const double* A, const double* B, double* C)
{
    DaABpbC(m, n, k, 1.0, A, B, 1.0, C);
}

extern "C" const char* orc_kind(void) { return "reference"; }

extern "C" int orc_flash_fimn_batch(const orc_fluid* fluid, const orc_batch* batch, double* res, double* resPc,
                                    int nthreads, double* seconds)
{
    if (!fluid || !batch || !res || !resPc || fluid->nc < 2 || fluid->nc > ORC_MAX_NC) return 1;
    return run_threads(batch->n, nthreads, seconds, [fluid, batch, res, resPc](int64_t lo, int64_t hi, double* s) {
        run_chunk_fimn(*fluid, *batch, res, resPc, lo, hi, s);
    });
}

extern "C" int orc_init_flash_fimn_batch(const orc_fluid* fluid, const orc_batch* batch, const double* Vpore,
                                         double* Ni, double* res, double* resPc, int nthreads, double* seconds)
{
    if (!fluid || !batch || !Vpore || !Ni || !res || !resPc || fluid->nc < 2 || fluid->nc > ORC_MAX_NC) return 1;
    return run_threads(batch->n, nthreads, seconds,
                       [fluid, batch, Vpore, Ni, res, resPc](int64_t lo, int64_t hi, double* s) {
                           run_chunk_init_fimn(*fluid, *batch, Vpore, Ni, res, resPc, lo, hi, s);
                       });
}
