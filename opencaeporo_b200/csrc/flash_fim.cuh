// flash_fim.cuh -- MixtureComp::FlashFIM for one cell on one thread
// (src/MixtureComp.cpp:494-573) and the copy-out of IsoT_FIM::PassFlashValue
// (src/OCPFluidMethod.cpp:1122-1187) into structure-of-arrays outputs.
#pragma once

#include "flash_cell.cuh"

namespace ocpf {

// Which of the reference's flash entry points a launch runs (bit flags):
// FlashFIM, FlashIMPEC, FlashFIMn (FM_FIMN), InitFlashFIM (FM_INIT),
// InitFlashIMPEC (FM_INIT | FM_IMPEC) or InitFlashFIMn (FM_INIT | FM_FIMN).
enum : int { FM_FIM = 0, FM_IMPEC = 1, FM_INIT = 2, FM_FIMN = 4 };

// The entry point of a launch and the arrays beyond ocpf_fim_in/out that it
// reads or writes. With FM_INIT, ocpf_fim_in.Ni holds the mole fractions z
// and ocpf_fim_in.S the initial saturations; lastNP and xij are not read.
struct FlashTail {
    int           mode;
    double*       vj;     // [3][n] phase volumes (FM_IMPEC), or null
    const double* vpore;  // [n] pore volumes, ft3 (FM_INIT)
    double*       ni;     // [numCom][n] moles after the flash (FM_INIT); may alias in.Ni
    double*       res;    // [3 (numCom + 1)][n] FlashFIMn's residual terms, first rows written (FM_FIMN)
    double*       resPc;  // [n] (FM_FIMN)
};

template <int NC>
struct FimCell : CellFlash<NC> {
    using Base = CellFlash<NC>;
    using Base::F;
    using Base::NUMCOM;
    using Base::NCOL;
    using Base::P;
    using Base::T;
    using Base::Nh;
    using Base::Ni;
    using Base::zi;
    using Base::Ai;
    using Base::Bi;
    using Base::sA;
    using Base::NP;
    using Base::lNP;
    using Base::ftype;
    using Base::flagSkip;
    using Base::nu;
    using Base::x;
    using Base::Aj;
    using Base::Bj;
    using Base::Zj;
    using Base::lKs;
    using Base::n;
    using Base::status;
    using Base::omb;

    double Sw0 = 0, Vp0 = 0;  // initial water saturation and pore volume (FM_INIT)

    __device__ __forceinline__ explicit FimCell(const FluidConst& f) : Base(f) {}

    // SkipStaAnaly::CalFtypeFIM / CalFtypeIMPEC / IfSkip,
    // src/AcceleratePVT.cpp:54-120 (IMPEC has no two-phase warm type 2)
    __device__ __forceinline__ int cal_ftype(const double* Sin, bool skflag, double skEig, double skP,
                                             double skT, const double* skz, bool impec = false) const
    {
        if (!F.use_skip) return 0;
        bool skip = false;
        if (skflag) {
            skip = true;
            if (fabs(1 - skP / P) >= skEig / 10) skip = false;
            if (fabs(skT - T) >= skEig * 10) skip = false;
#pragma unroll
            for (int i = 0; i < NC; i++)
                if (fabs(Ni[i] / Nh - skz[i]) >= skEig / 10) skip = false;
        }
        if (skip) return 1;
        if (impec) return 0;
        if (lNP >= 2) {
            if (Sin[0] < 1e-4 || Sin[1] < 1e-4) return 0;
            return 2;
        }
        return 0;
    }

    // Min eigenvalue of the skip-test matrix of the single phase,
    // CalPhiNSkip + AssembleSkipMatSTA + CalEigenSY (src/MixtureComp.cpp:5155-5232)
    __device__ double skip_min_eig() const
    {
        const double  aj = Aj[0], bj = Bj[0], zj = Zj[0], nu0 = nu[0];
        const double* xj = x[0];
        double        t[NC], An[NC], Bn[NC], Zn[NC];
        {
            double w[NC];
#pragma unroll
            for (int k = 0; k < NC; k++) w[k] = sA[k] * xj[k];
#pragma unroll
            for (int i = 0; i < NC; i++) {
                double s = 0;
#pragma unroll
                for (int k = 0; k < NC; k++) s += omb(i, k) * w[k];
                t[i] = sA[i] * s;
            }
        }
        const DzCoef dz(aj, bj, zj);
        const double inu = 1.0 / nu0;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            An[i] = 2 * inu * (t[i] - aj);
            Bn[i] = inu * (Bi[i] - bj);
            Zn[i] = dz(An[i], Bn[i]);
        }
        const double zmb  = zj - bj;
        const double G    = (zj + D1 * bj) / (zj + D2 * bj);
        const double lnG  = log(G);
        const double ib   = 1.0 / bj;
        const double zd2  = zj + D2 * bj;
        const double gfac = D1MD2 / (zd2 * zd2);
        const double efac = -1 / D1MD2 * (ib * ib);
        float        A[NC][NC];
#pragma unroll
        for (int i = 0; i < NC; i++) {
            const double E = -aj / (D1MD2 * bj) * (2 * t[i] / aj - Bi[i] * ib);
#pragma unroll
            for (int k = 0; k <= i; k++) {
                const double a_ik = omb(i, k) * sA[i] * sA[k];
                const double Cnk  = (Bn[k] - Zn[k]) / (zmb * zmb);
                const double Dnk  = Bi[i] * ib * (Zn[k] - (Bi[k] - bj) * (zj - 1) * inu * ib);
                const double Gnk  = gfac * (Bn[k] * zj - Zn[k] * bj);
                double       Enk  = efac * (2 * (bj * a_ik * inu + Bn[k] * (Bi[i] * aj * ib - t[i])) -
                                   An[k] * Bi[i] - aj * Bi[i] * inu);
                Enk -= E * inu;
                const double phiN = zmb * Cnk + Dnk + Enk * lnG + E / G * Gnk;
                A[i][k] = (float)(dlt(i, k) + nu0 * sqrt(xj[i] * xj[k]) * phiN);
                A[k][i] = A[i][k];
            }
        }
        return (double)min_eig_sym<NC>(A);
    }

    // Reads cell n_'s inputs (SoA with field stride `stride`) and decides the
    // flash type: FlashFIM up to CalFtypeFIM (src/MixtureComp.cpp:501-515),
    // with FM_IMPEC FlashIMPEC up to CalFtypeIMPEC (:451-461; S is not
    // read), with FM_INIT InitFlashFIM / InitFlashIMPEC up to InitPTZ
    // (:261-275, :195-209: flash type 0, no last phase count, z read as
    // given). Everything is read before any output is written, so the caller
    // may pass the same xij, S (and, with FM_INIT, z and Ni) arrays in and out.
    __device__ __forceinline__ void load_inputs(int64_t n_, int64_t stride, const ocpf_fim_in& in,
                                                const ocpf_skip& sk, const FlashTail& tl)
    {
        const int64_t N = stride;
        auto at = [N, n_](int f) { return (int64_t)f * N + n_; };
        const double Pin = in.P[n_];
        const double Tin = in.T[n_];
        this->it_ssmsta = this->it_nrsta = this->it_ssmsp = this->it_nrsp = this->it_rr = 0;
        status                                                                        = 0;
        this->ssmsta_conflag = this->nrsta_conflag = this->ssmsp_conflag = this->nrsp_conflag = false;
        this->ssmsta_realTol = this->nrsta_realTol = this->ssmsp_realTol = this->nrsp_realTol = 0;
        this->Yt                                                                      = 0;
        if (tl.mode & FM_INIT) {
            // InitPTZ, include/MixtureComp.hpp:171-176; Nh is set by the tail
            P  = Pin;
            T  = Tin + CONV5;
            Nh = 1;
#pragma unroll
            for (int i = 0; i < NC; i++) zi[i] = in.Ni[at(i)];
            Sw0   = in.S[at(2)];
            Vp0   = tl.vpore[n_];
            lNP   = 0;
            ftype = 0;
            return;
        }
        const bool impec = (tl.mode & FM_IMPEC) != 0;
#pragma unroll
        for (int i = 0; i < NUMCOM; i++) Ni[i] = in.Ni[at(i)];
        double Sin[2] = {0, 0};
        if (!impec) {
            Sin[0] = in.S[at(0)];
            Sin[1] = in.S[at(1)];
        }
        const uint32_t lastNP = in.lastNP[n_];
        lNP                   = lastNP > 0 ? (int)lastNP - 1 : 0;
        if (lNP == 2) {
#pragma unroll
            for (int i = 0; i < NC; i++) lKs[i] = in.xij[at(i)] / in.xij[at(i + NUMCOM)];
        }
        bool   skflag = false;
        double skEig = 0, skP = 0, skT = 0, skz[NC];
        if (F.use_skip) {
            skflag = sk.flag[n_] != 0;
            skEig  = sk.minEig[n_];
            skP    = sk.P[n_];
            skT    = sk.T[n_];
#pragma unroll
            for (int i = 0; i < NC; i++) skz[i] = sk.z[at(i)];
        }


        // InitPTN, include/MixtureComp.hpp:177-184
        P  = Pin;
        T  = Tin + CONV5;
        Nh = 0;
#pragma unroll
        for (int i = 0; i < NC; i++) Nh += fabs(Ni[i]);
#pragma unroll
        for (int i = 0; i < NC; i++) zi[i] = Ni[i] / Nh;

        ftype = cal_ftype(Sin, skflag, skEig, skP, skT, skz, impec);
    }

    // The whole flash of one cell on this thread (FlashFIM, FlashIMPEC,
    // InitFlashFIM or InitFlashIMPEC by tl.mode; FlashFIMn or InitFlashFIMn
    // with FIMN, which kernels of their own instantiate so that the FIMn tail
    // adds no registers to the others).
    template <bool FIMN = false>
    __device__ void run(int64_t n_, int64_t stride, const ocpf_fim_in& in, const ocpf_skip& sk,
                        const ocpf_fim_out& out, const FlashTail& tl)
    {
        load_inputs(n_, stride, in, sk, tl);
        this->phase_equilibrium();
        finalize<FIMN>(n_, stride, sk, out, tl);
    }

    // Everything after PhaseEquilibrium: CalFlash's property tail, the
    // derivatives, the water block, dXsdXp, the partials, the skip cache and
    // the copy-out of PassFlashValue. Needs load_inputs' state, cal_ai_bi's
    // Ai/Bi and the equilibrium (NP, x, nu as phase fractions, Aj/Bj/Zj of
    // each phase, n from the split, flagSkip, ePEC, counters, status).
    // With FM_IMPEC, FlashIMPEC's tail instead (src/MixtureComp.cpp:462-491)
    // and IsoT_IMPEC::PassFlashValue's outputs (src/OCPFluidMethod.cpp:
    // 275-305): no dXsdXp and no property partials; the phase volumes vj go
    // to tl.vj. With FM_INIT, the tails of InitFlashFIM / InitFlashIMPEC
    // (:276-353, :210-258): the properties are formed per mole of
    // hydrocarbon, then Nh = Vpore (1 - S_w) / vf scales the phase moles and
    // volumes, Ni = z Nh and N_w = Vpore S_w xi_w, and Ni goes to tl.ni.
    // With FIMN, FlashFIMn's tail (finalize_fimn) after the common part.
    template <bool FIMN = false>
    __device__ void finalize(int64_t n_, int64_t stride, const ocpf_skip& sk, const ocpf_fim_out& out,
                             const FlashTail& tl)
    {
        const int64_t N = stride;
        auto at = [N, n_](int f) { return (int64_t)f * N + n_; };
        const bool impec = (tl.mode & FM_IMPEC) != 0;
        const bool init  = (tl.mode & FM_INIT) != 0;

        // ---- CalFlash, src/MixtureComp.cpp:697-708 (after PhaseEquilibrium);
        // the initialisation keeps nu as phase fractions here
        if (!init) {
#pragma unroll
            for (int j = 0; j < 2; j++)
                if (j < NP) nu[j] *= Nh;
        }

        double MW[2], vC[2], xiC[2], rhoC[2], muC[2], muA[2][5];
        // CalMW, src/MixtureComp.cpp:1147-1156
#pragma unroll
        for (int j = 0; j < 2; j++) {
            MW[j] = 0;
#pragma unroll
            for (int i = 0; i < NC; i++) MW[j] += x[j][i] * F.MW[i];
        }
        // CalVfXiRho, src/MixtureComp.cpp:1158-1176
        double vf = 0;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            if (j < NP) {
                double tmp = Zj[j] * GAS_CONSTANT * T / P;
#pragma unroll
                for (int i = 0; i < NC; i++) tmp -= x[j][i] * F.Vshift[i];
                vC[j] = tmp * nu[j];
                vf += vC[j];
                xiC[j]  = 1 / tmp;
                rhoC[j] = MW[j] * xiC[j];
            }
        }
        // LBC temperature factors (T only), shared by CalViscoLBC and the mu partials
        double gT[NC];
#pragma unroll
        for (int i = 0; i < NC; i++) {
            const double Tri = T / F.Tc[i];
            gT[i] = (Tri <= 1.5) ? 34 * 1e-5 * pow(Tri, 0.94) : 17.78 * 1e-5 * pow((4.58 * Tri - 1.67), 0.625);
        }
        // CalViscoLBC, src/MixtureComp.cpp:2402-2446
        const double* L = F.L;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            if (j < NP) {
                const double sqMW = sqrt(MW[j]);
                double       m0 = 0, m1 = 0, xT = 0, xP = 0, xV = 0;
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    const double tmp = gT[i] / (F.lbc1[i] / sqMW / F.lbc2[i]);
                    m0 += x[j][i] * F.sqrtMW[i] * tmp;
                    m1 += x[j][i] * F.sqrtMW[i];
                    xT += x[j][i] * F.Tc[i];
                    xP += x[j][i] * F.Pc[i];
                    xV += x[j][i] * F.Vcvis[i];
                }
                muA[j][0] = m0;
                muA[j][1] = m1;
                muA[j][2] = 5.4402 * pow(xT, 1.0 / 6) / sqMW / pow(xP, 2.0 / 3);
                muA[j][3] = xiC[j] * xV;
                const double u = muA[j][3];
                muA[j][4]      = u * (u * (u * (L[4] * u + L[3]) + L[2]) + L[1]) + L[0];
                muC[j]         = muA[j][0] / muA[j][1] + 1e-4 * (pow(muA[j][4], 4) - 1) / muA[j][2];
            }
        }
        // IdentifyPhase, src/MixtureComp.cpp:2352-2384
        int  label[2];
        bool exist[NPH];
        exist[0] = exist[1] = false;
        exist[2]            = true;
        if (NP == 1) {
            double A = 0, B = 0;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                A += x[0][i] * F.Vc[i] * F.Tc[i];
                B += x[0][i] * F.Vc[i];
            }
            if (T > A / B) {
                label[0] = 1;
                exist[1] = true;
            } else {
                label[0] = 0;
                exist[0] = true;
            }
            label[1] = 1 - label[0];
        } else {
            if (MW[0] > MW[1]) {
                label[0] = 0;
                label[1] = 1;
            } else {
                label[0] = 1;
                label[1] = 0;
            }
            exist[0] = exist[1] = true;
        }
        // CopyPhase's nj (src/MixtureComp.cpp:2386-2398): the phase moles, or
        // in the initialisation the phase fractions (nu is rescaled after it)
        const double njC[2] = {nu[0], nu[1]};
        if (init) {
            // InitFlashFIM, src/MixtureComp.cpp:282-297 (InitFlashIMPEC :216-229)
            Nh = Vp0 * (1 - Sw0) / vf;
#pragma unroll
            for (int j = 0; j < 2; j++) {
                if (j < NP) {
                    nu[j] *= Nh;
                    vC[j] *= Nh;
                }
            }
            vf *= Nh;
#pragma unroll
            for (int i = 0; i < NC; i++) Ni[i] = zi[i] * Nh;
        }
        if constexpr (FIMN) {
            finalize_fimn(n_, stride, sk, out, tl, label, exist, MW, vC, xiC, rhoC, muC, muA, gT, njC, vf);
            return;
        }

        // ---- CalVfiVfp_full02, src/MixtureComp.cpp:3911-3989
        const double CgTP = GAS_CONSTANT * T / P;
        double       vfi[NUMCOM];
        double       vfP;
        double       Zp[2];
        double       vjpI[2] = {0, 0};         // dv_j/dP of hydrocarbon phase j (internal order)
        double       vjiI[2][NC];              // dv_j/dN_i
        double       X[NC][NC + 1];            // d n_k0 / d(P, N_1..N_nc)
        if (NP == 1) {
            const double aj = Aj[0], bj = Bj[0], zj = Zj[0], nu0 = nu[0];
            double       t[NC];
            {
                double w[NC];
#pragma unroll
                for (int k = 0; k < NC; k++) w[k] = sA[k] * x[0][k];
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    double s = 0;
#pragma unroll
                    for (int k = 0; k < NC; k++) s += omb(i, k) * w[k];
                    t[i] = sA[i] * s;
                }
            }
            const DzCoef dz(aj, bj, zj);
            const double inu = 1.0 / nu0;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                const double Zn = dz(2 * inu * (t[i] - aj), inu * (Bi[i] - bj));
                vfi[i]          = CgTP * (zj + nu0 * Zn) - F.Vshift[i];
            }
            Zp[0] = (dz.bmz * aj + dz.num_b * bj) / P * dz.inv_den;
            vfP   = CgTP * nu0 * (Zp[0] - zj / P);
        } else {
            double Sm[NC][NC], R1[NC][NC], Zn0[NC], Zn1[NC];
            this->fugn_phase(0, Sm, false, nullptr, Zn0);
            this->fugn_phase(1, Sm, true, R1, Zn1);
            // CalFugPAll, src/MixtureComp.cpp:2519-2579
            double fugP[2][NC];
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const double aj = Aj[j], bj = Bj[j], zj = Zj[j];
                const double Ap = aj / P, Bp = bj / P;
                const DzCoef dz(aj, bj, zj);
                Zp[j]            = dz(Ap, Bp);
                const double G   = (zj + D1 * bj) / (zj + D2 * bj);
                const double zd2 = zj + D2 * bj;
                const double Gp  = D1MD2 / (zd2 * zd2) * (Bp * zj - Zp[j] * bj);
                double       t[NC];
                {
                    double w[NC];
#pragma unroll
                    for (int k = 0; k < NC; k++) w[k] = sA[k] * x[j][k];
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        double s = 0;
#pragma unroll
                        for (int k = 0; k < NC; k++) s += omb(i, k) * w[k];
                        t[i] = sA[i] * s;
                    }
                }
                const double zmb = zj - bj;
                const double Cp  = (zmb - P * (Zp[j] - Bp)) / (zmb * zmb);
                const double iC  = zmb / P;
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    const double E  = -aj / (D1MD2 * bj) * (2 * t[i] / aj - Bi[i] / bj);
                    const double Dp = Bi[i] / bj * Zp[j];
                    fugP[j][i]      = Cp * iC + Dp + E / G * Gp;
                }
            }
            // LU solve with NC+1 right-hand sides (dgesv), src/MixtureComp.cpp:3948
#pragma unroll
            for (int i = 0; i < NC; i++) {
                X[i][0] = fugP[1][i] - fugP[0][i];
#pragma unroll
                for (int k = 0; k < NC; k++) X[i][k + 1] = R1[k][i];
            }
            if (!gauss_solve<NC, NC + 1>(Sm, X)) {
                status |= ST_SINGULAR;  // dgesv leaves the right-hand sides unchanged
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    X[i][0] = fugP[1][i] - fugP[0][i];
#pragma unroll
                    for (int k = 0; k < NC; k++) X[i][k + 1] = R1[k][i];
                }
            }
            double v0[NC], v1[NC];
#pragma unroll
            for (int k = 0; k < NC; k++) {
                v0[k] = CgTP * (Zj[0] + nu[0] * Zn0[k]) - F.Vshift[k];
                v1[k] = CgTP * (Zj[1] + nu[1] * Zn1[k]) - F.Vshift[k];
            }
            vjpI[0] = CgTP * nu[0] * (Zp[0] - Zj[0] / P);
            vjpI[1] = CgTP * nu[1] * (Zp[1] - Zj[1] / P);
#pragma unroll
            for (int k = 0; k < NC; k++) {
                vjpI[0] += v0[k] * X[k][0];
                vjpI[1] -= v1[k] * X[k][0];
            }
            vfP = vjpI[0] + vjpI[1];
#pragma unroll
            for (int i = 0; i < NC; i++) {
                double a0 = 0, a1 = 0;
#pragma unroll
                for (int k = 0; k < NC; k++) {
                    a0 += v0[k] * X[k][i + 1];
                    a1 += v1[k] * (dlt(i, k) - X[k][i + 1]);
                }
                vjiI[0][i] = a0;
                vjiI[1][i] = a1;
                vfi[i]     = a0 + a1;
            }
        }

        // ---- water, src/MixtureComp.cpp:517-546 (single-row PVTW: zero slopes);
        // the initialisation fills the water from the pore volume (:314)
        const double bw  = F.pvtw[1] * (1 - F.pvtw[2] * (P - F.pvtw[0]));
        const double bwp = -F.pvtw[2] * F.pvtw[1];
        const double xiW = 1 / (CONV1 * bw);
        if (init) Ni[NC] = Vp0 * Sw0 * xiW;
        const double Nw  = Ni[NC];
        const double Nt  = Nh + Nw;
        const double xiPW = -bwp / (bw * bw * CONV1);
        const double vw  = CONV1 * Nw * bw;
        vfi[NC]          = CONV1 * bw;
        const double vwp = CONV1 * Nw * bwp;
        vf += vw;
        vfP += vwp;

        // CalSaturation, src/MixtureComp.cpp:1178-1186
        double vj[NPH] = {0, 0, vw};
#pragma unroll
        for (int j = 0; j < 2; j++)
            if (j < NP) vj[label[j]] = vC[j];
        double S[NPH];
#pragma unroll
        for (int j = 0; j < NPH; j++) S[j] = exist[j] ? vj[j] / vf : 0;

        // ---- outputs of PassFlashValue: S, flags, per-phase properties
#pragma unroll
        for (int j = 0; j < NPH; j++) {
            out.S[at(j)]          = S[j];
            out.phaseExist[at(j)] = exist[j] ? 1u : 0u;
        }
        out.phaseNum[n_] = (uint32_t)(NP + 1);
        out.Nt[n_]       = Nt;
        out.vf[n_]       = vf;
        out.vfP[n_]      = vfP;
#pragma unroll
        for (int i = 0; i < NUMCOM; i++) out.vfi[at(i)] = vfi[i];
        if (tl.vj) {
#pragma unroll
            for (int j = 0; j < NPH; j++)
                if (exist[j]) tl.vj[at(j)] = vj[j];
        }
        if (init && tl.ni) {
#pragma unroll
            for (int i = 0; i < NUMCOM; i++) tl.ni[at(i)] = Ni[i];
        }
        if (impec) {
            finalize_impec(n_, stride, sk, out, label, exist, xiC, rhoC, muC, njC, bw, xiW, S, vf, vfP);
            return;
        }

        // ---- CaldXsdXpAPI02p, src/MixtureComp.cpp:4386-4493 (compact rows)
        const double vf2  = vf * vf;
        double*      dsd  = out.dSec_dPri;
        auto         dput = [&](int r, int c, double v) { dsd[at(r * NCOL + c)] = v; };
        uint32_t     rows;
        if (NP == 1) {
            const int    j1 = label[0];
            const double r0 = ((vfP - vwp) * vf - vfP * vj[j1]) / vf2;
            dput(0, 0, r0);
            dput(1, 0, -r0);
#pragma unroll
            for (int m = 0; m < NC; m++) {
                const double v = vfi[m] * vw / vf2;
                dput(0, 1 + m, v);
                dput(1, 1 + m, -v);
            }
            const double rw = -vfi[NC] * vj[j1] / vf2;
            dput(0, NC + 1, rw);
            dput(1, NC + 1, -rw);
#pragma unroll
            for (int i = 0; i < NC; i++) {
                dput(2 + i, 0, 0.0);
#pragma unroll
                for (int m = 0; m < NC; m++) dput(2 + i, 1 + m, (dlt(i, m) * Nh - Ni[i]) / (Nh * Nh));
                dput(2 + i, NC + 1, 0.0);
            }
            rows = NC + 2;
        } else {
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int j1 = label[j];
                dput(j1, 0, (vjpI[j] * vf - vfP * vj[j1]) / vf2);
#pragma unroll
                for (int m = 0; m < NC; m++) dput(j1, 1 + m, (vjiI[j][m] * vf - vfi[m] * vj[j1]) / vf2);
                dput(j1, NC + 1, (0.0 * vf - vfi[NC] * vj[j1]) / vf2);
            }
            dput(2, 0, (vwp * vf - vfP * vw) / vf2);
#pragma unroll
            for (int m = 0; m < NC; m++) dput(2, 1 + m, (0.0 * vf - vfi[m] * vw) / vf2);
            dput(2, NC + 1, (vfi[NC] * vf - vfi[NC] * vw) / vf2);
            const int r0 = 3 + label[0] * NC;
            const int r1 = 3 + label[1] * NC;
            double    sumP = 0;
#pragma unroll
            for (int i = 0; i < NC; i++) sumP += X[i][0];
            const double nu0 = nu[0], nu1 = nu[1];
#pragma unroll
            for (int i = 0; i < NC; i++) {
                dput(r0 + i, 0, (X[i][0] * nu0 - sumP * Nh * n[0][i]) / (nu0 * nu0));
                dput(r1 + i, 0, (-X[i][0] * nu1 + sumP * Nh * n[1][i]) / (nu1 * nu1));
                dput(r0 + i, NC + 1, 0.0);
                dput(r1 + i, NC + 1, 0.0);
            }
#pragma unroll
            for (int m = 0; m < NC; m++) {
                double s = 0;
#pragma unroll
                for (int i = 0; i < NC; i++) s += X[i][m + 1];
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    dput(r0 + i, 1 + m, (X[i][m + 1] * nu0 - s * Nh * n[0][i]) / (nu0 * nu0));
                    dput(r1 + i, 1 + m,
                         ((dlt(i, m) - X[i][m + 1]) * nu1 - (1 - s) * Nh * n[1][i]) / (nu1 * nu1));
                }
            }
            rows = 3 + 2 * NC;
        }
        out.bRowSizedSdP[n_] = rows;

        // ---- CalXiPNX_partial, CalRhoPX_partial, CalMuPXLBC_partial
        // (src/MixtureComp.cpp:3037-3213), written with CopyPhase's values
#pragma unroll
        for (int j = 0; j < 2; j++) {
            if (j < NP) {
                const int    j1 = label[j];
                const double aj = Aj[j], bj = Bj[j], zj = Zj[j];
                double       t[NC];
                {
                    double w[NC];
#pragma unroll
                    for (int k = 0; k < NC; k++) w[k] = sA[k] * x[j][k];
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        double s = 0;
#pragma unroll
                        for (int k = 0; k < NC; k++) s += omb(i, k) * w[k];
                        t[i] = sA[i] * s;
                    }
                }
                const DzCoef dz(aj, bj, zj);
                const double m2  = -xiC[j] * xiC[j];
                const double xiP = m2 * CgTP * (Zp[j] - Zj[j] / P);
                double       xix[NC];
#pragma unroll
                for (int i = 0; i < NC; i++) xix[i] = m2 * (CgTP * dz(2 * t[i], Bi[i]) - F.Vshift[i]);
                // LBC partials
                double xT = 0, xP = 0, xV = 0;
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    xT += x[j][i] * F.Tc[i];
                    xP += x[j][i] * F.Pc[i];
                    xV += x[j][i] * F.Vcvis[i];
                }
                const double u    = muA[j][3];
                const double poly = L[1] + u * (2 * L[2] + u * (3 * L[3] + u * 4 * L[4]));
                const double m4_3 = pow(muA[j][4], 3);
                const double m4_4 = pow(muA[j][4], 4);
                const double muP  = (4 * 1e-4) * m4_3 * (xV * xiP * poly) / muA[j][2];
                const double sqMW = sqrt(MW[j]);
                const double pT16 = pow(xT, 1.0 / 6), pT56 = pow(xT, -5.0 / 6), pP23 = pow(xP, 2.0 / 3);

                out.rho[at(j1)]  = rhoC[j];
                out.xi[at(j1)]   = xiC[j];
                out.mu[at(j1)]   = muC[j];
                out.xiP[at(j1)]  = xiP;
                out.rhoP[at(j1)] = xiP * MW[j];
                out.muP[at(j1)]  = muP;
                if (out.nj) out.nj[at(j1)] = njC[j];
#pragma unroll
                for (int k = 0; k < NC; k++) {
                    const int    o     = j1 * NUMCOM + k;
                    const double val1  = F.muAux1I[k] / sqMW;
                    const double der3  = F.sqrtMW[k] * (gT[k] / val1);
                    const double der4  = F.sqrtMW[k];
                    const double der6  = 5.4402 *
                                        (1.0 / 6 * pT56 * F.Tc[k] -
                                         pT16 * (0.5 / MW[j] * F.MW[k] + 2.0 / 3 / xP * F.Pc[k])) /
                                        (sqMW * pP23);
                    const double der7  = xix[k] * xV + xiC[j] * F.Vcvis[k];
                    const double der8  = der7 * poly;
                    const double mux   = (der3 * muA[j][1] - muA[j][0] * der4) / (muA[j][1] * muA[j][1]) +
                                       1e-4 * (4 * m4_3 * der8 * muA[j][2] - (m4_4 - 1) * der6) /
                                           (muA[j][2] * muA[j][2]);
                    out.xij[at(o)]  = x[j][k];
                    out.xix[at(o)]  = xix[k];
                    out.rhox[at(o)] = xix[k] * MW[j] + xiC[j] * F.MW[k];
                    out.mux[at(o)]  = mux;
                }
                const int ow     = j1 * NUMCOM + NC;  // water component of a hydrocarbon phase
                out.xij[at(ow)]  = 0.0;
                out.xix[at(ow)]  = 0.0;
                out.rhox[at(ow)] = 0.0;
                out.mux[at(ow)]  = 0.0;
            }
        }
        finish_fim(n_, stride, sk, out, exist, bw, xiW, xiPW, Nw, vf, vfP, S);
    }

    // FlashFIMn's tail after CalFlash (src/MixtureComp.cpp:627-694; with
    // FM_INIT, InitFlashFIMn's after the moles are scaled, :390-441) and
    // IsoT_FIMn::PassFlashValue's outputs (src/OCPFluidMethod.cpp:3179-3196).
    // The secondary variables are the saturations and the phase moles n_ij:
    // dSec_dPri holds dS/d(P, N) and dn_ij/d(P, N) (CaldXsdXpAPI03,
    // :4495-4631), the property partials are taken per n_ij, and the solve's
    // residual column goes to tl.res / tl.resPc.
    //
    // CaldXsdXp03 (:4633-4820) solves, by LU with partial pivoting, the
    // (3 + 2 nc)-square system of the saturation definitions, the fugacity
    // equalities and the component balances in the unknowns (S_0, S_1, S_w,
    // n_0, n_1). The saturation unknowns appear only in their own equations
    // (coefficient -1), so the first three pivots are those rows, they leave
    // the others unchanged, and the rest is the LU of the 2 nc-square
    // phase-mole block with its rows in the order the three row swaps leave
    // them. Here that block is solved so (one right-hand side per column: P,
    // N_1..N_nc, the residual; N_w moves no n_ij), then the saturation rows
    // by back substitution. (Eliminating n_1 = N - n_0 first, as FlashFIM's
    // derivatives do, gives the nc-square system fugN_0 + fugN_1, which is
    // far worse conditioned near the critical point.)
    __device__ void finalize_fimn(int64_t n_, int64_t stride, const ocpf_skip& sk, const ocpf_fim_out& out,
                                  const FlashTail& tl, const int* label, const bool* exist, const double* MW,
                                  const double* vC, const double* xiC, const double* rhoC, const double* muC,
                                  const double (*muA)[5], const double* gT, const double* njC, double vf)
    {
        const int64_t N = stride;
        auto at = [N, n_](int f) { return (int64_t)f * N + n_; };
        const bool   init = (tl.mode & FM_INIT) != 0;
        const double CgTP = GAS_CONSTANT * T / P;

        // ---- CalVjpVfpVfn_partial, src/MixtureComp.cpp:2581-2626 (internal
        // phase order; the reference files vji and vjp by phase label)
        double vji[2][NC], vjp[2] = {0, 0}, Zn[2][NC], Zp[2] = {0, 0};
        double vfP = 0;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            if (j < NP) {
                const double aj = Aj[j], bj = Bj[j], zj = Zj[j];
                double       t[NC];
                {
                    double w[NC];
#pragma unroll
                    for (int k = 0; k < NC; k++) w[k] = sA[k] * x[j][k];
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        double s = 0;
#pragma unroll
                        for (int k = 0; k < NC; k++) s += omb(i, k) * w[k];
                        t[i] = sA[i] * s;
                    }
                }
                const DzCoef dz(aj, bj, zj);
                const double inu = 1.0 / nu[j];
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    Zn[j][i]  = dz(2 * inu * (t[i] - aj), inu * (Bi[i] - bj));
                    vji[j][i] = CgTP * (zj + nu[j] * Zn[j][i]) - F.Vshift[i];
                }
                Zp[j]  = (dz.bmz * aj + dz.num_b * bj) / P * dz.inv_den;
                vjp[j] = CgTP * nu[j] * (Zp[j] - zj / P);
                vfP += vjp[j];
            }
        }

        // ---- water, src/MixtureComp.cpp:629-656 (InitFlashFIMn :392-418)
        const double bw   = F.pvtw[1] * (1 - F.pvtw[2] * (P - F.pvtw[0]));
        const double bwp  = -F.pvtw[2] * F.pvtw[1];
        const double xiW  = 1 / (CONV1 * bw);
        if (init) Ni[NC] = Vp0 * Sw0 * xiW;
        const double Nw   = Ni[NC];
        const double Nt   = Nh + Nw;
        const double xiPW = -bwp / (bw * bw * CONV1);
        const double vw   = CONV1 * Nw * bw;
        const double vfiW = CONV1 * bw;
        const double vwp  = CONV1 * Nw * bwp;
        vf += vw;
        vfP += vwp;

        // CalSaturation, src/MixtureComp.cpp:1178-1186
        double vj[NPH] = {0, 0, vw};
#pragma unroll
        for (int j = 0; j < 2; j++)
            if (j < NP) vj[label[j]] = vC[j];
        double S[NPH];
#pragma unroll
        for (int j = 0; j < NPH; j++) S[j] = exist[j] ? vj[j] / vf : 0;
#pragma unroll
        for (int j = 0; j < NPH; j++) {
            out.S[at(j)]          = S[j];
            out.phaseExist[at(j)] = exist[j] ? 1u : 0u;
        }
        out.phaseNum[n_] = (uint32_t)(NP + 1);
        out.Nt[n_]       = Nt;
        out.vf[n_]       = vf;
        if (init && tl.ni) {
#pragma unroll
            for (int i = 0; i < NUMCOM; i++) tl.ni[at(i)] = Ni[i];
        }

        // ---- CaldXsdXpAPI03 and CalVfiVfp_full03 (src/MixtureComp.cpp:4822-4848)
        const double vf2  = vf * vf;
        double*      dsd  = out.dSec_dPri;
        auto         dput = [&](int r, int c, double v) { dsd[at(r * NCOL + c)] = v; };
        double       vfi[NUMCOM];
        double       resPc = 0;
        uint32_t     rows;
        if (NP == 1) {
            const int    j0 = label[0];
            const double r0 = ((vfP - vwp) * vf - vfP * vj[j0]) / vf2;
            dput(0, 0, r0);
            dput(1, 0, -r0);
#pragma unroll
            for (int m = 0; m < NC; m++) {
                const double v = vji[0][m] * vw / vf2;
                dput(0, 1 + m, v);
                dput(1, 1 + m, -v);
            }
            const double rw = -vfiW * vj[j0] / vf2;
            dput(0, NC + 1, rw);
            dput(1, NC + 1, -rw);
#pragma unroll
            for (int i = 0; i < NC; i++)
#pragma unroll
                for (int c = 0; c < NCOL; c++) dput(2 + i, c, c == 1 + i ? 1.0 : 0.0);
            rows = NC + 2;
#pragma unroll
            for (int r = 0; r < NC + 2; r++) tl.res[at(r)] = 0.0;
            // CalVfiVfp_full03: vfP unchanged, vfi = vji
#pragma unroll
            for (int i = 0; i < NC; i++) vfi[i] = vji[0][i];
        } else {
            // fugN of both phases (CalFugNAll, :2168-2251) and fugP (CalFugPAll,
            // :2519-2579, with CalVjpVfpVfn_partial's Zp)
            double A0[NC][NC], A1[NC][NC], Zt[NC];
            this->fugn_phase(0, A0, false, nullptr, Zt);
            this->fugn_phase(1, A1, false, nullptr, Zt);
            double fugP[2][NC];
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const double aj = Aj[j], bj = Bj[j], zj = Zj[j];
                const double Bp  = bj / P;
                const double G   = (zj + D1 * bj) / (zj + D2 * bj);
                const double zd2 = zj + D2 * bj;
                const double Gp  = D1MD2 / (zd2 * zd2) * (Bp * zj - Zp[j] * bj);
                double       t[NC];
                {
                    double w[NC];
#pragma unroll
                    for (int k = 0; k < NC; k++) w[k] = sA[k] * x[j][k];
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        double s = 0;
#pragma unroll
                        for (int k = 0; k < NC; k++) s += omb(i, k) * w[k];
                        t[i] = sA[i] * s;
                    }
                }
                const double zmb = zj - bj;
                const double Cp  = (zmb - P * (Zp[j] - Bp)) / (zmb * zmb);
                const double iC  = zmb / P;
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    const double E  = -aj / (D1MD2 * bj) * (2 * t[i] / aj - Bi[i] / bj);
                    const double Dp = Bi[i] / bj * Zp[j];
                    fugP[j][i]      = Cp * iC + Dp + E / G * Gp;
                }
            }
            // residual column: resF = f_0 - f_1 (fugacities), resN = N - sum x nu
            double resN[NC];
#pragma unroll
            for (int i = 0; i < NC; i++) {
                double r = Ni[i];
                r -= x[0][i] * nu[0];
                r -= x[1][i] * nu[1];
                resN[i] = r;
            }
            // the phase-mole block: the fugacity rows -dF/dn_0 = -fugN_0,
            // -dF/dn_1 = fugN_1 and the balance rows (1 at n_0i and n_1i), in
            // the order dgetrf leaves them after swapping the first three
            // fugacity rows for the saturation rows: fugacity rows 3..nc-1,
            // balance rows 0..nc-1, fugacity rows 0..2
            constexpr int D = 2 * NC;
            constexpr int M = NC + 2;  // P, N_1..N_nc, residual
            static_assert(NC >= 3, "the row order below assumes at least three components");
            double Mx[D][D], X[D][M];
            auto   fill = [&]() {
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    const int rf = i >= 3 ? i - 3 : D - 3 + i;  // fugacity row of component i
                    const int rn = NC - 3 + i;                  // balance row of component i
#pragma unroll
                    for (int k = 0; k < NC; k++) {
                        Mx[rf][k]      = -A0[i][k];
                        Mx[rf][NC + k] = A1[i][k];
                        Mx[rn][k]      = k == i ? 1.0 : 0.0;
                        Mx[rn][NC + k] = k == i ? 1.0 : 0.0;
                    }
                    X[rf][0] = fugP[0][i] - fugP[1][i];
                    X[rn][0] = 0.0;
#pragma unroll
                    for (int m = 0; m < NC; m++) {
                        X[rf][1 + m] = 0.0;
                        X[rn][1 + m] = m == i ? 1.0 : 0.0;
                    }
                    X[rf][M - 1] = this->phi[0][i] * x[0][i] * P - this->phi[1][i] * x[1][i] * P;
                    X[rn][M - 1] = resN[i];
                }
            };
            fill();
            if (!gauss_solve_mem<D, M>(Mx, X)) {
                status |= ST_SINGULAR;  // dgesv leaves the right-hand sides unchanged
                fill();
            }
            auto dn = [&](int j, int i, int c) -> double { return X[j * NC + i][c]; };
            // saturation rows: dS_j = sum_mk c_jmk dn_mk - rhs_S_j
            const double rSP[3] = {(vfP * vj[label[0]] - vjp[0] * vf) / vf2,
                                   (vfP * vj[label[1]] - vjp[1] * vf) / vf2, (vfP * vw - vwp * vf) / vf2};
            const double rSW[3] = {vfiW * vj[label[0]] / vf2, vfiW * vj[label[1]] / vf2, vfiW * (vw - vf) / vf2};
            const double rSR[3] = {S[label[0]] - vj[label[0]] / vf, S[label[1]] - vj[label[1]] / vf,
                                   S[2] - vw / vf};
            double resv[3 + 2 * NC];
#pragma unroll
            for (int e = 0; e < 3; e++) {  // e: internal phase 0, 1, then water
                const double vje = e < 2 ? vj[label[e]] : vw;
                const int    row = e < 2 ? label[e] : 2;
#pragma unroll
                for (int c = 0; c < M; c++) {
                    // back substitution, last unknown first: (rhs - sum) / -1
                    double t = c == 0 ? rSP[e] : (c == M - 1 ? rSR[e] : 0.0);
#pragma unroll
                    for (int m = 1; m >= 0; m--) {
#pragma unroll
                        for (int k = NC - 1; k >= 0; k--) {
                            const double cf = (e == m) ? vji[m][k] * (vf - vje) / vf2 : -vji[m][k] * vje / vf2;
                            t -= cf * dn(m, k, c);
                        }
                    }
                    const double v = -t;
                    if (c < M - 1)
                        dput(row, c, v);
                    else
                        resv[row] = v;
                }
                dput(row, NC + 1, -rSW[e]);
            }
            // phase-mole rows, filed by phase label
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const int r0 = 3 + label[j] * NC;
#pragma unroll
                for (int i = 0; i < NC; i++) {
#pragma unroll
                    for (int c = 0; c < M - 1; c++) dput(r0 + i, c, dn(j, i, c));
                    dput(r0 + i, NC + 1, 0.0);
                    resv[r0 + i] = dn(j, i, M - 1);
                }
            }
            rows = 3 + 2 * NC;
#pragma unroll
            for (int r = 0; r < 3 + 2 * NC; r++) tl.res[at(r)] = resv[r];
            // resPc (:4589-4597): the reference pairs internal phase j's vji
            // with the residual block filed at position j
#pragma unroll
            for (int j = 0; j < 2; j++)
#pragma unroll
                for (int i = 0; i < NC; i++) resPc += vji[j][i] * resv[3 + j * NC + i];
            // CalVfiVfp_full03: phases in label order
#pragma unroll
            for (int i = 0; i < NC; i++) vfi[i] = 0;
#pragma unroll
            for (int j1 = 0; j1 < 2; j1++) {
                const int jj = (label[0] == j1) ? 0 : 1;
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    vfP += vji[jj][i] * dn(jj, i, 0);
#pragma unroll
                    for (int m = 0; m < NC; m++) vfi[m] += vji[jj][i] * dn(jj, i, 1 + m);
                }
            }
        }
        vfi[NC]              = vfiW;
        out.bRowSizedSdP[n_] = rows;
        tl.resPc[n_]         = resPc;
        out.vfP[n_]          = vfP;
#pragma unroll
        for (int i = 0; i < NUMCOM; i++) out.vfi[at(i)] = vfi[i];

        // ---- CalXiPn_partial, CalRhoPn_partial, CalMuPnLBC_partial
        // (src/MixtureComp.cpp:2628-2763): derivatives per n_ij
        const double* L = F.L;
#pragma unroll
        for (int j = 0; j < 2; j++) {
            if (j < NP) {
                const int    j1  = label[j];
                const double xi  = xiC[j];
                const double nuj = nu[j];
                const double tmp = -xi * xi * CgTP;
                const double xiP = tmp * (Zp[j] - Zj[j] / P);
                double       xT = 0, xP = 0, xV = 0;
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    xT += x[j][i] * F.Tc[i];
                    xP += x[j][i] * F.Pc[i];
                    xV += x[j][i] * F.Vcvis[i];
                }
                const double u    = muA[j][3];
                const double poly = L[1] + u * (2 * L[2] + u * (3 * L[3] + u * 4 * L[4]));
                const double m4_3 = pow(muA[j][4], 3);
                const double m4_4 = pow(muA[j][4], 4);
                const double muP  = (4 * 1e-4) * m4_3 * (xV * xiP * poly) / muA[j][2];
                const double sqMW = sqrt(MW[j]);
                const double pT16 = pow(xT, 1.0 / 6), pT56 = pow(xT, -5.0 / 6), pP23 = pow(xP, 2.0 / 3);
                double       val2[NC];
#pragma unroll
                for (int i = 0; i < NC; i++) val2[i] = gT[i] / (F.muAux1I[i] / sqMW);

                out.rho[at(j1)]  = rhoC[j];
                out.xi[at(j1)]   = xi;
                out.mu[at(j1)]   = muC[j];
                out.xiP[at(j1)]  = xiP;
                out.rhoP[at(j1)] = xiP * MW[j];
                out.muP[at(j1)]  = muP;
                out.nj[at(j1)]   = njC[j];
#pragma unroll
                for (int k = 0; k < NC; k++) {
                    const int    o     = j1 * NUMCOM + k;
                    const double xix   = tmp * Zn[j][k];
                    const double derxT = (F.Tc[k] - xT) / nuj;
                    const double derxP = (F.Pc[k] - xP) / nuj;
                    const double derMW = (F.MW[k] - MW[j]) / nuj;
                    // der1 and der2 of the reference vanish: they carry the
                    // factor -(1 / 2), an integer division
                    double der3 = 0, der4 = F.sqrtMW[k];
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        der3 += F.sqrtMW[i] * ((dlt(i, k) - x[j][i]) * val2[i] / nuj);
                        der4 -= x[j][i] * F.sqrtMW[i];
                    }
                    der4 /= nuj;
                    const double der6 = 5.4402 *
                                        (1.0 / 6 * pT56 * derxT - pT16 * (0.5 / MW[j] * derMW + 2.0 / 3 / xP * derxP)) /
                                        (sqMW * pP23);
                    const double der7 = xix * xV + (F.Vcvis[k] - xV) * xi / nuj;
                    const double der8 = der7 * poly;
                    const double mux  = (der3 * muA[j][1] - muA[j][0] * der4) / (muA[j][1] * muA[j][1]) +
                                       1e-4 * (4 * m4_3 * der8 * muA[j][2] - (m4_4 - 1) * der6) /
                                           (muA[j][2] * muA[j][2]);
                    out.xij[at(o)]  = x[j][k];
                    out.xix[at(o)]  = xix;
                    out.rhox[at(o)] = xix * MW[j] + xi / nuj * (F.MW[k] - MW[j]);
                    out.mux[at(o)]  = mux;
                }
                const int ow     = j1 * NUMCOM + NC;
                out.xij[at(ow)]  = 0.0;
                out.xix[at(ow)]  = 0.0;
                out.rhox[at(ow)] = 0.0;
                out.mux[at(ow)]  = 0.0;
            }
        }
        finish_fim(n_, stride, sk, out, exist, bw, xiW, xiPW, Nw, vf, vfP, S);
    }

    // The last outputs of the FIM copy-out (FlashFIM and FlashFIMn): the
    // water phase, pSderExist / pVnumCom, the skip cache and the diagnostics.
    __device__ void finish_fim(int64_t n_, int64_t stride, const ocpf_skip& sk, const ocpf_fim_out& out,
                               const bool* exist, double bw, double xiW, double xiPW, double Nw, double vf,
                               double vfP, const double* S)
    {
        const int64_t N = stride;
        auto at = [N, n_](int f) { return (int64_t)f * N + n_; };
        // water phase
        out.rho[at(2)]  = F.std_rho_w / bw;
        out.xi[at(2)]   = xiW;
        out.mu[at(2)]   = F.pvtw[3];
        out.xiP[at(2)]  = xiPW;
        out.rhoP[at(2)] = CONV1 * xiPW * F.std_rho_w;
        out.muP[at(2)]  = 0.0;
        if (out.nj) out.nj[at(2)] = Nw;
#pragma unroll
        for (int k = 0; k < NUMCOM; k++) {
            const int o     = 2 * NUMCOM + k;
            out.xij[at(o)]  = (k == NC) ? 1.0 : 0.0;
            out.xix[at(o)]  = 0.0;
            out.rhox[at(o)] = 0.0;
            out.mux[at(o)]  = 0.0;
        }
        // pSderExist / pVnumCom, src/MixtureComp.cpp:559-570 (FlashFIMn :681-692)
#pragma unroll
        for (int j = 0; j < 2; j++) {
            out.pSderExist[at(j)] = exist[j] ? 1u : 0u;
            out.pVnumCom[at(j)]   = exist[j] ? (uint32_t)NC : 0u;
        }
        out.pSderExist[at(2)] = 1u;
        out.pVnumCom[at(2)]   = 0u;

        // ---- CalSkipForNextStep, src/MixtureComp.cpp:5234-5254
        if (F.use_skip) {
            if (flagSkip && ftype == 0) {
                sk.minEig[n_] = skip_min_eig();
                sk.P[n_]      = P;
                sk.T[n_]      = T;
#pragma unroll
                for (int i = 0; i < NC; i++) sk.z[at(i)] = zi[i];
            }
            sk.flag[n_] = flagSkip ? 1u : 0u;
        }

        // ---- diagnostics
        if (!isfinite(vf) || !isfinite(vfP) || !isfinite(S[0]) || !isfinite(S[1])) status |= ST_NONFINITE;
        if (out.ePEC) out.ePEC[n_] = this->ePEC;
        if (out.ftype) out.ftype[n_] = (uint8_t)ftype;
        if (out.iters) {
            out.iters[at(0)] = this->it_ssmsta;
            out.iters[at(1)] = this->it_nrsta;
            out.iters[at(2)] = this->it_ssmsp;
            out.iters[at(3)] = this->it_nrsp;
            out.iters[at(4)] = this->it_rr;
        }
        if (out.status) out.status[n_] = status;
    }

    // FlashIMPEC's remaining outputs (IsoT_IMPEC::PassFlashValue): the
    // per-phase properties of the existing phases, the water phase, the skip
    // cache and the diagnostics.
    __device__ void finalize_impec(int64_t n_, int64_t stride, const ocpf_skip& sk, const ocpf_fim_out& out,
                                   const int* label, const bool* exist, const double* xiC, const double* rhoC,
                                   const double* muC, const double* njC, double bw, double xiW, const double* S,
                                   double vf, double vfP)
    {
        const int64_t N = stride;
        auto at = [N, n_](int f) { return (int64_t)f * N + n_; };
#pragma unroll
        for (int j = 0; j < 2; j++) {
            if (j < NP) {
                const int j1     = label[j];
                out.rho[at(j1)]  = rhoC[j];
                out.xi[at(j1)]   = xiC[j];
                out.mu[at(j1)]   = muC[j];
                if (out.nj) out.nj[at(j1)] = njC[j];
#pragma unroll
                for (int k = 0; k < NC; k++) out.xij[at(j1 * NUMCOM + k)] = x[j][k];
                out.xij[at(j1 * NUMCOM + NC)] = 0.0;
            }
        }
        out.rho[at(2)] = F.std_rho_w / bw;
        out.xi[at(2)]  = xiW;
        out.mu[at(2)]  = F.pvtw[3];
        if (out.nj) out.nj[at(2)] = Ni[NC];
#pragma unroll
        for (int k = 0; k < NUMCOM; k++) out.xij[at(2 * NUMCOM + k)] = (k == NC) ? 1.0 : 0.0;
        if (F.use_skip) {
            if (flagSkip && ftype == 0) {
                sk.minEig[n_] = skip_min_eig();
                sk.P[n_]      = P;
                sk.T[n_]      = T;
#pragma unroll
                for (int i = 0; i < NC; i++) sk.z[at(i)] = zi[i];
            }
            sk.flag[n_] = flagSkip ? 1u : 0u;
        }
        if (!isfinite(vf) || !isfinite(vfP) || !isfinite(S[0]) || !isfinite(S[1])) status |= ST_NONFINITE;
        if (out.ePEC) out.ePEC[n_] = this->ePEC;
        if (out.ftype) out.ftype[n_] = (uint8_t)ftype;
        if (out.iters) {
            out.iters[at(0)] = this->it_ssmsta;
            out.iters[at(1)] = this->it_nrsta;
            out.iters[at(2)] = this->it_ssmsp;
            out.iters[at(3)] = this->it_nrsp;
            out.iters[at(4)] = this->it_rr;
        }
        if (out.status) out.status[n_] = status;
    }
};

}  // namespace ocpf
