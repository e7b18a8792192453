// flash_batched.cuh -- the batched form of the FIM flash: a persistent
// equilibrium kernel in which every lane runs one cell's PhaseEquilibrium as
// a state machine and refills itself from a work queue when the cell is done,
// followed by a one-thread-per-cell finalize kernel (properties, derivatives,
// copy-out).
//
// Why: in a one-thread-per-cell kernel the cells of a warp need very
// different numbers of stability / split iterations (2 to 400+), so most
// lanes idle while the slowest cell iterates, and the fully inlined flash does
// not fit the instruction cache. Here each warp "tick" runs the light,
// divergent control logic of every lane (advance), then at most two fugacity
// evaluations -- the dominant cost -- with all lanes that need one converged
// on the same code. A lane whose cell finishes loads the next cell at once.
//
// The state machine takes exactly the reference's steps in the reference's
// order (src/MixtureComp.cpp:1279-1353 PhaseEquilibrium, :1355-1636
// PhaseStable/StableSSM01/StableSSM/StableNR, :1743-2156 PhaseSplit/
// SplitSSM2/RachfordRice2/SplitNR/CheckSplit); each stage names the loop it
// unrolls. Arithmetic is the plain form's (same helper functions).
#pragma once

#include "flash_fim.cuh"

namespace ocpf {

// Per-cell equilibrium results handed from the equilibrium kernel to the
// finalize kernel (structure of arrays, field stride `cap`).
struct EqBuf {
    uint32_t* meta;   // [cap]: NP | ftype << 4 | flagSkip << 8 | status << 16
    int32_t*  iters;  // [5][cap]
    double*   d;      // [EQ_DBL(nc)][cap]: ePEC, nu0, nu1, Aj0, Aj1, Bj0, Bj1, Zj0, Zj1, x0[nc], x1[nc], n0[nc], n1[nc]
    int64_t   cap;
};
__host__ __device__ constexpr int eq_dbl(int nc) { return 9 + 4 * nc; }
inline size_t eqbuf_bytes_per_cell(int nc) { return 4 + 5 * 4 + 8 * (size_t)eq_dbl(nc); }

template <int NC>
struct BatchedLane : FimCell<NC> {
    using Base = FimCell<NC>;
    using Base::F;
    using Base::NP;
    using Base::lNP;
    using Base::ftype;
    using Base::flagSkip;
    using Base::nu;
    using Base::x;
    using Base::phi;
    using Base::Aj;
    using Base::Bj;
    using Base::Zj;
    using Base::Ks;
    using Base::lKs;
    using Base::Kw0;
    using Base::zi;
    using Base::n;
    using Base::P;
    using Base::Yt;
    using Base::status;

    enum Stage : int {
        S_IDLE = 0,
        S_START,
        // strict stability test, StableSSM + StableNR
        S_STRICT_START,
        S_STRICT_E0,
        S_TRIAL_INIT,
        S_TRIAL_POST,
        S_SSM_STEP,
        S_SSM_POST,
        S_NR_START,
        S_NR_STEP,
        S_NR_POST,
        S_NR_END,
        // relaxed stability test, StableSSM01
        S01_START,
        S01_E0,
        S01_TRIAL,
        S01_STEP,
        S01_POST,
        S01_TEND,
        S01_DONE,
        S_STAB_DONE,
        // phase split
        S_SPLIT_BEGIN,
        S_SSM_BEGIN,
        S_SP_SSM_STEP,
        S_SP_SSM_POST,
        S_SP_SSM_END,
        S_SP_NR_BEGIN,
        S_SP_NR_STEP,
        S_SP_NR_POST,
        S_SP_NR_END,
        S_SPLIT_CTRL,
        S_FINAL_CHECK,
        S_EQ_END
    };

    int     stage;
    bool    needA, needB;  // evaluations requested for this tick
    int64_t cell;
    // stability test
    double di[NC];  // SSM01's d_i and previous Y (the strict test forms phi_z x_z on the fly)
    double Se_ssm, Se_nr, Sk;
    int    k, iter, nr_iter;
    bool   flag, have_e0, stab_result;
    // split
    double Stol, eNR, eNR0, en, Se_sp;
    int    maxIt, split_phase, guard;
    bool   restart;

    __device__ __forceinline__ explicit BatchedLane(const FluidConst& f) : Base(f) { stage = S_IDLE; }

    // fugacity of the test phase z: f_z = (phi_z x_z) P, as CalFugPhi forms it
    __device__ __forceinline__ double fz(int i) const { return phi[0][i] * x[0][i] * P; }
    // trial-phase fugacity (evaluation B)
    __device__ __forceinline__ double fy(int i) const { return phi[1][i] * x[1][i] * P; }

    // Evaluations: A on x[0] -> phi[0], Aj/Bj/Zj[0]; B on x[1] -> phi[1], Aj/Bj/Zj[1].
    __device__ __forceinline__ void eval(int j)
    {
        double fug_[NC];
        this->fug_phi(x[j], phi[j], fug_, Aj[j], Bj[j], Zj[j]);
    }

    __device__ void begin_cell(int64_t c, int64_t stride, const ocpf_fim_in& in, const ocpf_skip& sk)
    {
        cell = c;
        this->load_inputs(c, stride, in, sk);
        this->cal_ai_bi();
        stage = S_START;
    }

    __device__ void end_cell(int64_t stride, const EqBuf& eb) const
    {
        const int64_t C = eb.cap;
        const int64_t c = cell;
        eb.meta[c] = (uint32_t)NP | ((uint32_t)ftype << 4) | ((uint32_t)(flagSkip ? 1 : 0) << 8) |
                     ((uint32_t)status << 16);
        eb.iters[0 * C + c] = this->it_ssmsta;
        eb.iters[1 * C + c] = this->it_nrsta;
        eb.iters[2 * C + c] = this->it_ssmsp;
        eb.iters[3 * C + c] = this->it_nrsp;
        eb.iters[4 * C + c] = this->it_rr;
        double* d  = eb.d;
        d[0 * C + c] = this->ePEC;
        d[1 * C + c] = nu[0];
        d[2 * C + c] = nu[1];
        d[3 * C + c] = Aj[0];
        d[4 * C + c] = Aj[1];
        d[5 * C + c] = Bj[0];
        d[6 * C + c] = Bj[1];
        d[7 * C + c] = Zj[0];
        d[8 * C + c] = Zj[1];
#pragma unroll
        for (int i = 0; i < NC; i++) {
            d[(9 + i) * C + c]          = x[0][i];
            d[(9 + NC + i) * C + c]     = x[1][i];
            d[(9 + 2 * NC + i) * C + c] = n[0][i];
            d[(9 + 3 * NC + i) * C + c] = n[1][i];
        }
        (void)stride;
    }

    // Runs the lane's control logic until it needs an evaluation, or until
    // its cell is done (then stores it and takes the next cell from the
    // queue), or until the queue is empty (stage S_IDLE).
    __device__ void advance(int64_t count, int64_t stride, const ocpf_fim_in& in, const ocpf_skip& sk,
                            const EqBuf& eb, unsigned long long* queue)
    {
        needA = needB = false;
        // every path through the loop either requests an evaluation, finishes
        // a cell or changes stage towards one of those; the bound only guards
        // against a logic error turning into an endless loop
        for (int guard_ = 0; guard_ < 256; guard_++) {
            switch (stage) {
                case S_IDLE: return;
                case S_START:
                    this->ssmsta_conflag = this->nrsta_conflag = false;
                    if (ftype == 0) {
                        flagSkip = true;
                        NP       = 1;
                        nu[0]    = 1;
#pragma unroll
                        for (int i = 0; i < NC; i++) x[0][i] = zi[i];
                        this->cal_kwilson();
                        have_e0 = false;
                        stage   = (lNP == 0) ? S_STRICT_START : S01_START;
                    } else if (ftype == 1) {
                        // skip the stability test: single phase at z
                        flagSkip = true;
                        NP       = 1;
                        nu[0]    = 1;
#pragma unroll
                        for (int i = 0; i < NC; i++) x[0][i] = zi[i];
                        this->ePEC = 0.0;
                        needA      = true;
                        stage      = S_EQ_END;
                        return;
                    } else {
                        // skip the stability test: two phases from last K
                        flagSkip = false;
                        NP       = 2;
                        Yt       = 1.01;
                        this->cal_kwilson();
                        stage = S_SPLIT_BEGIN;
                    }
                    break;

                // ---------------- StableSSM (strict), :1492-1588
                case S_STRICT_START:
                    stage = S_STRICT_E0;
                    if (!have_e0) {
                        have_e0 = true;
                        needA   = true;  // CalFugPhi(phi[0], fug[0], z)
                        return;
                    }
                    break;
                case S_STRICT_E0:
                    k     = 0;
                    stage = S_TRIAL_INIT;
                    break;
                case S_TRIAL_INIT: {
                    Yt = 0;
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        x[1][i] = x[0][i] / this->kw(k, i);
                        Yt += x[1][i];
                    }
                    const double r = 1 / Yt;
#pragma unroll
                    for (int i = 0; i < NC; i++) x[1][i] *= r;
                    needB = true;
                    stage = S_TRIAL_POST;
                    return;
                }
                case S_TRIAL_POST:
                    Se_ssm = 0;
#pragma unroll
                    for (int i = 0; i < NC; i++) Se_ssm += sq(log(fy(i) / fz(i) * Yt));
                    iter  = 0;
                    stage = (Se_ssm > F.ssmsta_tol2) ? S_SSM_STEP : S_NR_START;
                    break;
                case S_SSM_STEP: {
                    Yt = 0;
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        x[1][i] = (phi[0][i] * x[0][i]) / phi[1][i];
                        Yt += x[1][i];
                    }
                    const double r = 1 / Yt;
#pragma unroll
                    for (int i = 0; i < NC; i++) x[1][i] *= r;
                    needB = true;
                    stage = S_SSM_POST;
                    return;
                }
                case S_SSM_POST:
                    Se_ssm = 0;
#pragma unroll
                    for (int i = 0; i < NC; i++) Se_ssm += sq(log(fy(i) / fz(i) * Yt));
                    iter++;
                    if (iter > F.ssmsta_maxit) {
                        status |= ST_SSMSTA_CAP;
                        stage = S_NR_START;
                    } else {
                        stage = (Se_ssm > F.ssmsta_tol2) ? S_SSM_STEP : S_NR_START;
                    }
                    break;
                // ---------------- StableNR, :1590-1636
                case S_NR_START:
                    this->it_ssmsta += iter;
                    Se_nr = 0;
#pragma unroll
                    for (int i = 0; i < NC; i++) Se_nr += sq(log(fz(i) / (fy(i) * Yt)));
                    Se_nr   = sqrt(Se_nr);
                    nr_iter = 0;
                    if (Se_nr > F.nrsta_tol) {
                        stage = S_NR_STEP;
                    } else {
                        this->nrsta_conflag = true;
                        this->nrsta_realTol = Se_nr;
                        flag                = true;
                        stage               = S_NR_END;
                    }
                    break;
                case S_NR_STEP: {
                    double res[NC];
#pragma unroll
                    for (int i = 0; i < NC; i++) res[i] = log(fz(i) / (fy(i) * Yt));
                    this->sta_nr_update(x[1], Yt, res, Aj[1], Bj[1], Zj[1]);
                    needB = true;
                    stage = S_NR_POST;
                    return;
                }
                case S_NR_POST:
                    Se_nr = 0;
#pragma unroll
                    for (int i = 0; i < NC; i++) Se_nr += sq(log(fz(i) / (fy(i) * Yt)));
                    Se_nr = sqrt(Se_nr);
                    nr_iter++;
                    if (nr_iter > F.nrsta_maxit) {
                        this->it_nrsta += nr_iter;
                        status |= ST_NRSTA_FAIL;
                        this->nrsta_conflag = false;
                        this->nrsta_realTol = Se_nr;
                        flag                = false;
                        stage               = S_NR_END;
                    } else if (Se_nr > F.nrsta_tol) {
                        stage = S_NR_STEP;
                    } else {
                        this->it_nrsta += nr_iter;
                        this->nrsta_conflag = true;
                        this->nrsta_realTol = Se_nr;
                        flag                = true;
                        stage               = S_NR_END;
                    }
                    break;
                case S_NR_END:
                    if (flag && Yt > 1 + F.ssmsta_eyt) {
                        this->ssmsta_conflag = true;
                        this->ssmsta_realTol = sqrt(Se_ssm);
                        stab_result          = false;
                        stage                = S_STAB_DONE;
                    } else if (++k < 4) {
                        stage = S_TRIAL_INIT;
                    } else {
                        this->ssmsta_realTol = sqrt(Se_ssm);
                        stab_result          = true;
                        stage                = S_STAB_DONE;
                    }
                    break;

                // ---------------- StableSSM01 (relaxed), :1392-1490
                case S01_START:
                    stage = S01_E0;
                    if (!have_e0) {
                        have_e0 = true;
                        needA   = true;
                        return;
                    }
                    break;
                case S01_E0:
                    k     = 0;
                    stage = S01_TRIAL;
                    break;
                case S01_TRIAL:
#pragma unroll
                    for (int i = 0; i < NC; i++) Ks[i] = this->kw(k, i);
                    iter  = 0;
                    flag  = false;
                    stage = S01_STEP;
                    break;
                case S01_STEP: {
                    Yt = 0;
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        x[1][i] = x[0][i] * Ks[i];
                        Yt += x[1][i];
                    }
                    const double r = 1 / Yt;
#pragma unroll
                    for (int i = 0; i < NC; i++) x[1][i] *= r;
                    if (iter > 0) {
                        double dY = 0;
#pragma unroll
                        for (int i = 0; i < NC; i++) dY += sq(x[1][i] - di[i]);
                        if (dY < 1e-6) {  // dYtol, include/MixtureComp.hpp:34
                            flag  = true;
                            stage = S01_TEND;
                            break;
                        }
                    }
                    needB = true;
                    stage = S01_POST;
                    return;
                }
                case S01_POST: {
                    Se_ssm = 0;
                    Sk     = 0;
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        const double d = fz(i) / (fy(i) * Yt);
                        Ks[i] *= d;
                        Se_ssm += sq(d - 1);
                        Sk += sq(log(Ks[i]));
                    }
                    iter++;
                    if (Se_ssm < F.ssmsta_tol2 || Sk < 1e-4) {  // Ktol, include/MixtureComp.hpp:33
                        flag  = true;
                        stage = S01_TEND;
                    } else if (iter > F.ssmsta_maxit) {
                        status |= ST_SSMSTA_CAP;
                        stage = S01_TEND;
                    } else {
#pragma unroll
                        for (int i = 0; i < NC; i++) di[i] = x[1][i];
                        stage = S01_STEP;
                    }
                    break;
                }
                case S01_TEND:
                    this->it_ssmsta += iter;
                    if (flag && Yt > 1 - 0.1 && Sk > 1) flagSkip = false;
                    if (flag && Yt > 1 + F.ssmsta_eyt) {
                        this->ssmsta_conflag = true;
                        this->ssmsta_realTol = sqrt(Se_ssm);
                        stab_result          = false;
                        stage                = S01_DONE;
                    } else if (++k < 2) {
                        stage = S01_TRIAL;
                    } else {
                        this->ssmsta_realTol = sqrt(Se_ssm);
                        stab_result          = true;
                        stage                = S01_DONE;
                    }
                    break;
                case S01_DONE: {
                    // PhaseStable: a verdict that disagrees with the last
                    // phase count falls back to the strict test
                    const int tmpNP = NP + (stab_result ? 0 : 1);
                    if (tmpNP != lNP) {
                        flagSkip = false;
                        stage    = S_STRICT_START;
                    } else {
                        stage = S_STAB_DONE;
                    }
                    break;
                }
                case S_STAB_DONE:
                    if (stab_result) {
                        this->ePEC = this->nrsta_conflag ? this->nrsta_realTol
                                     : (this->ssmsta_conflag ? this->ssmsta_realTol : 1e8);
                        stage = S_EQ_END;
                    } else {
                        NP    = 2;
                        stage = S_SPLIT_BEGIN;
                    }
                    break;

                // ---------------- PhaseSplit, :1743-1782
                case S_SPLIT_BEGIN:
                    this->ssmsp_conflag = false;
                    this->nrsp_conflag  = false;
                    split_phase         = 0;
                    guard               = 0;
                    restart             = false;
                    stage               = S_SSM_BEGIN;
                    break;
                // SplitSSM2, :1847-1903
                case S_SSM_BEGIN:
                    this->ssmsp_conflag = true;
                    Se_sp        = 1;
                    Stol                = F.ssmsp_tol2;
                    maxIt               = F.ssmsp_maxit;
                    if (!restart) {
#pragma unroll
                        for (int i = 0; i < NC; i++) Ks[i] = (lNP == 2) ? lKs[i] : Kw0[i];
                    } else {
                        Stol *= 1e-1;
                        maxIt *= 2;
                    }
                    if (Yt < 1.1) {
                        Stol *= 1e-1;
                        maxIt *= 2;
                    }
                    iter  = 0;
                    stage = (Se_sp > Stol) ? S_SP_SSM_STEP : S_SP_SSM_END;
                    break;
                case S_SP_SSM_STEP:
                    this->rachford_rice2();
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        const double tmp = 1 + nu[0] * (Ks[i] - 1);
                        x[1][i]          = zi[i] / tmp;
                        x[0][i]          = Ks[i] * x[1][i];
                    }
                    needA = needB = true;
                    stage         = S_SP_SSM_POST;
                    return;
                case S_SP_SSM_POST: {
                    double Se = 0;
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        Se += sq((phi[1][i] * x[1][i] * P) / (phi[0][i] * x[0][i] * P) - 1);
                        Ks[i] = phi[1][i] / phi[0][i];
                    }
                    Se_sp = Se;
                    iter++;
                    if (iter > maxIt) {
                        this->ssmsp_conflag = false;
                        stage               = S_SP_SSM_END;
                    } else {
                        stage = (Se > Stol) ? S_SP_SSM_STEP : S_SP_SSM_END;
                    }
                    break;
                }
                case S_SP_SSM_END:
                    this->ssmsp_realTol = sqrt(Se_sp);
                    this->it_ssmsp += iter;
                    stage = S_SP_NR_BEGIN;
                    break;
                // SplitNR, :2057-2156
                case S_SP_NR_BEGIN:
                    this->nrsp_conflag = false;
                    eNR                = 0;
#pragma unroll
                    for (int i = 0; i < NC; i++) {
                        n[0][i] = nu[0] * x[0][i];
                        n[1][i] = nu[1] * x[1][i];
                        eNR += sq(log((phi[1][i] * x[1][i] * P) / (phi[0][i] * x[0][i] * P)));
                    }
                    eNR   = sqrt(eNR);
                    eNR0  = eNR;
                    iter  = 0;
                    stage = (eNR > F.nrsp_tol) ? S_SP_NR_STEP : S_SP_NR_END;
                    break;
                case S_SP_NR_STEP: {
                    double res[NC];
#pragma unroll
                    for (int i = 0; i < NC; i++)
                        res[i] = log((phi[1][i] * x[1][i] * P) / (phi[0][i] * x[0][i] * P));
                    en    = this->sp_nr_update(res);
                    needA = needB = true;
                    stage         = S_SP_NR_POST;
                    return;
                }
                case S_SP_NR_POST:
                    eNR = 0;
#pragma unroll
                    for (int i = 0; i < NC; i++)
                        eNR += sq(log((phi[1][i] * x[1][i] * P) / (phi[0][i] * x[0][i] * P)));
                    eNR = sqrt(eNR);
                    iter++;
                    if (eNR > eNR0 || iter > F.nrsp_maxit) {
                        stage = S_SP_NR_END;
                    } else if (en / (2 * NC) < 1e-8) {
                        this->nrsp_conflag = true;
                        stage              = S_SP_NR_END;
                    } else {
                        stage = (eNR > F.nrsp_tol) ? S_SP_NR_STEP : S_SP_NR_END;
                    }
                    break;
                case S_SP_NR_END:
                    this->nrsp_realTol = eNR;
                    if (eNR < F.nrsp_tol) this->nrsp_conflag = true;
                    this->it_nrsp += iter;
                    stage = S_SPLIT_CTRL;
                    break;
                case S_SPLIT_CTRL:
                    // while (!NRsp.conflag) { SSM(true); NR(); if (!CheckSplit()) break;
                    //                          if (SSMsp.conflag) break; }
                    if (split_phase == 0) {
                        if (this->nrsp_conflag) {
                            stage = S_FINAL_CHECK;
                        } else {
                            split_phase = 1;
                            guard       = 1;
                            restart     = true;
                            stage       = S_SSM_BEGIN;
                        }
                    } else if (!this->check_split()) {
                        stage = S_FINAL_CHECK;  // collapsed: the final check is a no-op
                    } else if (this->ssmsp_conflag || this->nrsp_conflag) {
                        stage = S_FINAL_CHECK;
                    } else if (++guard > SPLIT_RESTART_CAP) {
                        status |= ST_SPLIT_CAP;
                        stage = S_FINAL_CHECK;
                    } else {
                        stage = S_SSM_BEGIN;
                    }
                    break;
                case S_FINAL_CHECK:
                    this->check_split();
                    if (!this->ssmsp_conflag) status |= ST_SSMSP_FAIL;
                    if (!this->nrsp_conflag) status |= ST_NRSP_FAIL;
                    if (ftype == 0) {
                        if (NP > 1) flagSkip = false;
                        if (NP == 1)
                            this->ePEC = this->nrsta_conflag ? this->nrsta_realTol
                                         : (this->ssmsta_conflag ? this->ssmsta_realTol : 1e8);
                        else
                            this->ePEC = this->nrsp_conflag ? this->nrsp_realTol
                                         : (this->ssmsp_conflag ? this->ssmsp_realTol : 1e8);
                    } else {
                        this->ePEC = this->nrsp_conflag ? this->nrsp_realTol
                                     : (this->ssmsp_conflag ? this->ssmsp_realTol : 1e8);
                    }
                    stage = S_EQ_END;
                    break;

                case S_EQ_END: {
                    end_cell(stride, eb);
                    const unsigned long long c = atomicAdd(queue, 1ull);
                    if ((int64_t)c < count) {
                        begin_cell((int64_t)c, stride, in, sk);
                    } else {
                        stage = S_IDLE;
                        return;
                    }
                    break;
                }
                default: stage = S_IDLE; return;
            }
        }
        // A control-flow error must not spin the lane: finish the cell with
        // the guard bit set; its next call stores it and moves on.
        status |= ST_GUARD;
        stage = S_EQ_END;
    }
};

// Persistent equilibrium kernel: each lane takes cells from `queue` (zeroed
// before the launch) until all `count` cells are done.
template <int NC>
__device__ __forceinline__ void eq_persistent_body(const FluidConst& F, int64_t count, int64_t stride,
                                                   const ocpf_fim_in& in, const ocpf_skip& sk,
                                                   const EqBuf& eb, unsigned long long* queue)
{
    BatchedLane<NC> L(F);
    const unsigned long long c0 = atomicAdd(queue, 1ull);
    if ((int64_t)c0 < count) L.begin_cell((int64_t)c0, stride, in, sk);
    while (true) {
        L.advance(count, stride, in, sk, eb, queue);
        const bool a = L.needA, b = L.needB;
        if (!__any_sync(0xffffffffu, L.stage != BatchedLane<NC>::S_IDLE)) break;
        if (a) L.eval(0);
        __syncwarp();
        if (b) L.eval(1);
        __syncwarp();
    }
}

// Finalize: properties, derivatives, skip cache and copy-out of one cell
// from its equilibrium (FimCell::finalize), one thread per cell.
template <int NC>
__device__ __forceinline__ void finalize_body(const FluidConst& F, int64_t count, int64_t stride,
                                              const ocpf_fim_in& in, const ocpf_skip& sk, const EqBuf& eb,
                                              const ocpf_fim_out& out)
{
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= count) return;
    FimCell<NC> f(F);
    f.load_inputs(c, stride, in, sk);
    f.cal_ai_bi();
    const int64_t  C  = eb.cap;
    const uint32_t m  = eb.meta[c];
    f.NP              = (int)(m & 0xF);
    f.ftype           = (int)((m >> 4) & 0xF);
    f.flagSkip        = ((m >> 8) & 1) != 0;
    f.status          = (uint16_t)(m >> 16);
    f.it_ssmsta       = eb.iters[0 * C + c];
    f.it_nrsta        = eb.iters[1 * C + c];
    f.it_ssmsp        = eb.iters[2 * C + c];
    f.it_nrsp         = eb.iters[3 * C + c];
    f.it_rr           = eb.iters[4 * C + c];
    const double* d   = eb.d;
    f.ePEC            = d[0 * C + c];
    f.nu[0]           = d[1 * C + c];
    f.nu[1]           = d[2 * C + c];
    f.Aj[0]           = d[3 * C + c];
    f.Aj[1]           = d[4 * C + c];
    f.Bj[0]           = d[5 * C + c];
    f.Bj[1]           = d[6 * C + c];
    f.Zj[0]           = d[7 * C + c];
    f.Zj[1]           = d[8 * C + c];
#pragma unroll
    for (int i = 0; i < NC; i++) {
        f.x[0][i] = d[(9 + i) * C + c];
        f.x[1][i] = d[(9 + NC + i) * C + c];
        f.n[0][i] = d[(9 + 2 * NC + i) * C + c];
        f.n[1][i] = d[(9 + 3 * NC + i) * C + c];
    }
    f.finalize(c, stride, sk, out);
}

}  // namespace ocpf
