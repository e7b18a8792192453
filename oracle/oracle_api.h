/*
 * oracle_api.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Shared C interface of the two CPU oracles for the compositional
 * Peng-Robinson FIM flash:
 *   - oracle/_ref/libocpref.so : the reference's own MixtureComp compiled from
 *     its sources (recipe: oracle/Makefile, harness: oracle/ref_harness.cpp);
 *   - oracle/libflashport.so   : a plain-C restatement of the same algorithm
 *     (oracle/flash_port.c).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * either library; the product path never does.
 *
 * Layout is the reference Bulk layout (array-of-structures per cell, as in
 * include/Bulk.hpp:304-357 and the compact dSec_dPri of
 * src/OCPFluidMethod.cpp:1056-1063, 1122-1187): with numCom = nc + 1 (water
 * last) and numPhase = 3 (oil, gas, water),
 *   Ni[n*numCom + i], S[n*3 + j], xij[n*3*numCom + j*numCom + i],
 *   dSec_dPri[n*(numCom+1)*(numCom+1)*3 + r*(numCom+1) + c].
 * Units are FIELD: psia, degF on input, ft3/lbmol, lbmol.
 */
#ifndef OCP_ORACLE_API_H
#define OCP_ORACLE_API_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_NC 16

/* Fluid and solver controls of one PVT region (one MixtureComp instance).
 * Mirrors ComponentParam (include/ParamReservoir.hpp:87-193) as consumed by
 * MixtureComp::MixtureComp (src/MixtureComp.cpp:28-165). */
typedef struct {
    int32_t nc;            /* hydrocarbon components */
    int32_t rr_maxit;      /* RR keyword */
    int32_t ssmsta_maxit;  /* SSMSTA keyword */
    int32_t nrsta_maxit;   /* NRSTA keyword */
    int32_t ssmsp_maxit;   /* SSMSP keyword */
    int32_t nrsp_maxit;    /* NRSP keyword */
    int32_t use_skip;      /* SkipStaAnaly::ifUseSkip */
    int32_t pad0;
    double rr_tol, ssmsta_tol, ssmsta_eyt, nrsta_tol, ssmsp_tol, nrsp_tol;
    double Tc[ORC_MAX_NC];     /* degR */
    double Pc[ORC_MAX_NC];     /* psia */
    double Vc[ORC_MAX_NC];     /* ft3/lbmol (VCRIT) */
    double MW[ORC_MAX_NC];
    double Acf[ORC_MAX_NC];
    double OmegaA[ORC_MAX_NC];
    double OmegaB[ORC_MAX_NC];
    double Vshift[ORC_MAX_NC]; /* dimensionless VSHIFT deck value */
    double BIC[ORC_MAX_NC * ORC_MAX_NC]; /* nc*nc row-major, symmetric */
    double LBCcoef[5];         /* LBCCOEF deck values (scaled x10 inside) */
    double pvtw[5];            /* PVTW row: Pref, Bw, Cw, muw, Cvw */
    double std_rho_w;          /* water density at surface, lb/ft3 */
} orc_fluid;

/* One batch of FlashFIM calls, one per cell, in Bulk layout. xij_in may alias
 * xij and S_in may alias S (in-place, as the Bulk arrays are). The skip_*
 * arrays are the per-bulk SkipStaAnaly cache (src/AcceleratePVT.cpp); they are
 * read and written when use_skip != 0. Outputs of absent phases are left
 * untouched, as PassFlashValue does (src/OCPFluidMethod.cpp:1141-1160). */
typedef struct {
    int64_t n;
    /* inputs */
    const double*  P;      /* [n] psia */
    const double*  T;      /* [n] degF */
    const double*  Ni;     /* [n*numCom] lbmol */
    const double*  S_in;   /* [n*3] */
    const int32_t* lastNP; /* [n] phase count of the last step, water included */
    const double*  xij_in; /* [n*3*numCom] */
    /* skip cache, in/out */
    int32_t* skip_flag;
    double*  skip_minEig;
    double*  skip_P;
    double*  skip_T;
    double*  skip_z;       /* [n*nc] */
    /* outputs */
    int32_t* phaseNum;     /* [n] */
    int32_t* phaseExist;   /* [n*3] */
    double*  S;            /* [n*3] */
    double*  Nt;           /* [n] */
    double*  vf;           /* [n] */
    double*  vfP;          /* [n] */
    double*  vfi;          /* [n*numCom] */
    double*  nj;           /* [n*3] */
    double*  rho;          /* [n*3] */
    double*  xi;           /* [n*3] */
    double*  mu;           /* [n*3] */
    double*  rhoP;         /* [n*3] */
    double*  xiP;          /* [n*3] */
    double*  muP;          /* [n*3] */
    double*  xij;          /* [n*3*numCom] */
    double*  rhox;         /* [n*3*numCom] */
    double*  xix;          /* [n*3*numCom] */
    double*  mux;          /* [n*3*numCom] */
    double*  dSec_dPri;    /* [n*(numCom+1)*(numCom+1)*3] compact rows */
    int32_t* bRowSizedSdP; /* [n] */
    int32_t* pSderExist;   /* [n*3] */
    int32_t* pVnumCom;     /* [n*3] */
    double*  ePEC;         /* [n] */
    int32_t* ftype;        /* [n] */
    int32_t* NPhc;         /* [n] hydrocarbon phase count */
    int32_t* iters;        /* [n*5] SSMSTA, NRSTA, SSMSP, NRSP, RR iterations */
    int32_t* restarts;     /* [n] PhaseSplit restarts (the restatement only; may be NULL) */
} orc_batch;

/* Runs FlashFIM over the batch with nthreads host threads (each owning its own
 * flash object). Returns 0 on success; *seconds receives the wall time of the
 * flash loop alone (construction excluded). */
int orc_flash_fim_batch(const orc_fluid* fluid, const orc_batch* batch,
                        int nthreads, double* seconds);

/* Runs FlashIMPEC over the batch (src/MixtureComp.cpp:444-492) with the
 * copy-out of IsoT_IMPEC::PassFlashValue (src/OCPFluidMethod.cpp:275-305):
 * phaseNum, phaseExist, S, Nt, vf, vfP, vfi, rho, xi, mu, xij of the batch
 * plus vj [n*3] (phase volumes); S_in is not read. The reference oracle
 * only. */
int orc_flash_impec_batch(const orc_fluid* fluid, const orc_batch* batch, double* vj,
                          int nthreads, double* seconds);

/* Runs InitFlashFIM (impec == 0, src/MixtureComp.cpp:261-353) or
 * InitFlashIMPEC (impec != 0, :195-259) over the batch, as IsoT_FIM::InitFlash
 * (src/OCPFluidMethod.cpp:1095-1106) and IsoT_IMPEC::InitFlash (:251-262)
 * make them: batch->Ni holds the initial mole fractions z [n*numCom] (water
 * entry ignored), batch->S_in the initial saturations (only S_w is read),
 * Vpore [n] the pore volumes (ft3); lastNP and xij_in are not read. Ni [n*numCom]
 * receives the flash object's Ni afterwards (may alias batch->Ni). The
 * copy-out is the FIM one (orc_flash_fim_batch's outputs) or, with impec, the
 * IMPEC one with the phase volumes in vj [n*3]. The reference oracle only. */
int orc_init_flash_batch(const orc_fluid* fluid, const orc_batch* batch, const double* Vpore, int impec,
                         double* Ni, double* vj, int nthreads, double* seconds);

/* Runs FlashFIMn over the batch (src/MixtureComp.cpp:575-695) with the
 * copy-out of IsoT_FIMn::PassFlashValue (src/OCPFluidMethod.cpp:3179-3196):
 * the orc_flash_fim_batch outputs (with FlashFIMn's dSec_dPri rows and
 * per-n_ij partials) plus res [n*3*(numCom+1)] (the first bRowSizedSdP
 * entries of each cell written) and resPc [n]. The reference oracle only. */
int orc_flash_fimn_batch(const orc_fluid* fluid, const orc_batch* batch, double* res, double* resPc,
                         int nthreads, double* seconds);

/* Runs InitFlashFIMn over the batch (src/MixtureComp.cpp:355-442), inputs as
 * orc_init_flash_batch, outputs as orc_flash_fimn_batch. */
int orc_init_flash_fimn_batch(const orc_fluid* fluid, const orc_batch* batch, const double* Vpore, double* Ni,
                              double* res, double* resPc, int nthreads, double* seconds);

/* Saturation functions of one region, as the SWOF and SGOF keywords list
 * them (row-major, 4 columns): Sw, krw, krow, Pcow and Sg, krg, krog, Pcgo. */
typedef struct {
    int32_t       nrow_swof, nrow_sgof;
    const double* swof;
    const double* sgof;
} orc_satfunc;

/* One batch of FlowUnit::CalKrPcDeriv (or CalKrPc) calls, cell-major (Bulk
 * layout): S [n*3] in; kr, Pc, Pj = P + Pc [n*3] and, with deriv,
 * dKr_dS, dPcj_dS [n*9] (row j: d/dS_k of phase j) out. */
typedef struct {
    int64_t        n;
    int32_t        deriv;
    const double*  P;      /* [n] */
    const double*  S;      /* [n*3] */
    const int32_t* satnum; /* [n] region of each cell, or null: region 0 */
    double*        kr;
    double*        Pc;
    double*        Pj;
    double*        dKr_dS;
    double*        dPcj_dS;
} orc_krpc_batch;

/* IsoT_FIM::CalKrPc (src/OCPFluidMethod.cpp:1189-1199) with the
 * compositional model's default flow unit, FlowUnit_ODGW01
 * (src/FlowUnit.cpp:183-349: SWOF / SGOF interpolation, Stone II oil
 * relative permeability). The reference oracle only. */
int orc_krpc(int nreg, const orc_satfunc* reg, const orc_krpc_batch* batch, int nthreads, double* seconds);

/* Saturation functions of one region in the SWFN / SGFN / SOF3 family
 * (row-major, 3 columns): Sw, krw, Pcow; Sg, krg, Pcgo; So, krow, krog. */
typedef struct {
    int32_t       nrow_swfn, nrow_sgfn, nrow_sof3, pad;
    const double* swfn;
    const double* sgfn;
    const double* sof3;
} orc_satfunc3;

/* The same with FlowUnit_ODGW02 (src/FlowUnit.cpp:522-671), the flow unit
 * the reference selects when SOF3 is given (src/Bulk.cpp:271-279). The
 * reference oracle only. */
int orc_krpc_sof3(int nreg, const orc_satfunc3* reg, const orc_krpc_batch* batch, int nthreads, double* seconds);

/* Identifies the implementation: "reference" or "port". */
const char* orc_kind(void);

#ifdef __cplusplus
}
#endif

#endif /* OCP_ORACLE_API_H */
