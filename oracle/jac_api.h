/* TEST INFRASTRUCTURE ONLY: C entry of the Jacobian-assembly oracle
 * (oracle/jac_harness.cpp -> oracle/_ref/libocpjac.so), which runs the
 * reference's own IsoT_FIM::AssembleMatBulksNew (src/OCPFluidMethod.cpp:
 * 1569-1840) on caller-given Bulk and BulkConn arrays. All arrays are in the
 * reference's Bulk layout (cell-major: bulk n's values contiguous). */
#ifndef OCP_ORACLE_JAC_API_H
#define OCP_ORACLE_JAC_API_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int64_t nb;        /* bulks */
    int32_t ncom;      /* components, water included (Bulk::numCom) */
    int32_t lend;      /* doubles per bulk of dSec_dPri (Bulk::maxLendSdP) */
    const double* v; const double* poroP; const double* vfP; const double* vfi;   /* vfi: nb x ncom */
    const int32_t* phaseExist; const int32_t* pSderExist; const int32_t* pVnumCom; /* nb x 3 */
    const double* Pj; const double* depth; const double* xi; const double* kr; const double* mu;
    const double* muP; const double* xiP; const double* rhoP;                    /* nb x 3 (depth nb) */
    const double* xij; const double* rhox; const double* xix; const double* mux; /* nb x 3 x ncom */
    const double* dPcj_dS; const double* dKr_dS;                                 /* nb x 3 x 3 */
    const double* dSec_dPri;                                                     /* nb x lend */
    int64_t nconn;
    const int64_t* bId; const int64_t* eId; const double* area;
    const int64_t* upblock; const double* upblock_Rho;                           /* nconn x 3 */
    double dt;
    double* diag;   /* out: nb x ncol^2, ncol = ncom + 1 */
    double* offEB;  /* out: nconn x ncol^2, the block at row eId, column bId */
    double* offBE;  /* out: nconn x ncol^2, the block at row bId, column eId */
} OrcJac;

/* 0 on success; 1 when the linear system's rows do not hold the blocks in
 * the expected order (a change in the reference's scatter). */
int orc_assemble_bulks(const OrcJac* j);

#ifdef __cplusplus
}
#endif
#endif
