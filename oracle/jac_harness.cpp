// TEST INFRASTRUCTURE ONLY: runs the reference's own bulk-part assembly of
// the FIM Jacobian, IsoT_FIM::AssembleMatBulksNew (src/OCPFluidMethod.cpp:
// 1569-1840), compiled from the reference sources (see oracle/Makefile,
// target `jac`), on Bulk and BulkConn arrays the caller fills, and returns
// the blocks it scattered into its LinearSystem.
//
// Only the members the assembly reads are set: the Reservoir's bulk and conn
// are constructed in place inside raw storage, and the method (which reads
// nothing of its object) is called through a pointer to unconstructed
// storage, so that none of the simulator's set-up (grid, wells, solvers,
// the FASP library) is needed or linked. The LinearSystem is sized as the
// reference sizes it (AllocateRowMem).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <new>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

// the reference's headers with every member reachable from this harness
// (standard headers above, so that only the reference's classes change)
#define private public
#define protected public
#include "OCPFluidMethod.hpp"
#undef private
#undef protected

#include "jac_api.h"

extern "C" __attribute__((visibility("default"))) int orc_assemble_bulks(const OrcJac* j)
{
    const OCP_USI nb   = (OCP_USI)j->nb;
    const USI     np   = 3;
    const USI     nc   = (USI)j->ncom;
    const USI     ncol = nc + 1;
    const USI     bs   = ncol * ncol;

    alignas(Reservoir) static thread_local unsigned char rs_raw[sizeof(Reservoir)];
    alignas(IsoT_FIM) static thread_local unsigned char fim_raw[sizeof(IsoT_FIM)];
    Reservoir* rs = reinterpret_cast<Reservoir*>(rs_raw);
    Bulk*      bk = new (&rs->bulk) Bulk();
    BulkConn*  cn = new (&rs->conn) BulkConn();

    auto dv = [](const double* p, size_t n) { return std::vector<OCP_DBL>(p, p + n); };
    auto bv = [](const int32_t* p, size_t n) {
        std::vector<OCP_BOOL> r(n);
        for (size_t i = 0; i < n; i++) r[i] = p[i] ? OCP_TRUE : OCP_FALSE;
        return r;
    };
    bk->numBulk    = nb;
    bk->numPhase   = np;
    bk->numCom     = nc;
    bk->maxLendSdP = (USI)j->lend;
    bk->v          = dv(j->v, nb);
    bk->poroP      = dv(j->poroP, nb);
    bk->vfP        = dv(j->vfP, nb);
    bk->vfi        = dv(j->vfi, (size_t)nb * nc);
    bk->phaseExist = bv(j->phaseExist, (size_t)nb * np);
    bk->pSderExist = bv(j->pSderExist, (size_t)nb * np);
    bk->pVnumCom.resize((size_t)nb * np);
    for (size_t i = 0; i < (size_t)nb * np; i++) bk->pVnumCom[i] = (USI)j->pVnumCom[i];
    bk->Pj        = dv(j->Pj, (size_t)nb * np);
    bk->depth     = dv(j->depth, nb);
    bk->xi        = dv(j->xi, (size_t)nb * np);
    bk->kr        = dv(j->kr, (size_t)nb * np);
    bk->mu        = dv(j->mu, (size_t)nb * np);
    bk->muP       = dv(j->muP, (size_t)nb * np);
    bk->xiP       = dv(j->xiP, (size_t)nb * np);
    bk->rhoP      = dv(j->rhoP, (size_t)nb * np);
    bk->xij       = dv(j->xij, (size_t)nb * np * nc);
    bk->rhox      = dv(j->rhox, (size_t)nb * np * nc);
    bk->xix       = dv(j->xix, (size_t)nb * np * nc);
    bk->mux       = dv(j->mux, (size_t)nb * np * nc);
    bk->dPcj_dS   = dv(j->dPcj_dS, (size_t)nb * np * np);
    bk->dKr_dS    = dv(j->dKr_dS, (size_t)nb * np * np);
    bk->dSec_dPri = dv(j->dSec_dPri, (size_t)nb * j->lend);

    cn->numConn = (OCP_USI)j->nconn;
    cn->iteratorConn.resize(j->nconn);
    cn->upblock.resize((size_t)j->nconn * np);
    cn->upblock_Rho.resize((size_t)j->nconn * np);
    for (int64_t c = 0; c < j->nconn; c++) {
        BulkPair& p = cn->iteratorConn[c];
        p.bId       = (OCP_USI)j->bId[c];
        p.eId       = (OCP_USI)j->eId[c];
        p.area      = j->area[c];
        for (USI k = 0; k < np; k++) {
            cn->upblock[c * np + k]     = (OCP_USI)j->upblock[c * np + k];
            cn->upblock_Rho[c * np + k] = j->upblock_Rho[c * np + k];
        }
    }

    LinearSystem ls;
    ls.AllocateRowMem(nb, ncol);
    const IsoT_FIM* fim = reinterpret_cast<const IsoT_FIM*>(fim_raw);
    fim->AssembleMatBulksNew(ls, *rs, j->dt);

    // read the rows back: the diagonal block first, then the off-diagonal
    // blocks in the order the connections inserted them
    int rc = 0;
    std::vector<size_t> next(nb, 1);
    for (OCP_USI n = 0; n < nb && rc == 0; n++) {
        if (ls.colId[n].empty() || ls.colId[n][0] != n || ls.val[n].size() < bs) rc = 1;
        else std::memcpy(j->diag + (size_t)n * bs, ls.val[n].data(), bs * sizeof(double));
    }
    for (int64_t c = 0; c < j->nconn && rc == 0; c++) {
        const OCP_USI b = (OCP_USI)j->bId[c], e = (OCP_USI)j->eId[c];
        const size_t  ke = next[e]++, kb = next[b]++;
        if (ls.colId[e].size() <= ke || ls.colId[e][ke] != b || ls.colId[b].size() <= kb || ls.colId[b][kb] != e) {
            rc = 1;
            break;
        }
        std::memcpy(j->offEB + (size_t)c * bs, ls.val[e].data() + ke * bs, bs * sizeof(double));
        std::memcpy(j->offBE + (size_t)c * bs, ls.val[b].data() + kb * bs, bs * sizeof(double));
    }
    cn->~BulkConn();
    bk->~Bulk();
    return rc;
}
