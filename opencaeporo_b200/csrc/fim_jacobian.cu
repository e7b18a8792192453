// fim_jacobian.cu -- the consumer of the flash's derivatives: the bulk part
// of the FIM Jacobian as IsoT_FIM::AssembleMatBulksNew builds it
// (src/OCPFluidMethod.cpp:1569-1840), and the upstream choice of every
// connection and phase that precedes it (src/BulkConn.cpp:170-215).
//
//   * k_upwind, one thread per (phase, connection): upstream bulk and mean
//     density;
//   * k_conn_block, a group of connections per block: thread (row,
//     connection) builds that row of dF/dXp and dF/dXs of both ends in
//     shared memory, then thread (column, connection) forms that column of
//     dt (dF/dXp + dF/dXs dSec_dPri) (DaABpbC, src/DenseMat.cpp:75-94) for
//     both ends, so that each dSec_dPri entry is read once per connection
//     end; stored as the connection's off-diagonal blocks;
//   * k_diag_rows, one thread per (row, bulk): the accumulation block plus
//     every incident connection's diagonal contribution, gathered through a
//     per-bulk list in connection order, which is the order the reference's
//     AddDiag calls sum them in.
// Every operation is an explicitly rounded intrinsic in the reference's
// left-to-right expression order (x / 2 as x * 0.5, the same value); the dense product sums over k in order
// and adds the dF/dXp entry last, as dgemm with beta = 1 does.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "ocp_flash.h"

namespace ocpf {
namespace {

constexpr double J_CONV1 = 5.61458;      // include/OCPConst.hpp
constexpr double J_CONV2 = 1.12712E-3;   // Darcy constant, field units
constexpr double J_GRAV  = 0.00694444;   // GRAVITY_FACTOR
constexpr int    J_NP    = 3;

__device__ __forceinline__ double M(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double A(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double S(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double D(double a, double b) { return __ddiv_rn(a, b); }

struct ConnDev {
    int64_t        nb, nconn;
    const int64_t* bId;
    const int64_t* eId;
    const double*  area;
    const int64_t* adj_off;  // [nb + 1]
    const int64_t* adj;      // c + 1 at the begin bulk, -(c + 1) at the end bulk, c increasing
};

__global__ void __launch_bounds__(256) k_upwind(const ConnDev C, const ocpf_jac_bulk B, int32_t* up, double* uprho)
{
    const int64_t nc = C.nconn, nb = C.nb;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < J_NP * nc;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int     j = (int)(t / nc);
        const int64_t c = t - j * nc;
        const int64_t b = C.bId[c], e = C.eId[c];
        const bool    xb = B.phaseExist[j * nb + b] != 0, xe = B.phaseExist[j * nb + e] != 0;
        double        rho;
        if (xb && xe) {
            const double sb = B.S[j * nb + b], se = B.S[j * nb + e];
            rho = D(A(M(B.rho[j * nb + b], sb), M(B.rho[j * nb + e], se)), A(sb, se));
        } else if (xb) {
            rho = B.rho[j * nb + b];
        } else if (xe) {
            rho = B.rho[j * nb + e];
        } else {
            up[j * nc + c]    = (int32_t)b;
            uprho[j * nc + c] = 0;
            continue;
        }
        const double gr = M(J_GRAV, rho);
        const double dP = S(S(B.Pj[j * nb + b], M(gr, B.depth[b])), S(B.Pj[j * nb + e], M(gr, B.depth[e])));
        up[j * nc + c]    = (int32_t)(dP < 0 ? e : b);
        uprho[j * nc + c] = rho;
    }
}

// The compact dSec_dPri layout of one bulk: sderivative flags and composition
// counts of its phases.
struct SecShape {
    bool sd[J_NP];
    int  vn[J_NP];
    int  ncol;  // rows of its dSec_dPri = columns of its dF/dXs
};

__device__ __forceinline__ SecShape sec_shape(const ocpf_jac_bulk& B, int64_t nb, int64_t n)
{
    SecShape s;
    s.ncol = 0;
#pragma unroll
    for (int j = 0; j < J_NP; j++) {
        s.sd[j] = B.pSderExist[j * nb + n] != 0;
        s.vn[j] = (int)B.pVnumCom[j * nb + n];
        s.ncol += s.vn[j] + (s.sd[j] ? 1 : 0);
    }
    return s;
}

// Connections per block of k_conn_block and its shared-memory size: the
// dF/dXs rows of both ends of every connection of the block.
template <int NCOM>
struct ConnBlock {
    static constexpr int NCOL = NCOM + 1;
    static constexpr int NSEC = 3 + 2 * (NCOM - 1);  // dSec_dPri rows of a two-phase bulk
    static constexpr int CPB  = NCOM <= 7 ? 16 : (NCOM <= 10 ? 8 : 4);
    static constexpr int TPC  = NCOL <= 8 ? 8 : 16;  // threads per connection (>= NCOL)
    static constexpr int THREADS = CPB * TPC;
    // per connection, staged once: 11 scalars of each phase's upstream
    // (dP, xi, kr, mu, muP, xiP, rhoP of upstream, begin and end, transJ,
    // upstream exists), the 9 saturation derivatives of each phase (dPc of
    // both ends, dKr of upstream), and 5 composition partials of each phase
    // and component (rhox, xix, mux of upstream, rhox of begin and end)
    static constexpr int STG = 3 * 11 + 3 * 9 + 3 * 5 * NCOM;
    static constexpr size_t SMEM =
        sizeof(double) * (size_t)CPB * (2 * (NSEC * NCOM + NCOM) + STG) + sizeof(int) * CPB * 3;
    static_assert(NCOL <= TPC, "one thread per column");
};

// Phase 1, thread (i, connection): row i + 1 of dF/dXp (column 0 only) and
// of dF/dXs of both ends, accumulated in shared memory in the reference's
// order. Phase 2, thread (column, connection): that column of
// dt (dF/dXp + dF/dXs dSec_dPri) (DaABpbC + Dscalar) for both ends, the sum
// over k in order and the dF/dXp entry last, as dgemm with beta = 1 forms
// it; stored as (row eId, col bId) = -bmatB and (row bId, col eId) = bmatE.
template <int NCOM>
__global__ void __launch_bounds__(ConnBlock<NCOM>::THREADS) k_conn_block(const ConnDev C, const ocpf_jac_bulk B,
                                                                           const int32_t* up, const double* uprho,
                                                                           double dt, ocpf_jac_out O)
{
    using CB = ConnBlock<NCOM>;
    constexpr int NCOL = CB::NCOL, NSEC = CB::NSEC, CPB = CB::CPB;
    extern __shared__ double sm[];
    // rows[end][k][i][cl], prow[end][i][cl], then nsec[end][cl], ok[cl]
    double* rows = sm;
    double* prow = sm + (size_t)2 * NSEC * NCOM * CPB;
    double* stg  = prow + (size_t)2 * NCOM * CPB;
    int*    meta = (int*)(stg + (size_t)CB::STG * CPB);
    // staged values: scalar v of phase j, derivative q (= 3 j1 + which) of
    // phase j, partial w of phase j and component k
    auto SC = [&](int j, int v, int cl) -> double& { return stg[(j * 11 + v) * CPB + cl]; };
    auto PK = [&](int j, int q, int cl) -> double& { return stg[(33 + j * 9 + q) * CPB + cl]; };
    auto CX = [&](int j, int k, int w, int cl) -> double& { return stg[(60 + (j * NCOM + k) * 5 + w) * CPB + cl]; };
    auto R  = [&](int end, int k, int i, int cl) -> double& { return rows[((end * NSEC + k) * NCOM + i) * CPB + cl]; };
    auto PR = [&](int end, int i, int cl) -> double& { return prow[(end * NCOM + i) * CPB + cl]; };
    const int64_t nc = C.nconn, nb = C.nb;
    const int     lane_c = threadIdx.x % CPB, part = threadIdx.x / CPB;
    for (int64_t g0 = (int64_t)blockIdx.x * CPB; g0 < nc; g0 += (int64_t)gridDim.x * CPB) {
        const int64_t c     = g0 + lane_c;
        const bool    live  = c < nc;
        const int     i     = part;  // phase 1: row i + 1
        __syncthreads();             // the previous group's phase 2 is done with the shared rows
        if (i < NCOM) {
            for (int k = 0; k < NSEC; k++) R(0, k, i, lane_c) = R(1, k, i, lane_c) = 0;
            PR(0, i, lane_c) = PR(1, i, lane_c) = 0;
        }
        // phase 0: each connection's per-phase upstream data, once
        if (live) {
            const int64_t bId = C.bId[c], eId = C.eId[c];
            const double  Akd    = M(J_CONV1 * J_CONV2, C.area[c]);
            const double  dGamma = M(J_GRAV, S(B.depth[bId], B.depth[eId]));
            for (int j = part; j < J_NP; j += CB::TPC) {
                const int64_t u   = up[j * nc + c];
                const bool    xb  = B.phaseExist[j * nb + bId] != 0, xe = B.phaseExist[j * nb + eId] != 0;
                const bool    val = (u == bId || u == eId);
                const bool    exU = val && (u == bId ? xb : xe);
                SC(j, 10, lane_c) = exU ? 1.0 : 0.0;
                if (exU) {
                    const int64_t uj = j * nb + u;
                    SC(j, 0, lane_c) = S(S(B.Pj[j * nb + bId], B.Pj[j * nb + eId]), M(uprho[j * nc + c], dGamma));
                    SC(j, 1, lane_c) = B.xi[uj];
                    SC(j, 2, lane_c) = B.kr[uj];
                    SC(j, 3, lane_c) = B.mu[uj];
                    SC(j, 4, lane_c) = B.muP[uj];
                    SC(j, 5, lane_c) = B.xiP[uj];
                    SC(j, 6, lane_c) = B.rhoP[uj];
                    SC(j, 7, lane_c) = xb ? B.rhoP[j * nb + bId] : 0.0;
                    SC(j, 8, lane_c) = xe ? B.rhoP[j * nb + eId] : 0.0;
                    SC(j, 9, lane_c) = D(M(Akd, B.kr[uj]), B.mu[uj]);
                }
            }
            for (int q = part; q < 9; q += CB::TPC) {
                const int     j = q / 3, j1 = q % 3;
                const int64_t u = up[j * nc + c];
                const int64_t f = (int64_t)(3 * j + j1) * nb;
                PK(j, 3 * j1 + 0, lane_c) = B.dPcj_dS[f + bId];
                PK(j, 3 * j1 + 1, lane_c) = B.dPcj_dS[f + eId];
                PK(j, 3 * j1 + 2, lane_c) = (u == bId || u == eId) ? B.dKr_dS[f + u] : 0.0;
            }
            for (int q = part; q < J_NP * NCOM; q += CB::TPC) {
                const int     j = q / NCOM, k = q % NCOM;
                const int64_t u = up[j * nc + c];
                const int64_t f = (int64_t)(j * NCOM + k) * nb;
                const bool    val = (u == bId || u == eId);
                CX(j, k, 0, lane_c) = val ? B.rhox[f + u] : 0.0;
                CX(j, k, 1, lane_c) = val ? B.xix[f + u] : 0.0;
                CX(j, k, 2, lane_c) = val ? B.mux[f + u] : 0.0;
                CX(j, k, 3, lane_c) = B.rhox[f + bId];
                CX(j, k, 4, lane_c) = B.rhox[f + eId];
            }
        }
        __syncthreads();
        if (live && i < NCOM) {
            const int64_t  bId = C.bId[c], eId = C.eId[c];
            const double   Akd    = M(J_CONV1 * J_CONV2, C.area[c]);
            const double   dGamma = M(J_GRAV, S(B.depth[bId], B.depth[eId]));
            const SecShape sB = sec_shape(B, nb, bId), sE = sec_shape(B, nb, eId);
            bool exB[J_NP], exE[J_NP];
#pragma unroll
            for (int j = 0; j < J_NP; j++) {
                exB[j] = B.phaseExist[j * nb + bId] != 0;
                exE[j] = B.phaseExist[j * nb + eId] != 0;
            }
            // shapes a flash writes: at most NCOM - 1 compositions per phase
            // and NSEC dSec_dPri rows; anything else (and an upstream bulk
            // that is neither end) gives NaN blocks instead of an access
            // outside the arrays
            bool ok = sB.ncol <= NSEC && sE.ncol <= NSEC;
#pragma unroll
            for (int j = 0; j < J_NP; j++) {
                ok = ok && sB.vn[j] >= 0 && sB.vn[j] < NCOM && sE.vn[j] >= 0 && sE.vn[j] < NCOM;
                const int64_t u = up[j * nc + c];
                ok = ok && (u == bId || u == eId);
            }
            if (i == 0) {
                meta[lane_c]           = ok ? sB.ncol : 0;
                meta[CPB + lane_c]     = ok ? sE.ncol : 0;
                meta[2 * CPB + lane_c] = ok ? 1 : 0;
            }
            if (ok) {
                double pB = 0, pE = 0;
                int    jxB = (sB.sd[0] ? 1 : 0) + (sB.sd[1] ? 1 : 0) + (sB.sd[2] ? 1 : 0);
                int    jxE = (sE.sd[0] ? 1 : 0) + (sE.sd[1] ? 1 : 0) + (sE.sd[2] ? 1 : 0);
                for (int j = 0; j < J_NP; j++) {
                    const int64_t uId = up[j * nc + c];
                    const bool    exU = SC(j, 10, lane_c) != 0;
                    if (!exU) {
                        jxB += sB.vn[j];
                        jxE += sE.vn[j];
                        continue;
                    }
                    const double dP = SC(j, 0, lane_c), xi = SC(j, 1, lane_c), mu = SC(j, 3, lane_c);
                    const double muP = SC(j, 4, lane_c), xiP = SC(j, 5, lane_c), rhoP = SC(j, 6, lane_c);
                    const double transJ  = SC(j, 9, lane_c);
                    const double xij     = B.xij[(int64_t)(j * NCOM + i) * nb + uId];
                    const double transIJ = M(M(xij, xi), transJ);
                    pB = A(pB, transIJ);
                    pE = S(pE, transIJ);
                    double tmp = M(M(M(xij, transJ), xiP), dP);
                    tmp        = A(tmp, M(D(M(-transIJ, muP), mu), dP));
                    if (!exE[j]) {
                        tmp = A(tmp, M(transIJ, M(-rhoP, dGamma)));
                        pB  = A(pB, tmp);
                    } else if (!exB[j]) {
                        tmp = A(tmp, M(transIJ, M(-rhoP, dGamma)));
                        pE  = A(pE, tmp);
                    } else {
                        pB = A(pB, M(M(transIJ, M(-SC(j, 7, lane_c), dGamma)), 0.5));
                        pE = A(pE, M(M(transIJ, M(-SC(j, 8, lane_c), dGamma)), 0.5));
                        if (bId == uId)
                            pB = A(pB, tmp);
                        else
                            pE = A(pE, tmp);
                    }
                    int          j1SB = 0, j1SE = 0;
                    const double fk   = D(M(M(Akd, xij), xi), mu);  // Akd xij xi / mu
                    if (bId == uId) {
#pragma unroll
                        for (int j1 = 0; j1 < J_NP; j1++) {
                            if (sB.sd[j1]) {
                                double& r = R(0, j1SB, i, lane_c);
                                r         = A(r, M(transIJ, PK(j, 3 * j1 + 0, lane_c)));
                                r         = A(r, M(M(fk, PK(j, 3 * j1 + 2, lane_c)), dP));
                                j1SB++;
                            }
                            if (sE.sd[j1]) {
                                double& r = R(1, j1SE, i, lane_c);
                                r         = S(r, M(transIJ, PK(j, 3 * j1 + 1, lane_c)));
                                j1SE++;
                            }
                        }
                        const int nv = sB.vn[j];
#pragma unroll
                        for (int k = 0; k < NCOM - 1; k++) {
                            if (k >= nv) break;
                            const double rx = exE[j] ? M(CX(j, k, 3, lane_c), 0.5) : CX(j, k, 0, lane_c);
                            double       v  = M(M(-transIJ, rx), dGamma);
                            v               = A(v, M(M(M(xij, transJ), CX(j, k, 1, lane_c)), dP));
                            v               = A(v, M(D(M(-transIJ, CX(j, k, 2, lane_c)), mu), dP));
                            double& r       = R(0, jxB + k, i, lane_c);
                            r               = A(r, v);
                            if (exE[j]) {
                                double& re = R(1, jxE + k, i, lane_c);
                                re         = A(re, M(M(M(-transIJ, CX(j, k, 4, lane_c)), 0.5), dGamma));
                            }
                        }
                        if (i < nv) {
                            double& r = R(0, jxB + i, i, lane_c);
                            r         = A(r, M(M(xi, transJ), dP));
                        }
                    } else {
#pragma unroll
                        for (int j1 = 0; j1 < J_NP; j1++) {
                            if (sB.sd[j1]) {
                                double& r = R(0, j1SB, i, lane_c);
                                r         = A(r, M(transIJ, PK(j, 3 * j1 + 0, lane_c)));
                                j1SB++;
                            }
                            if (sE.sd[j1]) {
                                double& r = R(1, j1SE, i, lane_c);
                                r         = S(r, M(transIJ, PK(j, 3 * j1 + 1, lane_c)));
                                r         = A(r, M(M(fk, PK(j, 3 * j1 + 2, lane_c)), dP));
                                j1SE++;
                            }
                        }
                        const int nv = sE.vn[j];
#pragma unroll
                        for (int k = 0; k < NCOM - 1; k++) {
                            if (k >= nv) break;
                            const double rx = exB[j] ? M(CX(j, k, 4, lane_c), 0.5) : CX(j, k, 0, lane_c);
                            double       v  = M(M(-transIJ, rx), dGamma);
                            v               = A(v, M(M(M(xij, transJ), CX(j, k, 1, lane_c)), dP));
                            v               = A(v, M(D(M(-transIJ, CX(j, k, 2, lane_c)), mu), dP));
                            double& r       = R(1, jxE + k, i, lane_c);
                            r               = A(r, v);
                            if (exB[j]) {
                                double& rb = R(0, jxB + k, i, lane_c);
                                rb         = A(rb, M(M(M(-transIJ, CX(j, k, 3, lane_c)), 0.5), dGamma));
                            }
                        }
                        if (i < nv) {
                            double& r = R(1, jxE + i, i, lane_c);
                            r         = A(r, M(M(xi, transJ), dP));
                        }
                    }
                    jxB += sB.vn[j];
                    jxE += sE.vn[j];
                }
                PR(0, i, lane_c) = pB;
                PR(1, i, lane_c) = pE;
            }
        }
        __syncthreads();
        const int col = part;  // phase 2: column col
        if (live && col < NCOL) {
            const int64_t bId = C.bId[c], eId = C.eId[c];
            const bool    ok  = meta[2 * CPB + lane_c] != 0;
            const double  nan = __longlong_as_double(0x7ff8000000000000LL);
            for (int end = 0; end < 2; end++) {
                const int64_t n    = end ? eId : bId;
                const int     nsec = meta[end * CPB + lane_c];
                double*       dst  = end ? O.offBE : O.offEB;
                dst[(int64_t)col * nc + c] = !ok ? nan : (end ? M(0.0, dt) : -M(0.0, dt));  // row 0
                double sec[NSEC];
#pragma unroll
                for (int k = 0; k < NSEC; k++) sec[k] = k < nsec ? B.dSec_dPri[(int64_t)(k * NCOL + col) * nb + n] : 0.0;
#pragma unroll
                for (int r = 1; r <= NCOM; r++) {
                    double v = nan;
                    if (ok) {
                        double s2 = 0;
#pragma unroll
                        for (int k = 0; k < NSEC; k++)
                            if (k < nsec) s2 = A(s2, M(R(end, k, r - 1, lane_c), sec[k]));
                        v = M(A(s2, col == 0 ? PR(end, r - 1, lane_c) : 0.0), dt);
                        if (!end) v = -v;
                    }
                    dst[(int64_t)(r * NCOL + col) * nc + c] = v;
                }
            }
        }
    }
}

template <int NCOM>
__global__ void __launch_bounds__(128) k_diag_rows(const ConnDev C, const ocpf_jac_bulk B, ocpf_jac_out O)
{
    constexpr int NCOL = NCOM + 1;
    const int64_t nb = C.nb, nc = C.nconn;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < NCOL * nb;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int     r = (int)(t / nb);
        const int64_t n = t - r * nb;
        double        d[NCOL];
        // accumulation block (src/OCPFluidMethod.cpp:1587-1596)
#pragma unroll
        for (int col = 0; col < NCOL; col++) d[col] = (r >= 1 && col == r) ? 1.0 : 0.0;
        if (r == 0) {
            d[0] = S(M(B.v[n], B.poroP[n]), B.vfP[n]);
#pragma unroll
            for (int k = 0; k < NCOM; k++) d[k + 1] = -B.vfi[(int64_t)k * nb + n];
        }
        for (int64_t q = C.adj_off[n]; q < C.adj_off[n + 1]; q++) {
            const int64_t a   = C.adj[q];
            const int64_t c   = a > 0 ? a - 1 : -a - 1;
            const double* src = a > 0 ? O.offEB : O.offBE;  // +bmatB = -offEB, -bmatE = -offBE
#pragma unroll
            for (int col = 0; col < NCOL; col++) d[col] = A(d[col], -src[(int64_t)(r * NCOL + col) * nc + c]);
        }
#pragma unroll
        for (int col = 0; col < NCOL; col++) O.diag[(int64_t)(r * NCOL + col) * nb + n] = d[col];
    }
}

template <int NCOM>
cudaError_t launch_jac(const ConnDev& C, const ocpf_jac_bulk& B, const int32_t* up, const double* uprho, double dt,
                       const ocpf_jac_out& O, int sms, cudaStream_t st)
{
    using CB = ConnBlock<NCOM>;
    // per device; cheap, so on every launch
    cudaFuncSetAttribute(k_conn_block<NCOM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CB::SMEM);
    const int64_t t2 = (NCOM + 1) * C.nb;
    const int     g1 = (int)std::min<int64_t>((C.nconn + CB::CPB - 1) / CB::CPB, (int64_t)sms * 8);
    const int     g2 = (int)std::min<int64_t>((t2 + 127) / 128, (int64_t)sms * 16);
    if (C.nconn > 0) k_conn_block<NCOM><<<g1, CB::THREADS, CB::SMEM, st>>>(C, B, up, uprho, dt, O);
    if (C.nb > 0) k_diag_rows<NCOM><<<g2, 128, 0, st>>>(C, B, O);
    return cudaGetLastError();
}

}  // namespace
}  // namespace ocpf

struct ocpf_conn {
    int              device, sms;
    ocpf::ConnDev    d;
    void*            mem;
};

extern "C" int ocpf_conn_create(int64_t nbulk, int64_t nconn, const int64_t* bId, const int64_t* eId,
                                const double* area, int device, ocpf_conn** out)
{
    using namespace ocpf;
    if (!out) return OCPF_EINVAL;
    *out = nullptr;
    if (nbulk < 1 || nconn < 0 || (nconn > 0 && (!bId || !eId || !area))) return OCPF_EINVAL;
    if (nconn > 0x3fffffffLL) return OCPF_EINVAL;
    for (int64_t c = 0; c < nconn; c++)
        if (bId[c] < 0 || bId[c] >= nbulk || eId[c] < 0 || eId[c] >= nbulk || bId[c] == eId[c]) return OCPF_EINVAL;
    // per-bulk incident connections in connection order
    std::vector<int64_t> off(nbulk + 1, 0), adj(2 * nconn);
    for (int64_t c = 0; c < nconn; c++) {
        off[bId[c] + 1]++;
        off[eId[c] + 1]++;
    }
    for (int64_t n = 0; n < nbulk; n++) off[n + 1] += off[n];
    std::vector<int64_t> pos(off.begin(), off.end() - 1);
    for (int64_t c = 0; c < nconn; c++) {
        adj[pos[bId[c]]++] = c + 1;
        adj[pos[eId[c]]++] = -(c + 1);
    }
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return OCPF_ECUDA;
    ocpf_conn* h = new (std::nothrow) ocpf_conn;
    int        rc = h ? OCPF_OK : OCPF_ENOMEM;
    if (rc == OCPF_OK) {
        std::memset(h, 0, sizeof(*h));
        h->device = device;
        cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device);
        const size_t b1 = sizeof(int64_t) * (size_t)nconn, b2 = sizeof(double) * (size_t)nconn;
        const size_t b3 = sizeof(int64_t) * (size_t)(nbulk + 1), b4 = sizeof(int64_t) * (size_t)(2 * nconn);
        const size_t tot = 2 * b1 + b2 + b3 + b4 + 5 * 256;
        if (cudaMalloc(&h->mem, tot) != cudaSuccess) {
            rc = OCPF_ENOMEM;
        } else {
            char* p    = (char*)h->mem;
            auto  take = [&p](size_t b) {
                char* q = p;
                p += (b + 255) / 256 * 256;
                return q;
            };
            int64_t* dB  = (int64_t*)take(b1);
            int64_t* dE  = (int64_t*)take(b1);
            double*  dA  = (double*)take(b2);
            int64_t* dO  = (int64_t*)take(b3);
            int64_t* dJ  = (int64_t*)take(b4);
            cudaError_t e = cudaSuccess;
            if (nconn > 0) {
                e = cudaMemcpy(dB, bId, b1, cudaMemcpyHostToDevice);
                if (e == cudaSuccess) e = cudaMemcpy(dE, eId, b1, cudaMemcpyHostToDevice);
                if (e == cudaSuccess) e = cudaMemcpy(dA, area, b2, cudaMemcpyHostToDevice);
                if (e == cudaSuccess) e = cudaMemcpy(dJ, adj.data(), b4, cudaMemcpyHostToDevice);
            }
            if (e == cudaSuccess) e = cudaMemcpy(dO, off.data(), b3, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) rc = OCPF_ECUDA;
            h->d = ConnDev{nbulk, nconn, dB, dE, dA, dO, dJ};
        }
    }
    if (rc != OCPF_OK && h) {
        if (h->mem) cudaFree(h->mem);
        delete h;
        h = nullptr;
    }
    if (prev != device) cudaSetDevice(prev);
    *out = h;
    return rc;
}

extern "C" int ocpf_conn_destroy(ocpf_conn* h)
{
    if (!h) return OCPF_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    cudaFree(h->mem);
    if (prev != h->device) cudaSetDevice(prev);
    delete h;
    return OCPF_OK;
}

extern "C" int ocpf_fim_upwind(ocpf_conn* h, const ocpf_jac_bulk* bk, int32_t* upblock, double* upblock_rho,
                               void* stream)
{
    using namespace ocpf;
    if (!h || !bk || !upblock || !upblock_rho || !bk->phaseExist || !bk->S || !bk->rho || !bk->Pj || !bk->depth)
        return OCPF_EINVAL;
    if (h->d.nconn == 0) return OCPF_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != h->device) cudaSetDevice(h->device);
    const int64_t t = J_NP * h->d.nconn;
    const int     g = (int)std::min<int64_t>((t + 255) / 256, (int64_t)h->sms * 8);
    k_upwind<<<g, 256, 0, (cudaStream_t)stream>>>(h->d, *bk, upblock, upblock_rho);
    const cudaError_t e = cudaGetLastError();
    if (prev != h->device) cudaSetDevice(prev);
    return e == cudaSuccess ? OCPF_OK : OCPF_ECUDA;
}

extern "C" int ocpf_fim_jacobian(ocpf_conn* h, int nc, double dt, const ocpf_jac_bulk* bk, const int32_t* upblock,
                                 const double* upblock_rho, ocpf_jac_out* out, void* stream)
{
    using namespace ocpf;
    if (!h || !bk || !out || !out->diag || !out->offEB || !out->offBE) return OCPF_EINVAL;
    if (h->d.nconn > 0 && (!upblock || !upblock_rho)) return OCPF_EINVAL;
    const ocpf_jac_bulk& B = *bk;
    if (!B.phaseExist || !B.pSderExist || !B.pVnumCom || !B.xi || !B.mu || !B.muP || !B.xiP || !B.rhoP || !B.xij ||
        !B.rhox || !B.xix || !B.mux || !B.dSec_dPri || !B.vfP || !B.vfi || !B.kr || !B.Pj || !B.dKr_dS ||
        !B.dPcj_dS || !B.v || !B.poroP || !B.depth)
        return OCPF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != h->device) cudaSetDevice(h->device);
    cudaError_t  e  = cudaSuccess;
    cudaStream_t st = (cudaStream_t)stream;
    switch (nc) {
        case 3: e = launch_jac<4>(h->d, B, upblock, upblock_rho, dt, *out, h->sms, st); break;
        case 6: e = launch_jac<7>(h->d, B, upblock, upblock_rho, dt, *out, h->sms, st); break;
        case 9: e = launch_jac<10>(h->d, B, upblock, upblock_rho, dt, *out, h->sms, st); break;
        case 12: e = launch_jac<13>(h->d, B, upblock, upblock_rho, dt, *out, h->sms, st); break;
        default:
            if (prev != h->device) cudaSetDevice(prev);
            return OCPF_EUNSUPPORTED;
    }
    if (prev != h->device) cudaSetDevice(prev);
    return e == cudaSuccess ? OCPF_OK : OCPF_ECUDA;
}
