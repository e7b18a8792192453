// flash_warp.cuh -- PhaseSplit's restart loop on one warp per cell, for the
// few cells whose split keeps restarting (near-critical mixtures whose
// successive substitution converges over tens of thousands of iterations).
//
// Such a cell is a chain of tens of thousands of dependent iterations, so
// its time is latency: on one thread an FP64 division costs ~115 cycles and
// independent divisions do not overlap, a logarithm ~270, acos + cos ~475.
// Here every lane holds the whole cell state (a CellFlash) and takes the
// same branches, while the operations of an iteration that are independent
// of one another run on different lanes and are then broadcast with
// shuffles:
//   * Rachford-Rice: lane i forms component i's residual term, lane 16 + i
//     its Jacobian term (two divisions); the sums are then taken on every
//     lane in the reference's order;
//   * compositions, fugacity ratios and K: one component per lane;
//   * fugacities: phase 0 on lanes 0-15 and phase 1 on lanes 16-31 at once;
//     within a half, lanes 0-2 polish the three roots of the cubic and form
//     the three pieces of the root choice, lanes 0-3 the two logarithms and
//     two reciprocals of CalFugPhi, and lane 16j + i the exponential of
//     phi_ij.
// Lanes that form different pieces run the same instructions on operands
// chosen per lane (one division, then one logarithm): different functions
// on different lanes of a warp would run one after another.
// Each value is formed by the same expression as in the one-thread form
// (shared helpers); the two agree to rounding (the compiler fuses
// multiply-adds per kernel), so an iteration count that ends on a
// convergence threshold can differ by a step.
#pragma once

#include "flash_cell.cuh"

namespace ocpf {

constexpr unsigned WARP_ALL = 0xffffffffu;

template <int NC>
struct WarpSplit {
    static_assert(NC <= 16, "one half-warp per phase holds at most 16 components");
    CellFlash<NC>& f;
    const int      lane, half, q;
    const unsigned hmask;

    __device__ __forceinline__ explicit WarpSplit(CellFlash<NC>& cell)
        : f(cell),
          lane(threadIdx.x & 31),
          half((threadIdx.x & 31) >> 4),
          q(threadIdx.x & 15),
          hmask(((threadIdx.x & 31) >> 4) ? 0xffff0000u : 0x0000ffffu)
    {
    }

    // component q's entry of a per-component register array
    __device__ __forceinline__ double pick(const double* v) const
    {
        double r = v[0];
#pragma unroll
        for (int i = 1; i < NC; i++)
            if (q == i) r = v[i];
        return r;
    }

    // RachfordRice2, src/MixtureComp.cpp:1907-1959 (CellFlash::rachford_rice2):
    // lane i forms component i's residual term, lane 16 + i its Jacobian
    // term; the sums run on every lane in the reference's order.
    __device__ void rachford_rice2()
    {
        double Kmin = f.Ks[0], Kmax = f.Ks[0];
#pragma unroll
        for (int i = 1; i < NC; i++) {
            if (f.Ks[i] < Kmin) Kmin = f.Ks[i];
            if (f.Ks[i] > Kmax) Kmax = f.Ks[i];
        }
        const double bound = 1 / (1 - (half ? Kmin : Kmax));
        const double numin = __shfl_sync(WARP_ALL, bound, 0);
        const double numax = __shfl_sync(WARP_ALL, bound, 16);
        double       v     = 0.5 * (numin + numax);
        // loop-invariant parts of component q's terms, formed as the
        // one-thread form forms them: z km1 / tmp and z km1 km1 / (tmp tmp)
        const double km1 = pick(f.Ks) - 1;
        const double zk  = pick(f.zi) * km1;
        const double num = half ? zk * km1 : zk;
        int          iter = 0;
        while (true) {
            const double tmp  = 1 + v * km1;
            const double term = num / (half ? tmp * tmp : tmp);
            double       rj = 0, J = 0;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                rj += __shfl_sync(WARP_ALL, term, i);
                J -= __shfl_sync(WARP_ALL, term, 16 + i);
            }
            if (fabs(rj) < f.F.rr_tol || iter > f.F.rr_maxit) break;
            const double dnuj  = -rj / J;
            const double tmpnu = v + dnuj;
            if (tmpnu < numax && tmpnu > numin)
                v = tmpnu;
            else if (dnuj > 0)
                v = (v + numax) / 2;
            else
                v = (v + numin) / 2;
            iter++;
        }
        f.it_rr += iter;
        f.nu[0] = v;
        f.nu[1] = 1 - v;
    }

    // UpdateXRR (src/MixtureComp.cpp:2030-2043): lane i forms x_1i and x_0i.
    __device__ __forceinline__ void update_x()
    {
        const double tmp = 1 + f.nu[0] * (pick(f.Ks) - 1);
        const double x1  = pick(f.zi) / tmp;
        const double x0  = pick(f.Ks) * x1;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            f.x[1][i] = __shfl_sync(WARP_ALL, x1, i);
            f.x[0][i] = __shfl_sync(WARP_ALL, x0, i);
        }
    }

    // One phase of CalFugPhi (src/MixtureComp.cpp:993-1101) on each half:
    // half j holds phase j's composition xj; returns phi of component q of
    // phase `half` and leaves the phase's a, b and Z on every lane of the
    // half. Within a half, lanes 0-2 polish the cubic's roots and lanes 0-3
    // form the two logarithms and two reciprocals.
    __device__ __forceinline__ double fug_lane(const double* xj, double& aj, double& bj, double& zj) const
    {
        double t[NC];
        mix_ab<NC>(f.F, f.sA, f.Bi, xj, t, aj, bj);
        zj              = sol_eos_group(aj, bj, hmask, half << 4, q);
        const int    base  = half << 4;
        const double piece = fug_piece(q < 4 ? q : 3, zj, aj, bj);
        const double L1  = __shfl_sync(WARP_ALL, piece, base);
        const double L2  = __shfl_sync(WARP_ALL, piece, base + 1);
        const double ib  = __shfl_sync(WARP_ALL, piece, base + 2);
        const double ia  = __shfl_sync(WARP_ALL, piece, base + 3);
        const double cf  = div_const(aj, D1MD2, RCPD1MD2) * ib;
        const double zm1 = zj - 1;
        double       tq = 0, bq = 0;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            if (q == i) {
                tq = t[i];
                bq = f.Bi[i];
            }
        }
        return q < NC ? phi_term(bq * ib, tq, ia, zm1, L1, cf, L2) : 0.0;
    }

    // The state of both phases on every lane from the per-lane pieces: a, b,
    // Z from lanes 0 and 16, phi_ji from lane 16 j + i, and f = phi x P.
    __device__ __forceinline__ void share_phases(double ph, double aj, double bj, double zj)
    {
#pragma unroll
        for (int j = 0; j < 2; j++) {
            f.Aj[j] = __shfl_sync(WARP_ALL, aj, 16 * j);
            f.Bj[j] = __shfl_sync(WARP_ALL, bj, 16 * j);
            f.Zj[j] = __shfl_sync(WARP_ALL, zj, 16 * j);
#pragma unroll
            for (int i = 0; i < NC; i++) {
                const double p = __shfl_sync(WARP_ALL, ph, 16 * j + i);
                f.phi[j][i]    = p;
                f.fug[j][i]    = p * f.x[j][i] * f.P;
            }
        }
    }

    // CalFugPhiAll for NP = 2 (src/MixtureComp.cpp:1103-1145) from f.x.
    __device__ __forceinline__ void fug_phi_all()
    {
        double xj[NC];
#pragma unroll
        for (int k = 0; k < NC; k++) xj[k] = half ? f.x[1][k] : f.x[0][k];
        double aj, bj, zj;
        const double ph = fug_lane(xj, aj, bj, zj);
        share_phases(ph, aj, bj, zj);
    }

    // SplitSSM2 with UpdateXRR, src/MixtureComp.cpp:1847-1903, 2030-2043
    // (CellFlash::split_ssm2 with the pieces above).
    __device__ void split_ssm2(bool restart)
    {
        f.ssmsp_conflag = true;
        double Se       = 1;
        double Stol     = f.F.ssmsp_tol2;
        int    maxIt    = f.F.ssmsp_maxit;
        if (restart) {
            Stol *= 1e-1;
            maxIt *= 2;
        }
        if (f.Yt < 1.1) {
            Stol *= 1e-1;
            maxIt *= 2;
        }
        int iter = 0;
        while (Se > Stol) {
            rachford_rice2();
            update_x();
            fug_phi_all();
            // lane i: component i's squared fugacity-ratio residual; lane
            // 16 + i: its new K (one division on every lane)
            const double quo = (half ? pick(f.phi[1]) : pick(f.fug[1])) / (half ? pick(f.phi[0]) : pick(f.fug[0]));
            const double v   = half ? quo : sq(quo - 1);
            Se               = 0;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                Se      = __dadd_rn(Se, __shfl_sync(WARP_ALL, v, i));
                f.Ks[i] = __shfl_sync(WARP_ALL, v, 16 + i);
            }
            iter++;
            if (iter > maxIt) {
                f.ssmsp_conflag = false;
                break;
            }
        }
        f.ssmsp_realTol = sqrt(Se);
        f.it_ssmsp += iter;
    }

    // ln(f_1i / f_0i) of every component, one per lane, and their squared sum
    __device__ __forceinline__ double residual(double* res) const
    {
        const double r   = log(pick(f.fug[1]) / pick(f.fug[0]));
        double       eNR = 0;
#pragma unroll
        for (int i = 0; i < NC; i++) {
            res[i] = __shfl_sync(WARP_ALL, r, i);
            eNR += res[i] * res[i];
        }
        return eNR;
    }

    // SplitNR, src/MixtureComp.cpp:2057-2166 (CellFlash::split_nr with the
    // pieces above; the Newton step itself runs on every lane).
    __device__ void split_nr()
    {
        f.nrsp_conflag = false;
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int i = 0; i < NC; i++) f.n[j][i] = f.nu[j] * f.x[j][i];
        double res[NC];
        double eNR        = sqrt(residual(res));
        const double eNR0 = eNR;
        int          iter = 0;
        while (eNR > f.F.nrsp_tol) {
            const double en = f.sp_nr_update(res);
            fug_phi_all();
            eNR = sqrt(residual(res));
            iter++;
            if (eNR > eNR0 || iter > f.F.nrsp_maxit) break;
            if (en / (2 * NC) < 1e-8) {
                f.nrsp_conflag = true;
                break;
            }
        }
        f.nrsp_realTol = eNR;
        if (eNR < f.F.nrsp_tol) f.nrsp_conflag = true;
        f.it_nrsp += iter;
    }
};

}  // namespace ocpf
