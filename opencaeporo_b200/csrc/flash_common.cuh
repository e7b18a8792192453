// flash_common.cuh -- constants, the per-fluid constant block and small
// helpers shared by the flash kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ocp_flash.h"

namespace ocpf {

constexpr int MAXNC = OCPF_MAX_NC;
constexpr int NPH   = OCPF_NUM_PHASE;  // oil, gas, water

// include/OCPConst.hpp:37-69 and include/MixtureComp.hpp:350-351
constexpr double GAS_CONSTANT = 10.73159;
constexpr double PI_TRUNC     = 3.141592653;  // truncated, as the reference uses it
constexpr double CONV1        = 5.61458;
constexpr double CONV5        = 459.67;
constexpr double D1           = 2.41421356237;
constexpr double D2           = -0.41421356237;
constexpr double D1PD2        = D1 + D2;
constexpr double D1MD2        = D1 - D2;
constexpr double D1TD2        = D1 * D2;

// x / d, correctly rounded, for a constant divisor d given with its
// correctly rounded reciprocal rd = RN(1/d): q = RN(x rd) lies within one
// ulp of x / d, so the remainder r = x - d q is exact in one fused
// multiply-add and RN(q + r rd) is the correctly rounded quotient
// (Markstein's theorem: P. Markstein, "Computation of elementary functions
// on the IBM RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990;
// J.-M. Muller et al., Handbook of Floating-Point Arithmetic, 2nd ed., 2018,
// ch. 4). Three dependent FP64 operations in place of a division, with the
// same result bits. Zeros, non-finite values and magnitudes outside
// [1e-270, 1e270] (where r or r rd could leave the normal range) take the
// ordinary division.
__device__ __forceinline__ double div_const(double x, double d, double rd)
{
    const double ax = fabs(x);
    if (!(ax > 1e-270 && ax < 1e270)) return x / d;
    const double q = x * rd;
    const double r = fma(-d, q, x);
    return fma(r, rd, q);
}
constexpr double RCP3     = 1.0 / 3;
constexpr double RCP9     = 1.0 / 9;
constexpr double RCP54    = 1.0 / 54;
constexpr double RCPD1MD2 = 1.0 / D1MD2;

// Everything a flash of one fluid reads that does not depend on the cell.
// Passed by value as a __grid_constant__ kernel parameter, so that with a
// compile-time component count every access is a constant-bank operand.
// Fixed row stride MAXNC keeps those offsets compile-time constants.
struct FluidConst {
    int32_t nc;
    int32_t use_skip;
    int32_t rr_maxit, ssmsta_maxit, nrsta_maxit, ssmsp_maxit, nrsp_maxit, pad;
    double  rr_tol, ssmsta_tol2, ssmsta_eyt, nrsta_tol, ssmsp_tol2, nrsp_tol;
    double  Tc[MAXNC], Pc[MAXNC], Vc[MAXNC], Vcvis[MAXNC], MW[MAXNC], Acf[MAXNC];
    double  OmegaA[MAXNC], OmegaB[MAXNC], Vshift[MAXNC];
    double  mwi[MAXNC];          // PR m(omega), src/MixtureComp.cpp:923-929
    double  sqrtMW[MAXNC];       // sqrtMWi, src/MixtureComp.cpp:2323-2324
    double  muAux1I[MAXNC];      // src/MixtureComp.cpp:2330-2333
    double  lbc1[MAXNC];         // 5.4402 Tc^(1/6)
    double  lbc2[MAXNC];         // Pc^(2/3)
    double  omb[MAXNC * MAXNC];  // 1 - BIC, row stride MAXNC
    double  L[5];                // LBC coefficients x 10
    double  pvtw[5];
    double  std_rho_w;
    float   ombf[MAXNC * MAXNC];  // omb in FP32, for the mixed form's fugacities
    // learned initialiser (OCPF_FORM_FAST): input normalisation, confidence
    float   lin_mean[MAXNC + 2], lin_scale[MAXNC + 2];
    float   learn_conf;
    int32_t learn_on;
};

// per-cell status bits mirror OCPF_CELL_*
constexpr uint16_t ST_SSMSTA_CAP = OCPF_CELL_SSMSTA_CAP;
constexpr uint16_t ST_NRSTA_FAIL = OCPF_CELL_NRSTA_FAIL;
constexpr uint16_t ST_SSMSP_FAIL = OCPF_CELL_SSMSP_FAIL;
constexpr uint16_t ST_NRSP_FAIL  = OCPF_CELL_NRSP_FAIL;
constexpr uint16_t ST_COLLAPSED  = OCPF_CELL_COLLAPSED;
constexpr uint16_t ST_SINGULAR   = OCPF_CELL_SINGULAR;
constexpr uint16_t ST_NONFINITE  = OCPF_CELL_NONFINITE;
constexpr uint16_t ST_SPLIT_CAP  = OCPF_CELL_SPLIT_CAP;
constexpr uint16_t ST_GUARD      = OCPF_CELL_GUARD;

// Bound on PhaseSplit's restart loop (src/MixtureComp.cpp:1752-1757 has none:
// a cell whose restarts never converge loops there for ever). Converging
// cells need few restarts (at most 78 in the 1M-state workload, at most 4 in
// 262,144 states of wider P, T and composition ranges); cells that do not
// converge within the bound are reported with OCPF_CELL_SPLIT_CAP.
constexpr int SPLIT_RESTART_CAP = 200;

__device__ __forceinline__ double sq(double v) { return v * v; }
__device__ __forceinline__ double dlt(int i, int k) { return i == k ? 1.0 : 0.0; }

// Host-side derivation of the constant block from the C-ABI fluid; returns
// false on invalid input.
bool make_fluid_const(const ocpf_fluid& in, FluidConst& out);

}  // namespace ocpf
