// flash_mixed.cuh -- the mixed-precision form's successive substitution:
// the iterations of the strict stability test (StableSSM) with the
// fugacities in FP32, while FP64 keeps
//   * the cubic's coefficients, its root count (the discriminant's sign) and
//     a Newton polish of every root, and the root choice where the Gibbs
//     difference is small (the full FP64 SolEoS where the discriminant
//     itself is small),
//   * the phase split: SplitSSM2 with its bracketed Rachford-Rice Newton,
//     and SplitNR. In FP32 the split's successive substitution changes the
//     outcome of the cells whose SplitNR the reference itself cannot settle
//     (it stops on a small step with a residual far above its tolerance;
//     such cells' results follow the exact arithmetic path), so it stays
//     FP64, the batched form's code,
//   * the end of every successive substitution: FP32 iterations stop at a
//     residual FP32 can resolve (SSM32_TOL2 below). A stability trial's end
//     point is then evaluated in FP64 and polished by StableNR; where that
//     Newton step fails (it has no globalisation), the trial continues by
//     FP64 substitution to the reference's tolerance and Newton runs again.
// Converged answers therefore agree with the FP64 form's to the reference's
// tolerances. Iteration counts differ from the reference's (they count FP32
// and FP64 iterations alike).
#pragma once

#include "flash_phased.cuh"

namespace ocpf {

// FP32 end test: the sum of squared log residuals. FP32 fugacities carry
// ~1e-6 relative error, so it sits two decades above that floor.
constexpr float SSM32_TOL2 = 1e-10f;

// FP32 mixing rule: t_i = sqrt(A_i) sum_k (1 - k_ik) sqrt(A_k) x_k,
// a = sum_i x_i t_i, b = sum_i B_i x_i (CalAjBj, src/MixtureComp.cpp:939-969).
template <int NC>
__device__ __forceinline__ void mix_ab32(const FluidConst& F, const float* sA, const float* Bi, const float* x,
                                         float* t, float& aj, float& bj)
{
    float w[NC];
#pragma unroll
    for (int k = 0; k < NC; k++) w[k] = sA[k] * x[k];
    aj = 0.f;
    bj = 0.f;
#pragma unroll
    for (int i = 0; i < NC; i++) {
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < NC; k++) s = fmaf(F.ombf[i * MAXNC + k], w[k], s);
        t[i] = sA[i] * s;
        aj   = fmaf(x[i], t[i], aj);
        bj   = fmaf(Bi[i], x[i], bj);
    }
}

// Z of the PR cubic for FP32 mixture parameters: coefficients, discriminant
// and root count in FP64; the trigonometric / Cardano root estimates in
// FP32; each root polished by FP64 Newton (NTcubicroot's rule); the
// smallest-or-largest choice by an FP32 Gibbs difference, redone in FP64
// when that difference is small. Close to the discriminant's zero (where
// FP32 root estimates are poor) the whole solve is the FP64 sol_eos.
// Follows SolEoS/CubicRoot, src/MixtureComp.cpp:889-914, 4999-5056.
__device__ __forceinline__ double sol_eos_mixed(double aj, double bj)
{
    const PrCubic cu(aj, bj);
    const double  scale = fmax(cu.R * cu.R, fabs(cu.Q3));
    if (!(fabs(cu.M) > 1e-6 * scale)) return sol_eos(aj, bj);
    if (cu.M > 0) {
        const float sM = sqrtf((float)cu.M);
        const float R  = (float)cu.R;
        const float t1 = -R + sM;
        const float t2 = R + sM;
        const float S  = copysignf(cbrtf(fabsf(t1)), t1);
        const float T  = -copysignf(cbrtf(fabsf(t2)), t2);
        return nt_polish((double)(S + T) - cu.a / 3, cu.a, cu.b, cu.c);
    }
    const float  theta = acosf((float)(cu.R / sqrt(cu.Q3)));
    const float  s2    = -2.f * sqrtf((float)cu.Q);
    const double a3    = cu.a / 3;
    const float  pt    = 2.f * (float)PI_TRUNC;
    const double z0    = nt_polish((double)(s2 * cosf(theta / 3.f)) - a3, cu.a, cu.b, cu.c);
    const double z1    = nt_polish((double)(s2 * cosf((theta + pt) / 3.f)) - a3, cu.a, cu.b, cu.c);
    const double z2    = nt_polish((double)(s2 * cosf((theta - pt) / 3.f)) - a3, cu.a, cu.b, cu.c);
    const double zmin  = fmin(z0, fmin(z1, z2));
    const double zmax  = fmax(z0, fmax(z1, z2));
    const float  g1    = __logf((float)((zmin - bj) / (zmax - bj)));
    const float  g2    = __logf((float)((zmin + D1 * bj) * (zmax + D2 * bj) / ((zmin + D2 * bj) * (zmax + D1 * bj))));
    const double k2    = aj / (bj * (D2 - D1));
    const double dG    = (zmax - zmin) + (double)g1 - k2 * (double)g2;
    if (fabs(dG) > 1e-4 * (fabs(zmax - zmin) + fabs((double)g1) + fabs(k2 * (double)g2)))
        return dG > 0 ? zmin : zmax;
    return pick_root(z0, z1, z2, aj, bj);
}

// FP32 fugacity coefficients ln(phi_i) of composition x (CalFugPhi,
// src/MixtureComp.cpp:993-1101) with the cubic of sol_eos_mixed.
template <int NC>
__device__ __forceinline__ void ln_phi32(const FluidConst& F, const float* sA, const float* Bi, const float* x,
                                         float* lnphi)
{
    float t[NC], aj, bj;
    mix_ab32<NC>(F, sA, Bi, x, t, aj, bj);
    const double Z   = sol_eos_mixed((double)aj, (double)bj);
    const double bd  = (double)bj;
    const float  L1  = __logf((float)(Z - bd));
    const float  L2  = __logf((float)((Z + D1 * bd) / (Z + D2 * bd)));
    const float  ib  = 1.f / bj;
    const float  ia  = 1.f / aj;
    const float  cf  = aj / (float)D1MD2 * ib;
    const float  zm1 = (float)(Z - 1);
#pragma unroll
    for (int i = 0; i < NC; i++) {
        const float bi = Bi[i] * ib;
        lnphi[i]       = bi * zm1 - L1 - cf * (2.f * t[i] * ia - bi) * L2;
    }
}

// ------------------------------------------------ strict stability (FP32)
// StableSSM trial k's successive substitution (src/MixtureComp.cpp:1525-1564)
// in FP32 on a persistent grid, ending at SSM32_TOL2, at the reference's
// tolerance, or at its iteration cap. The end point (ln Y, Yt) goes to
// sta_verdict, which evaluates it in FP64 before StableNR; trials whose
// Newton step fails from there continue in FP64 (sta_ssm on L_STC_k). The
// trial composition is carried as ln Y (normalised, set up by sta_prep), so
// components whose Y falls below FP32's range keep their values: with
// Y_i = d_i / phi_i / Yt the residual ln(phi_i(Y) Y_i Yt / d_i) is
// ln phi_i(Y) + ln Y_i - ln d_i + ln Yt.
template <int NC>
__device__ void sta_ssm32_body(const FluidConst& F, const PhasedArgs& a, int k)
{
    using F_ = SF<NC>;
    const StateBuf& S    = a.S;
    const int       list = stab_list(L_STA_0 + k, a.sdup != 0);
    const uint32_t  n    = a.L.len(list);
    const float     tol2 = fmaxf(SSM32_TOL2, (float)F.ssmsta_tol2);
    float           lnY[NC], lndi[NC], sA[NC], Bi[NC];
    float           lnYt = 0;
    int             iter = 0;
    bool            first = true;
    int64_t         c     = a.L.take(list, n);
    auto load = [&]() {
        lnYt = __logf((float)S.D(F_::Yt, c));
#pragma unroll
        for (int i = 0; i < NC; i++) {
            lnY[i]  = (float)S.D(F_::lnY + i, c);
            lndi[i] = (float)S.D(F_::lndi + i, c);
            sA[i]   = (float)S.D(F_::sA + i, c);
            Bi[i]   = (float)S.D(F_::Bi + i, c);
        }
        iter  = 0;
        first = true;
    };
    auto finish = [&]() {
#pragma unroll
        for (int i = 0; i < NC; i++) S.D(F_::lnY + i, c) = (double)lnY[i];
        S.D(F_::Yt, c) = (double)__expf(lnYt);
        S.I(IF_IT0, c) += iter;
        S.I(IF_MAXIT, c) = F.ssmsta_maxit > iter ? F.ssmsta_maxit - iter : 0;
        c = a.L.take(list, n);
        if (c >= 0) load();
    };
    if (c >= 0) load();
    while (__any_sync(0xffffffffu, c >= 0)) {
        if (c >= 0) {
            float Y[NC], lnphi[NC];
#pragma unroll
            for (int i = 0; i < NC; i++) Y[i] = __expf(lnY[i]);
            ln_phi32<NC>(F, sA, Bi, Y, lnphi);
            float Se = 0.f;
#pragma unroll
            for (int i = 0; i < NC; i++) {
                const float r = lnphi[i] + lnY[i] - lndi[i] + lnYt;
                Se            = fmaf(r, r, Se);
            }
            bool done;
            if (first) {
                first = false;
                done  = !(Se > tol2);
            } else {
                iter++;
                done = (iter > F.ssmsta_maxit) || !(Se > tol2);
                if (iter > F.ssmsta_maxit) S.I(IF_STATUS, c) |= ST_SSMSTA_CAP;
            }
            if (done) {
                finish();
            } else {
                float Yt = 0.f;
#pragma unroll
                for (int i = 0; i < NC; i++) {
                    lnY[i] = lndi[i] - lnphi[i];
                    Yt += __expf(lnY[i]);
                }
                lnYt = __logf(Yt);
#pragma unroll
                for (int i = 0; i < NC; i++) lnY[i] -= lnYt;
            }
        }
    }
}

}  // namespace ocpf
