// flash_math.cuh -- per-thread FP64 building blocks of the flash: the
// Peng-Robinson cubic with its root choice, dZ derivatives, and small dense
// solves and eigenvalues held in registers.
#pragma once

#include "flash_common.cuh"

namespace ocpf {

// Newton polish of one cubic root, keeping the best iterate
// (NTcubicroot, src/MixtureComp.cpp:5078-5102).
__device__ __forceinline__ double nt_polish(double root, double a, double b, double c)
{
    double e       = root * (root * (root + a) + b) + c;
    double optroot = root;
    double opte    = fabs(e);
    int    iter    = 0;
    while (fabs(e) > 1e-8) {
        const double df = root * (3 * root + 2 * a) + b;
        root            = root - e / df;
        iter++;
        if (iter > 10) break;
        e = root * (root * (root + a) + b) + c;
        if (fabs(e) <= opte) {
            opte    = fabs(e);
            optroot = root;
        }
    }
    return optroot;
}

__device__ __forceinline__ double signD(double d) { return d > 0 ? 1.0 : (d < 0 ? -1.0 : 0.0); }

// The PR cubic Z^3 + a Z^2 + b Z + c = 0 of mixture parameters (aj, bj) with
// Cardano's Q, R and discriminant M = R^2 - Q^3 (CubicRoot,
// src/MixtureComp.cpp:4999-5013).
struct PrCubic {
    double a, b, c, Q, R, Q3, M;
    __device__ __forceinline__ PrCubic(double aj, double bj)
    {
        a  = (D1PD2 - 1) * bj - 1;
        b  = (aj + D1TD2 * bj * bj - D1PD2 * bj * (bj + 1));
        c  = -(aj * bj + D1TD2 * bj * bj * (bj + 1));
        Q  = div_const(a * a - 3 * b, 9, RCP9);
        R  = div_const(2 * a * a * a - 9 * a * b + 27 * c, 54, RCP54);
        Q3 = Q * Q * Q;
        M  = R * R - Q3;
    }
    // Root k (0, 1, 2) of the trigonometric form (M <= 0), polished; theta =
    // acos(R / sqrt(Q^3)), with the reference's truncated pi.
    __device__ __forceinline__ double trig_root(int k, double theta) const
    {
        const double s2  = -2 * sqrt(Q);
        const double a3  = div_const(a, 3, RCP3);
        const double arg = div_const(k == 1 ? theta + 2 * PI_TRUNC : (k == 2 ? theta - 2 * PI_TRUNC : theta), 3, RCP3);
        return nt_polish(s2 * cos(arg) - a3, a, b, c);
    }
    // The single real root (M > 0), polished.
    __device__ __forceinline__ double cardano_root() const
    {
        const double sM = sqrt(M);
        const double t1 = -R + sM;
        const double t2 = R + sM;
        const double S  = signD(t1) * cbrt(fabs(t1));
        const double T  = -signD(t2) * cbrt(fabs(t2));
        return nt_polish(S + T - div_const(a, 3, RCP3), a, b, c);
    }
};

// SolEoS's choice among three real roots: the smallest or the largest by the
// sign of the Gibbs-energy difference (src/MixtureComp.cpp:895-911), in
// pieces (two logarithms and a coefficient) that a warp can form on
// different lanes; pick_root_from combines them in one fixed expression.
//   k = 0: ln((zmin - b) / (zmax - b)),
//   k = 1: ln((zmin + d1 b)(zmax + d2 b) / ((zmin + d2 b)(zmax + d1 b))),
//   k = 2: a / (b (d2 - d1)).
// One division and at most one logarithm, with the operands chosen by k, so
// that lanes forming different pieces run one instruction stream; explicit
// fused multiply-adds keep the value independent of how a kernel contracts.
__device__ __forceinline__ double gibbs_piece(int k, double zmin, double zmax, double aj, double bj)
{
    const double num = k == 0 ? zmin - bj : (k == 1 ? fma(D1, bj, zmin) * fma(D2, bj, zmax) : aj);
    const double den = k == 0 ? zmax - bj : (k == 1 ? fma(D2, bj, zmin) * fma(D1, bj, zmax) : bj * (D2 - D1));
    const double d   = num / den;
    return k <= 1 ? log(d) : d;
}
__device__ __forceinline__ double pick_root_from(double zmin, double zmax, double g1, double g2, double k)
{
    const double dG = (zmax - zmin) + g1 - k * g2;
    return dG > 0 ? zmin : zmax;
}
__device__ __forceinline__ double pick_root(double z0, double z1, double z2, double aj, double bj)
{
    const double zmin = fmin(z0, fmin(z1, z2));
    const double zmax = fmax(z0, fmax(z1, z2));
    return pick_root_from(zmin, zmax, gibbs_piece(0, zmin, zmax, aj, bj), gibbs_piece(1, zmin, zmax, aj, bj),
                          gibbs_piece(2, zmin, zmax, aj, bj));
}

// Z factor of the PR cubic for mixture parameters (aj, bj): Cardano /
// trigonometric roots with the reference's truncated pi, Newton polish, and
// for three roots the Gibbs-energy choice between the smallest and largest
// (SolEoS + CubicRoot, src/MixtureComp.cpp:889-914, 4999-5056).
__device__ __forceinline__ double sol_eos(double aj, double bj)
{
    const PrCubic cu(aj, bj);
    if (cu.M <= 0) {
        const double theta = acos(cu.R / sqrt(cu.Q3));
        const double z0    = cu.trig_root(0, theta);
        const double z1    = cu.trig_root(1, theta);
        const double z2    = cu.trig_root(2, theta);
        return pick_root(z0, z1, z2, aj, bj);
    } else {
        return cu.cardano_root();
    }
}

// sol_eos for a group of lanes that all hold the same (aj, bj): lanes
// `base`, `base`+1 and `base`+2 each polish one of the three trigonometric
// roots and then form one piece of the Gibbs-energy choice; every lane of
// `mask` (which holds them) picks the same root. Same value as sol_eos, bit
// for bit.
__device__ __forceinline__ double sol_eos_group(double aj, double bj, unsigned mask, int base, int rank)
{
    const PrCubic cu(aj, bj);
    if (cu.M <= 0) {
        const double theta = acos(cu.R / sqrt(cu.Q3));
        const double zk    = cu.trig_root(rank < 3 ? rank : 0, theta);
        const double z0    = __shfl_sync(mask, zk, base);
        const double z1    = __shfl_sync(mask, zk, base + 1);
        const double z2    = __shfl_sync(mask, zk, base + 2);
        const double zmin  = fmin(z0, fmin(z1, z2));
        const double zmax  = fmax(z0, fmax(z1, z2));
        const double piece = gibbs_piece(rank < 3 ? rank : 2, zmin, zmax, aj, bj);
        const double g1 = __shfl_sync(mask, piece, base);
        const double g2 = __shfl_sync(mask, piece, base + 1);
        const double k  = __shfl_sync(mask, piece, base + 2);
        return pick_root_from(zmin, zmax, g1, g2, k);
    } else {
        return cu.cardano_root();
    }
}

// dZ for a perturbation (dA, dB) of the mixture parameters: the implicit
// derivative of the PR cubic used by CalFugXSTA, CalFugNAll, CalFugPAll,
// CalVfiVfp_full02 and CalXiPNX_partial (e.g. src/MixtureComp.cpp:1664-1670).
struct DzCoef {
    double num_b, inv_den, bmz;
    __device__ __forceinline__ DzCoef(double aj, double bj, double zj)
    {
        bmz   = bj - zj;
        num_b = (aj + D1TD2 * (3 * bj * bj + 2 * bj)) +
                (D1PD2 * (2 * bj + 1) - 2 * D1TD2 * bj) * zj - (D1PD2 - 1) * zj * zj;
        inv_den = 1.0 / (3 * zj * zj + 2 * ((D1PD2 - 1) * bj - 1) * zj +
                         (aj + D1TD2 * bj * bj - D1PD2 * bj * (bj + 1)));
    }
    __device__ __forceinline__ double operator()(double dA, double dB) const
    {
        return (bmz * dA + num_b * dB) * inv_den;
    }
};

// Solves A X = B (A: N x N, B: N x M, both row-major in registers) by
// Gaussian elimination with partial pivoting, the same pivot rule as LAPACK
// dgetf2 (first largest magnitude). Row swaps are predicated so every index
// stays a compile-time constant. Returns false on an exactly zero pivot;
// A and B are then partially reduced and the caller restores B.
template <int N, int M>
__device__ __forceinline__ bool gauss_solve(double (&A)[N][N], double (&B)[N][M])
{
    bool ok = true;
#pragma unroll
    for (int j = 0; j < N; j++) {
        int    p  = j;
        double mx = fabs(A[j][j]);
#pragma unroll
        for (int i = j + 1; i < N; i++) {
            const double v = fabs(A[i][j]);
            if (v > mx) {
                mx = v;
                p  = i;
            }
        }
#pragma unroll
        for (int i = j + 1; i < N; i++) {
            const bool sw = (p == i);
#pragma unroll
            for (int c = j; c < N; c++) {
                const double t = A[j][c];
                A[j][c]        = sw ? A[i][c] : A[j][c];
                A[i][c]        = sw ? t : A[i][c];
            }
#pragma unroll
            for (int c = 0; c < M; c++) {
                const double t = B[j][c];
                B[j][c]        = sw ? B[i][c] : B[j][c];
                B[i][c]        = sw ? t : B[i][c];
            }
        }
        if (A[j][j] == 0.0) ok = false;
        const double r = 1.0 / A[j][j];
#pragma unroll
        for (int i = j + 1; i < N; i++) {
            const double l = A[i][j] * r;
#pragma unroll
            for (int c = j + 1; c < N; c++) A[i][c] -= l * A[j][c];
#pragma unroll
            for (int c = 0; c < M; c++) B[i][c] -= l * B[j][c];
        }
    }
#pragma unroll
    for (int j = N - 1; j >= 0; j--) {
#pragma unroll
        for (int c = 0; c < M; c++) {
            double s = B[j][c];
#pragma unroll
            for (int k = j + 1; k < N; k++) s -= A[j][k] * B[k][c];
            B[j][c] = s / A[j][j];
        }
    }
    return ok;
}

// gauss_solve for systems too large for registers: the same elimination
// and pivot rule with rolled loops over arrays in local memory, rows
// swapped in place.
template <int N, int M>
__device__ __noinline__ bool gauss_solve_mem(double (&A)[N][N], double (&B)[N][M])
{
    bool ok = true;
#pragma unroll 1
    for (int j = 0; j < N; j++) {
        int    p  = j;
        double mx = fabs(A[j][j]);
        for (int i = j + 1; i < N; i++) {
            const double v = fabs(A[i][j]);
            if (v > mx) {
                mx = v;
                p  = i;
            }
        }
        if (p != j) {
            for (int c = j; c < N; c++) {
                const double t = A[j][c];
                A[j][c]        = A[p][c];
                A[p][c]        = t;
            }
            for (int c = 0; c < M; c++) {
                const double t = B[j][c];
                B[j][c]        = B[p][c];
                B[p][c]        = t;
            }
        }
        if (A[j][j] == 0.0) ok = false;
        const double r = 1.0 / A[j][j];
#pragma unroll 1
        for (int i = j + 1; i < N; i++) {
            const double l = A[i][j] * r;
            for (int c = j + 1; c < N; c++) A[i][c] -= l * A[j][c];
#pragma unroll
            for (int c = 0; c < M; c++) B[i][c] -= l * B[j][c];
        }
    }
#pragma unroll 1
    for (int j = N - 1; j >= 0; j--) {
#pragma unroll
        for (int c = 0; c < M; c++) {
            double s = B[j][c];
            for (int k = j + 1; k < N; k++) s -= A[j][k] * B[k][c];
            B[j][c] = s / A[j][j];
        }
    }
    return ok;
}

// Smallest eigenvalue of a symmetric matrix given in single precision (what
// CalEigenSY / ssyevd returns first, src/DenseMat.cpp:14-26): cyclic Jacobi in
// FP64 on the single-precision entries, rounded to single precision.
template <int N>
__device__ __forceinline__ float min_eig_sym(float (&Af)[N][N])
{
    double a[N][N];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
        for (int j = 0; j < N; j++) a[i][j] = (double)Af[i][j];
    for (int sweep = 0; sweep < 30; sweep++) {
        double off = 0, dia = 0;
#pragma unroll
        for (int p = 0; p < N; p++) {
            dia += a[p][p] * a[p][p];
#pragma unroll
            for (int q = p + 1; q < N; q++) off += a[p][q] * a[p][q];
        }
        if (off <= 1e-36 * dia) break;
#pragma unroll
        for (int p = 0; p < N - 1; p++) {
#pragma unroll
            for (int q = p + 1; q < N; q++) {
                const double apq = a[p][q];
                if (apq != 0.0) {
                    const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
                    const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    const double c = rsqrt(t * t + 1.0);
                    const double s = t * c;
#pragma unroll
                    for (int k = 0; k < N; k++) {
                        const double akp = a[k][p], akq = a[k][q];
                        a[k][p] = c * akp - s * akq;
                        a[k][q] = s * akp + c * akq;
                    }
#pragma unroll
                    for (int k = 0; k < N; k++) {
                        const double apk = a[p][k], aqk = a[q][k];
                        a[p][k] = c * apk - s * aqk;
                        a[q][k] = s * apk + c * aqk;
                    }
                }
            }
        }
    }
    double m = a[0][0];
#pragma unroll
    for (int i = 1; i < N; i++) m = fmin(m, a[i][i]);
    return (float)m;
}

}  // namespace ocpf
