/*
 * flash_port.c -- TEST INFRASTRUCTURE ONLY (the "port" oracle).
 *
 * A plain-C restatement of the reference's compositional Peng-Robinson FIM
 * flash (MixtureComp::FlashFIM and everything it calls), written from the
 * algorithm in src/MixtureComp.cpp, src/AcceleratePVT.cpp and the LAPACK
 * routines it relies on (dsysv 'U' = Bunch-Kaufman; dgesv = partial-pivot LU;
 * ssyevd = symmetric eigenvalues). It is checked against the reference itself
 * (oracle/_ref) on the golden fixtures and serves as the debugging twin of the
 * CUDA kernels and as a CPU baseline. The product never links or calls it.
 *
 * State mirrors one MixtureComp instance (include/MixtureComp.hpp:125-606);
 * every function names the reference lines it follows.
 */
#define _POSIX_C_SOURCE 199309L
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "oracle_api.h"

#define MXC ORC_MAX_NC
#define NPH 3 /* numPhase: oil, gas, water */

/* include/OCPConst.hpp:37-69 */
static const double GAS_CONSTANT = 10.73159;
static const double PI_TRUNC     = 3.141592653;
static const double CONV1        = 5.61458;
static const double CONV5        = 459.67;
static const int    OIL = 0, GAS = 1;

/* include/MixtureComp.hpp:350-351 */
static const double delta1 = 2.41421356237;
static const double delta2 = -0.41421356237;

typedef struct {
    /* fluid (src/MixtureComp.cpp:28-165) */
    int    NC, numCom;
    double Tc[MXC], Pc[MXC], Vc[MXC], MWC[MXC], Acf[MXC], OmegaA[MXC], OmegaB[MXC];
    double Vshift[MXC], Vcvis[MXC], BIC[MXC * MXC], LBCcoef[5];
    double sqrtMWi[MXC], muAux1I[MXC];
    double pvtw[5], std_RhoW;
    /* controls */
    int    rr_maxit, ssmsta_maxit, nrsta_maxit, ssmsp_maxit, nrsp_maxit, use_skip;
    double rr_tol, ssmsta_tol, ssmsta_tol2, ssmsta_eyt, nrsta_tol, ssmsp_tol2, nrsp_tol;
    double Ktol, dYtol;
    /* convergence bookkeeping (include/MixtureComp.hpp:28-92) */
    int    ssmsta_conflag, nrsta_conflag, ssmsp_conflag, nrsp_conflag;
    double ssmsta_realTol, nrsta_realTol, ssmsp_realTol, nrsp_realTol;
    int    it_ssmsta, it_nrsta, it_ssmsp, it_nrsp, it_rr; /* per call */
    int    restarts;                                    /* PhaseSplit restarts, per call */
    double ePEC;
    /* state */
    double P, T, Nh, Nt, vf, vfP;
    double Ni[MXC + 1], zi[MXC];
    double Ai[MXC], Bi[MXC], Aj[2], Bj[2], Zj[2];
    int    NP, lNP, ftype, flagSkip, testPId;
    double nu[2], x[2][MXC], phi[2][MXC], fug[2][MXC], n[2][MXC], ln[2][MXC];
    double Kw[4][MXC], Ks[MXC], lKs[MXC];
    double Y[MXC], Yt, di[MXC], phiSta[MXC], fugSta[MXC], resSTA[MXC];
    double Asta, Bsta, Zsta;
    double fugX[MXC * MXC], JmatSTA[MXC * MXC], Ax[MXC], Zx[MXC];
    double resSP[MXC], JmatSP[MXC * MXC], fugN[2][MXC * MXC], Zn[2][MXC], An[MXC], Bn[MXC];
    double fugP[2][MXC], Zp[2];
    double JmatDer[MXC * MXC], rhsDer[MXC * (MXC + 1)];
    double MW[2], vC[2], xiC[2], rhoC[2], muC[2], muAux[2][5];
    int    phaseLabel[2];
    /* Mixture outputs (include/Mixture.hpp:255-283) */
    int    phaseExist[NPH];
    double S[NPH], vj[NPH], nj[NPH], xij[NPH * (MXC + 1)], rho[NPH], xi[NPH], mu[NPH];
    double vfi[MXC + 1], rhoP[NPH], xiP[NPH], muP[NPH];
    double rhox[NPH * (MXC + 1)], xix[NPH * (MXC + 1)], mux[NPH * (MXC + 1)];
    double dXsdXp[(MXC + 2) * (NPH + NPH * (MXC + 1))];
    double vjp[NPH], vji[NPH][MXC + 1], xixC[2 * MXC], xiPC[2];
    int    pSderExist[NPH], pVnumCom[NPH];
    /* skip cache of the current cell (src/AcceleratePVT.cpp) */
    int    sk_flag;
    double sk_minEig, sk_P, sk_T, sk_z[MXC];
} Mix;

static double sq(double v) { return v * v; }
static double dlt(int i, int j) { return i == j ? 1.0 : 0.0; } /* delta(), :5069-5075 */
static double signD(double d) { return d > 0 ? 1.0 : (d < 0 ? -1.0 : 0.0); }

/* ---- small dense kernels standing in for the BLAS/LAPACK calls -------- */

static double dnorm2(int n, const double* v)
{
    double s = 0;
    for (int i = 0; i < n; i++) s += v[i] * v[i];
    return sqrt(s);
}

/* dsysv(uplo='U') on a symmetric matrix held column-major in A (only A(r,c),
 * r<=c are read): Bunch-Kaufman factorisation U D U^T (LAPACK dsytf2, upper)
 * followed by the triangular solves (dsytrs). If a zero pivot is met (info>0)
 * the right-hand side is left unchanged, as dsysv does. Returns info. */
static int sysv_upper(int N, double* A, double* b)
{
#define AM(r, c) A[(c) * N + (r)]
    int          ipiv[MXC];
    const double alpha = (1.0 + sqrt(17.0)) / 8.0;
    int          info  = 0;
    int          k     = N - 1;
    while (k >= 0) {
        int    kstep = 1, kp, imax = 0;
        double absakk = fabs(AM(k, k)), colmax = 0, rowmax;
        if (k > 0) {
            imax   = 0;
            colmax = fabs(AM(0, k));
            for (int i = 1; i < k; i++)
                if (fabs(AM(i, k)) > colmax) {
                    colmax = fabs(AM(i, k));
                    imax   = i;
                }
        }
        if (fmax(absakk, colmax) == 0.0 || isnan(absakk)) {
            if (info == 0) info = k + 1;
            kp = k;
        } else {
            if (absakk >= alpha * colmax) {
                kp = k;
            } else {
                /* largest off-diagonal magnitude in row/column imax */
                rowmax = fabs(AM(imax, imax + 1));
                for (int j = imax + 2; j <= k; j++) rowmax = fmax(rowmax, fabs(AM(imax, j)));
                for (int r = 0; r < imax; r++) rowmax = fmax(rowmax, fabs(AM(r, imax)));
                if (absakk >= alpha * colmax * (colmax / rowmax)) {
                    kp = k;
                } else if (fabs(AM(imax, imax)) >= alpha * rowmax) {
                    kp = imax;
                } else {
                    kp    = imax;
                    kstep = 2;
                }
            }
            const int kk = k - kstep + 1;
            if (kp != kk) {
                double t;
                for (int i = 0; i < kp; i++) {
                    t          = AM(i, kk);
                    AM(i, kk)  = AM(i, kp);
                    AM(i, kp)  = t;
                }
                for (int j = kp + 1; j < kk; j++) {
                    t          = AM(j, kk);
                    AM(j, kk)  = AM(kp, j);
                    AM(kp, j)  = t;
                }
                t          = AM(kk, kk);
                AM(kk, kk) = AM(kp, kp);
                AM(kp, kp) = t;
                if (kstep == 2) {
                    t            = AM(k - 1, k);
                    AM(k - 1, k) = AM(kp, k);
                    AM(kp, k)    = t;
                }
            }
            if (kstep == 1) {
                const double r1 = 1.0 / AM(k, k);
                for (int j = 0; j < k; j++) {
                    const double tmp = -r1 * AM(j, k);
                    for (int i = 0; i <= j; i++) AM(i, j) += AM(i, k) * tmp;
                }
                for (int i = 0; i < k; i++) AM(i, k) *= r1;
            } else if (k > 1) {
                double       d12 = AM(k - 1, k);
                const double d22 = AM(k - 1, k - 1) / d12;
                const double d11 = AM(k, k) / d12;
                const double t   = 1.0 / (d11 * d22 - 1.0);
                d12              = t / d12;
                for (int j = k - 2; j >= 0; j--) {
                    const double wkm1 = d12 * (d11 * AM(j, k - 1) - AM(j, k));
                    const double wk   = d12 * (d22 * AM(j, k) - AM(j, k - 1));
                    for (int i = j; i >= 0; i--)
                        AM(i, j) = AM(i, j) - AM(i, k) * wk - AM(i, k - 1) * wkm1;
                    AM(j, k)     = wk;
                    AM(j, k - 1) = wkm1;
                }
            }
        }
        if (kstep == 1) {
            ipiv[k] = kp;
        } else {
            ipiv[k]     = -(kp + 1);
            ipiv[k - 1] = -(kp + 1);
        }
        k -= kstep;
    }
    if (info > 0) return info;
    /* solve U D y = b */
    k = N - 1;
    while (k >= 0) {
        if (ipiv[k] >= 0) {
            const int kp = ipiv[k];
            if (kp != k) {
                double t = b[k];
                b[k]     = b[kp];
                b[kp]    = t;
            }
            for (int i = 0; i < k; i++) b[i] -= AM(i, k) * b[k];
            b[k] *= 1.0 / AM(k, k);
            k -= 1;
        } else {
            const int kp = -ipiv[k] - 1;
            if (kp != k - 1) {
                double t  = b[k - 1];
                b[k - 1]  = b[kp];
                b[kp]     = t;
            }
            for (int i = 0; i < k - 1; i++) b[i] -= AM(i, k) * b[k];
            for (int i = 0; i < k - 1; i++) b[i] -= AM(i, k - 1) * b[k - 1];
            const double akm1k = AM(k - 1, k);
            const double akm1  = AM(k - 1, k - 1) / akm1k;
            const double ak    = AM(k, k) / akm1k;
            const double denom = akm1 * ak - 1.0;
            const double bkm1  = b[k - 1] / akm1k;
            const double bk    = b[k] / akm1k;
            b[k - 1]           = (ak * bkm1 - bk) / denom;
            b[k]               = (akm1 * bk - bkm1) / denom;
            k -= 2;
        }
    }
    /* solve U^T x = y */
    k = 0;
    while (k < N) {
        if (ipiv[k] >= 0) {
            for (int i = 0; i < k; i++) b[k] -= AM(i, k) * b[i];
            const int kp = ipiv[k];
            if (kp != k) {
                double t = b[k];
                b[k]     = b[kp];
                b[kp]    = t;
            }
            k += 1;
        } else {
            for (int i = 0; i < k; i++) b[k] -= AM(i, k) * b[i];
            for (int i = 0; i < k; i++) b[k + 1] -= AM(i, k + 1) * b[i];
            const int kp = -ipiv[k] - 1;
            if (kp != k) {
                double t = b[k];
                b[k]     = b[kp];
                b[kp]    = t;
            }
            k += 2;
        }
    }
    return 0;
#undef AM
}

/* dgesv: LU with partial pivoting of the column-major N x N matrix A, then
 * nrhs column-major right-hand sides in B. On a zero pivot B is unchanged. */
static int gesv(int N, int nrhs, double* A, double* B)
{
#define AM(r, c) A[(c) * N + (r)]
    int piv[MXC];
    int info = 0;
    for (int j = 0; j < N; j++) {
        int    p = j;
        double m = fabs(AM(j, j));
        for (int i = j + 1; i < N; i++)
            if (fabs(AM(i, j)) > m) {
                m = fabs(AM(i, j));
                p = i;
            }
        piv[j] = p;
        if (AM(p, j) != 0.0) {
            if (p != j)
                for (int c = 0; c < N; c++) {
                    double t = AM(j, c);
                    AM(j, c) = AM(p, c);
                    AM(p, c) = t;
                }
            const double r = 1.0 / AM(j, j);
            for (int i = j + 1; i < N; i++) AM(i, j) *= r;
        } else if (info == 0) {
            info = j + 1;
        }
        for (int c = j + 1; c < N; c++)
            for (int i = j + 1; i < N; i++) AM(i, c) -= AM(i, j) * AM(j, c);
    }
    if (info > 0) return info;
    for (int r = 0; r < nrhs; r++) {
        double* b = B + r * N;
        for (int j = 0; j < N; j++)
            if (piv[j] != j) {
                double t    = b[j];
                b[j]        = b[piv[j]];
                b[piv[j]]   = t;
            }
        for (int j = 0; j < N; j++)
            for (int i = j + 1; i < N; i++) b[i] -= AM(i, j) * b[j];
        for (int j = N - 1; j >= 0; j--) {
            b[j] /= AM(j, j);
            for (int i = 0; i < j; i++) b[i] -= AM(i, j) * b[j];
        }
    }
    return 0;
#undef AM
}

/* Smallest eigenvalue of a symmetric single-precision matrix (what
 * CalEigenSY/ssyevd returns first, src/DenseMat.cpp:14-26): cyclic Jacobi in
 * double on the single-precision entries, rounded to single. */
static float min_eig_sym(int N, const float* Af)
{
    double a[MXC * MXC];
    for (int i = 0; i < N * N; i++) a[i] = (double)Af[i];
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0, dia = 0;
        for (int p = 0; p < N; p++) {
            dia += a[p * N + p] * a[p * N + p];
            for (int q = p + 1; q < N; q++) off += a[p * N + q] * a[p * N + q];
        }
        if (off <= 1e-36 * dia || off == 0.0) break;
        for (int p = 0; p < N - 1; p++)
            for (int q = p + 1; q < N; q++) {
                const double apq = a[p * N + q];
                if (apq == 0.0) continue;
                const double app = a[p * N + p], aqq = a[q * N + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) /
                                 (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < N; k++) {
                    const double akp = a[k * N + p], akq = a[k * N + q];
                    a[k * N + p] = c * akp - s * akq;
                    a[k * N + q] = s * akp + c * akq;
                }
                for (int k = 0; k < N; k++) {
                    const double apk = a[p * N + k], aqk = a[q * N + k];
                    a[p * N + k] = c * apk - s * aqk;
                    a[q * N + k] = s * apk + c * aqk;
                }
            }
    }
    double m = a[0];
    for (int i = 1; i < N; i++) m = fmin(m, a[i * N + i]);
    return (float)m;
}

/* ---- EoS ------------------------------------------------------------- */

/* NTcubicroot, src/MixtureComp.cpp:5078-5102 */
static double nt_cubic_root(double root, double a, double b, double c)
{
    double e       = root * (root * (root + a) + b) + c;
    double optroot = root, opte = fabs(e);
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

/* CubicRoot with NT polish, src/MixtureComp.cpp:4999-5056; Z[] ascending */
static int cubic_root(double a, double b, double c, double Z[3])
{
    const double Q  = (a * a - 3 * b) / 9;
    const double R  = (2 * a * a * a - 9 * a * b + 27 * c) / 54;
    const double Q3 = Q * Q * Q;
    const double M  = R * R - Q3;
    if (M <= 0) {
        const double theta = acos(R / sqrt(Q3));
        Z[0] = -2 * sqrt(Q) * cos(theta / 3) - a / 3;
        Z[1] = -2 * sqrt(Q) * cos((theta + 2 * PI_TRUNC) / 3) - a / 3;
        Z[2] = -2 * sqrt(Q) * cos((theta - 2 * PI_TRUNC) / 3) - a / 3;
        for (int i = 0; i < 3; i++) Z[i] = nt_cubic_root(Z[i], a, b, c);
        /* sort ascending */
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2 - i; j++)
                if (Z[j + 1] < Z[j]) {
                    double t = Z[j];
                    Z[j]     = Z[j + 1];
                    Z[j + 1] = t;
                }
        return 3;
    } else {
        const double t1 = -R + sqrt(M);
        const double t2 = R + sqrt(M);
        const double S  = signD(t1) * pow(fabs(t1), 1.0 / 3);
        const double T  = -signD(t2) * pow(fabs(t2), 1.0 / 3);
        Z[0]            = nt_cubic_root(S + T - a / 3, a, b, c);
        return 1;
    }
}

/* SolEoS, src/MixtureComp.cpp:889-914 */
static double sol_eos(double aj, double bj)
{
    const double a = (delta1 + delta2 - 1) * bj - 1;
    const double b = (aj + delta1 * delta2 * bj * bj - (delta1 + delta2) * bj * (bj + 1));
    const double c = -(aj * bj + delta1 * delta2 * bj * bj * (bj + 1));
    double       Z[3];
    if (cubic_root(a, b, c, Z) == 1) return Z[0];
    const double z1 = Z[0], z2 = Z[2];
    const double dG = (z2 - z1) + log((z1 - bj) / (z2 - bj)) -
                      aj / (bj * (delta2 - delta1)) *
                          log((z1 + delta1 * bj) * (z2 + delta2 * bj) /
                              ((z1 + delta2 * bj) * (z2 + delta1 * bj)));
    return dG > 0 ? z1 : z2;
}

/* CalAiBi, src/MixtureComp.cpp:916-937 */
static void cal_ai_bi(Mix* m)
{
    for (int i = 0; i < m->NC; i++) {
        const double acf = m->Acf[i];
        double       mwi;
        if (acf <= 0.49)
            mwi = 0.37464 + 1.54226 * acf - 0.26992 * sq(acf);
        else
            mwi = 0.379642 + 1.48503 * acf - 0.164423 * sq(acf) + 0.016667 * pow(acf, 3);
        const double Pri = m->P / m->Pc[i];
        const double Tri = m->T / m->Tc[i];
        m->Ai[i] = m->OmegaA[i] * Pri / sq(Tri) * sq(1 + mwi * (1 - sqrt(Tri)));
        m->Bi[i] = m->OmegaB[i] * Pri / Tri;
    }
}

/* (1 - k_ik) sqrt(A_i A_k) */
static double aik(const Mix* m, int i, int k)
{
    return (1 - m->BIC[i * m->NC + k]) * sqrt(m->Ai[i] * m->Ai[k]);
}

/* CalAjBj, src/MixtureComp.cpp:939-969 */
static void cal_aj_bj(const Mix* m, double* AjT, double* BjT, const double* xj)
{
    double a = 0, b = 0;
    for (int i1 = 0; i1 < m->NC; i1++) {
        b += m->Bi[i1] * xj[i1];
        a += xj[i1] * xj[i1] * m->Ai[i1] * (1 - m->BIC[i1 * m->NC + i1]);
        for (int i2 = 0; i2 < i1; i2++)
            a += 2 * xj[i1] * xj[i2] * sqrt(m->Ai[i1] * m->Ai[i2]) *
                 (1 - m->BIC[i1 * m->NC + i2]);
    }
    *AjT = a;
    *BjT = b;
}

/* CalFugPhi (all three overloads), src/MixtureComp.cpp:993-1101. phiT may be
 * NULL (fugacity only). Records Asta, Bsta, Zsta. */
static void cal_fug_phi(Mix* m, double* phiT, double* fugT, const double* xj)
{
    double aj, bj;
    cal_aj_bj(m, &aj, &bj, xj);
    const double zj = sol_eos(aj, bj);
    for (int i = 0; i < m->NC; i++) {
        double tmp = 0;
        for (int k = 0; k < m->NC; k++) tmp += 2 * aik(m, i, k) * xj[k];
        const double ph = exp(m->Bi[i] / bj * (zj - 1) - log(zj - bj) -
                              aj / (delta1 - delta2) / bj * (tmp / aj - m->Bi[i] / bj) *
                                  log((zj + delta1 * bj) / (zj + delta2 * bj)));
        if (phiT) phiT[i] = ph;
        fugT[i] = ph * xj[i] * m->P;
    }
    m->Asta = aj;
    m->Bsta = bj;
    m->Zsta = zj;
}

/* CalFugPhiAll, src/MixtureComp.cpp:1103-1145 */
static void cal_fug_phi_all(Mix* m)
{
    for (int j = 0; j < m->NP; j++) {
        cal_aj_bj(m, &m->Aj[j], &m->Bj[j], m->x[j]);
        m->Zj[j] = sol_eos(m->Aj[j], m->Bj[j]);
        const double aj = m->Aj[j], bj = m->Bj[j], zj = m->Zj[j];
        for (int i = 0; i < m->NC; i++) {
            double tmp = 0;
            for (int k = 0; k < m->NC; k++) tmp += 2 * aik(m, i, k) * m->x[j][k];
            m->phi[j][i] = exp(m->Bi[i] / bj * (zj - 1) - log(zj - bj) -
                               aj / (delta1 - delta2) / bj * (tmp / aj - m->Bi[i] / bj) *
                                   log((zj + delta1 * bj) / (zj + delta2 * bj)));
            m->fug[j][i] = m->phi[j][i] * m->x[j][i] * m->P;
        }
    }
}

/* dZ/dq for a perturbation (dA, dB) of the mixture parameters; the formula
 * shared by CalFugXSTA, CalFugNAll, CalFugPAll, CalVfiVfp_full02 and
 * CalXiPNX_partial (e.g. src/MixtureComp.cpp:1664-1670). */
static double dz_of(double aj, double bj, double zj, double dA, double dB)
{
    return ((bj - zj) * dA +
            ((aj + delta1 * delta2 * (3 * bj * bj + 2 * bj)) +
             ((delta1 + delta2) * (2 * bj + 1) - 2 * delta1 * delta2 * bj) * zj -
             (delta1 + delta2 - 1) * zj * zj) *
                dB) /
           (3 * zj * zj + 2 * ((delta1 + delta2 - 1) * bj - 1) * zj +
            (aj + delta1 * delta2 * bj * bj - (delta1 + delta2) * bj * (bj + 1)));
}

/* CalKwilson, src/MixtureComp.cpp:1269-1277 */
static void cal_kwilson(Mix* m)
{
    for (int i = 0; i < m->NC; i++) {
        m->Kw[0][i] = (m->Pc[i] / m->P) * exp(5.373 * (1 + m->Acf[i]) * (1 - m->Tc[i] / m->T));
        m->Kw[1][i] = 1 / m->Kw[0][i];
        m->Kw[2][i] = pow(m->Kw[0][i], 1.0 / 3);
        m->Kw[3][i] = pow(m->Kw[1][i], 1.0 / 3);
    }
}

/* ---- stability ------------------------------------------------------- */

/* CalFugXSTA, src/MixtureComp.cpp:1638-1714 */
static void cal_fugx_sta(Mix* m)
{
    const int    NC = m->NC;
    const double aj = m->Asta, bj = m->Bsta, zj = m->Zsta, P = m->P;
    const double m1Mm2 = delta1 - delta2;
    for (int i = 0; i < NC; i++) {
        double tmp = 0;
        for (int k = 0; k < NC; k++) tmp += m->Y[k] * aik(m, i, k);
        m->Ax[i] = 2 * tmp;
        m->Zx[i] = dz_of(aj, bj, zj, m->Ax[i], m->Bi[i]);
    }
    const double G = (zj + delta1 * bj) / (zj + delta2 * bj);
    for (int i = 0; i < NC; i++) {
        const double C = m->Y[i] * P / (zj - bj);
        const double E = -aj / (m1Mm2 * bj) * (m->Ax[i] / aj - m->Bi[i] / bj);
        for (int k = 0; k < NC; k++) {
            const double a_ik = aik(m, i, k);
            const double Cxk  = ((zj - bj) * dlt(i, k) - m->Y[i] * (m->Zx[k] - m->Bi[k])) * P /
                               ((zj - bj) * (zj - bj));
            const double Dxk = m->Bi[i] / bj * (m->Zx[k] - m->Bi[k] * (zj - 1) / bj);
            double       Exk = (2 * (aj / bj * m->Bi[k] * m->Bi[i] + bj * a_ik) -
                          m->Ax[i] * m->Bi[k] - m->Ax[k] * m->Bi[i]) /
                         (bj * bj);
            Exk /= -m1Mm2;
            const double Gxk = m1Mm2 / (zj + delta2 * bj) / (zj + delta2 * bj) *
                               (zj * m->Bi[k] - m->Zx[k] * bj);
            m->fugX[i * NC + k] = 1 / C * Cxk + Dxk + Exk * log(G) + E / G * Gxk;
        }
    }
}

/* AssembleJmatSTA, src/MixtureComp.cpp:1716-1741 (row-major, as the reference
 * stores it; dsysv 'U' then reads its lower triangle as the upper one of the
 * column-major matrix). */
static void assemble_jmat_sta(Mix* m)
{
    const int NC = m->NC;
    for (int i = 0; i < NC; i++) {
        double tmp = 0;
        for (int k = 0; k < NC; k++) tmp += m->Y[k] * m->fugX[i * NC + k];
        for (int j = 0; j < NC; j++) m->JmatSTA[i * NC + j] = (m->fugX[i * NC + j] - tmp + 1) / m->Yt;
    }
}

/* StableNR, src/MixtureComp.cpp:1590-1636 */
static int stable_nr(Mix* m, int Id)
{
    const int NC = m->NC;
    for (int i = 0; i < NC; i++) m->resSTA[i] = log(m->fug[Id][i] / (m->fugSta[i] * m->Yt));
    double Se   = dnorm2(NC, m->resSTA);
    int    iter = 0;
    while (Se > m->nrsta_tol) {
        cal_fugx_sta(m);
        assemble_jmat_sta(m);
        sysv_upper(NC, m->JmatSTA, m->resSTA);
        for (int i = 0; i < NC; i++) m->Y[i] *= m->Yt;
        for (int i = 0; i < NC; i++) m->Y[i] += 1.0 * m->resSTA[i];
        m->Yt = 0;
        for (int i = 0; i < NC; i++) m->Yt += m->Y[i];
        const double r = 1 / m->Yt;
        for (int i = 0; i < NC; i++) m->Y[i] *= r;
        cal_fug_phi(m, NULL, m->fugSta, m->Y);
        for (int i = 0; i < NC; i++) m->resSTA[i] = log(m->fug[Id][i] / (m->fugSta[i] * m->Yt));
        Se = dnorm2(NC, m->resSTA);
        iter++;
        if (iter > m->nrsta_maxit) {
            m->it_nrsta += iter;
            m->nrsta_conflag = 0;
            m->nrsta_realTol = Se;
            return 0;
        }
    }
    m->it_nrsta += iter;
    m->nrsta_conflag = 1;
    m->nrsta_realTol = Se;
    return 1;
}

/* StableSSM (strict), src/MixtureComp.cpp:1492-1588 */
static int stable_ssm(Mix* m, int Id)
{
    const int     NC    = m->NC;
    const double* xj    = m->x[Id];
    cal_fug_phi(m, m->phi[Id], m->fug[Id], xj);
    const double* fugId = m->fug[Id];
    for (int i = 0; i < NC; i++) m->di[i] = m->phi[Id][i] * xj[i];
    double Se = 0;
    for (int k = 0; k < 4; k++) {
        m->Yt = 0;
        for (int i = 0; i < NC; i++) {
            m->Y[i] = xj[i] / m->Kw[k][i];
            m->Yt += m->Y[i];
        }
        double r = 1 / m->Yt;
        for (int i = 0; i < NC; i++) m->Y[i] *= r;
        cal_fug_phi(m, m->phiSta, m->fugSta, m->Y);
        Se = 0;
        for (int i = 0; i < NC; i++) Se += sq(log(m->fugSta[i] / fugId[i] * m->Yt));
        int iter = 0;
        while (Se > m->ssmsta_tol2) {
            m->Yt = 0;
            for (int i = 0; i < NC; i++) {
                m->Y[i] = m->di[i] / m->phiSta[i];
                m->Yt += m->Y[i];
            }
            r = 1 / m->Yt;
            for (int i = 0; i < NC; i++) m->Y[i] *= r;
            cal_fug_phi(m, m->phiSta, m->fugSta, m->Y);
            Se = 0;
            for (int i = 0; i < NC; i++) Se += sq(log(m->fugSta[i] / fugId[i] * m->Yt));
            iter++;
            if (iter > m->ssmsta_maxit) break;
        }
        m->it_ssmsta += iter;
        const int flag = stable_nr(m, Id);
        if (flag && m->Yt > 1 + m->ssmsta_eyt) {
            m->ssmsta_conflag = 1;
            m->ssmsta_realTol = sqrt(Se);
            return 0;
        }
    }
    m->ssmsta_realTol = sqrt(Se);
    return 1;
}

/* StableSSM01 (relaxed), src/MixtureComp.cpp:1392-1490 */
static int stable_ssm01(Mix* m, int Id)
{
    const int     NC = m->NC;
    const double* xj = m->x[Id];
    cal_fug_phi(m, m->phi[Id], m->fug[Id], xj);
    const double* fugId = m->fug[Id];
    double        Se = 0, Sk = 0;
    double*       ks = m->Ks;
    for (int k = 0; k < 2; k++) {
        memcpy(ks, m->Kw[k], sizeof(double) * NC);
        int iter = 0, flag = 0;
        while (1) {
            m->Yt = 0;
            for (int i = 0; i < NC; i++) {
                m->Y[i] = xj[i] * ks[i];
                m->Yt += m->Y[i];
            }
            const double r = 1 / m->Yt;
            for (int i = 0; i < NC; i++) m->Y[i] *= r;
            if (iter > 0) {
                double dY = 0;
                for (int i = 0; i < NC; i++) dY += sq(m->Y[i] - m->di[i]);
                if (dY < m->dYtol) {
                    flag = 1;
                    break;
                }
            }
            cal_fug_phi(m, NULL, m->fugSta, m->Y);
            Se = 0;
            Sk = 0;
            for (int i = 0; i < NC; i++) {
                m->di[i] = fugId[i] / (m->fugSta[i] * m->Yt);
                ks[i] *= m->di[i];
                Se += sq(m->di[i] - 1);
                Sk += sq(log(ks[i]));
            }
            iter++;
            if (Se < m->ssmsta_tol2) {
                flag = 1;
                break;
            }
            if (Sk < m->Ktol) {
                flag = 1;
                break;
            }
            if (iter > m->ssmsta_maxit) break;
            memcpy(m->di, m->Y, sizeof(double) * NC);
        }
        m->it_ssmsta += iter;
        if (flag && m->Yt > 1 - 0.1 && Sk > 1) m->flagSkip = 0;
        if (flag && m->Yt > 1 + m->ssmsta_eyt) {
            m->ssmsta_conflag = 1;
            m->ssmsta_realTol = sqrt(Se);
            return 0;
        }
    }
    m->ssmsta_realTol = sqrt(Se);
    return 1;
}

/* CalMW, src/MixtureComp.cpp:1147-1156 */
static void cal_mw(Mix* m)
{
    for (int j = 0; j < m->NP; j++) {
        m->MW[j] = 0;
        for (int i = 0; i < m->NC; i++) m->MW[j] += m->x[j][i] * m->MWC[i];
    }
}

/* PhaseStable, src/MixtureComp.cpp:1355-1390 */
static int phase_stable(Mix* m)
{
    if (m->NP == 1) {
        m->testPId = 0;
    } else {
        cal_mw(m);
        m->testPId = m->MW[1] > m->MW[0] ? 1 : 0; /* FindMWmax */
    }
    m->ssmsta_conflag = 0;
    m->nrsta_conflag  = 0;
    int flag;
    int tmpNP = m->NP;
    if (m->lNP == 0) {
        flag = stable_ssm(m, m->testPId);
    } else {
        flag = stable_ssm01(m, m->testPId);
        if (!flag) tmpNP++;
        if (tmpNP != m->lNP) {
            flag        = stable_ssm(m, m->testPId);
            m->flagSkip = 0;
        }
    }
    return flag;
}

/* ---- phase split ----------------------------------------------------- */

/* RachfordRice2, src/MixtureComp.cpp:1907-1959 */
static void rachford_rice2(Mix* m)
{
    const int     NC = m->NC;
    const double* K  = m->Ks;
    double        Kmin = K[0], Kmax = K[0];
    for (int i = 1; i < NC; i++) {
        if (K[i] < Kmin) Kmin = K[i];
        if (K[i] > Kmax) Kmax = K[i];
    }
    const double numin = 1 / (1 - Kmax);
    const double numax = 1 / (1 - Kmin);
    m->nu[0]           = 0.5 * (numin + numax);
    int iter           = 0;
    while (1) {
        double rj = 0, J = 0;
        for (int i = 0; i < NC; i++) {
            const double tmp = 1 + m->nu[0] * (K[i] - 1);
            rj += m->zi[i] * (K[i] - 1) / tmp;
            J -= m->zi[i] * (K[i] - 1) * (K[i] - 1) / (tmp * tmp);
        }
        if (fabs(rj) < m->rr_tol || iter > m->rr_maxit) break;
        const double dnuj  = -rj / J;
        const double tmpnu = m->nu[0] + dnuj;
        if (tmpnu < numax && tmpnu > numin) {
            m->nu[0] = tmpnu;
        } else if (dnuj > 0) {
            m->nu[0] = (m->nu[0] + numax) / 2;
        } else {
            m->nu[0] = (m->nu[0] + numin) / 2;
        }
        iter++;
    }
    m->it_rr += iter;
    m->nu[1] = 1 - m->nu[0];
}

/* UpdateXRR, src/MixtureComp.cpp:2030-2043 (NP = 2) */
static void update_x_rr(Mix* m)
{
    for (int i = 0; i < m->NC; i++) {
        const double tmp = 1 + m->nu[0] * (m->Ks[i] - 1);
        m->x[1][i]       = m->zi[i] / tmp;
        m->x[0][i]       = m->Ks[i] * m->x[1][i];
    }
}

/* SplitSSM2, src/MixtureComp.cpp:1847-1903 */
static void split_ssm2(Mix* m, int restart)
{
    const int NC     = m->NC;
    m->ssmsp_conflag = 1;
    double Se        = 1;
    double Stol      = m->ssmsp_tol2;
    int    maxIt     = m->ssmsp_maxit;
    if (!restart) {
        if (m->lNP == 2)
            memcpy(m->Ks, m->lKs, sizeof(double) * NC);
        else
            memcpy(m->Ks, m->Kw[0], sizeof(double) * NC);
    } else {
        Stol *= 1e-1;
        maxIt *= 2;
    }
    if (m->Yt < 1.1) {
        Stol *= 1e-1;
        maxIt *= 2;
    }
    int iter = 0;
    while (Se > Stol) {
        rachford_rice2(m);
        update_x_rr(m);
        cal_fug_phi_all(m);
        Se = 0;
        for (int i = 0; i < NC; i++) {
            Se += sq(m->fug[1][i] / m->fug[0][i] - 1);
            m->Ks[i] = m->phi[1][i] / m->phi[0][i];
        }
        iter++;
        if (iter > maxIt) {
            m->ssmsp_conflag = 0;
            break;
        }
    }
    m->ssmsp_realTol = sqrt(Se);
    m->it_ssmsp += iter;
}

/* CalFugNAll, src/MixtureComp.cpp:2168-2250 (Znflag = true) */
static void cal_fugn_all(Mix* m)
{
    const int NC = m->NC;
    for (int j = 0; j < m->NP; j++) {
        double*       fugn = m->fugN[j];
        const double  aj = m->Aj[j], bj = m->Bj[j], zj = m->Zj[j], nuj = m->nu[j];
        const double* xj = m->x[j];
        double*       Znj = m->Zn[j];
        for (int i = 0; i < NC; i++) {
            double tmp = 0;
            for (int k = 0; k < NC; k++) tmp += aik(m, i, k) * xj[k];
            m->An[i] = 2 / nuj * (tmp - aj);
            m->Bn[i] = 1 / nuj * (m->Bi[i] - bj);
            Znj[i]   = dz_of(aj, bj, zj, m->An[i], m->Bn[i]);
        }
        const double G = (zj + delta1 * bj) / (zj + delta2 * bj);
        for (int i = 0; i < NC; i++) {
            const double C = xj[i] * m->P / (zj - bj);
            double       tmp = 0;
            for (int k = 0; k < NC; k++) tmp += aik(m, i, k) * xj[k];
            const double E = -aj / ((delta1 - delta2) * bj) * (2 * tmp / aj - m->Bi[i] / bj);
            for (int k = 0; k <= i; k++) {
                const double a_ik = aik(m, i, k);
                const double Cnk  = m->P / (zj - bj) / (zj - bj) *
                                   ((zj - bj) / nuj * (dlt(i, k) - xj[i]) - xj[i] * (Znj[k] - m->Bn[k]));
                const double Dnk = m->Bi[i] / bj * (Znj[k] - (m->Bi[k] - bj) * (zj - 1) / (nuj * bj));
                const double Gnk = (delta1 - delta2) / ((zj + delta2 * bj) * (zj + delta2 * bj)) *
                                   (m->Bn[k] * zj - Znj[k] * bj);
                double Enk = -1 / (delta1 - delta2) / (bj * bj) *
                             (2 * (bj * a_ik / nuj + m->Bn[k] * (m->Bi[i] * aj / bj - tmp)) -
                              m->An[k] * m->Bi[i] - aj * m->Bi[i] / nuj);
                Enk -= E / nuj;
                fugn[i * NC + k] = 1 / C * Cnk + Dnk + Enk * log(G) + E / G * Gnk;
                fugn[k * NC + i] = fugn[i * NC + k];
            }
        }
    }
}

/* SplitNR, src/MixtureComp.cpp:2057-2156, with CalResSP (:2158-2166),
 * AssembleJmatSP (:2265-2299) and CalStepNRsp (:2301-2319) for NP = 2 */
static void split_nr(Mix* m)
{
    const int NC     = m->NC;
    m->nrsp_conflag  = 0;
    for (int j = 0; j < 2; j++)
        for (int i = 0; i < NC; i++) m->n[j][i] = m->nu[j] * m->x[j][i];
    for (int i = 0; i < NC; i++) m->resSP[i] = log(m->fug[1][i] / m->fug[0][i]);
    double       eNR  = dnorm2(NC, m->resSP);
    const double eNR0 = eNR;
    int          iter = 0;
    while (eNR > m->nrsp_tol) {
        memcpy(m->ln, m->n, sizeof(m->n));
        cal_fugn_all(m);
        for (int i = 0; i < NC; i++)
            for (int k = 0; k < NC; k++)
                m->JmatSP[i * NC + k] = m->fugN[0][i * NC + k] + m->fugN[1][i * NC + k];
        sysv_upper(NC, m->JmatSP, m->resSP);
        double alpha = 1;
        for (int i = 0; i < NC; i++) {
            const double tmp = m->n[0][i] + alpha * m->resSP[i];
            if (tmp < 0) alpha *= 0.9 * fabs(m->n[0][i] / m->resSP[i]);
        }
        memcpy(m->n[1], m->zi, sizeof(double) * NC);
        for (int i = 0; i < NC; i++) m->n[0][i] += alpha * m->resSP[i];
        for (int i = 0; i < NC; i++) m->n[1][i] += -1 * m->n[0][i];
        m->nu[0] = 0;
        for (int i = 0; i < NC; i++) m->nu[0] += m->n[0][i];
        for (int i = 0; i < NC; i++) m->x[0][i] = fabs(m->n[0][i] / m->nu[0]);
        m->nu[1] = 0;
        for (int i = 0; i < NC; i++) m->nu[1] += m->n[1][i];
        for (int i = 0; i < NC; i++) m->x[1][i] = fabs(m->n[1][i] / m->nu[1]);
        cal_fug_phi_all(m);
        for (int i = 0; i < NC; i++) m->resSP[i] = log(m->fug[1][i] / m->fug[0][i]);
        eNR = dnorm2(NC, m->resSP);
        iter++;
        if (eNR > eNR0 || iter > m->nrsp_maxit) break;
        double en = 0;
        for (int j = 0; j < 2; j++) {
            double d[MXC];
            for (int i = 0; i < NC; i++) d[i] = m->ln[j][i] + -1 * m->n[j][i];
            en += dnorm2(NC, d);
        }
        if (en / (2 * NC) < 1e-8) {
            m->nrsp_conflag = 1;
            break;
        }
    }
    m->nrsp_realTol = eNR;
    if (eNR < m->nrsp_tol) m->nrsp_conflag = 1;
    m->it_nrsp += iter;
}

/* CheckSplit, src/MixtureComp.cpp:1784-1836. The Gibbs-energy evaluation
 * there only feeds a diagnostic print and is omitted. */
static int check_split(Mix* m)
{
    if (m->NP == 2) {
        double       eX    = 0;
        const double nuMax = (m->nu[0] < m->nu[1]) ? m->nu[1] : m->nu[0];
        for (int i = 0; i < m->NC; i++) eX += (m->x[0][i] - m->x[1][i]) * (m->x[0][i] - m->x[1][i]);
        if (nuMax < 1 && m->nrsp_conflag && isfinite(eX)) {
            /* accept */
        } else if (!isfinite(eX) || 1 - nuMax < 1e-3) {
            m->NP    = 1;
            memcpy(m->x[0], m->zi, sizeof(double) * m->NC);
            m->nu[0] = 1;
            cal_aj_bj(m, &m->Aj[0], &m->Bj[0], m->x[0]);
            m->Zj[0]          = sol_eos(m->Aj[0], m->Bj[0]);
            m->ssmsta_conflag = 0;
            m->nrsta_conflag  = 0;
            return 0;
        }
    }
    return 1;
}

/* PhaseSplit, src/MixtureComp.cpp:1743-1782 (restart loop bounded at 200,
 * as the CUDA library bounds it; the reference's is unbounded) */
static void phase_split(Mix* m)
{
    m->ssmsp_conflag = 0;
    m->nrsp_conflag  = 0;
    split_ssm2(m, 0);
    split_nr(m);
    int guard = 0;
    while (!m->nrsp_conflag && guard++ < 200) {
        split_ssm2(m, 1);
        split_nr(m);
        m->restarts++;
        if (!check_split(m)) break;
        if (m->ssmsp_conflag) break;
    }
    check_split(m);
}

/* PhaseEquilibrium, src/MixtureComp.cpp:1279-1353 (NPmax = 2) */
static void phase_equilibrium(Mix* m)
{
    switch (m->ftype) {
        case 0:
            m->flagSkip = 1;
            m->NP       = 1;
            m->nu[0]    = 1;
            memcpy(m->x[0], m->zi, sizeof(double) * m->NC);
            cal_ai_bi(m);
            cal_aj_bj(m, &m->Aj[0], &m->Bj[0], m->x[0]);
            m->Zj[0] = sol_eos(m->Aj[0], m->Bj[0]);
            cal_kwilson(m);
            while (!phase_stable(m)) {
                m->NP++;
                phase_split(m);
                if (m->NP == 2 || m->NP == 1) break;
            }
            if (m->NP > 1) m->flagSkip = 0;
            if (m->NP == 1) {
                m->ePEC = m->nrsta_conflag ? m->nrsta_realTol
                          : m->ssmsta_conflag ? m->ssmsta_realTol : 1e8;
            } else {
                m->ePEC = m->nrsp_conflag ? m->nrsp_realTol
                          : m->ssmsp_conflag ? m->ssmsp_realTol : 1e8;
            }
            break;
        case 1:
            m->flagSkip = 1;
            m->NP       = 1;
            m->nu[0]    = 1;
            memcpy(m->x[0], m->zi, sizeof(double) * m->NC);
            cal_ai_bi(m);
            cal_aj_bj(m, &m->Aj[0], &m->Bj[0], m->x[0]);
            m->Zj[0] = sol_eos(m->Aj[0], m->Bj[0]);
            m->ePEC  = 0.0;
            break;
        default: /* 2 */
            m->flagSkip = 0;
            m->NP       = 2;
            m->Yt       = 1.01;
            cal_ai_bi(m);
            cal_kwilson(m);
            phase_split(m);
            m->ePEC = m->nrsp_conflag ? m->nrsp_realTol
                      : m->ssmsp_conflag ? m->ssmsp_realTol : 1e8;
            break;
    }
}

/* ---- properties ------------------------------------------------------ */

/* CalVfXiRho, src/MixtureComp.cpp:1158-1176 */
static void cal_vf_xi_rho(Mix* m)
{
    m->vf = 0;
    for (int j = 0; j < m->NP; j++) {
        double tmp = m->Zj[j] * GAS_CONSTANT * m->T / m->P;
        for (int i = 0; i < m->NC; i++) tmp -= m->x[j][i] * m->Vshift[i];
        m->vC[j] = tmp * m->nu[j];
        m->vf += m->vC[j];
        m->xiC[j]  = 1 / tmp;
        m->rhoC[j] = m->MW[j] * m->xiC[j];
    }
}

/* CalViscoLBC, src/MixtureComp.cpp:2402-2446 */
static void cal_visco_lbc(Mix* m)
{
    const double* L = m->LBCcoef;
    for (int j = 0; j < m->NP; j++) {
        const double* xj  = m->x[j];
        double*       muA = m->muAux[j];
        double        xijT = 0, xijP = 0, xijV = 0;
        for (int k = 0; k < 5; k++) muA[k] = 0;
        for (int i = 0; i < m->NC; i++) {
            double tmp = 5.4402 * pow(m->Tc[i], 1.0 / 6) / sqrt(m->MW[j]) / pow(m->Pc[i], 2.0 / 3);
            const double Tri = m->T / m->Tc[i];
            if (Tri <= 1.5)
                tmp = 34 * 1e-5 * pow(Tri, 0.94) / tmp;
            else
                tmp = 17.78 * 1e-5 * pow((4.58 * Tri - 1.67), 0.625) / tmp;
            muA[0] += xj[i] * sqrt(m->MWC[i]) * tmp;
            muA[1] += xj[i] * sqrt(m->MWC[i]);
            xijT += xj[i] * m->Tc[i];
            xijP += xj[i] * m->Pc[i];
            xijV += xj[i] * m->Vcvis[i];
        }
        muA[2] = 5.4402 * pow(xijT, 1.0 / 6) / sqrt(m->MW[j]) / pow(xijP, 2.0 / 3);
        muA[3] = m->xiC[j] * xijV;
        muA[4] = muA[3] * (muA[3] * (muA[3] * (L[4] * muA[3] + L[3]) + L[2]) + L[1]) + L[0];
        m->muC[j] = muA[0] / muA[1] + 1e-4 * (pow(muA[4], 4) - 1) / muA[2];
    }
}

/* IdentifyPhase, src/MixtureComp.cpp:2352-2384 */
static void identify_phase(Mix* m)
{
    m->phaseExist[0] = 0;
    m->phaseExist[1] = 0;
    if (m->NP == 1) {
        double A = 0, B = 0;
        for (int i = 0; i < m->NC; i++) {
            A += m->x[0][i] * m->Vc[i] * m->Tc[i];
            B += m->x[0][i] * m->Vc[i];
        }
        const double Tcm = A / B;
        if (m->T > Tcm) {
            m->phaseLabel[0] = GAS;
            m->phaseExist[1] = 1;
        } else {
            m->phaseLabel[0] = OIL;
            m->phaseExist[0] = 1;
        }
    } else {
        if (m->MW[0] > m->MW[1]) {
            m->phaseLabel[0] = OIL;
            m->phaseLabel[1] = GAS;
        } else {
            m->phaseLabel[0] = GAS;
            m->phaseLabel[1] = OIL;
        }
        m->phaseExist[0] = 1;
        m->phaseExist[1] = 1;
    }
}

/* CopyPhase, src/MixtureComp.cpp:2386-2398 */
static void copy_phase(Mix* m)
{
    for (int j = 0; j < m->NP; j++) {
        const int j1 = m->phaseLabel[j];
        m->vj[j1]    = m->vC[j];
        for (int i = 0; i < m->NC; i++) m->xij[j1 * m->numCom + i] = m->x[j][i];
        m->mu[j1]  = m->muC[j];
        m->xi[j1]  = m->xiC[j];
        m->rho[j1] = m->rhoC[j];
        m->nj[j1]  = m->nu[j];
    }
}

/* CalFlash, src/MixtureComp.cpp:697-708 */
static void cal_flash(Mix* m)
{
    phase_equilibrium(m);
    for (int j = 0; j < m->NP; j++) m->nu[j] *= m->Nh;
    cal_mw(m);
    cal_vf_xi_rho(m);
    cal_visco_lbc(m);
    identify_phase(m);
    copy_phase(m);
}

/* CalFugPAll, src/MixtureComp.cpp:2519-2579 (Zpflag = true) */
static void cal_fugp_all(Mix* m)
{
    const int NC = m->NC;
    for (int j = 0; j < m->NP; j++) {
        const double aj = m->Aj[j], bj = m->Bj[j], zj = m->Zj[j], P = m->P;
        const double Ap = aj / P, Bp = bj / P;
        m->Zp[j]        = dz_of(aj, bj, zj, Ap, Bp);
        const double G  = (zj + delta1 * bj) / (zj + delta2 * bj);
        const double Gp = (delta1 - delta2) / ((zj + delta2 * bj) * (zj + delta2 * bj)) *
                          (Bp * zj - m->Zp[j] * bj);
        for (int i = 0; i < NC; i++) {
            const double C   = P / (zj - bj);
            double       tmp = 0;
            for (int k = 0; k < NC; k++) tmp += aik(m, i, k) * m->x[j][k];
            const double E  = -aj / ((delta1 - delta2) * bj) * (2 * tmp / aj - m->Bi[i] / bj);
            const double Cp = ((zj - bj) - P * (m->Zp[j] - Bp)) / ((zj - bj) * (zj - bj));
            const double Dp = m->Bi[i] / bj * m->Zp[j];
            m->fugP[j][i]   = Cp / C + Dp + E / G * Gp;
        }
    }
}

/* CalVfiVfp_full02, src/MixtureComp.cpp:3911-3989, with
 * AssembleMatVfiVfp_full02 / AssembleRhsVfiVfp_full02 (:3991-4025) */
static void cal_vfi_vfp_full02(Mix* m)
{
    const int    NC   = m->NC;
    const double CgTP = GAS_CONSTANT * m->T / m->P;
    if (m->NP == 1) {
        const double aj = m->Aj[0], bj = m->Bj[0], zj = m->Zj[0], nu0 = m->nu[0];
        for (int i = 0; i < NC; i++) {
            double tmp = 0;
            for (int k = 0; k < NC; k++) tmp += aik(m, i, k) * m->x[0][k];
            m->An[i]    = 2 / nu0 * (tmp - aj);
            m->Bn[i]    = 1 / nu0 * (m->Bi[i] - bj);
            m->Zn[0][i] = dz_of(aj, bj, zj, m->An[i], m->Bn[i]);
            m->vfi[i]   = CgTP * (zj + nu0 * m->Zn[0][i]) - m->Vshift[i];
        }
        m->Zp[0] = ((bj - zj) * aj +
                    ((aj + delta1 * delta2 * (3 * bj * bj + 2 * bj)) +
                     ((delta1 + delta2) * (2 * bj + 1) - 2 * delta1 * delta2 * bj) * zj -
                     (delta1 + delta2 - 1) * zj * zj) *
                        bj) /
                   m->P /
                   (3 * zj * zj + 2 * ((delta1 + delta2 - 1) * bj - 1) * zj +
                    (aj + delta1 * delta2 * bj * bj - (delta1 + delta2) * bj * (bj + 1)));
        m->vfP = CgTP * nu0 * (m->Zp[0] - zj / m->P);
    } else {
        cal_fugn_all(m);
        cal_fugp_all(m);
        for (int i = 0; i < NC; i++)
            for (int k = 0; k < NC; k++)
                m->JmatDer[i * NC + k] = m->fugN[0][i * NC + k] + m->fugN[1][i * NC + k];
        double* rhs = m->rhsDer;
        for (int i = 0; i < NC; i++) rhs[i] = m->fugP[1][i] - m->fugP[0][i];
        for (int k = 0; k < NC; k++)
            for (int i = 0; i < NC; i++) rhs[(k + 1) * NC + i] = m->fugN[1][k * NC + i];
        gesv(NC, NC + 1, m->JmatDer, m->rhsDer);
        const double* dn = m->rhsDer;
        const int     j0 = m->phaseLabel[0], j1 = m->phaseLabel[1];
        m->vjp[j0] = CgTP * m->nu[0] * (m->Zp[0] - m->Zj[0] / m->P);
        m->vjp[j1] = CgTP * m->nu[1] * (m->Zp[1] - m->Zj[1] / m->P);
        for (int k = 0; k < NC; k++) {
            m->vjp[j0] += (CgTP * (m->Zj[0] + m->nu[0] * m->Zn[0][k]) - m->Vshift[k]) * dn[k];
            m->vjp[j1] -= (CgTP * (m->Zj[1] + m->nu[1] * m->Zn[1][k]) - m->Vshift[k]) * dn[k];
        }
        m->vfP = m->vjp[j0] + m->vjp[j1];
        dn += NC;
        for (int i = 0; i < NC; i++) {
            m->vfi[i]     = 0;
            m->vji[j0][i] = 0;
            m->vji[j1][i] = 0;
            for (int k = 0; k < NC; k++) {
                m->vji[j0][i] += (CgTP * (m->Zj[0] + m->nu[0] * m->Zn[0][k]) - m->Vshift[k]) * dn[k];
                m->vji[j1][i] += (CgTP * (m->Zj[1] + m->nu[1] * m->Zn[1][k]) - m->Vshift[k]) *
                                 (dlt(i, k) - dn[k]);
            }
            m->vfi[i] = m->vji[j0][i] + m->vji[j1][i];
            dn += NC;
        }
    }
}

/* CaldXsdXpAPI02p, src/MixtureComp.cpp:4386-4493 */
static void cal_dxsdxp_api02p(Mix* m)
{
    const int NC = m->NC, numCom = m->numCom, numPhase = NPH, ncol = numCom + 1;
    memset(m->dXsdXp, 0, sizeof(m->dXsdXp));
    const double vf2 = m->vf * m->vf;
    const double vwp = m->vjp[numPhase - 1];
    const double vw  = m->vj[numPhase - 1];
    if (m->NP == 1) {
        const int j1  = m->phaseLabel[0];
        double*   bId = m->dXsdXp;
        bId[0]        = ((m->vfP - vwp) * m->vf - m->vfP * m->vj[j1]) / vf2;
        bId++;
        for (int k = 0; k < NC; k++) bId[k] = m->vfi[k] * vw / vf2;
        bId += NC;
        bId[0] = -m->vfi[numCom - 1] * m->vj[j1] / vf2;
        bId++;
        for (int k = 0; k < ncol; k++) bId[k] = -m->dXsdXp[k];
        bId += ncol + 1;
        for (int i = 0; i < NC; i++) {
            for (int k = 0; k < NC; k++)
                bId[k] = (dlt(i, k) * m->Nh - m->Ni[i]) / (m->Nh * m->Nh);
            bId += ncol;
        }
    } else {
        double* bId;
        for (int j = 0; j < 2; j++) {
            const int j1 = m->phaseLabel[j];
            bId          = &m->dXsdXp[j1 * ncol];
            bId[0]       = (m->vjp[j1] * m->vf - m->vfP * m->vj[j1]) / vf2;
            bId++;
            for (int k = 0; k < numCom; k++)
                bId[k] = (m->vji[j1][k] * m->vf - m->vfi[k] * m->vj[j1]) / vf2;
        }
        bId    = &m->dXsdXp[(numPhase - 1) * ncol];
        bId[0] = (vwp * m->vf - m->vfP * vw) / vf2;
        bId++;
        for (int k = 0; k < numCom; k++)
            bId[k] = (m->vji[numPhase - 1][k] * m->vf - m->vfi[k] * vw) / vf2;
        bId += numCom;
        const int     j0 = m->phaseLabel[0], j1 = m->phaseLabel[1];
        const double* dn = m->rhsDer;
        double*       b1 = bId + j0 * NC * ncol;
        double*       b2 = bId + j1 * NC * ncol;
        double        sum = 0;
        for (int i = 0; i < NC; i++) sum += dn[i];
        for (int i = 0; i < NC; i++) {
            b1[0] = (dn[i] * m->nu[0] - sum * m->Nh * m->n[0][i]) / (m->nu[0] * m->nu[0]);
            b2[0] = (-dn[i] * m->nu[1] + sum * m->Nh * m->n[1][i]) / (m->nu[1] * m->nu[1]);
            b1 += ncol;
            b2 += ncol;
        }
        dn += NC;
        for (int k = 0; k < NC; k++) {
            sum = 0;
            for (int i = 0; i < NC; i++) sum += dn[i];
            b1 = bId + j0 * NC * ncol + k + 1;
            b2 = bId + j1 * NC * ncol + k + 1;
            for (int i = 0; i < NC; i++) {
                b1[0] = (dn[i] * m->nu[0] - sum * m->Nh * m->n[0][i]) / (m->nu[0] * m->nu[0]);
                b2[0] = ((dlt(i, k) - dn[i]) * m->nu[1] - (1 - sum) * m->Nh * m->n[1][i]) /
                        (m->nu[1] * m->nu[1]);
                b1 += ncol;
                b2 += ncol;
            }
            dn += NC;
        }
    }
}

/* CalXiPNX_partial, src/MixtureComp.cpp:3037-3092 */
static void cal_xi_pnx_partial(Mix* m)
{
    const int    NC   = m->NC;
    const double CgTP = GAS_CONSTANT * m->T / m->P;
    for (int j = 0; j < m->NP; j++) {
        const double aj = m->Aj[j], bj = m->Bj[j], zj = m->Zj[j];
        for (int i = 0; i < NC; i++) {
            double tmp = 0;
            for (int k = 0; k < NC; k++)
                tmp += m->x[j][k] * (1 - m->BIC[i * NC + k]) * sqrt(m->Ai[i] * m->Ai[k]);
            m->Ax[i] = 2 * tmp;
            m->Zx[i] = dz_of(aj, bj, zj, m->Ax[i], m->Bi[i]);
        }
        const double tmp = -m->xiC[j] * m->xiC[j];
        for (int i = 0; i < NC; i++) m->xixC[j * NC + i] = tmp * (CgTP * m->Zx[i] - m->Vshift[i]);
        m->xiPC[j] = tmp * CgTP * (m->Zp[j] - m->Zj[j] / m->P);
    }
    for (int j = 0; j < m->NP; j++) {
        const int j1 = m->phaseLabel[j];
        m->xiP[j1]   = m->xiPC[j];
        for (int i = 0; i < NC; i++) m->xix[j1 * m->numCom + i] = m->xixC[j * NC + i];
    }
}

/* CalRhoPX_partial, src/MixtureComp.cpp:3094-3114 */
static void cal_rho_px_partial(Mix* m)
{
    for (int j = 0; j < m->NP; j++) {
        const int j1 = m->phaseLabel[j];
        m->rhoP[j1]  = m->xiP[j1] * m->MW[j];
        for (int i = 0; i < m->NC; i++)
            m->rhox[j1 * m->numCom + i] =
                m->xix[j1 * m->numCom + i] * m->MW[j] + m->xi[j1] * m->MWC[i];
    }
}

/* CalMuPXLBC_partial, src/MixtureComp.cpp:3125-3213. der1IJ is identically
 * zero there (the factor -(1 / 2) is integer division), so der2IJ vanishes
 * and der3J reduces to sqrt(MW_k) * val2_kk. */
static void cal_mu_px_lbc_partial(Mix* m)
{
    const double* L = m->LBCcoef;
    for (int j = 0; j < m->NP; j++) {
        const int     j1   = m->phaseLabel[j];
        const double* xj   = m->x[j];
        const double* muA  = m->muAux[j];
        double        xTj = 0, xPj = 0, xVj = 0;
        for (int i = 0; i < m->NC; i++) {
            xTj += xj[i] * m->Tc[i];
            xPj += xj[i] * m->Pc[i];
            xVj += xj[i] * m->Vcvis[i];
        }
        double der7J = xVj * m->xiP[j1];
        double der8J = der7J * (L[1] + muA[3] * (2 * L[2] + muA[3] * (3 * L[3] + muA[3] * 4 * L[4])));
        m->muP[j1]   = (4 * 1e-4) * pow(muA[4], 3) * der8J / muA[2];
        const int bId = m->numCom * j1;
        for (int k = 0; k < m->NC; k++) {
            const double derxTj = m->Tc[k], derxPj = m->Pc[k], derMWj = m->MWC[k];
            const double val1 = m->muAux1I[k] / sqrt(m->MW[j]);
            const double Tri  = m->T / m->Tc[k];
            double       tmp;
            if (Tri <= 1.5)
                tmp = 34 * 1e-5 * pow(Tri, 0.94);
            else
                tmp = 17.78 * 1e-5 * pow(4.58 * Tri - 1.67, 0.625);
            const double der3J = m->sqrtMWi[k] * (tmp / val1);
            const double der4J = m->sqrtMWi[k];
            const double der6J =
                5.4402 *
                (1.0 / 6 * pow(xTj, -5.0 / 6) * derxTj -
                 pow(xTj, 1.0 / 6) * (0.5 / m->MW[j] * derMWj + 2.0 / 3 / xPj * derxPj)) /
                (sqrt(m->MW[j]) * pow(xPj, 2.0 / 3));
            der7J = m->xix[j1 * m->numCom + k] * xVj + m->xi[j1] * m->Vcvis[k];
            der8J = der7J * (L[1] + muA[3] * (2 * L[2] + muA[3] * (3 * L[3] + muA[3] * 4 * L[4])));
            m->mux[bId + k] = (der3J * muA[1] - muA[0] * der4J) / (muA[1] * muA[1]) +
                              1e-4 * (4 * pow(muA[4], 3) * der8J * muA[2] - (pow(muA[4], 4) - 1) * der6J) /
                                  (muA[2] * muA[2]);
        }
    }
}

/* CalPhiNSkip + AssembleSkipMatSTA + CalEigenSY, src/MixtureComp.cpp:5155-5232 */
static double skip_min_eig(Mix* m)
{
    const int    NC = m->NC;
    const double aj = m->Aj[0], bj = m->Bj[0], zj = m->Zj[0], nu0 = m->nu[0];
    const double* xj = m->x[0];
    double       phiN[MXC * MXC];
    for (int i = 0; i < NC; i++) {
        double tmp = 0;
        for (int k = 0; k < NC; k++) tmp += aik(m, i, k) * xj[k];
        m->An[i]    = 2 / nu0 * (tmp - aj);
        m->Bn[i]    = 1 / nu0 * (m->Bi[i] - bj);
        m->Zn[0][i] = dz_of(aj, bj, zj, m->An[i], m->Bn[i]);
    }
    const double G = (zj + delta1 * bj) / (zj + delta2 * bj);
    for (int i = 0; i < NC; i++) {
        const double C   = 1 / (zj - bj);
        double       tmp = 0;
        for (int k = 0; k < NC; k++) tmp += aik(m, i, k) * xj[k];
        const double E = -aj / ((delta1 - delta2) * bj) * (2 * tmp / aj - m->Bi[i] / bj);
        for (int k = 0; k <= i; k++) {
            const double a_ik = aik(m, i, k);
            const double Cnk  = (m->Bn[k] - m->Zn[0][k]) / ((zj - bj) * (zj - bj));
            const double Dnk  = m->Bi[i] / bj * (m->Zn[0][k] - (m->Bi[k] - bj) * (zj - 1) / (nu0 * bj));
            const double Gnk  = (delta1 - delta2) / ((zj + delta2 * bj) * (zj + delta2 * bj)) *
                               (m->Bn[k] * zj - m->Zn[0][k] * bj);
            double Enk = -1 / (delta1 - delta2) / (bj * bj) *
                         (2 * (bj * a_ik / nu0 + m->Bn[k] * (m->Bi[i] * aj / bj - tmp)) -
                          m->An[k] * m->Bi[i] - aj * m->Bi[i] / nu0);
            Enk -= E / nu0;
            phiN[i * NC + k] = 1 / C * Cnk + Dnk + Enk * log(G) + E / G * Gnk;
            phiN[k * NC + i] = phiN[i * NC + k];
        }
    }
    float A[MXC * MXC];
    for (int i = 0; i < NC; i++)
        for (int j = 0; j <= i; j++) {
            A[i * NC + j] = (float)(dlt(i, j) + nu0 * sqrt(xj[i] * xj[j]) * phiN[i * NC + j]);
            A[j * NC + i] = A[i * NC + j];
        }
    return (double)min_eig_sym(NC, A);
}

/* SkipStaAnaly::IfSkip / CalFtypeFIM, src/AcceleratePVT.cpp:54-120 */
static int cal_ftype_fim(const Mix* m, const double* Sjin)
{
    if (!m->use_skip) return 0;
    int skip = 0;
    if (m->sk_flag) {
        skip = 1;
        if (fabs(1 - m->sk_P / m->P) >= m->sk_minEig / 10) skip = 0;
        else if (fabs(m->sk_T - m->T) >= m->sk_minEig * 10) skip = 0;
        else
            for (int i = 0; i < m->NC; i++)
                if (fabs(m->Ni[i] / m->Nh - m->sk_z[i]) >= m->sk_minEig / 10) {
                    skip = 0;
                    break;
                }
    }
    if (skip) return 1;
    if (m->lNP >= 2) {
        for (int j = 0; j < 2; j++)
            if (Sjin[j] < 1e-4) return 0;
        return 2;
    }
    return 0;
}

/* FlashFIM, src/MixtureComp.cpp:494-573 */
static void flash_fim(Mix* m, double Pin, double Tin, const double* Niin, const double* Sjin,
                      int lastNP, const double* xijin)
{
    const int NC = m->NC, numCom = m->numCom;
    m->it_ssmsta = m->it_nrsta = m->it_ssmsp = m->it_nrsp = m->it_rr = 0;
    m->restarts  = 0;
    m->lNP = lastNP > 0 ? lastNP - 1 : 0;
    if (m->lNP == 2)
        for (int i = 0; i < NC; i++) m->lKs[i] = xijin[i] / xijin[i + numCom];
    /* InitPTN, include/MixtureComp.hpp:177-184 */
    m->P = Pin;
    m->T = Tin + CONV5;
    memcpy(m->Ni, Niin, sizeof(double) * numCom);
    m->Nh = 0;
    for (int i = 0; i < NC; i++) m->Nh += fabs(m->Ni[i]);
    for (int i = 0; i < NC; i++) m->zi[i] = m->Ni[i] / m->Nh;

    m->ftype = cal_ftype_fim(m, Sjin);
    cal_flash(m);
    cal_vfi_vfp_full02(m);

    /* water, src/MixtureComp.cpp:517-546 (single-row PVTW: zero slopes) */
    const int Wp = NPH - 1, Wc = numCom - 1;
    m->phaseExist[Wp]         = 1;
    m->xij[Wp * numCom + Wc]  = 1.0;
    m->nj[Wp]                 = m->Ni[Wc];
    m->Nt                     = m->Nh + m->Ni[Wc];
    const double Pw0 = m->pvtw[0], bw0 = m->pvtw[1], cbw = m->pvtw[2];
    const double bw  = bw0 * (1 - cbw * (m->P - Pw0));
    const double bwp = -cbw * bw0;
    m->mu[Wp]   = m->pvtw[3];
    m->xi[Wp]   = 1 / (CONV1 * bw);
    m->rho[Wp]  = m->std_RhoW / bw;
    m->muP[Wp]  = 0.0;
    m->xiP[Wp]  = -bwp / (bw * bw * CONV1);
    m->rhoP[Wp] = CONV1 * m->xiP[Wp] * m->std_RhoW;
    m->vj[Wp]   = CONV1 * m->Ni[Wc] * bw;
    m->vfi[Wc]  = CONV1 * bw;
    const double vwp = CONV1 * m->Ni[Wc] * bwp;
    m->vf += m->vj[Wp];
    m->vfP += vwp;
    m->vji[Wp][Wc] = m->vfi[Wc];
    m->vjp[Wp]     = vwp;
    /* CalSaturation, src/MixtureComp.cpp:1178-1186 */
    for (int j = 0; j < NPH; j++) m->S[j] = m->phaseExist[j] ? m->vj[j] / m->vf : 0;

    cal_dxsdxp_api02p(m);
    cal_xi_pnx_partial(m);
    cal_rho_px_partial(m);
    cal_mu_px_lbc_partial(m);

    for (int j = 0; j < NPH; j++) {
        m->pSderExist[j] = 0;
        m->pVnumCom[j]   = 0;
    }
    if (m->phaseExist[0]) {
        m->pSderExist[0] = 1;
        m->pVnumCom[0]   = NC;
    }
    if (m->phaseExist[1]) {
        m->pSderExist[1] = 1;
        m->pVnumCom[1]   = NC;
    }
    m->pSderExist[2] = 1;

    /* CalSkipForNextStep, src/MixtureComp.cpp:5234-5254 */
    if (m->use_skip) {
        if (m->flagSkip && m->ftype == 0) {
            m->sk_minEig = skip_min_eig(m);
            m->sk_P      = m->P;
            m->sk_T      = m->T;
            memcpy(m->sk_z, m->zi, sizeof(double) * NC);
        }
        m->sk_flag = m->flagSkip;
    }
}

/* MixtureComp constructor pieces, src/MixtureComp.cpp:28-165, 2321-2350 */
static void mix_init(Mix* m, const orc_fluid* f)
{
    memset(m, 0, sizeof(*m));
    const int NC = f->nc;
    m->NC        = NC;
    m->numCom    = NC + 1;
    for (int i = 0; i < NC; i++) {
        m->Tc[i]     = f->Tc[i];
        m->Pc[i]     = f->Pc[i];
        m->Vc[i]     = f->Vc[i];
        m->Vcvis[i]  = f->Vc[i];
        m->MWC[i]    = f->MW[i];
        m->Acf[i]    = f->Acf[i];
        m->OmegaA[i] = f->OmegaA[i];
        m->OmegaB[i] = f->OmegaB[i];
        m->Vshift[i] = f->Vshift[i] * (GAS_CONSTANT * f->OmegaB[i] * f->Tc[i] / f->Pc[i]);
        m->sqrtMWi[i] = sqrt(f->MW[i]);
        m->muAux1I[i] = 5.4402 * pow(f->Tc[i], 1.0 / 6) / pow(f->Pc[i], 2.0 / 3);
    }
    for (int i = 0; i < NC * NC; i++) m->BIC[i] = f->BIC[(i / NC) * NC + (i % NC)];
    for (int k = 0; k < 5; k++) {
        m->LBCcoef[k] = f->LBCcoef[k] * 10;
        m->pvtw[k]    = f->pvtw[k];
    }
    m->std_RhoW     = f->std_rho_w;
    m->rr_maxit     = f->rr_maxit;
    m->rr_tol       = f->rr_tol;
    m->ssmsta_maxit = f->ssmsta_maxit;
    m->ssmsta_tol   = f->ssmsta_tol;
    m->ssmsta_tol2  = f->ssmsta_tol * f->ssmsta_tol;
    m->ssmsta_eyt   = f->ssmsta_eyt;
    m->nrsta_maxit  = f->nrsta_maxit;
    m->nrsta_tol    = f->nrsta_tol;
    m->ssmsp_maxit  = f->ssmsp_maxit;
    m->ssmsp_tol2   = f->ssmsp_tol * f->ssmsp_tol;
    m->nrsp_maxit   = f->nrsp_maxit;
    m->nrsp_tol     = f->nrsp_tol;
    m->use_skip     = f->use_skip;
    m->Ktol         = 1e-4;
    m->dYtol        = 1e-6;
}

typedef struct {
    const orc_fluid* f;
    const orc_batch* b;
    int64_t          lo, hi;
    double           secs;
} Job;

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void* run_job(void* arg)
{
    Job*             J = (Job*)arg;
    const orc_fluid* f = J->f;
    const orc_batch* b = J->b;
    Mix*             m = (Mix*)malloc(sizeof(Mix));
    mix_init(m, f);
    const int NC = f->nc, numCom = NC + 1, ncol = numCom + 1, maxLen = ncol * ncol * NPH;
    double    Sin[NPH], xin[NPH * (MXC + 1)];
    const double t0 = now_s();
    for (int64_t n = J->lo; n < J->hi; n++) {
        memcpy(Sin, b->S_in + n * NPH, sizeof(Sin));
        memcpy(xin, b->xij_in + n * NPH * numCom, sizeof(double) * NPH * numCom);
        if (f->use_skip) {
            m->sk_flag   = b->skip_flag[n];
            m->sk_minEig = b->skip_minEig[n];
            m->sk_P      = b->skip_P[n];
            m->sk_T      = b->skip_T[n];
            memcpy(m->sk_z, b->skip_z + n * NC, sizeof(double) * NC);
        }
        flash_fim(m, b->P[n], b->T[n], b->Ni + n * numCom, Sin, b->lastNP[n], xin);
        /* copy-out as IsoT_FIM::PassFlashValue, src/OCPFluidMethod.cpp:1122-1187 */
        int pn = 0, len = 0;
        for (int j = 0; j < NPH; j++) {
            b->S[n * NPH + j]          = m->S[j];
            b->phaseExist[n * NPH + j] = m->phaseExist[j];
            if (m->phaseExist[j]) {
                pn++;
                b->rho[n * NPH + j]  = m->rho[j];
                b->xi[n * NPH + j]   = m->xi[j];
                b->mu[n * NPH + j]   = m->mu[j];
                b->rhoP[n * NPH + j] = m->rhoP[j];
                b->xiP[n * NPH + j]  = m->xiP[j];
                b->muP[n * NPH + j]  = m->muP[j];
                b->nj[n * NPH + j]   = m->nj[j];
                for (int i = 0; i < numCom; i++) {
                    const int64_t o = (n * NPH + j) * numCom + i;
                    b->xij[o]       = m->xij[j * numCom + i];
                    b->rhox[o]      = m->rhox[j * numCom + i];
                    b->xix[o]       = m->xix[j * numCom + i];
                    b->mux[o]       = m->mux[j * numCom + i];
                }
            }
            b->pSderExist[n * NPH + j] = m->pSderExist[j];
            b->pVnumCom[n * NPH + j]   = m->pVnumCom[j];
            len += m->pSderExist[j] + m->pVnumCom[j];
        }
        b->phaseNum[n] = pn;
        b->Nt[n]       = m->Nt;
        b->vf[n]       = m->vf;
        b->vfP[n]      = m->vfP;
        for (int i = 0; i < numCom; i++) b->vfi[n * numCom + i] = m->vfi[i];
        b->bRowSizedSdP[n] = len;
        memcpy(b->dSec_dPri + n * maxLen, m->dXsdXp, sizeof(double) * len * ncol);
        b->ePEC[n]         = m->ePEC;
        b->ftype[n]        = m->ftype;
        b->NPhc[n]         = m->NP;
        b->iters[n * 5 + 0] = m->it_ssmsta;
        b->iters[n * 5 + 1] = m->it_nrsta;
        b->iters[n * 5 + 2] = m->it_ssmsp;
        b->iters[n * 5 + 3] = m->it_nrsp;
        b->iters[n * 5 + 4] = m->it_rr;
        if (b->restarts) b->restarts[n] = m->restarts;
        if (f->use_skip) {
            b->skip_flag[n]   = m->sk_flag;
            b->skip_minEig[n] = m->sk_minEig;
            b->skip_P[n]      = m->sk_P;
            b->skip_T[n]      = m->sk_T;
            memcpy(b->skip_z + n * NC, m->sk_z, sizeof(double) * NC);
        }
    }
    J->secs = now_s() - t0;
    free(m);
    return NULL;
}

int orc_flash_fim_batch(const orc_fluid* fluid, const orc_batch* batch, int nthreads,
                        double* seconds)
{
    if (!fluid || !batch || fluid->nc < 2 || fluid->nc > ORC_MAX_NC) return 1;
    const int64_t n = batch->n;
    if (n <= 0) {
        if (seconds) *seconds = 0;
        return 0;
    }
    if (nthreads < 1) nthreads = 1;
    if (nthreads > n) nthreads = (int)n;
    pthread_t* th   = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    Job*       jobs = (Job*)malloc(sizeof(Job) * nthreads);
    for (int t = 0; t < nthreads; t++) {
        jobs[t].f    = fluid;
        jobs[t].b    = batch;
        jobs[t].lo   = n * t / nthreads;
        jobs[t].hi   = n * (t + 1) / nthreads;
        jobs[t].secs = 0;
        pthread_create(&th[t], NULL, run_job, &jobs[t]);
    }
    double mx = 0;
    for (int t = 0; t < nthreads; t++) {
        pthread_join(th[t], NULL);
        if (jobs[t].secs > mx) mx = jobs[t].secs;
    }
    free(th);
    free(jobs);
    if (seconds) *seconds = mx;
    return 0;
}

const char* orc_kind(void) { return "port"; }
