/*
 * blas_shim.c -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference declares Fortran BLAS/LAPACK prototypes (include/DenseMat.hpp)
 * and links a system library. This image has none; SciPy ships an LP64
 * OpenBLAS whose symbols carry a "scipy_" prefix. These forwarders give the
 * reference's objects the unprefixed names they expect.
 */
extern void scipy_dsysv_(const char*, const int*, const int*, double*, const int*,
                         int*, double*, const int*, double*, const int*, int*);
extern void scipy_dgesv_(const int*, const int*, double*, const int*, int*, double*,
                         const int*, int*);
extern void scipy_ssyevd_(const char*, const char*, const int*, float*, const int*,
                          float*, float*, const int*, int*, const int*, int*);
extern double scipy_dnrm2_(const int*, const double*, const int*);
extern double scipy_dasum_(const int*, const double*, const int*);
extern void scipy_dcopy_(const int*, const double*, const int*, double*, const int*);
extern void scipy_daxpy_(const int*, const double*, const double*, const int*, double*,
                         const int*);
extern void scipy_dscal_(const int*, const double*, double*, const int*);
extern double scipy_ddot_(const int*, const double*, const int*, const double*,
                          const int*);
extern void scipy_dgemm_(const char*, const char*, const int*, const int*, const int*,
                         const double*, const double*, const int*, const double*,
                         const int*, const double*, double*, const int*);

void dsysv_(const char* uplo, const int* n, const int* nrhs, double* a, const int* lda,
            int* ipiv, double* b, const int* ldb, double* work, const int* lwork,
            int* info)
{
    scipy_dsysv_(uplo, n, nrhs, a, lda, ipiv, b, ldb, work, lwork, info);
}

void dgesv_(const int* n, const int* nrhs, double* a, const int* lda, int* ipiv,
            double* b, const int* ldb, int* info)
{
    scipy_dgesv_(n, nrhs, a, lda, ipiv, b, ldb, info);
}

void ssyevd_(const char* jobz, const char* uplo, const int* n, float* a, const int* lda,
             float* w, float* work, const int* lwork, int* iwork, const int* liwork,
             int* info)
{
    scipy_ssyevd_(jobz, uplo, n, a, lda, w, work, lwork, iwork, liwork, info);
}

double dnrm2_(const int* n, const double* x, const int* incx)
{
    return scipy_dnrm2_(n, x, incx);
}

double dasum_(const int* n, const double* x, const int* incx)
{
    return scipy_dasum_(n, x, incx);
}

void dcopy_(const int* n, const double* x, const int* incx, double* y, const int* incy)
{
    scipy_dcopy_(n, x, incx, y, incy);
}

void daxpy_(const int* n, const double* a, const double* x, const int* incx, double* y,
            const int* incy)
{
    scipy_daxpy_(n, a, x, incx, y, incy);
}

void dscal_(const int* n, const double* a, double* x, const int* incx)
{
    scipy_dscal_(n, a, x, incx);
}

double ddot_(const int* n, const double* x, const int* incx, const double* y,
             const int* incy)
{
    return scipy_ddot_(n, x, incx, y, incy);
}

void dgemm_(const char* ta, const char* tb, const int* m, const int* n, const int* k,
            const double* alpha, const double* a, const int* lda, const double* b,
            const int* ldb, const double* beta, double* c, const int* ldc)
{
    scipy_dgemm_(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}
