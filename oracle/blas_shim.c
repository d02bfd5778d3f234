/*
 * Forward the Fortran BLAS/LAPACK names that the reference's SparseLDL calls
 * to the prefixed exports of the OpenBLAS build bundled with scipy, so the
 * oracle needs no system BLAS.  Oracle-only (test infrastructure).
 */
#define FWD(ret, name, params, args)       \
  extern ret scipy_##name params;          \
  ret name params { return scipy_##name args; }

FWD(int, idamax_, (const int* n, const double* a, const int* inc), (n, a, inc))
FWD(void, dcopy_, (const int* n, const double* x, const int* incx, double* y, const int* incy),
    (n, x, incx, y, incy))
FWD(void, dswap_, (const int* n, double* x, const int* incx, double* y, const int* incy),
    (n, x, incx, y, incy))
FWD(void, dscal_, (const int* n, const double* a, double* x, const int* incx), (n, a, x, incx))
FWD(void, dsyrk_, (const char* uplo, const char* trans, const int* n, const int* k,
                   const double* alpha, const double* a, const int* lda, const double* beta,
                   double* c, const int* ldc),
    (uplo, trans, n, k, alpha, a, lda, beta, c, ldc))
FWD(void, dgemm_, (const char* ta, const char* tb, const int* m, const int* n, const int* k,
                   const double* alpha, const double* a, const int* lda, const double* b,
                   const int* ldb, const double* beta, double* c, const int* ldc),
    (ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc))
FWD(void, dgemv_, (const char* t, const int* m, const int* n, const double* alpha,
                   const double* a, const int* lda, const double* x, const int* incx,
                   const double* beta, double* y, const int* incy),
    (t, m, n, alpha, a, lda, x, incx, beta, y, incy))
FWD(void, dtrsm_, (const char* side, const char* uplo, const char* ta, const char* diag,
                   const int* m, const int* n, const double* alpha, const double* a,
                   const int* lda, double* b, const int* ldb),
    (side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb))
FWD(void, dpotrf_, (const char* uplo, const int* n, double* a, const int* lda, int* info),
    (uplo, n, a, lda, info))
FWD(void, dsytrf_, (const char* uplo, const int* n, double* a, const int* lda, int* ipiv,
                    double* work, const int* lwork, int* info),
    (uplo, n, a, lda, ipiv, work, lwork, info))
FWD(void, dsytrs_, (const char* uplo, const int* n, const int* nrhs, const double* a,
                    const int* lda, const int* ipiv, double* b, const int* ldb, int* info),
    (uplo, n, nrhs, a, lda, ipiv, b, ldb, info))
