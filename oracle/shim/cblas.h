/* Declaration-only CBLAS header used to compile the reference CPU sources
 * (delayed_lu/delayed_dgetrf.cpp, delayed_dgetrf_column.cpp, lapack_dgetrf.cpp and
 * delayed-bunch-kaufman/delayed_sytrf.cpp, delayed_sytrf_blocked.cpp, lapack_dsytrf.cpp)
 * unmodified against SciPy's bundled OpenBLAS, whose exported symbols carry a
 * `scipy_` prefix.  Enumerator values are the netlib CBLAS values.  Only the
 * routines that the reference calls are declared.
 *
 * Test infrastructure: nothing in the product library includes this file. */
#ifndef DP_ORACLE_CBLAS_SHIM_H
#define DP_ORACLE_CBLAS_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;
typedef enum { CblasLeft = 141, CblasRight = 142 } CBLAS_SIDE;
typedef CBLAS_ORDER CBLAS_LAYOUT;

#define cblas_idamax scipy_cblas_idamax
#define cblas_dswap scipy_cblas_dswap
#define cblas_dscal scipy_cblas_dscal
#define cblas_dger scipy_cblas_dger
#define cblas_dtrsm scipy_cblas_dtrsm
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_dsyr scipy_cblas_dsyr
#define cblas_dsyr2 scipy_cblas_dsyr2
#define cblas_dsyr2k scipy_cblas_dsyr2k

/* OpenBLAS LP64: blasint == int, CBLAS_INDEX == size_t. */
unsigned long cblas_idamax(const int n, const double *x, const int incx);
void cblas_dswap(const int n, double *x, const int incx, double *y, const int incy);
void cblas_dscal(const int n, const double alpha, double *x, const int incx);
void cblas_dger(CBLAS_ORDER order, const int m, const int n, const double alpha,
                const double *x, const int incx, const double *y, const int incy,
                double *a, const int lda);
void cblas_dtrsm(CBLAS_ORDER order, CBLAS_SIDE side, CBLAS_UPLO uplo,
                 CBLAS_TRANSPOSE transa, CBLAS_DIAG diag, const int m, const int n,
                 const double alpha, const double *a, const int lda, double *b,
                 const int ldb);
void cblas_dgemm(CBLAS_ORDER order, CBLAS_TRANSPOSE transa, CBLAS_TRANSPOSE transb,
                 const int m, const int n, const int k, const double alpha,
                 const double *a, const int lda, const double *b, const int ldb,
                 const double beta, double *c, const int ldc);
void cblas_dgemv(CBLAS_ORDER order, CBLAS_TRANSPOSE trans, const int m, const int n,
                 const double alpha, const double *a, const int lda, const double *x,
                 const int incx, const double beta, double *y, const int incy);
void cblas_dsyr(CBLAS_ORDER order, CBLAS_UPLO uplo, const int n, const double alpha,
                const double *x, const int incx, double *a, const int lda);
void cblas_dsyr2(CBLAS_ORDER order, CBLAS_UPLO uplo, const int n, const double alpha,
                 const double *x, const int incx, const double *y, const int incy,
                 double *a, const int lda);
void cblas_dsyr2k(CBLAS_ORDER order, CBLAS_UPLO uplo, CBLAS_TRANSPOSE trans, const int n,
                  const int k, const double alpha, const double *a, const int lda,
                  const double *b, const int ldb, const double beta, double *c,
                  const int ldc);

#ifdef __cplusplus
}
#endif
#endif
