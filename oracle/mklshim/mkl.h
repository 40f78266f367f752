/* Minimal stand-in for <mkl.h> so the reference trainer (tensorsvm-train.cu) compiles
 * against the OpenBLAS 0.3.30 build that ships with scipy (LP64, symbols prefixed
 * "scipy_").  Only the CBLAS/LAPACKE entry points the reference calls are declared:
 *   cblas_{ddot,dnrm2,dscal,idamax,idamin,dgemv,dsyrk}   (tensorsvm-train.cu:1536-1837)
 *   LAPACKE_{dpotrf,dpotrs,dsyevd,spotrf,spstrf}        (tensorsvm-train.cu:1709,1834,2191,2279,2285)
 * The enum values are the standard CBLAS / LAPACKE ones.
 * This header is test infrastructure: it is used only by oracle/build_ref.sh. */
#ifndef TSVM_MKL_SHIM_H
#define TSVM_MKL_SHIM_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int lapack_int;
typedef int MKL_INT;

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

double scipy_cblas_ddot(int n, const double *x, int incx, const double *y, int incy);
double scipy_cblas_dnrm2(int n, const double *x, int incx);
void scipy_cblas_dscal(int n, double alpha, double *x, int incx);
size_t scipy_cblas_idamax(int n, const double *x, int incx);
size_t scipy_cblas_idamin(int n, const double *x, int incx);
void scipy_cblas_dgemv(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE trans, int m, int n,
                       double alpha, const double *a, int lda, const double *x, int incx,
                       double beta, double *y, int incy);
void scipy_cblas_dsyrk(enum CBLAS_ORDER order, enum CBLAS_UPLO uplo, enum CBLAS_TRANSPOSE trans,
                       int n, int k, double alpha, const double *a, int lda, double beta,
                       double *c, int ldc);
lapack_int scipy_LAPACKE_dpotrf(int layout, char uplo, lapack_int n, double *a, lapack_int lda);
lapack_int scipy_LAPACKE_dpotrs(int layout, char uplo, lapack_int n, lapack_int nrhs,
                                const double *a, lapack_int lda, double *b, lapack_int ldb);
lapack_int scipy_LAPACKE_dsyevd(int layout, char jobz, char uplo, lapack_int n, double *a,
                                lapack_int lda, double *w);
lapack_int scipy_LAPACKE_spotrf(int layout, char uplo, lapack_int n, float *a, lapack_int lda);
lapack_int scipy_LAPACKE_spstrf(int layout, char uplo, lapack_int n, float *a, lapack_int lda,
                                lapack_int *piv, lapack_int *rank, float tol);

#ifdef __cplusplus
}
#endif

#define cblas_ddot scipy_cblas_ddot
#define cblas_dnrm2 scipy_cblas_dnrm2
#define cblas_dscal scipy_cblas_dscal
#define cblas_idamax scipy_cblas_idamax
#define cblas_idamin scipy_cblas_idamin
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_dsyrk scipy_cblas_dsyrk
#define LAPACKE_dpotrf scipy_LAPACKE_dpotrf
#define LAPACKE_dpotrs scipy_LAPACKE_dpotrs
#define LAPACKE_dsyevd scipy_LAPACKE_dsyevd
#define LAPACKE_spotrf scipy_LAPACKE_spotrf
#define LAPACKE_spstrf scipy_LAPACKE_spstrf

#endif
