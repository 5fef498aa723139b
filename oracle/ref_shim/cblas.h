/* Prototype-only CBLAS header used to compile the reference's CPU path
 * against the OpenBLAS build that ships inside scipy (its exported symbols
 * carry a "scipy_" prefix).  Only the routines the reference calls are
 * declared.  Test infrastructure: never part of the product library. */
#ifndef ORACLE_REF_SHIM_CBLAS_H
#define ORACLE_REF_SHIM_CBLAS_H
#ifdef __cplusplus
extern "C" {
#endif
typedef int blasint;
typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef CBLAS_ORDER CBLAS_LAYOUT;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;

#define cblas_sgemv scipy_cblas_sgemv
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_sgemm scipy_cblas_sgemm
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_snrm2 scipy_cblas_snrm2
#define cblas_dnrm2 scipy_cblas_dnrm2
#define cblas_sscal scipy_cblas_sscal
#define cblas_dscal scipy_cblas_dscal
#define cblas_saxpy scipy_cblas_saxpy
#define cblas_daxpy scipy_cblas_daxpy
#define cblas_scopy scipy_cblas_scopy
#define cblas_dcopy scipy_cblas_dcopy
#define cblas_strsv scipy_cblas_strsv
#define cblas_dtrsv scipy_cblas_dtrsv

void cblas_sgemv(CBLAS_ORDER, CBLAS_TRANSPOSE, int m, int n, float alpha,
                 const float* a, int lda, const float* x, int incx, float beta,
                 float* y, int incy);
void cblas_dgemv(CBLAS_ORDER, CBLAS_TRANSPOSE, int m, int n, double alpha,
                 const double* a, int lda, const double* x, int incx,
                 double beta, double* y, int incy);
void cblas_sgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int m, int n,
                 int k, float alpha, const float* a, int lda, const float* b,
                 int ldb, float beta, float* c, int ldc);
void cblas_dgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int m, int n,
                 int k, double alpha, const double* a, int lda,
                 const double* b, int ldb, double beta, double* c, int ldc);
float cblas_snrm2(int n, const float* x, int incx);
double cblas_dnrm2(int n, const double* x, int incx);
void cblas_sscal(int n, float alpha, float* x, int incx);
void cblas_dscal(int n, double alpha, double* x, int incx);
void cblas_saxpy(int n, float alpha, const float* x, int incx, float* y, int incy);
void cblas_daxpy(int n, double alpha, const double* x, int incx, double* y, int incy);
void cblas_scopy(int n, const float* x, int incx, float* y, int incy);
void cblas_dcopy(int n, const double* x, int incx, double* y, int incy);
void cblas_strsv(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_DIAG, int n,
                 const float* a, int lda, float* x, int incx);
void cblas_dtrsv(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_DIAG, int n,
                 const double* a, int lda, double* x, int incx);
#ifdef __cplusplus
}
#endif
#endif
