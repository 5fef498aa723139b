/* Prototype-only LAPACKE header for compiling the reference's CPU path
 * against scipy's bundled OpenBLAS ("scipy_"-prefixed exports).  Test
 * infrastructure only. */
#ifndef ORACLE_REF_SHIM_LAPACKE_H
#define ORACLE_REF_SHIM_LAPACKE_H
#ifdef __cplusplus
extern "C" {
#endif
typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
#define LAPACKE_sgeqrf scipy_LAPACKE_sgeqrf
#define LAPACKE_dgeqrf scipy_LAPACKE_dgeqrf
#define LAPACKE_sgeqrf_work scipy_LAPACKE_sgeqrf_work
#define LAPACKE_dgeqrf_work scipy_LAPACKE_dgeqrf_work
#define LAPACKE_strtri scipy_LAPACKE_strtri
#define LAPACKE_dtrtri scipy_LAPACKE_dtrtri
lapack_int LAPACKE_sgeqrf(int layout, lapack_int m, lapack_int n, float* a,
                          lapack_int lda, float* tau);
lapack_int LAPACKE_dgeqrf(int layout, lapack_int m, lapack_int n, double* a,
                          lapack_int lda, double* tau);
lapack_int LAPACKE_sgeqrf_work(int layout, lapack_int m, lapack_int n, float* a,
                               lapack_int lda, float* tau, float* work,
                               lapack_int lwork);
lapack_int LAPACKE_dgeqrf_work(int layout, lapack_int m, lapack_int n,
                               double* a, lapack_int lda, double* tau,
                               double* work, lapack_int lwork);
lapack_int LAPACKE_strtri(int layout, char uplo, char diag, lapack_int n,
                          float* a, lapack_int lda);
lapack_int LAPACKE_dtrtri(int layout, char uplo, char diag, lapack_int n,
                          double* a, lapack_int lda);
#ifdef __cplusplus
}
#endif
#endif
