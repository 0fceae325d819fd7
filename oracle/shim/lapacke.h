/* Minimal LAPACKE declarations (LP64) for the reference build; the symbols
 * come from the image's OpenBLAS 0.3.15 (test infrastructure only). */
#ifndef ORACLE_SHIM_LAPACKE_H_
#define ORACLE_SHIM_LAPACKE_H_
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
typedef int lapack_int;
#ifdef __cplusplus
extern "C" {
#endif
lapack_int LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double* a,
                          lapack_int lda, lapack_int* ipiv);
lapack_int LAPACKE_dgetrs(int layout, char trans, lapack_int n,
                          lapack_int nrhs, const double* a, lapack_int lda,
                          const lapack_int* ipiv, double* b, lapack_int ldb);
lapack_int LAPACKE_dgeqp3(int layout, lapack_int m, lapack_int n, double* a,
                          lapack_int lda, lapack_int* jpvt, double* tau);
lapack_int LAPACKE_dtrtrs(int layout, char uplo, char trans, char diag,
                          lapack_int n, lapack_int nrhs, const double* a,
                          lapack_int lda, double* b, lapack_int ldb);
lapack_int LAPACKE_dgeev(int layout, char jobvl, char jobvr, lapack_int n,
                         double* a, lapack_int lda, double* wr, double* wi,
                         double* vl, lapack_int ldvl, double* vr,
                         lapack_int ldvr);
#ifdef __cplusplus
}
#endif
#endif
