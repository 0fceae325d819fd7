/* Minimal CBLAS declarations so the reference's ki_mat.cpp compiles against
 * the LP64 OpenBLAS 0.3.15 shipped in the image (test infrastructure only). */
#ifndef ORACLE_SHIM_CBLAS_H_
#define ORACLE_SHIM_CBLAS_H_
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta,
                 enum CBLAS_TRANSPOSE tb, int m, int n, int k, double alpha,
                 const double* a, int lda, const double* b, int ldb,
                 double beta, double* c, int ldc);
#ifdef __cplusplus
}
#endif
#endif
