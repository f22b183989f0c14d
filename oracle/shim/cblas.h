/*
 * Test-infrastructure shim: lets the reference's unmodified
 * src/dense/matrixops.cpp (which includes <cblas.h>) compile against the
 * OpenBLAS 0.3.30 (LP64) bundled with scipy, whose exports carry a
 * "scipy_" prefix.  Only the two CBLAS routines the reference calls are
 * declared.  Used only by oracle/Makefile to build oracle/_ref.
 */
#ifndef ORACLE_SHIM_CBLAS_H
#define ORACLE_SHIM_CBLAS_H
#ifdef __cplusplus
extern "C" {
#endif

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };

void scipy_cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE ta,
                       enum CBLAS_TRANSPOSE tb, int m, int n, int k,
                       double alpha, const double *a, int lda, const double *b,
                       int ldb, double beta, double *c, int ldc);
void scipy_cblas_dsyrk(enum CBLAS_ORDER order, enum CBLAS_UPLO uplo,
                       enum CBLAS_TRANSPOSE trans, int n, int k, double alpha,
                       const double *a, int lda, double beta, double *c,
                       int ldc);

#define cblas_dgemm scipy_cblas_dgemm
#define cblas_dsyrk scipy_cblas_dsyrk

#ifdef __cplusplus
}
#endif
#endif
