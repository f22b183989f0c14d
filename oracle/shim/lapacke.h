/*
 * Test-infrastructure shim: maps the four LAPACKE routines that the
 * reference's src/dense/matrixops.cpp calls onto the "scipy_"-prefixed
 * exports of scipy's bundled OpenBLAS 0.3.30 (LP64, 32-bit lapack_int).
 * Used only by oracle/Makefile to build oracle/_ref.
 */
#ifndef ORACLE_SHIM_LAPACKE_H
#define ORACLE_SHIM_LAPACKE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

lapack_int scipy_LAPACKE_dgesvd(int matrix_layout, char jobu, char jobvt,
                                lapack_int m, lapack_int n, double *a,
                                lapack_int lda, double *s, double *u,
                                lapack_int ldu, double *vt, lapack_int ldvt,
                                double *superb);
lapack_int scipy_LAPACKE_dgeqrf(int matrix_layout, lapack_int m, lapack_int n,
                                double *a, lapack_int lda, double *tau);
lapack_int scipy_LAPACKE_dorgqr(int matrix_layout, lapack_int m, lapack_int n,
                                lapack_int k, double *a, lapack_int lda,
                                const double *tau);
lapack_int scipy_LAPACKE_dsyevd(int matrix_layout, char jobz, char uplo,
                                lapack_int n, double *a, lapack_int lda,
                                double *w);

#define LAPACKE_dgesvd scipy_LAPACKE_dgesvd
#define LAPACKE_dgeqrf scipy_LAPACKE_dgeqrf
#define LAPACKE_dorgqr scipy_LAPACKE_dorgqr
#define LAPACKE_dsyevd scipy_LAPACKE_dsyevd

#ifdef __cplusplus
}
#endif
#endif
