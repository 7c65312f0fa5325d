/*
 * Minimal LAPACKE prototype header for compiling H2Pack's own sources.
 *
 * Build support.  H2Pack's src/linalg_lib_wrapper.h:17 includes
 * <lapacke.h>.  The construction and matvec/matmul sources call no LAPACKE routine;
 * the HSS ULV factorizations (src/H2Pack_HSS_ULV.c, through the LAPACK_* names of
 * src/H2Pack_config.h:37-46) call the four below.  Layout constants, the lapack_int
 * type and the prototypes are written from the public LAPACKE API; the library that
 * provides them is the OpenBLAS the builds link.
 */
#ifndef H2B_ORACLE_LAPACKE_H
#define H2B_ORACLE_LAPACKE_H

#ifdef __cplusplus
extern "C" {
#endif

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
typedef int lapack_int;

lapack_int LAPACKE_dgeqrf(int matrix_layout, lapack_int m, lapack_int n, double *a, lapack_int lda, double *tau);
lapack_int LAPACKE_dormqr(int matrix_layout, char side, char trans, lapack_int m, lapack_int n, lapack_int k,
                          const double *a, lapack_int lda, const double *tau, double *c, lapack_int ldc);
lapack_int LAPACKE_dpotrf(int matrix_layout, char uplo, lapack_int n, double *a, lapack_int lda);
lapack_int LAPACKE_dgetrf(int matrix_layout, lapack_int m, lapack_int n, double *a, lapack_int lda, lapack_int *ipiv);

#ifdef __cplusplus
}
#endif

#endif
