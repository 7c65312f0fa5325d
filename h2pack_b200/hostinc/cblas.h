/*
 * Minimal CBLAS prototype header for compiling H2Pack's own sources.
 *
 * Build support: H2Pack (src/linalg_lib_wrapper.h:16 includes <cblas.h>) is
 * compiled unchanged against the OpenBLAS shared object that ships inside the
 * Python environment, which has no development headers.  It declares only the enums and routines that the
 * reference's construction and matvec/matmul files call, with the standard
 * CBLAS enum values (Netlib CBLAS ABI), written from the public CBLAS API.
 */
#ifndef H2B_ORACLE_CBLAS_H
#define H2B_ORACLE_CBLAS_H

#include <stddef.h>
#include <stdint.h>  /* OpenBLAS's cblas.h provides <stdint.h> transitively; src/H2Pack_utils.c:139 relies on it */

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef CBLAS_LAYOUT CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;
typedef enum { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef enum { CblasNonUnit = 131, CblasUnit = 132 } CBLAS_DIAG;
typedef enum { CblasLeft = 141, CblasRight = 142 } CBLAS_SIDE;

double cblas_dnrm2(const int n, const double *x, const int incx);
float  cblas_snrm2(const int n, const float *x, const int incx);
double cblas_ddot(const int n, const double *x, const int incx, const double *y, const int incy);
float  cblas_sdot(const int n, const float *x, const int incx, const float *y, const int incy);

void cblas_dgemv(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE trans, const int m, const int n,
                 const double alpha, const double *a, const int lda, const double *x, const int incx,
                 const double beta, double *y, const int incy);
void cblas_sgemv(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE trans, const int m, const int n,
                 const float alpha, const float *a, const int lda, const float *x, const int incx,
                 const float beta, float *y, const int incy);

void cblas_dgemm(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE transa, const CBLAS_TRANSPOSE transb,
                 const int m, const int n, const int k, const double alpha, const double *a, const int lda,
                 const double *b, const int ldb, const double beta, double *c, const int ldc);
void cblas_sgemm(const CBLAS_LAYOUT layout, const CBLAS_TRANSPOSE transa, const CBLAS_TRANSPOSE transb,
                 const int m, const int n, const int k, const float alpha, const float *a, const int lda,
                 const float *b, const int ldb, const float beta, float *c, const int ldc);

void cblas_dsyrk(const CBLAS_LAYOUT layout, const CBLAS_UPLO uplo, const CBLAS_TRANSPOSE trans,
                 const int n, const int k, const double alpha, const double *a, const int lda,
                 const double beta, double *c, const int ldc);
void cblas_dtrsm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side, const CBLAS_UPLO uplo,
                 const CBLAS_TRANSPOSE transa, const CBLAS_DIAG diag, const int m, const int n,
                 const double alpha, const double *a, const int lda, double *b, const int ldb);
void cblas_dtrmm(const CBLAS_LAYOUT layout, const CBLAS_SIDE side, const CBLAS_UPLO uplo,
                 const CBLAS_TRANSPOSE transa, const CBLAS_DIAG diag, const int m, const int n,
                 const double alpha, const double *a, const int lda, double *b, const int ldb);

void openblas_set_num_threads(int num_threads);

#ifdef __cplusplus
}
#endif

#endif
