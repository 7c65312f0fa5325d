/*
 * Minimal LAPACKE prototype header for compiling H2Pack's own sources.
 *
 * Build support.  H2Pack's src/linalg_lib_wrapper.h:17 includes
 * <lapacke.h>; the construction and matvec/matmul sources compiled by the oracle
 * recipe call no LAPACKE routine, so this header only supplies the layout
 * constants and the lapack_int type, written from the public LAPACKE API.
 */
#ifndef H2B_ORACLE_LAPACKE_H
#define H2B_ORACLE_LAPACKE_H

#ifdef __cplusplus
extern "C" {
#endif

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
typedef int lapack_int;

#ifdef __cplusplus
}
#endif

#endif
