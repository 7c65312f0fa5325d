/*
 * h2p_dropin.h -- GPU drop-in for H2Pack's apply path.
 *
 * libH2Pack_gpu.so exports H2Pack's own apply entry points with byte-identical
 * signatures, so a program built against H2Pack links this library in place of
 * H2Pack_matvec.o / H2Pack_matmul.o and runs the four phases on the GPU:
 *
 *   H2P_matvec                       src/H2Pack_matvec.h:17
 *   H2P_permute_vector_forward       src/H2Pack_matvec.h:29
 *   H2P_permute_vector_backward      src/H2Pack_matvec.h:30
 *   H2P_matmul                       src/H2Pack_matmul.h:25-28
 *   H2P_permute_matrix_row_forward   src/H2Pack_matmul.h:47-50
 *   H2P_permute_matrix_row_backward  src/H2Pack_matmul.h:51-54
 *
 * The first call on an H2Pack handle uploads its representation (tree, pair
 * lists, U, B, D, coordinates, permutations) into a device image kept in a
 * registry keyed by the handle; later calls reuse it.  A fingerprint of the
 * handle (sizes, array addresses and a strided sample of the array contents) is
 * checked on every call, so a handle rebuilt or changed in place is re-uploaded.
 * Calls on one handle are serialised by a lock of that handle; calls on different
 * handles run concurrently.  Like the reference (ASSERT_PRINTF, src/utils.h:56-66)
 * the void entry points print the reason and abort on failure; the H2P_gpu_*
 * variants return an h2gpu status instead.
 *
 *   H2P_destroy                      src/H2Pack_typedef.h (src/H2Pack_typedef.c:210):
 *                                    releases the handle's device image, then frees
 *                                    the handle as H2Pack does
 *
 * JIT-mode handles carry their kernel only as a function pointer and a parameter
 * pointer (src/H2Pack_typedef.h:160, :193).  The drop-in calls that function on a
 * fixed probe point set and matches the values against Coulomb, Gaussian,
 * Matern-3/2 and RPY with the handle's parameter; a JIT handle whose kernel matches
 * none of them is refused with H2GPU_ERR_UNSUPPORTED (there is no CPU fallback).
 *
 * Extra entry points (no counterpart in the reference):
 *   H2P_gpu_set_kernel     name the kernel of a JIT-mode handle explicitly instead of
 *                          identifying it
 *   H2P_gpu_kernel_of      the kernel id and parameters the drop-in uses for a handle
 *   H2P_gpu_build_uj       construction: U / J of scalar kernels on the GPU (off by default)
 *   H2P_gpu_set_precision  H2GPU_PREC_FP64 (default) or H2GPU_PREC_MIXED
 *   H2P_gpu_matvec / H2P_gpu_matmul   status-returning forms
 *   H2P_gpu_image          the handle's device image (for h2gpu_get_stats)
 *   H2P_gpu_release        free the handle's device image early (H2P_destroy does it too)
 *   H2P_gpu_ULV_solve      status-returning form of the HSS ULV solves
 *   H2P_gpu_ULV_release    free the handle's device ULV factors early
 *   H2P_gpu_last_error     message of the last failure
 *
 * Handles in HSS mode are applied over their HSS pair lists and minimum admissible
 * level, as H2Pack does (src/H2Pack_matvec.c:101, :308, :773, :904), and their ULV
 * solves run on the GPU after H2Pack's own factorization.  RPY-Ewald /
 * periodic handles and H2ERI handles are rejected with H2GPU_ERR_UNSUPPORTED.
 */
#ifndef H2P_DROPIN_H
#define H2P_DROPIN_H

#include "h2gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

struct H2Pack;

/* Same signatures as H2Pack (DTYPE = double, CBLAS_LAYOUT passed as its int value). */
void H2P_matvec(struct H2Pack *h2pack, const double *x, double *y);
void H2P_permute_vector_forward(struct H2Pack *h2pack, const double *x, double *pmt_x);
void H2P_permute_vector_backward(struct H2Pack *h2pack, const double *x, double *pmt_x);
void H2P_matmul(struct H2Pack *h2pack, const int layout, const int n_vec,
                const double *mat_x, const int ldx, double *mat_y, const int ldy);
void H2P_permute_matrix_row_forward(struct H2Pack *h2pack, const int layout, const int n_vec,
                                    const double *mat_x, const int ldx, double *pmt_mat_x, const int ldp);
void H2P_permute_matrix_row_backward(struct H2Pack *h2pack, const int layout, const int n_vec,
                                     const double *mat_x, const int ldx, double *pmt_mat_x, const int ldp);

void H2P_destroy(struct H2Pack **h2pack_);

/* HSS ULV solves on the GPU (replace src/H2Pack_HSS_ULV.c:981 and :429, same
   signatures, checks and messages; the factorizations H2P_HSS_ULV_Cholesky_factorize /
   H2P_HSS_ULV_LU_factorize stay H2Pack's).  The handle's factors are uploaded on the
   first solve after each factorization; a device failure prints the reason and aborts. */
void H2P_HSS_ULV_Cholesky_solve(struct H2Pack *h2pack, const int op, const double *b, double *x);
void H2P_HSS_ULV_LU_solve(struct H2Pack *h2pack, const int op, const double *b, double *x);

int  H2P_gpu_set_kernel(struct H2Pack *h2pack, int kernel_id, const double *param, int n_param);
int  H2P_gpu_kernel_of(struct H2Pack *h2pack, int *kernel_id, double *param4, int *n_param);

/* Construction on the GPU: with on = 1 (or H2GPU_BUILD_UJ=1 in the environment), later
   H2P_build calls of scalar-kernel H2 handles (Coulomb, Gaussian, Matern 3/2, relative-
   norm stop, 3-D) compute the projection matrices U and skeleton sets J on the device
   (h2gpu_id_batch, one batch per tree level) in place of H2P_build_H2_UJ_proxy
   (src/H2Pack_build.c:32-270); other handles, HSS mode and on = 0 (the default) run
   H2Pack's CPU code.  A device failure prints a message and falls back to it.  The
   skeletons match H2Pack's in accuracy (pivots can differ where column norms tie). */
void H2P_gpu_build_uj(int on);
/* How many H2P_build calls so far had their U / J computed on the device. */
int  H2P_gpu_build_uj_count(void);
/* Numerical proxy points on the GPU: with on = 1 (or H2GPU_BUILD_PP=1), later
   H2P_generate_proxy_point_ID_file calls of scalar kernels select each level's proxy
   points on the device (H2P_generate_proxy_point_nlayer, src/H2Pack_gen_proxy_point.c:
   56-330, algorithm 2, reltol >= 1e-12, H2Pack's own random candidates); off by
   default, since late pivots can differ from H2Pack's where column norms tie to
   rounding.  The proxy points give H2Pack's accuracy. */
void H2P_gpu_build_pp(int on);
/* How many proxy-point levels so far were selected on the device. */
int  H2P_gpu_build_pp_count(void);
int  H2P_gpu_set_precision(struct H2Pack *h2pack, int precision);
int  H2P_gpu_matvec(struct H2Pack *h2pack, const double *x, double *y);
int  H2P_gpu_matmul(struct H2Pack *h2pack, int layout, int n_vec,
                    const double *mat_x, int ldx, double *mat_y, int ldy);
h2gpu_image *H2P_gpu_image(struct H2Pack *h2pack);
int  H2P_gpu_release(struct H2Pack *h2pack);
const char *H2P_gpu_last_error(void);
/* Status-returning form of the two ULV solves (lu = 1: LU factors, 0: Cholesky). */
int  H2P_gpu_ULV_solve(struct H2Pack *h2pack, int lu, int op, const double *b, double *x);
/* Free the handle's device ULV factors early (H2P_destroy does it too). */
int  H2P_gpu_ULV_release(struct H2Pack *h2pack);

#ifdef __cplusplus
}
#endif

#endif
