/*
 * h2gpu.h -- C ABI of the B200 (sm_100a) H2 matrix apply engine.
 *
 * The engine multiplies an H2 matrix representation produced by H2Pack's
 * construction (H2P_partition_points + H2P_build) by vectors and matrices on one
 * GPU.  Everything here is plain C: pointers, sizes and status codes; no CUDA or
 * torch types appear in the signatures (streams are passed as void*).
 *
 * What each entry point replaces in the reference (paths are within the
 * H2Pack project):
 *   h2gpu_image_create   the per-handle state that H2P_matvec/H2P_matmul keep in
 *                        struct H2Pack (src/H2Pack_typedef.h:88-205): y0/y1
 *                        buffers (src/H2Pack_matvec.c:68-92, :234-269), thread
 *                        buffers, B_blk/D_blk task partitions
 *                        (src/H2Pack_build.c:762-764, :1006-1008)
 *   h2gpu_matvec         H2P_matvec (src/H2Pack_matvec.h:17, src/H2Pack_matvec.c:1162-1284)
 *   h2gpu_matmul         H2P_matmul (src/H2Pack_matmul.h:25-28, src/H2Pack_matmul.c:455-583)
 *   h2gpu_permute_*      H2P_permute_vector_{forward,backward} (src/H2Pack_matvec.h:29-30)
 *                        and H2P_permute_matrix_row_{forward,backward}
 *                        (src/H2Pack_matmul.h:47-54)
 *   h2gpu_direct_sum     direct_nbody (examples/direct_nbody.h:2-54)
 *   h2gpu_id_batch       the interpolative decompositions of H2P_build_H2_UJ_proxy
 *                        (src/H2Pack_build.c:32-270, src/H2Pack_ID_compress.c:491-576)
 *   h2gpu_get_stats      the timers[] / mat_size[] / JIT_flops[] counters
 *                        (src/H2Pack_typedef.h:200-204, :226-239) read by
 *                        H2P_print_statistic (src/H2Pack_typedef.c:345-524)
 *
 * All functions return H2GPU_OK (0) or a negative status; h2gpu_last_error()
 * returns a thread-local message for the last failure.  No function traps on the
 * device and there is no CPU fallback: a missing GPU is an error.
 */
#ifndef H2GPU_H
#define H2GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define H2GPU_ABI_VERSION 2

/* Status codes */
#define H2GPU_OK               0
#define H2GPU_ERR_INVALID     -1   /* malformed descriptor or argument          */
#define H2GPU_ERR_UNSUPPORTED -2   /* mode the engine does not implement        */
#define H2GPU_ERR_CUDA        -3   /* CUDA runtime error (no GPU, launch, ...)  */
#define H2GPU_ERR_NOMEM       -4   /* device or host allocation failed          */
#define H2GPU_ERR_STATE       -5   /* call out of order / handle destroyed      */
#define H2GPU_ERR_DEVICE      -6   /* device-side check failed (status word)    */

/* Kernel functions K(x, y).  The reference keeps only function pointers to
 * static functions (src/H2Pack_typedef.h:193-196, src/H2Pack_3D_kernels.h), so
 * the kernel identity crosses the ABI as an id plus its parameter array. */
#define H2GPU_KRNL_NONE      0    /* AOT only: B and D are stored               */
#define H2GPU_KRNL_COULOMB   1    /* 1/r, param[0] on r == 0 (0 if no param),    src/H2Pack_3D_kernels.h:50-161 */
#define H2GPU_KRNL_GAUSSIAN  2    /* exp(-l r^2), l = param[0],                  src/H2Pack_3D_kernels.h:167-268 */
#define H2GPU_KRNL_MATERN32  3    /* (1+sqrt3 l r) exp(-sqrt3 l r), l = param[0], src/H2Pack_3D_kernels.h:384-497 */
#define H2GPU_KRNL_RPY       4    /* 3x3 Rotne-Prager-Yamakawa, eta = param[0], radius in coord row 3,
                                     src/H2Pack_3D_kernels.h:893-959, :1310-1430 */

/* Arithmetic of the apply */
#define H2GPU_PREC_FP64   0       /* plain drop-in: every product and sum in FP64       */
#define H2GPU_PREC_MIXED  1       /* FP32 blocks / FP32 re-centred kernel evaluation,
                                     FP32 sums inside one block, FP64 across blocks     */

/* Matrix layouts of h2gpu_matmul (numerically equal to CBLAS_LAYOUT) */
#define H2GPU_ROW_MAJOR 101
#define H2GPU_COL_MAJOR 102

/*
 * Plain-pointer view of one H2 representation.  Every field has the meaning of
 * the struct H2Pack field of the same name (src/H2Pack_typedef.h:88-205); arrays
 * are read during h2gpu_image_create only and may be freed afterwards.
 */
typedef struct h2gpu_desc
{
    int n_point;            /* number of points                                    */
    int pt_dim;             /* point dimension (3)                                 */
    int xpt_dim;            /* coordinate rows (4 for RPY: x, y, z, radius)        */
    int krnl_dim;           /* kernel block dimension (1, or 3 for RPY)            */
    int n_node;
    int n_leaf_node;
    int max_child;          /* 2^pt_dim                                            */
    int max_level;
    int min_adm_level;      /* H2 mode value (HSS mode is rejected)                */
    int BD_JIT;             /* 1: B and D are evaluated on the fly                 */

    const int *n_child;     /* [n_node]                                            */
    const int *children;    /* [n_node * max_child]                                */
    const int *node_level;  /* [n_node]                                            */
    const int *pt_cluster;  /* [2 * n_node] first and last (inclusive) point       */
    const int *mat_cluster; /* [2 * n_node] first and last (inclusive) vector row  */
    const int *level_n_node;/* [max_level + 1]                                     */
    const int *level_nodes; /* [(max_level + 1) * n_leaf_node]                     */
    const int *leaf_nodes;  /* [n_leaf_node] = height_nodes row 0: order of the
                               diagonal D blocks (src/H2Pack_build.c:948-968)       */

    const int *U_nrow;      /* [n_node]                                            */
    const int *U_ncol;      /* [n_node]                                            */
    const int *U_ld;        /* [n_node] row stride of U[i] (>= U_ncol[i])          */
    const double *const *U; /* [n_node] row-major U[i]; NULL when empty            */

    int n_r_adm_pair;
    const int *r_adm_pairs;   /* [2 * n_r_adm_pair]                                */
    int n_r_inadm_pair;
    const int *r_inadm_pairs; /* [2 * n_r_inadm_pair]                              */

    int n_B;                  /* == n_r_adm_pair                                    */
    const int *B_nrow;        /* [n_B]                                              */
    const int *B_ncol;        /* [n_B]                                              */
    const size_t *B_ptr;      /* [n_B + 1] element offsets into B_data              */
    const double *B_data;     /* AOT only (NULL when BD_JIT)                        */
    int n_D;                  /* == n_leaf_node + n_r_inadm_pair                    */
    const int *D_nrow;
    const int *D_ncol;
    const size_t *D_ptr;
    const double *D_data;     /* AOT only                                           */

    const double *coord;      /* [xpt_dim * n_point], row d at coord + d * n_point,
                                 points in H2Pack's sorted order                    */
    const int *J_n;           /* [n_node] skeleton point counts                     */
    const double *const *J_coord; /* [n_node] xpt_dim x J_n[i], ld = J_n[i]        */

    const int *fwd_pmt_idx;   /* [krnl_dim * n_point]                               */
    const int *bwd_pmt_idx;   /* [krnl_dim * n_point]                               */

    int kernel_id;            /* H2GPU_KRNL_*; required when BD_JIT                 */
    int n_krnl_param;         /* 0 .. 4                                             */
    double krnl_param[4];
} h2gpu_desc;

/* Where the stored B / D blocks of an image come from (h2gpu_options.blocks) */
#define H2GPU_BLOCKS_GIVEN    0   /* AOT descriptors: uploaded from B_data / D_data;
                                     JIT descriptors: evaluated on the fly (default)  */
#define H2GPU_BLOCKS_GENERATE 1   /* stored blocks generated on the device from the kernel,
                                     the coordinates and the skeleton points, in H2Pack's
                                     packing (B_ptr / D_ptr): what H2P_build_B_AOT and
                                     H2P_build_D_AOT compute (src/H2Pack_build.c:789-889,
                                     :1034-1140); B_data / D_data are not read, so a
                                     descriptor of a handle built with BD_JIT = 1 works.
                                     The arena is FP64 for an FP64 image and FP32 only
                                     for a mixed one (such an image refuses FP64 applies). */

/* Options of an image */
typedef struct h2gpu_options
{
    int precision;      /* H2GPU_PREC_FP64 or H2GPU_PREC_MIXED                        */
    int max_n_vec;      /* widest right-hand-side panel per pass, <= 64 (default 64;
                           mixed stored-block images take 32 / 64, others up to 16)   */
    int device;         /* CUDA device ordinal (default: current device)              */
    int blocks;         /* H2GPU_BLOCKS_GIVEN (default) or H2GPU_BLOCKS_GENERATE      */
} h2gpu_options;

typedef struct h2gpu_image h2gpu_image;

/* Phase statistics, accumulated over calls (the reference's timers[] and
 * mat_size[] plus the device-side view). */
typedef struct h2gpu_stats
{
    long long n_matvec;       /* right-hand sides applied (src/H2Pack_matvec.c:1283)  */
    double ms_total;          /* device time of all applies                           */
    double ms_phase[5];       /* gather/up, B, down, D, assemble (device events)      */
    double bytes_U;           /* U bytes read by one upward + one downward sweep       */
    double bytes_B;           /* stored B bytes (AOT)                                  */
    double bytes_D;           /* stored D bytes (AOT)                                  */
    double ref_mv_bytes;      /* 8*(mat_size[MV_FWD]+[MV_MID]+[MV_BWD]+[MV_DEN]) model */
    double jit_pairs_B;       /* kernel evaluations of the B phase per RHS panel       */
    double jit_pairs_D;       /* kernel evaluations of the D phase per RHS panel       */
    long long n_tasks_B, n_tasks_D;
    long long device_bytes;   /* device memory held by the image                      */
    long long n_launches;     /* kernels launched by all applies so far               */
} h2gpu_stats;

int  h2gpu_abi_version(void);
const char *h2gpu_last_error(void);
void h2gpu_default_options(h2gpu_options *opt);

int h2gpu_image_create(const h2gpu_desc *desc, const h2gpu_options *opt, h2gpu_image **out);
int h2gpu_image_destroy(h2gpu_image *img);
int h2gpu_set_precision(h2gpu_image *img, int precision);

/* y := A x with host vectors in the caller's original point order. */
int h2gpu_matvec(h2gpu_image *img, const double *x, double *y);

/* Y := A X, n_vec right-hand sides, host matrices, CBLAS-style layout. */
int h2gpu_matmul(h2gpu_image *img, int layout, int n_vec,
                 const double *X, int ldx, double *Y, int ldy);

/* Device-resident forms: X and Y are device pointers, row-major
 * (krnl_mat_size x n_vec, leading dimensions ldx / ldy >= n_vec), original
 * order; stream is a cudaStream_t or NULL for the image's own stream. */
int h2gpu_matmul_device(h2gpu_image *img, int n_vec, const double *dX, int ldx,
                        double *dY, int ldy, void *stream);

/* Permutations between the caller's order and H2Pack's sorted order, on host data. */
int h2gpu_permute_vector(h2gpu_image *img, int forward, const double *x, double *px);
int h2gpu_permute_matrix_rows(h2gpu_image *img, int forward, int layout, int n_vec,
                              const double *X, int ldx, double *PX, int ldp);

/*
 * y := A x for one device-resident vector (original order) without allocating:
 * no cudaMalloc, cudaFree or allocating library routine is called.  No counterpart
 * in the reference.  It is for callers that cannot allocate device memory when they
 * apply the matrix -- code whose device memory is owned by another allocator (a
 * framework's caching allocator or a pool reserved up front, where cudaMalloc fails
 * or fragments memory) and code that must not stall on cudaMalloc / cudaFree, which
 * synchronize the device.  The image is created beforehand.  Work buffers come from
 * a fixed 16 MiB device array in the library (held by every GPU that loads it);
 * images needing more work space for one right-hand side are rejected with
 * H2GPU_ERR_INVALID.  Calls share that array, so calls that overlap on the GPU race;
 * the first call on a device looks up the array's address and should come before
 * any stream capture.  A mixed-precision image is refused with H2GPU_ERR_STATE until
 * one allocating apply (h2gpu_matvec / h2gpu_matmul / h2gpu_matmul_device) has made
 * its FP32 copies of U, B and D; FP64 images need no such call.  The caller's current
 * device is restored before returning.  stream: a cudaStream_t or NULL for the
 * image's own stream.
 */
int h2gpu_matvec_device_noalloc(h2gpu_image *img, const double *d_x, double *d_y, void *stream);

/*
 * Batched form: one image for n_desc independent representations with the same
 * kernel, kernel parameters, krnl_dim and mode.  Every phase runs as one launch per
 * tree level over all of them (flattened cross-matrix task lists).  Vectors of the
 * batch are the members' vectors stacked in order (rows sum of krnl_dim * n_point).
 * No counterpart in the reference (its callers loop over handles).
 */
int h2gpu_batch_create(const h2gpu_desc *descs, int n_desc, const h2gpu_options *opt, h2gpu_image **out);

/*
 * Capture the device-resident apply of n_vec right-hand sides (dX -> dY, row-major,
 * fixed pointers) in a CUDA graph, and replay it on a stream (NULL: the image's).
 * No counterpart in the reference.
 */
int h2gpu_graph_capture(h2gpu_image *img, int n_vec, const double *dX, int ldx, double *dY, int ldy);
int h2gpu_graph_launch(h2gpu_image *img, void *stream);

/*
 * Autotuner: time the device apply of n_vec right-hand sides for each candidate
 * panel width and, for FP32 images, each kernel variant (h2gpu_set_jit_variant), and
 * keep the fastest for this image.  dY is overwritten.  *best_variant receives
 * H2GPU_JIT_SIMT (CUDA cores), H2GPU_JIT_TC (tensor cores, every target evaluates
 * its own sources) or H2GPU_JIT_PAIR (tensor cores, each unordered pair of leaves /
 * nodes evaluated once and applied in both directions).  No counterpart in the
 * reference.
 */
#define H2GPU_JIT_SIMT 0
#define H2GPU_JIT_TC   1
#define H2GPU_JIT_PAIR 2
#define H2GPU_BLK_TCGEN05 3   /* stored-block images: block products on tcgen05 (BF16x3 pieces, TMEM accumulators) */
int h2gpu_autotune(h2gpu_image *img, int n_vec, const double *dX, int ldx, double *dY, int ldy,
                   int *best_nv, int *best_variant);

/*
 * Select the kernel variant used by FP32 panels: for JIT images H2GPU_JIT_SIMT,
 * H2GPU_JIT_TC (default) or H2GPU_JIT_PAIR (needs a scalar kernel; panels of 8 or
 * 16 right-hand sides, others use H2GPU_JIT_TC); for stored-block images
 * H2GPU_JIT_TC (default: block products of panels of 8 or 16 on the tensor cores with
 * warp-level MMAs, 3xTF32), H2GPU_BLK_TCGEN05 (the same on tcgen05: values split into
 * three BF16 pieces, six products kept, accumulators in tensor memory) or
 * H2GPU_JIT_SIMT (CUDA cores).  FP64 panels always use the CUDA cores; a captured
 * graph keeps the variant it was captured with.  No counterpart in the reference.
 */
int h2gpu_set_jit_variant(h2gpu_image *img, int variant);

/*
 * Lock-step conjugate gradients on (K + mu I) for up to 16 requests ("slots") of one
 * image, on the device.  Each PCG slot runs H2Pack's left-preconditioned CG with the
 * identity preconditioner (examples/PCG/pcg.c:11-152) on the shifted operator of
 * examples/SPDHSS-H2/pcg_tests.c:13-20, with FP64 vectors and inner products and
 * the operator in the image's precision at h2gpu_cg_create; a MATVEC slot computes
 * (K + mu I) b once.  All 16 slots are the columns of one panel, so each iteration
 * is one H2 matmul plus five small kernels, enqueued on the image's stream; the host
 * reads the slot records with h2gpu_cg_sync once per batch of iterations.
 *
 * A slot whose recursive residual reaches tol ||b|| (or max_iter, or, for a mixed
 * operator, `refresh` iterations since its last restart) enters H2GPU_CG_CHECK;
 * h2gpu_cg_check recomputes b - (K + mu I) x with the FP64 operator and the slot
 * either finishes (H2GPU_CG_DONE; relres is then the true relative residual) or
 * restarts CG from that residual.  Reductions have a fixed order and columns are
 * independent.  d_b / d_x are device vectors of krnl_dim * n_point doubles in the
 * caller's (original) order; the caller orders its own writes of d_b before
 * h2gpu_cg_admit.  One engine per image (it uses the image's work buffers and
 * stream).  No counterpart in the reference (pcg.c runs one vector on the host).
 */
typedef struct h2gpu_cg h2gpu_cg;
#define H2GPU_CG_FREE   0
#define H2GPU_CG_RUN    1
#define H2GPU_CG_CHECK  2
#define H2GPU_CG_DONE   3
#define H2GPU_CG_MATVEC 0
#define H2GPU_CG_PCG    1
int h2gpu_cg_create(h2gpu_image *img, double mu, int refresh, h2gpu_cg **out);
int h2gpu_cg_destroy(h2gpu_cg *cg);
int h2gpu_cg_admit(h2gpu_cg *cg, int slot, int kind, const double *d_b, double tol, int max_iter);
int h2gpu_cg_step(h2gpu_cg *cg, int n_iter);
int h2gpu_cg_check(h2gpu_cg *cg);
int h2gpu_cg_sync(h2gpu_cg *cg, int *state, int *iters, double *relres);   /* 16 entries each */
/* 1 when the work of the last h2gpu_cg_step / h2gpu_cg_check has finished on the device,
 * 0 while it runs (no waiting): a scheduler polls its engines and collects each one as
 * soon as it is done, so engines of small and large matrices do not wait for each other. */
int h2gpu_cg_query(h2gpu_cg *cg);
/* Free a slot whatever its state (a request given up, e.g. past its deadline); work
 * already enqueued finishes first, then the slot may be admitted again. */
int h2gpu_cg_cancel(h2gpu_cg *cg, int slot);
int h2gpu_cg_take(h2gpu_cg *cg, int slot, double *d_x);
int h2gpu_cg_history(h2gpu_cg *cg, int slot, double *out, int max_n);      /* ||r|| per iteration; returns count */

/*
 * Copy the image's stored blocks (which = 0: B, 1: D) to host memory as doubles, in
 * H2Pack's packing (element B_ptr[i] / D_ptr[i] starts block i); n_elems must be the
 * total (B_ptr[n_B] / D_ptr[n_D]).  An image holding FP32 blocks only returns them
 * widened.  For checking generated blocks against H2P_build_B_AOT / H2P_build_D_AOT;
 * no counterpart in the reference.
 */
int h2gpu_get_blocks(h2gpu_image *img, int which, double *host, size_t n_elems);

int h2gpu_get_stats(h2gpu_image *img, h2gpu_stats *st);
int h2gpu_reset_stats(h2gpu_image *img);
size_t h2gpu_image_bytes(const h2gpu_image *img);

/*
 * Host-only self-check of the apply plan: builds the plan h2gpu_image_create would
 * upload for desc (no device is touched, no GPU is needed) and verifies that
 *   - the upward tasks sweep every column of every node's U once and the downward
 *     tasks every row at most once, inside the node's U; the stored-block tasks
 *     cover every row of every B / D block once;
 *   - every partial-space row is written by one producer and summed by one
 *     consumer, every push-down / y1 row a downward task reads is written, and the
 *     assembly writes every output row once (for each plan an image holds);
 *   - JIT: every target's source sets are exactly those H2Pack's pair lists name
 *     for its node (near: the leaf itself and its inadmissible partners; far: the
 *     admissible partners, skeleton or leaf points as the levels say), the point
 *     pairs total what the lists imply, the source tiles and 8-point panel groups
 *     cover every source set once
 *     in order, and the pair plan (scalar kernels) owns every unordered pair once;
 *   - every index a kernel takes from a task record (block offsets, input rows, point
 *     ranges) lies inside the array it indexes (kernels do not bounds-check them).
 * counts (H2GPU_PLAN_COUNTS entries, may be NULL): upward tasks, downward tasks,
 * stored-block tasks, JIT target chunks, source tiles, panel groups, partial-space
 * rows, JIT point pairs evaluated per right-hand side.  Returns H2GPU_OK or
 * H2GPU_ERR_INVALID naming the first violated invariant in h2gpu_last_error().
 */
#define H2GPU_PLAN_COUNTS 8
int h2gpu_plan_check(const h2gpu_desc *desc, long long *counts);
/* The same for the merged representation h2gpu_batch_create would build from descs. */
int h2gpu_batch_plan_check(const h2gpu_desc *descs, int n_desc, long long *counts);

/*
 * Measured pipe peaks of a device (-1: the current one), the denominators of the JIT
 * kernels' roofline: FP32 FMA throughput (TFLOP/s, packed FP32x2 FMA chains on every SM)
 * and MUFU throughput (10^12 ex2.approx operations/s).  No counterpart in the reference.
 */
int h2gpu_measure_peaks(int device, double *fp32_tflops, double *mufu_tops);

/*
 * FP64 direct sum on the device: y_t = sum_s K(x_t, x_s) v_s for n_trg targets
 * and n_src sources (coordinates xpt_dim x n, ld = n, host arrays; values are
 * krnl_dim-interleaved per point as in the H2 vectors).
 */
int h2gpu_direct_sum(int kernel_id, const double *krnl_param, int n_krnl_param,
                     int xpt_dim, int krnl_dim,
                     const double *src_coord, int n_src, const double *src_val,
                     const double *trg_coord, int n_trg, double *trg_val);

/*
 * Interpolative decompositions of a batch of kernel blocks on the device: the
 * construction step of the projection matrices for scalar kernels
 * (H2P_build_H2_UJ_proxy, src/H2Pack_build.c:32-270, its per-node
 * H2P_ID_compress, src/H2Pack_ID_compress.c:491-576).  Block b is the kernel
 * matrix of ncand[b] candidate points (3 x ncand[b], dim-major, blocks one after the
 * other in cand) against the npp proxy points (3 x npp, dim-major) of one level:
 * A_b[i][j] = K(c_i, p_j).  A_b^T is factored by column-pivoted Householder QR with
 * H2Pack's relative-norm stopping rule at reltol (H2P_partial_pivot_QR,
 * src/H2Pack_ID_compress.c:51-189), and E_b = R11^-1 R12 is formed.  Outputs:
 * rank[b]; perm (sum of ncand, blocks one after the other): the column order of the
 * QR, whose first rank[b] entries are the skeleton candidates; *E: a buffer allocated
 * here (release with h2gpu_free) holding E_b (rank x (ncand - rank), column-major,
 * ld = rank) from element e_off[b] (e_off has n_blk + 1 entries); with E = NULL only
 * rank and perm are computed (e_off unused).  Each block takes one CTA, except
 * blocks whose work space exceeds a CTA's shared memory and blocks of at least 2^20
 * entries in a batch with fewer than 64 of them: those are decomposed one at a time
 * over the whole GPU (two launches per pivot step), with the same arithmetic.  Pivot
 * choices can differ from the CPU's where two downdated column norms agree to
 * rounding, so skeletons match the reference's in accuracy, not always index by
 * index.  No counterpart beyond H2Pack's internal function.
 */
int h2gpu_id_batch(int kernel_id, const double *krnl_param, int n_krnl_param, double reltol, int n_blk,
                   const int *ncand, int npp, const double *cand, const double *prox, int *rank, int *perm,
                   double **E, long long *e_off);

/* Release a buffer allocated by the library (h2gpu_id_batch). */
void h2gpu_free(void *p);

/*
 * The candidate reduction of proxy-point generation on the device
 * (H2P_generate_proxy_point_nlayer, src/H2Pack_gen_proxy_point.c:106-159): the
 * sketch W = K(X0, Y0) S of nx candidate points X0 against ny outer points Y0 (both
 * 3 x n, dim-major), S given as S^T in CSR (nx rows: st_rowptr[nx + 1], st_col,
 * st_val; H2P_gen_rand_sparse_mat_trans's output), followed by the interpolative
 * decomposition of W's rows at reltol (as h2gpu_id_batch, skeletons only, over the
 * whole GPU): rank and
 * perm (nx; the first rank entries are the selected candidates).
 */
int h2gpu_pp_sketch_id(int kernel_id, const double *krnl_param, int n_krnl_param, double reltol, int nx,
                       const double *X0, int ny, const double *Y0, const int *st_rowptr, const int *st_col,
                       const double *st_val, int *rank, int *perm);

/* ------------------------------------------------------------------ HSS ULV solve
 *
 * The ULV factors of an HSS-mode matrix (H2P_HSS_ULV_Cholesky_factorize,
 * src/H2Pack_HSS_ULV.c:601-979, or H2P_HSS_ULV_LU_factorize, :16-427; the handle's
 * ULV_Ls / ULV_idx / ULV_p / ULV_Q / ULV_L, src/H2Pack_typedef.h:153-191) uploaded to
 * the device, and the ULV solve there (replaces H2P_HSS_ULV_Cholesky_solve, :981-1159,
 * and H2P_HSS_ULV_LU_solve, :429-599).  All descriptor arrays are host memory, read
 * during h2gpu_ulv_create only.  Per node i (every node of levels 0 .. max_level):
 *   Ls[i]               ULV_Ls[i];
 *   m[i], idx[i]        ULV_idx[i]: m[i] indices into the permuted vector;
 *   q_ncol[i], Q[i]     ULV_Q[i]: (m[i] + 1) x q_ncol[i] row-major (ld q_ncol[i]): the
 *                       Householder vectors of a row-major GEQRF below the diagonal and
 *                       tau in the last row; ignored at the root (level 0);
 *   L[i], l_ld[i]       ULV_L[i]: m[i] x m[i] row-major;
 *   p[i]                LU only: ULV_p[i], m[i] - Ls[i] entries.
 * The device keeps each node's explicit Q (formed from the reflectors at create) and
 * L, both m x m, and runs one launch per tree level per sweep (one CTA per node, the
 * node's vector in shared memory: nodes of more than 13,872 rows are refused with
 * H2GPU_ERR_UNSUPPORTED).
 */
typedef struct h2gpu_ulv h2gpu_ulv;

typedef struct h2gpu_ulv_desc
{
    int lu;                        /* 0: Cholesky factors, 1: LU factors              */
    int n_node, max_level, n_leaf_node, krnl_mat_size;
    const int *level_n_node;       /* max_level + 1                                   */
    const int *level_nodes;        /* (max_level + 1) x n_leaf_node; level 0 = root   */
    const int *fwd_pmt_idx;        /* krnl_mat_size: permuted[i] = b[fwd_pmt_idx[i]]  */
    const int *bwd_pmt_idx;        /* krnl_mat_size: x[i] = permuted[bwd_pmt_idx[i]]  */
    const int *Ls, *m, *q_ncol, *l_ld;          /* n_node each                        */
    const int *const *idx;                      /* n_node pointers                    */
    const double *const *Q, *const *L;          /* n_node pointers                    */
    const int *const *p;                        /* n_node pointers (LU), else NULL    */
    int device;                    /* CUDA device ordinal, -1: current device         */
} h2gpu_ulv_desc;

int h2gpu_ulv_create(const h2gpu_ulv_desc *desc, h2gpu_ulv **out);
int h2gpu_ulv_destroy(h2gpu_ulv *u);
/* x = the ULV solve of b, as the reference's op: 1 the first sweep (Cholesky: L^-1;
   LU: U^-1 part, levels max_level .. 0), 2 the second (Cholesky: L^-T; LU: L^-1
   part), 3 both (the solve with the factored matrix).  Host arrays of krnl_mat_size. */
int h2gpu_ulv_solve(h2gpu_ulv *u, int op, const double *b, double *x);
/* The same on device arrays, enqueued on `stream` (a cudaStream_t; NULL: the
   library's stream of this factorization); returns once enqueued.  Every solve of one
   h2gpu_ulv works in that object's permuted-vector buffer, so solves of one object
   must not overlap on the device (enqueue them on one stream; the drop-in serialises
   per handle); different objects are independent. */
int h2gpu_ulv_solve_device(h2gpu_ulv *u, int op, const double *d_b, double *d_x, void *stream);
size_t h2gpu_ulv_bytes(const h2gpu_ulv *u);

#ifdef __cplusplus
}
#endif

#endif
