/*
 * h2p_pp.c -- numerical proxy points of H2Pack's construction on the GPU.
 *
 * For every level H2Pack selects proxy points for a box [-L1/2, L1/2]^3 from random
 * candidates in the shells between L2 and L3 (H2P_generate_proxy_point_nlayer,
 * src/H2Pack_gen_proxy_point.c:56-330, algorithm 2, called per level by
 * H2P_generate_proxy_point_ID_file, :451-616):
 *   1. X0 = X0_size random points in the box, Y0 = n_layer shells of Y0_lsize random
 *      points each (the same random streams: srand(1924), srand48(1112), H2Pack's own
 *      generators, so the candidates are H2Pack's);
 *   2. the sketch K(X0, Y0) S with a sparse random S (H2Pack's generator), and an
 *      interpolative decomposition of its rows at reltol / 100: the skeleton Xp of X0;
 *   3. shell by shell: the rows of K([Yp, shell], Xp) decomposed at reltol / 100, the
 *      skeleton rows become the new Yp.
 * Steps 2 and 3 run on the device (h2gpu_pp_sketch_id, h2gpu_id_batch); the result
 * is Yp, H2Pack's output for reltol >= 1e-12.
 *
 * This file replaces that function inside libH2Pack_gpu.so when the device selection is
 * on (H2P_gpu_build_pp(1) or H2GPU_BUILD_PP=1): scalar kernels (identified from the
 * kernel function), 3-D, algorithm 2, reltol >= 1e-12.  Everything else, and the
 * default, runs H2Pack's own function (compiled under the name
 * H2P_generate_proxy_point_nlayer_host).  Each level's 2000 x 2000 sketch is decomposed
 * by the grid-wide QR (Matern-3/2 N = 250,000, no cache file: construction 5.93 ->
 * 4.86 s, 2.70 s with U / J on the device too).  It is opt-in because late pivots can
 * differ from the CPU's where two downdated column norms agree to rounding: the proxy
 * points then match H2Pack's in the accuracy they give, not point by point.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "H2Pack.h"
#include "H2Pack_utils.h"
#include "h2gpu.h"

#define DROPIN_API __attribute__((visibility("default")))

void H2P_generate_proxy_point_nlayer_host(const int pt_dim, const int krnl_dim, const DTYPE reltol,
                                          const void *krnl_param, kernel_eval_fptr krnl_eval, const DTYPE L1,
                                          const DTYPE L2, const DTYPE L3, const int alg, const int X0_size,
                                          const int Y0_lsize, const int max_layer, H2P_dense_mat_p pp,
                                          double *timers);
int h2p_identify_kernel_fn(kernel_eval_fptr krnl_eval, const void *krnl_param, int xd, int kd, int *kid,
                           double *param, int *n_param);

static int g_pp_gpu = -1;    /* -1: read H2GPU_BUILD_PP once */
static int g_pp_built = 0;   /* levels whose proxy points the device selected */

/* Switch the device selection of proxy points on (1) or off (0) for later calls. */
DROPIN_API void H2P_gpu_build_pp(int on) { g_pp_gpu = on ? 1 : 0; }

/* How many proxy-point levels so far were selected on the device. */
DROPIN_API int H2P_gpu_build_pp_count(void) { return g_pp_built; }

static int pp_gpu_enabled(void)
{
    if (g_pp_gpu < 0)
    {
        const char *e = getenv("H2GPU_BUILD_PP");
        g_pp_gpu = (e != NULL && e[0] == '1') ? 1 : 0;
    }
    return g_pp_gpu;
}

static int cmp_int(const void *a, const void *b)
{
    const int x = *(const int *) a, y = *(const int *) b;
    return (x > y) - (x < y);
}

/* columns idx[0 .. k-1] of a 3 x n dim-major set into a 3 x k one */
static void take_columns(const double *src, int n, const int *idx, int k, double *dst)
{
    for (int d = 0; d < 3; d++)
        for (int j = 0; j < k; j++) dst[(size_t) d * k + j] = src[(size_t) d * n + idx[j]];
}

static int proxy_gpu(int kid, const double *param, int n_param, DTYPE reltol, DTYPE L1, DTYPE L2, DTYPE L3,
                     int X0_size, int Y0_lsize, int max_layer, H2P_dense_mat_p pp)
{
    int n_layer = (int) round((L3 - L2) / L1);
    if (n_layer > max_layer) n_layer = max_layer;
    if (n_layer < 1) return 1;
    const int Y0_size = n_layer * Y0_lsize;
    int st = 0;
    double *X0 = (double *) malloc(sizeof(double) * 3 * X0_size);
    double *Y0 = (double *) malloc(sizeof(double) * 3 * (size_t) Y0_size);
    int *perm = (int *) malloc(sizeof(int) * (X0_size > Y0_lsize ? X0_size : Y0_lsize) * 2 + 16);
    H2P_dense_mat_p sval = NULL;
    H2P_int_vec_p sidx = NULL;
    double *Xp = NULL, *Yp = NULL, *tmp = NULL;
    int nxp = 0, nyp = 0;
    if (!X0 || !Y0 || !perm) { st = 1; goto done; }
    /* 1. candidates: H2Pack's random streams and generators, in its order */
    srand(1924);
    srand48(1112);
    H2P_gen_coord_in_ring(X0_size, 3, 0.0, L1, X0, X0_size);
    const DTYPE w = (L3 - L2) / (DTYPE) n_layer;
    for (int i = 0; i < n_layer; i++)
        H2P_gen_coord_in_ring(Y0_lsize, 3, L2 + w * (DTYPE) i, L2 + w * (DTYPE) (i + 1), Y0 + (size_t) i * Y0_lsize,
                              Y0_size);
    /* 2. sketch and its decomposition: the skeleton of X0 */
    H2P_dense_mat_init(&sval, 1, 1);
    H2P_int_vec_init(&sidx, 1);
    H2P_gen_rand_sparse_mat_trans(32, Y0_size, X0_size, sval, sidx);
    int r = 0;
    if (h2gpu_pp_sketch_id(kid, param, n_param, reltol * 1e-2, X0_size, X0, Y0_size, Y0, sidx->data,
                           sidx->data + X0_size + 1, sval->data, &r, perm) != H2GPU_OK)
    {
        st = 1;
        goto done;
    }
    qsort(perm, r, sizeof(int), cmp_int);
    nxp = r;
    Xp = (double *) malloc(sizeof(double) * 3 * (nxp > 0 ? nxp : 1));
    if (!Xp) { st = 1; goto done; }
    take_columns(X0, X0_size, perm, nxp, Xp);
    /* 3. shell by shell: the skeleton rows of K([Yp, shell], Xp) */
    tmp = (double *) malloc(sizeof(double) * 3 * ((size_t) Y0_lsize + Y0_size));
    Yp = (double *) malloc(sizeof(double) * 3 * ((size_t) Y0_lsize + Y0_size));
    if (!tmp || !Yp) { st = 1; goto done; }
    for (int i = 0; i < n_layer && st == 0; i++)
    {
        const int nt = nyp + Y0_lsize;
        for (int d = 0; d < 3; d++)
        {
            memcpy(tmp + (size_t) d * nt, Yp + (size_t) d * nyp, sizeof(double) * nyp);
            memcpy(tmp + (size_t) d * nt + nyp, Y0 + (size_t) d * Y0_size + (size_t) i * Y0_lsize,
                   sizeof(double) * Y0_lsize);
        }
        int *pt = (int *) malloc(sizeof(int) * nt);
        int rk = 0;
        if (!pt || h2gpu_id_batch(kid, param, n_param, reltol * 1e-2, 1, &nt, nxp, tmp, Xp, &rk, pt, NULL, NULL) !=
                       H2GPU_OK)
        {
            st = 1;
        } else {
            qsort(pt, rk, sizeof(int), cmp_int);
            take_columns(tmp, nt, pt, rk, Yp);
            nyp = rk;
        }
        free(pt);
    }
    if (st == 0)
    {
        H2P_dense_mat_resize(pp, 3, nyp);
        for (int d = 0; d < 3; d++)
            for (int j = 0; j < nyp; j++) pp->data[(size_t) d * pp->ld + j] = Yp[(size_t) d * nyp + j];
    }
done:
    if (st != 0) fprintf(stderr, "H2Pack GPU proxy points: %s; selecting on the CPU\n", h2gpu_last_error());
    if (sval) H2P_dense_mat_destroy(&sval);
    if (sidx) H2P_int_vec_destroy(&sidx);
    free(X0); free(Y0); free(perm); free(Xp); free(Yp); free(tmp);
    return st;
}

/* Replaces H2Pack's function of this name (src/H2Pack_gen_proxy_point.c:56), which
   H2P_generate_proxy_point_ID_file calls per level. */
DROPIN_API void H2P_generate_proxy_point_nlayer(const int pt_dim, const int krnl_dim, const DTYPE reltol,
                                                const void *krnl_param, kernel_eval_fptr krnl_eval, const DTYPE L1,
                                                const DTYPE L2, const DTYPE L3, const int alg, const int X0_size,
                                                const int Y0_lsize, const int max_layer, H2P_dense_mat_p pp,
                                                double *timers)
{
    int kid = 0, n_param = 0;
    double param[4] = {0.0, 0.0, 0.0, 0.0};
    if (pp_gpu_enabled() && pt_dim == 3 && krnl_dim == 1 && alg == 2 && reltol >= 1e-12 &&
        h2p_identify_kernel_fn(krnl_eval, krnl_param, 3, 1, &kid, param, &n_param) == H2GPU_OK &&
        kid != H2GPU_KRNL_RPY &&
        proxy_gpu(kid, param, n_param, reltol, L1, L2, L3, X0_size, Y0_lsize, max_layer, pp) == 0)
    {
        __atomic_add_fetch(&g_pp_built, 1, __ATOMIC_RELAXED);
        return;
    }
    H2P_generate_proxy_point_nlayer_host(pt_dim, krnl_dim, reltol, krnl_param, krnl_eval, L1, L2, L3, alg, X0_size,
                                         Y0_lsize, max_layer, pp, timers);
}
