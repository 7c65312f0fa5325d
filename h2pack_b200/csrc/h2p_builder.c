/*
 * h2p_builder.c -- construction driver and plain-pointer description of an
 * H2Pack representation.
 *
 * Construction of the H2 representation is H2Pack's own CPU code, called
 * unchanged through its public API in the order its example drivers use
 * (examples/example_H2.c:47-88, examples/example_H2_RPY.c:47-108):
 *   H2P_init -> [H2P_run_RPY] -> H2P_calc_enclosing_box -> H2P_partition_points
 *   -> proxy points (numerical ID, src/H2Pack_gen_proxy_point.c:451, or box
 *      surface, :620) -> H2P_build (src/H2Pack_build.c:1143).
 * This file is compiled against the H2Pack headers; it is the piece a caller of
 * the GPU drop-in already has in some form (its own driver program).
 *
 * h2pb_describe() flattens the fields of struct H2Pack that the apply path reads
 * (src/H2Pack_typedef.h:88-205) into an h2gpu_desc of plain pointers.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#include "H2Pack.h"
#include "H2Pack_kernels.h"
#include "h2gpu.h"

#define H2PB_EXPORT __attribute__((visibility("default")))

typedef struct h2pb_handle
{
    H2Pack_p h2pack;
    DTYPE   *krnl_param;     /* owned; H2P_destroy does not free it (src/H2Pack_typedef.c) */
    int      n_krnl_param;
    H2P_dense_mat_p *pp;     /* owned; H2P_destroy leaves pp to the caller (src/H2Pack_typedef.c:272) */
    int      n_pp;
    int      kernel_id;
    double   build_sec;
    /* arrays behind every h2pb_describe() of this handle, newest first; each
       descriptor stays valid until h2pb_destroy */
    struct desc_store *descs;
} h2pb_handle;

typedef struct desc_store
{
    int *ints;
    const double **ptrs;
    struct desc_store *next;
} desc_store;

static int krnl_dim_of(int kernel_id) { return kernel_id == H2GPU_KRNL_RPY ? 3 : 1; }

static void select_kernel(int kernel_id, kernel_eval_fptr *ev, kernel_bimv_fptr *bimv, int *flops)
{
    switch (kernel_id)
    {
        case H2GPU_KRNL_COULOMB:
            *ev = Coulomb_3D_eval_intrin_t;  *bimv = Coulomb_3D_krnl_bimv_intrin_t;  *flops = Coulomb_3D_krnl_bimv_flop;  break;
        case H2GPU_KRNL_GAUSSIAN:
            *ev = Gaussian_3D_eval_intrin_t; *bimv = Gaussian_3D_krnl_bimv_intrin_t; *flops = Gaussian_3D_krnl_bimv_flop; break;
        case H2GPU_KRNL_MATERN32:
            *ev = Matern32_3D_eval_intrin_t; *bimv = Matern32_3D_krnl_bimv_intrin_t; *flops = Matern32_3D_krnl_bimv_flop; break;
        case H2GPU_KRNL_RPY:
            *ev = RPY_eval_std;              *bimv = RPY_krnl_bimv_intrin_t;         *flops = RPY_krnl_bimv_flop;         break;
        default:
            *ev = NULL; *bimv = NULL; *flops = 0;
    }
}

/*
 * Build an H2 representation.
 *   coord          : xpt_dim x n_point, row d at coord + d * n_point (xpt_dim = 4 for RPY)
 *   proxy_kind     : 0 numerical proxy points (ID), 1 proxy points on a box surface
 *   pp_fname       : proxy point cache file for proxy_kind 0 (may be NULL)
 *   use_bimv       : 1 pass the kernel's bi-matvec to H2P_build, 0 pass NULL
 *   n_thread       : OpenMP threads for the build (<= 0: OpenMP default)
 *   hss            : 1 build in HSS mode (H2P_run_HSS, examples/example_HSS.c:55)
 */
H2PB_EXPORT h2pb_handle *h2pb_build(
    int kernel_id, const double *param, int n_param,
    int n_point, const double *coord, double reltol,
    int max_leaf_points, double max_leaf_size, int BD_JIT,
    int proxy_kind, const char *pp_fname, int use_bimv, int n_thread, int hss)
{
    kernel_eval_fptr krnl_eval;
    kernel_bimv_fptr krnl_bimv;
    int bimv_flops;
    select_kernel(kernel_id, &krnl_eval, &krnl_bimv, &bimv_flops);
    if (krnl_eval == NULL || n_point <= 0 || coord == NULL || n_param < 0 || n_param > 4) return NULL;
    if (kernel_id != H2GPU_KRNL_COULOMB && n_param < 1) return NULL;
    if (n_thread > 0) omp_set_num_threads(n_thread);

    h2pb_handle *hd = (h2pb_handle *) calloc(1, sizeof(h2pb_handle));
    if (hd == NULL) return NULL;
    hd->kernel_id = kernel_id;
    hd->n_krnl_param = n_param;
    if (n_param > 0)
    {
        hd->krnl_param = (DTYPE *) malloc(sizeof(DTYPE) * 4);
        memset(hd->krnl_param, 0, sizeof(DTYPE) * 4);
        for (int i = 0; i < n_param; i++) hd->krnl_param[i] = param[i];
    }

    double st = omp_get_wtime();
    const int pt_dim = 3, krnl_dim = krnl_dim_of(kernel_id);
    DTYPE rel_tol = reltol;
    H2Pack_p h2pack;
    H2P_init(&h2pack, pt_dim, krnl_dim, QR_REL_NRM, &rel_tol);
    if (kernel_id == H2GPU_KRNL_RPY) H2P_run_RPY(h2pack);
    if (hss) H2P_run_HSS(h2pack);
    const int xpt_dim = h2pack->xpt_dim;

    H2P_calc_enclosing_box(pt_dim, n_point, coord, proxy_kind == 0 ? pp_fname : NULL, &h2pack->root_enbox);
    H2P_partition_points(h2pack, n_point, coord, max_leaf_points, max_leaf_size);

    H2P_dense_mat_p *pp = NULL;
    if (proxy_kind == 0)
    {
        H2P_generate_proxy_point_ID_file(h2pack, hd->krnl_param, krnl_eval, pp_fname, &pp);
    } else {
        /* Heuristic of examples/example_H2.c:69-76 */
        DTYPE max_L = h2pack->root_enbox[pt_dim];
        int num_pp_dim = (int) ceil(-log10(reltol));
        if (num_pp_dim < 4)  num_pp_dim = 4;
        if (num_pp_dim > 10) num_pp_dim = 10;
        int num_pp = 2 * pt_dim * num_pp_dim * num_pp_dim;
        /* xpt_dim rows so that RPY's radius row exists (zero-filled, src/H2Pack_gen_proxy_point.c:718-722) */
        H2P_generate_proxy_point_surface(pt_dim, xpt_dim, num_pp, h2pack->max_level,
                                         hss ? h2pack->HSS_min_adm_level : h2pack->min_adm_level, max_L, &pp);
    }
    hd->pp = pp;
    hd->n_pp = h2pack->max_level + 1;

    H2P_build(h2pack, pp, BD_JIT, hd->krnl_param, krnl_eval, use_bimv ? krnl_bimv : NULL, bimv_flops);
    hd->build_sec = omp_get_wtime() - st;
    /* H2P_build ends with BLAS_SET_NUM_THREADS(n_thread) (src/H2Pack_build.c:269), but
       the CPU matvec calls BLAS from inside its own OpenMP regions; with the pthreads
       OpenBLAS available here that nests thread pools, so BLAS is kept single-threaded
       as an OpenMP-built OpenBLAS would be inside a parallel region. */
    BLAS_SET_NUM_THREADS(1);
    hd->h2pack = h2pack;
    return hd;
}

H2PB_EXPORT H2Pack_p h2pb_h2pack(h2pb_handle *hd) { return hd ? hd->h2pack : NULL; }
H2PB_EXPORT double h2pb_build_seconds(h2pb_handle *hd) { return hd ? hd->build_sec : -1.0; }
H2PB_EXPORT int h2pb_kernel_id(h2pb_handle *hd) { return hd ? hd->kernel_id : 0; }
H2PB_EXPORT const double *h2pb_krnl_param(h2pb_handle *hd) { return hd ? hd->krnl_param : NULL; }
H2PB_EXPORT int h2pb_n_krnl_param(h2pb_handle *hd) { return hd ? hd->n_krnl_param : 0; }

H2PB_EXPORT void h2pb_destroy(h2pb_handle *hd)
{
    if (hd == NULL) return;
    if (hd->h2pack != NULL) H2P_destroy(&hd->h2pack);
    if (hd->pp != NULL)
    {
        for (int i = 0; i < hd->n_pp; i++) H2P_dense_mat_destroy(&hd->pp[i]);
        free(hd->pp);
    }
    free(hd->krnl_param);
    while (hd->descs != NULL)
    {
        desc_store *ds = hd->descs;
        hd->descs = ds->next;
        free(ds->ints);
        free((void *) ds->ptrs);
        free(ds);
    }
    free(hd);
}

/*
 * Integer summary of a built representation:
 *   out[0..15] = n_point, krnl_dim, xpt_dim, n_node, n_leaf_node, max_level,
 *                min_adm_level, n_r_adm_pair, n_r_inadm_pair, n_B, n_D, BD_JIT,
 *                krnl_mat_size, max_leaf_points, n_thread, mm_max_n_vec
 */
H2PB_EXPORT void h2pb_info(H2Pack_p h, long long *out)
{
    out[0] = h->n_point;  out[1] = h->krnl_dim;  out[2] = h->xpt_dim;  out[3] = h->n_node;
    out[4] = h->n_leaf_node;  out[5] = h->max_level;  out[6] = h->min_adm_level;
    out[7] = h->n_r_adm_pair;  out[8] = h->n_r_inadm_pair;  out[9] = h->n_B;  out[10] = h->n_D;
    out[11] = h->BD_JIT;  out[12] = h->krnl_mat_size;  out[13] = h->max_leaf_points;
    out[14] = h->n_thread;  out[15] = h->mm_max_n_vec;
}

/* Copies of the reference's statistics counters (src/H2Pack_typedef.h:200-204). */
H2PB_EXPORT void h2pb_counters(H2Pack_p h, double *mat_size11, double *timers11, double *jit_flops2, long long *n_matvec)
{
    for (int i = 0; i < 11; i++) { mat_size11[i] = (double) h->mat_size[i]; timers11[i] = h->timers[i]; }
    jit_flops2[0] = h->JIT_flops[0];
    jit_flops2[1] = h->JIT_flops[1];
    *n_matvec = h->n_matvec;
}

H2PB_EXPORT void h2pb_reset_timers(H2Pack_p h) { H2P_reset_timers(h); }

/* Sorted coordinates (xpt_dim x n_point) and the original index of each sorted point. */
H2PB_EXPORT const double *h2pb_coord(H2Pack_p h) { return h->coord; }
H2PB_EXPORT const int *h2pb_coord_idx(H2Pack_p h) { return h->coord_idx; }

/*
 * Fill an h2gpu_desc from struct H2Pack.  The per-node arrays U_nrow/U_ncol/U_ld/
 * J_n and the pointer tables are allocated into *ints_out / *ptrs_out, which the
 * caller frees with free() once the descriptor is no longer needed.
 */
H2PB_EXPORT int h2pb_describe_h2pack(H2Pack_p h, int kernel_id, const double *param, int n_param,
                                     h2gpu_desc *d, int **ints_out, const double ***ptrs_out)
{
    if (h == NULL || d == NULL) return H2GPU_ERR_INVALID;
    if (h->is_RPY_Ewald || h->is_H2ERI) return H2GPU_ERR_UNSUPPORTED;
    /* HSS mode applies the same phases over its own pair lists and minimum admissible
       level (src/H2Pack_matvec.c:101, :308, :773, :904) */
    const int hss = h->is_HSS;
    if (h->U == NULL || h->pt_cluster == NULL) return H2GPU_ERR_STATE;
    int n_node = h->n_node;
    int *ints = (int *) malloc(sizeof(int) * 4 * (size_t) n_node);
    const double **ptrs = (const double **) malloc(sizeof(double *) * 2 * (size_t) n_node);
    if (ints == NULL || ptrs == NULL) { free(ints); free(ptrs); return H2GPU_ERR_NOMEM; }
    int *U_nrow = ints, *U_ncol = ints + n_node, *U_ld = ints + 2 * n_node, *J_n = ints + 3 * n_node;
    const double **U = ptrs, **J_coord = ptrs + n_node;
    for (int i = 0; i < n_node; i++)
    {
        H2P_dense_mat_p Ui = h->U[i];
        U_nrow[i] = Ui ? Ui->nrow : 0;
        U_ncol[i] = Ui ? Ui->ncol : 0;
        U_ld[i]   = Ui ? Ui->ld   : 0;
        U[i] = (Ui && Ui->nrow > 0 && Ui->ncol > 0) ? Ui->data : NULL;
        H2P_dense_mat_p Ji = (h->J_coord != NULL) ? h->J_coord[i] : NULL;
        J_n[i] = Ji ? Ji->ncol : 0;
        J_coord[i] = (Ji && Ji->ncol > 0) ? Ji->data : NULL;
    }
    memset(d, 0, sizeof(*d));
    d->n_point = h->n_point;  d->pt_dim = h->pt_dim;  d->xpt_dim = h->xpt_dim;  d->krnl_dim = h->krnl_dim;
    d->n_node = n_node;  d->n_leaf_node = h->n_leaf_node;  d->max_child = h->max_child;
    d->max_level = h->max_level;  d->BD_JIT = h->BD_JIT;
    d->min_adm_level = hss ? h->HSS_min_adm_level : h->min_adm_level;
    d->n_child = h->n_child;  d->children = h->children;  d->node_level = h->node_level;
    d->pt_cluster = h->pt_cluster;  d->mat_cluster = h->mat_cluster;
    d->level_n_node = h->level_n_node;  d->level_nodes = h->level_nodes;
    d->leaf_nodes = h->height_nodes;
    d->U_nrow = U_nrow;  d->U_ncol = U_ncol;  d->U_ld = U_ld;  d->U = U;
    d->n_r_adm_pair = hss ? h->HSS_n_r_adm_pair : h->n_r_adm_pair;
    d->r_adm_pairs = hss ? h->HSS_r_adm_pairs : h->r_adm_pairs;
    d->n_r_inadm_pair = hss ? h->HSS_n_r_inadm_pair : h->n_r_inadm_pair;
    d->r_inadm_pairs = hss ? h->HSS_r_inadm_pairs : h->r_inadm_pairs;
    d->n_B = h->n_B;  d->B_nrow = h->B_nrow;  d->B_ncol = h->B_ncol;  d->B_ptr = h->B_ptr;  d->B_data = h->B_data;
    d->n_D = h->n_D;  d->D_nrow = h->D_nrow;  d->D_ncol = h->D_ncol;  d->D_ptr = h->D_ptr;  d->D_data = h->D_data;
    d->coord = h->coord;  d->J_n = J_n;  d->J_coord = J_coord;
    d->fwd_pmt_idx = h->fwd_pmt_idx;  d->bwd_pmt_idx = h->bwd_pmt_idx;
    d->kernel_id = kernel_id;
    d->n_krnl_param = n_param;
    for (int i = 0; i < n_param && i < 4; i++) d->krnl_param[i] = param[i];
    *ints_out = ints;
    *ptrs_out = ptrs;
    return H2GPU_OK;
}

/* Descriptor of a handle built by h2pb_build.  Its arrays are owned by the handle
   and stay valid until h2pb_destroy: every call gets storage of its own, so a caller
   may keep several descriptors of one handle (a batch listing a matrix twice, a
   descriptor kept across a plan check). */
H2PB_EXPORT int h2pb_describe(h2pb_handle *hd, h2gpu_desc *d)
{
    if (hd == NULL) return H2GPU_ERR_INVALID;
    desc_store *ds = (desc_store *) calloc(1, sizeof(desc_store));
    if (ds == NULL) return H2GPU_ERR_NOMEM;
    int st = h2pb_describe_h2pack(hd->h2pack, hd->kernel_id, hd->krnl_param, hd->n_krnl_param,
                                  d, &ds->ints, &ds->ptrs);
    if (st != H2GPU_OK) { free(ds); return st; }
    ds->next = hd->descs;
    hd->descs = ds;
    return H2GPU_OK;
}

/* The ULV factors of an HSS handle (after H2P_HSS_ULV_Cholesky_factorize, lu = 0, or
   H2P_HSS_ULV_LU_factorize, lu = 1) as an h2gpu_ulv_desc over the handle's own arrays
   (ULV_Ls / ULV_idx / ULV_p / ULV_Q / ULV_L, src/H2Pack_typedef.h:153-191).  *buf holds
   the descriptor's per-node tables; release it with h2pb_free after the last use of d.
   Returns H2GPU_ERR_STATE without factors of that kind. */
H2PB_EXPORT int h2pb_describe_ulv(H2Pack_p h, int lu, h2gpu_ulv_desc *d, void **buf)
{
    if (h == NULL || d == NULL || buf == NULL) return H2GPU_ERR_INVALID;
    *buf = NULL;
    if (!h->is_HSS || h->ULV_idx == NULL || h->ULV_L == NULL || h->ULV_Q == NULL || (lu && h->ULV_p == NULL))
        return H2GPU_ERR_STATE;
    const int n = h->n_node;
    char *mem = (char *) malloc(sizeof(int) * 4 * (size_t) n + sizeof(void *) * 4 * (size_t) n);
    if (mem == NULL) return H2GPU_ERR_NOMEM;
    const void **ptrs = (const void **) mem;
    int *ints = (int *) (mem + sizeof(void *) * 4 * (size_t) n);
    int *m = ints, *qn = ints + n, *ld = ints + 2 * n, *Ls = ints + 3 * n;
    const int **idx = (const int **) ptrs;
    const double **Q = (const double **) (ptrs + n), **L = (const double **) (ptrs + 2 * n);
    const int **p = (const int **) (ptrs + 3 * n);
    const int root = h->level_nodes[0];
    for (int i = 0; i < n; i++)
    {
        if (h->ULV_idx[i] == NULL || h->ULV_L[i] == NULL || h->ULV_Q[i] == NULL || (lu && h->ULV_p[i] == NULL))
        {
            free(mem);
            return H2GPU_ERR_STATE;
        }
        m[i] = h->ULV_idx[i]->length;
        Ls[i] = h->ULV_Ls[i];
        ld[i] = h->ULV_L[i]->ld;
        qn[i] = i == root ? 0 : h->ULV_Q[i]->ncol;
        idx[i] = h->ULV_idx[i]->data;
        L[i] = h->ULV_L[i]->data;
        Q[i] = i == root ? NULL : h->ULV_Q[i]->data;
        p[i] = lu ? h->ULV_p[i]->data : NULL;
    }
    memset(d, 0, sizeof(*d));
    d->lu = lu;
    d->n_node = n;
    d->max_level = h->max_level;
    d->n_leaf_node = h->n_leaf_node;
    d->krnl_mat_size = h->krnl_mat_size;
    d->level_n_node = h->level_n_node;
    d->level_nodes = h->level_nodes;
    d->fwd_pmt_idx = h->fwd_pmt_idx;
    d->bwd_pmt_idx = h->bwd_pmt_idx;
    d->Ls = Ls;
    d->m = m;
    d->q_ncol = qn;
    d->l_ld = ld;
    d->idx = idx;
    d->Q = Q;
    d->L = L;
    d->p = lu ? p : NULL;
    d->device = -1;
    *buf = mem;
    return H2GPU_OK;
}

H2PB_EXPORT void h2pb_free(void *p) { free(p); }
