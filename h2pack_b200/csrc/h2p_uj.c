/*
 * h2p_uj.c -- the projection matrices of H2Pack's construction on the GPU.
 *
 * H2Pack builds U and the skeleton sets J node by node, bottom-up
 * (H2P_build_H2_UJ_proxy, src/H2Pack_build.c:32-270): the candidate points of a
 * node (its points for a leaf, the union of its children's skeletons otherwise),
 * shifted to the node's box center, against its level's proxy points give a kernel
 * matrix A; an interpolative decomposition of A's rows (H2P_ID_compress,
 * src/H2Pack_ID_compress.c:491-576: column-pivoted QR of A^T with the relative-norm
 * stop at QR_stop_tol, then E = R11^-1 R12) picks the skeleton rows J and gives
 * U = P [I; E^T].
 *
 * This file replaces that function inside libH2Pack_gpu.so.  With the GPU path on
 * (H2P_gpu_build_uj(1), or H2GPU_BUILD_UJ=1 in the environment) every level's nodes
 * go to the device in one batch (h2gpu_id_batch: kernel matrices, pivoted QR and the
 * triangular solve, one CTA per node) and U / J / J_coord are assembled here in
 * H2Pack's own structures, exactly as H2P_ID_compress and the build loop assemble
 * them from the QR's output.  Scalar kernels only (Coulomb, Gaussian, Matern 3/2,
 * identified from the handle's kernel function), relative-norm stop, 3-D points;
 * everything else, and the default, runs H2Pack's own function (compiled under the
 * name H2P_build_H2_UJ_proxy_host).  Pivot choices can differ from the CPU's where
 * two column norms agree to rounding, so the skeletons match H2Pack's in accuracy,
 * not index by index.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "H2Pack.h"
#include "H2Pack_utils.h"
#include "h2gpu.h"

#define DROPIN_API __attribute__((visibility("default")))

void H2P_build_H2_UJ_proxy_host(H2Pack_p h2pack);
int h2p_identify_kernel(H2Pack_p h, int *kid, double *param, int *n_param);

static int g_uj_gpu = -1;   /* -1: read H2GPU_BUILD_UJ once */
static int g_uj_built = 0;  /* handles whose U / J the device computed */

/* Switch the GPU construction of U / J on (1) or off (0) for later H2P_build calls. */
DROPIN_API void H2P_gpu_build_uj(int on) { g_uj_gpu = on ? 1 : 0; }

/* How many H2P_build calls so far had their U / J computed on the device. */
DROPIN_API int H2P_gpu_build_uj_count(void) { return g_uj_built; }

static int h2p_uj_gpu_enabled(void)
{
    if (g_uj_gpu < 0)
    {
        const char *e = getenv("H2GPU_BUILD_UJ");
        g_uj_gpu = (e != NULL && e[0] == '1') ? 1 : 0;
    }
    return g_uj_gpu;
}

/* U, J and J_coord of one node from its QR output (the tail of H2P_ID_compress and
   step (6) of the build loop): perm = the QR's column order of the candidates, r the
   rank, E = R11^-1 R12 (r x (nc - r), column-major, ld = r). */
static void assemble_node(H2Pack_p h2pack, int node, int nc, int r, const int *perm, const double *E,
                          H2P_int_vec_p cand)
{
    H2P_dense_mat_p *U = h2pack->U, *J_coord = h2pack->J_coord;
    H2P_int_vec_p *J = h2pack->J;
    const int xpt_dim = h2pack->xpt_dim, n_point = h2pack->n_point;
    /* skeleton positions (into the candidate list), sorted, with their QR positions */
    int *sk = (int *) malloc(sizeof(int) * (nc > 0 ? nc : 1));
    int *p0 = (int *) malloc(sizeof(int) * (nc > 0 ? nc : 1) * 4);
    int *i0 = p0 + nc, *i1 = i0 + nc, *p1 = i1 + nc;
    for (int i = 0; i < nc; i++) { sk[i] = perm[i]; p0[perm[i]] = i; i0[i] = i; }
    if (r > 0) H2P_qsort_int_key_val(sk, i0, 0, r - 1);
    for (int i = 0; i < nc; i++) i1[i0[i]] = i;
    for (int i = 0; i < nc; i++) p1[i] = i1[p0[i]];
    /* U = rows permuted by p1 of [I_r; E^T with columns in sorted-skeleton order] */
    H2P_dense_mat_p Un;
    if (r == 0)
    {
        H2P_dense_mat_init(&Un, 1, 1);
        Un->nrow = nc;
        Un->ncol = 0;
        Un->ld = 0;
    } else {
        H2P_dense_mat_init(&Un, nc, r);
        for (int i = 0; i < r; i++)
        {
            memset(Un->data + (size_t) i * r, 0, sizeof(double) * r);
            Un->data[(size_t) i * r + i] = 1.0;
        }
        double *UL = Un->data + (size_t) r * r;
        for (int icol = 0; icol < r; icol++)
            for (int irow = 0; irow < nc - r; irow++)
                UL[(size_t) irow * r + icol] = E[(size_t) i0[icol] + (size_t) irow * r];
        H2P_dense_mat_permute_rows(Un, p1);
    }
    U[node] = Un;
    /* the node's skeleton points, their coordinates */
    H2P_int_vec_init(&J[node], 0);
    H2P_int_vec_set_capacity(J[node], r > 0 ? r : 1);
    for (int k = 0; k < r; k++) J[node]->data[k] = cand->data[sk[k]];
    J[node]->length = r;
    H2P_dense_mat_init(&J_coord[node], xpt_dim, r > 0 ? r : 1);
    J_coord[node]->ncol = r;
    J_coord[node]->ld = r;
    if (r > 0)
        H2P_gather_matrix_columns(h2pack->coord, n_point, J_coord[node]->data, r, xpt_dim, J[node]->data, r);
    free(sk);
    free(p0);
}

/* The GPU construction; returns 0, or nonzero with U / J / J_coord released (the
   caller then runs H2Pack's own function). */
static int build_uj_gpu(H2Pack_p h2pack, int kid, const double *param, int n_param)
{
    const int n_node = h2pack->n_node, n_point = h2pack->n_point, max_child = h2pack->max_child;
    const int pt_dim = h2pack->pt_dim;
    h2pack->n_UJ = n_node;
    h2pack->U = (H2P_dense_mat_p *) calloc(n_node, sizeof(H2P_dense_mat_p));
    h2pack->J = (H2P_int_vec_p *) calloc(n_node, sizeof(H2P_int_vec_p));
    h2pack->J_coord = (H2P_dense_mat_p *) calloc(n_node, sizeof(H2P_dense_mat_p));
    int st = (h2pack->U && h2pack->J && h2pack->J_coord) ? 0 : 1;
    for (int L = h2pack->max_level; L >= 0 && st == 0; L--)
    {
        const int nb = h2pack->level_n_node[L];
        const int *nodes = h2pack->level_nodes + (size_t) L * h2pack->n_leaf_node;
        H2P_dense_mat_p pp = h2pack->pp[L];
        const int npp = (pp != NULL) ? pp->ncol : 0;
        /* candidates of every node of the level, shifted to the node's box center */
        H2P_int_vec_p *cand = (H2P_int_vec_p *) calloc(nb > 0 ? nb : 1, sizeof(H2P_int_vec_p));
        int *ncand = (int *) malloc(sizeof(int) * (nb > 0 ? nb : 1));
        long long tot = 0;
        for (int b = 0; b < nb; b++)
        {
            const int node = nodes[b];
            if (h2pack->n_child[node] == 0)
            {
                const int s = h2pack->pt_cluster[2 * node], e = h2pack->pt_cluster[2 * node + 1];
                H2P_int_vec_init(&cand[b], 0);
                H2P_int_vec_set_capacity(cand[b], e - s + 1);
                for (int k = s; k <= e; k++) cand[b]->data[k - s] = k;
                cand[b]->length = e - s + 1;
            } else {
                int sz = 0;
                for (int c = 0; c < h2pack->n_child[node]; c++)
                    sz += h2pack->J[h2pack->children[(size_t) node * max_child + c]]->length;
                H2P_int_vec_init(&cand[b], 0);
                H2P_int_vec_set_capacity(cand[b], sz > 0 ? sz : 1);
                cand[b]->length = 0;
                for (int c = 0; c < h2pack->n_child[node]; c++)
                    H2P_int_vec_concatenate(cand[b], h2pack->J[h2pack->children[(size_t) node * max_child + c]]);
            }
            ncand[b] = cand[b]->length;
            tot += ncand[b];
        }
        double *cc = (double *) malloc(sizeof(double) * 3 * (tot > 0 ? tot : 1));
        double *prox = (double *) malloc(sizeof(double) * 3 * (npp > 0 ? npp : 1));
        int *perm = (int *) malloc(sizeof(int) * (tot > 0 ? tot : 1));
        int *rank = (int *) malloc(sizeof(int) * (nb > 0 ? nb : 1));
        long long *e_off = (long long *) malloc(sizeof(long long) * (nb + 1));
        double *E = NULL;
        long long o = 0;
        for (int b = 0; b < nb; b++)
        {
            const double *box = h2pack->enbox + (size_t) nodes[b] * 2 * pt_dim;
            for (int d = 0; d < 3; d++)
            {
                const double ctr = box[d] + 0.5 * box[pt_dim + d];
                for (int k = 0; k < ncand[b]; k++)
                    cc[3 * o + (size_t) d * ncand[b] + k] = h2pack->coord[(size_t) d * n_point + cand[b]->data[k]] - ctr;
            }
            o += ncand[b];
        }
        for (int d = 0; d < 3; d++)
            for (int j = 0; j < npp; j++) prox[(size_t) d * npp + j] = pp->data[(size_t) d * pp->ld + j];
        if (h2gpu_id_batch(kid, param, n_param, h2pack->QR_stop_tol, nb, ncand, npp, cc, prox, rank, perm, &E,
                           e_off) != H2GPU_OK)
        {
            fprintf(stderr, "H2Pack GPU construction of U / J: %s; building on the CPU\n", h2gpu_last_error());
            st = 1;
        } else {
            o = 0;
            for (int b = 0; b < nb; b++)
            {
                assemble_node(h2pack, nodes[b], ncand[b], rank[b], perm + o, E + e_off[b], cand[b]);
                o += ncand[b];
            }
        }
        h2gpu_free(E);
        for (int b = 0; b < nb; b++) H2P_int_vec_destroy(&cand[b]);
        free(cand); free(ncand); free(cc); free(prox); free(perm); free(rank); free(e_off);
    }
    if (st != 0)
    {
        for (int i = 0; i < n_node; i++)
        {
            if (h2pack->U && h2pack->U[i]) H2P_dense_mat_destroy(&h2pack->U[i]);
            if (h2pack->J && h2pack->J[i]) H2P_int_vec_destroy(&h2pack->J[i]);
            if (h2pack->J_coord && h2pack->J_coord[i]) H2P_dense_mat_destroy(&h2pack->J_coord[i]);
        }
        free(h2pack->U); free(h2pack->J); free(h2pack->J_coord);
        h2pack->U = NULL; h2pack->J = NULL; h2pack->J_coord = NULL;
        return st;
    }
    /* statistics, as the reference's step 3 */
    for (int i = 0; i < n_node; i++)
    {
        H2P_dense_mat_p Ui = h2pack->U[i];
        h2pack->mat_size[U_SIZE_IDX] += (size_t) Ui->nrow * Ui->ncol;
        h2pack->mat_size[MV_FWD_SIZE_IDX] += (size_t) Ui->nrow * Ui->ncol + Ui->nrow + Ui->ncol;
        h2pack->mat_size[MV_BWD_SIZE_IDX] += (size_t) Ui->nrow * Ui->ncol + Ui->nrow + Ui->ncol;
    }
    return 0;
}

/* Replaces H2Pack's function of this name (src/H2Pack_build.c:32), which H2P_build calls. */
DROPIN_API void H2P_build_H2_UJ_proxy(H2Pack_p h2pack)
{
    int kid = 0, n_param = 0;
    double param[4] = {0.0, 0.0, 0.0, 0.0};
    if (h2p_uj_gpu_enabled() && h2pack->krnl_dim == 1 && h2pack->pt_dim == 3 && h2pack->QR_stop_type == QR_REL_NRM &&
        h2p_identify_kernel(h2pack, &kid, param, &n_param) == H2GPU_OK && kid != H2GPU_KRNL_RPY &&
        build_uj_gpu(h2pack, kid, param, n_param) == 0)
    {
        __atomic_add_fetch(&g_uj_built, 1, __ATOMIC_RELAXED);
        return;
    }
    H2P_build_H2_UJ_proxy_host(h2pack);
}
