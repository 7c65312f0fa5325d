/*
 * h2_oracle.c -- CPU restatement of H2Pack's H2 matvec / matmul apply path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the GPU engine:
 * it is called by tests/, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline leg, never by the product path.  It restates, in plain sequential
 * FP64 C over the plain-pointer h2gpu_desc view, the algorithm of the reference
 * files (paths within the H2Pack project):
 *
 *   h2o_matvec   H2P_matvec                 src/H2Pack_matvec.c:1162-1284
 *     permute    H2P_permute_vector_*       src/H2Pack_matvec.c:1149-1159, src/utils.c:124
 *     upward     H2P_matvec_fwd_transform   src/H2Pack_matvec.c:95-177
 *     B (AOT)    H2P_matvec_intmd_mult_AOT  src/H2Pack_matvec.c:303-437
 *     B (JIT)    H2P_matvec_intmd_mult_JIT  src/H2Pack_matvec.c:586-764 (krnl_eval + bi-GEMV form, :558-582)
 *     downward   H2P_matvec_bwd_transform   src/H2Pack_matvec.c:767-861
 *     D (AOT)    H2P_matvec_dense_mult_AOT  src/H2Pack_matvec.c:864-998
 *     D (JIT)    H2P_matvec_dense_mult_JIT  src/H2Pack_matvec.c:1002-1145
 *     bi-GEMV    CBLAS_BI_GEMV              src/H2Pack_matvec.c:26-65
 *   h2o_matmul   H2P_matmul                 src/H2Pack_matmul.c:455-583, per-node CSR
 *                traversal of B/D blocks     src/H2Pack_matmul.c:140-245, :353-418,
 *                block lookup                src/H2Pack_utils.c:330-451,
 *                CSR of pair -> block index  src/H2Pack_build.c:742-753, :1009-1021
 *   h2o_eval     kernel matrix evaluation   src/H2Pack_3D_kernels.h (Coulomb :50-161,
 *                Gaussian :167-268, Matern 3/2 :384-497, RPY :893-959)
 *   h2o_direct_sum  direct_nbody            examples/direct_nbody.h:2-54
 *   h2o_ulv_solve  H2P_HSS_ULV_Cholesky_solve src/H2Pack_HSS_ULV.c:981-1159 and
 *                H2P_HSS_ULV_LU_solve       src/H2Pack_HSS_ULV.c:429-599 over the
 *                plain h2gpu_ulv_desc view of the factors; Q applied from its
 *                Householder vectors as ORMQR does
 *
 * Parity of this restatement is pinned against the reference library itself
 * (built from the reference sources into oracle/_ref) by tests/test_oracle_pin.py.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "h2gpu.h"

#define H2O_EXPORT __attribute__((visibility("default")))

/* ---------------------------------------------------------------- kernels */

/* K(coordA[:, i], coordB[:, j]) blocks, krnl_dim rows/cols per point, written
 * mat[(kd*i + a) * ldm + kd*j + b] as krnl_eval does (src/H2Pack_typedef.h:25-29). */
H2O_EXPORT void h2o_eval(int kernel_id, const double *param, int n_param,
                         const double *cA, int ldA, int nA,
                         const double *cB, int ldB, int nB,
                         double *mat, int ldm)
{
    const double *xa = cA, *ya = cA + ldA, *za = cA + 2 * ldA;
    const double *xb = cB, *yb = cB + ldB, *zb = cB + 2 * ldB;
    if (kernel_id == H2GPU_KRNL_COULOMB)
    {
        const double diag = (n_param > 0) ? param[0] : 0.0;   /* src/H2Pack_3D_kernels.h:56 */
        for (int i = 0; i < nA; i++)
            for (int j = 0; j < nB; j++)
            {
                double dx = xa[i] - xb[j], dy = ya[i] - yb[j], dz = za[i] - zb[j];
                double r2 = dx * dx + dy * dy + dz * dz;
                mat[i * ldm + j] = (r2 == 0.0) ? diag : 1.0 / sqrt(r2);
            }
    } else if (kernel_id == H2GPU_KRNL_GAUSSIAN) {
        const double neg_l = -param[0];                          /* :173 */
        for (int i = 0; i < nA; i++)
            for (int j = 0; j < nB; j++)
            {
                double dx = xa[i] - xb[j], dy = ya[i] - yb[j], dz = za[i] - zb[j];
                double r2 = dx * dx + dy * dy + dz * dz;
                mat[i * ldm + j] = exp(neg_l * r2);
            }
    } else if (kernel_id == H2GPU_KRNL_MATERN32) {
        const double nsqrt3_l = -1.7320508075688772 * param[0];  /* :386, :392 */
        for (int i = 0; i < nA; i++)
            for (int j = 0; j < nB; j++)
            {
                double dx = xa[i] - xb[j], dy = ya[i] - yb[j], dz = za[i] - zb[j];
                double t = nsqrt3_l * sqrt(dx * dx + dy * dy + dz * dz);
                mat[i * ldm + j] = (1.0 - t) * exp(t);
            }
    } else if (kernel_id == H2GPU_KRNL_RPY) {
        const double *aa = cA + 3 * ldA, *ab = cB + 3 * ldB;
        const double C = 1.0 / (6.0 * M_PI * param[0]);          /* :900 */
        for (int i = 0; i < nA; i++)
            for (int j = 0; j < nB; j++)
            {
                double dx = xa[i] - xb[j], dy = ya[i] - yb[j], dz = za[i] - zb[j];
                double ta = aa[i], sa = ab[j];
                double r2 = dx * dx + dy * dy + dz * dz;
                double r = sqrt(r2);
                double inv_r = (r == 0.0) ? 0.0 : 1.0 / r;
                double inv_r2 = inv_r * inv_r;
                dx *= inv_r;  dy *= inv_r;  dz *= inv_r;
                double t1, t2;
                double ta_p_sa = ta + sa, ta_m_sa = ta - sa;
                if (r > ta_p_sa)                       /* well separated, :918-923 */
                {
                    double tmp0 = C * 0.75 * inv_r;
                    double tmp1 = (ta * ta + sa * sa) * inv_r2;
                    t1 = tmp0 * (1.0 + tmp1 / 3.0);
                    t2 = tmp0 * (1.0 - tmp1);
                } else if (r > fabs(ta_m_sa)) {        /* overlapping, :924-930 */
                    double tmp0 = ta_m_sa * ta_m_sa;
                    double tmp1 = (inv_r2 * inv_r * C) / (ta * sa * 32.0);
                    t1 = tmp0 + 3.0 * r2;
                    t1 = tmp1 * (16.0 * r2 * r * ta_p_sa - t1 * t1);
                    t2 = tmp0 - r2;
                    t2 = tmp1 * 3.0 * t2 * t2;
                } else {                               /* one inside the other, :931-934 */
                    t1 = C / (ta > sa ? ta : sa);
                    t2 = 0.0;
                }
                double *k = mat + 3 * i * ldm + 3 * j;
                double u[3] = {dx, dy, dz};
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        k[a * ldm + b] = t2 * u[a] * u[b] + (a == b ? t1 : 0.0);
            }
    }
}

/* ---------------------------------------------------------------- helpers */

/* out0 += A in0 and out1 += A^T in1 in one pass over A, restated from CBLAS_BI_GEMV */
static void bi_gemv(int nrow, int ncol, const double *A, int lda,
                    const double *in0, const double *in1, double *out0, double *out1)
{
    for (int i = 0; i < nrow; i++)
    {
        const double *a = A + (size_t) i * lda;
        double s = 0.0, w = in1[i];
        for (int j = 0; j < ncol; j++)
        {
            s += a[j] * in0[j];
            out1[j] += w * a[j];
        }
        out0[i] += s;
    }
}

static void gemv_n(int nrow, int ncol, const double *A, int lda, const double *x, double beta, double *y)
{
    for (int i = 0; i < nrow; i++)
    {
        const double *a = A + (size_t) i * lda;
        double s = 0.0;
        for (int j = 0; j < ncol; j++) s += a[j] * x[j];
        y[i] = (beta == 0.0) ? s : beta * y[i] + s;   /* BLAS: y is not read when beta == 0 */
    }
}

static void gemv_t(int nrow, int ncol, const double *A, int lda, const double *x, double beta, double *y)
{
    for (int j = 0; j < ncol; j++) y[j] = (beta == 0.0) ? 0.0 : y[j] * beta;   /* y not read when beta == 0 */
    for (int i = 0; i < nrow; i++)
    {
        const double *a = A + (size_t) i * lda;
        for (int j = 0; j < ncol; j++) y[j] += a[j] * x[i];
    }
}

/* Gather the xpt_dim x n points [s, s+n) of the sorted coordinates into a packed block. */
static void gather_pts(const h2gpu_desc *d, int s, int n, double *dst)
{
    for (int k = 0; k < d->xpt_dim; k++)
        memcpy(dst + (size_t) k * n, d->coord + (size_t) k * d->n_point + s, sizeof(double) * n);
}

static int node_npt(const h2gpu_desc *d, int node) { return d->pt_cluster[2 * node + 1] - d->pt_cluster[2 * node] + 1; }

/* Kernel block for an admissible pair (n0, n1) in JIT mode, restated from
 * H2P_get_Bij_block (src/H2Pack_utils.c:356-401).  Returns nrow x ncol in *mat. */
static void eval_B_block(const h2gpu_desc *d, int n0, int n1, double *mat, double *cbuf, int *nrow, int *ncol)
{
    int l0 = d->node_level[n0], l1 = d->node_level[n1], kd = d->krnl_dim;
    const double *cA, *cB;
    int nA, nB, ldA, ldB;
    if (l0 == l1 || l0 > l1) { cA = d->J_coord[n0]; nA = d->J_n[n0]; ldA = nA; }
    else { nA = node_npt(d, n0); gather_pts(d, d->pt_cluster[2 * n0], nA, cbuf); cA = cbuf; ldA = nA; }
    if (l0 == l1 || l0 < l1) { cB = d->J_coord[n1]; nB = d->J_n[n1]; ldB = nB; }
    else
    {
        nB = node_npt(d, n1);
        double *cb = cbuf + (size_t) d->xpt_dim * 4096;
        gather_pts(d, d->pt_cluster[2 * n1], nB, cb);
        cB = cb; ldB = nB;
    }
    h2o_eval(d->kernel_id, d->krnl_param, d->n_krnl_param, cA, ldA, nA, cB, ldB, nB, mat, nB * kd);
    *nrow = nA * kd;
    *ncol = nB * kd;
}

static void eval_D_block(const h2gpu_desc *d, int n0, int n1, double *mat, double *cbuf, int *nrow, int *ncol)
{
    int kd = d->krnl_dim;
    int nA = node_npt(d, n0), nB = node_npt(d, n1);
    double *ca = cbuf, *cb = cbuf + (size_t) d->xpt_dim * 4096;
    gather_pts(d, d->pt_cluster[2 * n0], nA, ca);
    gather_pts(d, d->pt_cluster[2 * n1], nB, cb);
    h2o_eval(d->kernel_id, d->krnl_param, d->n_krnl_param, ca, nA, nA, cb, nB, nB, mat, nB * kd);
    *nrow = nA * kd;
    *ncol = nB * kd;
}

static int max_block_rows(const h2gpu_desc *d)
{
    int m = 1;
    for (int i = 0; i < d->n_node; i++)
    {
        int r = node_npt(d, i) * d->krnl_dim;
        if (r > m) m = r;
        if (d->U_ncol[i] > m) m = d->U_ncol[i];
        if (d->U_nrow[i] > m) m = d->U_nrow[i];
    }
    return m;
}

/* --------------------------------------------------------------- matvec */

H2O_EXPORT int h2o_matvec(const h2gpu_desc *d, const double *x, double *y)
{
    const int N = d->krnl_dim * d->n_point, n_node = d->n_node, kd = d->krnl_dim;
    const int *mc = d->mat_cluster;
    double *px = (double *) malloc(sizeof(double) * N);
    double *py = (double *) calloc(N, sizeof(double));
    double **y0 = (double **) calloc(n_node, sizeof(double *));
    double **y1 = (double **) calloc(n_node, sizeof(double *));
    int mb = max_block_rows(d);
    double *blk = (double *) malloc(sizeof(double) * (size_t) mb * mb);
    double *cbuf = (double *) malloc(sizeof(double) * (size_t) d->xpt_dim * 4096 * 2);
    double *tmp = (double *) malloc(sizeof(double) * mb);
    if (!px || !py || !y0 || !y1 || !blk || !cbuf || !tmp) return H2GPU_ERR_NOMEM;
    for (int i = 0; i < n_node; i++)
    {
        y0[i] = (double *) calloc(d->U_ncol[i] + 1, sizeof(double));
        y1[i] = (double *) calloc(d->U_ncol[i] + 1, sizeof(double));
    }

    /* 1. forward permutation (src/H2Pack_matvec.c:1174-1179) */
    for (int i = 0; i < N; i++) px[i] = x[d->fwd_pmt_idx[i]];

    /* 2. upward sweep (src/H2Pack_matvec.c:113-160) */
    for (int lvl = d->max_level; lvl >= d->min_adm_level; lvl--)
    {
        const int *nodes = d->level_nodes + (size_t) lvl * d->n_leaf_node;
        for (int j = 0; j < d->level_n_node[lvl]; j++)
        {
            int node = nodes[j];
            int nr = d->U_nrow[node], nc = d->U_ncol[node], ld = d->U_ld[node];
            if (nc == 0) continue;
            if (d->n_child[node] == 0)
            {
                gemv_t(nr, nc, d->U[node], ld, px + mc[2 * node], 0.0, y0[node]);
            } else {
                int srow = 0;
                for (int k = 0; k < d->n_child[node]; k++)
                {
                    int c = d->children[node * d->max_child + k];
                    int cr = d->U_ncol[c];
                    gemv_t(cr, nc, d->U[node] + (size_t) srow * ld, ld, y0[c], k == 0 ? 0.0 : 1.0, y0[node]);
                    srow += cr;
                }
            }
        }
    }

    /* 3. intermediate multiplication (src/H2Pack_matvec.c:303-381, :586-764) */
    for (int i = 0; i < d->n_r_adm_pair; i++)
    {
        int n0 = d->r_adm_pairs[2 * i], n1 = d->r_adm_pairs[2 * i + 1];
        int l0 = d->node_level[n0], l1 = d->node_level[n1];
        int nr, nc;
        const double *B;
        if (d->BD_JIT) { eval_B_block(d, n0, n1, blk, cbuf, &nr, &nc); B = blk; }
        else { nr = d->B_nrow[i]; nc = d->B_ncol[i]; B = d->B_data + d->B_ptr[i]; }
        if (l0 == l1) bi_gemv(nr, nc, B, nc, y0[n1], y0[n0], y1[n0], y1[n1]);
        if (l0 > l1)  bi_gemv(nr, nc, B, nc, px + mc[2 * n1], y0[n0], y1[n0], py + mc[2 * n1]);
        if (l0 < l1)  bi_gemv(nr, nc, B, nc, y0[n1], px + mc[2 * n0], py + mc[2 * n0], y1[n1]);
    }

    /* 4. downward sweep (src/H2Pack_matvec.c:783-841) */
    for (int lvl = d->min_adm_level; lvl <= d->max_level; lvl++)
    {
        const int *nodes = d->level_nodes + (size_t) lvl * d->n_leaf_node;
        for (int j = 0; j < d->level_n_node[lvl]; j++)
        {
            int node = nodes[j];
            int nr = d->U_nrow[node], nc = d->U_ncol[node], ld = d->U_ld[node];
            if (nc == 0 || nr == 0) continue;
            gemv_n(nr, nc, d->U[node], ld, y1[node], 0.0, tmp);
            if (d->n_child[node] == 0)
            {
                for (int k = 0; k < nr; k++) py[mc[2 * node] + k] += tmp[k];
            } else {
                int off = 0;
                for (int k = 0; k < d->n_child[node]; k++)
                {
                    int c = d->children[node * d->max_child + k];
                    for (int l = 0; l < d->U_ncol[c]; l++) y1[c][l] += tmp[off + l];
                    off += d->U_ncol[c];
                }
            }
        }
    }

    /* 5. dense multiplication (src/H2Pack_matvec.c:864-934, :1002-1145) */
    for (int i = 0; i < d->n_leaf_node; i++)
    {
        int node = d->leaf_nodes[i];
        int nr, nc;
        const double *D;
        if (d->BD_JIT) { eval_D_block(d, node, node, blk, cbuf, &nr, &nc); D = blk; }
        else { nr = d->D_nrow[i]; nc = d->D_ncol[i]; D = d->D_data + d->D_ptr[i]; }
        gemv_n(nr, nc, D, nc, px + mc[2 * node], 1.0, py + mc[2 * node]);
    }
    for (int i = 0; i < d->n_r_inadm_pair; i++)
    {
        int n0 = d->r_inadm_pairs[2 * i], n1 = d->r_inadm_pairs[2 * i + 1];
        int nr, nc;
        const double *D;
        if (d->BD_JIT) { eval_D_block(d, n0, n1, blk, cbuf, &nr, &nc); D = blk; }
        else
        {
            int ii = d->n_leaf_node + i;
            nr = d->D_nrow[ii]; nc = d->D_ncol[ii]; D = d->D_data + d->D_ptr[ii];
        }
        bi_gemv(nr, nc, D, nc, px + mc[2 * n1], px + mc[2 * n0], py + mc[2 * n0], py + mc[2 * n1]);
    }

    /* 6. backward permutation (src/H2Pack_matvec.c:1277-1278) */
    for (int i = 0; i < N; i++) y[i] = py[d->bwd_pmt_idx[i]];
    (void) kd;

    for (int i = 0; i < n_node; i++) { free(y0[i]); free(y1[i]); }
    free(y0); free(y1); free(px); free(py); free(blk); free(cbuf); free(tmp);
    return H2GPU_OK;
}

/* --------------------------------------------------------------- matmul */

/* C (m x n, ldc) += op(A) (m x k) * B (k x n, ldb), op(A) = A (lda) or A^T (A is k x m, lda) */
static void gemm_acc(int transA, int m, int n, int k, const double *A, int lda,
                     const double *B, int ldb, double *C, int ldc)
{
    for (int i = 0; i < m; i++)
        for (int p = 0; p < k; p++)
        {
            double a = transA ? A[(size_t) p * lda + i] : A[(size_t) i * lda + p];
            if (a == 0.0) continue;
            const double *b = B + (size_t) p * ldb;
            double *c = C + (size_t) i * ldc;
            for (int j = 0; j < n; j++) c[j] += a * b[j];
        }
}

/* CSR of the signed pair -> block index map, restated from src/H2Pack_build.c:716-753 */
static void build_p2i(int n_node, int n_pair, const int *pairs, int diag_first_n, const int *diag_nodes,
                      int **rowptr, int **colidx, int **val)
{
    int nnz = diag_first_n + 2 * n_pair;
    int *rp = (int *) calloc(n_node + 1, sizeof(int));
    int *ci = (int *) malloc(sizeof(int) * (nnz + 1));
    int *vv = (int *) malloc(sizeof(int) * (nnz + 1));
    for (int i = 0; i < diag_first_n; i++) rp[diag_nodes[i] + 1]++;
    for (int i = 0; i < n_pair; i++) { rp[pairs[2 * i] + 1]++; rp[pairs[2 * i + 1] + 1]++; }
    for (int i = 0; i < n_node; i++) rp[i + 1] += rp[i];
    int *pos = (int *) malloc(sizeof(int) * n_node);
    memcpy(pos, rp, sizeof(int) * n_node);
    for (int i = 0; i < diag_first_n; i++)
    {
        int r = diag_nodes[i];
        ci[pos[r]] = r; vv[pos[r]] = i + 1; pos[r]++;
    }
    for (int i = 0; i < n_pair; i++)
    {
        int a = pairs[2 * i], b = pairs[2 * i + 1], idx = diag_first_n + i + 1;
        ci[pos[a]] = b; vv[pos[a]] = idx;  pos[a]++;
        ci[pos[b]] = a; vv[pos[b]] = -idx; pos[b]++;
    }
    free(pos);
    *rowptr = rp; *colidx = ci; *val = vv;
}

/*
 * Y = A X for n_vec right-hand sides in row-major (layout 101) or column-major
 * (102) storage, following the per-node traversal of src/H2Pack_matmul.c.
 */
H2O_EXPORT int h2o_matmul(const h2gpu_desc *d, int layout, int n_vec,
                          const double *X, int ldx, double *Y, int ldy)
{
    const int N = d->krnl_dim * d->n_point, n_node = d->n_node, nv = n_vec;
    const int *mc = d->mat_cluster;
    double *px = (double *) malloc(sizeof(double) * (size_t) N * nv);
    double *py = (double *) calloc((size_t) N * nv, sizeof(double));
    double **y0 = (double **) calloc(n_node, sizeof(double *));
    double **y1 = (double **) calloc(n_node, sizeof(double *));
    int mb = max_block_rows(d);
    double *blk = (double *) malloc(sizeof(double) * (size_t) mb * mb);
    double *cbuf = (double *) malloc(sizeof(double) * (size_t) d->xpt_dim * 4096 * 2);
    double *tmp = (double *) malloc(sizeof(double) * (size_t) mb * nv);
    if (!px || !py || !y0 || !y1 || !blk || !cbuf || !tmp) return H2GPU_ERR_NOMEM;
    for (int i = 0; i < n_node; i++)
    {
        y0[i] = (double *) calloc((size_t) (d->U_ncol[i] + 1) * nv, sizeof(double));
        y1[i] = (double *) calloc((size_t) (d->U_ncol[i] + 1) * nv, sizeof(double));
    }
    /* row-major work copies px/py with ld = nv (src/H2Pack_matmul.c:480-495 keeps the layout;
       the products are the same, only the storage of the work arrays differs) */
    for (int i = 0; i < N; i++)
        for (int v = 0; v < nv; v++)
        {
            int src = d->fwd_pmt_idx[i];
            px[(size_t) i * nv + v] = (layout == H2GPU_ROW_MAJOR) ? X[(size_t) src * ldx + v] : X[(size_t) v * ldx + src];
        }

    /* upward (src/H2Pack_matmul.c:63-111) */
    for (int lvl = d->max_level; lvl >= d->min_adm_level; lvl--)
    {
        const int *nodes = d->level_nodes + (size_t) lvl * d->n_leaf_node;
        for (int j = 0; j < d->level_n_node[lvl]; j++)
        {
            int node = nodes[j], nr = d->U_nrow[node], nc = d->U_ncol[node], ld = d->U_ld[node];
            if (nc == 0) continue;
            memset(y0[node], 0, sizeof(double) * (size_t) nc * nv);
            if (d->n_child[node] == 0)
                gemm_acc(1, nc, nv, nr, d->U[node], ld, px + (size_t) mc[2 * node] * nv, nv, y0[node], nv);
            else
            {
                int srow = 0;
                for (int k = 0; k < d->n_child[node]; k++)
                {
                    int c = d->children[node * d->max_child + k];
                    gemm_acc(1, nc, nv, d->U_ncol[c], d->U[node] + (size_t) srow * ld, ld, y0[c], nv, y0[node], nv);
                    srow += d->U_ncol[c];
                }
            }
        }
    }

    /* intermediate: per node0 CSR row, owner computes, symmetric pairs double
       counted (src/H2Pack_matmul.c:160-244) */
    int *rp, *ci, *vv;
    build_p2i(n_node, d->n_r_adm_pair, d->r_adm_pairs, 0, NULL, &rp, &ci, &vv);
    for (int n0 = 0; n0 < n_node; n0++)
    {
        for (int t = rp[n0]; t < rp[n0 + 1]; t++)
        {
            int n1 = ci[t], idx = vv[t];
            int trans = idx < 0;
            int bi = (trans ? -idx : idx) - 1;
            int a0 = trans ? n1 : n0, a1 = trans ? n0 : n1;  /* stored orientation */
            int nr, nc;
            const double *B;
            if (d->BD_JIT) { eval_B_block(d, a0, a1, blk, cbuf, &nr, &nc); B = blk; }
            else { nr = d->B_nrow[bi]; nc = d->B_ncol[bi]; B = d->B_data + d->B_ptr[bi]; }
            int m = trans ? nc : nr, k = trans ? nr : nc;   /* op(B_ij) is m x k */
            int l0 = d->node_level[n0], l1 = d->node_level[n1];
            const double *in = (l0 > l1) ? px + (size_t) mc[2 * n1] * nv : y0[n1];
            double *out = (l0 < l1) ? py + (size_t) mc[2 * n0] * nv : y1[n0];
            gemm_acc(trans, m, nv, k, B, nc, in, nv, out, nv);
        }
    }
    free(rp); free(ci); free(vv);

    /* downward (src/H2Pack_matmul.c:268-350) */
    for (int lvl = d->min_adm_level; lvl <= d->max_level; lvl++)
    {
        const int *nodes = d->level_nodes + (size_t) lvl * d->n_leaf_node;
        for (int j = 0; j < d->level_n_node[lvl]; j++)
        {
            int node = nodes[j], nr = d->U_nrow[node], nc = d->U_ncol[node], ld = d->U_ld[node];
            if (nc == 0 || nr == 0) continue;
            memset(tmp, 0, sizeof(double) * (size_t) nr * nv);
            gemm_acc(0, nr, nv, nc, d->U[node], ld, y1[node], nv, tmp, nv);
            if (d->n_child[node] == 0)
            {
                for (size_t k = 0; k < (size_t) nr * nv; k++) py[(size_t) mc[2 * node] * nv + k] += tmp[k];
            } else {
                int off = 0;
                for (int k = 0; k < d->n_child[node]; k++)
                {
                    int c = d->children[node * d->max_child + k];
                    for (size_t l = 0; l < (size_t) d->U_ncol[c] * nv; l++) y1[c][l] += tmp[(size_t) off * nv + l];
                    off += d->U_ncol[c];
                }
            }
        }
    }

    /* dense: per node0 CSR row (src/H2Pack_matmul.c:372-417) */
    build_p2i(n_node, d->n_r_inadm_pair, d->r_inadm_pairs, d->n_leaf_node, d->leaf_nodes, &rp, &ci, &vv);
    for (int n0 = 0; n0 < n_node; n0++)
    {
        for (int t = rp[n0]; t < rp[n0 + 1]; t++)
        {
            int n1 = ci[t], idx = vv[t];
            int trans = idx < 0;
            int di = (trans ? -idx : idx) - 1;
            int a0 = trans ? n1 : n0, a1 = trans ? n0 : n1;
            int nr, nc;
            const double *D;
            if (d->BD_JIT) { eval_D_block(d, a0, a1, blk, cbuf, &nr, &nc); D = blk; }
            else { nr = d->D_nrow[di]; nc = d->D_ncol[di]; D = d->D_data + d->D_ptr[di]; }
            int m = trans ? nc : nr, k = trans ? nr : nc;
            gemm_acc(trans, m, nv, k, D, nc, px + (size_t) mc[2 * n1] * nv, nv, py + (size_t) mc[2 * n0] * nv, nv);
        }
    }
    free(rp); free(ci); free(vv);

    /* backward permutation into the caller's layout */
    for (int i = 0; i < N; i++)
        for (int v = 0; v < nv; v++)
        {
            double val = py[(size_t) d->bwd_pmt_idx[i] * nv + v];
            if (layout == H2GPU_ROW_MAJOR) Y[(size_t) i * ldy + v] = val;
            else Y[(size_t) v * ldy + i] = val;
        }

    for (int i = 0; i < n_node; i++) { free(y0[i]); free(y1[i]); }
    free(y0); free(y1); free(px); free(py); free(blk); free(cbuf); free(tmp);
    return H2GPU_OK;
}

/* ----------------------------------------------------------- direct sum */

/* trg_val (n_trg x kd) = K(trg, src) src_val, restated from examples/direct_nbody.h:2-54
 * (blocks of 256 points, kernel block then GEMV). */
H2O_EXPORT void h2o_direct_sum(int kernel_id, const double *param, int n_param, int xpt_dim, int kd,
                               const double *src, int ld_src, int n_src, const double *src_val,
                               const double *trg, int ld_trg, int n_trg, double *trg_val)
{
    const int B = 256;
    double *mat = (double *) malloc(sizeof(double) * (size_t) B * kd * B * kd);
    double *cs = (double *) malloc(sizeof(double) * (size_t) xpt_dim * B);
    double *ct = (double *) malloc(sizeof(double) * (size_t) xpt_dim * B);
    memset(trg_val, 0, sizeof(double) * (size_t) n_trg * kd);
    for (int t0 = 0; t0 < n_trg; t0 += B)
    {
        int nt = (t0 + B > n_trg) ? n_trg - t0 : B;
        for (int k = 0; k < xpt_dim; k++) memcpy(ct + (size_t) k * nt, trg + (size_t) k * ld_trg + t0, sizeof(double) * nt);
        for (int s0 = 0; s0 < n_src; s0 += B)
        {
            int ns = (s0 + B > n_src) ? n_src - s0 : B;
            for (int k = 0; k < xpt_dim; k++) memcpy(cs + (size_t) k * ns, src + (size_t) k * ld_src + s0, sizeof(double) * ns);
            h2o_eval(kernel_id, param, n_param, ct, nt, nt, cs, ns, ns, mat, ns * kd);
            gemv_n(nt * kd, ns * kd, mat, ns * kd, src_val + (size_t) s0 * kd, 1.0, trg_val + (size_t) t0 * kd);
        }
    }
    free(mat); free(cs); free(ct);
}

/* ---------------------------------------------------------------- HSS ULV solve */

/* b = Q^T b (trans) or Q b, Q = H(0) .. H(k-1) from a row-major GEQRF of m rows (A:
   m x k, ld k, vector j below the diagonal of column j with an implicit 1; tau: the
   row after A), as LAPACK's ORMQR with side 'L' */
static void ulv_apply_q(const double *A, int m, int k, int trans, double *b)
{
    const double *tau = A + (size_t) m * k;
    for (int t = 0; t < k; t++)
    {
        const int j = trans ? t : k - 1 - t;
        double s = b[j];
        for (int i = j + 1; i < m; i++) s += A[(size_t) i * k + j] * b[i];
        s *= tau[j];
        b[j] -= s;
        for (int i = j + 1; i < m; i++) b[i] -= s * A[(size_t) i * k + j];
    }
}

/* one node of one sweep (src/H2Pack_HSS_ULV.c:1030-1067 / :1107-1148 Cholesky,
   :480-520 / :545-590 LU) on b0 = the node's entries of the permuted vector */
static void ulv_node(const h2gpu_ulv_desc *d, int node, int has_q, int up, double *b0, double *tmp)
{
    const int m = d->m[node], I = d->Ls[node], n2 = m - I, ld = d->l_ld[node];
    const double *L = d->L[node];
    double *b1 = b0, *b2 = b0 + I;
    const double *T = L + (size_t) I * ld + I;
    if (up)
    {
        if (has_q) ulv_apply_q(d->Q[node], m, d->q_ncol[node], 1, b0);
        if (d->lu)
        {
            memcpy(tmp, b2, sizeof(double) * (size_t) n2);
            for (int j = 0; j < n2; j++) b2[j] = tmp[d->p[node][j]];
        }
        for (int r = 0; r < n2; r++)                 /* b2 = L22 \ b2 (LU: unit diagonal) */
        {
            double s = b2[r];
            for (int c = 0; c < r; c++) s -= T[(size_t) r * ld + c] * b2[c];
            b2[r] = d->lu ? s : s / T[(size_t) r * ld + r];
        }
        for (int r = 0; r < I; r++)                  /* b1 -= L12 b2 */
        {
            double s = 0.0;
            for (int c = 0; c < n2; c++) s += L[(size_t) r * ld + I + c] * b2[c];
            b1[r] -= s;
        }
    } else {
        if (!d->lu)
        {
            for (int c = 0; c < n2; c++)             /* b2 -= L12^T b1 */
            {
                double s = 0.0;
                for (int r = 0; r < I; r++) s += L[(size_t) r * ld + I + c] * b1[r];
                b2[c] -= s;
            }
            for (int r = n2 - 1; r >= 0; r--)        /* b2 = L22^T \ b2 */
            {
                double s = b2[r];
                for (int c = r + 1; c < n2; c++) s -= T[(size_t) c * ld + r] * b2[c];
                b2[r] = s / T[(size_t) r * ld + r];
            }
        } else {
            for (int r = 0; r < n2; r++)             /* b2 -= LD21 b1 */
            {
                double s = 0.0;
                for (int c = 0; c < I; c++) s += L[(size_t) (I + r) * ld + c] * b1[c];
                b2[r] -= s;
            }
            for (int r = n2 - 1; r >= 0; r--)        /* b2 = U0 \ b2 */
            {
                double s = b2[r];
                for (int c = r + 1; c < n2; c++) s -= T[(size_t) r * ld + c] * b2[c];
                b2[r] = s / T[(size_t) r * ld + r];
            }
        }
        if (has_q) ulv_apply_q(d->Q[node], m, d->q_ncol[node], 0, b0);
    }
}

/* x = the ULV solve of b (op 1, 2 or 3 as the reference's); the root (level 0) has no
   Q.  Returns 0, or -1 on a bad argument or allocation failure. */
H2O_EXPORT int h2o_ulv_solve(const h2gpu_ulv_desc *d, int op, const double *b, double *x)
{
    if (d == NULL || b == NULL || x == NULL || op < 1 || op > 3) return -1;
    const int n = d->krnl_mat_size;
    int mmax = 1;
    for (int i = 0; i < d->n_node; i++) mmax = d->m[i] > mmax ? d->m[i] : mmax;
    double *px = (double *) malloc(sizeof(double) * (size_t) n);
    double *b0 = (double *) malloc(sizeof(double) * (size_t) mmax);
    double *tmp = (double *) malloc(sizeof(double) * (size_t) mmax);
    if (px == NULL || b0 == NULL || tmp == NULL)
    {
        free(px); free(b0); free(tmp);
        return -1;
    }
    for (int i = 0; i < n; i++) px[i] = b[d->fwd_pmt_idx[i]];
    for (int pass = 0; pass < 2; pass++)
    {
        const int up = pass == 0;
        if (!(op & (up ? 1 : 2))) continue;
        for (int t = 0; t <= d->max_level; t++)
        {
            const int lvl = up ? d->max_level - t : t;
            for (int j = 0; j < d->level_n_node[lvl]; j++)
            {
                const int node = d->level_nodes[(size_t) lvl * d->n_leaf_node + j];
                const int m = d->m[node];
                const int has_q = lvl > 0 && d->q_ncol[node] > 0;
                for (int k = 0; k < m; k++) b0[k] = px[d->idx[node][k]];
                ulv_node(d, node, has_q, up, b0, tmp);
                for (int k = 0; k < m; k++) px[d->idx[node][k]] = b0[k];
            }
        }
    }
    for (int i = 0; i < n; i++) x[i] = px[d->bwd_pmt_idx[i]];
    free(px); free(b0); free(tmp);
    return 0;
}
