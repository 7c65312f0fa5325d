/*
 * h2p_dropin.c -- H2Pack's apply entry points on the GPU engine.
 *
 * Compiled against H2Pack's own headers so that struct H2Pack is read exactly as
 * H2Pack lays it out; every entry point keeps the reference signature
 * (src/H2Pack_matvec.h:17-30, src/H2Pack_matmul.h:25-54) and its side effects on
 * the handle: n_matvec (src/H2Pack_matvec.c:1283, src/H2Pack_matmul.c:582) and the
 * phase timers timers[MV_*_TIMER_IDX] (src/H2Pack_typedef.h:226-239) that
 * H2P_print_statistic reads.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "H2Pack.h"
#include "h2gpu.h"

#define DROPIN_API __attribute__((visibility("default")))

_Static_assert(sizeof(DTYPE) == sizeof(double), "the GPU drop-in is built for DTYPE = double");

/* h2p_builder.c */
int h2pb_describe_h2pack(H2Pack_p h, int kernel_id, const double *param, int n_param,
                         h2gpu_desc *d, int **ints_out, const double ***ptrs_out);

typedef struct reg_entry
{
    H2Pack_p key;
    uint64_t fingerprint;
    h2gpu_image *img;
    int kernel_id, n_param, precision;
    double param[4];
    double ms_seen[5];
    struct reg_entry *next;
} reg_entry;

static reg_entry *g_reg = NULL;
static pthread_mutex_t g_mu = PTHREAD_MUTEX_INITIALIZER;
static __thread char g_msg[512];

static uint64_t mix(uint64_t h, uint64_t v)
{
    h ^= v + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
    return h;
}

/* Identity of the arrays the image was built from. */
static uint64_t fingerprint(H2Pack_p h)
{
    uint64_t f = 1469598103934665603ULL;
    f = mix(f, (uint64_t) h->n_point);   f = mix(f, (uint64_t) h->n_node);
    f = mix(f, (uint64_t) h->n_B);       f = mix(f, (uint64_t) h->n_D);
    f = mix(f, (uint64_t) h->BD_JIT);    f = mix(f, (uint64_t) h->krnl_dim);
    f = mix(f, (uint64_t) (uintptr_t) h->U);        f = mix(f, (uint64_t) (uintptr_t) h->B_data);
    f = mix(f, (uint64_t) (uintptr_t) h->D_data);   f = mix(f, (uint64_t) (uintptr_t) h->coord);
    f = mix(f, (uint64_t) (uintptr_t) h->r_adm_pairs);  f = mix(f, (uint64_t) (uintptr_t) h->fwd_pmt_idx);
    f = mix(f, (uint64_t) (uintptr_t) h->J_coord);
    return f;
}

static reg_entry *find(H2Pack_p h)
{
    for (reg_entry *e = g_reg; e != NULL; e = e->next)
        if (e->key == h) return e;
    return NULL;
}

static reg_entry *find_or_add(H2Pack_p h)
{
    reg_entry *e = find(h);
    if (e != NULL) return e;
    e = (reg_entry *) calloc(1, sizeof(reg_entry));
    if (e == NULL) return NULL;
    e->key = h;
    e->precision = H2GPU_PREC_FP64;
    e->next = g_reg;
    g_reg = e;
    return e;
}

static int set_msg(int st, const char *what)
{
    snprintf(g_msg, sizeof(g_msg), "%s: %s", what, st == H2GPU_OK ? "ok" : h2gpu_last_error());
    return st;
}

/* Device image of a handle, created or refreshed as needed (caller holds g_mu). */
static int image_of(H2Pack_p h, reg_entry **out)
{
    if (h == NULL) return set_msg(H2GPU_ERR_INVALID, "H2Pack handle is NULL");
    reg_entry *e = find_or_add(h);
    if (e == NULL) return set_msg(H2GPU_ERR_NOMEM, "registry allocation");
    uint64_t fp = fingerprint(h);
    if (e->img != NULL && e->fingerprint == fp) { *out = e; return H2GPU_OK; }
    if (e->img != NULL) { h2gpu_image_destroy(e->img); e->img = NULL; }
    if (h->BD_JIT && e->kernel_id == 0)
    {
        snprintf(g_msg, sizeof(g_msg),
                 "JIT-mode handle has no kernel id: call H2P_gpu_set_kernel() before the first apply");
        return H2GPU_ERR_STATE;
    }
    h2gpu_desc d;
    int *ints = NULL;
    const double **ptrs = NULL;
    int st = h2pb_describe_h2pack(h, e->kernel_id, e->param, e->n_param, &d, &ints, &ptrs);
    if (st != H2GPU_OK)
    {
        snprintf(g_msg, sizeof(g_msg), "handle not supported by the GPU apply path (status %d): "
                 "HSS, periodic and H2ERI handles are not accelerated", st);
        return st;
    }
    h2gpu_options opt;
    h2gpu_default_options(&opt);
    opt.precision = e->precision;
    st = h2gpu_image_create(&d, &opt, &e->img);
    free(ints);
    free(ptrs);
    if (st != H2GPU_OK) return set_msg(st, "h2gpu_image_create");
    e->fingerprint = fp;
    memset(e->ms_seen, 0, sizeof(e->ms_seen));
    *out = e;
    return H2GPU_OK;
}

/* Add the device phase times of the last call to the handle's timers (seconds). */
static void account(H2Pack_p h, reg_entry *e)
{
    h2gpu_stats s;
    if (h2gpu_get_stats(e->img, &s) != H2GPU_OK) return;
    static const int idx[5] = {MV_FWD_TIMER_IDX, MV_MID_TIMER_IDX, MV_BWD_TIMER_IDX, MV_DEN_TIMER_IDX, MV_VOP_TIMER_IDX};
    for (int k = 0; k < 5; k++)
    {
        h->timers[idx[k]] += 1e-3 * (s.ms_phase[k] - e->ms_seen[k]);
        e->ms_seen[k] = s.ms_phase[k];
    }
}

DROPIN_API int H2P_gpu_set_kernel(H2Pack_p h, int kernel_id, const double *param, int n_param)
{
    if (h == NULL || n_param < 0 || n_param > 4 || (n_param > 0 && param == NULL))
        return set_msg(H2GPU_ERR_INVALID, "H2P_gpu_set_kernel arguments");
    if (kernel_id < H2GPU_KRNL_COULOMB || kernel_id > H2GPU_KRNL_RPY)
        return set_msg(H2GPU_ERR_INVALID, "unknown kernel id");
    pthread_mutex_lock(&g_mu);
    reg_entry *e = find_or_add(h);
    int st = H2GPU_OK;
    if (e == NULL) st = H2GPU_ERR_NOMEM;
    else
    {
        e->kernel_id = kernel_id;
        e->n_param = n_param;
        memset(e->param, 0, sizeof(e->param));
        for (int i = 0; i < n_param; i++) e->param[i] = param[i];
        if (e->img) { h2gpu_image_destroy(e->img); e->img = NULL; }
    }
    pthread_mutex_unlock(&g_mu);
    return st;
}

DROPIN_API int H2P_gpu_set_precision(H2Pack_p h, int precision)
{
    if (h == NULL || (precision != H2GPU_PREC_FP64 && precision != H2GPU_PREC_MIXED))
        return set_msg(H2GPU_ERR_INVALID, "H2P_gpu_set_precision arguments");
    pthread_mutex_lock(&g_mu);
    reg_entry *e = find_or_add(h);
    int st = H2GPU_OK;
    if (e == NULL) st = H2GPU_ERR_NOMEM;
    else
    {
        e->precision = precision;
        if (e->img) st = h2gpu_set_precision(e->img, precision);
    }
    pthread_mutex_unlock(&g_mu);
    return st;
}

DROPIN_API int H2P_gpu_matvec(H2Pack_p h, const double *x, double *y)
{
    pthread_mutex_lock(&g_mu);
    reg_entry *e = NULL;
    int st = image_of(h, &e);
    if (st == H2GPU_OK)
    {
        st = h2gpu_matvec(e->img, x, y);
        if (st == H2GPU_OK) { h->n_matvec++; account(h, e); }
        else set_msg(st, "h2gpu_matvec");
    }
    pthread_mutex_unlock(&g_mu);
    return st;
}

DROPIN_API int H2P_gpu_matmul(H2Pack_p h, int layout, int n_vec, const double *mat_x, int ldx, double *mat_y, int ldy)
{
    pthread_mutex_lock(&g_mu);
    reg_entry *e = NULL;
    int st = image_of(h, &e);
    if (st == H2GPU_OK)
    {
        st = h2gpu_matmul(e->img, layout, n_vec, mat_x, ldx, mat_y, ldy);
        if (st == H2GPU_OK) { h->n_matvec += n_vec; account(h, e); }
        else set_msg(st, "h2gpu_matmul");
    }
    pthread_mutex_unlock(&g_mu);
    return st;
}

DROPIN_API h2gpu_image *H2P_gpu_image(H2Pack_p h)
{
    pthread_mutex_lock(&g_mu);
    reg_entry *e = NULL;
    h2gpu_image *img = (image_of(h, &e) == H2GPU_OK) ? e->img : NULL;
    pthread_mutex_unlock(&g_mu);
    return img;
}

DROPIN_API int H2P_gpu_release(H2Pack_p h)
{
    pthread_mutex_lock(&g_mu);
    reg_entry **pp = &g_reg;
    while (*pp != NULL && (*pp)->key != h) pp = &(*pp)->next;
    if (*pp != NULL)
    {
        reg_entry *e = *pp;
        *pp = e->next;
        if (e->img) h2gpu_image_destroy(e->img);
        free(e);
    }
    pthread_mutex_unlock(&g_mu);
    return H2GPU_OK;
}

DROPIN_API const char *H2P_gpu_last_error(void) { return g_msg; }

static void die(const char *what)
{
    fprintf(stderr, "[FATAL] H2Pack GPU drop-in, %s failed: %s\n", what, g_msg);
    fflush(stderr);
    abort();
}

/* ----- H2Pack signatures ----- */

DROPIN_API void H2P_matvec(H2Pack_p h2pack, const DTYPE *x, DTYPE *y)
{
    if (H2P_gpu_matvec(h2pack, x, y) != H2GPU_OK) die("H2P_matvec");
}

DROPIN_API void H2P_matmul(H2Pack_p h2pack, const CBLAS_LAYOUT layout, const int n_vec,
                           const DTYPE *mat_x, const int ldx, DTYPE *mat_y, const int ldy)
{
    if (H2P_gpu_matmul(h2pack, (int) layout, n_vec, mat_x, ldx, mat_y, ldy) != H2GPU_OK) die("H2P_matmul");
}

static void permute(H2Pack_p h, int forward, int layout, int n_vec, const double *x, int ldx, double *px, int ldp,
                    const char *what)
{
    pthread_mutex_lock(&g_mu);
    reg_entry *e = NULL;
    int st = image_of(h, &e);
    if (st == H2GPU_OK)
    {
        st = h2gpu_permute_matrix_rows(e->img, forward, layout, n_vec, x, ldx, px, ldp);
        if (st != H2GPU_OK) set_msg(st, what);
    }
    pthread_mutex_unlock(&g_mu);
    if (st != H2GPU_OK) die(what);
}

DROPIN_API void H2P_permute_vector_forward(H2Pack_p h2pack, const DTYPE *x, DTYPE *pmt_x)
{
    permute(h2pack, 1, H2GPU_COL_MAJOR, 1, x, h2pack->krnl_mat_size, pmt_x, h2pack->krnl_mat_size,
            "H2P_permute_vector_forward");
}

DROPIN_API void H2P_permute_vector_backward(H2Pack_p h2pack, const DTYPE *x, DTYPE *pmt_x)
{
    permute(h2pack, 0, H2GPU_COL_MAJOR, 1, x, h2pack->krnl_mat_size, pmt_x, h2pack->krnl_mat_size,
            "H2P_permute_vector_backward");
}

DROPIN_API void H2P_permute_matrix_row_forward(H2Pack_p h2pack, const CBLAS_LAYOUT layout, const int n_vec,
                                               const DTYPE *mat_x, const int ldx, DTYPE *pmt_mat_x, const int ldp)
{
    permute(h2pack, 1, (int) layout, n_vec, mat_x, ldx, pmt_mat_x, ldp, "H2P_permute_matrix_row_forward");
}

DROPIN_API void H2P_permute_matrix_row_backward(H2Pack_p h2pack, const CBLAS_LAYOUT layout, const int n_vec,
                                                const DTYPE *mat_x, const int ldx, DTYPE *pmt_mat_x, const int ldp)
{
    permute(h2pack, 0, (int) layout, n_vec, mat_x, ldx, pmt_mat_x, ldp, "H2P_permute_matrix_row_backward");
}
