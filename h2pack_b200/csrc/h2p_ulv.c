/*
 * h2p_ulv.c -- H2Pack's HSS ULV solves on the GPU engine.
 *
 * H2P_HSS_ULV_Cholesky_solve and H2P_HSS_ULV_LU_solve (src/H2Pack_HSS_ULV.h,
 * src/H2Pack_HSS_ULV.c:981-1159 and :429-599) are replaced inside libH2Pack_gpu.so:
 * H2Pack_HSS_ULV.c is compiled with one function per section and both solves weakened
 * and aliased (H2P_HSS_ULV_Cholesky_solve_host, H2P_HSS_ULV_LU_solve_host), so the
 * factorizations stay H2Pack's own code and a program's solve calls land here.  The
 * replacements keep the reference's signature, its argument checks and messages, and
 * its side effects on the handle (n_ULV_solve, timers[ULV_SLV_TIMER_IDX]).
 *
 * Each handle's factors are uploaded once (h2gpu_ulv_create) and reused while their
 * fingerprint holds: factor kind, sizes, array addresses and a strided sample of every
 * node's L.  A new factorization of the handle (another shift, LU after Cholesky)
 * allocates new factors and is uploaded on the next solve.  Calls on one handle are
 * serialised (the reference's solve is not reentrant per handle either: it works in
 * the handle's pmt_x); calls on different handles run concurrently.  H2P_destroy
 * (h2p_dropin.c) releases the handle's factors through H2P_gpu_ULV_release.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include "H2Pack.h"
#include "h2gpu.h"

#define DROPIN_API __attribute__((visibility("default")))

/* h2p_dropin.c: record a failure in H2P_gpu_last_error's message */
int h2p_dropin_fail(int st, const char *what, const char *msg);
const char *H2P_gpu_last_error(void);

typedef struct ulv_entry
{
    H2Pack_p key;
    pthread_mutex_t mu;       /* held across one solve on this handle              */
    int refs, dead;
    int lu;
    uint64_t fingerprint;
    h2gpu_ulv *ulv;
    struct ulv_entry *next;
} ulv_entry;

static ulv_entry *g_ulv = NULL;
static pthread_mutex_t g_ulv_mu = PTHREAD_MUTEX_INITIALIZER;   /* registry links and refs only */

static double wtime(void)
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return (double) tv.tv_sec + 1e-6 * (double) tv.tv_usec;
}

static uint64_t mix(uint64_t h, uint64_t v)
{
    h ^= v + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
    return h;
}

static uint64_t fingerprint(H2Pack_p h, int lu)
{
    uint64_t f = mix(1469598103934665603ULL, (uint64_t) lu);
    f = mix(f, (uint64_t) h->n_node);
    f = mix(f, (uint64_t) h->krnl_mat_size);
    f = mix(f, (uint64_t) (uintptr_t) h->ULV_idx);
    f = mix(f, (uint64_t) (uintptr_t) h->ULV_Q);
    f = mix(f, (uint64_t) (uintptr_t) h->ULV_L);
    f = mix(f, (uint64_t) (uintptr_t) h->ULV_p);
    f = mix(f, (uint64_t) (uintptr_t) h->fwd_pmt_idx);
    for (int i = 0; i < h->n_node; i++)
    {
        H2P_dense_mat_p L = h->ULV_L[i];
        if (L == NULL) continue;
        f = mix(f, (uint64_t) (uintptr_t) L->data);
        f = mix(f, (uint64_t) L->nrow);
        const size_t n = (size_t) L->nrow * L->ld;
        const size_t step = n > 8 ? n / 8 : 1;
        for (size_t k = 0; k < n; k += step)
        {
            uint64_t b;
            memcpy(&b, &L->data[k], sizeof(b));
            f = mix(f, b);
        }
    }
    return f;
}

static ulv_entry *acquire(H2Pack_p h)
{
    pthread_mutex_lock(&g_ulv_mu);
    ulv_entry *e = g_ulv;
    while (e != NULL && (e->key != h || e->dead)) e = e->next;
    if (e == NULL)
    {
        e = (ulv_entry *) calloc(1, sizeof(ulv_entry));
        if (e != NULL)
        {
            e->key = h;
            pthread_mutex_init(&e->mu, NULL);
            e->next = g_ulv;
            g_ulv = e;
        }
    }
    if (e != NULL) e->refs++;
    pthread_mutex_unlock(&g_ulv_mu);
    return e;
}

static void release_ref(ulv_entry *e)
{
    int last = 0;
    pthread_mutex_lock(&g_ulv_mu);
    e->refs--;
    last = e->dead && e->refs == 0;
    pthread_mutex_unlock(&g_ulv_mu);
    if (last)
    {
        h2gpu_ulv_destroy(e->ulv);
        pthread_mutex_destroy(&e->mu);
        free(e);
    }
}

/* Free the handle's device factors (H2P_destroy calls this before H2Pack frees the
   handle).  Returns H2GPU_OK. */
DROPIN_API int H2P_gpu_ULV_release(H2Pack_p h)
{
    ulv_entry *e = NULL;
    pthread_mutex_lock(&g_ulv_mu);
    for (ulv_entry **pp = &g_ulv; *pp != NULL; pp = &(*pp)->next)
    {
        if ((*pp)->key == h && !(*pp)->dead)
        {
            e = *pp;
            *pp = e->next;
            e->dead = 1;
            e->refs++;
            break;
        }
    }
    pthread_mutex_unlock(&g_ulv_mu);
    if (e != NULL) release_ref(e);
    return H2GPU_OK;
}

/* h2p_builder.c: the handle's factors as an h2gpu_ulv_desc */
int h2pb_describe_ulv(H2Pack_p h, int lu, h2gpu_ulv_desc *d, void **buf);

/* the handle's factors onto the device; records its own failure message */
static int upload(H2Pack_p h, int lu, h2gpu_ulv **out)
{
    const char *what = "H2P_HSS_ULV_solve";
    h2gpu_ulv_desc d;
    void *buf = NULL;
    int st = h2pb_describe_ulv(h, lu, &d, &buf);
    if (st == H2GPU_ERR_STATE)
        return h2p_dropin_fail(st, what, lu ? "the handle holds no LU factors (H2P_HSS_ULV_LU_factorize)"
                                            : "the handle's ULV factors are incomplete");
    if (st != H2GPU_OK) return h2p_dropin_fail(st, what, "host allocation");
    /* the reference's solve assumes these shapes (src/H2Pack_HSS_ULV.c:1036-1046) */
    const int root = h->level_nodes[0];
    for (int i = 0; i < h->n_node && st == H2GPU_OK; i++)
    {
        H2P_dense_mat_p q = h->ULV_Q[i], l = h->ULV_L[i];
        if (l->nrow != d.m[i] || l->ncol != d.m[i] ||
            (i != root && q->ncol > 0 && (q->nrow != d.m[i] + 1 || q->ld != q->ncol)) ||
            (lu && h->ULV_p[i]->length != d.m[i] - d.Ls[i]))
            st = h2p_dropin_fail(H2GPU_ERR_INVALID, what, "factor shapes differ from H2Pack's layout");
    }
    if (st == H2GPU_OK)
    {
        st = h2gpu_ulv_create(&d, out);
        if (st != H2GPU_OK) h2p_dropin_fail(st, "uploading the ULV factors", NULL);
    }
    free(buf);
    return st;
}

/* x = the ULV solve of b on the GPU (lu: the factors of H2P_HSS_ULV_LU_factorize, else
   of H2P_HSS_ULV_Cholesky_factorize; op as the reference's).  Status-returning form of
   the two replaced solves; counts the solve and its time on the handle. */
DROPIN_API int H2P_gpu_ULV_solve(H2Pack_p h, int lu, int op, const double *b, double *x)
{
    const char *what = "H2P_HSS_ULV_solve";
    if (h == NULL || b == NULL || x == NULL) return h2p_dropin_fail(H2GPU_ERR_INVALID, what, "NULL argument");
    if (!h->is_HSS) return h2p_dropin_fail(H2GPU_ERR_STATE, what, "H2Pack is not running in HSS mode");
    if (h->ULV_idx == NULL) return h2p_dropin_fail(H2GPU_ERR_STATE, what, "no ULV factorization on the handle");
    if (op < 1 || op > 3) return h2p_dropin_fail(H2GPU_ERR_INVALID, what, "op must be 1, 2 or 3");
    const double st0 = wtime();
    ulv_entry *e = acquire(h);
    if (e == NULL) return h2p_dropin_fail(H2GPU_ERR_NOMEM, what, "host allocation");
    pthread_mutex_lock(&e->mu);
    int st = H2GPU_OK;
    const uint64_t f = fingerprint(h, lu);
    if (e->ulv == NULL || e->fingerprint != f || e->lu != lu)
    {
        if (e->ulv != NULL) h2gpu_ulv_destroy(e->ulv);
        e->ulv = NULL;
        st = upload(h, lu, &e->ulv);   /* records its own failure message */
        e->fingerprint = f;
        e->lu = lu;
    }
    if (st == H2GPU_OK)
    {
        st = h2gpu_ulv_solve(e->ulv, op, b, x);
        if (st != H2GPU_OK) h2p_dropin_fail(st, what, NULL);
    }
    pthread_mutex_unlock(&e->mu);
    release_ref(e);
    if (st == H2GPU_OK)
    {
        h->n_ULV_solve++;
        h->timers[ULV_SLV_TIMER_IDX] += wtime() - st0;
    }
    return st;
}

static void solve_or_die(H2Pack_p h, int lu, int op, const DTYPE *b, DTYPE *x, const char *name, const char *factor)
{
    /* the reference's checks and messages (src/H2Pack_HSS_ULV.c:983-997) */
    if (!h->is_HSS)
    {
        ERROR_PRINTF("H2Pack is not running in HSS mode!\n");
        return;
    }
    if (h->ULV_idx == NULL)
    {
        ERROR_PRINTF("Need to call %s() first!\n", factor);
        return;
    }
    if (op < 1 || op > 3)
    {
        ERROR_PRINTF("Invalid operation type %d, should be 1, 2, or 3\n", op);
        return;
    }
    const int st = H2P_gpu_ULV_solve(h, lu, op, b, x);
    if (st != H2GPU_OK)
    {
        fprintf(stderr, "[FATAL] H2Pack GPU drop-in, %s failed (status %d): %s\n", name, st, H2P_gpu_last_error());
        abort();
    }
}

/* Replaces src/H2Pack_HSS_ULV.c:981 (same signature and checks). */
DROPIN_API void H2P_HSS_ULV_Cholesky_solve(H2Pack_p h2pack, const int op, const DTYPE *b, DTYPE *x)
{
    solve_or_die(h2pack, 0, op, b, x, "H2P_HSS_ULV_Cholesky_solve", "H2P_HSS_ULV_Cholesky_factorize");
}

/* Replaces src/H2Pack_HSS_ULV.c:429 (same signature and checks). */
DROPIN_API void H2P_HSS_ULV_LU_solve(H2Pack_p h2pack, const int op, const DTYPE *b, DTYPE *x)
{
    solve_or_die(h2pack, 1, op, b, x, "H2P_HSS_ULV_LU_solve", "H2P_HSS_ULV_LU_factorize");
}
