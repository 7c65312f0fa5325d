/*
 * Scalar-lane stand-in for the ASTER SIMD wrapper used by H2Pack.
 *
 * Build support for compiling H2Pack's own sources.  H2Pack includes "ASTER/include/aster.h"
 * (src/H2Pack_config.h:109, src/H2Pack_3D_kernels.h:7), a git submodule
 * (https://github.com/huanghua1994/ASTER, pinned commit not recoverable) whose
 * directory is empty in the reference tree.  This header is NOT the ASTER source:
 * it gives each name the reference calls the meaning its call sites require,
 * implemented with GCC vector extensions and lane-wise libm calls:
 *
 *   vec_t                 SIMD_LEN lanes of DTYPE (8 doubles / 16 floats)
 *   vec_load/loadu/store/storeu_t   (un)aligned vector memory access
 *   vec_zero/set1/bcast_t  zero vector, broadcast of a value / of *pointer
 *   vec_add/sub/mul/div/max_t       lane-wise arithmetic
 *   vec_fmadd_t(a,b,c) = a*b + c,  vec_fmsub_t(a,b,c) = a*b - c
 *   vec_sqrt/exp/log/pow_t          lane-wise libm
 *   vec_frsqrt_t(x)       1/sqrt(x) lane-wise, and 0 where x == 0 (the RPY and
 *                         Stokes kernels multiply dx*inv_r without a blend,
 *                         src/H2Pack_3D_kernels.h:1348-1354)
 *   vec_frsqrt_pf_t()     prefactor p with p*vec_frsqrt_t(x) == 1/sqrt(x); 1 here
 *   vec_cmp_{eq,gt,le}_t  lane masks (all ones where true)
 *   vec_blend_t(a,b,m)    b where m is set, a elsewhere (src/H2Pack_3D_kernels.h:80)
 *   vec_reduce_add_t      sum of all lanes
 *
 * Because the fast approximate exp/rsqrt of the real ASTER are replaced by libm,
 * kernel values here are plain FP64 libm values.
 */
#ifndef H2B_ORACLE_ASTER_SHIM_H
#define H2B_ORACLE_ASTER_SHIM_H

#include <math.h>
#include <string.h>

#define SIMD_LEN_D 8
#define SIMD_LEN_S 16

#if defined(ASTER_DTYPE_FLOAT)
#define ASTER_SHIM_T     float
#define ASTER_SHIM_IT    int
#define ASTER_SHIM_LEN   SIMD_LEN_S
#define ASTER_SHIM_SQRT  sqrtf
#define ASTER_SHIM_EXP   expf
#define ASTER_SHIM_LOG   logf
#define ASTER_SHIM_POW   powf
#else
#define ASTER_SHIM_T     double
#define ASTER_SHIM_IT    long long
#define ASTER_SHIM_LEN   SIMD_LEN_D
#define ASTER_SHIM_SQRT  sqrt
#define ASTER_SHIM_EXP   exp
#define ASTER_SHIM_LOG   log
#define ASTER_SHIM_POW   pow
#endif

typedef ASTER_SHIM_T  vec_t     __attribute__((vector_size(ASTER_SHIM_LEN * sizeof(ASTER_SHIM_T))));
typedef ASTER_SHIM_IT vec_cmp_t __attribute__((vector_size(ASTER_SHIM_LEN * sizeof(ASTER_SHIM_IT))));

static inline vec_t vec_zero_t(void) { vec_t r = {0}; return r; }
static inline vec_t vec_set1_t(const ASTER_SHIM_T a) { vec_t r = {0}; return r + a; }
static inline vec_t vec_bcast_t(const ASTER_SHIM_T *p) { return vec_set1_t(*p); }
static inline vec_t vec_loadu_t(const ASTER_SHIM_T *p) { vec_t r; memcpy(&r, p, sizeof(r)); return r; }
static inline vec_t vec_load_t(const ASTER_SHIM_T *p) { return vec_loadu_t(p); }
static inline void  vec_storeu_t(ASTER_SHIM_T *p, const vec_t v) { memcpy(p, &v, sizeof(v)); }
static inline void  vec_store_t(ASTER_SHIM_T *p, const vec_t v) { vec_storeu_t(p, v); }

static inline vec_t vec_add_t(const vec_t a, const vec_t b) { return a + b; }
static inline vec_t vec_sub_t(const vec_t a, const vec_t b) { return a - b; }
static inline vec_t vec_mul_t(const vec_t a, const vec_t b) { return a * b; }
static inline vec_t vec_div_t(const vec_t a, const vec_t b) { return a / b; }
static inline vec_t vec_fmadd_t(const vec_t a, const vec_t b, const vec_t c) { return a * b + c; }
static inline vec_t vec_fmsub_t(const vec_t a, const vec_t b, const vec_t c) { return a * b - c; }

static inline vec_cmp_t vec_cmp_eq_t(const vec_t a, const vec_t b) { return (vec_cmp_t) (a == b); }
static inline vec_cmp_t vec_cmp_gt_t(const vec_t a, const vec_t b) { return (vec_cmp_t) (a >  b); }
static inline vec_cmp_t vec_cmp_le_t(const vec_t a, const vec_t b) { return (vec_cmp_t) (a <= b); }

static inline vec_t vec_blend_t(const vec_t a, const vec_t b, const vec_cmp_t m)
{
    vec_cmp_t ai, bi;
    memcpy(&ai, &a, sizeof(ai));
    memcpy(&bi, &b, sizeof(bi));
    vec_cmp_t ri = (ai & ~m) | (bi & m);
    vec_t r;
    memcpy(&r, &ri, sizeof(r));
    return r;
}

static inline vec_t vec_max_t(const vec_t a, const vec_t b)
{
    vec_t r;
    for (int i = 0; i < ASTER_SHIM_LEN; i++) r[i] = (a[i] > b[i]) ? a[i] : b[i];
    return r;
}

static inline vec_t vec_sqrt_t(const vec_t a)
{
    vec_t r;
    for (int i = 0; i < ASTER_SHIM_LEN; i++) r[i] = ASTER_SHIM_SQRT(a[i]);
    return r;
}

static inline vec_t vec_frsqrt_pf_t(void) { return vec_set1_t((ASTER_SHIM_T) 1); }

static inline vec_t vec_frsqrt_t(const vec_t a)
{
    vec_t r;
    for (int i = 0; i < ASTER_SHIM_LEN; i++)
        r[i] = (a[i] == (ASTER_SHIM_T) 0) ? (ASTER_SHIM_T) 0 : (ASTER_SHIM_T) 1 / ASTER_SHIM_SQRT(a[i]);
    return r;
}

static inline vec_t vec_exp_t(const vec_t a)
{
    vec_t r;
    for (int i = 0; i < ASTER_SHIM_LEN; i++) r[i] = ASTER_SHIM_EXP(a[i]);
    return r;
}

static inline vec_t vec_log_t(const vec_t a)
{
    vec_t r;
    for (int i = 0; i < ASTER_SHIM_LEN; i++) r[i] = ASTER_SHIM_LOG(a[i]);
    return r;
}

static inline vec_t vec_pow_t(const vec_t a, const vec_t b)
{
    vec_t r;
    for (int i = 0; i < ASTER_SHIM_LEN; i++) r[i] = ASTER_SHIM_POW(a[i], b[i]);
    return r;
}

static inline ASTER_SHIM_T vec_reduce_add_t(const vec_t a)
{
    ASTER_SHIM_T s = 0;
    for (int i = 0; i < ASTER_SHIM_LEN; i++) s += a[i];
    return s;
}

#endif
