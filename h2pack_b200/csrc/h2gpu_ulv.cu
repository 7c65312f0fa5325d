// h2gpu_ulv.cu -- the ULV solve of an HSS matrix on the device (include/h2gpu.h,
// h2gpu_ulv_*).
//
// The reference solves level by level on the host (H2P_HSS_ULV_Cholesky_solve,
// src/H2Pack_HSS_ULV.c:981-1159; H2P_HSS_ULV_LU_solve, :429-599).  Per node it gathers
// the node's entries of the permuted vector, applies Q^T (or Q), solves with the
// node's triangular factor, updates with the off-diagonal part of the factor and
// scatters back.  Nodes of one level touch disjoint entries, so here each level is one
// launch with one CTA per node, the node's vector in shared memory:
//
//   Cholesky, first sweep (levels max .. 0)   b = Q^T b;  b2 = L22 \ b2;  b1 -= L12 b2
//   Cholesky, second sweep (levels 0 .. max)  b2 -= L12^T b1;  b2 = L22^T \ b2;  b = Q b
//   LU, first sweep (levels max .. 0)         b = Q^T b;  b2 = b2(p);  b2 = L0 \ b2 (unit);
//                                             b1 -= DU12 b2
//   LU, second sweep (levels 0 .. max)        b2 -= LD21 b1;  b2 = U0 \ b2;  b = Q b
//
// with b1 / b2 the first Ls / last m - Ls entries and L12, L22, DU12, LD21, L0, U0 the
// blocks of the node's m x m factor.  The root (level 0) has no Q and Ls = 0.
//
// Layout.  Q is kept explicitly (m x m per node, stored as Q^T row-major, i.e. row r
// = column r of Q), formed once from the reflectors at create by k_ulv_form_q, so
// that Q^T b and Q b are plain products instead of a chain of k dependent reflector
// steps; L as H2Pack stores it (m x m row-major).  Triangular solves run in blocks of
// 32 rows: the CTA's warps compute the off-diagonal products of a block (row segments
// read contiguously), one warp solves the 32 x 32 diagonal block from shared memory.
// FP64 throughout; every sum has a fixed order, so results are deterministic.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "h2gpu.h"

#define H2G_API extern "C" __attribute__((visibility("default")))

namespace h2gpu {
int set_error(int code, const char* msg);
}

namespace {

constexpr int kUT = 256, kUW = kUT / 32;   // threads and warps of a node's CTA
constexpr int kDiag = 32 * 33;             // diagonal block in shared memory (padded)
constexpr int kMaxSmem = 227 * 1024;

struct UlvNode {
    long long q_off;     // Q^T (m x m row-major) in the Q arena; -1: no Q
    long long l_off;     // L (m x m row-major) in the L arena
    long long idx_off;   // m indices into the permuted vector
    long long p_off;     // LU: m - I pivots; -1: none
    int m, I, pad0, pad1;
};

struct UlvQJob {
    long long v_off;     // k reflectors of length m, reflector j at v + j m (1 at j,
                         // zeros above), then tau (k entries)
    long long q_off;
    int m, k, pad0, pad1;
};

enum { CH_UP = 0, CH_DOWN = 1, LU_UP = 2, LU_DOWN = 3 };

__device__ __forceinline__ double warp_sum(double s)
{
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// y[r] (+)= alpha sum_c A[r lda + c] x[c], r < nr, c < nc: one warp per row.  The
// caller synchronises before (x ready) and after.
__device__ void gemv_rows(const double* __restrict__ A, int lda, int nr, int nc, const double* x, double* y,
                          double alpha, bool acc)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r = warp; r < nr; r += kUW)
    {
        const double* a = A + (long long) r * lda;
        double s = 0.0;
        for (int c = lane; c < nc; c += 32) s += a[c] * x[c];
        s = warp_sum(s);
        if (lane == 0) y[r] = acc ? y[r] + alpha * s : alpha * s;
    }
}

// y[c] (+)= alpha sum_r A[r lda + c] x[r], c < nc, r < nr: one thread per column
// (consecutive threads read consecutive entries of a row).
__device__ void gemv_cols(const double* __restrict__ A, int lda, int nr, int nc, const double* x, double* y,
                          double alpha, bool acc)
{
    for (int c = threadIdx.x; c < nc; c += kUT)
    {
        double s = 0.0;
        for (int r = 0; r < nr; r++) s += A[(long long) r * lda + c] * x[r];
        y[c] = acc ? y[c] + alpha * s : alpha * s;
    }
}

// the diagonal block T[r0 .. r0 + bs)^2 into sD (row i at sD + 33 i)
__device__ void load_diag(const double* __restrict__ T, int ld, int r0, int bs, double* sD)
{
    for (int e = threadIdx.x; e < bs * 32; e += kUT)
    {
        const int i = e >> 5, j = e & 31;
        if (j < bs) sD[i * 33 + j] = T[(long long) (r0 + i) * ld + r0 + j];
    }
}

// x = T \ x, T lower triangular (row-major, ld), unit diagonal if `unit`
__device__ void trsv_lower(const double* __restrict__ T, int ld, int n, double* x, bool unit, double* sD)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r0 = 0; r0 < n; r0 += 32)
    {
        const int bs = min(32, n - r0);
        for (int i = warp; i < bs; i += kUW)
        {
            const double* t = T + (long long) (r0 + i) * ld;
            double s = 0.0;
            for (int c = lane; c < r0; c += 32) s += t[c] * x[c];
            s = warp_sum(s);
            if (lane == 0) x[r0 + i] -= s;
        }
        load_diag(T, ld, r0, bs, sD);
        __syncthreads();
        if (warp == 0)
        {
            double v = lane < bs ? x[r0 + lane] : 0.0;
            for (int j = 0; j < bs; j++)
            {
                double xj = __shfl_sync(0xffffffffu, v, j);
                if (!unit) xj = xj / sD[j * 33 + j];
                if (lane == j) v = xj;
                if (lane > j && lane < bs) v -= sD[lane * 33 + j] * xj;
            }
            if (lane < bs) x[r0 + lane] = v;
        }
        __syncthreads();
    }
}

// x = T \ x, T upper triangular (row-major, ld), non-unit diagonal
__device__ void trsv_upper(const double* __restrict__ T, int ld, int n, double* x, double* sD)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r0 = ((n - 1) / 32) * 32; n > 0 && r0 >= 0; r0 -= 32)
    {
        const int bs = min(32, n - r0), r1 = r0 + bs;
        for (int i = warp; i < bs; i += kUW)
        {
            const double* t = T + (long long) (r0 + i) * ld;
            double s = 0.0;
            for (int c = r1 + lane; c < n; c += 32) s += t[c] * x[c];
            s = warp_sum(s);
            if (lane == 0) x[r0 + i] -= s;
        }
        load_diag(T, ld, r0, bs, sD);
        __syncthreads();
        if (warp == 0)
        {
            double v = lane < bs ? x[r0 + lane] : 0.0;
            for (int j = bs - 1; j >= 0; j--)
            {
                const double xj = __shfl_sync(0xffffffffu, v, j) / sD[j * 33 + j];
                if (lane == j) v = xj;
                if (lane < j) v -= sD[lane * 33 + j] * xj;
            }
            if (lane < bs) x[r0 + lane] = v;
        }
        __syncthreads();
    }
}

// x = T^T \ x, T lower triangular (row-major, ld), non-unit diagonal: the products of
// a block's rows are sums over later rows c of T[c, r0 .. r0 + 32) x[c], each warp
// taking every 8th c (contiguous 32-entry segments), summed over warps in order
__device__ void trsv_lower_t(const double* __restrict__ T, int ld, int n, double* x, double* sD, double* sP)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int r0 = ((n - 1) / 32) * 32; n > 0 && r0 >= 0; r0 -= 32)
    {
        const int bs = min(32, n - r0), r1 = r0 + bs;
        double s = 0.0;
        if (lane < bs)
            for (int c = r1 + warp; c < n; c += kUW) s += T[(long long) c * ld + r0 + lane] * x[c];
        sP[warp * 32 + lane] = s;
        load_diag(T, ld, r0, bs, sD);
        __syncthreads();
        if (warp == 0)
        {
            double v = 0.0;
            if (lane < bs)
            {
                double p = 0.0;
                for (int w = 0; w < kUW; w++) p += sP[w * 32 + lane];
                v = x[r0 + lane] - p;
            }
            for (int j = bs - 1; j >= 0; j--)
            {
                const double xj = __shfl_sync(0xffffffffu, v, j) / sD[j * 33 + j];
                if (lane == j) v = xj;
                if (lane < j) v -= sD[j * 33 + lane] * xj;
            }
            if (lane < bs) x[r0 + lane] = v;
        }
        __syncthreads();
    }
}

// one level of one sweep: CTA b takes node list[b]
template <int MODE>
__global__ void __launch_bounds__(kUT) k_ulv_level(const UlvNode* __restrict__ nodes, const int* __restrict__ list,
                                                   int m_cap, const double* __restrict__ Qt,
                                                   const double* __restrict__ Lf, const int* __restrict__ idxs,
                                                   const int* __restrict__ piv, double* __restrict__ px)
{
    extern __shared__ __align__(16) double ulv_sm[];
    const UlvNode N = nodes[list[blockIdx.x]];
    const int m = N.m, I = N.I, n2 = m - I;
    double* const sb = ulv_sm;
    double* const st = sb + m_cap;
    double* const sD = st + m_cap;
    double* const sP = sD + kDiag;
    const int* const idx = idxs + N.idx_off;
    const double* const L = Lf + N.l_off;
    const double* const Q = N.q_off >= 0 ? Qt + N.q_off : nullptr;
    if (MODE == CH_UP || MODE == LU_UP)
    {
        if (Q)
        {
            for (int i = threadIdx.x; i < m; i += kUT) st[i] = px[idx[i]];
            __syncthreads();
            gemv_rows(Q, m, m, m, st, sb, 1.0, false);   // Q^T b
        } else {
            for (int i = threadIdx.x; i < m; i += kUT) sb[i] = px[idx[i]];
        }
        __syncthreads();
        if (MODE == LU_UP)
        {
            const int* const p = piv + N.p_off;
            for (int j = threadIdx.x; j < n2; j += kUT) st[j] = sb[I + j];
            __syncthreads();
            for (int j = threadIdx.x; j < n2; j += kUT) sb[I + j] = st[p[j]];
            __syncthreads();
        }
        trsv_lower(L + (long long) I * m + I, m, n2, sb + I, MODE == LU_UP, sD);
        gemv_rows(L + I, m, I, n2, sb + I, sb, -1.0, true);   // b1 -= L12 b2 (DU12 b2)
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += kUT) px[idx[i]] = sb[i];
    } else {
        for (int i = threadIdx.x; i < m; i += kUT) sb[i] = px[idx[i]];
        __syncthreads();
        if (MODE == CH_DOWN)
        {
            gemv_cols(L + I, m, I, n2, sb, sb + I, -1.0, true);   // b2 -= L12^T b1
            __syncthreads();
            trsv_lower_t(L + (long long) I * m + I, m, n2, sb + I, sD, sP);
        } else {
            gemv_rows(L + (long long) I * m, m, n2, I, sb, sb + I, -1.0, true);   // b2 -= LD21 b1
            __syncthreads();
            trsv_upper(L + (long long) I * m + I, m, n2, sb + I, sD);
        }
        if (Q)
        {
            gemv_cols(Q, m, m, m, sb, st, 1.0, false);   // Q b
            __syncthreads();
            for (int i = threadIdx.x; i < m; i += kUT) px[idx[i]] = st[i];
        } else {
            for (int i = threadIdx.x; i < m; i += kUT) px[idx[i]] = sb[i];
        }
    }
}

// Q^T of each job: warp w of CTA (x, y) forms column c = 8 x + w of job y's Q, i.e.
// Q e_c = H(0) H(1) .. H(k-1) e_c, into row c of Q^T
__global__ void __launch_bounds__(kUT) k_ulv_form_q(const UlvQJob* __restrict__ jobs, const double* __restrict__ V,
                                                    double* __restrict__ Qt)
{
    const UlvQJob J = jobs[blockIdx.y];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * kUW + warp;
    if (c >= J.m) return;
    const int m = J.m;
    double* const x = Qt + J.q_off + (long long) c * m;
    for (int i = lane; i < m; i += 32) x[i] = i == c ? 1.0 : 0.0;
    __syncwarp();
    const double* const v = V + J.v_off;
    const double* const tau = v + (long long) J.k * m;
    for (int j = J.k - 1; j >= 0; j--)
    {
        const double* const vj = v + (long long) j * m;
        double s = 0.0;
        for (int i = j + lane; i < m; i += 32) s += vj[i] * x[i];
        s = warp_sum(s) * tau[j];
        for (int i = j + lane; i < m; i += 32) x[i] -= s * vj[i];
        __syncwarp();
    }
}

__global__ void k_ulv_gather(int n, const double* __restrict__ src, const int* __restrict__ map,
                             double* __restrict__ dst)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[map[i]];
}

int smem_bytes(int m_cap) { return (int) sizeof(double) * (2 * m_cap + kDiag + kUW * 32); }

}  // namespace

struct h2gpu_ulv {
    int lu = 0, device = 0, n = 0, max_level = 0, m_cap = 0;
    cudaStream_t stream = nullptr;
    std::vector<int> lvl_off;            // max_level + 2 offsets into the node list
    UlvNode* d_nodes = nullptr;
    int* d_list = nullptr;
    double *d_Q = nullptr, *d_L = nullptr, *d_px = nullptr, *d_b = nullptr, *d_x = nullptr;
    int *d_idx = nullptr, *d_p = nullptr, *d_fwd = nullptr, *d_bwd = nullptr;
    size_t bytes = 0;
};

namespace {

int ulv_fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int ulv_fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return h2gpu::set_error(code, buf);
}

int cuda_status(cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return H2GPU_OK;
    return ulv_fail(e == cudaErrorMemoryAllocation ? H2GPU_ERR_NOMEM : H2GPU_ERR_CUDA, "ULV %s: %s", what,
                    cudaGetErrorString(e));
}

void free_ulv(h2gpu_ulv* u)
{
    for (void* p : {(void*) u->d_nodes, (void*) u->d_list, (void*) u->d_Q, (void*) u->d_L, (void*) u->d_px,
                    (void*) u->d_b, (void*) u->d_x, (void*) u->d_idx, (void*) u->d_p, (void*) u->d_fwd,
                    (void*) u->d_bwd})
        if (p) cudaFree(p);
    if (u->stream) cudaStreamDestroy(u->stream);
    delete u;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int enqueue_solve(h2gpu_ulv* u, int op, const double* d_b, double* d_x, cudaStream_t st)
{
    const int gb = std::max(1, std::min((u->n + 255) / 256, 4096));
    k_ulv_gather<<<gb, 256, 0, st>>>(u->n, d_b, u->d_fwd, u->d_px);
    const int sm = smem_bytes(u->m_cap);
    auto level = [&](int mode, int l) {
        const int cnt = u->lvl_off[l + 1] - u->lvl_off[l];
        if (cnt <= 0) return;
        const int* list = u->d_list + u->lvl_off[l];
        switch (mode)
        {
            case CH_UP:   k_ulv_level<CH_UP><<<cnt, kUT, sm, st>>>(u->d_nodes, list, u->m_cap, u->d_Q, u->d_L, u->d_idx, u->d_p, u->d_px); break;
            case CH_DOWN: k_ulv_level<CH_DOWN><<<cnt, kUT, sm, st>>>(u->d_nodes, list, u->m_cap, u->d_Q, u->d_L, u->d_idx, u->d_p, u->d_px); break;
            case LU_UP:   k_ulv_level<LU_UP><<<cnt, kUT, sm, st>>>(u->d_nodes, list, u->m_cap, u->d_Q, u->d_L, u->d_idx, u->d_p, u->d_px); break;
            default:      k_ulv_level<LU_DOWN><<<cnt, kUT, sm, st>>>(u->d_nodes, list, u->m_cap, u->d_Q, u->d_L, u->d_idx, u->d_p, u->d_px); break;
        }
    };
    if (op & 1)
        for (int l = u->max_level; l >= 0; l--) level(u->lu ? LU_UP : CH_UP, l);
    if (op & 2)
        for (int l = 0; l <= u->max_level; l++) level(u->lu ? LU_DOWN : CH_DOWN, l);
    k_ulv_gather<<<gb, 256, 0, st>>>(u->n, u->d_px, u->d_bwd, d_x);
    return cuda_status(cudaGetLastError(), "solve launch");
}

}  // namespace

H2G_API int h2gpu_ulv_create(const h2gpu_ulv_desc* d, h2gpu_ulv** out)
{
    if (!out) return ulv_fail(H2GPU_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!d || d->n_node <= 0 || d->max_level < 0 || d->n_leaf_node <= 0 || d->krnl_mat_size <= 0 ||
        !d->level_n_node || !d->level_nodes || !d->fwd_pmt_idx || !d->bwd_pmt_idx || !d->Ls || !d->m ||
        !d->q_ncol || !d->l_ld || !d->idx || !d->Q || !d->L || (d->lu && !d->p))
        return ulv_fail(H2GPU_ERR_INVALID, "malformed ULV descriptor");
    const int n = d->krnl_mat_size;
    for (int i = 0; i < n; i++)
        if (d->fwd_pmt_idx[i] < 0 || d->fwd_pmt_idx[i] >= n || d->bwd_pmt_idx[i] < 0 || d->bwd_pmt_idx[i] >= n)
            return ulv_fail(H2GPU_ERR_INVALID, "permutation entry %d out of range", i);
    // nodes in level order, and their arena offsets
    std::vector<int> list, lvl_off(1, 0), level_of(d->n_node, -1);
    for (int l = 0; l <= d->max_level; l++)
    {
        const int cnt = d->level_n_node[l];
        if (cnt < 0 || cnt > d->n_leaf_node) return ulv_fail(H2GPU_ERR_INVALID, "level %d: %d nodes", l, cnt);
        if (l == 0 && cnt != 1) return ulv_fail(H2GPU_ERR_INVALID, "level 0 must hold the root alone");
        for (int j = 0; j < cnt; j++)
        {
            const int node = d->level_nodes[(size_t) l * d->n_leaf_node + j];
            if (node < 0 || node >= d->n_node || level_of[node] >= 0)
                return ulv_fail(H2GPU_ERR_INVALID, "level %d: bad or repeated node %d", l, node);
            level_of[node] = l;
            list.push_back(node);
        }
        lvl_off.push_back((int) list.size());
    }
    std::vector<UlvNode> nodes(d->n_node);
    std::vector<UlvQJob> jobs;
    long long nq = 0, nl = 0, ni = 0, np = 0, nv = 0;
    int m_cap = 1;
    for (int node : list)
    {
        const int m = d->m[node], I = d->Ls[node], k = d->q_ncol[node];
        const bool root = level_of[node] == 0;
        if (m < 0 || I < 0 || I > m) return ulv_fail(H2GPU_ERR_INVALID, "node %d: m %d, Ls %d", node, m, I);
        if (m > 0 && (!d->idx[node] || !d->L[node] || d->l_ld[node] < m))
            return ulv_fail(H2GPU_ERR_INVALID, "node %d: factor or index set missing", node);
        for (int i = 0; i < m; i++)
            if (d->idx[node][i] < 0 || d->idx[node][i] >= n)
                return ulv_fail(H2GPU_ERR_INVALID, "node %d: index %d out of range", node, d->idx[node][i]);
        UlvNode& N = nodes[node];
        N.m = m; N.I = I; N.pad0 = N.pad1 = 0;
        N.l_off = nl; nl += (long long) m * m;
        N.idx_off = ni; ni += m;
        N.q_off = -1;
        N.p_off = -1;
        if (!root && k > 0 && m > 0)
        {
            if (k > m) return ulv_fail(H2GPU_ERR_UNSUPPORTED, "node %d: %d reflectors of length %d", node, k, m);
            if (!d->Q[node]) return ulv_fail(H2GPU_ERR_INVALID, "node %d: Q missing", node);
            N.q_off = nq; nq += (long long) m * m;
            jobs.push_back(UlvQJob{nv, N.q_off, m, k, 0, 0});
            nv += (long long) k * m + k;
        }
        if (d->lu)
        {
            if (m - I > 0 && !d->p[node]) return ulv_fail(H2GPU_ERR_INVALID, "node %d: pivots missing", node);
            for (int j = 0; j < m - I; j++)
                if (d->p[node][j] < 0 || d->p[node][j] >= m - I)
                    return ulv_fail(H2GPU_ERR_INVALID, "node %d: pivot %d out of range", node, d->p[node][j]);
            N.p_off = np; np += m - I;
        }
        m_cap = std::max(m_cap, m);
    }
    for (int i = 0; i < d->n_node; i++)
        if (level_of[i] < 0) { nodes[i].m = 0; nodes[i].I = 0; nodes[i].q_off = nodes[i].p_off = -1; }
    if (smem_bytes(m_cap) > kMaxSmem)
        return ulv_fail(H2GPU_ERR_UNSUPPORTED, "a node of %d rows exceeds one CTA's shared memory", m_cap);
    int dev = d->device;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return ulv_fail(H2GPU_ERR_CUDA, "no CUDA device");
    DeviceGuard guard(dev);
    h2gpu_ulv* u = new h2gpu_ulv;
    u->lu = d->lu ? 1 : 0; u->device = dev; u->n = n; u->max_level = d->max_level; u->m_cap = m_cap;
    u->lvl_off = lvl_off;
    // host staging of the small arrays and of the reflectors (transposed: reflector j
    // contiguous, with its implicit 1 and the zeros above it written out)
    std::vector<int> hidx((size_t) std::max<long long>(ni, 1)), hp((size_t) std::max<long long>(np, 1));
    std::vector<double> hv((size_t) std::max<long long>(nv, 1));
    size_t ji = 0;
    for (int node : list)
    {
        const UlvNode& N = nodes[node];
        if (N.m > 0) memcpy(&hidx[N.idx_off], d->idx[node], sizeof(int) * N.m);
        if (N.p_off >= 0 && N.m - N.I > 0) memcpy(&hp[N.p_off], d->p[node], sizeof(int) * (N.m - N.I));
        if (N.q_off >= 0)
        {
            const UlvQJob& J = jobs[ji++];
            const double* A = d->Q[node];
            const int m = J.m, k = J.k;
            double* v = &hv[J.v_off];
            for (int j = 0; j < k; j++)
                for (int i = 0; i < m; i++)
                    v[(size_t) j * m + i] = i < j ? 0.0 : i == j ? 1.0 : A[(size_t) i * k + j];
            for (int j = 0; j < k; j++) v[(size_t) k * m + j] = A[(size_t) m * k + j];   // tau: the last row
        }
    }
    double* d_v = nullptr;
    UlvQJob* d_jobs = nullptr;
    int st = H2GPU_OK;
    auto step = [&](cudaError_t e, const char* what) {
        if (st == H2GPU_OK) st = cuda_status(e, what);
        return st == H2GPU_OK;
    };
    auto alloc = [&](void** p, size_t b) {
        if (!step(cudaMalloc(p, std::max<size_t>(b, 16)), "device allocation")) return false;
        u->bytes += std::max<size_t>(b, 16);
        return true;
    };
    if (step(cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking), "stream") &&
        alloc((void**) &u->d_nodes, sizeof(UlvNode) * nodes.size()) &&
        alloc((void**) &u->d_list, sizeof(int) * list.size()) &&
        alloc((void**) &u->d_Q, 8 * (size_t) nq) && alloc((void**) &u->d_L, 8 * (size_t) nl) &&
        alloc((void**) &u->d_idx, 4 * (size_t) ni) && alloc((void**) &u->d_p, 4 * (size_t) np) &&
        alloc((void**) &u->d_fwd, 4 * (size_t) n) && alloc((void**) &u->d_bwd, 4 * (size_t) n) &&
        alloc((void**) &u->d_px, 8 * (size_t) n) && alloc((void**) &u->d_b, 8 * (size_t) n) &&
        alloc((void**) &u->d_x, 8 * (size_t) n) &&
        step(cudaMemcpy(u->d_nodes, nodes.data(), sizeof(UlvNode) * nodes.size(), cudaMemcpyHostToDevice), "upload") &&
        step(cudaMemcpy(u->d_list, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice), "upload") &&
        step(cudaMemcpy(u->d_idx, hidx.data(), 4 * (size_t) ni, cudaMemcpyHostToDevice), "upload") &&
        step(np ? cudaMemcpy(u->d_p, hp.data(), 4 * (size_t) np, cudaMemcpyHostToDevice) : cudaSuccess, "upload") &&
        step(cudaMemcpy(u->d_fwd, d->fwd_pmt_idx, 4 * (size_t) n, cudaMemcpyHostToDevice), "upload") &&
        step(cudaMemcpy(u->d_bwd, d->bwd_pmt_idx, 4 * (size_t) n, cudaMemcpyHostToDevice), "upload"))
    {
        for (int node : list)
        {
            const UlvNode& N = nodes[node];
            if (N.m == 0) continue;
            if (!step(cudaMemcpy2D(u->d_L + N.l_off, 8 * (size_t) N.m, d->L[node], 8 * (size_t) d->l_ld[node],
                                   8 * (size_t) N.m, (size_t) N.m, cudaMemcpyHostToDevice), "factor upload"))
                break;
        }
    }
    if (st == H2GPU_OK && !jobs.empty() && step(cudaMalloc(&d_v, 8 * (size_t) nv), "reflector staging") &&
        step(cudaMalloc(&d_jobs, sizeof(UlvQJob) * jobs.size()), "reflector staging") &&
        step(cudaMemcpy(d_v, hv.data(), 8 * (size_t) nv, cudaMemcpyHostToDevice), "reflector upload") &&
        step(cudaMemcpy(d_jobs, jobs.data(), sizeof(UlvQJob) * jobs.size(), cudaMemcpyHostToDevice), "reflector upload"))
    {
        int mq = 1;
        for (const UlvQJob& J : jobs) mq = std::max(mq, J.m);
        for (size_t j0 = 0; j0 < jobs.size() && st == H2GPU_OK; j0 += 65535)
        {
            const unsigned cnt = (unsigned) std::min<size_t>(65535, jobs.size() - j0);
            k_ulv_form_q<<<dim3((unsigned) ((mq + kUW - 1) / kUW), cnt), kUT, 0, u->stream>>>(d_jobs + j0, d_v, u->d_Q);
            step(cudaGetLastError(), "forming Q");
        }
        step(cudaStreamSynchronize(u->stream), "forming Q");
    }
    if (d_v) cudaFree(d_v);
    if (d_jobs) cudaFree(d_jobs);
    if (st == H2GPU_OK)
    {
        // The limit is a per-function setting of the process: it is set to the device's
        // opt-in maximum, the same value for every object, so that creating a
        // factorization with smaller nodes never lowers it under another's launches.
        int optin = 0;
        if (step(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "device query") &&
            smem_bytes(m_cap) > optin)
            st = ulv_fail(H2GPU_ERR_UNSUPPORTED, "a node of %d rows exceeds one CTA's shared memory", m_cap);
        for (auto kern : {k_ulv_level<CH_UP>, k_ulv_level<CH_DOWN>, k_ulv_level<LU_UP>, k_ulv_level<LU_DOWN>})
            if (st == H2GPU_OK)
                step(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin),
                     "shared memory of the solve kernels");
    }
    if (st != H2GPU_OK)
    {
        free_ulv(u);
        return st;
    }
    *out = u;
    return H2GPU_OK;
}

H2G_API int h2gpu_ulv_destroy(h2gpu_ulv* u)
{
    if (!u) return H2GPU_OK;
    DeviceGuard guard(u->device);
    cudaStreamSynchronize(u->stream);
    free_ulv(u);
    return H2GPU_OK;
}

H2G_API int h2gpu_ulv_solve_device(h2gpu_ulv* u, int op, const double* d_b, double* d_x, void* stream)
{
    if (!u || !d_b || !d_x) return ulv_fail(H2GPU_ERR_INVALID, "ULV solve: NULL argument");
    if (op < 1 || op > 3) return ulv_fail(H2GPU_ERR_INVALID, "ULV solve: op %d, should be 1, 2 or 3", op);
    DeviceGuard guard(u->device);
    return enqueue_solve(u, op, d_b, d_x, stream ? (cudaStream_t) stream : u->stream);
}

H2G_API int h2gpu_ulv_solve(h2gpu_ulv* u, int op, const double* b, double* x)
{
    if (!u || !b || !x) return ulv_fail(H2GPU_ERR_INVALID, "ULV solve: NULL argument");
    if (op < 1 || op > 3) return ulv_fail(H2GPU_ERR_INVALID, "ULV solve: op %d, should be 1, 2 or 3", op);
    DeviceGuard guard(u->device);
    const size_t nb = 8 * (size_t) u->n;
    int st = cuda_status(cudaMemcpyAsync(u->d_b, b, nb, cudaMemcpyHostToDevice, u->stream), "upload");
    if (st == H2GPU_OK) st = enqueue_solve(u, op, u->d_b, u->d_x, u->stream);
    if (st == H2GPU_OK) st = cuda_status(cudaMemcpyAsync(x, u->d_x, nb, cudaMemcpyDeviceToHost, u->stream), "download");
    const int s2 = cuda_status(cudaStreamSynchronize(u->stream), "solve");
    return st != H2GPU_OK ? st : s2;
}

H2G_API size_t h2gpu_ulv_bytes(const h2gpu_ulv* u) { return u ? u->bytes : 0; }
