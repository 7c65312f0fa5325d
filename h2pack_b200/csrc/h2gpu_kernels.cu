// h2gpu_kernels.cu -- sm_100a kernels of the H2 apply engine.
//
// Phases (reference: H2P_matvec, src/H2Pack_matvec.c:1162-1284; H2P_matmul,
// src/H2Pack_matmul.c:455-583):
//   k_gather      forward permutation of the input panel into XS          (matvec.c:1174-1179)
//   k_up          upward sweep y0 = U^T x, one CTA per node                 (matvec.c:95-177)
//   k_blk         stored B / D block chunks, one read feeds A*v and A^T*w  (matvec.c:303-437, 864-998)
//   k_jit         on-the-fly B / D kernel blocks, owner computes           (matvec.c:586-764, 1002-1145)
//   k_down        downward sweep U * y1 with slot sums and push-down       (matvec.c:767-861)
//   k_asm         sum of a leaf's partial slots + backward permutation     (matvec.c:1251-1278)
//   k_direct      FP64 direct sum (examples/direct_nbody.h:2-54)
// All right-hand-side panels are NV wide (NV in {1,2,4,8,16}); vector spaces are
// row-major with row stride NV.  Sums inside one block use the block's warps; sums
// across blocks go through PS slots in a fixed order, so results are bitwise
// reproducible run to run.
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include "h2gpu_internal.cuh"
#include "h2gpu_launch.h"

namespace h2gpu {

constexpr int kWarps = 8;               // warps per CTA of the sweep / block kernels
constexpr int kThreads = kWarps * 32;
constexpr unsigned kFull = 0xffffffffu;

template <int NV> struct SV { static constexpr int v = (NV > 1) ? NV + 1 : 1; };  // padded smem row stride

// A stored-block task's offset and row stride in the arena of element type TA (the FP32
// arena pads its rows, BlkTask)
template <typename TA>
__device__ __forceinline__ long long blk_off(const BlkTask& T)
{
    if constexpr (sizeof(TA) == 4) return T.a32;
    else return T.a_off;
}
template <typename TA>
__device__ __forceinline__ int blk_ld(const BlkTask& T)
{
    if constexpr (sizeof(TA) == 4) return T.ld32;
    else return T.ncol;
}

__device__ __forceinline__ double to_d(double x) { return x; }
__device__ __forceinline__ double to_d(float x) { return (double) x; }

// Reduce NV per-lane values over the 32 lanes of a warp.  After the call a[0] of
// lane l holds the warp sum for right-hand side v = nv_of_lane(l); the lanes with
// (lane & (32/NV - 1)) == 0 hold distinct v.  Uses NV-1 + log2(32/NV) shuffles.
template <int NV>
__device__ __forceinline__ void warp_transpose_reduce(double (&a)[NV], int lane)
{
    int m = NV;
    int o = 16;
#pragma unroll
    for (int s = 0; (1 << s) < NV; s++)
    {
        const int half = m >> 1;
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < NV / 2; i++)
        {
            if (i < half)
            {
                double send = up ? a[i] : a[i + half];
                double keep = up ? a[i + half] : a[i];
                double recv = __shfl_xor_sync(kFull, send, o);
                a[i] = keep + recv;
            }
        }
        m = half;
        o >>= 1;
    }
#pragma unroll
    for (; o >= 1; o >>= 1) a[0] += __shfl_xor_sync(kFull, a[0], o);
}

template <int NV>
__device__ __forceinline__ int nv_of_lane(int lane)
{
    // bits of v from MSB: lane bit 16 -> v bit log2(NV)-1, lane bit 8 -> next, ...
    int v = 0, o = 16;
#pragma unroll
    for (int s = 0; (1 << s) < NV; s++) { v = (v << 1) | ((lane & o) ? 1 : 0); o >>= 1; }
    return v;
}

template <int NV>
__device__ __forceinline__ bool lane_writes(int lane) { return (lane & (32 / NV - 1)) == 0; }

// ------------------------------------------------------------------ gather

// XS[r][v] = X[fwd[r]][v] (v < nv), zero-padded to NV columns.
template <int NV>
__global__ void k_gather(const double* __restrict__ X, long long x_rs, long long x_cs, int nv,
                         const int* __restrict__ fwd, int N, double* __restrict__ XS)
{
    long long total = (long long) N * NV;
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < total;
         i += (long long) gridDim.x * blockDim.x)
    {
        int r = (int) (i / NV), v = (int) (i % NV);
        XS[i] = (v < nv) ? X[(long long) fwd[r] * x_rs + (long long) v * x_cs] : 0.0;
    }
}

// Y[i][v] = X[idx[i]][v] for general strides (H2P_permute_* on device)
__global__ void k_permute(const double* __restrict__ X, long long x_rs, long long x_cs, const int* __restrict__ idx,
                          int n, int nv, double* __restrict__ Y, long long y_rs, long long y_cs)
{
    long long total = (long long) n * nv;
    for (long long i = blockIdx.x * (long long) blockDim.x + threadIdx.x; i < total;
         i += (long long) gridDim.x * blockDim.x)
    {
        int r = (int) (i / nv), v = (int) (i % nv);
        Y[(long long) r * y_rs + (long long) v * y_cs] = X[(long long) idx[r] * x_rs + (long long) v * x_cs];
    }
}

// ---------------------------------------------------------------- upward

// y0 = U^T w for one column tile (<= 64 columns) of a node per CTA (narrow panels).
// Lane l owns columns c0 + l and c0 + 32 + l; warp w takes rows w, w + 8, ... of each
// 256-row chunk of the node's rows, eight rows per step (16 loads in flight per lane);
// the chunk's inputs are staged in shared memory first, and the 8 warps' column sums
// are added in warp order at the end.
template <typename TA, int NV>
__global__ void __launch_bounds__(kThreads) k_up(const UpTask* __restrict__ tasks, const TA* __restrict__ Uar,
                                                 double* __restrict__ XS)
{
    constexpr int RC = 256;
    __shared__ double s_w[RC * NV];
    __shared__ double s_red[kWarps][64][NV];
    const UpTask t = tasks[blockIdx.x];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const TA* U = Uar + t.u_off;
    const int cend = t.c0 + t.nc, ca = t.c0 + lane, cb = ca + 32;
    const bool va = ca < cend, vb = cb < cend;
    double acc[2][NV];
#pragma unroll
    for (int v = 0; v < NV; v++) { acc[0][v] = 0.0; acc[1][v] = 0.0; }
    for (int rc = 0; rc < t.nrow; rc += RC)
    {
        const int nr = min(RC, t.nrow - rc);
        __syncthreads();
        for (int i = threadIdx.x; i < nr * NV; i += kThreads) s_w[i] = XS[(long long) (t.in_row + rc) * NV + i];
        __syncthreads();
        int r = w;
        for (; r + 56 < nr; r += 64)
        {
            TA a[8], b[8];
#pragma unroll
            for (int k = 0; k < 8; k++)
            {
                const TA* row = U + (long long) (rc + r + 8 * k) * t.ld;
                a[k] = va ? row[ca] : TA(0);
                b[k] = vb ? row[cb] : TA(0);
            }
#pragma unroll
            for (int k = 0; k < 8; k++)
#pragma unroll
                for (int v = 0; v < NV; v++)
                {
                    const double x = s_w[(r + 8 * k) * NV + v];
                    acc[0][v] = fma(to_d(a[k]), x, acc[0][v]);
                    acc[1][v] = fma(to_d(b[k]), x, acc[1][v]);
                }
        }
        for (; r < nr; r += 8)
        {
            const TA* row = U + (long long) (rc + r) * t.ld;
            const double a = va ? to_d(row[ca]) : 0.0, b = vb ? to_d(row[cb]) : 0.0;
#pragma unroll
            for (int v = 0; v < NV; v++)
            {
                acc[0][v] = fma(a, s_w[r * NV + v], acc[0][v]);
                acc[1][v] = fma(b, s_w[r * NV + v], acc[1][v]);
            }
        }
    }
#pragma unroll
    for (int v = 0; v < NV; v++) { s_red[w][lane][v] = acc[0][v]; s_red[w][lane + 32][v] = acc[1][v]; }
    __syncthreads();
    for (int i = threadIdx.x; i < t.nc * NV; i += kThreads)
    {
        const int cc = i / NV, v = i % NV;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < kWarps; k++) s += s_red[k][cc][v];
        XS[(long long) (t.out_row + t.c0 + cc) * NV + v] = s;
    }
}

// Sweep products for panels of NV >= 4 right-hand sides as small tiled GEMMs:
//   upward   (UP):  C[m][v] = sum_k U[k][c0 + m] * XS[in_row + k][v]      (m < nc, a column tile)
//   downward (!UP): C[m][v] = sum_k U[r0 + m][k] * (Y1 + PUSH)[k][v]       (m < 64, a row chunk)
// A 64 x 32 tile of U and a 32 x NV tile of the right-hand sides are staged in shared
// memory per step (coalesced global reads along the contiguous index); each thread
// accumulates (NV * 64 / 256) outputs of one row in FP64.
template <typename TA, int NV, bool UP>
__global__ void __launch_bounds__(256) k_sweep_gemm(const UpTask* __restrict__ ups, const DownTask* __restrict__ dns,
                                                    const TA* __restrict__ Uar, double* __restrict__ XS,
                                                    const double* __restrict__ Y1, double* __restrict__ PS,
                                                    double* __restrict__ PUSH)
{
    constexpr int MT = 64, KT = 32;
    constexpr int VPT = (NV * MT) / 256;
    constexpr int NG = NV / VPT;
    static_assert(VPT >= 1 && NG * VPT == NV, "panel width");
    __shared__ double sA[KT][MT + 1];
    __shared__ double sB[KT][NV];
    const int t = threadIdx.x;
    const int m = t / NG, v0 = (t % NG) * VPT;
    int K, M, lda, brow = 0, y1_row = -1, push_row = -1;
    const TA* A;
    double* out;
    if constexpr (UP)
    {
        const UpTask T = ups[blockIdx.x];
        K = T.nrow; M = T.nc; lda = T.ld;
        A = Uar + T.u_off + T.c0;
        brow = T.in_row;
        out = XS + (long long) (T.out_row + T.c0) * NV;
    } else {
        const DownTask T = dns[blockIdx.x];
        K = T.ncol; M = T.nrow; lda = T.ld;
        A = Uar + T.u_off;
        y1_row = T.y1_row; push_row = T.push_row;
        out = (T.dst_ps ? PS : PUSH) + (long long) T.dst_row * NV;
    }
    double acc[VPT];
#pragma unroll
    for (int j = 0; j < VPT; j++) acc[j] = 0.0;
    for (int k0 = 0; k0 < K; k0 += KT)
    {
        __syncthreads();
        if constexpr (UP)
        {
            for (int i = t; i < KT * MT; i += 256)
            {
                int k = i / MT, mm = i % MT;
                sA[k][mm] = (k0 + k < K && mm < M) ? to_d(A[(long long) (k0 + k) * lda + mm]) : 0.0;
            }
            for (int i = t; i < KT * NV; i += 256)
            {
                int k = i / NV, v = i % NV;
                sB[k][v] = (k0 + k < K) ? XS[(long long) (brow + k0 + k) * NV + v] : 0.0;
            }
        } else {
            for (int i = t; i < KT * MT; i += 256)
            {
                int mm = i / KT, k = i % KT;
                sA[k][mm] = (k0 + k < K && mm < M) ? to_d(A[(long long) mm * lda + k0 + k]) : 0.0;
            }
            for (int i = t; i < KT * NV; i += 256)
            {
                int k = i / NV, v = i % NV;
                double b = 0.0;
                if (k0 + k < K)
                {
                    if (y1_row >= 0) b = Y1[(long long) (y1_row + k0 + k) * NV + v];
                    if (push_row >= 0) b += PUSH[(long long) (push_row + k0 + k) * NV + v];
                }
                sB[k][v] = b;
            }
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < KT; k++)
        {
            const double a = sA[k][m];
#pragma unroll
            for (int j = 0; j < VPT; j++) acc[j] = fma(a, sB[k][v0 + j], acc[j]);
        }
    }
    if (m < M)
#pragma unroll
        for (int j = 0; j < VPT; j++) out[(long long) m * NV + v0 + j] = acc[j];
}

// ------------------------------------------------- row-chunk block apply

// Input of the "A * v" product for a column tile: either rows of XS, or (downward
// sweep) the node's summed y1 plus the parent's push-down slice.
struct VFromXS {
    const double* XS; int row;
    __device__ double operator()(int c, int v, int NVs) const { return XS[(long long) (row + c) * NVs + v]; }
};
struct VFromY1 {
    const double* Y1; const double* PUSH; int y1_row, push_row;
    __device__ double operator()(int c, int v, int NVs) const
    {
        double s = (y1_row >= 0) ? Y1[(long long) (y1_row + c) * NVs + v] : 0.0;
        if (push_row >= 0) s += PUSH[(long long) (push_row + c) * NVs + v];
        return s;
    }
};

// One chunk of R <= 64 rows of a row-major block (ld = ncol):
//   out0[r][v] = sum_c A[r][c] vin[c][v]     (if out0 != nullptr)
//   out1[c][v] = sum_r A[r][c] win[r][v]     (if out1 != nullptr)
template <int NV>
constexpr int chunk_smem_bytes() { return 8 * (64 * SV<NV>::v + 32 * SV<NV>::v + 64 * NV + kWarps * 32 * NV); }

template <typename TA, int NV, typename VIN>
__device__ __forceinline__ void chunk_apply(const TA* __restrict__ A, int R, int ncol, int lda, VIN vin,
                                            const double* __restrict__ win_XS, int win_row,
                                            double* __restrict__ out0, double* __restrict__ out1,
                                            double* __restrict__ smem, bool add1 = false)
{
    constexpr int S = SV<NV>::v;
    double* s_w = smem;
    double* s_v = s_w + 64 * S;
    double* s_o0 = s_v + 32 * S;
    double (*s_red)[32][NV] = reinterpret_cast<double (*)[32][NV]>(s_o0 + 64 * NV);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool do0 = out0 != nullptr, do1 = out1 != nullptr;
    if (do1)
        for (int i = threadIdx.x; i < R * NV; i += kThreads)
            s_w[(i / NV) * S + (i % NV)] = win_XS[(long long) (win_row + i / NV) * NV + (i % NV)];
    for (int i = threadIdx.x; i < R * NV; i += kThreads) s_o0[i] = 0.0;
    for (int ct = 0; ct < ncol; ct += 32)
    {
        const int c = ct + lane;
        const bool cin = c < ncol;
        __syncthreads();
        if (do0)
            for (int i = threadIdx.x; i < 32 * NV; i += kThreads)
            {
                int cc = i / NV, v = i % NV;
                s_v[cc * S + v] = (ct + cc < ncol) ? vin(ct + cc, v, NV) : 0.0;
            }
        __syncthreads();
        double acc1[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) acc1[v] = 0.0;
        for (int r = w; r < R; r += kWarps)
        {
            double a = cin ? to_d(A[(long long) r * lda + c]) : 0.0;
            if (do1)
            {
#pragma unroll
                for (int v = 0; v < NV; v++) acc1[v] = fma(a, s_w[r * S + v], acc1[v]);
            }
            if (do0)
            {
                double p[NV];
#pragma unroll
                for (int v = 0; v < NV; v++) p[v] = a * s_v[lane * S + v];
                warp_transpose_reduce<NV>(p, lane);
                if (lane_writes<NV>(lane)) s_o0[r * NV + nv_of_lane<NV>(lane)] += p[0];
            }
        }
        if (do1)
        {
#pragma unroll
            for (int v = 0; v < NV; v++) s_red[w][lane][v] = acc1[v];
            __syncthreads();
            for (int i = threadIdx.x; i < 32 * NV; i += kThreads)
            {
                int cc = i / NV, v = i % NV;
                if (ct + cc < ncol)
                {
                    double s = 0.0;
#pragma unroll
                    for (int k = 0; k < kWarps; k++) s += s_red[k][cc][v];
                    double* o = out1 + (long long) (ct + cc) * NV + v;
                    *o = add1 ? *o + s : s;
                }
            }
        }
    }
    __syncthreads();
    if (do0)
        for (int i = threadIdx.x; i < R * NV; i += kThreads) out0[i] = s_o0[i];
}

// Stored blocks, single right-hand side (the matvec path, memory bound).  One launch.
// A task of at most 256 columns, 512 rows and 128 KB (blk1_fits: the B blocks of the
// usual leaf sizes, and their D blocks in FP32) is one warp's, 8 per CTA.  The lane owns
// columns lane + 32j; their A^T w sums (and, for FP32 blocks, their inputs) live in the
// warp's rows of shared memory for the whole block (only the lane touches its columns:
// no barrier; registers stay free for the loads in flight).  The rows are walked 8
// at a time with all of a pass's loads in flight (FP32: two 32-column passes, 16 loads
// per lane), and the 8 rows' A v partials are combined with one transposed butterfly.
// Every warp runs its own task, so 24 independent load chains per SM hide each other's
// latency (one CTA per task left long serial chains of task, input, block loads,
// barriers and output per ~100 KB block).  Larger tasks get a CTA each (blk1_cta): one
// warp per 200 KB FP64 block measured slower (fewer warps than slots in the last
// wave).  The plan orders each task list small-first; n_small is the count for TA.
// Sums: FP64 blocks in FP64; FP32 blocks in FP32 over one pass (8 rows, or the <= 8
// column passes of a row) and widened per sum.
template <typename TA>
__device__ __forceinline__ void blk1_warp(const BlkTask& T, const TA* __restrict__ arena,
                                          const double* __restrict__ XS, double* __restrict__ PS,
                                          double* __restrict__ sq, float* __restrict__ sv, int lane)
{
    constexpr bool F32 = sizeof(TA) == 4;
    constexpr int PASS = F32 ? 2 : 1;          // 32-column passes whose loads are issued together
    const int ncol = T.ncol, nrow = T.nrow;
    const bool do0 = T.out0_row >= 0, do1 = T.out1_row >= 0;
    const int J = (ncol + 31) >> 5;
    const TA* A = arena + blk_off<TA>(T);
    const int lda = blk_ld<TA>(T);
#pragma unroll
    for (int j = 0; j < 8; j++)
    {
        const int c = lane + 32 * j;
        sq[c] = 0.0;
        if constexpr (F32) sv[c] = (do0 && c < ncol) ? (float) XS[T.in0_row + c] : 0.f;
    }
    for (int r0 = 0; r0 < nrow; r0 += 8)
    {
        const int nr = min(8, nrow - r0);
        double wr[8];
#pragma unroll
        for (int k = 0; k < 8; k++) wr[k] = (do1 && k < nr) ? XS[T.in1_row + r0 + k] : 0.0;
        double p[8];
        float pf[8];
#pragma unroll
        for (int k = 0; k < 8; k++) { p[k] = 0.0; pf[k] = 0.f; }
#pragma unroll 1
        for (int j0 = 0; j0 < J; j0 += PASS)
        {
            TA a[PASS][8];
#pragma unroll
            for (int u = 0; u < PASS; u++)
            {
                const int c = lane + 32 * (j0 + u);
                const bool cv = c < ncol;
#pragma unroll
                for (int k = 0; k < 8; k++) a[u][k] = (cv && k < nr) ? A[(long long) (r0 + k) * lda + c] : TA(0);
            }
#pragma unroll
            for (int u = 0; u < PASS; u++)
            {
                const int j = j0 + u;
                if constexpr (F32)
                {
                    const float v = sv[lane + 32 * j];
                    float q = 0.f;
#pragma unroll
                    for (int k = 0; k < 8; k++)
                    {
                        q = fmaf(a[u][k], (float) wr[k], q);
                        pf[k] = fmaf(a[u][k], v, pf[k]);
                    }
                    sq[lane + 32 * j] += (double) q;
                } else {
                    const int c = lane + 32 * j;
                    const double v = (do0 && c < ncol) ? XS[T.in0_row + c] : 0.0;
                    double q = 0.0;
#pragma unroll
                    for (int k = 0; k < 8; k++)
                    {
                        q = fma(to_d(a[u][k]), wr[k], q);
                        p[k] = fma(to_d(a[u][k]), v, p[k]);
                    }
                    sq[lane + 32 * j] += q;
                }
            }
        }
        if (do0)
        {
            if constexpr (F32)
            {
#pragma unroll
                for (int k = 0; k < 8; k++) p[k] = (double) pf[k];
            }
            warp_transpose_reduce<8>(p, lane);
            const int row = nv_of_lane<8>(lane);
            if (lane_writes<8>(lane) && row < nr) PS[T.out0_row + r0 + row] = p[0];
        }
    }
    if (do1)
    {
#pragma unroll
        for (int j = 0; j < 8; j++)
        {
            const int c = lane + 32 * j;
            if (c < ncol) PS[T.out1_row + c] = sq[c];
        }
    }
}

// A task walked by the whole CTA (chunks of 64 rows; warp w owns rows 8w..8w+7 of a
// chunk and its lanes sweep the columns 32 at a time).  A v completes per lane across
// the sweep and is combined with one transposed butterfly per chunk; the 8 warps'
// partials of A^T w are summed in warp order through shared memory every 256 columns
// and added into the task's single out1 slot (stored by the first chunk, added by the
// later ones; the same thread owns the same column in every chunk).
template <typename TA>
__device__ __forceinline__ void blk1_cta(const BlkTask& T, const TA* __restrict__ arena,
                                         const double* __restrict__ XS, double* __restrict__ PS,
                                         double (*s_q)[256])
{
    constexpr int CPL = 1;
    constexpr int CW = 256;                       // columns per shared reduction of A^T w
    const int ncol = T.ncol, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool do0 = T.out0_row >= 0, do1 = T.out1_row >= 0;
    for (int rc = 0; rc < T.nrow; rc += 64)
    {
        const int nr = max(0, min(8, min(64, T.nrow - rc) - 8 * w));   // rows of this warp
        const int r0 = rc + 8 * w;
        const TA* A = arena + blk_off<TA>(T) + (long long) r0 * blk_ld<TA>(T);
        double wr[8];
#pragma unroll
        for (int k = 0; k < 8; k++) wr[k] = (do1 && k < nr) ? XS[T.in1_row + r0 + k] : 0.0;
        double p[8];
#pragma unroll
        for (int k = 0; k < 8; k++) p[k] = 0.0;
        for (int cw = 0; cw < ncol; cw += CW)
        {
            const int cend = min(ncol, cw + CW);
            // the out1 value this thread adds to after the window, read now so its latency
            // hides behind the window's loads (one column per thread: CW = blockDim)
            double o1 = 0.0;
            if (do1 && rc > 0 && threadIdx.x < cend - cw) o1 = PS[T.out1_row + cw + threadIdx.x];
            for (int cs = cw; cs < cend; cs += 32 * CPL)
            {
                int c[CPL];
                bool cv[CPL];
                double vc[CPL];
                TA a[CPL][8];            // raw loads in flight, widened at use
#pragma unroll
                for (int j = 0; j < CPL; j++)
                {
                    c[j] = cs + lane + 32 * j;
                    cv[j] = c[j] < cend;
                    vc[j] = (do0 && cv[j]) ? XS[T.in0_row + c[j]] : 0.0;
#pragma unroll
                    for (int k = 0; k < 8; k++) a[j][k] = (cv[j] && k < nr) ? A[(long long) k * blk_ld<TA>(T) + c[j]] : TA(0);
                }
                if constexpr (sizeof(TA) == 4)
                {
                    // FP32 blocks: products and the sums over one pass (8 rows, or CPL
                    // columns) in FP32, widened once per sum
#pragma unroll
                    for (int j = 0; j < CPL; j++)
                    {
                        float q = 0.f;
#pragma unroll
                        for (int k = 0; k < 8; k++) q = fmaf(a[j][k], (float) wr[k], q);
                        if (do1) s_q[w][cs - cw + lane + 32 * j] = (double) q;
                    }
#pragma unroll
                    for (int k = 0; k < 8; k++)
                    {
                        float pk = 0.f;
#pragma unroll
                        for (int j = 0; j < CPL; j++) pk = fmaf(a[j][k], (float) vc[j], pk);
                        p[k] += (double) pk;
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < CPL; j++)
                    {
                        double q = 0.0;
#pragma unroll
                        for (int k = 0; k < 8; k++)
                        {
                            const double ad = to_d(a[j][k]);
                            q = fma(ad, wr[k], q);
                            p[k] = fma(ad, vc[j], p[k]);
                        }
                        if (do1) s_q[w][cs - cw + lane + 32 * j] = q;
                    }
                }
            }
            if (do1)
            {
                __syncthreads();
                const int t = threadIdx.x;
                if (t < cend - cw)
                {
                    double sum = 0.0;
#pragma unroll
                    for (int k = 0; k < kWarps; k++) sum += s_q[k][t];
                    PS[T.out1_row + cw + t] = (rc == 0) ? sum : o1 + sum;
                }
                __syncthreads();
            }
        }
        if (do0)
        {
            warp_transpose_reduce<8>(p, lane);
            const int row = nv_of_lane<8>(lane);
            if (lane_writes<8>(lane) && row < nr) PS[T.out0_row + r0 + row] = p[0];
        }
    }
}


// CTAs [0, ceil(n_small / 8)): 8 small tasks each, one per warp; the rest: one larger
// task each (tasks [n_small, n)).
template <typename TA>
__global__ void __launch_bounds__(256, 3) k_blk1(const BlkTask* __restrict__ tasks, int n, int n_small,
                                              const TA* __restrict__ arena, const double* __restrict__ XS,
                                              double* __restrict__ PS)
{
    __shared__ double s_q[kWarps][256];
    __shared__ float s_v[sizeof(TA) == 4 ? kWarps : 1][256];
    const int nw = (n_small + kWarps - 1) / kWarps;
    if ((int) blockIdx.x < nw)
    {
        const int w = threadIdx.x >> 5;
        const int t = blockIdx.x * kWarps + w;
        if (t < n_small)
        {
            const BlkTask T = tasks[t];
            blk1_warp<TA>(T, arena, XS, PS, s_q[w], s_v[sizeof(TA) == 4 ? w : 0], threadIdx.x & 31);
        }
        return;
    }
    const int t = n_small + (int) blockIdx.x - nw;
    if (t < n)
    {
        const BlkTask T = tasks[t];
        blk1_cta<TA>(T, arena, XS, PS, s_q);
    }
}

// Stored block chunk for panels of NV >= 4: the R x 32 tile of A staged in shared
// memory feeds both products, C0 = A V (accumulated over the column tiles in
// registers) and C1 = A^T W (complete per column tile, written at once).
template <typename TA, int NV>
__global__ void __launch_bounds__(256) k_blk_gemm(const BlkTask* __restrict__ tasks, const TA* __restrict__ arena,
                                                  const double* __restrict__ XS, double* __restrict__ PS)
{
    constexpr int RT = 64, CT = 32;
    constexpr int VPT0 = (NV * RT) / 256;        // C0 outputs per thread
    constexpr int NG0 = NV / VPT0;
    constexpr int VPT1 = (NV * CT + 255) / 256;  // C1 outputs per thread
    constexpr int NG1 = NV / VPT1;
    __shared__ double sA[RT][CT + 1];
    __shared__ double sV[CT][NV];
    __shared__ double sW[RT][NV];
    const BlkTask T = tasks[blockIdx.x];
    const int t = threadIdx.x, ncol = T.ncol;
    const bool do0 = T.out0_row >= 0, do1 = T.out1_row >= 0;
    const int m = t / NG0, v0 = (t % NG0) * VPT0;
    const int c1 = t / NG1, w0 = (t % NG1) * VPT1;
    // the task's rows in chunks of RT; the chunks' C1 parts add into one slot
    for (int rc = 0; rc < T.nrow; rc += RT)
    {
    const int lda = blk_ld<TA>(T);
    const TA* A = arena + blk_off<TA>(T) + (long long) rc * lda;
    const int R = min(RT, T.nrow - rc);
    double acc0[VPT0];
#pragma unroll
    for (int j = 0; j < VPT0; j++) acc0[j] = 0.0;
    __syncthreads();
    if (do1)
        for (int i = t; i < RT * NV; i += 256)
        {
            int r = i / NV, v = i % NV;
            sW[r][v] = (r < R) ? XS[(long long) (T.in1_row + rc + r) * NV + v] : 0.0;
        }
    for (int ct = 0; ct < ncol; ct += CT)
    {
        __syncthreads();
        for (int i = t; i < RT * CT; i += 256)
        {
            int r = i / CT, c = i % CT;
            sA[r][c] = (r < R && ct + c < ncol) ? to_d(A[(long long) r * lda + ct + c]) : 0.0;
        }
        if (do0)
            for (int i = t; i < CT * NV; i += 256)
            {
                int c = i / NV, v = i % NV;
                sV[c][v] = (ct + c < ncol) ? XS[(long long) (T.in0_row + ct + c) * NV + v] : 0.0;
            }
        __syncthreads();
        if (do0)
        {
#pragma unroll 8
            for (int c = 0; c < CT; c++)
            {
                const double a = sA[m][c];
#pragma unroll
                for (int j = 0; j < VPT0; j++) acc0[j] = fma(a, sV[c][v0 + j], acc0[j]);
            }
        }
        if (do1 && c1 < CT && ct + c1 < ncol)
        {
            double acc1[VPT1];
#pragma unroll
            for (int j = 0; j < VPT1; j++) acc1[j] = 0.0;
            for (int r = 0; r < R; r++)
            {
                const double a = sA[r][c1];
#pragma unroll
                for (int j = 0; j < VPT1; j++) acc1[j] = fma(a, sW[r][w0 + j], acc1[j]);
            }
#pragma unroll
            for (int j = 0; j < VPT1; j++)
            {
                double* o = PS + (long long) (T.out1_row + ct + c1) * NV + w0 + j;
                *o = (rc == 0) ? acc1[j] : *o + acc1[j];
            }
        }
    }
    if (do0 && m < R)
#pragma unroll
        for (int j = 0; j < VPT0; j++) PS[(long long) (T.out0_row + rc + m) * NV + v0 + j] = acc0[j];
    }
}

template <typename TA, int NV>
__global__ void __launch_bounds__(kThreads) k_blk(const BlkTask* __restrict__ tasks, const TA* __restrict__ arena,
                                                  const double* __restrict__ XS, double* __restrict__ PS)
{
    extern __shared__ double dsm[];
    const BlkTask t = tasks[blockIdx.x];
    VFromXS vin{XS, t.in0_row};
    // the task's rows in chunks of 64; the chunks' A^T w parts add into one slot
    for (int rc = 0; rc < t.nrow; rc += 64)
    {
        chunk_apply<TA, NV>(arena + blk_off<TA>(t) + (long long) rc * blk_ld<TA>(t), min(64, t.nrow - rc), t.ncol,
                            blk_ld<TA>(t), vin, XS,
                            t.in1_row + rc, t.out0_row >= 0 ? PS + (long long) (t.out0_row + rc) * NV : nullptr,
                            t.out1_row >= 0 ? PS + (long long) t.out1_row * NV : nullptr, dsm, rc > 0);
        __syncthreads();
    }
}

// Downward product of one chunk of <= 64 rows of U per CTA (narrow panels):
// dst[r] = U[r] (y1 + push).  Warp w owns rows 8w..8w+7; lanes stride the columns, eight
// loads (one per row) in flight per step; the column inputs y1 + push are staged in
// shared memory per 256 columns; the eight row sums of a warp meet in one transposed
// butterfly per right-hand side.
template <typename TA, int NV>
__global__ void __launch_bounds__(kThreads) k_down(const DownTask* __restrict__ tasks, const TA* __restrict__ Uar,
                                                   const double* __restrict__ Y1, double* __restrict__ PS,
                                                   double* __restrict__ PUSH)
{
    constexpr int CW = 256;
    __shared__ double s_x[CW * NV];
    const DownTask t = tasks[blockIdx.x];
    const VFromY1 vin{Y1, PUSH, t.y1_row, t.push_row};
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, ncol = t.ncol, ld = t.ld;
    const int r0 = 8 * w, nr = max(0, min(8, t.nrow - r0));
    const TA* A = Uar + t.u_off + (long long) r0 * ld;
    double p[NV][8];
#pragma unroll
    for (int v = 0; v < NV; v++)
#pragma unroll
        for (int k = 0; k < 8; k++) p[v][k] = 0.0;
    for (int cw = 0; cw < ncol; cw += CW)
    {
        const int cend = min(ncol, cw + CW);
        __syncthreads();
        for (int i = threadIdx.x; i < (cend - cw) * NV; i += kThreads) s_x[i] = vin(cw + i / NV, i % NV, NV);
        __syncthreads();
        for (int c = cw + lane; c < cend; c += 32)
        {
            TA a[8];
#pragma unroll
            for (int k = 0; k < 8; k++) a[k] = (k < nr) ? A[(long long) k * ld + c] : TA(0);
#pragma unroll
            for (int k = 0; k < 8; k++)
#pragma unroll
                for (int v = 0; v < NV; v++) p[v][k] = fma(to_d(a[k]), s_x[(c - cw) * NV + v], p[v][k]);
        }
    }
    double* dst = (t.dst_ps ? PS : PUSH) + (long long) (t.dst_row + r0) * NV;
    const int row = nv_of_lane<8>(lane);
#pragma unroll
    for (int v = 0; v < NV; v++)
    {
        warp_transpose_reduce<8>(p[v], lane);
        if (lane_writes<8>(lane) && row < nr) dst[(long long) row * NV + v] = p[v][0];
    }
}

// y1 of a node = sum of its PS slots (fixed order); rows indexed like the y0 region.
template <int NV>
__global__ void k_y1sum(const Y1Task* __restrict__ tasks, const int* __restrict__ slots,
                        const double* __restrict__ PS, double* __restrict__ Y1)
{
    const Y1Task t = tasks[blockIdx.x];
    for (int i = threadIdx.x; i < t.nrow * NV; i += blockDim.x)
    {
        double s = 0.0;
        for (int k = t.slot_beg; k < t.slot_end; k++) s += PS[(long long) slots[k] * NV + i];
        Y1[(long long) t.row * NV + i] = s;
    }
}

// --------------------------------------------------------------- assemble

// Y[fwd[row0 + r]][v] = sum over the leaf's slots (fixed order)
template <int NV>
__global__ void k_asm(const AsmTask* __restrict__ tasks, const int* __restrict__ slots,
                      const double* __restrict__ PS, const int* __restrict__ fwd,
                      double* __restrict__ Y, long long y_rs, long long y_cs, int nv)
{
    const AsmTask t = tasks[blockIdx.x];
    for (int i = threadIdx.x; i < t.nrow * NV; i += blockDim.x)
    {
        int r = i / NV, v = i % NV;
        if (v >= nv) continue;
        double s = 0.0;
        for (int k = t.slot_beg; k < t.slot_end; k++) s += PS[(long long) (slots[k] + r) * NV + v];
        Y[(long long) fwd[t.row0 + r] * y_rs + (long long) v * y_cs] = s;
    }
}

// ------------------------------------------------------------------- kernels

// Kernel functions, restated from src/H2Pack_3D_kernels.h (Coulomb :98-161,
// Gaussian :209-268, Matern 3/2 :435-497, RPY :893-959).
template <typename T> struct Math;
template <> struct Math<double> {
    static __device__ __forceinline__ double rsqrt_(double x) { return 1.0 / sqrt(x); }
    static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
    static __device__ __forceinline__ double exp_(double x) { return exp(x); }
    static __device__ __forceinline__ double div_(double a, double b) { return a / b; }
};
// FP32 path: the hardware approximations (MUFU ex2 / rsqrt, flush-to-zero),
// relative error below 2^-22, written as PTX so no library code is involved.
__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rsqrt_approx(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kLog2e = 1.4426950408889634f;

template <> struct Math<float> {
    static __device__ __forceinline__ float rsqrt_(float x) { return rsqrt_approx(x); }
    static __device__ __forceinline__ float sqrt_(float x) { return x * rsqrt_approx(fmaxf(x, 1e-30f)); }
    static __device__ __forceinline__ float exp_(float x) { return ex2_approx(x * kLog2e); }
    static __device__ __forceinline__ float div_(float a, float b) { return __fdividef(a, b); }
};

template <int KID, typename T> struct Scalar;
template <typename T> struct Scalar<KRNL_COULOMB_ID, T> {
    static __device__ __forceinline__ T f(T r2, T p0, T) { return r2 == T(0) ? p0 : Math<T>::rsqrt_(r2); }
};
template <typename T> struct Scalar<KRNL_GAUSSIAN_ID, T> {
    static __device__ __forceinline__ T f(T r2, T p0, T) { return Math<T>::exp_(-p0 * r2); }
};
template <typename T> struct Scalar<KRNL_MATERN32_ID, T> {
    static __device__ __forceinline__ T f(T r2, T, T c0)
    {
        T t = c0 * Math<T>::sqrt_(r2);   // c0 = -sqrt(3) l
        return (T(1) - t) * Math<T>::exp_(t);
    }
};
// (1 - t) e^t = e - t e with e = 2^(t log2 e): 7 instructions, 2 of them MUFU
template <> struct Scalar<KRNL_MATERN32_ID, float> {
    static __device__ __forceinline__ float f(float r2, float, float c0)
    {
        float t = c0 * (r2 * rsqrt_approx(fmaxf(r2, 1e-30f)));
        float e = ex2_approx(t * kLog2e);
        return fmaf(-t, e, e);
    }
};

// The FP32 kernels of two values at once with packed FP32x2 arithmetic, the same
// operations and roundings as Scalar<K, float>::f (coincident points included).
template <int KID> struct ScalarF2;
template <> struct ScalarF2<KRNL_COULOMB_ID> {
    static __device__ __forceinline__ float2 f2(float2 r2, float p0, float)
    {
        return make_float2(r2.x == 0.f ? p0 : rsqrt_approx(r2.x), r2.y == 0.f ? p0 : rsqrt_approx(r2.y));
    }
};
template <> struct ScalarF2<KRNL_GAUSSIAN_ID> {
    static __device__ __forceinline__ float2 f2(float2 r2, float p0, float)
    {
        // exp(-p0 r^2) = 2^((-p0 r^2) log2 e)
        const float2 t = __fmul2_rn(__fmul2_rn(make_float2(-p0, -p0), r2), make_float2(kLog2e, kLog2e));
        return make_float2(ex2_approx(t.x), ex2_approx(t.y));
    }
};
template <> struct ScalarF2<KRNL_MATERN32_ID> {
    static __device__ __forceinline__ float2 f2(float2 r2, float, float c0)
    {
        const float2 rs = make_float2(rsqrt_approx(fmaxf(r2.x, 1e-30f)), rsqrt_approx(fmaxf(r2.y, 1e-30f)));
        const float2 t = __fmul2_rn(make_float2(c0, c0), __fmul2_rn(r2, rs));
        const float2 u = __fmul2_rn(t, make_float2(kLog2e, kLog2e));
        const float2 e = make_float2(ex2_approx(u.x), ex2_approx(u.y));
        return __ffma2_rn(make_float2(-t.x, -t.y), e, e);
    }
};

// Exact-difference form of the near field (Coulomb): a coordinate is carried as
// hi + lo (both FP32, hi = the re-centred coordinate rounded to FP32).  The target's
// coordinate in the source set's frame is a + s with s the frame shift, which the
// host makes exactly representable; two_sum returns the rounded sum and the low part
// a' + (rounding error of a + s) (Knuth's TwoSum).  A difference is then
// (ahi - bhi) + (alo - blo): the first term is exact or rounded relative to itself,
// so r keeps ~FP32 relative accuracy however close two points are (the plain
// difference of rounded coordinates loses eps * box / r).
__device__ __forceinline__ void two_sum(float a, float s, float alo, float& hi, float& lo)
{
    hi = a + s;
    const float bp = hi - a;
    lo = ((a - (hi - bp)) + (s - bp)) + alo;
}

// FP32 kernel values for admissible (well-separated) pairs only: r2 > 0 always, so the
// coincident-point cases drop out.  They take r^2 scaled by KParam::sigma (the callers
// scale |a|^2, -2a and the panels' |b|^2), which folds a constant multiply into the
// r^2 form: Gaussian exp(-l r^2) = 2^-(sigma r^2) with sigma = l log2 e; Matern
// (1 + s ln 2) 2^-s with s = sqrt(sigma r^2) = sqrt(3) log2 e r / l.  prep folds the
// remaining constants once per launch.  f2: two values at once (packed FP32x2).
template <int KID> struct ScalarFar;
template <> struct ScalarFar<KRNL_COULOMB_ID> {    // sigma = 1
    static __device__ __forceinline__ void prep(float, float, float& q0, float& q1) { q0 = 0.f; q1 = 0.f; }
    static __device__ __forceinline__ float2 f2(float2 r2, float, float)
    {
        return make_float2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
    }
};
template <> struct ScalarFar<KRNL_GAUSSIAN_ID> {
    static __device__ __forceinline__ void prep(float, float, float& q0, float& q1) { q0 = 0.f; q1 = 0.f; }
    static __device__ __forceinline__ float2 f2(float2 r2s, float, float)
    {
        return make_float2(ex2_approx(-r2s.x), ex2_approx(-r2s.y));
    }
};
template <> struct ScalarFar<KRNL_MATERN32_ID> {
    static __device__ __forceinline__ void prep(float, float, float& q0, float& q1) { q0 = 0.6931471805599453f; q1 = 0.f; }
    static __device__ __forceinline__ float2 f2(float2 r2s, float ln2, float)
    {
        const float2 s = __fmul2_rn(r2s, make_float2(rsqrt_approx(r2s.x), rsqrt_approx(r2s.y)));
        const float2 e = make_float2(ex2_approx(-s.x), ex2_approx(-s.y));
        return __fmul2_rn(__ffma2_rn(s, make_float2(ln2, ln2), make_float2(1.f, 1.f)), e);
    }
};

// RPY 3x3 block: K_ab = t2 u_a u_b + t1 delta_ab, u = (dx,dy,dz)/r (0 at r = 0)
template <typename T>
__device__ __forceinline__ void rpy_coef(T dx, T dy, T dz, T ta, T sa, T C, T& t1, T& t2, T& ux, T& uy, T& uz)
{
    T r2 = dx * dx + dy * dy + dz * dz;
    T r = Math<T>::sqrt_(r2);
    T inv_r = (r == T(0)) ? T(0) : Math<T>::div_(T(1), r);
    T inv_r2 = inv_r * inv_r;
    ux = dx * inv_r; uy = dy * inv_r; uz = dz * inv_r;
    T ta_p_sa = ta + sa, ta_m_sa = ta - sa;
    if (r > ta_p_sa)
    {
        T tmp0 = C * T(0.75) * inv_r;
        T tmp1 = (ta * ta + sa * sa) * inv_r2;
        t1 = tmp0 * (T(1) + tmp1 / T(3));
        t2 = tmp0 * (T(1) - tmp1);
    } else if (r > fabs(ta_m_sa)) {
        T tmp0 = ta_m_sa * ta_m_sa;
        T tmp1 = Math<T>::div_(inv_r2 * inv_r * C, ta * sa * T(32));
        T a = tmp0 + T(3) * r2;
        t1 = tmp1 * (T(16) * r2 * r * ta_p_sa - a * a);
        T b = tmp0 - r2;
        t2 = tmp1 * T(3) * b * b;
    } else {
        t1 = Math<T>::div_(C, (ta > sa ? ta : sa));
        t2 = T(0);
    }
}

template <typename T> struct Vec4;
template <> struct Vec4<double> { using t = double4; };
template <> struct Vec4<float> { using t = float4; };

// ------------------------------------------------------------ JIT owner kernel

// One CTA per chunk of <= 128 target points, 128/TPT threads, TPT targets per thread.
// For every source set of the target, source points and their inputs are staged in
// shared memory in tiles; each thread evaluates its targets against every staged
// source point and accumulates K * in (the one-sided form of H2P_ext_krnl_bimv,
// src/H2Pack_matvec.c:463-539).  With T = float the products of one tile are summed
// in FP32 and every tile sum is added to FP64 accumulators, so an FP32 sum never
// spans more than one tile of sources.  Outputs are written once, no atomics.
template <int KID, typename T, int NV, int KD, int TPT>
__global__ void __launch_bounds__(128 / TPT, sizeof(T) == 4 ? 5 * TPT : 4 * TPT) k_jit(const JitTarget* __restrict__ tgts, const JitSource* __restrict__ srcs,
                                                   const typename Vec4<T>::t* __restrict__ pts, KParam kp, int use_shift,
                                                   const double* __restrict__ XS, double* __restrict__ PS,
                                                   double* __restrict__ Y1)
{
    using T4 = typename Vec4<T>::t;
    constexpr int NT = 128 / TPT;
    constexpr int W = KD * NV;
    constexpr bool SPLIT = sizeof(T) < sizeof(double);
    // FP32: 64-point tiles keep shared memory at ~21 KB so 10 CTAs fit an SM
    constexpr int TILE = (SPLIT || 128 * W * (int) sizeof(T) > 32768) ? 64 : 128;
    __shared__ T4 s_pt[TILE];
    __shared__ T s_in[TILE * W];
    // FP64 sums of the FP32 tile sums, one column per thread (conflict-free)
    __shared__ double s_acc[SPLIT ? TPT * W * NT : 1];
    const JitTarget tg = tgts[blockIdx.x];
    const T p0 = (T) kp.p0, c0 = (T) kp.c0;

    T4 xi[TPT];
    bool valid[TPT];
    T acc[TPT][W];
#pragma unroll
    for (int q = 0; q < TPT; q++)
    {
        int i = threadIdx.x + q * NT;
        valid[q] = i < tg.npt;
        xi[q] = pts[tg.pt0 + (valid[q] ? i : 0)];
#pragma unroll
        for (int k = 0; k < W; k++) acc[q][k] = T(0);
        if constexpr (SPLIT)
        {
#pragma unroll
            for (int k = 0; k < W; k++) s_acc[(q * W + k) * NT + threadIdx.x] = 0.0;
        }
    }

    for (int s = tg.src_beg; s < tg.src_end; s++)
    {
        const JitSource sc = srcs[s];
        T4 xs[TPT];
#pragma unroll
        for (int q = 0; q < TPT; q++)
        {
            xs[q] = xi[q];
            if (use_shift) { xs[q].x += (T) sc.sx; xs[q].y += (T) sc.sy; xs[q].z += (T) sc.sz; }
        }
        for (int j0 = 0; j0 < sc.npt; j0 += TILE)
        {
            const int nj = min(TILE, sc.npt - j0);
            __syncthreads();
            for (int j = threadIdx.x; j < nj; j += NT) s_pt[j] = pts[sc.pt0 + j0 + j];
            for (int i = threadIdx.x; i < nj * W; i += NT)
                s_in[i] = (T) XS[(long long) (sc.in_row + KD * j0) * NV + i];
            __syncthreads();
#pragma unroll 2
            for (int j = 0; j < nj; j++)
            {
                const T4 pj = s_pt[j];
                const T* inj = s_in + j * W;
                T in[W];
#pragma unroll
                for (int k = 0; k < W; k++) in[k] = inj[k];
#pragma unroll
                for (int q = 0; q < TPT; q++)
                {
                    T dx = xs[q].x - pj.x, dy = xs[q].y - pj.y, dz = xs[q].z - pj.z;
                    if constexpr (KD == 1)
                    {
                        T r2 = dx * dx + dy * dy + dz * dz;
                        T k = Scalar<KID, T>::f(r2, p0, c0);
#pragma unroll
                        for (int v = 0; v < NV; v++) acc[q][v] = fma(k, in[v], acc[q][v]);
                    } else {
                        T t1, t2, ux, uy, uz;
                        rpy_coef<T>(dx, dy, dz, xi[q].w, pj.w, c0, t1, t2, ux, uy, uz);
#pragma unroll
                        for (int v = 0; v < NV; v++)
                        {
                            T bx = in[0 * NV + v], by = in[1 * NV + v], bz = in[2 * NV + v];
                            T dot = t2 * (ux * bx + uy * by + uz * bz);
                            acc[q][0 * NV + v] = fma(dot, ux, fma(t1, bx, acc[q][0 * NV + v]));
                            acc[q][1 * NV + v] = fma(dot, uy, fma(t1, by, acc[q][1 * NV + v]));
                            acc[q][2 * NV + v] = fma(dot, uz, fma(t1, bz, acc[q][2 * NV + v]));
                        }
                    }
                }
            }
            if constexpr (SPLIT)
            {
#pragma unroll
                for (int q = 0; q < TPT; q++)
#pragma unroll
                    for (int k = 0; k < W; k++)
                    {
                        s_acc[(q * W + k) * NT + threadIdx.x] += (double) acc[q][k];
                        acc[q][k] = T(0);
                    }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < TPT; q++)
    {
        if (!valid[q]) continue;
        int i = threadIdx.x + q * NT;
        double* o = (tg.out_y1 ? Y1 : PS) + (long long) (tg.out_row + KD * i) * NV;
#pragma unroll
        for (int k = 0; k < W; k++)
        {
            if constexpr (SPLIT) o[k] = s_acc[(q * W + k) * NT + threadIdx.x];
            else o[k] = (double) acc[q][k];
        }
    }
}

// FP32 scalar kernels on the CUDA cores (the panels the tensor-core kernel does not
// take, e.g. the narrow panels of the served form): k_jit's work split (one CTA of 64
// threads per 128-target chunk, two targets per thread) with the thread's two targets
// as one FP32x2 pair.  Sources are staged in shared memory with every coordinate and
// input stored twice (the FP32x2 operand that meets both targets), so a source costs
// packed instructions only.  FAR (admissible pairs): r^2 = |a|^2 + |b|^2 - 2 a.b as in
// k_jit_tc; otherwise differences (exact-difference form for Coulomb, see two_sum).
// FP32 sums per 64-source tile, FP64 across tiles.
template <int KID, int NV, bool FAR>
__global__ void __launch_bounds__(64, NV >= 16 ? 8 : 10) k_jit2(const JitTarget* __restrict__ tgts, const JitSource* __restrict__ srcs,
                                                 const float4* __restrict__ pts, KParam kp,
                                                 const double* __restrict__ XS, double* __restrict__ PS,
                                                 double* __restrict__ Y1, const float4* __restrict__ plo)
{
    constexpr bool EX = KID == KRNL_COULOMB_ID && !FAR;
    constexpr int TILE = 64, NT = 64;
    __shared__ float4 s_p[TILE][2];          // {x, x, y, y}, {z, z, w, w}; w = |p|^2 (FAR), z' (EX)
    __shared__ float4 s_l[EX ? TILE : 1];    // {x', x', y', y'} (EX)
    __shared__ float2 s_in[TILE * NV];       // (in, in)
    __shared__ double s_acc[2 * NV][NT];     // FP64 sums of the tile sums, [target q x NV + v][thread]
    const JitTarget tg = tgts[blockIdx.x];
    const float p0 = (float) kp.p0, c0 = (float) kp.c0;
    float q0 = 0.f, q1 = 0.f;
    if constexpr (FAR) ScalarFar<KID>::prep(p0, c0, q0, q1);
    const int i0 = threadIdx.x, i1 = threadIdx.x + NT;
    const bool v0 = i0 < tg.npt, v1 = i1 < tg.npt;
    const float4 x0 = pts[tg.pt0 + (v0 ? i0 : 0)], x1 = pts[tg.pt0 + (v1 ? i1 : 0)];
    float4 l0 = make_float4(0.f, 0.f, 0.f, 0.f), l1 = l0;
    if constexpr (EX) { l0 = plo[tg.pt0 + (v0 ? i0 : 0)]; l1 = plo[tg.pt0 + (v1 ? i1 : 0)]; }
    float2 acc[NV];
#pragma unroll
    for (int v = 0; v < NV; v++)
    {
        acc[v] = make_float2(0.f, 0.f);
        s_acc[v][threadIdx.x] = 0.0;
        s_acc[NV + v][threadIdx.x] = 0.0;
    }
    const float2 m1 = make_float2(-1.f, -1.f);
    for (int s = tg.src_beg; s < tg.src_end; s++)
    {
        const JitSource sc = srcs[s];
        const float ax = x0.x + sc.sx, ay = x0.y + sc.sy, az = x0.z + sc.sz;
        const float bx = x1.x + sc.sx, by = x1.y + sc.sy, bz = x1.z + sc.sz;
        const float2 X = make_float2(ax, bx), Y = make_float2(ay, by), Z = make_float2(az, bz);
        // far form, scaled by sigma (ScalarFar)
        const float m2s = -2.f * kp.sigma;
        const float2 MX = make_float2(m2s * ax, m2s * bx), MY = make_float2(m2s * ay, m2s * by),
                     MZ = make_float2(m2s * az, m2s * bz);
        const float2 S2 = make_float2(kp.sigma * (ax * ax + ay * ay + az * az), kp.sigma * (bx * bx + by * by + bz * bz));
        float2 XH = X, YH = Y, ZH = Z, XL = make_float2(0.f, 0.f), YL = XL, ZL = XL;
        if constexpr (EX)
        {
            two_sum(x0.x, sc.sx, l0.x, XH.x, XL.x); two_sum(x1.x, sc.sx, l1.x, XH.y, XL.y);
            two_sum(x0.y, sc.sy, l0.y, YH.x, YL.x); two_sum(x1.y, sc.sy, l1.y, YH.y, YL.y);
            two_sum(x0.z, sc.sz, l0.z, ZH.x, ZL.x); two_sum(x1.z, sc.sz, l1.z, ZH.y, ZL.y);
        }
        for (int j0 = 0; j0 < sc.npt; j0 += TILE)
        {
            const int nj = min(TILE, sc.npt - j0);
            __syncthreads();
            if (threadIdx.x < nj)
            {
                float4 q = pts[sc.pt0 + j0 + threadIdx.x];
                if (FAR) q.w = kp.sigma * (q.x * q.x + q.y * q.y + q.z * q.z);
                if constexpr (EX)
                {
                    const float4 ql = plo[sc.pt0 + j0 + threadIdx.x];
                    q.w = ql.z;
                    s_l[threadIdx.x] = make_float4(ql.x, ql.x, ql.y, ql.y);
                }
                s_p[threadIdx.x][0] = make_float4(q.x, q.x, q.y, q.y);
                s_p[threadIdx.x][1] = make_float4(q.z, q.z, q.w, q.w);
            }
            for (int i = threadIdx.x; i < nj * NV; i += NT)
            {
                const float x = (float) XS[(long long) (sc.in_row + j0) * NV + i];
                s_in[i] = make_float2(x, x);
            }
            __syncthreads();
#pragma unroll 2
            for (int j = 0; j < nj; j++)
            {
                const float4 P0 = s_p[j][0], P1 = s_p[j][1];
                float2 k;
                if constexpr (FAR)
                {
                    float2 r2 = __fadd2_rn(S2, make_float2(P1.z, P1.w));
                    r2 = __ffma2_rn(MZ, make_float2(P1.x, P1.y), r2);
                    r2 = __ffma2_rn(MY, make_float2(P0.z, P0.w), r2);
                    r2 = __ffma2_rn(MX, make_float2(P0.x, P0.y), r2);
                    k = ScalarFar<KID>::f2(r2, q0, q1);
                } else if constexpr (EX) {
                    const float4 L = s_l[j];
                    const float2 dx = __fadd2_rn(__ffma2_rn(make_float2(P0.x, P0.y), m1, XH),
                                                 __ffma2_rn(make_float2(L.x, L.y), m1, XL));
                    const float2 dy = __fadd2_rn(__ffma2_rn(make_float2(P0.z, P0.w), m1, YH),
                                                 __ffma2_rn(make_float2(L.z, L.w), m1, YL));
                    const float2 dz = __fadd2_rn(__ffma2_rn(make_float2(P1.x, P1.y), m1, ZH),
                                                 __ffma2_rn(make_float2(P1.z, P1.w), m1, ZL));
                    k = ScalarF2<KID>::f2(__ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz))), p0, c0);
                } else {
                    const float2 dx = __ffma2_rn(make_float2(P0.x, P0.y), m1, X);
                    const float2 dy = __ffma2_rn(make_float2(P0.z, P0.w), m1, Y);
                    const float2 dz = __ffma2_rn(make_float2(P1.x, P1.y), m1, Z);
                    k = ScalarF2<KID>::f2(__ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz))), p0, c0);
                }
#pragma unroll
                for (int v = 0; v < NV; v++) acc[v] = __ffma2_rn(k, s_in[j * NV + v], acc[v]);
            }
#pragma unroll
            for (int v = 0; v < NV; v++)
            {
                s_acc[v][threadIdx.x] += (double) acc[v].x;
                s_acc[NV + v][threadIdx.x] += (double) acc[v].y;
                acc[v] = make_float2(0.f, 0.f);
            }
        }
    }
    double* o = tg.out_y1 ? Y1 : PS;
#pragma unroll
    for (int v = 0; v < NV; v++)
    {
        if (v0) o[(long long) (tg.out_row + i0) * NV + v] = s_acc[v][threadIdx.x];
        if (v1) o[(long long) (tg.out_row + i1) * NV + v] = s_acc[NV + v][threadIdx.x];
    }
}

// ------------------------------------------------ JIT owner kernel, tensor cores

// TF32 pieces of an FP32 value: hi = rna(x), lo = rna(x - hi); hi*b + lo*b recovers
// ~22 bits, the 3xTF32 split (hi*hi + hi*lo + lo*hi) keeps products at ~2^-21.
__device__ __forceinline__ uint32_t tf32_rna(float x)
{
    // round to nearest (ties away from zero) at 10 mantissa bits with two integer ops;
    // finite inputs far below FLT_MAX only, which holds for kernel values and inputs here
    return (__float_as_uint(x) + 0x1000u) & 0xffffe000u;
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1)
{
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Shared-window address of a shared-memory pointer (32-bit, for PTX operands)
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t) __cvta_generic_to_shared(p); }

// cp.async: 16 bytes global -> shared without registers (L2 only), in commit groups
__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Source panels of k_jit_tc (one PanelGroup per 8 points of a source set).
// Points: per group 8 float4, entry [t][0] = {x, x', y, y'}, [t][1] = {z, z', s|p|^2, s|p'|^2}
// (s = KParam::sigma, the far field's scale of r^2)
// of the set's points 8g + t and 8g + t + 4 (t < 4): the two sources of one B-fragment
// register pair, as FP32x2 operands.  Points past the set's end are far away (their
// inputs are zero).
__global__ void k_panel_pts(const PanelGroup* __restrict__ pg, int n, const float4* __restrict__ pts, float sigma,
                            float4* __restrict__ out)
{
    const long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if (e >= 8LL * n) return;
    const int g = (int) (e >> 3), j = (int) (e & 7), t = j & 3, h = j >> 2;
    const PanelGroup G = pg[g];
    float4 q = (j < G.nvalid) ? pts[G.pt0 + j] : make_float4(1e6f, 1e6f, 1e6f, 0.f);
    q.w = sigma * (q.x * q.x + q.y * q.y + q.z * q.z);
    float* d = reinterpret_cast<float*>(out + 8LL * g + 2 * t);
    d[h] = q.x; d[2 + h] = q.y; d[4 + h] = q.z; d[6 + h] = q.w;
}

// Low parts of the panel points (Coulomb near field): per group 6 float4 = 24 floats,
// [4t + h] = x', [4t + 2 + h] = y', [16 + 2t + h] = z' of point 8g + t + 4h (t < 4), the
// same pairing as k_panel_pts; points past the set's end have zero low parts.
__global__ void k_panel_lo(const PanelGroup* __restrict__ pg, int n, const float4* __restrict__ lo,
                           float4* __restrict__ out)
{
    const long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if (e >= 8LL * n) return;
    const int g = (int) (e >> 3), j = (int) (e & 7), t = j & 3, h = j >> 2;
    const PanelGroup G = pg[g];
    const float4 q = (j < G.nvalid) ? lo[G.pt0 + j] : make_float4(0.f, 0.f, 0.f, 0.f);
    float* d = reinterpret_cast<float*>(out + 6LL * g);
    d[4 * t + h] = q.x; d[4 * t + 2 + h] = q.y; d[16 + 2 * t + h] = q.z;
}


// Inputs: per group 2 x 32 uint4, the m16n8k8 A fragment of in^T (16 right-hand sides
// x the group's 8 points; right-hand sides >= NV are zero) split into TF32 hi (first 32)
// and lo (last 32): lane l (r = l/4, t = l%4) holds in[t][r], in[t][r+8], in[t+4][r],
// in[t+4][r+8], each rounded to FP32, hi = rna(x), lo = rna(x - hi).
template <int NV>
__global__ void k_panel_in(const PanelGroup* __restrict__ pg, int g0, int n, const double* __restrict__ XS,
                           uint4* __restrict__ out)
{
    const long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if (e >= 32LL * n) return;
    const int g = g0 + (int) (e >> 5), ln = (int) (e & 31), r = ln >> 2, t = ln & 3;
    const PanelGroup G = pg[g];
    auto in = [&](int s, int c) -> float {
        return (s < G.nvalid && c < NV) ? (float) XS[(long long) (G.row0 + s) * NV + c] : 0.f;
    };
    const float x[4] = {in(t, r), in(t, r + 8), in(t + 4, r), in(t + 4, r + 8)};
    uint32_t h[4], l[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
    {
        h[q] = tf32_rna(x[q]);
        l[q] = tf32_rna(x[q] - __uint_as_float(h[q]));
    }
    out[64LL * g + ln] = make_uint4(h[0], h[1], h[2], h[3]);
    out[64LL * g + 32 + ln] = make_uint4(l[0], l[1], l[2], l[3]);
}

// Shared memory of k_jit_tc (dynamic, 52 KB)
struct JitTcSmem {
    float4 pt[2][16][4][2];     // points of the tile being computed and of the next one
    uint4 in[2][16][2][32];     // their inputs (A fragments, hi / lo)
    double acc[8][8][32];       // FP64 sums of the FP32 segment sums, [warp][n-tile x 4 + q][lane]
    TileRec rec[4];             // records of the next tiles
};
// ... with the low parts of the points (Coulomb near field, 55 KB: still 4 CTAs per SM)
struct JitTcSmemEx : JitTcSmem {
    float4 lo[2][16][6];
};

// Same work split as k_jit (one CTA per 128-target chunk, owner computes), with the
// right-hand-side products on the tensor cores.  Warp w owns targets 16w..16w+15.
// The kernel block is the B operand of m16n8k8 (k = 8 sources x n = 8 targets) and the
// inputs the A operand (16 right-hand sides x 8 sources), so a lane (g = lane/4,
// t = lane%4) evaluates, per group of 8 sources and for each of its targets 16w + g and
// 16w + 8 + g, the values against sources t and t + 4: one FP32x2 pair that is also
// its B-fragment register pair.  Values are split into TF32 hi / lo and multiplied
// with the inputs' hi / lo (3xTF32: lo.hi + hi.lo + hi.hi, 3 MMAs per 8 targets).
// FP32 accumulation over 64 sources (a segment), FP64 sums across segments.
// Sources come from the panels, already paired and split; a tile of up to 128 sources
// (16 groups) is two contiguous copies, moved by cp.async into a shared-memory double
// buffer while the previous tile is computed, so the CTA meets one barrier per 128
// sources and no registers carry the next tile.
// FAR (admissible pairs only): r^2 = |a|^2 + |b|^2 - 2 a.b with a the target in the
// source set's frame (|a|^2 and -2a once per tile, |b|^2 from the panel): 4
// instructions per 2 values.  Admissible boxes keep r above the box size, so the
// cancellation stays at a few FP32 ulps of r^2 (the near field keeps differences).
// Warps whose 16 target rows are all past the end of the chunk only take part in the
// barriers.
template <int KID, int NV, bool FAR>
__global__ void __launch_bounds__(256, 4) k_jit_tc(const JitTarget* __restrict__ tgts, const TileRec* __restrict__ tiles,
                                                   const float4* __restrict__ pts, const float4* __restrict__ ppts,
                                                   const uint4* __restrict__ pin, KParam kp, double* __restrict__ PS,
                                                   double* __restrict__ Y1, const float4* __restrict__ plo,
                                                   const float4* __restrict__ pplo)
{
    // EX: exact differences (Coulomb near field; plo / pplo = low parts of the points / panels)
    constexpr bool EX = KID == KRNL_COULOMB_ID && !FAR;
    using SM = typename std::conditional<EX, JitTcSmemEx, JitTcSmem>::type;
    extern __shared__ __align__(16) unsigned char jtc_raw[];
    SM& sm = *reinterpret_cast<SM*>(jtc_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
    const JitTarget tg = tgts[blockIdx.x];
    const bool busy = warp * 16 < tg.npt;
    const float p0 = (float) kp.p0, c0 = (float) kp.c0;
    float q0 = 0.f, q1 = 0.f;
    if constexpr (FAR) ScalarFar<KID>::prep(p0, c0, q0, q1);
    // the lane's two targets (as B-fragment columns of n-tiles 0 and 1)
    const int i0 = warp * 16 + g, i1 = i0 + 8;
    const float4 x0 = pts[tg.pt0 + (i0 < tg.npt ? i0 : 0)], x1 = pts[tg.pt0 + (i1 < tg.npt ? i1 : 0)];
    float acc[2][4];
#pragma unroll
    for (int n = 0; n < 2; n++)
#pragma unroll
        for (int q = 0; q < 4; q++) { acc[n][q] = 0.f; sm.acc[warp][n * 4 + q][lane] = 0.0; }
    auto flush = [&]() {
#pragma unroll
        for (int n = 0; n < 2; n++)
#pragma unroll
            for (int q = 0; q < 4; q++) { sm.acc[warp][n * 4 + q][lane] += (double) acc[n][q]; acc[n][q] = 0.f; }
    };
    // one group: the lane's 2 x 2 values (targets i0, i1 x sources t, t+4) as B-fragment
    // pairs k0, k1, against the group's inputs
    auto mma_group = [&](float2 k0, float2 k1, int buf, int grp) {
        const uint4 ah = sm.in[buf][grp][0][lane], al = sm.in[buf][grp][1][lane];
        const float2 m1 = make_float2(-1.f, -1.f);
        const uint32_t h00 = tf32_rna(k0.x), h01 = tf32_rna(k0.y), h10 = tf32_rna(k1.x), h11 = tf32_rna(k1.y);
        const float2 l0 = __ffma2_rn(make_float2(__uint_as_float(h00), __uint_as_float(h01)), m1, k0);
        const float2 l1 = __ffma2_rn(make_float2(__uint_as_float(h10), __uint_as_float(h11)), m1, k1);
        mma_tf32(acc[0], ah.x, ah.y, ah.z, ah.w, __float_as_uint(l0.x), __float_as_uint(l0.y));
        mma_tf32(acc[1], ah.x, ah.y, ah.z, ah.w, __float_as_uint(l1.x), __float_as_uint(l1.y));
        mma_tf32(acc[0], al.x, al.y, al.z, al.w, h00, h01);
        mma_tf32(acc[1], al.x, al.y, al.z, al.w, h10, h11);
        mma_tf32(acc[0], ah.x, ah.y, ah.z, ah.w, h00, h01);
        mma_tf32(acc[1], ah.x, ah.y, ah.z, ah.w, h10, h11);
    };

    // Pipeline over the chunk's tiles k = 0 .. nt-1: tile k is computed from buffer
    // k & 1 while tile k+1 sits in the other buffer; after the tile's barrier tile k+2
    // is copied into buffer k & 1, and the record of tile k+4 into ring slot k & 3.
    const TileRec* rec = tiles + tg.tile_beg;
    const int nt = tg.tile_end - tg.tile_beg;
    auto issue_rec = [&](int k) {   // threads 0, 1: the two 16-byte halves
        if (threadIdx.x < 2 && k < nt)
            cp_async16(reinterpret_cast<uint4*>(&sm.rec[k & 3]) + threadIdx.x, reinterpret_cast<const uint4*>(rec + k) + threadIdx.x);
    };
    auto issue = [&](int k, int buf) {
        if (k >= nt) return;
        const int gb = sm.rec[k & 3].gb, ng = sm.rec[k & 3].ng;
        const float4* gp = ppts + 8LL * gb;
        const uint4* gi = pin + 64LL * gb;
        const int np = ng * 8, nin = np + ng * 64, nall = nin + (EX ? ng * 6 : 0);
        for (int c = threadIdx.x; c < nall; c += 256)
        {
            if (c < np) cp_async16(&sm.pt[buf][0][0][0] + c, gp + c);
            else if (c < nin) cp_async16(&sm.in[buf][0][0][0] + (c - np), gi + (c - np));
            else if constexpr (EX) cp_async16(&sm.lo[buf][0][0] + (c - nin), pplo + 6LL * gb + (c - nin));
        }
    };
    issue_rec(0); issue_rec(1); issue_rec(2); issue_rec(3);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    issue(0, 0); issue(1, 1);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    for (int k = 0; k < nt; k++)
    {
        const int buf = k & 1;
        if (busy)
        {
            const TileRec r = sm.rec[k & 3];
            const float ax = x0.x + r.sx, ay = x0.y + r.sy, az = x0.z + r.sz;
            const float bx = x1.x + r.sx, by = x1.y + r.sy, bz = x1.z + r.sz;
            // segments of 8 groups (64 sources) summed in FP32
            for (int h = 0; h < r.ng; h += 8)
            {
                const int ge = min(r.ng, h + 8);
                if constexpr (FAR)
                {
                    // -2a and |a|^2 of each target in the source set's frame, scaled by
                    // sigma as the panels' |b|^2 (ScalarFar), broadcast
                    const float m2s = -2.f * kp.sigma;
                    const float2 max2 = make_float2(m2s * ax, m2s * ax), may2 = make_float2(m2s * ay, m2s * ay),
                                 maz2 = make_float2(m2s * az, m2s * az);
                    const float2 mbx2 = make_float2(m2s * bx, m2s * bx), mby2 = make_float2(m2s * by, m2s * by),
                                 mbz2 = make_float2(m2s * bz, m2s * bz);
                    const float sa2 = kp.sigma * (ax * ax + ay * ay + az * az), sb2 = kp.sigma * (bx * bx + by * by + bz * bz);
                    const float2 sa22 = make_float2(sa2, sa2), sb22 = make_float2(sb2, sb2);
#pragma unroll 2
                    for (int grp = h; grp < ge; grp++)
                    {
                        const float4 P0 = sm.pt[buf][grp][tq][0], P1 = sm.pt[buf][grp][tq][1];
                        const float2 px = make_float2(P0.x, P0.y), py = make_float2(P0.z, P0.w);
                        const float2 pz = make_float2(P1.x, P1.y), pw = make_float2(P1.z, P1.w);
                        // r^2 of one target against the source pair: 4 packed instructions
                        // for two values.  No clamp: admissible pairs keep r^2 far from 0.
                        auto r2p = [&](float2 s, float2 mx, float2 my, float2 mz) {
                            float2 t = __fadd2_rn(s, pw);
                            t = __ffma2_rn(mz, pz, t);
                            t = __ffma2_rn(my, py, t);
                            return __ffma2_rn(mx, px, t);
                        };
                        const float2 k0 = ScalarFar<KID>::f2(r2p(sa22, max2, may2, maz2), q0, q1);
                        const float2 k1 = ScalarFar<KID>::f2(r2p(sb22, mbx2, mby2, mbz2), q0, q1);
                        mma_group(k0, k1, buf, grp);
                    }
                } else if constexpr (EX) {
                    // targets as hi + lo in the source set's frame (the shift is exact); the
                    // low parts are read per tile (few registers stay live across tiles)
                    const float4 l0 = plo[tg.pt0 + (i0 < tg.npt ? i0 : 0)], l1 = plo[tg.pt0 + (i1 < tg.npt ? i1 : 0)];
                    float ahx, ahy, ahz, alx, aly, alz, bhx, bhy, bhz, blx, bly, blz;
                    two_sum(x0.x, r.sx, l0.x, ahx, alx); two_sum(x0.y, r.sy, l0.y, ahy, aly);
                    two_sum(x0.z, r.sz, l0.z, ahz, alz);
                    two_sum(x1.x, r.sx, l1.x, bhx, blx); two_sum(x1.y, r.sy, l1.y, bhy, bly);
                    two_sum(x1.z, r.sz, l1.z, bhz, blz);
#pragma unroll 1
                    for (int grp = h; grp < ge; grp++)
                    {
                        const float4 P0 = sm.pt[buf][grp][tq][0], P1 = sm.pt[buf][grp][tq][1];
                        const float4 L0 = sm.lo[buf][grp][tq], LZ = sm.lo[buf][grp][4 + (tq >> 1)];
                        const float2 lz = (tq & 1) ? make_float2(LZ.z, LZ.w) : make_float2(LZ.x, LZ.y);
                        const float2 m1 = make_float2(-1.f, -1.f);
                        // (th - p) + (tl - p') per coordinate, both sources of the pair at once
                        auto d2 = [&](float th, float tl, float2 p, float2 q) {
                            return __fadd2_rn(__ffma2_rn(p, m1, make_float2(th, th)), __ffma2_rn(q, m1, make_float2(tl, tl)));
                        };
                        const float2 PX = make_float2(P0.x, P0.y), PY = make_float2(P0.z, P0.w), PZ = make_float2(P1.x, P1.y);
                        const float2 QX = make_float2(L0.x, L0.y), QY = make_float2(L0.z, L0.w);
                        float2 dx = d2(ahx, alx, PX, QX), dy = d2(ahy, aly, PY, QY), dz = d2(ahz, alz, PZ, lz);
                        const float2 k0 = ScalarF2<KID>::f2(__ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz))), p0, c0);
                        dx = d2(bhx, blx, PX, QX); dy = d2(bhy, bly, PY, QY); dz = d2(bhz, blz, PZ, lz);
                        const float2 k1 = ScalarF2<KID>::f2(__ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz))), p0, c0);
                        mma_group(k0, k1, buf, grp);
                    }
                } else {
                    const float2 ax2 = make_float2(ax, ax), ay2 = make_float2(ay, ay), az2 = make_float2(az, az);
                    const float2 bx2 = make_float2(bx, bx), by2 = make_float2(by, by), bz2 = make_float2(bz, bz);
#pragma unroll 1
                    for (int grp = h; grp < ge; grp++)
                    {
                        const float4 P0 = sm.pt[buf][grp][tq][0], P1 = sm.pt[buf][grp][tq][1];
                        const float2 px = make_float2(-P0.x, -P0.y), py = make_float2(-P0.z, -P0.w);
                        const float2 pz = make_float2(-P1.x, -P1.y);
                        // differences of one target to the source pair, packed
                        auto r2d = [&](float2 x, float2 y, float2 z) {
                            const float2 dx = __fadd2_rn(x, px), dy = __fadd2_rn(y, py), dz = __fadd2_rn(z, pz);
                            return __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
                        };
                        const float2 k0 = ScalarF2<KID>::f2(r2d(ax2, ay2, az2), p0, c0);
                        const float2 k1 = ScalarF2<KID>::f2(r2d(bx2, by2, bz2), p0, c0);
                        mma_group(k0, k1, buf, grp);
                    }
                }
                flush();
            }
        }
        cp_async_wait_all();                     // tile k+1 and record k+3 have landed (this thread's copies)
        __syncthreads();                         // ... everyone's, and tile k / record k are no longer read
        issue(k + 2, buf);
        issue_rec(k + 4);
        cp_async_commit();
    }
    // accumulator (n, q) of lane (g, t): right-hand side g + 8 (q >> 1), target
    // 16w + 8n + 2t + (q & 1)
    double* base = (tg.out_y1 ? Y1 : PS) + (long long) tg.out_row * NV;
#pragma unroll
    for (int n = 0; n < 2; n++)
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            const int row = warp * 16 + 8 * n + 2 * tq + (q & 1), rhs = g + 8 * (q >> 1);
            if (row < tg.npt && rhs < NV) base[(long long) row * NV + rhs] = sm.acc[warp][n * 4 + q][lane];
        }
}

constexpr int jit_tc_smem_bytes(bool ex) { return (int) (ex ? sizeof(JitTcSmemEx) : sizeof(JitTcSmem)); }

// ---------------------------------------- JIT pair kernel (both directions at once)

// One CTA (8 warps) per work unit: up to 128 points of an owner a (longer owners are
// walked in chunks of 128; warp w owns rows 16w..16w+15 of a chunk) and a run of a's
// partners.  For every partner b, source tiles of 64 points are
// staged as in k_jit_tc (double-buffered: the next tile is read from global memory
// while the current one is computed).  Per group of 8 points of b each lane evaluates
// the 4 kernel values of its m16n8k8 A fragment once and uses them twice:
//   direction a <- b:  out_a (16 rows x NV) += K (16 x 8) * in_b (8 x NV)   [A = K]
//   direction b <- a:  out_b^T (16 RHS x 8) += in_a^T (16 RHS x 16) * K (16 x 8)
//                      [A = in_a^T, kept in registers; B = K, transposed through a
//                       warp-private shared tile]
// 3xTF32 products, FP32 accumulation.  Each warp stores its b-side partial of a tile
// in its own shared region; the 8 partials are then summed in warp order (fixed, so
// the result does not depend on scheduling) and written to b's slot (FP64): stored by
// the first chunk of a, added by the later ones (the same thread owns the same
// element in every chunk, so program order keeps the sum ordered).  The a-side sums
// go to FP64 per tile as in k_jit_tc.
constexpr int kPairWarps = 8;
constexpr int kPairChunk = 16 * kPairWarps;

template <int NV>
struct PairSmem {
    static constexpr int NT = NV / 8, TS = 64, NG = TS / 8, NW = kPairWarps;
    float4 pt[2][TS];
    float4 lo[2][TS];          // low parts of the points (Coulomb near field)
    uint4 b[2][NG][NT][32];
    double acc[NW][NT * 4][32];
    float d2[NW][TS][NV];
    float k[NW][16][9];
};

template <int KID, int NV, bool FAR>
__global__ void __launch_bounds__(32 * kPairWarps, 3) k_jit_pair(const PairOwner* __restrict__ owners,
                                                                 const PairPartner* __restrict__ partners,
                                                                 const float4* __restrict__ pts, KParam kp,
                                                                 const double* __restrict__ XS, double* __restrict__ PS,
                                                                 const float4* __restrict__ plo)
{
    constexpr bool EX = KID == KRNL_COULOMB_ID && !FAR;   // exact differences (see two_sum)
    using SM = PairSmem<NV>;
    constexpr int NT = SM::NT, TS = SM::TS, NG = SM::NG, NW = SM::NW, NTH = 32 * NW;
    constexpr int NB = NG * NT * 32 / NTH;        // B-fragment entries staged per thread and tile
    static_assert(NB >= 1 && NB * NTH == NG * NT * 32, "staging split");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SM& sm = *reinterpret_cast<SM*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
    const PairOwner ow = owners[blockIdx.x];
    const float p0 = (float) kp.p0, c0 = (float) kp.c0;
    float q0 = 0.f, q1 = 0.f;
    if constexpr (FAR) ScalarFar<KID>::prep(p0, c0, q0, q1);
    float* sk = &sm.k[warp][0][0];
    float* d2w = &sm.d2[warp][0][0];

    // staging of one tile (points of b and its inputs split into TF32 hi / lo)
    float4 rp = make_float4(0.f, 0.f, 0.f, 0.f), rl = rp;
    double rxa[NB], rxb[NB];
    auto load_tile = [&](int pi, int j0) {
        const PairPartner pb = partners[pi];
        const int nj = min(TS, pb.nb - j0);
        if (threadIdx.x < TS)
        {
            rp = (threadIdx.x < nj) ? pts[pb.pb + j0 + threadIdx.x] : make_float4(1e6f, 1e6f, 1e6f, 0.f);
            if constexpr (EX) rl = (threadIdx.x < nj) ? plo[pb.pb + j0 + threadIdx.x] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < NB; u++)
        {
            const int e = threadIdx.x + u * NTH;
            const int ln = e & 31, n = (e >> 5) % NT, grp = e / (32 * NT);
            const int sa = grp * 8 + (ln & 3), sb = sa + 4, r = n * 8 + (ln >> 2);
            rxa[u] = (sa < nj) ? XS[(long long) (pb.in_b + j0 + sa) * NV + r] : 0.0;
            rxb[u] = (sb < nj) ? XS[(long long) (pb.in_b + j0 + sb) * NV + r] : 0.0;
        }
    };
    auto store_tile = [&](int buf) {
        if (threadIdx.x < TS)
        {
            float4 q = rp;
            if (FAR) q.w = kp.sigma * (q.x * q.x + q.y * q.y + q.z * q.z);   // s |b|^2 for the far form of r^2
            sm.pt[buf][threadIdx.x] = q;
            if constexpr (EX) sm.lo[buf][threadIdx.x] = rl;
        }
#pragma unroll
        for (int u = 0; u < NB; u++)
        {
            const int e = threadIdx.x + u * NTH;
            const int ln = e & 31, n = (e >> 5) % NT, grp = e / (32 * NT);
            const float xa = (float) rxa[u], xb = (float) rxb[u];
            const uint32_t ha = tf32_rna(xa), hb = tf32_rna(xb);
            sm.b[buf][grp][n][ln] = make_uint4(ha, hb, __float_as_uint(xa - __uint_as_float(ha)),
                                               __float_as_uint(xb - __uint_as_float(hb)));
        }
    };
    auto advance = [&](int& pi, int& j0) {
        j0 += TS;
        if (j0 >= partners[pi].nb) { pi++; j0 = 0; }
    };

    for (int ch = 0; ch < ow.na; ch += kPairChunk)
    {
        const int na = min(kPairChunk, ow.na - ch);
        const int i0 = warp * 16 + g, i1 = i0 + 8;
        const bool v0 = i0 < na, v1 = i1 < na;
        const bool warp_on = warp * 16 < na;
        const int n_on = (na + 15) >> 4;
        const float4 x0 = pts[ow.pa + ch + (v0 ? i0 : 0)], x1 = pts[ow.pa + ch + (v1 ? i1 : 0)];
        // in_a^T fragments (16 RHS x 8 rows of a per k-step), hi / lo
        uint32_t ah[2][4], al[2][4];
#pragma unroll
        for (int ks = 0; ks < 2; ks++)
        {
            const int ra = warp * 16 + 8 * ks + tq, rb = ra + 4;
            const long long ia = (long long) (ow.in_a + ch + ra) * NV, ib = (long long) (ow.in_a + ch + rb) * NV;
            float v[4];
            v[0] = (ra < na && g < NV) ? (float) XS[ia + g] : 0.f;
            v[1] = (ra < na && g + 8 < NV) ? (float) XS[ia + g + 8] : 0.f;
            v[2] = (rb < na && g < NV) ? (float) XS[ib + g] : 0.f;
            v[3] = (rb < na && g + 8 < NV) ? (float) XS[ib + g + 8] : 0.f;
#pragma unroll
            for (int q = 0; q < 4; q++)
            {
                ah[ks][q] = tf32_rna(v[q]);
                al[ks][q] = __float_as_uint(v[q] - __uint_as_float(ah[ks][q]));
            }
        }
        float acc[NT][4];
#pragma unroll
        for (int n = 0; n < NT; n++)
#pragma unroll
            for (int q = 0; q < 4; q++) { acc[n][q] = 0.f; sm.acc[warp][n * 4 + q][lane] = 0.0; }

        int ls = ow.p_beg, lj = 0;              // tile being loaded
        __syncthreads();                        // previous chunk's readers of the buffers are done
        if (ls < ow.p_end)
        {
            load_tile(ls, lj);
            store_tile(0);
            advance(ls, lj);
        }
        __syncthreads();
        int cs = ow.p_beg, cj = 0, buf = 0;     // tile being computed
        while (cs < ow.p_end)
        {
            const bool more = ls < ow.p_end;
            if (more) load_tile(ls, lj);
            const PairPartner pb = partners[cs];
            const int nj = min(TS, pb.nb - cj);
            if (warp_on)
            {
                const float ax = x0.x + pb.sx, ay = x0.y + pb.sy, az = x0.z + pb.sz;
                const float bx = x1.x + pb.sx, by = x1.y + pb.sy, bz = x1.z + pb.sz;
                // rows (g, g+8) of a as packed pairs; far form: -2a and |a|^2 in b's frame,
                // scaled by sigma (ScalarFar)
                const float m2s = -2.f * kp.sigma;
                const float2 m_x = make_float2(m2s * ax, m2s * bx), m_y = make_float2(m2s * ay, m2s * by),
                             m_z = make_float2(m2s * az, m2s * bz);
                const float2 s2 = make_float2(kp.sigma * (ax * ax + ay * ay + az * az), kp.sigma * (bx * bx + by * by + bz * bz));
                // exact-difference form: rows (g, g+8) of a as hi + lo pairs in b's frame
                float2 hx = make_float2(ax, bx), hy = make_float2(ay, by), hz = make_float2(az, bz);
                float2 lx = make_float2(0.f, 0.f), ly = lx, lz = lx;
                if constexpr (EX)
                {
                    // the low parts of a's rows, read per tile (fewer live registers)
                    const float4 l0 = plo[ow.pa + ch + (v0 ? i0 : 0)], l1 = plo[ow.pa + ch + (v1 ? i1 : 0)];
                    two_sum(x0.x, pb.sx, l0.x, hx.x, lx.x); two_sum(x1.x, pb.sx, l1.x, hx.y, lx.y);
                    two_sum(x0.y, pb.sy, l0.y, hy.x, ly.x); two_sum(x1.y, pb.sy, l1.y, hy.y, ly.y);
                    two_sum(x0.z, pb.sz, l0.z, hz.x, lz.x); two_sum(x1.z, pb.sz, l1.z, hz.y, lz.y);
                }
                const int ngrp = (nj + 7) >> 3;
                for (int grp = 0; grp < ngrp; grp++)
                {
                    const float4 pa = sm.pt[buf][grp * 8 + tq], pc = sm.pt[buf][grp * 8 + tq + 4];
                    float k[4];
                    if constexpr (FAR)
                    {
                        auto r2p = [&](const float4& p) {
                            float2 t = __fadd2_rn(s2, make_float2(p.w, p.w));
                            t = __ffma2_rn(m_z, make_float2(p.z, p.z), t);
                            t = __ffma2_rn(m_y, make_float2(p.y, p.y), t);
                            return __ffma2_rn(m_x, make_float2(p.x, p.x), t);
                        };
                        const float2 ka = ScalarFar<KID>::f2(r2p(pa), q0, q1);   // (a g, b t), (a g+8, b t)
                        const float2 kb = ScalarFar<KID>::f2(r2p(pc), q0, q1);   // (a g, b t+4), (a g+8, b t+4)
                        k[0] = ka.x; k[1] = ka.y; k[2] = kb.x; k[3] = kb.y;
                    } else if constexpr (EX) {
                        auto r2e = [&](const float4& p, const float4& q) {
                            const float2 dx = __fadd2_rn(__fadd2_rn(hx, make_float2(-p.x, -p.x)),
                                                         __fadd2_rn(lx, make_float2(-q.x, -q.x)));
                            const float2 dy = __fadd2_rn(__fadd2_rn(hy, make_float2(-p.y, -p.y)),
                                                         __fadd2_rn(ly, make_float2(-q.y, -q.y)));
                            const float2 dz = __fadd2_rn(__fadd2_rn(hz, make_float2(-p.z, -p.z)),
                                                         __fadd2_rn(lz, make_float2(-q.z, -q.z)));
                            return __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
                        };
                        const float2 ra2 = r2e(pa, sm.lo[buf][grp * 8 + tq]), rc2 = r2e(pc, sm.lo[buf][grp * 8 + tq + 4]);
                        k[0] = Scalar<KID, float>::f(ra2.x, p0, c0);
                        k[1] = Scalar<KID, float>::f(ra2.y, p0, c0);
                        k[2] = Scalar<KID, float>::f(rc2.x, p0, c0);
                        k[3] = Scalar<KID, float>::f(rc2.y, p0, c0);
                    } else {
                        auto r2d = [&](const float4& p) {
                            const float2 dx = __fadd2_rn(make_float2(ax, bx), make_float2(-p.x, -p.x));
                            const float2 dy = __fadd2_rn(make_float2(ay, by), make_float2(-p.y, -p.y));
                            const float2 dz = __fadd2_rn(make_float2(az, bz), make_float2(-p.z, -p.z));
                            return __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
                        };
                        const float2 ra2 = r2d(pa), rc2 = r2d(pc);
                        k[0] = Scalar<KID, float>::f(ra2.x, p0, c0);   // (a g,   b t)
                        k[1] = Scalar<KID, float>::f(ra2.y, p0, c0);   // (a g+8, b t)
                        k[2] = Scalar<KID, float>::f(rc2.x, p0, c0);   // (a g,   b t+4)
                        k[3] = Scalar<KID, float>::f(rc2.y, p0, c0);   // (a g+8, b t+4)
                    }
                    // rows of a beyond the chunk contribute nothing to b
                    if (!v0) { k[0] = 0.f; k[2] = 0.f; }
                    if (!v1) { k[1] = 0.f; k[3] = 0.f; }
                    // K tile (16 rows of a x 8 points of b) to the warp's shared tile
                    sk[g * 9 + tq] = k[0];
                    sk[(g + 8) * 9 + tq] = k[1];
                    sk[g * 9 + tq + 4] = k[2];
                    sk[(g + 8) * 9 + tq + 4] = k[3];
                    uint32_t hi[4], lo[4];
#pragma unroll
                    for (int q = 0; q < 4; q++)
                    {
                        hi[q] = tf32_rna(k[q]);
                        lo[q] = __float_as_uint(k[q] - __uint_as_float(hi[q]));
                    }
                    uint4 b[NT];
#pragma unroll
                    for (int n = 0; n < NT; n++) b[n] = sm.b[buf][grp][n][lane];
#pragma unroll
                    for (int n = 0; n < NT; n++) mma_tf32(acc[n], lo[0], lo[1], lo[2], lo[3], b[n].x, b[n].y);
#pragma unroll
                    for (int n = 0; n < NT; n++) mma_tf32(acc[n], hi[0], hi[1], hi[2], hi[3], b[n].z, b[n].w);
#pragma unroll
                    for (int n = 0; n < NT; n++) mma_tf32(acc[n], hi[0], hi[1], hi[2], hi[3], b[n].x, b[n].y);
                    __syncwarp();
                    float kt[4];
                    kt[0] = sk[tq * 9 + g];          // k-step 0: K[a = tq][b = g]
                    kt[1] = sk[(tq + 4) * 9 + g];    //           K[a = tq + 4][b = g]
                    kt[2] = sk[(tq + 8) * 9 + g];    // k-step 1: K[a = 8 + tq][b = g]
                    kt[3] = sk[(tq + 12) * 9 + g];   //           K[a = 12 + tq][b = g]
                    __syncwarp();
                    uint32_t th[4], tl[4];
#pragma unroll
                    for (int q = 0; q < 4; q++)
                    {
                        th[q] = tf32_rna(kt[q]);
                        tl[q] = __float_as_uint(kt[q] - __uint_as_float(th[q]));
                    }
                    // two independent chains (one per k-step), summed at the end
                    float da[4] = {0.f, 0.f, 0.f, 0.f}, db[4] = {0.f, 0.f, 0.f, 0.f};
                    mma_tf32(da, al[0][0], al[0][1], al[0][2], al[0][3], th[0], th[1]);
                    mma_tf32(db, al[1][0], al[1][1], al[1][2], al[1][3], th[2], th[3]);
                    mma_tf32(da, ah[0][0], ah[0][1], ah[0][2], ah[0][3], tl[0], tl[1]);
                    mma_tf32(db, ah[1][0], ah[1][1], ah[1][2], ah[1][3], tl[2], tl[3]);
                    mma_tf32(da, ah[0][0], ah[0][1], ah[0][2], ah[0][3], th[0], th[1]);
                    mma_tf32(db, ah[1][0], ah[1][1], ah[1][2], ah[1][3], th[2], th[3]);
                    // rows = RHS (g, g+8), columns = points of b (2t, 2t+1)
                    float* row0 = d2w + (grp * 8 + 2 * tq) * NV;
                    row0[g] = da[0] + db[0];
                    row0[NV + g] = da[1] + db[1];
                    if (NV > 8)
                    {
                        row0[g + 8] = da[2] + db[2];
                        row0[NV + g + 8] = da[3] + db[3];
                    }
                }
#pragma unroll
                for (int n = 0; n < NT; n++)
#pragma unroll
                    for (int q = 0; q < 4; q++)
                    {
                        sm.acc[warp][n * 4 + q][lane] += (double) acc[n][q];
                        acc[n][q] = 0.f;
                    }
            }
            if (more) store_tile(buf ^ 1);
            __syncthreads();                    // all partials of this tile written; next tile staged
            for (int e = threadIdx.x; e < nj * NV; e += NTH)
            {
                float t = 0.f;
                for (int w = 0; w < n_on; w++) t += (&sm.d2[w][0][0])[e];
                double* o = PS + (long long) (pb.out_b + cj) * NV + e;
                *o = (ch == 0) ? (double) t : *o + (double) t;
            }
            __syncthreads();                    // partials read before the next tile overwrites them
            cs = ls; cj = lj; buf ^= 1;
            if (more) advance(ls, lj);
        }
        if (warp_on)
        {
            double* base = PS + (long long) (ow.out_a + ch) * NV;
#pragma unroll
            for (int n = 0; n < NT; n++)
#pragma unroll
                for (int q = 0; q < 4; q++)
                {
                    const int row = (q < 2) ? i0 : i1;
                    const bool ok = (q < 2) ? v0 : v1;
                    if (ok) base[(long long) row * NV + n * 8 + 2 * tq + (q & 1)] = sm.acc[warp][n * 4 + q][lane];
                }
        }
    }
}

template <int NV>
constexpr int pair_smem_bytes()
{
    return (int) sizeof(PairSmem<NV>);
}

// --------------------------------------- stored blocks on the tensor cores (FP32)

// Stored block task (up to 1024 rows x ncol, FP32 copy, walked in chunks of R <= 64
// rows) for panels of 8 / 16 right-hand sides, both products on the tensor cores with
// the right-hand sides as the M = 16 side of m16n8k8 (3xTF32, FP32 accumulation):
//   C1^T (NV x ncol) = W^T (NV x R) A        [B operand = A, k = rows]      warps 0-3
//   C0^T (NV x R)    = V^T (NV x ncol) A^T   [B operand = A^T, k = columns] warps 4-7
// Column tiles of 64 are copied to shared memory by 4-byte cp.async one tile ahead of
// the math (double buffer, 58 KB of dynamic shared memory, 3 CTAs per SM, one barrier
// per 64 columns); each tile feeds both products.  Warp w < 4 owns columns
// 16w..16w+15 of every tile and completes the chunk's part of C1 for them over its R
// rows (two FP32 chains over alternate 8-row steps), stored by the first chunk into the
// task's single C1 slot and added by the later ones (FP64; the same thread owns the same
// element in every chunk; the value it adds to is read before the MMAs); warp 4 + u
// owns rows 16u..16u+15 of the chunk and sums C0 over the tiles (FP32 per 32 columns,
// FP64 across).
struct BlkTcSmem {
    float a[2][64][68];          // A tiles (64 rows x 64 columns, padded rows), double-buffered
    uint4 w[8][32][2];           // W^T fragments per k-step of 8 rows: hi, lo
    uint4 v[2][8][32][2];        // V^T fragments per k-step of 8 columns: hi, lo
};

template <int NV>
__global__ void __launch_bounds__(256, 3) k_blk_tc(const BlkTask* __restrict__ tasks, const float* __restrict__ arena,
                                                   const double* __restrict__ XS, double* __restrict__ PS)
{
    constexpr int CT = 64, S = CT + 4;            // tile width; padded shared row
    extern __shared__ __align__(16) unsigned char blktc_raw[];
    BlkTcSmem& sm = *reinterpret_cast<BlkTcSmem*>(blktc_raw);
    const BlkTask T = tasks[blockIdx.x];
    const int ncol = T.ncol;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
    const bool do0 = T.out0_row >= 0, do1 = T.out1_row >= 0;

    // A-fragment of an (NV x 8) slice of X^T: X rows k0 + {tq, tq+4}, right-hand sides {g, g+8}
    auto frag = [&](int row0, int nrows, int k0, uint4& hi, uint4& lo) {
        float v[4];
        const int ra = k0 + tq, rb = ra + 4;
        v[0] = (ra < nrows && g < NV) ? (float) XS[(long long) (row0 + ra) * NV + g] : 0.f;
        v[1] = (ra < nrows && g + 8 < NV) ? (float) XS[(long long) (row0 + ra) * NV + g + 8] : 0.f;
        v[2] = (rb < nrows && g < NV) ? (float) XS[(long long) (row0 + rb) * NV + g] : 0.f;
        v[3] = (rb < nrows && g + 8 < NV) ? (float) XS[(long long) (row0 + rb) * NV + g + 8] : 0.f;
        uint32_t h[4], l[4];
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            h[q] = tf32_rna(v[q]);
            l[q] = __float_as_uint(v[q] - __uint_as_float(h[q]));
        }
        hi = make_uint4(h[0], h[1], h[2], h[3]);
        lo = make_uint4(l[0], l[1], l[2], l[3]);
    };

    for (int rc = 0; rc < T.nrow; rc += 64)
    {
        const float* A = arena + T.a32 + (long long) rc * T.ld32;
        const int R = min(64, T.nrow - rc);
        __syncthreads();
        if (do1)
            frag(T.in1_row + rc, R, 8 * warp, sm.w[warp][lane][0], sm.w[warp][lane][1]);
        const int nct = (ncol + CT - 1) / CT;
        auto issue_tile = [&](int t) {
            if (t < nct)
            {
                const int c0 = t * CT;
                float* dst = &sm.a[t & 1][0][0];
#pragma unroll
                for (int u = 0; u < 16; u++)
                {
                    const int e = threadIdx.x + 256 * u, r = e >> 6, c = e & 63;
                    const bool in = r < R && c0 + c < ncol;
                    const float* src = in ? A + (long long) r * T.ld32 + c0 + c : A;
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;"
                                 ::"r"(smem_u32(dst + r * S + c)), "l"(src), "r"(in ? 4 : 0) : "memory");
                }
            }
            cp_async_commit();
        };
        uint4 rvh = make_uint4(0, 0, 0, 0), rvl = rvh;
        auto load_v = [&](int c0) {
            if (do0) frag(T.in0_row + c0, ncol - c0, 8 * warp, rvh, rvl);
        };
        auto store_v = [&](int buf) {
            if (do0) { sm.v[buf][warp][lane][0] = rvh; sm.v[buf][warp][lane][1] = rvl; }
        };

        double c0acc[2][4];
#pragma unroll
        for (int n = 0; n < 2; n++)
#pragma unroll
            for (int q = 0; q < 4; q++) c0acc[n][q] = 0.0;

        issue_tile(0);
        if (ncol > 0) { load_v(0); store_v(0); }
        cp_async_wait_all();
        __syncthreads();
        int buf = 0;
        for (int c0 = 0; c0 < ncol; c0 += CT)
        {
            const int t = c0 / CT;
            const bool more = c0 + CT < ncol;
            issue_tile(t + 1);                    // into the other buffer, read two tiles ago
            if (more) load_v(c0 + CT);
            if (warp < 4)
            {
                if (do1)
                {
                    // C1^T for columns c0 + 16w .. +15 (two n-tiles): k over the R rows
                    double old[2][4];
#pragma unroll
                    for (int j = 0; j < 2; j++)
#pragma unroll
                        for (int q = 0; q < 4; q++)
                        {
                            const int rhs = (q < 2) ? g : g + 8, col = c0 + 16 * warp + 8 * j + 2 * tq + (q & 1);
                            old[j][q] = (rc > 0 && rhs < NV && col < ncol) ? PS[(long long) (T.out1_row + col) * NV + rhs] : 0.0;
                        }
                    float d[2][2][4] = {};                // [n-tile][two chains over alternate k-steps]
                    const int ksteps = (R + 7) >> 3;
#pragma unroll
                    for (int ks = 0; ks < 8; ks++)
                    {
                        if (ks >= ksteps) break;
                        const uint4 wh = sm.w[ks][lane][0], wl = sm.w[ks][lane][1];
#pragma unroll
                        for (int j = 0; j < 2; j++)
                        {
                            const float b0 = sm.a[buf][8 * ks + tq][16 * warp + 8 * j + g];
                            const float b1 = sm.a[buf][8 * ks + tq + 4][16 * warp + 8 * j + g];
                            const uint32_t h0 = tf32_rna(b0), h1 = tf32_rna(b1);
                            const uint32_t l0 = __float_as_uint(b0 - __uint_as_float(h0)),
                                           l1 = __float_as_uint(b1 - __uint_as_float(h1));
                            float (&dd)[4] = d[j][ks & 1];
                            mma_tf32(dd, wl.x, wl.y, wl.z, wl.w, h0, h1);
                            mma_tf32(dd, wh.x, wh.y, wh.z, wh.w, l0, l1);
                            mma_tf32(dd, wh.x, wh.y, wh.z, wh.w, h0, h1);
                        }
                    }
#pragma unroll
                    for (int j = 0; j < 2; j++)
#pragma unroll
                        for (int q = 0; q < 4; q++)
                        {
                            const int rhs = (q < 2) ? g : g + 8, col = c0 + 16 * warp + 8 * j + 2 * tq + (q & 1);
                            if (rhs < NV && col < ncol)
                            {
                                const double v = (double) (d[j][0][q] + d[j][1][q]);
                                PS[(long long) (T.out1_row + col) * NV + rhs] = (rc == 0) ? v : old[j][q] + v;
                            }
                        }
                }
            } else if (do0) {
                // C0^T for rows 16u .. 16u+15 (two n-tiles of 8): k over the tile's 64 columns
                const int u = warp - 4;
                if (16 * u < R)
#pragma unroll
                for (int half = 0; half < 2; half++)   // FP32 sums over 32 columns, FP64 across
                {
                    float d[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
                    for (int ks = 4 * half; ks < 4 * half + 4; ks++)
                    {
                        const uint4 vh = sm.v[buf][ks][lane][0], vl = sm.v[buf][ks][lane][1];
#pragma unroll
                        for (int n = 0; n < 2; n++)
                        {
                            const int row = 16 * u + 8 * n + g;
                            const float b0 = sm.a[buf][row][8 * ks + tq], b1 = sm.a[buf][row][8 * ks + tq + 4];
                            const uint32_t h0 = tf32_rna(b0), h1 = tf32_rna(b1);
                            const uint32_t l0 = __float_as_uint(b0 - __uint_as_float(h0)),
                                           l1 = __float_as_uint(b1 - __uint_as_float(h1));
                            mma_tf32(d[n], vl.x, vl.y, vl.z, vl.w, h0, h1);
                            mma_tf32(d[n], vh.x, vh.y, vh.z, vh.w, l0, l1);
                            mma_tf32(d[n], vh.x, vh.y, vh.z, vh.w, h0, h1);
                        }
                    }
#pragma unroll
                    for (int n = 0; n < 2; n++)
#pragma unroll
                        for (int q = 0; q < 4; q++) c0acc[n][q] += (double) d[n][q];
                }
            }
            if (more) store_v(buf ^ 1);
            cp_async_wait_all();                  // tile t+1 has landed
            __syncthreads();                      // ... for every thread; tile t no longer read
            buf ^= 1;
        }
        if (do0 && warp >= 4)
        {
            const int u = warp - 4;
#pragma unroll
            for (int n = 0; n < 2; n++)
#pragma unroll
                for (int q = 0; q < 4; q++)
                {
                    const int rhs = (q < 2) ? g : g + 8, row = 16 * u + 8 * n + 2 * tq + (q & 1);
                    if (rhs < NV && row < R) PS[(long long) (T.out0_row + rc + row) * NV + rhs] = c0acc[n][q];
                }
        }
    }
}

template <int NV>
constexpr int blk_tc_smem_bytes() { return (int) sizeof(BlkTcSmem); }

// ------------------------------------ stored blocks on tcgen05 (TMEM accumulators)

// PTX wrappers (sm_100a).  Shared addresses are 32-bit shared-window addresses.

// Shared-memory matrix descriptor: start address, leading / stride byte offsets (16-byte
// units), version 1, layout type (0 = no swizzle, 2 = 128-byte swizzle).
__device__ __forceinline__ uint64_t umma_desc(uint32_t start, uint32_t lbo_bytes, uint32_t sbo_bytes, uint32_t layout)
{
    return (uint64_t) ((start >> 4) & 0x3FFFu) | ((uint64_t) ((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           ((uint64_t) ((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t) layout << 61);
}

__device__ __forceinline__ void umma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
    return ok != 0;
}

// ----------------------------- stored blocks on tcgen05, BF16x3 split (one tile layout)

// Instruction descriptor, kind::f16 with BF16 A and B, FP32 accumulator: A K-major (0)
// or MN-major (1), B K-major, N = n, M = 64.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n, int a_mn_major)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) a_mn_major << 15) | ((uint32_t) (n >> 3) << 17) |
           ((uint32_t) (64 >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc) : "memory");
}

// x = h + m + l exactly up to the last bits of l: three BF16 pieces (8 significant bits
// each) of an FP32 value, each the round-to-nearest of the remainder.
__device__ __forceinline__ void bf16x3(float x, uint16_t& h, uint16_t& m, uint16_t& l)
{
    const __nv_bfloat16 bh = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(bh);
    const __nv_bfloat16 bm = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(bm);
    const __nv_bfloat16 bl = __float2bfloat16_rn(r2);
    h = __bfloat16_as_ushort(bh); m = __bfloat16_as_ushort(bm); l = __bfloat16_as_ushort(bl);
}

// One stored block task (up to 1024 rows x ncol, FP32 copy) for panels of 8 / 16
// right-hand sides on the 5th-generation tensor cores, both products per 64 x 64 tile
// of A with the tile read from HBM once:
//   C0 (64 rows x NV) += A_tile V_tile       A K-major  (k = the tile's columns) -> TMEM columns 0-15
//   C1 (64 cols x NV)  = A_tile^T W_chunk    A MN-major (k = the tile's rows)    -> TMEM columns 16-31
// Each value is split into three BF16 pieces h + m + l (24 significant bits, the whole
// FP32 value) and the products keep the six terms down to 2^-16 relative
// (l.h + h.l + m.m + m.h + h.m + h.h, smallest first), summed in FP32 in TMEM over one
// tile (64 terms deep) and in FP64 across tiles.  With 16-bit pieces one 128-byte-
// swizzled copy of each piece (rows of 64 columns) serves both the K-major and the
// MN-major view, so a tile takes 24 KB of shared memory and several CTAs fit an SM.
// Per tile: the threads store the tile's pieces (loaded into registers while the
// previous tile's MMAs ran), one thread issues the 48 MMAs and commits them to an
// mbarrier, the threads load the next tile, then read the accumulators: C1 is added
// into the task's C1 slot, C0 into FP64 registers written when the 64-row chunk ends.
// Every wait on the mbarrier is bounded: on expiry the kernel records a status and
// stops issuing work.
struct Bf3Smem {
    uint16_t a[3][64 * 64];    // A tile pieces h, m, l: 64 rows of 128 B, 128-byte swizzle
    uint16_t v[3][16 * 64];    // V^T pieces (NV rows of the tile's 64 columns)
    uint16_t w[3][16 * 64];    // W^T pieces (NV rows of the chunk's 64 rows)
    double c0acc[64][17];      // the chunk's C0 rows in FP64 (row 16 warp + lane; padded)
    unsigned long long mbar;
    uint32_t tmem;
};
constexpr int kBf3Threads = 128;

// byte offset of 16-byte granule q (8 BF16) of row r in a 128-byte-swizzled tile
__device__ __forceinline__ int sw128(int r, int q) { return r * 128 + ((q ^ (r & 7)) << 4); }

template <int NV>
__global__ void __launch_bounds__(kBf3Threads, 5) k_blk_bf3(const BlkTask* __restrict__ tasks,
                                                            const float* __restrict__ arena,
                                                            const double* __restrict__ XS, double* __restrict__ PS,
                                                            int* __restrict__ status)
{
    constexpr uint32_t IDESC0 = umma_idesc_bf16(NV, 0), IDESC1 = umma_idesc_bf16(NV, 1);
    extern __shared__ __align__(1024) unsigned char bf3_raw[];
    Bf3Smem& sm = *reinterpret_cast<Bf3Smem*>(bf3_raw + ((1024 - (smem_u32(bf3_raw) & 1023)) & 1023));
    const BlkTask T = tasks[blockIdx.x];
    const int ncol = T.ncol, nrow = T.nrow;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool do0 = T.out0_row >= 0, do1 = T.out1_row >= 0;
    const int ntc = (ncol + 63) / 64, nt = ntc * ((nrow + 63) / 64);
    const float* A0 = arena + T.a32;

    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(smem_u32(&sm.tmem)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sm.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem, mbar = smem_u32(&sm.mbar);
    unsigned char* const a_b = reinterpret_cast<unsigned char*>(sm.a);
    unsigned char* const v_b = reinterpret_cast<unsigned char*>(sm.v);
    unsigned char* const w_b = reinterpret_cast<unsigned char*>(sm.w);
    const uint32_t a_s = smem_u32(sm.a), v_s = smem_u32(sm.v), w_s = smem_u32(sm.w);

    // registers of the tile being loaded: thread t holds 4 granules (8 columns each) of A
    // and one granule of V^T and of W^T (rows n < NV of 8 consecutive k)
    float ra[4][8];
    float rv[8], rw[8];
    auto load_tile = [&](int t) {
        const int rc = (t / ntc) * 64, c0 = (t % ntc) * 64, R = min(64, nrow - rc);
        const float* A = A0 + (long long) rc * T.ld32 + c0;
#pragma unroll
        for (int u = 0; u < 4; u++)
        {
            const int gi = tid + kBf3Threads * u, r = gi >> 3, q = gi & 7;
#pragma unroll
            for (int j = 0; j < 8; j++)
            {
                const int c = 8 * q + j;
                ra[u][j] = (r < R && c0 + c < ncol) ? A[(long long) r * T.ld32 + c] : 0.f;
            }
        }
        const int n = tid >> 3, q = tid & 7;          // V^T / W^T granule: row n, k = 8q .. 8q+7
#pragma unroll
        for (int j = 0; j < 8; j++)
        {
            const int k = 8 * q + j;
            rv[j] = (n < NV && do0 && c0 + k < ncol) ? (float) XS[(long long) (T.in0_row + c0 + k) * NV + n] : 0.f;
            rw[j] = (n < NV && do1 && c0 == 0 && k < R) ? (float) XS[(long long) (T.in1_row + rc + k) * NV + n] : 0.f;
        }
    };
    auto put = [&](unsigned char* base, int stride, int off, const float (&x)[8]) {
        uint16_t h[8], m[8], l[8];
#pragma unroll
        for (int j = 0; j < 8; j++) bf16x3(x[j], h[j], m[j], l[j]);
        auto pack = [](const uint16_t (&e)[8]) {
            return make_uint4(e[0] | ((uint32_t) e[1] << 16), e[2] | ((uint32_t) e[3] << 16),
                              e[4] | ((uint32_t) e[5] << 16), e[6] | ((uint32_t) e[7] << 16));
        };
        *reinterpret_cast<uint4*>(base + off) = pack(h);
        *reinterpret_cast<uint4*>(base + stride + off) = pack(m);
        *reinterpret_cast<uint4*>(base + 2 * stride + off) = pack(l);
    };
    auto store_tile = [&](int t) {
        const int c0 = (t % ntc) * 64;
#pragma unroll
        for (int u = 0; u < 4; u++)
        {
            const int gi = tid + kBf3Threads * u, r = gi >> 3, q = gi & 7;
            put(a_b, 64 * 64 * 2, sw128(r, q), ra[u]);
        }
        const int n = tid >> 3, q = tid & 7;
        if (n < NV)
        {
            put(v_b, 16 * 64 * 2, sw128(n, q), rv);
            if (c0 == 0) put(w_b, 16 * 64 * 2, sw128(n, q), rw);
        }
    };

    bool ok = true;
    uint32_t phase = 0;
    // lanes 0-15: the chunk's C0 row 16 warp + lane, summed in shared memory
    double* const c0acc = sm.c0acc[(16 * warp + lane) & 63];
    if (lane < 16)
#pragma unroll
        for (int n = 0; n < NV; n++) c0acc[n] = 0.0;
    // read back the tile just multiplied: C1 into its slot, C0 into the chunk's FP64 sums
    auto drain = [&](int t) {
        int good = 1;
        if (tid == 0)
        {
            int it = 0;
            while (!mbar_try_wait(mbar, phase))
                if (++it > (1 << 22)) { good = 0; break; }
            if (!good) atomicExch(status, 1);
        }
        phase ^= 1;
        ok = __syncthreads_and(good) != 0;
        if (!ok) return;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t d[32];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                     "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                     : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
                       "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
                       "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]),
                       "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
                     : "r"(tmem + ((uint32_t) (32 * warp) << 16)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int rc = (t / ntc) * 64, c0 = (t % ntc) * 64, R = min(64, nrow - rc);
        const int m = 16 * warp + lane;
        if (lane < 16)
        {
            if (do1 && c0 + m < ncol)
            {
                double* o = PS + (long long) (T.out1_row + c0 + m) * NV;
#pragma unroll
                for (int n = 0; n < NV; n++)
                {
                    const double v = (double) __uint_as_float(d[16 + n]);
                    o[n] = (rc == 0) ? v : o[n] + v;
                }
            }
            if (do0)
            {
#pragma unroll
                for (int n = 0; n < NV; n++) c0acc[n] += (double) __uint_as_float(d[n]);
                if (c0 + 64 >= ncol)
                {
                    if (m < R)
                    {
                        double* o = PS + (long long) (T.out0_row + rc + m) * NV;
#pragma unroll
                        for (int n = 0; n < NV; n++) o[n] = c0acc[n];
                    }
#pragma unroll
                    for (int n = 0; n < NV; n++) c0acc[n] = 0.0;
                }
            }
        }
    };

    // the six products of one K-step: (A piece, B piece), smallest first
    constexpr int PA[6] = {2, 0, 1, 1, 0, 0}, PB[6] = {0, 2, 1, 0, 1, 0};
    if (nt > 0) load_tile(0);
    for (int t = 0; t < nt; t++)
    {
        if (t > 0) drain(t - 1);
        if (!ok) break;
        store_tile(t);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0)
        {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int ks = 0; ks < 4; ks++)          // K-steps of 16
#pragma unroll
                for (int p = 0; p < 6; p++)
                {
                    // C0: A K-major (32-byte step along the row), B = V^T K-major
                    if (do0)
                        umma_f16(tmem, umma_desc(a_s + PA[p] * 8192 + ks * 32, 16, 1024, 2),
                                 umma_desc(v_s + PB[p] * 2048 + ks * 32, 16, 1024, 2), IDESC0,
                                 (ks == 0 && p == 0) ? 0u : 1u);
                    // C1: A MN-major (16 rows = two 8-row swizzle atoms per step), B = W^T K-major
                    if (do1)
                        umma_f16(tmem + 16u, umma_desc(a_s + PA[p] * 8192 + ks * 2048, 8192, 1024, 2),
                                 umma_desc(w_s + PB[p] * 2048 + ks * 32, 16, 1024, 2), IDESC1,
                                 (ks == 0 && p == 0) ? 0u : 1u);
                }
            umma_commit(mbar);
        }
        if (t + 1 < nt) load_tile(t + 1);
    }
    if (ok && nt > 0) drain(nt - 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
    {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
    }
}

template <int NV>
constexpr int bf3_smem_bytes() { return (int) sizeof(Bf3Smem) + 1024; }

// --------------------------- stored blocks on tcgen05, wide panels (32 / 64 right-hand sides)

// The k_blk_bf3 scheme for panels of NV = 32 or 64 right-hand sides, so that a matmul of
// up to 64 right-hand sides streams every stored block once (H2P_matmul applies each
// block to up to mm_max_n_vec right-hand sides per read, src/H2Pack_matmul.c:497).
// Per 64 x 64 tile of A (FP32, read from HBM once, split into BF16 pieces h + m + l):
//   C0 (64 rows x NV) += A_tile V_tile   (MMA M = 64, N = NV, A K-major)  TMEM columns [0, NV)
//   C1 (64 cols x NV)  = A_tile^T W      (MMA M = 64, N = NV, A MN-major) TMEM columns [NV, 2 NV)
// six products per 16-deep K step (l.h + h.l + m.m + m.h + h.m + h.h), FP32 in TMEM over
// one tile (64 terms), FP64 across tiles (C0 in shared memory per 64-row chunk, C1 added
// into the task's slot).  V^T / W^T are NV rows of 64 BF16 (128 B, 128-byte swizzle),
// B operands K-major, as k_blk_bf3.  The accumulators are read back 32 columns at a time.
// 105 KB of shared memory: two CTAs per SM, whose tile loads and MMAs interleave.
template <int NV>
struct Bf3wSmem {
    uint16_t a[3][64 * 64];    // A tile pieces h, m, l: 64 rows of 128 B, 128-byte swizzle
    uint16_t v[3][NV * 64];    // V^T pieces (NV rows of the tile's 64 columns)
    uint16_t w[3][NV * 64];    // W^T pieces (NV rows of the chunk's 64 rows)
    double c0acc[64][NV + 1];  // the chunk's C0 rows in FP64 (row 16 warp + lane; padded)
    unsigned long long mbar;
    uint32_t tmem;
};

template <int NV>
constexpr int bf3w_smem_bytes() { return (int) sizeof(Bf3wSmem<NV>) + 1024; }

template <int NV>
__global__ void __launch_bounds__(kBf3Threads, 2) k_blk_bf3w(const BlkTask* __restrict__ tasks,
                                                             const float* __restrict__ arena,
                                                             const double* __restrict__ XS, double* __restrict__ PS,
                                                             int* __restrict__ status)
{
    static_assert(NV == 32 || NV == 64, "wide panels of 32 or 64 right-hand sides");
    constexpr uint32_t IDESC0 = umma_idesc_bf16(NV, 0), IDESC1 = umma_idesc_bf16(NV, 1);
    constexpr uint32_t TCOLS = 2 * NV;            // C0 and C1 (a power of two >= 32)
    constexpr int VG = NV / 16;                   // granules of V^T / W^T per thread
    constexpr int PIECE_VW = NV * 64 * 2;         // bytes of one piece of V^T / W^T
    extern __shared__ __align__(1024) unsigned char bf3w_raw[];
    Bf3wSmem<NV>& sm = *reinterpret_cast<Bf3wSmem<NV>*>(bf3w_raw + ((1024 - (smem_u32(bf3w_raw) & 1023)) & 1023));
    const BlkTask T = tasks[blockIdx.x];
    const int ncol = T.ncol, nrow = T.nrow;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool do0 = T.out0_row >= 0, do1 = T.out1_row >= 0;
    const int ntc = (ncol + 63) / 64, nt = ntc * ((nrow + 63) / 64);
    const float* A0 = arena + T.a32;

    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&sm.tmem)), "n"(TCOLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sm.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem, mbar = smem_u32(&sm.mbar);
    unsigned char* const a_b = reinterpret_cast<unsigned char*>(sm.a);
    unsigned char* const v_b = reinterpret_cast<unsigned char*>(sm.v);
    unsigned char* const w_b = reinterpret_cast<unsigned char*>(sm.w);
    const uint32_t a_s = smem_u32(sm.a), v_s = smem_u32(sm.v), w_s = smem_u32(sm.w);

    // registers of the tile being loaded: thread t holds 4 granules (8 columns each) of A
    // and VG granules of V^T and of W^T (row n, 8 consecutive k each)
    float ra[4][8];
    float rv[VG][8], rw[VG][8];
    auto load_tile = [&](int t) {
        const int rc = (t / ntc) * 64, c0 = (t % ntc) * 64, R = min(64, nrow - rc);
        const float* A = A0 + (long long) rc * T.ld32 + c0;
#pragma unroll
        for (int u = 0; u < 4; u++)
        {
            const int gi = tid + kBf3Threads * u, r = gi >> 3, q = gi & 7;
#pragma unroll
            for (int j = 0; j < 8; j++)
            {
                const int c = 8 * q + j;
                ra[u][j] = (r < R && c0 + c < ncol) ? A[(long long) r * T.ld32 + c] : 0.f;
            }
        }
#pragma unroll
        for (int u = 0; u < VG; u++)
        {
            const int gi = tid + kBf3Threads * u, n = gi >> 3, q = gi & 7;
#pragma unroll
            for (int j = 0; j < 8; j++)
            {
                const int k = 8 * q + j;
                rv[u][j] = (do0 && c0 + k < ncol) ? (float) XS[(long long) (T.in0_row + c0 + k) * NV + n] : 0.f;
                rw[u][j] = (do1 && c0 == 0 && k < R) ? (float) XS[(long long) (T.in1_row + rc + k) * NV + n] : 0.f;
            }
        }
    };
    auto put = [&](unsigned char* base, int stride, int off, const float (&x)[8]) {
        uint16_t h[8], m[8], l[8];
#pragma unroll
        for (int j = 0; j < 8; j++) bf16x3(x[j], h[j], m[j], l[j]);
        auto pack = [](const uint16_t (&e)[8]) {
            return make_uint4(e[0] | ((uint32_t) e[1] << 16), e[2] | ((uint32_t) e[3] << 16),
                              e[4] | ((uint32_t) e[5] << 16), e[6] | ((uint32_t) e[7] << 16));
        };
        *reinterpret_cast<uint4*>(base + off) = pack(h);
        *reinterpret_cast<uint4*>(base + stride + off) = pack(m);
        *reinterpret_cast<uint4*>(base + 2 * stride + off) = pack(l);
    };
    auto store_tile = [&](int t) {
        const int c0 = (t % ntc) * 64;
#pragma unroll
        for (int u = 0; u < 4; u++)
        {
            const int gi = tid + kBf3Threads * u, r = gi >> 3, q = gi & 7;
            put(a_b, 64 * 64 * 2, sw128(r, q), ra[u]);
        }
#pragma unroll
        for (int u = 0; u < VG; u++)
        {
            const int gi = tid + kBf3Threads * u, n = gi >> 3, q = gi & 7;
            put(v_b, PIECE_VW, sw128(n, q), rv[u]);
            if (c0 == 0) put(w_b, PIECE_VW, sw128(n, q), rw[u]);
        }
    };

    bool ok = true;
    uint32_t phase = 0;
    // lanes 0-15: the chunk's C0 row 16 warp + lane, summed in shared memory
    double* const c0acc = sm.c0acc[(16 * warp + lane) & 63];
    if (lane < 16)
        for (int n = 0; n < NV; n++) c0acc[n] = 0.0;
    // read back the tile just multiplied: C1 into its slot, C0 into the chunk's FP64 sums
    auto drain = [&](int t) {
        int good = 1;
        if (tid == 0)
        {
            int it = 0;
            while (!mbar_try_wait(mbar, phase))
                if (++it > (1 << 22)) { good = 0; break; }
            if (!good) atomicExch(status, 1);
        }
        phase ^= 1;
        ok = __syncthreads_and(good) != 0;
        if (!ok) return;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int rc = (t / ntc) * 64, c0 = (t % ntc) * 64, R = min(64, nrow - rc);
        const int m = 16 * warp + lane;
        const bool last_tc = c0 + 64 >= ncol;
#pragma unroll
        for (int h = 0; h < 2 * NV / 32; h++)        // 32 accumulator columns at a time
        {
            uint32_t d[32];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                         "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                         : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
                           "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
                           "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]),
                           "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
                         : "r"(tmem + ((uint32_t) (32 * warp) << 16) + (uint32_t) (32 * h)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (lane >= 16) continue;
            const bool is_c1 = 32 * h >= NV;
            const int n0 = is_c1 ? 32 * h - NV : 32 * h;
            if (is_c1)
            {
                if (do1 && c0 + m < ncol)
                {
                    double* o = PS + (long long) (T.out1_row + c0 + m) * NV + n0;
#pragma unroll
                    for (int n = 0; n < 32; n++)
                    {
                        const double v = (double) __uint_as_float(d[n]);
                        o[n] = (rc == 0) ? v : o[n] + v;
                    }
                }
            } else if (do0) {
#pragma unroll
                for (int n = 0; n < 32; n++) c0acc[n0 + n] += (double) __uint_as_float(d[n]);
                if (last_tc)
                {
                    if (m < R)
                    {
                        double* o = PS + (long long) (T.out0_row + rc + m) * NV + n0;
#pragma unroll
                        for (int n = 0; n < 32; n++) o[n] = c0acc[n0 + n];
                    }
#pragma unroll
                    for (int n = 0; n < 32; n++) c0acc[n0 + n] = 0.0;
                }
            }
        }
    };

    // the six products of one K-step: (A piece, B piece), smallest first
    constexpr int PA[6] = {2, 0, 1, 1, 0, 0}, PB[6] = {0, 2, 1, 0, 1, 0};
    if (nt > 0) load_tile(0);
    for (int t = 0; t < nt; t++)
    {
        if (t > 0) drain(t - 1);
        if (!ok) break;
        store_tile(t);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0)
        {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int ks = 0; ks < 4; ks++)          // K-steps of 16
#pragma unroll
                for (int p = 0; p < 6; p++)
                {
                    // C0: A K-major (32-byte step along the row), B = V^T K-major
                    if (do0)
                        umma_f16(tmem, umma_desc(a_s + PA[p] * 8192 + ks * 32, 16, 1024, 2),
                                 umma_desc(v_s + PB[p] * PIECE_VW + ks * 32, 16, 1024, 2), IDESC0,
                                 (ks == 0 && p == 0) ? 0u : 1u);
                    // C1: A MN-major (16 rows = two 8-row swizzle atoms per step), B = W^T K-major
                    if (do1)
                        umma_f16(tmem + (uint32_t) NV, umma_desc(a_s + PA[p] * 8192 + ks * 2048, 8192, 1024, 2),
                                 umma_desc(w_s + PB[p] * PIECE_VW + ks * 32, 16, 1024, 2), IDESC1,
                                 (ks == 0 && p == 0) ? 0u : 1u);
                }
            umma_commit(mbar);
        }
        if (t + 1 < nt) load_tile(t + 1);
    }
    if (ok && nt > 0) drain(nt - 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
    {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(TCOLS) : "memory");
    }
}


// ------------------------ stored blocks on tcgen05, 64-wide panels as two GEMM passes

// Instruction descriptor, kind::f16 with BF16 A and B, FP32 accumulator, M = 64, N = n,
// A and B each K-major (0) or MN-major (1).
__host__ __device__ constexpr uint32_t umma_idesc_bf16_ab(int n, int a_mn_major, int b_mn_major)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) a_mn_major << 15) | ((uint32_t) b_mn_major << 16) |
           ((uint32_t) (n >> 3) << 17) | ((uint32_t) (64 >> 4) << 24);
}

// A panel of 64 right-hand sides applied to the stored blocks as two passes over the block
// tasks, each a plain GEMM whose outputs are written once (the one-pass kernel's per-tile
// read-modify-write of the transposed-product slot dominated its memory traffic):
//   pass 0, one unit per 64-row chunk of a task:     C0 = A_chunk V    (over the column tiles)
//   pass 1, one unit per 64-column tile of a task:   C1 = A_tile^T W   (over the task's rows)
// Each 64 x 64 tile of A (FP32) is split into BF16 pieces h + m + l in shared memory
// (rows of 128 B, 128-byte swizzle).  The right-hand sides of a tile (64 rows of the
// input space, row-major with the 64 right-hand sides contiguous) are split the same way
// and used as an MN-major B operand, so they are read with coalesced loads and need no
// transpose.  Six products per 16-deep K step (l.h + h.l + m.m + m.h + h.m + h.h), FP32 in
// TMEM over one tile (64 terms), FP64 across tiles in shared memory; the unit's 64 output
// rows are written once.  The next tile is loaded into registers while the MMAs of the
// current one run.  Bounded waits record a status and stop.
struct WideSmem {
    uint16_t a[3][64 * 64];    // A tile pieces: 64 rows (of A) of 64 BF16, 128-byte swizzle
    uint16_t b[2][3][64 * 64]; // right-hand-side pieces, two stages: 64 rows (k) of 64 BF16, swizzled
    double acc[64][65];        // FP64 sums of the unit's 64 output rows (padded)
    unsigned long long mbar;
    uint32_t tmem;
};

constexpr int wide_smem_bytes() { return (int) sizeof(WideSmem) + 1024; }

// Three BF16 pieces h + m + l of a pair of FP32 values, packed two per 32-bit word (element
// order: the first value in the low half): each piece the round-to-nearest of the
// remainder, the remainders formed in packed FP32x2 arithmetic (exact: h and m are the
// leading bits of the value they are subtracted from).
__device__ __forceinline__ void bf16x3_pair(float x0, float x1, uint32_t& h, uint32_t& m, uint32_t& l)
{
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(h) : "f"(x1), "f"(x0));
    const float2 m1 = make_float2(-1.f, -1.f);
    const float2 r1 = __ffma2_rn(make_float2(__uint_as_float(h << 16), __uint_as_float(h & 0xffff0000u)), m1,
                                 make_float2(x0, x1));
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(m) : "f"(r1.y), "f"(r1.x));
    const float2 r2 = __ffma2_rn(make_float2(__uint_as_float(m << 16), __uint_as_float(m & 0xffff0000u)), m1, r1);
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(l) : "f"(r2.y), "f"(r2.x));
}

constexpr int kWideThreads = 256;

// 16-byte global -> shared copy whose bytes past src_bytes (0 or 16) are zero-filled
__device__ __forceinline__ void cp_async16_zfill(void* dst, const void* src, int src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}

// The 64-wide input space split once per panel into BF16 pieces h + m + l (bf16x3_pair),
// piece p of row r at XS3[(p * rows + r) * 64 + v]: the B operands of the 64-wide block
// passes are then copied tile by tile with no conversion.
__global__ void k_split3(const double* __restrict__ XS, long long row0, long long n, long long rows,
                         uint16_t* __restrict__ XS3)
{
    const long long ng = n * 8;   // granules of 8 right-hand sides
    for (long long g = blockIdx.x * (long long) blockDim.x + threadIdx.x; g < ng; g += (long long) gridDim.x * blockDim.x)
    {
        const long long r = row0 + g / 8;
        const int q = (int) (g % 8);
        const double* x = XS + r * 64 + 8 * q;
        uint32_t h[4], m[4], l[4];
#pragma unroll
        for (int j = 0; j < 4; j++) bf16x3_pair((float) x[2 * j], (float) x[2 * j + 1], h[j], m[j], l[j]);
        uint4* o = reinterpret_cast<uint4*>(XS3 + r * 64 + 8 * q);
        const long long ps = rows * 64 / 8;   // one piece, in uint4
        o[0] = make_uint4(h[0], h[1], h[2], h[3]);
        o[ps] = make_uint4(m[0], m[1], m[2], m[3]);
        o[2 * ps] = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

template <int MODE>
__global__ void __launch_bounds__(kWideThreads, 2) k_blk_wide(const BlkTask* __restrict__ tasks,
                                                              const WideUnit* __restrict__ units, int n_units,
                                                              const float* __restrict__ arena,
                                                              const uint16_t* __restrict__ XS3, long long rows3,
                                                              double* __restrict__ PS, int* __restrict__ status)
{
    constexpr int NV = 64;
    // pass 0: A K-major, B (V rows) MN-major; pass 1: A MN-major (A^T), B (W rows) MN-major
    constexpr uint32_t IDESC = umma_idesc_bf16_ab(NV, MODE == 1 ? 1 : 0, 1);
    constexpr int STAGE_B = 3 * 64 * 64 * 2;      // bytes of one stage of right-hand-side pieces
    extern __shared__ __align__(1024) unsigned char wide_raw[];
    WideSmem& sm = *reinterpret_cast<WideSmem*>(wide_raw + ((1024 - (smem_u32(wide_raw) & 1023)) & 1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(smem_u32(&sm.tmem)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0)
    {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sm.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sm.tmem, mbar = smem_u32(&sm.mbar);
    unsigned char* const a_b = reinterpret_cast<unsigned char*>(sm.a);
    unsigned char* const b_b = reinterpret_cast<unsigned char*>(sm.b);
    const uint32_t a_s = smem_u32(sm.a), b_s = smem_u32(sm.b);
    bool ok = true;
    uint32_t phase = 0;
    // warp w reads TMEM lane quadrant w % 4 (rows 16 (w % 4) + lane, lane < 16) and the 32
    // accumulator columns 32 (w / 4) .. + 31
    const int quad = warp & 3, half = warp >> 2;
    double* const acc = sm.acc[(16 * quad + lane) & 63] + 32 * half;
    constexpr int PA[6] = {2, 0, 1, 1, 0, 0}, PB[6] = {0, 2, 1, 0, 1, 0};

    // persistent: the CTA takes units blockIdx.x, + gridDim.x, ...
    for (int ui = blockIdx.x; ui < n_units && ok; ui += gridDim.x)
    {
        const WideUnit U = units[ui];
        const BlkTask T = tasks[U.task];
        const int ncol = T.ncol, nrow = T.nrow;
        // the unit's fixed 64-row chunk (pass 0) or 64-column tile (pass 1), and the tiles it walks
        const int nt = MODE == 0 ? (ncol + 63) / 64 : (nrow + 63) / 64;
        const float* A0 = arena + T.a32;
        const int lda = T.ld32;
        auto tile_of = [&](int t, int& rc, int& c0) {
            if (MODE == 0) { rc = U.off; c0 = 64 * t; }
            else { rc = 64 * t; c0 = U.off; }
        };
        // the A tile is loaded into registers (thread t: 2 granules, row r, 8 consecutive
        // columns q, as two 16-byte loads: FP32 rows are padded to 16 bytes with zeros, so
        // a vector that starts before the row's end stays in the row) and split into shared
        // memory; the right-hand-side pieces of a tile are copied from XS3 by cp.async into
        // one of two stages (rows past the tile's extent zero-filled)
        float4 ra[2][2];
        auto load_a = [&](int t) {
            int rc, c0;
            tile_of(t, rc, c0);
            const int R = min(64, nrow - rc), C = min(64, ncol - c0);
            const float* A = A0 + (long long) rc * lda + c0;
#pragma unroll
            for (int u = 0; u < 2; u++)
            {
                const int gi = tid + kWideThreads * u, r = gi >> 3, q = gi & 7;
#pragma unroll
                for (int h = 0; h < 2; h++)
                {
                    const int c = 8 * q + 4 * h;
                    ra[u][h] = (r < R && c < C) ? *reinterpret_cast<const float4*>(A + (long long) r * lda + c)
                                                : make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
        };
        auto issue_b = [&](int t, int stage) {
            int rc, c0;
            tile_of(t, rc, c0);
            const int nk = MODE == 0 ? min(64, ncol - c0) : min(64, nrow - rc);
            const long long row0 = MODE == 0 ? (long long) T.in0_row + c0 : (long long) T.in1_row + rc;
#pragma unroll
            for (int u = 0; u < 6; u++)
            {
                const int i = tid + kWideThreads * u, pc = i >> 9, r = (i >> 3) & 63, q = i & 7;
                const uint16_t* src = XS3 + ((long long) pc * rows3 + row0 + (r < nk ? r : 0)) * 64 + 8 * q;
                cp_async16_zfill(b_b + stage * STAGE_B + pc * 8192 + sw128(r, q), src, r < nk ? 16 : 0);
            }
            cp_async_commit();
        };
        auto store_a = [&]() {
#pragma unroll
            for (int u = 0; u < 2; u++)
            {
                const int gi = tid + kWideThreads * u, r = gi >> 3, q = gi & 7;
                uint32_t h[4], m[4], l[4];
                bf16x3_pair(ra[u][0].x, ra[u][0].y, h[0], m[0], l[0]);
                bf16x3_pair(ra[u][0].z, ra[u][0].w, h[1], m[1], l[1]);
                bf16x3_pair(ra[u][1].x, ra[u][1].y, h[2], m[2], l[2]);
                bf16x3_pair(ra[u][1].z, ra[u][1].w, h[3], m[3], l[3]);
                const int off = sw128(r, q);
                *reinterpret_cast<uint4*>(a_b + off) = make_uint4(h[0], h[1], h[2], h[3]);
                *reinterpret_cast<uint4*>(a_b + 8192 + off) = make_uint4(m[0], m[1], m[2], m[3]);
                *reinterpret_cast<uint4*>(a_b + 16384 + off) = make_uint4(l[0], l[1], l[2], l[3]);
            }
        };
        // wait for the tile's MMAs and add its FP32 products into the unit's FP64 sums (the
        // unit's first tile initialises them)
        auto drain = [&](bool first) {
            int good = 1;
            if (tid == 0)
            {
                int it = 0;
                while (!mbar_try_wait(mbar, phase))
                    if (++it > (1 << 22)) { good = 0; break; }
                if (!good) atomicExch(status, 1);
            }
            phase ^= 1;
            ok = __syncthreads_and(good) != 0;
            if (!ok) return;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint32_t d[32];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                         "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                         : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
                           "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
                           "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]),
                           "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
                         : "r"(tmem + ((uint32_t) (32 * quad) << 16) + (uint32_t) (32 * half)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (lane < 16)
            {
                if (first)
#pragma unroll
                    for (int n = 0; n < 32; n++) acc[n] = (double) __uint_as_float(d[n]);
                else
#pragma unroll
                    for (int n = 0; n < 32; n++) acc[n] += (double) __uint_as_float(d[n]);
            }
        };

        issue_b(0, 0);
        load_a(0);
        for (int t = 0; t < nt; t++)
        {
            if (t > 0) drain(t == 1);
            if (!ok) break;
            store_a();
            cp_async_wait_all();                     // this thread's copies of tile t's inputs
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            if (tid == 0)
            {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t bs = b_s + (uint32_t) ((t & 1) * STAGE_B);
#pragma unroll
                for (int ks = 0; ks < 4; ks++)          // K-steps of 16
#pragma unroll
                    for (int p = 0; p < 6; p++)
                    {
                        // pass 0: A K-major (32-byte step along a row); pass 1: A MN-major
                        // (16 rows = two 8-row swizzle atoms per step); B MN-major in both
                        const uint64_t ad = MODE == 0 ? umma_desc(a_s + PA[p] * 8192 + ks * 32, 16, 1024, 2)
                                                      : umma_desc(a_s + PA[p] * 8192 + ks * 2048, 8192, 1024, 2);
                        umma_f16(tmem, ad, umma_desc(bs + PB[p] * 8192 + ks * 2048, 8192, 1024, 2), IDESC,
                                 (ks == 0 && p == 0) ? 0u : 1u);
                    }
                umma_commit(mbar);
            }
            if (t + 1 < nt)
            {
                issue_b(t + 1, (t + 1) & 1);         // that stage's previous tile (t - 1) was waited on
                load_a(t + 1);
            }
        }
        if (ok && nt > 0) drain(nt == 1);
        // the unit's outputs, written once (each thread writes the sums it added)
        if (ok && lane < 16)
        {
            const int m = 16 * quad + lane;
            const int lim = MODE == 0 ? min(64, nrow - U.off) : min(64, ncol - U.off);
            if (m < lim)
            {
                double* o = PS + (long long) ((MODE == 0 ? T.out0_row : T.out1_row) + U.off + m) * NV + 32 * half;
#pragma unroll 8
                for (int n = 0; n < 32; n++) o[n] = acc[n];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
    {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(tmem) : "memory");
    }
}

// ------------------------------------ interpolative decompositions (construction of U)

// The construction step of the projection matrices (H2P_build_H2_UJ_proxy,
// src/H2Pack_build.c:32-270, with H2P_ID_compress / H2P_partial_pivot_QR,
// src/H2Pack_ID_compress.c:51-189 and :491-576), for scalar kernels.  Block b is the
// kernel matrix of a node's candidate points (shifted to its box center) against its
// level's proxy points, A[i][j] = K(c_i, p_j), stored row-major (ncand x npp) -- that
// is, A^T column-major, whose columns (one per candidate) are what the pivoted QR
// ranks.

// A of every block: one CTA per (block, 64 candidate rows)
template <int KID>
__global__ void __launch_bounds__(256) k_id_eval(const IdBlock* __restrict__ blks, const double* __restrict__ cand,
                                                 const double* __restrict__ prox, KParam kp, double* __restrict__ W)
{
    const IdBlock B = blks[blockIdx.y];
    const int r0 = 64 * blockIdx.x;
    if (r0 >= B.ncand) return;
    const int nr = min(64, B.ncand - r0);
    const double* c = cand + B.cand_off;
    const double* q = prox + B.prox_off;
    double* w = W + B.w_off;
    for (long long e = threadIdx.x; e < (long long) nr * B.npp; e += blockDim.x)
    {
        const int i = r0 + (int) (e / B.npp), j = (int) (e % B.npp);
        const double dx = c[i] - q[j], dy = c[B.ncand + i] - q[B.npp + j], dz = c[2 * B.ncand + i] - q[2 * B.npp + j];
        w[(long long) i * B.npp + j] = Scalar<KID, double>::f(dx * dx + dy * dy + dz * dz, kp.p0, kp.c0);
    }
}

// The reduced candidate matrix of proxy-point generation (H2P_generate_proxy_point_nlayer,
// src/H2Pack_gen_proxy_point.c:106-131): W = K(X0, Y0) S with S a sparse random matrix
// given as S^T in CSR (nx rows), W nx x nx row-major; the kernel values are evaluated
// where S has nonzeros, never stored.  One thread per element of W.
template <int KID>
__global__ void __launch_bounds__(256) k_pp_sketch(int nx, const double* __restrict__ X0, int ny,
                                                   const double* __restrict__ Y0, const int* __restrict__ rowptr,
                                                   const int* __restrict__ col, const double* __restrict__ val,
                                                   KParam kp, double* __restrict__ W)
{
    const long long e = blockIdx.x * (long long) blockDim.x + threadIdx.x;
    if (e >= (long long) nx * nx) return;
    const int i = (int) (e / nx), c = (int) (e % nx);
    const double x = X0[i], y = X0[nx + i], z = X0[2 * nx + i];
    double s = 0.0;
    for (int p = rowptr[c]; p < rowptr[c + 1]; p++)
    {
        const int k = col[p];
        const double dx = x - Y0[k], dy = y - Y0[ny + k], dz = z - Y0[2 * ny + k];
        s += val[p] * Scalar<KID, double>::f(dx * dx + dy * dy + dz * dz, kp.p0, kp.c0);
    }
    W[e] = s;
}

constexpr int kIdThreads = 512, kIdWarps = kIdThreads / 32;
static_assert(kIdWarps == kIdQrWarps, "shared-memory layout of k_id_qr");

// block-wide sum (all threads get it); scratch: kIdWarps doubles
__device__ __forceinline__ double id_block_sum(double v, double* scratch)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) scratch[w] = v;
    __syncthreads();
    double s = 0.0;
    for (int k = 0; k < kIdWarps; k++) s += scratch[k];   // fixed order
    return s;
}

// block-wide argmax of val[j] over j in [j0, n): the largest value, the smallest index
// among equal ones (as a first-strictly-greater scan); scratch: kIdWarps (double, int)
__device__ __forceinline__ void id_block_argmax(const double* val, int j0, int n, double* sv, int* si, double& best,
                                                int& arg)
{
    double b = -1.0;
    int a = n;
    for (int j = j0 + (int) threadIdx.x; j < n; j += blockDim.x)
        if (val[j] > b) { b = val[j]; a = j; }
    for (int o = 16; o > 0; o >>= 1)
    {
        const double ob = __shfl_xor_sync(0xffffffffu, b, o);
        const int oa = __shfl_xor_sync(0xffffffffu, a, o);
        if (ob > b || (ob == b && oa < a)) { b = ob; a = oa; }
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) { sv[w] = b; si[w] = a; }
    __syncthreads();
    b = -1.0;
    a = n;
    for (int k = 0; k < kIdWarps; k++)
        if (sv[k] > b || (sv[k] == b && si[k] < a)) { b = sv[k]; a = si[k]; }
    best = b;
    arg = a;
}

// Column-pivoted Householder QR of A^T (m = npp rows, n = ncand columns, column j at
// W + j m) with H2Pack's stopping rule (stop when the largest remaining column norm
// falls below max(sqrt(m) 1e-15, reltol) times the largest initial one, H2P_ID_QR with
// QR_REL_NRM), its column-norm downdates (recomputed when the downdated square falls to
// 1e-10 or below), then E = R11^-1 R12 in place (columns r .. n-1, rows 0 .. r-1).
// One CTA per block; outputs rank and the column permutation.
__global__ void __launch_bounds__(kIdThreads) k_id_qr(const IdBlock* __restrict__ blks, double* __restrict__ W,
                                                      double reltol, int* __restrict__ rank_out,
                                                      int* __restrict__ perm_out, int want_e)
{
    extern __shared__ __align__(16) unsigned char id_raw[];
    const IdBlock B = blks[blockIdx.x];
    const int m = B.npp, n = B.ncand;
    double* const cn = reinterpret_cast<double*>(id_raw);          // n column norms
    double* const v = cn + n;                                       // m: Householder vector
    double* const sv = v + m;                                       // kIdWarps
    int* const perm = reinterpret_cast<int*>(sv + kIdWarps);        // n
    int* const si = perm + n;                                       // kIdWarps
    double* const A = W + B.w_off;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int max_iter = min(m, n);
    for (int j = warp; j < n; j += kIdWarps)
    {
        double s = 0.0;
        for (int k = lane; k < m; k += 32) { const double x = A[(long long) j * m + k]; s += x * x; }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) { cn[j] = sqrt(s); perm[j] = j; }
    }
    __syncthreads();
    double norm_p;
    int pivot;
    id_block_argmax(cn, 0, n, sv, si, norm_p, pivot);
    if (pivot >= n) { norm_p = 0.0; pivot = 0; }
    const double stop_norm = fmax(sqrt((double) m) * 1e-15, reltol) * norm_p;
    int r = max_iter;
    for (int i = 0; i < max_iter; i++)
    {
        // (a zero remaining column ends it too: nothing left to orthogonalise)
        if (norm_p < stop_norm || !(norm_p > 0.0)) { r = i; break; }
        // swap column i with the pivot column
        if (pivot != i)
        {
            double* ci = A + (long long) i * m;
            double* cp = A + (long long) pivot * m;
            for (int k = tid; k < m; k += kIdThreads) { const double t = ci[k]; ci[k] = cp[k]; cp[k] = t; }
            if (tid == 0)
            {
                const int tp = perm[i]; perm[i] = perm[pivot]; perm[pivot] = tp;
                const double tn = cn[i]; cn[i] = cn[pivot]; cn[pivot] = tn;
            }
        }
        __syncthreads();
        // Householder vector of column i, rows i .. m-1
        double* const h = A + (long long) i * m + i;
        const int hl = m - i;
        double s = 0.0;
        for (int k = tid; k < hl; k += kIdThreads) s += h[k] * h[k];
        const double h_norm = sqrt(id_block_sum(s, sv));
        const double x0 = h[0];
        const double sign = x0 > 0.0 ? 1.0 : -1.0;
        const double v0 = x0 + sign * h_norm;
        s = 0.0;
        for (int k = tid; k < hl; k += kIdThreads) { const double x = k == 0 ? v0 : h[k]; s += x * x; }
        const double inv = 1.0 / sqrt(id_block_sum(s, sv));
        for (int k = tid; k < hl; k += kIdThreads) v[k] = (k == 0 ? v0 : h[k]) * inv;
        __syncthreads();
        // trailing columns: one warp per column
        for (int j = i + 1 + warp; j < n; j += kIdWarps)
        {
            double* const c = A + (long long) j * m + i;
            double d = 0.0;
            for (int k = lane; k < hl; k += 32) d += v[k] * c[k];
            for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
            d *= 2.0;
            for (int k = lane; k < hl; k += 32) c[k] -= d * v[k];
            __syncwarp();
            if (cn[j] < stop_norm)
            {
                if (lane == 0) cn[j] = 0.0;
                continue;
            }
            const double c0 = c[0];
            const double t = cn[j] * cn[j] - c0 * c0;
            if (t <= 1e-10)
            {
                double q = 0.0;
                for (int k = 1 + lane; k < hl; k += 32) q += c[k] * c[k];
                for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
                if (lane == 0) cn[j] = sqrt(q);
            } else if (lane == 0) {
                cn[j] = sqrt(t);
            }
        }
        for (int k = tid; k < hl; k += kIdThreads) h[k] = k == 0 ? -sign * h_norm : 0.0;
        __syncthreads();
        id_block_argmax(cn, i + 1, n, sv, si, norm_p, pivot);
        if (pivot >= n) { norm_p = 0.0; pivot = i + 1; }
    }
    // E = R11^-1 R12: one thread per column of R12 (back substitution)
    for (int c = r + tid; want_e && c < n; c += kIdThreads)
    {
        double* const b = A + (long long) c * m;
        for (int k = r - 1; k >= 0; k--)
        {
            double x = b[k];
            for (int l = k + 1; l < r; l++) x -= A[(long long) l * m + k] * b[l];
            b[k] = x / A[(long long) k * m + k];
        }
    }
    if (tid == 0) rank_out[blockIdx.x] = r;
    for (int j = tid; j < n; j += kIdThreads) perm_out[B.perm_off + j] = perm[j];
}

// The same QR for one large matrix (the proxy-point sketch, large nodes of a level with
// few of them), spread over the whole GPU: per iteration i one single-CTA launch picks
// the pivot, swaps it in and forms the Householder vector (k_qrg_pivot), then a grid of
// CTAs updates the trailing columns, one warp per column (k_qrg_update).  Launches past
// the stopping point return at once (the state's done flag).  Same arithmetic, pivot
// order and stopping rule as k_id_qr.
struct QrgState {
    double stop_norm;   // reltol until the first pivot step scales it
    int done, rank;
};

__global__ void __launch_bounds__(kIdThreads) k_qrg_init(const double* __restrict__ A, int m, int n, double reltol,
                                                         double* __restrict__ cn, int* __restrict__ perm,
                                                         QrgState* __restrict__ st)
{
    // column norms: the grid's warps over the columns
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int j = gw; j < n; j += nw)
    {
        double s = 0.0;
        for (int k = lane; k < m; k += 32) { const double x = A[(long long) j * m + k]; s += x * x; }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) { cn[j] = sqrt(s); perm[j] = j; }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) { st->done = 0; st->rank = min(m, n); st->stop_norm = reltol; }
}

// one CTA: stop test, pivot swap, Householder vector v (m - i entries) and the finished
// column i; step 0 also scales the stopping norm by the largest initial column norm
__global__ void __launch_bounds__(kIdThreads) k_qrg_pivot(double* __restrict__ A, int m, int n, int i,
                                                          double* __restrict__ cn, int* __restrict__ perm,
                                                          double* __restrict__ v, QrgState* __restrict__ st)
{
    __shared__ double sv[kIdWarps];
    __shared__ int si[kIdWarps];
    if (st->done) return;
    const int tid = threadIdx.x;
    double norm_p;
    int pivot;
    id_block_argmax(cn, i, n, sv, si, norm_p, pivot);   // (holds barriers: every thread has read st)
    if (pivot >= n) { norm_p = 0.0; pivot = i; }
    double stop_norm = st->stop_norm;
    if (i == 0) stop_norm = fmax(sqrt((double) m) * 1e-15, stop_norm) * norm_p;
    __syncthreads();
    if (tid == 0 && i == 0) st->stop_norm = stop_norm;
    if (norm_p < stop_norm || !(norm_p > 0.0))
    {
        if (tid == 0) { st->done = 1; st->rank = i; }
        return;
    }
    if (pivot != i)
    {
        double* ci = A + (long long) i * m;
        double* cp = A + (long long) pivot * m;
        for (int k = tid; k < m; k += kIdThreads) { const double t = ci[k]; ci[k] = cp[k]; cp[k] = t; }
        if (tid == 0)
        {
            const int tp = perm[i]; perm[i] = perm[pivot]; perm[pivot] = tp;
            const double tn = cn[i]; cn[i] = cn[pivot]; cn[pivot] = tn;
        }
    }
    __syncthreads();
    double* const h = A + (long long) i * m + i;
    const int hl = m - i;
    double s = 0.0;
    for (int k = tid; k < hl; k += kIdThreads) s += h[k] * h[k];
    const double h_norm = sqrt(id_block_sum(s, sv));
    const double x0 = h[0];
    const double sign = x0 > 0.0 ? 1.0 : -1.0;
    const double v0 = x0 + sign * h_norm;
    s = 0.0;
    for (int k = tid; k < hl; k += kIdThreads) { const double x = k == 0 ? v0 : h[k]; s += x * x; }
    const double inv = 1.0 / sqrt(id_block_sum(s, sv));
    for (int k = tid; k < hl; k += kIdThreads) v[k] = (k == 0 ? v0 : h[k]) * inv;
    __syncthreads();
    for (int k = tid; k < hl; k += kIdThreads) h[k] = k == 0 ? -sign * h_norm : 0.0;
}

// trailing columns j = i + 1 .. n - 1, one warp per column across the grid
__global__ void __launch_bounds__(256) k_qrg_update(double* __restrict__ A, int m, int n, int i,
                                                    double* __restrict__ cn, const double* __restrict__ v,
                                                    const QrgState* __restrict__ st)
{
    if (st->done) return;
    const double stop_norm = st->stop_norm;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int hl = m - i;
    for (int j = i + 1 + gw; j < n; j += nw)
    {
        double* const c = A + (long long) j * m + i;
        double d = 0.0;
        for (int k = lane; k < hl; k += 32) d += v[k] * c[k];
        for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        d *= 2.0;
        for (int k = lane; k < hl; k += 32) c[k] -= d * v[k];
        __syncwarp();
        if (cn[j] < stop_norm)
        {
            if (lane == 0) cn[j] = 0.0;
            continue;
        }
        const double c0 = c[0];
        const double t = cn[j] * cn[j] - c0 * c0;
        if (t <= 1e-10)
        {
            double q = 0.0;
            for (int k = 1 + lane; k < hl; k += 32) q += c[k] * c[k];
            for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
            if (lane == 0) cn[j] = sqrt(q);
        } else if (lane == 0) {
            cn[j] = sqrt(t);
        }
    }
}

// the rank out, then (want_e) E = R11^-1 R12 in place, one thread per column of R12
__global__ void __launch_bounds__(256) k_qrg_trsm(double* __restrict__ A, int m, int n,
                                                  const QrgState* __restrict__ st, int want_e, int* __restrict__ rank_out)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) rank_out[0] = st->rank;
    if (!want_e) return;
    const int r = st->rank;
    for (int c = r + blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        double* const b = A + (long long) c * m;
        for (int k = r - 1; k >= 0; k--)
        {
            double x = b[k];
            for (int l = k + 1; l < r; l++) x -= A[(long long) l * m + k] * b[l];
            b[k] = x / A[(long long) k * m + k];
        }
    }
}

// ---------------------------------------------- sweeps on the tensor cores (FP32 U)

// Upward / downward sweep products for FP32 U and panels of 8 / 16 right-hand sides on
// the tensor cores (3xTF32, FP32 accumulation per 32-deep k tile, FP64 across tiles),
// right-hand sides as the M = 16 side of m16n8k8:
//   upward   (UP):  C^T (NV x nc) = X^T (NV x nrow) U[:, c0 : c0 + nc]    B = U,   k = rows of U
//   downward (!UP): C^T (NV x 64) = Y^T (NV x ncol) U[r0 : r0 + 64, :]^T  B = U^T, k = columns of U
// (Y = the node's summed y1 plus the parent's push-down slice).  Warp w owns output
// columns (UP) / rows (DOWN) 8w..8w+7.  The 32-deep k tiles of U come through a
// three-stage shared-memory ring filled by 16-byte cp.async (two tiles in flight
// without registers); the X^T / Y^T fragments are split by warps 0-3 one tile ahead
// and double-buffered in shared memory.
// STRIDE: row stride of the vector spaces.  A 64-wide panel (STRIDE = 64) runs as four
// 16-column sub-panels, blockIdx.y = sub-panel (columns 16 blockIdx.y .. + 15).
template <int NV, bool UP, int STRIDE = NV>
__global__ void __launch_bounds__(256, 4) k_sweep_tc(const UpTask* __restrict__ ups, const DownTask* __restrict__ dns,
                                                     const float* __restrict__ Uar, double* __restrict__ XS,
                                                     const double* __restrict__ Y1, double* __restrict__ PS,
                                                     double* __restrict__ PUSH)
{
    static_assert(STRIDE == NV || NV == 16, "sub-panels are 16 columns wide");
    const int v0 = STRIDE == NV ? 0 : 16 * (int) blockIdx.y;
    constexpr int KT = 32, NS = 3;                          // tile depth, U ring stages
    constexpr int ROWS = UP ? KT : 64, LD = UP ? 72 : 36;   // padded: conflict-free fragment reads
    __shared__ __align__(16) float s_u[NS][ROWS][LD];
    __shared__ uint4 s_x[2][4][32][2];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3;
    int K, M, lda, xrow = 0, y1_row = -1, push_row = -1;
    const float* A;
    double* out;
    if constexpr (UP)
    {
        const UpTask T = ups[blockIdx.x];
        K = T.nrow; M = T.nc; lda = T.ld;
        A = Uar + T.u_off + T.c0;
        xrow = T.in_row;
        out = XS + (long long) (T.out_row + T.c0) * STRIDE + v0;
    } else {
        const DownTask T = dns[blockIdx.x];
        K = T.ncol; M = T.nrow; lda = T.ld;
        A = Uar + T.u_off;
        y1_row = T.y1_row; push_row = T.push_row;
        out = (T.dst_ps ? PS : PUSH) + (long long) T.dst_row * STRIDE + v0;
    }
    auto xin = [&](int k, int v) -> double {
        if constexpr (UP) return XS[(long long) (xrow + k) * STRIDE + v0 + v];
        double b = (y1_row >= 0) ? Y1[(long long) (y1_row + k) * STRIDE + v0 + v] : 0.0;
        if (push_row >= 0) b += PUSH[(long long) (push_row + k) * STRIDE + v0 + v];
        return b;
    };
    const int nt = (K + KT - 1) / KT;
    // U tiles: a ring of NS stages filled by 16-byte cp.async (U rows are padded to a
    // multiple of 4 elements with zeros and start on 16-byte boundaries, so a vector that
    // starts inside a row stays in it; vectors past the tile's extent are zero-filled), so
    // NS - 1 tiles are in flight without registers.  One commit group per tile (empty
    // past the end), so that wait_group(NS - 2) means "tile t has landed".
    auto issue_u = [&](int t) {
        if (t < nt)
        {
            const int k0 = t * KT;
            float* st = &s_u[t % NS][0][0];
#pragma unroll
            for (int u = 0; u < 2; u++)
            {
                const int e = threadIdx.x + 256 * u;
                int r, c;
                bool in;
                if constexpr (UP) { r = e >> 4; c = (e & 15) * 4; in = k0 + r < K && c < M; }
                else { r = e >> 3; c = (e & 7) * 4; in = r < M && k0 + c < K; }
                const float* src = !in ? A : (UP ? A + (long long) (k0 + r) * lda + c : A + (long long) r * lda + k0 + c);
                cp_async16_zfill(st + r * LD + c, src, in ? 16 : 0);
            }
        }
        cp_async_commit();
    };
    // input fragments of a tile (warps 0-3, one k-step each), split into TF32 hi / lo
    uint4 rxh = make_uint4(0, 0, 0, 0), rxl = rxh;
    auto load_x = [&](int t) {
        if (warp < 4)
        {
            const int k0 = t * KT;
            const int ka = k0 + 8 * warp + tq, kb = ka + 4;
            float v[4];
            v[0] = (ka < K && g < NV) ? (float) xin(ka, g) : 0.f;
            v[1] = (ka < K && g + 8 < NV) ? (float) xin(ka, g + 8) : 0.f;
            v[2] = (kb < K && g < NV) ? (float) xin(kb, g) : 0.f;
            v[3] = (kb < K && g + 8 < NV) ? (float) xin(kb, g + 8) : 0.f;
            uint32_t h[4], l[4];
#pragma unroll
            for (int q = 0; q < 4; q++)
            {
                h[q] = tf32_rna(v[q]);
                l[q] = __float_as_uint(v[q] - __uint_as_float(h[q]));
            }
            rxh = make_uint4(h[0], h[1], h[2], h[3]);
            rxl = make_uint4(l[0], l[1], l[2], l[3]);
        }
    };
    auto store_x = [&](int buf) {
        if (warp < 4) { s_x[buf][warp][lane][0] = rxh; s_x[buf][warp][lane][1] = rxl; }
    };

    double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int t = 0; t < NS - 1; t++) issue_u(t);
    if (nt > 0)
    {
        load_x(0);
        store_x(0);
    }
    for (int t = 0; t < nt; t++)
    {
        cp_async_wait_group<NS - 2>();     // this thread's copies of tile t have landed
        __syncthreads();                   // everyone's; tile t - 1 (its stage, its x buffer) is no longer read
        issue_u(t + NS - 1);               // into the stage tile t - 1 used
        const bool more = t + 1 < nt;
        if (more) load_x(t + 1);
        const int st = t % NS, buf = t & 1;
        if (8 * warp < M)
        {
            float d[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
            for (int ks = 0; ks < 4; ks++)
            {
                const uint4 xh = s_x[buf][ks][lane][0], xl = s_x[buf][ks][lane][1];
                float b0, b1;
                if constexpr (UP)
                {
                    b0 = s_u[st][8 * ks + tq][8 * warp + g];
                    b1 = s_u[st][8 * ks + tq + 4][8 * warp + g];
                } else {
                    b0 = s_u[st][8 * warp + g][8 * ks + tq];
                    b1 = s_u[st][8 * warp + g][8 * ks + tq + 4];
                }
                const uint32_t h0 = tf32_rna(b0), h1 = tf32_rna(b1);
                const uint32_t l0 = __float_as_uint(b0 - __uint_as_float(h0)), l1 = __float_as_uint(b1 - __uint_as_float(h1));
                float (&dd)[4] = d[ks & 1];
                mma_tf32(dd, xl.x, xl.y, xl.z, xl.w, h0, h1);
                mma_tf32(dd, xh.x, xh.y, xh.z, xh.w, l0, l1);
                mma_tf32(dd, xh.x, xh.y, xh.z, xh.w, h0, h1);
            }
#pragma unroll
            for (int q = 0; q < 4; q++) acc[q] += (double) (d[0][q] + d[1][q]);
        }
        if (more) store_x(buf ^ 1);        // read by tile t + 1 after the next barrier
    }
    cp_async_wait_all();
    // rows of the fragment = right-hand sides (g, g+8), columns = outputs (2tq, 2tq+1)
#pragma unroll
    for (int q = 0; q < 4; q++)
    {
        const int rhs = (q < 2) ? g : g + 8, m = 8 * warp + 2 * tq + (q & 1);
        if (rhs < NV && m < M) out[(long long) m * STRIDE + rhs] = acc[q];
    }
}

// --------------------------------------------------------------- direct sum

template <int KID, int KD>
__global__ void __launch_bounds__(128) k_direct(const double4* __restrict__ trg, int n_trg,
                                                const double4* __restrict__ src, int n_src,
                                                const double* __restrict__ val, KParam kp, double* __restrict__ out)
{
    constexpr int TILE = 128;
    __shared__ double4 s_pt[TILE];
    __shared__ double s_v[TILE * KD];
    const int i = blockIdx.x * 128 + threadIdx.x;
    const double4 xi = trg[i < n_trg ? i : 0];
    double acc[KD];
#pragma unroll
    for (int a = 0; a < KD; a++) acc[a] = 0.0;
    for (int j0 = 0; j0 < n_src; j0 += TILE)
    {
        const int nj = min(TILE, n_src - j0);
        __syncthreads();
        for (int j = threadIdx.x; j < nj; j += 128) s_pt[j] = src[j0 + j];
        for (int j = threadIdx.x; j < nj * KD; j += 128) s_v[j] = val[(long long) j0 * KD + j];
        __syncthreads();
        for (int j = 0; j < nj; j++)
        {
            double dx = xi.x - s_pt[j].x, dy = xi.y - s_pt[j].y, dz = xi.z - s_pt[j].z;
            if constexpr (KD == 1)
            {
                double r2 = dx * dx + dy * dy + dz * dz;
                acc[0] = fma(Scalar<KID, double>::f(r2, kp.p0, kp.c0), s_v[j], acc[0]);
            } else {
                double t1, t2, ux, uy, uz;
                rpy_coef<double>(dx, dy, dz, xi.w, s_pt[j].w, kp.c0, t1, t2, ux, uy, uz);
                double bx = s_v[3 * j], by = s_v[3 * j + 1], bz = s_v[3 * j + 2];
                double dot = t2 * (ux * bx + uy * by + uz * bz);
                acc[0] += dot * ux + t1 * bx;
                acc[1] += dot * uy + t1 * by;
                acc[2] += dot * uz + t1 * bz;
            }
        }
    }
    if (i < n_trg)
#pragma unroll
        for (int a = 0; a < KD; a++) out[(long long) i * KD + a] = acc[a];
}

// ------------------------------------------------- stored-block generation

// One CTA per GenTask: up to 16 row points of one B / D block against all its column
// points, in FP64 from the same formulas as the JIT and direct-sum kernels (the values
// of H2Pack's krnl_eval on the same points, src/H2Pack_build.c:818-860, :1063-1110), then
// stored in the arena's type.  Column points are staged in shared memory 256 at a time;
// thread j owns column point j of the stage and writes its kd x kd entries of every row
// point (consecutive threads write consecutive kd-wide runs of a row).
constexpr int kGenThreads = 256;

template <int KID, int KD, typename TO>
__global__ void __launch_bounds__(kGenThreads) k_gen(const GenTask* __restrict__ tasks,
                                                     const double4* __restrict__ pts, KParam kp,
                                                     TO* __restrict__ arena)
{
    __shared__ double4 s_row[16];
    const GenTask t = tasks[blockIdx.x];
    const int tid = threadIdx.x;
    // FP64: H2Pack's packing; FP32: rows padded to 16 bytes (the padding is zeroed by the host)
    const long long ld = sizeof(TO) == 4 ? (long long) f32_ld(KD * t.ncp) : (long long) KD * t.ncp;
    const long long a0 = sizeof(TO) == 4 ? t.a32 : t.a_off;
    if (tid < t.nrp) s_row[tid] = pts[t.row_pt0 + tid];
    __syncthreads();
    for (int j0 = 0; j0 < t.ncp; j0 += kGenThreads)
    {
        const int j = j0 + tid;
        if (j >= t.ncp) break;
        const double4 q = pts[t.col_pt0 + j];
        TO* col = arena + a0 + (long long) KD * j;
        for (int i = 0; i < t.nrp; i++)
        {
            const double4 p = s_row[i];
            const double dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
            if constexpr (KD == 1)
            {
                const double r2 = dx * dx + dy * dy + dz * dz;
                col[(long long) i * ld] = (TO) Scalar<KID, double>::f(r2, kp.p0, kp.c0);
            } else {
                double t1, t2, ux, uy, uz;
                rpy_coef<double>(dx, dy, dz, p.w, q.w, kp.c0, t1, t2, ux, uy, uz);
                const double u[3] = {ux, uy, uz};
                TO* row = col + (long long) (3 * i) * ld;
#pragma unroll
                for (int a = 0; a < 3; a++)
                {
                    const double ta = t2 * u[a];
#pragma unroll
                    for (int b = 0; b < 3; b++) row[(long long) a * ld + b] = (TO) (ta * u[b] + (a == b ? t1 : 0.0));
                }
            }
        }
    }
}

// ------------------------------------------------ measured pipe peaks (roofline)

// FP32 FMA pipe: 8 independent packed FP32x2 FMA chains per thread (16 FMAs per
// iteration step, 32 flop), so the pipe, not a dependency, bounds the rate.
__global__ void __launch_bounds__(256) k_peak_ffma2(int iters, float seed, float* __restrict__ out)
{
    float2 a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = make_float2(seed + k + threadIdx.x, seed - k);
    const float2 m = make_float2(0.999999f, 1.000001f), c = make_float2(1e-7f, -1e-7f);
    // unrolled by 16 so that the loop's own instructions are < 1 % of the issued ones
#pragma unroll 16
    for (int i = 0; i < iters; i++)
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = __ffma2_rn(a[k], m, c);
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k].x + a[k].y;
    if (s == 1234.5f) out[blockIdx.x] = s;   // keeps the chains live
}

// MUFU pipe: 8 independent ex2.approx chains per thread (the FP32 path's exponential).
__global__ void __launch_bounds__(256) k_peak_mufu(int iters, float seed, float* __restrict__ out)
{
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = -1e-3f * (seed + k + (threadIdx.x & 7));
#pragma unroll 16
    for (int i = 0; i < iters; i++)
#pragma unroll
        for (int k = 0; k < 8; k++) a[k] = -ex2_approx(a[k]);
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == 1234.5f) out[blockIdx.x] = s;
}

cudaError_t launch_peak(int which, int blocks, int iters, float* out, cudaStream_t st)
{
    if (which == 0) k_peak_ffma2<<<blocks, 256, 0, st>>>(iters, 1.0f, out);
    else k_peak_mufu<<<blocks, 256, 0, st>>>(iters, 1.0f, out);
    return cudaGetLastError();
}

// ------------------------------------------------------------- launchers

static inline unsigned grid_for(long long n, int threads)
{
    long long g = (n + threads - 1) / threads;
    if (g > 148LL * 64) g = 148LL * 64;
    return (unsigned) (g < 1 ? 1 : g);
}

#define NV_DISPATCH(nv, ...)                                  \
    switch (nv) {                                             \
        case 1:  { constexpr int NVc = 1;  __VA_ARGS__; } break; \
        case 2:  { constexpr int NVc = 2;  __VA_ARGS__; } break; \
        case 4:  { constexpr int NVc = 4;  __VA_ARGS__; } break; \
        case 8:  { constexpr int NVc = 8;  __VA_ARGS__; } break; \
        case 16: { constexpr int NVc = 16; __VA_ARGS__; } break; \
        default: return cudaErrorInvalidValue;                \
    }

// The same with the wide panels of the mixed stored-block path (gather, sweeps, sums).
#define NV_DISPATCH_WIDE(nv, ...)                             \
    switch (nv) {                                             \
        case 1:  { constexpr int NVc = 1;  __VA_ARGS__; } break; \
        case 2:  { constexpr int NVc = 2;  __VA_ARGS__; } break; \
        case 4:  { constexpr int NVc = 4;  __VA_ARGS__; } break; \
        case 8:  { constexpr int NVc = 8;  __VA_ARGS__; } break; \
        case 16: { constexpr int NVc = 16; __VA_ARGS__; } break; \
        case 32: { constexpr int NVc = 32; __VA_ARGS__; } break; \
        case 64: { constexpr int NVc = 64; __VA_ARGS__; } break; \
        default: return cudaErrorInvalidValue;                \
    }

cudaError_t launch_gather(int NV, const double* X, long long x_rs, long long x_cs, int nv, const int* fwd, int N,
                          double* XS, cudaStream_t st)
{
    NV_DISPATCH_WIDE(NV, k_gather<NVc><<<grid_for((long long) N * NVc, 256), 256, 0, st>>>(X, x_rs, x_cs, nv, fwd, N, XS));
    return cudaGetLastError();
}

cudaError_t launch_permute(const double* X, long long x_rs, long long x_cs, const int* idx, int n, int nv, double* Y,
                           long long y_rs, long long y_cs, cudaStream_t st)
{
    k_permute<<<grid_for((long long) n * nv, 256), 256, 0, st>>>(X, x_rs, x_cs, idx, n, nv, Y, y_rs, y_cs);
    return cudaGetLastError();
}

template <typename TA>
cudaError_t launch_up(int NV, const UpTask* t, int n, const TA* U, double* XS, cudaStream_t st, int use_tc)
{
    if (n <= 0) return cudaSuccess;
    if constexpr (sizeof(TA) == 4)
    {
        if (use_tc && NV == 64)
        {
            k_sweep_tc<16, true, 64><<<dim3(n, 4), 256, 0, st>>>(t, nullptr, U, XS, nullptr, nullptr, nullptr);
            return cudaGetLastError();
        }
        if (use_tc && (NV == 8 || NV == 16))
        {
            if (NV == 16) k_sweep_tc<16, true><<<n, 256, 0, st>>>(t, nullptr, U, XS, nullptr, nullptr, nullptr);
            else k_sweep_tc<8, true><<<n, 256, 0, st>>>(t, nullptr, U, XS, nullptr, nullptr, nullptr);
            return cudaGetLastError();
        }
    }
    NV_DISPATCH_WIDE(NV, {
        if constexpr (NVc >= 4)
            k_sweep_gemm<TA, NVc, true><<<n, 256, 0, st>>>(t, nullptr, U, XS, nullptr, nullptr, nullptr);
        else
            k_up<TA, NVc><<<n, kThreads, 0, st>>>(t, U, XS);
    });
    return cudaGetLastError();
}

template <typename K>
static cudaError_t allow_smem(K kern, int bytes)
{
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

template <typename TA>
cudaError_t launch_blk(int NV, const BlkTask* t, int n, const TA* arena, const double* XS, double* PS, cudaStream_t st,
                       int use_tc, int* status, int n_small)
{
    if constexpr (sizeof(TA) == 4)
    {
        if (n > 0 && (NV == 32 || NV == 64))
        {
            // wide panels: tcgen05 kernel only (BF16x3 pieces, TMEM accumulators)
            if (!status) return cudaErrorInvalidValue;
            if (NV == 64)
            {
                constexpr int b = bf3w_smem_bytes<64>();
                cudaError_t e = allow_smem(k_blk_bf3w<64>, b);
                if (e != cudaSuccess) return e;
                k_blk_bf3w<64><<<n, kBf3Threads, b, st>>>(t, arena, XS, PS, status);
            } else {
                constexpr int b = bf3w_smem_bytes<32>();
                cudaError_t e = allow_smem(k_blk_bf3w<32>, b);
                if (e != cudaSuccess) return e;
                k_blk_bf3w<32><<<n, kBf3Threads, b, st>>>(t, arena, XS, PS, status);
            }
            return cudaGetLastError();
        }
        if (use_tc && n > 0 && (NV == 8 || NV == 16))
        {
            if (use_tc == 2 && status)
            {
                // tcgen05 kernel (BF16x3 pieces, TMEM accumulators)
                if (NV == 16)
                {
                    constexpr int b = bf3_smem_bytes<16>();
                    cudaError_t e = allow_smem(k_blk_bf3<16>, b);
                    if (e != cudaSuccess) return e;
                    k_blk_bf3<16><<<n, kBf3Threads, b, st>>>(t, arena, XS, PS, status);
                } else {
                    constexpr int b = bf3_smem_bytes<8>();
                    cudaError_t e = allow_smem(k_blk_bf3<8>, b);
                    if (e != cudaSuccess) return e;
                    k_blk_bf3<8><<<n, kBf3Threads, b, st>>>(t, arena, XS, PS, status);
                }
                return cudaGetLastError();
            }
            // the dynamic shared-memory opt-in is a per-device function attribute (cheap,
            // and legal inside a stream capture), so it is set at every launch
            constexpr int b = blk_tc_smem_bytes<16>();
            auto kern = NV == 16 ? k_blk_tc<16> : k_blk_tc<8>;
            cudaError_t e = allow_smem(kern, b);
            if (e != cudaSuccess) return e;
            kern<<<n, 256, b, st>>>(t, arena, XS, PS);
            return cudaGetLastError();
        }
    }
    if (n <= 0) return cudaSuccess;
    NV_DISPATCH(NV, {
        if constexpr (NVc >= 4)
        {
            k_blk_gemm<TA, NVc><<<n, 256, 0, st>>>(t, arena, XS, PS);
        } else if constexpr (NVc == 1) {
            const int ns = n_small < 0 ? 0 : (n_small > n ? n : n_small);
            k_blk1<TA><<<(ns + kWarps - 1) / kWarps + (n - ns), 256, 0, st>>>(t, n, ns, arena, XS, PS);
        } else {
            constexpr int b = chunk_smem_bytes<NVc>();
            cudaError_t e = allow_smem(k_blk<TA, NVc>, b);
            if (e != cudaSuccess) return e;
            k_blk<TA, NVc><<<n, kThreads, b, st>>>(t, arena, XS, PS);
        }
    });
    return cudaGetLastError();
}

cudaError_t launch_split3(const double* XS, long long row0, long long n, long long rows, uint16_t* XS3,
                          cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    k_split3<<<grid_for(n * 8, 256), 256, 0, st>>>(XS, row0, n, rows, XS3);
    return cudaGetLastError();
}

cudaError_t launch_blk_wide(int mode, const BlkTask* t, const WideUnit* u, int n, const float* arena,
                            const uint16_t* XS3, long long rows3, double* PS, cudaStream_t st, int* status)
{
    if (n <= 0) return cudaSuccess;
    if (!status) return cudaErrorInvalidValue;
    constexpr int b = wide_smem_bytes();
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int g = n < 2 * sms ? n : 2 * sms;   // persistent: two CTAs per SM walk the units
    if (mode == 0)
    {
        cudaError_t e = allow_smem(k_blk_wide<0>, b);
        if (e != cudaSuccess) return e;
        k_blk_wide<0><<<g, kWideThreads, b, st>>>(t, u, n, arena, XS3, rows3, PS, status);
    } else {
        cudaError_t e = allow_smem(k_blk_wide<1>, b);
        if (e != cudaSuccess) return e;
        k_blk_wide<1><<<g, kWideThreads, b, st>>>(t, u, n, arena, XS3, rows3, PS, status);
    }
    return cudaGetLastError();
}

template <typename TA>
cudaError_t launch_down(int NV, const DownTask* t, int n, const TA* U, const double* Y1, double* PS, double* PUSH,
                        cudaStream_t st, int use_tc)
{
    if (n <= 0) return cudaSuccess;
    if constexpr (sizeof(TA) == 4)
    {
        if (use_tc && NV == 64)
        {
            k_sweep_tc<16, false, 64><<<dim3(n, 4), 256, 0, st>>>(nullptr, t, U, nullptr, Y1, PS, PUSH);
            return cudaGetLastError();
        }
        if (use_tc && (NV == 8 || NV == 16))
        {
            if (NV == 16) k_sweep_tc<16, false><<<n, 256, 0, st>>>(nullptr, t, U, nullptr, Y1, PS, PUSH);
            else k_sweep_tc<8, false><<<n, 256, 0, st>>>(nullptr, t, U, nullptr, Y1, PS, PUSH);
            return cudaGetLastError();
        }
    }
    NV_DISPATCH_WIDE(NV, {
        if constexpr (NVc >= 4)
        {
            k_sweep_gemm<TA, NVc, false><<<n, 256, 0, st>>>(nullptr, t, U, nullptr, Y1, PS, PUSH);
        } else {
            k_down<TA, NVc><<<n, kThreads, 0, st>>>(t, U, Y1, PS, PUSH);
        }
    });
    return cudaGetLastError();
}

cudaError_t launch_y1sum(int NV, const Y1Task* t, int n, const int* slots, const double* PS, double* Y1, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    NV_DISPATCH_WIDE(NV, k_y1sum<NVc><<<n, 256, 0, st>>>(t, slots, PS, Y1));
    return cudaGetLastError();
}

cudaError_t launch_asm(int NV, const AsmTask* t, int n, const int* slots, const double* PS, const int* fwd,
                       double* Y, long long y_rs, long long y_cs, int nv, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    NV_DISPATCH_WIDE(NV, k_asm<NVc><<<n, 256, 0, st>>>(t, slots, PS, fwd, Y, y_rs, y_cs, nv));
    return cudaGetLastError();
}

template <int KID, typename T, int KD>
static cudaError_t launch_jit_k(int NV, const JitTarget* tg, int n, const JitSource* sr, const void* pts, KParam kp,
                                int use_shift, int use_tc, const double* XS, double* PS, double* Y1, cudaStream_t st,
                                int far, const float4* ppts, const uint4* pin, const TileRec* tiles,
                                const float4* lo, const float4* plo)
{
    using T4 = typename Vec4<T>::t;
    const T4* p = (const T4*) pts;
    // the FP32 Coulomb near field reads the low parts of the points
    if (KID == KRNL_COULOMB_ID && sizeof(T) == 4 && !far && !lo) return cudaErrorInvalidValue;
    // FP32 scalar kernels on panels of 8 or 16: right-hand-side products on the tensor
    // cores unless the image chose the CUDA-core kernel (autotuner, H2G_JIT_TC=0)
    if constexpr (KD == 1 && sizeof(T) == 4)
    {
        if (use_tc && (NV == 16 || NV == 8) && use_shift)
        {
            // the tensor-core kernel reads the source panels and tile lists
            if (!ppts || !pin || !tiles) return cudaErrorInvalidValue;
            if (KID == KRNL_COULOMB_ID && !far && !plo) return cudaErrorInvalidValue;
            const float4* p4 = (const float4*) pts;
            const int b = jit_tc_smem_bytes(KID == KRNL_COULOMB_ID && !far);
            // the dynamic shared-memory opt-in is a per-device function attribute (cheap,
            // and legal inside a stream capture), so it is set at every launch
            auto kern = NV == 16 ? (far ? k_jit_tc<KID, 16, true> : k_jit_tc<KID, 16, false>)
                                 : (far ? k_jit_tc<KID, 8, true> : k_jit_tc<KID, 8, false>);
            cudaError_t e = allow_smem(kern, b);
            if (e != cudaSuccess) return e;
            kern<<<n, 256, b, st>>>(tg, tiles, p4, ppts, pin, kp, PS, Y1, lo, plo);
            return cudaGetLastError();
        }
    }
    // FP32: two targets per thread (64 threads per 128-point chunk) where the accumulators
    // allow it; FP64: one target per thread, 4 CTAs per SM (two targets per thread took
    // 188 registers and left 7 warps per SM to hide the FP64 latencies: 1.4x slower)
    NV_DISPATCH(NV, {
        if constexpr (KD == 3 && NVc > 8)
            return cudaErrorInvalidValue;   // tensor kernels run in panels of <= 8 right-hand sides
        else if constexpr (KD == 1 && sizeof(T) == 4)
        {
            // scalar FP32 kernels: the two targets of a thread as one FP32x2 pair
            if (!use_shift) return cudaErrorInvalidValue;   // FP32 evaluation is re-centred
            if (far) k_jit2<KID, NVc, true><<<n, 64, 0, st>>>(tg, sr, (const float4*) pts, kp, XS, PS, Y1, lo);
            else k_jit2<KID, NVc, false><<<n, 64, 0, st>>>(tg, sr, (const float4*) pts, kp, XS, PS, Y1, lo);
        }
        else if constexpr (KD * NVc <= 16 && sizeof(T) == 4)
            k_jit<KID, T, NVc, KD, 2><<<n, 64, 0, st>>>(tg, sr, p, kp, use_shift, XS, PS, Y1);
        else
            k_jit<KID, T, NVc, KD, 1><<<n, 128, 0, st>>>(tg, sr, p, kp, use_shift, XS, PS, Y1);
    });
    return cudaGetLastError();
}

cudaError_t launch_jit(int kid, int fp32, int NV, const JitTarget* tg, int n, const JitSource* sr, const void* pts,
                       KParam kp, int use_shift, int use_tc, const double* XS, double* PS, double* Y1, cudaStream_t st,
                       int far, const float4* ppts, const uint4* pin, const TileRec* tiles, const float4* lo,
                       const float4* plo)
{
    if (n <= 0) return cudaSuccess;
#define H2G_JIT_ARGS NV, tg, n, sr, pts, kp, use_shift, use_tc, XS, PS, Y1, st, far, ppts, pin, tiles, lo, plo
    switch (kid)
    {
        case KRNL_COULOMB_ID:  return fp32 ? launch_jit_k<KRNL_COULOMB_ID, float, 1>(H2G_JIT_ARGS)
                                           : launch_jit_k<KRNL_COULOMB_ID, double, 1>(H2G_JIT_ARGS);
        case KRNL_GAUSSIAN_ID: return fp32 ? launch_jit_k<KRNL_GAUSSIAN_ID, float, 1>(H2G_JIT_ARGS)
                                           : launch_jit_k<KRNL_GAUSSIAN_ID, double, 1>(H2G_JIT_ARGS);
        case KRNL_MATERN32_ID: return fp32 ? launch_jit_k<KRNL_MATERN32_ID, float, 1>(H2G_JIT_ARGS)
                                           : launch_jit_k<KRNL_MATERN32_ID, double, 1>(H2G_JIT_ARGS);
        case KRNL_RPY_ID:      return fp32 ? launch_jit_k<KRNL_RPY_ID, float, 3>(H2G_JIT_ARGS)
                                           : launch_jit_k<KRNL_RPY_ID, double, 3>(H2G_JIT_ARGS);
        default: return cudaErrorInvalidValue;
    }
#undef H2G_JIT_ARGS
}

cudaError_t launch_panel_pts(const PanelGroup* pg, int n, const float4* pts, float sigma, float4* ppts, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    const long long t = 8LL * n;
    k_panel_pts<<<(unsigned) ((t + 255) / 256), 256, 0, st>>>(pg, n, pts, sigma, ppts);
    return cudaGetLastError();
}

cudaError_t launch_panel_lo(const PanelGroup* pg, int n, const float4* lo, float4* out, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    const long long t = 8LL * n;
    k_panel_lo<<<(unsigned) ((t + 255) / 256), 256, 0, st>>>(pg, n, lo, out);
    return cudaGetLastError();
}

cudaError_t launch_panel_in(int NV, const PanelGroup* pg, int g0, int n, const double* XS, uint4* pin, cudaStream_t st)
{
    if (n <= 0 || !pin || (NV != 8 && NV != 16)) return cudaSuccess;
    const long long t = 32LL * n;
    if (NV == 16) k_panel_in<16><<<(unsigned) ((t + 255) / 256), 256, 0, st>>>(pg, g0, n, XS, pin);
    else k_panel_in<8><<<(unsigned) ((t + 255) / 256), 256, 0, st>>>(pg, g0, n, XS, pin);
    return cudaGetLastError();
}

template <int KID, bool FAR>
static cudaError_t launch_pair_kf(int NV, const PairOwner* ow, int n, const PairPartner* pp, const float4* pts, KParam kp,
                                  const double* XS, double* PS, cudaStream_t st, const float4* lo)
{
    if (KID == KRNL_COULOMB_ID && !FAR && !lo) return cudaErrorInvalidValue;
    if (NV == 16)
    {
        constexpr int b = pair_smem_bytes<16>();
        cudaError_t e = allow_smem(k_jit_pair<KID, 16, FAR>, b);
        if (e != cudaSuccess) return e;
        k_jit_pair<KID, 16, FAR><<<n, 32 * kPairWarps, b, st>>>(ow, pp, pts, kp, XS, PS, lo);
    } else if (NV == 8) {
        constexpr int b = pair_smem_bytes<8>();
        cudaError_t e = allow_smem(k_jit_pair<KID, 8, FAR>, b);
        if (e != cudaSuccess) return e;
        k_jit_pair<KID, 8, FAR><<<n, 32 * kPairWarps, b, st>>>(ow, pp, pts, kp, XS, PS, lo);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int KID>
static cudaError_t launch_pair_k(int NV, const PairOwner* ow, int n, const PairPartner* pp, const float4* pts, KParam kp,
                                 const double* XS, double* PS, cudaStream_t st, int far, const float4* lo)
{
    return far ? launch_pair_kf<KID, true>(NV, ow, n, pp, pts, kp, XS, PS, st, lo)
               : launch_pair_kf<KID, false>(NV, ow, n, pp, pts, kp, XS, PS, st, lo);
}

cudaError_t launch_pair(int kid, int NV, const PairOwner* ow, int n, const PairPartner* pp, const void* pts, KParam kp,
                        const double* XS, double* PS, cudaStream_t st, int far, const float4* lo)
{
    if (n <= 0) return cudaSuccess;
    const float4* p = (const float4*) pts;
    switch (kid)
    {
        case KRNL_COULOMB_ID:  return launch_pair_k<KRNL_COULOMB_ID>(NV, ow, n, pp, p, kp, XS, PS, st, far, lo);
        case KRNL_GAUSSIAN_ID: return launch_pair_k<KRNL_GAUSSIAN_ID>(NV, ow, n, pp, p, kp, XS, PS, st, far, lo);
        case KRNL_MATERN32_ID: return launch_pair_k<KRNL_MATERN32_ID>(NV, ow, n, pp, p, kp, XS, PS, st, far, lo);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_id_eval(int kid, const IdBlock* blks, int n, int max_ncand, const double* cand, const double* prox,
                           KParam kp, double* W, cudaStream_t st)
{
    if (n <= 0 || max_ncand <= 0 || !cand) return cudaErrorInvalidValue;
    const dim3 ge((unsigned) ((max_ncand + 63) / 64), (unsigned) n);
    switch (kid)
    {
        case KRNL_COULOMB_ID:  k_id_eval<KRNL_COULOMB_ID><<<ge, 256, 0, st>>>(blks, cand, prox, kp, W); break;
        case KRNL_GAUSSIAN_ID: k_id_eval<KRNL_GAUSSIAN_ID><<<ge, 256, 0, st>>>(blks, cand, prox, kp, W); break;
        case KRNL_MATERN32_ID: k_id_eval<KRNL_MATERN32_ID><<<ge, 256, 0, st>>>(blks, cand, prox, kp, W); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_id(int kid, const IdBlock* blks, int n, int max_ncand, int max_npp, const double* cand,
                      const double* prox, KParam kp, double* W, double reltol, int* rank, int* perm, cudaStream_t st,
                      int want_e)
{
    if (n <= 0 || max_ncand <= 0 || max_npp <= 0) return cudaErrorInvalidValue;
    if (cand)   // kernel matrices from coordinates (else W already holds the matrices)
    {
        cudaError_t e = launch_id_eval(kid, blks, n, max_ncand, cand, prox, kp, W, st);
        if (e != cudaSuccess) return e;
    }
    const int b = id_qr_smem_bytes(max_ncand, max_npp);
    cudaError_t e = allow_smem(k_id_qr, b);
    if (e != cudaSuccess) return e;
    k_id_qr<<<n, kIdThreads, b, st>>>(blks, W, reltol, rank, perm, want_e);
    return cudaGetLastError();
}

size_t qr_grid_work_bytes(int m, int n)
{
    const size_t a = (sizeof(QrgState) + 15) & ~(size_t) 15;
    return a + 8 * ((size_t) std::max(n, 1) + (size_t) std::max(m, 1));
}

cudaError_t launch_qr_grid(double* A, int m, int n, double reltol, void* work, int* rank, int* perm, int sms,
                           int want_e, cudaStream_t st)
{
    if (m <= 0 || n <= 0 || sms <= 0) return cudaErrorInvalidValue;
    QrgState* S = (QrgState*) work;
    double* const cn = (double*) ((char*) work + ((sizeof(QrgState) + 15) & ~(size_t) 15));
    double* const v = cn + n;
    const int gu = std::max(1, std::min(4 * sms, (n + 7) / 8));   // 8 warps per CTA of k_qrg_update
    k_qrg_init<<<std::max(1, std::min(sms, (n + 15) / 16)), kIdThreads, 0, st>>>(A, m, n, reltol, cn, perm, S);
    cudaError_t e = cudaGetLastError();
    const int mi = std::min(m, n);
    for (int i = 0; i < mi && e == cudaSuccess; i++)
    {
        k_qrg_pivot<<<1, kIdThreads, 0, st>>>(A, m, n, i, cn, perm, v, S);
        if (i + 1 < n) k_qrg_update<<<gu, 256, 0, st>>>(A, m, n, i, cn, v, S);
        e = cudaGetLastError();
        if (e == cudaSuccess && (i & 63) == 63 && i + 1 < mi)
        {
            // past the stopping point the launches only return: end the loop there
            int done = 0;
            e = cudaMemcpyAsync(&done, &S->done, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e == cudaSuccess && done) break;
        }
    }
    if (e != cudaSuccess) return e;
    const int gt = want_e ? std::max(1, std::min(4 * sms, (n + 255) / 256)) : 1;
    k_qrg_trsm<<<gt, 256, 0, st>>>(A, m, n, S, want_e, rank);
    return cudaGetLastError();
}

cudaError_t launch_pp_sketch(int kid, int nx, const double* X0, int ny, const double* Y0, const int* rowptr,
                             const int* col, const double* val, KParam kp, double* W, cudaStream_t st)
{
    if (nx <= 0 || ny <= 0) return cudaErrorInvalidValue;
    const long long t = (long long) nx * nx;
    const unsigned g = (unsigned) ((t + 255) / 256);
    switch (kid)
    {
        case KRNL_COULOMB_ID:  k_pp_sketch<KRNL_COULOMB_ID><<<g, 256, 0, st>>>(nx, X0, ny, Y0, rowptr, col, val, kp, W); break;
        case KRNL_GAUSSIAN_ID: k_pp_sketch<KRNL_GAUSSIAN_ID><<<g, 256, 0, st>>>(nx, X0, ny, Y0, rowptr, col, val, kp, W); break;
        case KRNL_MATERN32_ID: k_pp_sketch<KRNL_MATERN32_ID><<<g, 256, 0, st>>>(nx, X0, ny, Y0, rowptr, col, val, kp, W); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_direct(int kid, const double4* trg, int n_trg, const double4* src, int n_src, const double* val,
                          KParam kp, double* out, cudaStream_t st)
{
    unsigned g = (unsigned) ((n_trg + 127) / 128);
    switch (kid)
    {
        case KRNL_COULOMB_ID:  k_direct<KRNL_COULOMB_ID, 1><<<g, 128, 0, st>>>(trg, n_trg, src, n_src, val, kp, out); break;
        case KRNL_GAUSSIAN_ID: k_direct<KRNL_GAUSSIAN_ID, 1><<<g, 128, 0, st>>>(trg, n_trg, src, n_src, val, kp, out); break;
        case KRNL_MATERN32_ID: k_direct<KRNL_MATERN32_ID, 1><<<g, 128, 0, st>>>(trg, n_trg, src, n_src, val, kp, out); break;
        case KRNL_RPY_ID:      k_direct<KRNL_RPY_ID, 3><<<g, 128, 0, st>>>(trg, n_trg, src, n_src, val, kp, out); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename TO>
static cudaError_t gen_typed(int kid, const GenTask* t, int n, const double4* pts, KParam kp, TO* arena,
                             cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    switch (kid)
    {
        case KRNL_COULOMB_ID:  k_gen<KRNL_COULOMB_ID, 1, TO><<<n, kGenThreads, 0, st>>>(t, pts, kp, arena); break;
        case KRNL_GAUSSIAN_ID: k_gen<KRNL_GAUSSIAN_ID, 1, TO><<<n, kGenThreads, 0, st>>>(t, pts, kp, arena); break;
        case KRNL_MATERN32_ID: k_gen<KRNL_MATERN32_ID, 1, TO><<<n, kGenThreads, 0, st>>>(t, pts, kp, arena); break;
        case KRNL_RPY_ID:      k_gen<KRNL_RPY_ID, 3, TO><<<n, kGenThreads, 0, st>>>(t, pts, kp, arena); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_gen(int kid, int kd, int fp32, const GenTask* t, int n, const double4* pts, KParam kp, void* arena,
                       cudaStream_t st)
{
    if ((kid == KRNL_RPY_ID) != (kd == 3)) return cudaErrorInvalidValue;
    return fp32 ? gen_typed<float>(kid, t, n, pts, kp, (float*) arena, st)
                : gen_typed<double>(kid, t, n, pts, kp, (double*) arena, st);
}

template cudaError_t launch_up<double>(int, const UpTask*, int, const double*, double*, cudaStream_t, int);
template cudaError_t launch_up<float>(int, const UpTask*, int, const float*, double*, cudaStream_t, int);
template cudaError_t launch_blk<double>(int, const BlkTask*, int, const double*, const double*, double*, cudaStream_t, int, int*, int);
template cudaError_t launch_blk<float>(int, const BlkTask*, int, const float*, const double*, double*, cudaStream_t, int, int*, int);
template cudaError_t launch_down<double>(int, const DownTask*, int, const double*, const double*, double*, double*, cudaStream_t, int);
template cudaError_t launch_down<float>(int, const DownTask*, int, const float*, const double*, double*, double*, cudaStream_t, int);

}  // namespace h2gpu
