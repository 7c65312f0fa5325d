// h2gpu_launch.h -- host-side launchers of the engine's kernels (internal).
#pragma once
#include <cuda_runtime.h>
#include "h2gpu_internal.cuh"

namespace h2gpu {

// kernel ids as in include/h2gpu.h
constexpr int KRNL_COULOMB_ID = 1;
constexpr int KRNL_GAUSSIAN_ID = 2;
constexpr int KRNL_MATERN32_ID = 3;
constexpr int KRNL_RPY_ID = 4;

cudaError_t launch_gather(int NV, const double* X, long long x_rs, long long x_cs, int nv, const int* fwd, int N,
                          double* XS, cudaStream_t st);
template <typename TA>
cudaError_t launch_up(int NV, const UpTask* t, int n, const TA* U, double* XS, cudaStream_t st, int use_tc = 0);
template <typename TA>
cudaError_t launch_blk(int NV, const BlkTask* t, int n, const TA* arena, const double* XS, double* PS, cudaStream_t st,
                       int use_tc = 0, int* status = nullptr,    // use_tc: 1 mma.sync, 2 tcgen05
                       int n_small = 0);   // NV 1: leading tasks that blk1_fits for TA (one warp each)
// 64-wide panels of FP32 stored blocks on tcgen05: pass 0 (mode 0, units = 64-row chunks:
// A V) or pass 1 (mode 1, units = 64-column tiles: A^T W), outputs written once
cudaError_t launch_blk_wide(int mode, const BlkTask* t, const WideUnit* u, int n, const float* arena,
                            const uint16_t* XS3, long long rows3, double* PS, cudaStream_t st, int* status);
// rows [row0, row0 + n) of the 64-wide input space (row stride 64) into its BF16 pieces
cudaError_t launch_split3(const double* XS, long long row0, long long n, long long rows, uint16_t* XS3,
                          cudaStream_t st);
template <typename TA>
cudaError_t launch_down(int NV, const DownTask* t, int n, const TA* U, const double* Y1, double* PS, double* PUSH,
                        cudaStream_t st, int use_tc = 0);
cudaError_t launch_y1sum(int NV, const Y1Task* t, int n, const int* slots, const double* PS, double* Y1, cudaStream_t st);
cudaError_t launch_asm(int NV, const AsmTask* t, int n, const int* slots, const double* PS, const int* fwd,
                       double* Y, long long y_rs, long long y_cs, int nv, cudaStream_t st);
// far: every source set is admissible for its target (r > 0); ppts / pin / tiles: the
// source panels and tile lists, which the tensor-core kernel (FP32 scalar kernels,
// NV 8 / 16, use_tc) reads; lo / plo: the low parts of the FP32 points and of the
// panels, which the FP32 Coulomb near field needs (exact differences)
cudaError_t launch_jit(int kid, int fp32, int NV, const JitTarget* tg, int n, const JitSource* sr, const void* pts,
                       KParam kp, int use_shift, int use_tc, const double* XS, double* PS, double* Y1, cudaStream_t st,
                       int far = 0, const float4* ppts = nullptr, const uint4* pin = nullptr,
                       const TileRec* tiles = nullptr, const float4* lo = nullptr, const float4* plo = nullptr);
// source panels: the points (once per image) and the inputs of groups [g0, g0 + n) for a
// panel of NV right-hand sides (NV 8 / 16; other widths do nothing)
cudaError_t launch_panel_pts(const PanelGroup* pg, int n, const float4* pts, float sigma, float4* ppts, cudaStream_t st);
// the low parts of the panel points (6 float4 per group)
cudaError_t launch_panel_lo(const PanelGroup* pg, int n, const float4* lo, float4* out, cudaStream_t st);
cudaError_t launch_panel_in(int NV, const PanelGroup* pg, int g0, int n, const double* XS, uint4* pin, cudaStream_t st);
cudaError_t launch_pair(int kid, int NV, const PairOwner* ow, int n, const PairPartner* pp, const void* pts, KParam kp,
                        const double* XS, double* PS, cudaStream_t st,
                        int far = 0, const float4* lo = nullptr);
// stored-block generation: tasks [0, n) into arena (double or float, per fp32)
cudaError_t launch_gen(int kid, int kd, int fp32, const GenTask* t, int n, const double4* pts, KParam kp, void* arena,
                       cudaStream_t st);
// pipe peak micro-benchmarks: which 0 = FP32 FMA (packed FP32x2), 1 = MUFU ex2
cudaError_t launch_peak(int which, int blocks, int iters, float* out, cudaStream_t st);
cudaError_t launch_direct(int kid, const double4* trg, int n_trg, const double4* src, int n_src, const double* val,
                          KParam kp, double* out, cudaStream_t st);
// dynamic shared memory of the pivoted-QR kernel for blocks of up to ncand candidates and
// npp proxy points (column norms, Householder vector, permutation, reduction scratch)
constexpr int kIdQrWarps = 16;
constexpr int id_qr_smem_bytes(int ncand, int npp) { return 8 * (ncand + npp + kIdQrWarps) + 4 * (ncand + kIdQrWarps); }
// interpolative decompositions of n kernel blocks (scalar kernels): kernel matrices
// into W, pivoted QR, E = R11^-1 R12 in place; rank[b], perm[perm_off + j]
// (cand == nullptr: W already holds the blocks' matrices; want_e = 0: no E)
cudaError_t launch_id(int kid, const IdBlock* blks, int n, int max_ncand, int max_npp, const double* cand,
                      const double* prox, KParam kp, double* W, double reltol, int* rank, int* perm, cudaStream_t st,
                      int want_e = 1);
// the pivoted QR (and E, if want_e) of one large matrix A^T (m x n, column j at A + j m)
// over the whole GPU, 2 launches per iteration (k_id_qr's arithmetic and stopping rule);
// work: qr_grid_work_bytes(m, n) of device memory (16-byte aligned); rank: 1 device int;
// perm: n device ints; sms: the device's SM count
size_t qr_grid_work_bytes(int m, int n);
cudaError_t launch_qr_grid(double* A, int m, int n, double reltol, void* work, int* rank, int* perm, int sms,
                           int want_e, cudaStream_t st);
// the kernel matrices of launch_id alone (W[b] = K(cand_b, prox)^T, column j = candidate j)
cudaError_t launch_id_eval(int kid, const IdBlock* blks, int n, int max_ncand, const double* cand, const double* prox,
                           KParam kp, double* W, cudaStream_t st);
// proxy-point generation: W = K(X0, Y0) S (nx x nx), S^T in CSR with nx rows
cudaError_t launch_pp_sketch(int kid, int nx, const double* X0, int ny, const double* Y0, const int* rowptr,
                             const int* col, const double* val, KParam kp, double* W, cudaStream_t st);

}  // namespace h2gpu
