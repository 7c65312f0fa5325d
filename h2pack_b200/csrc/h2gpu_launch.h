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
                       int use_tc = 0, int* status = nullptr);   // use_tc: 1 mma.sync, 2 tcgen05
template <typename TA>
cudaError_t launch_down(int NV, const DownTask* t, int n, const TA* U, const double* Y1, double* PS, double* PUSH,
                        cudaStream_t st, int use_tc = 0);
cudaError_t launch_y1sum(int NV, const Y1Task* t, int n, const int* slots, const double* PS, double* Y1, cudaStream_t st);
cudaError_t launch_asm(int NV, const AsmTask* t, int n, const int* slots, const double* PS, const int* fwd,
                       double* Y, long long y_rs, long long y_cs, int nv, cudaStream_t st);
cudaError_t launch_jit(int kid, int fp32, int NV, const JitTarget* tg, int n, const JitSource* sr, const void* pts,
                       KParam kp, int use_shift, int use_tc, const double* XS, double* PS, double* Y1, cudaStream_t st,
                       int far = 0);   // far: every source set is admissible for its target (r > 0)
cudaError_t launch_pair(int kid, int NV, const PairOwner* ow, int n, const PairPartner* pp, const void* pts, KParam kp,
                        const double* XS, double* PS, cudaStream_t st,
                        int far = 0);
cudaError_t launch_direct(int kid, const double4* trg, int n_trg, const double4* src, int n_src, const double* val,
                          KParam kp, double* out, cudaStream_t st);

}  // namespace h2gpu
