// h2gpu_solve.cu -- lock-step conjugate gradients on (K + mu I) for the slots of one
// image, entirely on the device (include/h2gpu.h, h2gpu_cg_*).
//
// The solver is H2Pack's left-preconditioned CG with the identity preconditioner
// (examples/PCG/pcg.c:11-152) on the shifted operator of
// examples/SPDHSS-H2/pcg_tests.c:13-20, run for up to 16 right-hand sides ("slots")
// at once: the slots are the columns of one 16-wide panel, so every iteration is one
// H2 matmul (of the panel's columns up to the highest busy slot) plus five small
// kernels (direction update, p'Ap, alpha, x/r update with ||r||^2, status).  The host only enqueues iterations and reads the
// 16 slot records once per batch of iterations; it never waits per iteration.
//
// Precision: vectors, inner products and the residual recomputation are FP64; the
// operator runs in the image's precision.  A slot whose recursive residual claims
// convergence (or that ran `refresh` iterations since its last restart, for a mixed
// operator) moves to CHECK; h2gpu_cg_check recomputes b - (K + mu I) x with the FP64
// operator, and the slot either finishes or restarts CG from the true residual --
// iterative refinement, so a mixed operator still reaches an FP64 tolerance.
//
// Determinism: every reduction has a fixed order (row ranges per block, a fixed tree
// in shared memory, partials summed in block order by one block), and every kernel
// treats the 16 columns independently.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "h2gpu.h"

#define H2G_API extern "C" __attribute__((visibility("default")))

namespace h2gpu {
int set_error(int code, const char* msg);
int image_apply_quiet(h2gpu_image* im, int precision, int n_vec, const double* dX, int ldx, double* dY, int ldy);
int image_info(const h2gpu_image* im, int* N, int* device, int* precision, void** stream);
}  // namespace h2gpu

namespace {

constexpr int kS = 16;          // slots = panel width
constexpr int kHist = 8192;     // residual norms kept per slot
constexpr int kRedBlocks = 592; // 148 SMs x 4

struct CgSlot {
    double bnorm2;      // ||b||^2
    double tol2;        // (tol ||b||)^2
    double rho;         // r'r of the current residual
    double rho_prev;    // r'r one iteration earlier
    double alpha;
    double rr;          // ||r||^2: recursive while running, true after a check
    int state, kind, it, it_total, max_iter, restart, first, pad;
};

struct CgCtx {
    double mu;
    int N, G;
    const double* B;
    double *X, *R, *P, *AP;
    double* part;       // [G][kS]
    CgSlot* sl;
    double* hist;       // [kS][kHist]
};

__device__ __forceinline__ bool running_pcg(const CgSlot& s) { return s.state == H2GPU_CG_RUN && s.kind == H2GPU_CG_PCG; }

// Fixed-order reduction of per-thread column sums (thread t: column t % 16, row lane
// t / 16) into part[blockIdx.x][col].  256 threads.
__device__ __forceinline__ void block_col_reduce(double v, double* part)
{
    __shared__ double s[256];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int w = 128; w >= kS; w >>= 1)
    {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < kS) part[blockIdx.x * kS + threadIdx.x] = s[threadIdx.x];
}

// Row range of block b: contiguous, fixed by N and G only.
__device__ __forceinline__ void rows_of(int N, int G, int b, int& r0, int& r1)
{
    const int per = (N + G - 1) / G;
    r0 = min(N, b * per);
    r1 = min(N, r0 + per);
}

// One block of 256 threads: per column, the sum of part[0..G)[col] in a fixed order.
// The result is valid in threads 0..15 (column = threadIdx.x).
__device__ __forceinline__ double sum_parts(const double* part, int G)
{
    __shared__ double s[256];
    const int col = threadIdx.x / kS, j = threadIdx.x % kS;   // 16 threads per column
    double v = 0.0;
    for (int b = j; b < G; b += kS) v += part[b * kS + col];
    s[threadIdx.x] = v;
    __syncthreads();
    double tot = 0.0;
    if (threadIdx.x < kS)
        for (int q = 0; q < kS; q++) tot += s[threadIdx.x * kS + q];
    __syncthreads();
    return tot;
}

__global__ void k_cg_dir(CgCtx c)
{
    __shared__ double beta[kS];
    __shared__ int on[kS], first[kS];
    if (threadIdx.x < kS)
    {
        const CgSlot s = c.sl[threadIdx.x];
        on[threadIdx.x] = running_pcg(s);
        first[threadIdx.x] = s.first;
        beta[threadIdx.x] = s.first ? 0.0 : s.rho / s.rho_prev;
    }
    __syncthreads();
    const long long n = (long long) c.N * kS;
    for (long long e = blockIdx.x * 256LL + threadIdx.x; e < n; e += (long long) gridDim.x * 256)
    {
        const int k = (int) (e & (kS - 1));
        if (!on[k]) continue;
        c.P[e] = first[k] ? c.R[e] : c.R[e] + beta[k] * c.P[e];
    }
}

__global__ void k_cg_dot(CgCtx c)
{
    const int k = threadIdx.x % kS, lane = threadIdx.x / kS;
    const bool on = running_pcg(c.sl[k]);
    int r0, r1;
    rows_of(c.N, c.G, blockIdx.x, r0, r1);
    double v = 0.0;
    if (on)
        for (int i = r0 + lane; i < r1; i += 256 / kS)
        {
            const long long e = (long long) i * kS + k;
            const double p = c.P[e];
            v += p * (c.AP[e] + c.mu * p);
        }
    block_col_reduce(v, c.part);
}

__global__ void k_cg_alpha(CgCtx c)
{
    const double pap = sum_parts(c.part, c.G);
    if (threadIdx.x < kS)
    {
        CgSlot& s = c.sl[threadIdx.x];
        if (running_pcg(s)) s.alpha = s.rho / pap;
    }
}

__global__ void k_cg_update(CgCtx c)
{
    const int k = threadIdx.x % kS, lane = threadIdx.x / kS;
    const CgSlot s = c.sl[k];
    int r0, r1;
    rows_of(c.N, c.G, blockIdx.x, r0, r1);
    double v = 0.0;
    if (running_pcg(s))
    {
        for (int i = r0 + lane; i < r1; i += 256 / kS)
        {
            const long long e = (long long) i * kS + k;
            const double p = c.P[e];
            const double r = c.R[e] - s.alpha * (c.AP[e] + c.mu * p);
            c.X[e] += s.alpha * p;
            c.R[e] = r;
            v += r * r;
        }
    } else if (s.state == H2GPU_CG_RUN && s.kind == H2GPU_CG_MATVEC) {
        for (int i = r0 + lane; i < r1; i += 256 / kS)
        {
            const long long e = (long long) i * kS + k;
            c.X[e] = c.AP[e] + c.mu * c.P[e];
        }
    }
    block_col_reduce(v, c.part);
}

__global__ void k_cg_finish(CgCtx c)
{
    const double rr = sum_parts(c.part, c.G);
    if (threadIdx.x < kS)
    {
        CgSlot& s = c.sl[threadIdx.x];
        if (running_pcg(s))
        {
            s.rr = rr;
            s.it++;
            s.it_total++;
            if (s.it_total <= kHist) c.hist[threadIdx.x * kHist + s.it_total - 1] = sqrt(rr);
            s.rho_prev = s.rho;
            s.rho = rr;
            s.first = 0;
            if (rr <= s.tol2 || s.it_total >= s.max_iter || (s.restart > 0 && s.it >= s.restart))
                s.state = H2GPU_CG_CHECK;
        } else if (s.state == H2GPU_CG_RUN && s.kind == H2GPU_CG_MATVEC) {
            s.rr = 0.0;
            s.it_total = 1;
            s.state = H2GPU_CG_DONE;
        }
    }
}

// True residual r = b - (K + mu I) x of the CHECK slots (AP holds K x in FP64).
__global__ void k_cg_resid(CgCtx c)
{
    const int k = threadIdx.x % kS, lane = threadIdx.x / kS;
    const bool on = c.sl[k].state == H2GPU_CG_CHECK;
    int r0, r1;
    rows_of(c.N, c.G, blockIdx.x, r0, r1);
    double v = 0.0;
    if (on)
        for (int i = r0 + lane; i < r1; i += 256 / kS)
        {
            const long long e = (long long) i * kS + k;
            const double r = c.B[e] - (c.AP[e] + c.mu * c.X[e]);
            c.R[e] = r;
            v += r * r;
        }
    block_col_reduce(v, c.part);
}

__global__ void k_cg_check_finish(CgCtx c)
{
    const double rr = sum_parts(c.part, c.G);
    if (threadIdx.x < kS)
    {
        CgSlot& s = c.sl[threadIdx.x];
        if (s.state == H2GPU_CG_CHECK)
        {
            s.rr = rr;
            if (rr <= s.tol2 || s.it_total >= s.max_iter) s.state = H2GPU_CG_DONE;
            else
            {
                s.state = H2GPU_CG_RUN;      // restart CG from the true residual
                s.first = 1;
                s.it = 0;
                s.rho = rr;
                s.rho_prev = rr;
            }
        }
    }
}

// ||b||^2 of a new slot and its record (one block of 256 threads).
__global__ void k_cg_admit(CgCtx c, int slot, int kind, double tol, int max_iter, int restart)
{
    __shared__ double s[256];
    double v = 0.0;
    for (int i = threadIdx.x; i < c.N; i += 256)
    {
        const double b = c.B[(long long) i * kS + slot];
        v += b * b;
    }
    s[threadIdx.x] = v;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1)
    {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        CgSlot r;
        memset(&r, 0, sizeof(r));
        r.bnorm2 = s[0];
        r.tol2 = tol * tol * s[0];
        r.rho = r.rho_prev = r.rr = s[0];
        r.kind = kind;
        r.max_iter = max_iter;
        r.restart = restart;
        r.first = 1;
        // b = 0: x = 0 is the solution (pcg.c's loop does not start)
        r.state = (kind == H2GPU_CG_PCG && s[0] == 0.0) ? H2GPU_CG_DONE : H2GPU_CG_RUN;
        c.sl[slot] = r;
    }
}

__global__ void k_cg_free(CgSlot* sl, int slot) { sl[slot].state = H2GPU_CG_FREE; }

}  // namespace

struct h2gpu_cg {
    std::mutex lock;
    h2gpu_image* img = nullptr;
    int N = 0, device = 0, precision = H2GPU_PREC_FP64;
    cudaStream_t stream = nullptr;
    CgCtx c{};
    double* mem = nullptr;
    CgSlot* d_sl = nullptr;
    CgSlot* h_sl = nullptr;     // pinned mirror, refreshed by h2gpu_cg_sync
    double* d_hist = nullptr;
    int refresh = 0;
    cudaEvent_t done = nullptr; // recorded after the work each h2gpu_cg_step / h2gpu_cg_check enqueues
};

#define CGCK(call)                                                                     \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) return h2gpu::set_error(                                \
            e_ == cudaErrorMemoryAllocation ? H2GPU_ERR_NOMEM : H2GPU_ERR_CUDA,         \
            cudaGetErrorString(e_));                                                   \
    } while (0)

static void cg_free_all(h2gpu_cg* g)
{
    if (g->mem) cudaFree(g->mem);
    if (g->d_sl) cudaFree(g->d_sl);
    if (g->d_hist) cudaFree(g->d_hist);
    if (g->h_sl) cudaFreeHost(g->h_sl);
    if (g->done) cudaEventDestroy(g->done);
    g->mem = nullptr; g->d_sl = nullptr; g->d_hist = nullptr; g->h_sl = nullptr; g->done = nullptr;
}

H2G_API int h2gpu_cg_create(h2gpu_image* img, double mu, int refresh, h2gpu_cg** out)
{
    if (!img || !out) return h2gpu::set_error(H2GPU_ERR_INVALID, "image or out is NULL");
    *out = nullptr;
    if (!(mu >= 0.0) || refresh < 0) return h2gpu::set_error(H2GPU_ERR_INVALID, "mu must be >= 0 and refresh >= 0");
    h2gpu_cg* g = new h2gpu_cg();
    g->img = img;
    void* st = nullptr;
    h2gpu::image_info(img, &g->N, &g->device, &g->precision, &st);
    g->stream = (cudaStream_t) st;
    g->refresh = refresh;
    const int N = g->N;
    const int G = std::max(1, std::min(kRedBlocks, (N + 63) / 64));
    int stc = H2GPU_OK;
    do {
        if (cudaSetDevice(g->device) != cudaSuccess) { stc = h2gpu::set_error(H2GPU_ERR_CUDA, "cudaSetDevice failed"); break; }
        const size_t panel = (size_t) N * kS;
        if (cudaMalloc(&g->mem, sizeof(double) * (5 * panel + (size_t) G * kS)) != cudaSuccess ||
            cudaMalloc(&g->d_sl, sizeof(CgSlot) * kS) != cudaSuccess ||
            cudaMalloc(&g->d_hist, sizeof(double) * kS * kHist) != cudaSuccess ||
            cudaMallocHost(&g->h_sl, sizeof(CgSlot) * kS) != cudaSuccess ||
            cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming) != cudaSuccess)
        {
            stc = h2gpu::set_error(H2GPU_ERR_NOMEM, "CG engine allocation failed");
            break;
        }
        g->c.mu = mu; g->c.N = N; g->c.G = G;
        double* m = g->mem;
        g->c.B = m; g->c.X = m + panel; g->c.R = m + 2 * panel; g->c.P = m + 3 * panel; g->c.AP = m + 4 * panel;
        g->c.part = m + 5 * panel;
        g->c.sl = g->d_sl;
        g->c.hist = g->d_hist;
        if (cudaMemsetAsync(g->mem, 0, sizeof(double) * 5 * panel, g->stream) != cudaSuccess ||
            cudaMemsetAsync(g->d_sl, 0, sizeof(CgSlot) * kS, g->stream) != cudaSuccess ||
            cudaStreamSynchronize(g->stream) != cudaSuccess)
        {
            stc = h2gpu::set_error(H2GPU_ERR_CUDA, "CG engine initialisation failed");
            break;
        }
        memset(g->h_sl, 0, sizeof(CgSlot) * kS);
    } while (0);
    if (stc != H2GPU_OK)
    {
        cg_free_all(g);
        delete g;
        return stc;
    }
    *out = g;
    return H2GPU_OK;
}

H2G_API int h2gpu_cg_destroy(h2gpu_cg* g)
{
    if (!g) return H2GPU_OK;
    cudaSetDevice(g->device);
    cudaStreamSynchronize(g->stream);
    cg_free_all(g);
    delete g;
    return H2GPU_OK;
}

H2G_API int h2gpu_cg_admit(h2gpu_cg* g, int slot, int kind, const double* d_b, double tol, int max_iter)
{
    if (!g || !d_b) return h2gpu::set_error(H2GPU_ERR_INVALID, "engine or b is NULL");
    if (slot < 0 || slot >= kS) return h2gpu::set_error(H2GPU_ERR_INVALID, "slot out of range [0, 16)");
    if (kind != H2GPU_CG_MATVEC && kind != H2GPU_CG_PCG) return h2gpu::set_error(H2GPU_ERR_INVALID, "unknown request kind");
    if (!(tol > 0.0) || max_iter < 1) return h2gpu::set_error(H2GPU_ERR_INVALID, "tol must be > 0 and max_iter >= 1");
    std::lock_guard<std::mutex> lk(g->lock);
    if (g->h_sl[slot].state != H2GPU_CG_FREE) return h2gpu::set_error(H2GPU_ERR_STATE, "slot is busy");
    CGCK(cudaSetDevice(g->device));
    const size_t pitch = sizeof(double) * kS, col = sizeof(double);
    double* B = const_cast<double*>(g->c.B);
    CGCK(cudaMemcpy2DAsync(B + slot, pitch, d_b, col, col, g->N, cudaMemcpyDeviceToDevice, g->stream));
    CGCK(cudaMemcpy2DAsync(g->c.R + slot, pitch, d_b, col, col, g->N, cudaMemcpyDeviceToDevice, g->stream));
    CGCK(cudaMemset2DAsync(g->c.X + slot, pitch, 0, col, g->N, g->stream));
    if (kind == H2GPU_CG_MATVEC)
        CGCK(cudaMemcpy2DAsync(g->c.P + slot, pitch, d_b, col, col, g->N, cudaMemcpyDeviceToDevice, g->stream));
    else
        CGCK(cudaMemset2DAsync(g->c.P + slot, pitch, 0, col, g->N, g->stream));
    const int restart = g->precision == H2GPU_PREC_FP64 ? 0 : g->refresh;
    k_cg_admit<<<1, 256, 0, g->stream>>>(g->c, slot, kind, tol, max_iter, restart);
    CGCK(cudaGetLastError());
    g->h_sl[slot].state = H2GPU_CG_RUN;     // host view until the next sync
    return H2GPU_OK;
}

// Columns the operator must be applied to: up to the highest slot in `state` (by the
// host's latest view: the last sync plus admissions since, an upper bound of the
// device's), so a panel with few busy slots applies a narrower panel.
static int busy_width(const h2gpu_cg* g, int state)
{
    int hi = 0;
    for (int k = 0; k < kS; k++)
        if (g->h_sl[k].state == state) hi = k + 1;
    return hi;
}

H2G_API int h2gpu_cg_step(h2gpu_cg* g, int n_iter)
{
    if (!g || n_iter < 1) return h2gpu::set_error(H2GPU_ERR_INVALID, "bad engine or n_iter");
    std::lock_guard<std::mutex> lk(g->lock);
    CGCK(cudaSetDevice(g->device));
    const int G = g->c.G;
    const int ge = std::max(1, std::min(kRedBlocks, (g->N * kS + 255) / 256));
    const int width = busy_width(g, H2GPU_CG_RUN);
    if (width == 0) return H2GPU_OK;
    for (int t = 0; t < n_iter; t++)
    {
        k_cg_dir<<<ge, 256, 0, g->stream>>>(g->c);
        int st = h2gpu::image_apply_quiet(g->img, g->precision, width, g->c.P, kS, g->c.AP, kS);
        if (st != H2GPU_OK) return st;
        k_cg_dot<<<G, 256, 0, g->stream>>>(g->c);
        k_cg_alpha<<<1, 256, 0, g->stream>>>(g->c);
        k_cg_update<<<G, 256, 0, g->stream>>>(g->c);
        k_cg_finish<<<1, 256, 0, g->stream>>>(g->c);
    }
    CGCK(cudaGetLastError());
    CGCK(cudaEventRecord(g->done, g->stream));
    return H2GPU_OK;
}

H2G_API int h2gpu_cg_check(h2gpu_cg* g)
{
    if (!g) return h2gpu::set_error(H2GPU_ERR_INVALID, "engine is NULL");
    std::lock_guard<std::mutex> lk(g->lock);
    CGCK(cudaSetDevice(g->device));
    const int width = busy_width(g, H2GPU_CG_CHECK);
    if (width == 0) return H2GPU_OK;
    int st = h2gpu::image_apply_quiet(g->img, H2GPU_PREC_FP64, width, g->c.X, kS, g->c.AP, kS);
    if (st != H2GPU_OK) return st;
    k_cg_resid<<<g->c.G, 256, 0, g->stream>>>(g->c);
    k_cg_check_finish<<<1, 256, 0, g->stream>>>(g->c);
    CGCK(cudaGetLastError());
    CGCK(cudaEventRecord(g->done, g->stream));
    // a checked slot either finished or restarts: until the next sync the host view
    // counts it as running, so the next step's panel covers it
    for (int k = 0; k < kS; k++)
        if (g->h_sl[k].state == H2GPU_CG_CHECK) g->h_sl[k].state = H2GPU_CG_RUN;
    return H2GPU_OK;
}

// 1 when the work enqueued by the last h2gpu_cg_step / h2gpu_cg_check has finished (a
// following h2gpu_cg_sync then returns without waiting on the device), 0 while it runs.
H2G_API int h2gpu_cg_query(h2gpu_cg* g)
{
    if (!g) return h2gpu::set_error(H2GPU_ERR_INVALID, "engine is NULL");
    std::lock_guard<std::mutex> lk(g->lock);
    CGCK(cudaSetDevice(g->device));
    cudaError_t e = cudaEventQuery(g->done);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) return 0;
    return h2gpu::set_error(H2GPU_ERR_CUDA, cudaGetErrorString(e));
}

// Free a slot whatever its state (a request given up by its caller): iterations already
// enqueued finish first (stream order), then the slot takes no further part and may be
// admitted again.
H2G_API int h2gpu_cg_cancel(h2gpu_cg* g, int slot)
{
    if (!g) return h2gpu::set_error(H2GPU_ERR_INVALID, "engine is NULL");
    if (slot < 0 || slot >= kS) return h2gpu::set_error(H2GPU_ERR_INVALID, "slot out of range [0, 16)");
    std::lock_guard<std::mutex> lk(g->lock);
    CGCK(cudaSetDevice(g->device));
    k_cg_free<<<1, 1, 0, g->stream>>>(g->d_sl, slot);
    CGCK(cudaGetLastError());
    g->h_sl[slot].state = H2GPU_CG_FREE;
    return H2GPU_OK;
}

H2G_API int h2gpu_cg_sync(h2gpu_cg* g, int* state, int* iters, double* relres)
{
    if (!g) return h2gpu::set_error(H2GPU_ERR_INVALID, "engine is NULL");
    std::lock_guard<std::mutex> lk(g->lock);
    CGCK(cudaSetDevice(g->device));
    CGCK(cudaMemcpyAsync(g->h_sl, g->d_sl, sizeof(CgSlot) * kS, cudaMemcpyDeviceToHost, g->stream));
    CGCK(cudaStreamSynchronize(g->stream));
    for (int k = 0; k < kS; k++)
    {
        const CgSlot& s = g->h_sl[k];
        if (state) state[k] = s.state;
        if (iters) iters[k] = s.it_total;
        if (relres) relres[k] = s.bnorm2 > 0.0 ? std::sqrt(s.rr / s.bnorm2) : 0.0;
    }
    return H2GPU_OK;
}

H2G_API int h2gpu_cg_take(h2gpu_cg* g, int slot, double* d_x)
{
    if (!g || !d_x) return h2gpu::set_error(H2GPU_ERR_INVALID, "engine or x is NULL");
    if (slot < 0 || slot >= kS) return h2gpu::set_error(H2GPU_ERR_INVALID, "slot out of range [0, 16)");
    std::lock_guard<std::mutex> lk(g->lock);
    if (g->h_sl[slot].state != H2GPU_CG_DONE)
        return h2gpu::set_error(H2GPU_ERR_STATE, "slot has no finished result (call h2gpu_cg_sync first)");
    CGCK(cudaSetDevice(g->device));
    const size_t pitch = sizeof(double) * kS, col = sizeof(double);
    CGCK(cudaMemcpy2DAsync(d_x, col, g->c.X + slot, pitch, col, g->N, cudaMemcpyDeviceToDevice, g->stream));
    k_cg_free<<<1, 1, 0, g->stream>>>(g->d_sl, slot);
    CGCK(cudaGetLastError());
    CGCK(cudaStreamSynchronize(g->stream));
    g->h_sl[slot].state = H2GPU_CG_FREE;
    return H2GPU_OK;
}

H2G_API int h2gpu_cg_history(h2gpu_cg* g, int slot, double* out, int max_n)
{
    if (!g || !out || max_n < 0) return h2gpu::set_error(H2GPU_ERR_INVALID, "bad history arguments");
    if (slot < 0 || slot >= kS) return h2gpu::set_error(H2GPU_ERR_INVALID, "slot out of range [0, 16)");
    std::lock_guard<std::mutex> lk(g->lock);
    CGCK(cudaSetDevice(g->device));
    const int n = std::min(std::min(max_n, kHist), g->h_sl[slot].it_total);
    if (n > 0)
    {
        CGCK(cudaMemcpyAsync(out, g->d_hist + (size_t) slot * kHist, sizeof(double) * n, cudaMemcpyDeviceToHost,
                             g->stream));
        CGCK(cudaStreamSynchronize(g->stream));
    }
    return n;
}
