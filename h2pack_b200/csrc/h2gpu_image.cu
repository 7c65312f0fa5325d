// h2gpu_image.cu -- device image of one H2 representation and the C ABI (include/h2gpu.h).
//
// h2gpu_image_create turns the plain-pointer view of struct H2Pack into flat task
// lists per phase (built once on the host, uploaded once):
//   * upward / downward tasks per tree level (levels are the only serial
//     dependency, src/H2Pack_matvec.c:113, :314),
//   * AOT: one record per <= 64-row chunk of every stored B / D block
//     (replacing the static B_blk / D_blk thread partitions, src/H2Pack_build.c:762-764,
//     :1006-1008, and the per-thread output copies, src/H2Pack_matvec.c:1191-1263),
//   * JIT: one record per target chunk with the list of its source point sets
//     (the admissible / inadmissible pair lists of src/H2Pack_partition.c:327-432
//     turned into per-node interaction lists),
//   * slot lists that say which partial results sum into which output rows.
// Applying the matrix is then a fixed sequence of kernel launches per panel of
// right-hand sides; nothing is allocated or built in the apply path once the
// buffers for the widest panel exist.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <map>
#include <vector>

#include <cuda_runtime.h>

#include "h2gpu.h"
#include "h2gpu_internal.cuh"
#include "h2gpu_launch.h"

using namespace h2gpu;

#define H2G_API extern "C" __attribute__((visibility("default")))

static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                                       \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return fail(e_ == cudaErrorMemoryAllocation ? H2GPU_ERR_NOMEM : H2GPU_ERR_CUDA,            \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);  \
    } while (0)

#define REQ(cond, ...)                                               \
    do {                                                             \
        if (!(cond)) return fail(H2GPU_ERR_INVALID, __VA_ARGS__);    \
    } while (0)

#define TRY(expr)                        \
    do {                                 \
        int s_ = (expr);                 \
        if (s_ != H2GPU_OK) return s_;   \
    } while (0)

namespace {

template <typename T>
int upload(const std::vector<T>& h, T** d, size_t& total)
{
    *d = nullptr;
    if (h.empty()) return H2GPU_OK;
    CK(cudaMalloc((void**) d, sizeof(T) * h.size()));
    CK(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    total += sizeof(T) * h.size();
    return H2GPU_OK;
}

struct Ev {
    cudaEvent_t e[8] = {};
};

}  // namespace

struct h2gpu_image {
    std::mutex mu;
    int device = 0;
    cudaStream_t stream = nullptr;
    int precision = H2GPU_PREC_FP64;
    int max_nv = 16;

    // dimensions
    int n_point = 0, kd = 1, xpt_dim = 3, n_node = 0, n_leaf = 0, max_level = 0, min_adm = 0, BD_JIT = 0;
    int kernel_id = 0, n_kp = 0;
    double kp[4] = {0, 0, 0, 0};
    int N = 0;
    long long y0_rows = 0, ps_rows = 0;

    // plan (host copies kept for launches by level)
    std::vector<int> up_beg, dn_beg;     // task ranges per level step
    int n_up = 0, n_dn = 0, n_y1 = 0, n_blkB = 0, n_blkD = 0, n_jtN = 0, n_jtF = 0, n_asm = 0;

    // device plan
    UpTask* d_up = nullptr;
    DownTask* d_dn = nullptr;
    Y1Task* d_y1t = nullptr;
    int* d_y1_slots = nullptr;
    BlkTask* d_blkB = nullptr;
    BlkTask* d_blkD = nullptr;
    WideUnit* d_wide = nullptr;   // units of the 64-wide passes: B pass 0, B pass 1, D pass 0, D pass 1
    int n_wide[4] = {0, 0, 0, 0};
    JitTarget* d_jtN = nullptr;
    JitTarget* d_jtF = nullptr;
    JitSource* d_js = nullptr;
    AsmTask* d_asm = nullptr;
    int* d_asm_slots = nullptr;
    int* d_fwd = nullptr;
    int* d_bwd = nullptr;

    // data
    double* d_U64 = nullptr;
    float* d_U32 = nullptr;
    size_t U_elems = 0;
    double* d_B64 = nullptr;
    float* d_B32 = nullptr;
    size_t B_elems = 0;
    size_t B32_elems = 0, D32_elems = 0;   // FP32 arenas (rows padded, BlkTask)
    // per block: FP64 offset (H2Pack's packing), FP32 offset, rows, columns ([0] B, [1] D)
    struct BlkMap { long long off64, off32; int nrow, ncol; };
    std::vector<BlkMap> bmap[2];
    double* d_D64 = nullptr;
    float* d_D32 = nullptr;
    size_t D_elems = 0;
    double4* d_pts64 = nullptr;   // global coordinates (x, y, z, radius)
    float4* d_pts32 = nullptr;    // coordinates relative to their node's box center
    float4* d_pts32lo = nullptr;  // Coulomb: their low parts (coordinate - FP32 coordinate)
    size_t n_pts = 0;
    // source panels of the FP32 tensor-core JIT kernel
    PanelGroup* d_pg = nullptr;
    int n_pg = 0, n_pg_pts = 0;   // groups; groups of point sets (the rest are skeleton sets)
    float4* d_ppts = nullptr;     // 8 float4 per group: the points, paired as the B fragment holds them
    float4* d_pplo = nullptr;     // Coulomb: 6 float4 per group, the low parts of those points
    TileRec* d_tiles = nullptr;   // source tiles of every JIT target chunk
    uint4* d_pin = nullptr;       // 64 uint4 per group (NV <= 16): inputs split into TF32 hi / lo

    // work buffers sized for panels of width NVb
    int NVb = 0;
    double* d_XS = nullptr;
    double* d_PS = nullptr;
    double* d_Y1 = nullptr;
    double* d_PUSH = nullptr;
    uint16_t* d_XS3 = nullptr;   // 64-wide panels of mixed stored-block images: XS split into BF16 pieces
    // host-API staging
    double* d_io = nullptr;
    size_t io_elems = 0;

    size_t bytes = 0;        // plan + data
    size_t work_bytes = 0;   // work buffers
    h2gpu_stats st{};
    Ev ev;

    // pair plan: each unordered JIT pair evaluated once (FP32 tensor-core path)
    int has_pair = 0;
    int blk1_small[2][2] = {{0, 0}, {0, 0}};   // [B, D][FP64, FP32]: leading tasks that blk1_fits
    // FP32 far field in the difference form: some admissible pair's boxes are too close
    // for r^2 = |a|^2 + |b|^2 - 2 a.b (HSS mode: siblings are admissible and may touch)
    int far_diff = 0;
    PairOwner* d_owN = nullptr;
    PairOwner* d_owF = nullptr;
    PairPartner* d_pp = nullptr;
    JitTarget* d_jtN2 = nullptr;
    JitTarget* d_jtF2 = nullptr;
    Y1Task* d_y1t2 = nullptr;
    int* d_y1_slots2 = nullptr;
    AsmTask* d_asm2 = nullptr;
    int* d_asm_slots2 = nullptr;
    int n_owN = 0, n_owF = 0, n_jtN2 = 0, n_jtF2 = 0, n_y12 = 0, n_asm2 = 0;

    // tuning (h2gpu_autotune) and captured graph (h2gpu_graph_capture)
    int jit_tc = 1;          // tensor-core JIT kernel for FP32 panels of 8 / 16
    int jit_pair = 0;        // with jit_tc: the pair kernel (each unordered pair once)
    int blk_tc = 1;          // stored-block kernel for FP32 panels of 8 / 16: 1 mma.sync, 2 tcgen05, 0 CUDA cores
    int* d_status = nullptr; // device status word (bounded waits of the tcgen05 kernel)
    int* h_status = nullptr; // pinned host copy, read back at the end of every timed panel
    int tuned_nv = 0;        // panel width chosen by the autotuner (0: default rule)
    int gen = 0;             // stored blocks generated on the device (H2GPU_BLOCKS_GENERATE)
    int f32_only = 0;        // the stored blocks exist in FP32 only (generated for a mixed image)
    int n_images = 1;        // matrices in this image (batched images hold several)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
};

namespace {

void free_all(h2gpu_image* im)
{
    void* ptrs[] = {im->d_up, im->d_dn, im->d_y1t, im->d_y1_slots, im->d_blkB, im->d_blkD, im->d_jtN, im->d_jtF,
                    im->d_js, im->d_asm, im->d_asm_slots, im->d_fwd, im->d_bwd, im->d_U64, im->d_U32, im->d_B64,
                    im->d_B32, im->d_D64, im->d_D32, im->d_pts64, im->d_pts32, im->d_XS, im->d_PS, im->d_Y1,
                    im->d_PUSH, im->d_io, im->d_owN, im->d_owF, im->d_pp, im->d_jtN2, im->d_jtF2, im->d_y1t2,
                    im->d_y1_slots2, im->d_asm2, im->d_asm_slots2, im->d_status, im->d_pg, im->d_ppts,
                    im->d_pin, im->d_tiles, im->d_wide, im->d_XS3, im->d_pts32lo, im->d_pplo};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (im->h_status) cudaFreeHost(im->h_status);
    for (auto& e : im->ev.e)
        if (e) cudaEventDestroy(e);
    if (im->graph_exec) cudaGraphExecDestroy(im->graph_exec);
    if (im->graph) cudaGraphDestroy(im->graph);
    if (im->stream) cudaStreamDestroy(im->stream);
}

int npt_of(const h2gpu_desc* d, int n) { return d->pt_cluster[2 * n + 1] - d->pt_cluster[2 * n] + 1; }

// Structural checks of the descriptor; every index used by a kernel is checked here,
// so the device code indexes without bounds checks.
int validate(const h2gpu_desc* d, bool gen = false)
{
    REQ(d != nullptr, "descriptor is NULL");
    REQ(d->n_point > 0 && d->n_node > 0 && d->n_leaf_node > 0, "empty representation");
    REQ(d->pt_dim == 3, "pt_dim %d: only 3-D kernels are supported", d->pt_dim);
    REQ(d->krnl_dim == 1 || d->krnl_dim == 3, "krnl_dim %d not supported", d->krnl_dim);
    REQ(d->xpt_dim >= 3 && d->xpt_dim <= 4, "xpt_dim %d not supported", d->xpt_dim);
    REQ(d->max_child == 8, "max_child must be 8 for 3-D trees");
    REQ(d->max_level >= 0 && d->min_adm_level >= 0, "bad level data");
    REQ((long long) d->krnl_dim * d->n_point < (1LL << 30), "problem too large for 32-bit row indices");
    REQ(d->n_child && d->children && d->node_level && d->pt_cluster && d->mat_cluster && d->level_n_node &&
            d->level_nodes && d->leaf_nodes && d->U_nrow && d->U_ncol && d->U_ld && d->U && d->fwd_pmt_idx &&
            d->bwd_pmt_idx,
        "descriptor is missing a required array");
    REQ(d->n_r_adm_pair == 0 || d->r_adm_pairs, "r_adm_pairs missing");
    REQ(d->n_r_inadm_pair == 0 || d->r_inadm_pairs, "r_inadm_pairs missing");
    REQ(d->n_D == d->n_leaf_node + d->n_r_inadm_pair, "n_D != n_leaf_node + n_r_inadm_pair");
    const int kd = d->krnl_dim;
    for (int n = 0; n < d->n_node; n++)
    {
        int s = d->pt_cluster[2 * n], e = d->pt_cluster[2 * n + 1];
        REQ(s >= 0 && e < d->n_point && s <= e, "node %d: bad pt_cluster [%d, %d]", n, s, e);
        REQ(d->mat_cluster[2 * n] == kd * s && d->mat_cluster[2 * n + 1] == kd * (e + 1) - 1,
            "node %d: mat_cluster does not match pt_cluster", n);
        REQ(d->n_child[n] >= 0 && d->n_child[n] <= d->max_child, "node %d: bad n_child", n);
        for (int k = 0; k < d->n_child[n]; k++)
        {
            int c = d->children[n * d->max_child + k];
            REQ(c >= 0 && c < d->n_node && c != n, "node %d: bad child index", n);
        }
        REQ(d->node_level[n] >= 0 && d->node_level[n] <= d->max_level, "node %d: bad level", n);
        REQ(d->U_nrow[n] >= 0 && d->U_ncol[n] >= 0, "node %d: negative U size", n);
        if (d->U_nrow[n] > 0 && d->U_ncol[n] > 0)
            REQ(d->U[n] != nullptr && d->U_ld[n] >= d->U_ncol[n], "node %d: U data missing", n);
    }
    for (int l = 0; l <= d->max_level; l++)
    {
        REQ(d->level_n_node[l] >= 0 && d->level_n_node[l] <= d->n_leaf_node, "level %d: bad node count", l);
        for (int j = 0; j < d->level_n_node[l]; j++)
        {
            int n = d->level_nodes[(size_t) l * d->n_leaf_node + j];
            REQ(n >= 0 && n < d->n_node && d->node_level[n] == l, "level %d: bad node list", l);
        }
    }
    for (int i = 0; i < d->n_leaf_node; i++)
    {
        int n = d->leaf_nodes[i];
        REQ(n >= 0 && n < d->n_node && d->n_child[n] == 0, "leaf_nodes[%d] is not a leaf", i);
    }
    for (int i = 0; i < d->n_r_adm_pair; i++)
    {
        int a = d->r_adm_pairs[2 * i], b = d->r_adm_pairs[2 * i + 1];
        REQ(a >= 0 && a < d->n_node && b >= 0 && b < d->n_node && a != b, "admissible pair %d out of range", i);
    }
    for (int i = 0; i < d->n_r_inadm_pair; i++)
    {
        int a = d->r_inadm_pairs[2 * i], b = d->r_inadm_pairs[2 * i + 1];
        REQ(a >= 0 && a < d->n_node && b >= 0 && b < d->n_node, "inadmissible pair %d out of range", i);
        REQ(d->n_child[a] == 0 && d->n_child[b] == 0, "inadmissible pair %d is not leaf-leaf", i);
    }
    const int N = kd * d->n_point;
    std::vector<char> seen(N, 0);
    for (int i = 0; i < N; i++)
    {
        int f = d->fwd_pmt_idx[i], b = d->bwd_pmt_idx[i];
        REQ(f >= 0 && f < N && b >= 0 && b < N, "permutation index out of range");
        REQ(!seen[f], "fwd_pmt_idx is not a permutation");
        seen[f] = 1;
        REQ(d->bwd_pmt_idx[f] == i, "bwd_pmt_idx is not the inverse of fwd_pmt_idx");
    }
    if (d->BD_JIT)
    {
        REQ(d->kernel_id >= H2GPU_KRNL_COULOMB && d->kernel_id <= H2GPU_KRNL_RPY,
            "JIT mode needs a kernel id (H2GPU_KRNL_*), got %d", d->kernel_id);
        REQ((d->kernel_id == H2GPU_KRNL_RPY) == (kd == 3), "kernel id does not match krnl_dim");
        REQ(d->kernel_id != H2GPU_KRNL_RPY || d->xpt_dim == 4, "RPY needs 4 coordinate rows");
        REQ(d->kernel_id == H2GPU_KRNL_COULOMB || d->n_krnl_param >= 1, "kernel needs a parameter");
        REQ(d->coord && d->J_n && d->J_coord, "JIT mode needs coordinates and skeleton points");
    } else {
        REQ(d->n_B == d->n_r_adm_pair, "n_B != n_r_adm_pair");
        REQ(d->n_B == 0 || (d->B_nrow && d->B_ncol && d->B_ptr && (gen || d->B_data)), "AOT mode needs B blocks");
        REQ(d->D_nrow && d->D_ncol && d->D_ptr && (gen || d->D_data), "AOT mode needs D blocks");
    }
    if (gen)
    {
        // the blocks are generated from the kernel, the points and the skeleton points
        REQ(d->kernel_id >= H2GPU_KRNL_COULOMB && d->kernel_id <= H2GPU_KRNL_RPY,
            "generated blocks need a kernel id (H2GPU_KRNL_*), got %d", d->kernel_id);
        REQ((d->kernel_id == H2GPU_KRNL_RPY) == (kd == 3), "kernel id does not match krnl_dim");
        REQ(d->kernel_id != H2GPU_KRNL_RPY || d->xpt_dim == 4, "RPY needs 4 coordinate rows");
        REQ(d->kernel_id == H2GPU_KRNL_COULOMB || d->n_krnl_param >= 1, "kernel needs a parameter");
        REQ(d->coord && d->J_n && d->J_coord, "generated blocks need coordinates and skeleton points");
    }
    return H2GPU_OK;
}

// Center of the bounding box of every node's points.
void node_centers(const h2gpu_desc* d, std::vector<double>& c, std::vector<double>* half = nullptr)
{
    c.assign(3 * (size_t) d->n_node, 0.0);
    if (half) half->assign(3 * (size_t) d->n_node, 0.0);
    for (int n = 0; n < d->n_node; n++)
    {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int p = d->pt_cluster[2 * n]; p <= d->pt_cluster[2 * n + 1]; p++)
            for (int k = 0; k < 3; k++)
            {
                double x = d->coord[(size_t) k * d->n_point + p];
                lo[k] = std::min(lo[k], x);
                hi[k] = std::max(hi[k], x);
            }
        for (int k = 0; k < 3; k++) c[3 * n + k] = 0.5 * (lo[k] + hi[k]);
        if (half)
            for (int k = 0; k < 3; k++) (*half)[3 * n + k] = 0.5 * std::max(0.0, hi[k] - lo[k]);
    }
    // Centers on a grid of 2^(e - 21) with 2^e >= max |center|: every center is an
    // integer multiple of the quantum below 2^21 in magnitude, so the difference of two
    // centers (a frame shift) is exact in FP32.  Moving a frame's origin by less than
    // a quantum changes nothing else.
    double m = 0.0;
    for (double v : c) m = std::max(m, std::fabs(v));
    if (m > 0.0)
    {
        int e = 0;
        std::frexp(m, &e);   // m < 2^e
        const double q = std::ldexp(1.0, e - 21);
        for (double& v : c) v = std::nearbyint(v / q) * q;
    }
}

// Everything build_plan produces on the host; uploaded by upload_plan once a device is known.
// points of an owner set per pair-plan work unit (one CTA's rows)
constexpr int kPairOwnerChunk = 128;

struct HostPlan {
    std::vector<double> U;
    std::vector<UpTask> up;
    std::vector<DownTask> dn;
    std::vector<Y1Task> y1t;
    std::vector<int> y1_slots;
    std::vector<BlkTask> blkB, blkD;
    std::vector<WideUnit> wide;   // B pass 0, B pass 1, D pass 0, D pass 1 (counts in n_wide)
    std::vector<JitTarget> jtN, jtF;
    std::vector<JitSource> js;
    std::vector<AsmTask> at;
    std::vector<int> at_slots;
    std::vector<int> fw, bw;
    std::vector<double4> p64;
    std::vector<float4> p32;
    std::vector<float4> p32lo;    // Coulomb only
    // pair plan (FP32 tensor-core path of scalar JIT kernels)
    std::vector<PairOwner> owN, owF;
    std::vector<PairPartner> partners;
    std::vector<JitTarget> jtN2, jtF2;
    std::vector<Y1Task> y1t2;
    std::vector<int> y1_slots2;
    std::vector<AsmTask> at2;
    std::vector<int> at_slots2;
    // source panels: groups of the point sets first (filled after the gather), then
    // those of the skeleton sets (filled after the upward sweep)
    std::vector<PanelGroup> pg;
    int pg_pts = 0;
    std::vector<TileRec> tiles;
};

// FP32 arena offsets of n blocks stored one after the other with rows of f32_ld(ncol)
// elements (every offset a multiple of 4); returns the arena's element count
long long pack_f32(int n, const int* nrow, const int* ncol, std::vector<long long>& off)
{
    off.assign(n, 0);
    long long e = 0;
    for (int i = 0; i < n; i++)
    {
        off[i] = e;
        e += (long long) nrow[i] * f32_ld(ncol[i]);
    }
    return e;
}

int build_plan(h2gpu_image* im, const h2gpu_desc* d, HostPlan& hp)
{
    const int kd = d->krnl_dim, N = kd * d->n_point, n_node = d->n_node, min_adm = d->min_adm_level;
    const int* lvl = d->node_level;
    const int* mc = d->mat_cluster;
    im->n_point = d->n_point; im->kd = kd; im->xpt_dim = d->xpt_dim; im->n_node = n_node;
    im->n_leaf = d->n_leaf_node; im->max_level = d->max_level; im->min_adm = min_adm; im->BD_JIT = d->BD_JIT;
    im->kernel_id = d->kernel_id; im->n_kp = d->n_krnl_param; im->N = N;
    for (int i = 0; i < 4; i++) im->kp[i] = d->krnl_param[i];

    // ---- parents, and the y0 layout with each node's children contiguous
    std::vector<int> parent(n_node, -1);
    for (int n = 0; n < n_node; n++)
        for (int k = 0; k < d->n_child[n]; k++) parent[d->children[n * d->max_child + k]] = n;
    std::vector<int> y0r(n_node, -1);
    long long cur = 0;
    for (int p = 0; p < n_node; p++)
        for (int k = 0; k < d->n_child[p]; k++)
        {
            int c = d->children[p * d->max_child + k];
            if (lvl[c] >= min_adm) { y0r[c] = (int) cur; cur += d->U_ncol[c]; }
        }
    for (int n = 0; n < n_node; n++)
        if (parent[n] < 0 && lvl[n] >= min_adm) { y0r[n] = (int) cur; cur += d->U_ncol[n]; }
    REQ(cur < (1LL << 30), "skeleton space too large");
    im->y0_rows = cur;

    // ---- U shapes and arena
    std::vector<long long> u_off(n_node, 0);
    long long ue = 0;
    for (int n = 0; n < n_node; n++)
    {
        int nr = d->U_nrow[n], nc = d->U_ncol[n];
        if (nr == 0 || nc == 0 || lvl[n] < min_adm) continue;
        if (d->n_child[n] == 0)
            REQ(nr == kd * npt_of(d, n), "leaf %d: U has %d rows, expected %d", n, nr, kd * npt_of(d, n));
        else
        {
            int s = 0;
            for (int k = 0; k < d->n_child[n]; k++) s += d->U_ncol[d->children[n * d->max_child + k]];
            REQ(nr == s, "node %d: U has %d rows, children ranks sum to %d", n, nr, s);
        }
        u_off[n] = ue;                                  // a multiple of 4: every stride is
        ue += (long long) nr * ((nc + 3) & ~3);
    }
    std::vector<double>& U = hp.U;
    U.assign(ue, 0.0);                                  // zero padding
    for (int n = 0; n < n_node; n++)
    {
        int nr = d->U_nrow[n], nc = d->U_ncol[n], ld = d->U_ld[n];
        if (nr == 0 || nc == 0 || lvl[n] < min_adm) continue;
        const int ld4 = (nc + 3) & ~3;
        for (int r = 0; r < nr; r++) memcpy(&U[u_off[n] + (long long) r * ld4], d->U[n] + (size_t) r * ld, 8 * nc);
    }
    im->U_elems = ue;

    // ---- upward tasks, levels max_level .. min_adm
    std::vector<UpTask>& up = hp.up;
    im->up_beg.clear();
    for (int L = d->max_level; L >= min_adm; L--)
    {
        im->up_beg.push_back((int) up.size());
        for (int j = 0; j < d->level_n_node[L]; j++)
        {
            int n = d->level_nodes[(size_t) L * d->n_leaf_node + j];
            int nr = d->U_nrow[n], nc = d->U_ncol[n];
            if (nr == 0 || nc == 0) continue;
            for (int c0 = 0; c0 < nc; c0 += 64)
            {
                UpTask t;
                t.u_off = u_off[n];
                t.nrow = nr;
                t.ld = (nc + 3) & ~3;
                t.c0 = c0;
                t.nc = std::min(64, nc - c0);
                t.in_row = d->n_child[n] == 0 ? mc[2 * n] : N + y0r[d->children[n * d->max_child]];
                t.out_row = N + y0r[n];
                up.push_back(t);
            }
        }
    }
    im->up_beg.push_back((int) up.size());
    im->n_up = (int) up.size();

    // ---- partial slots
    long long ps = 0;
    auto alloc = [&](int rows) { long long r = ps; ps += rows; return (int) r; };
    std::vector<std::vector<int>> y1s(n_node), asms(n_node);
    // pair plan slots of a node: (slot, first row) -- a slot of the node's full size
    // (first row -1), or one of an owner unit covering rows [first row, + 128) of it
    std::vector<std::vector<std::pair<int, int>>> pair_y1, pair_asm;
    std::vector<char> has_y1(n_node, 0);
    // Stored blocks: one task per block of up to RB rows (larger blocks split evenly
    // into tasks of a multiple of 64 rows).  A task's kernel walks its rows in chunks
    // of 64 and adds the chunks' transposed products into the task's single slot, so
    // a block has one A^T w slot per task instead of one per 64-row chunk.
    const int RB = 1024;
    auto rows_per_task = [&](int nr) {
        const int nt = (nr + RB - 1) / RB;
        return ((nr + nt - 1) / nt + 63) / 64 * 64;
    };
    std::vector<BlkTask>& blkB = hp.blkB;
    std::vector<BlkTask>& blkD = hp.blkD;
    std::vector<JitTarget>& jtN = hp.jtN;
    std::vector<JitTarget>& jtF = hp.jtF;
    std::vector<JitSource>& js = hp.js;
    std::vector<double> ctr;

    if (!d->BD_JIT)
    {
        std::vector<long long> off32B, off32D;
        im->B32_elems = (size_t) pack_f32(d->n_B, d->B_nrow, d->B_ncol, off32B);
        im->D32_elems = (size_t) pack_f32(d->n_D, d->D_nrow, d->D_ncol, off32D);
        for (int k = 0; k < 2; k++) im->bmap[k].clear();
        for (int i = 0; i < d->n_B; i++)
            im->bmap[0].push_back({(long long) d->B_ptr[i], off32B[i], d->B_nrow[i], d->B_ncol[i]});
        for (int i = 0; i < d->n_D; i++)
            im->bmap[1].push_back({(long long) d->D_ptr[i], off32D[i], d->D_nrow[i], d->D_ncol[i]});
        for (int i = 0; i < d->n_B; i++)
        {
            int n0 = d->r_adm_pairs[2 * i], n1 = d->r_adm_pairs[2 * i + 1];
            int l0 = lvl[n0], l1 = lvl[n1];
            int nr = d->B_nrow[i], nc = d->B_ncol[i];
            int er = (l0 >= l1) ? d->U_ncol[n0] : kd * npt_of(d, n0);
            int ec = (l1 >= l0) ? d->U_ncol[n1] : kd * npt_of(d, n1);
            REQ(nr == er && nc == ec, "B block %d is %dx%d, expected %dx%d", i, nr, nc, er, ec);
            REQ(l0 < l1 || (l0 >= min_adm && y0r[n0] >= 0), "B block %d: node %d has no skeleton", i, n0);
            REQ(l1 < l0 || (l1 >= min_adm && y0r[n1] >= 0), "B block %d: node %d has no skeleton", i, n1);
            if (nr == 0 || nc == 0) continue;
            int in0 = (l0 > l1) ? mc[2 * n1] : N + y0r[n1];
            int in1 = (l0 < l1) ? mc[2 * n0] : N + y0r[n0];
            int s0 = alloc(nr);
            if (l0 < l1) asms[n0].push_back(s0); else { y1s[n0].push_back(s0); }
            const int R = rows_per_task(nr);
            for (int r0 = 0; r0 < nr; r0 += R)
            {
                int rr = std::min(R, nr - r0);
                int s1 = alloc(nc);
                if (l0 > l1) asms[n1].push_back(s1); else y1s[n1].push_back(s1);
                BlkTask t;
                t.a_off = (long long) d->B_ptr[i] + (long long) r0 * nc;
                t.nrow = rr; t.ncol = nc; t.in0_row = in0; t.in1_row = in1 + r0;
                t.out0_row = s0 + r0; t.out1_row = s1;
                t.ld32 = f32_ld(nc); t.a32 = off32B[i] + (long long) r0 * t.ld32; t.pad = 0;
                blkB.push_back(t);
            }
        }
        for (int i = 0; i < d->n_D; i++)
        {
            int n0, n1;
            if (i < d->n_leaf_node) n0 = n1 = d->leaf_nodes[i];
            else { n0 = d->r_inadm_pairs[2 * (i - d->n_leaf_node)]; n1 = d->r_inadm_pairs[2 * (i - d->n_leaf_node) + 1]; }
            int nr = d->D_nrow[i], nc = d->D_ncol[i];
            REQ(nr == kd * npt_of(d, n0) && nc == kd * npt_of(d, n1), "D block %d has a wrong shape", i);
            bool diag = i < d->n_leaf_node;
            int s0 = alloc(nr);
            asms[n0].push_back(s0);
            const int R = rows_per_task(nr);
            for (int r0 = 0; r0 < nr; r0 += R)
            {
                int rr = std::min(R, nr - r0);
                int s1 = -1;
                if (!diag) { s1 = alloc(nc); asms[n1].push_back(s1); }
                BlkTask t;
                t.a_off = (long long) d->D_ptr[i] + (long long) r0 * nc;
                t.nrow = rr; t.ncol = nc; t.in0_row = mc[2 * n1]; t.in1_row = mc[2 * n0] + r0;
                t.out0_row = s0 + r0; t.out1_row = s1;
                t.ld32 = f32_ld(nc); t.a32 = off32D[i] + (long long) r0 * t.ld32; t.pad = 0;
                blkD.push_back(t);
            }
        }
        for (int n = 0; n < n_node; n++) has_y1[n] = !y1s[n].empty();
        // one-RHS kernel (k_blk1): tasks one warp takes first, those within the FP64
        // limit before those within the FP32 limit only; stable, so the tasks of one row
        // node stay adjacent within a class (the outputs do not depend on task order)
        for (int li = 0; li < 2; li++)
        {
            std::vector<BlkTask>& ts = li == 0 ? blkB : blkD;
            auto cls = [](const BlkTask& t) {
                return blk1_fits(t.nrow, t.ncol, 8) ? 0 : (blk1_fits(t.nrow, t.ncol, 4) ? 1 : 2);
            };
            std::stable_sort(ts.begin(), ts.end(), [&](const BlkTask& a, const BlkTask& b) { return cls(a) < cls(b); });
            int n64 = 0, n32 = 0;
            for (const BlkTask& t : ts)
            {
                n64 += cls(t) == 0;
                n32 += cls(t) <= 1;
            }
            im->blk1_small[li][0] = n64;
            im->blk1_small[li][1] = n32;
        }
        // units of the 64-wide passes: pass 0 per 64-row chunk of a task (A V), pass 1 per
        // 64-column tile of a task (A^T W)
        // Pass-0 units are ordered by their input rows (the column node's y0 / x slice),
        // so that consecutive units, walked by the persistent CTAs in order, read the same
        // 64-wide input rows from L2; pass-1 units read their task's own rows and keep the
        // task order (tasks of one row node are adjacent).
        auto units = [&](const std::vector<BlkTask>& ts, int pass) {
            std::vector<WideUnit> us;
            for (int i = 0; i < (int) ts.size(); i++)
            {
                const BlkTask& t = ts[i];
                if ((pass == 0 ? t.out0_row : t.out1_row) < 0) continue;
                for (int o = 0; o < (pass == 0 ? t.nrow : t.ncol); o += 64) us.push_back(WideUnit{i, o});
            }
            if (pass == 0)
                std::stable_sort(us.begin(), us.end(), [&](const WideUnit& a, const WideUnit& b) {
                    return ts[a.task].in0_row < ts[b.task].in0_row;
                });
            hp.wide.insert(hp.wide.end(), us.begin(), us.end());
            return (int) us.size();
        };
        im->n_wide[0] = units(blkB, 0);
        im->n_wide[1] = units(blkB, 1);
        im->n_wide[2] = units(blkD, 0);
        im->n_wide[3] = units(blkD, 1);
    } else {
        // ---- JIT: point space = sorted points, then the skeleton points of every node
        std::vector<double> half;
        node_centers(d, ctr, &half);
        // The FP32 far field forms r^2 = |a|^2 + |b|^2 - 2 a.b in the source box's frame;
        // its rounding error relative to r^2 is a few eps times
        // F = (max |a|^2 + max |b|^2) / min r^2, with |b| <= the source box's half-diagonal,
        // |a| <= the center distance + the target box's, r >= the gap between the boxes.
        // H2Pack's admissibility (a gap of one box width) keeps F near 10, or ~30 with
        // pairs two levels apart; touching boxes (HSS mode: every sibling pair is
        // admissible) make it unbounded.  Any pair with F > 64, in either direction,
        // switches the image's FP32 far field to the difference form.
        im->far_diff = 0;
        for (int i = 0; i < d->n_r_adm_pair && !im->far_diff; i++)
        {
            const int a = d->r_adm_pairs[2 * i], b = d->r_adm_pairs[2 * i + 1];
            double gap2 = 0.0, dc2 = 0.0, ha2 = 0.0, hb2 = 0.0;
            for (int k = 0; k < 3; k++)
            {
                const double dc = std::fabs(ctr[3 * a + k] - ctr[3 * b + k]);
                const double g = dc - half[3 * a + k] - half[3 * b + k];
                if (g > 0.0) gap2 += g * g;
                dc2 += dc * dc;
                ha2 += half[3 * a + k] * half[3 * a + k];
                hb2 += half[3 * b + k] * half[3 * b + k];
            }
            const double dcn = std::sqrt(dc2), ha = std::sqrt(ha2), hb = std::sqrt(hb2);
            const double num = std::max((dcn + ha) * (dcn + ha) + hb2, (dcn + hb) * (dcn + hb) + ha2);
            if (!(num <= 64.0 * gap2)) im->far_diff = 1;
        }
        std::vector<int> jp0(n_node, 0);
        long long np = d->n_point;
        for (int n = 0; n < n_node; n++) { jp0[n] = (int) np; np += d->J_n[n]; }
        REQ(np < (1LL << 31), "too many points");
        im->n_pts = np;
        std::vector<int> leaf_of(d->n_point, -1);
        for (int i = 0; i < d->n_leaf_node; i++)
        {
            int n = d->leaf_nodes[i];
            for (int p = d->pt_cluster[2 * n]; p <= d->pt_cluster[2 * n + 1]; p++) leaf_of[p] = n;
        }
        std::vector<double4>& p64 = hp.p64;
        std::vector<float4>& p32 = hp.p32;
        p64.resize(np);
        p32.resize(np);
        const bool rad = d->xpt_dim >= 4;
        // Coulomb (singular at r = 0): the FP32 near field forms differences from hi + lo
        // coordinates, so nearby points keep their relative distance accuracy
        const bool lo_parts = d->kernel_id == H2GPU_KRNL_COULOMB;
        if (lo_parts) hp.p32lo.resize(np);
        auto rel32 = [&](size_t p, double x, double y, double z, double a, const double* c) {
            const double rx = x - c[0], ry = y - c[1], rz = z - c[2];
            p32[p] = make_float4((float) rx, (float) ry, (float) rz, (float) a);
            if (lo_parts)
                hp.p32lo[p] = make_float4((float) (rx - (double) p32[p].x), (float) (ry - (double) p32[p].y),
                                          (float) (rz - (double) p32[p].z), 0.f);
        };
        for (int p = 0; p < d->n_point; p++)
        {
            double x = d->coord[p], y = d->coord[(size_t) d->n_point + p], z = d->coord[2 * (size_t) d->n_point + p];
            double a = rad ? d->coord[3 * (size_t) d->n_point + p] : 0.0;
            REQ(leaf_of[p] >= 0, "point %d belongs to no leaf", p);
            const double* c = &ctr[3 * leaf_of[p]];
            p64[p] = make_double4(x, y, z, a);
            rel32(p, x, y, z, a, c);
        }
        for (int n = 0; n < n_node; n++)
        {
            int nj = d->J_n[n];
            if (nj > 0) REQ(d->J_coord[n] != nullptr, "node %d: skeleton coordinates missing", n);
            const double* c = &ctr[3 * n];
            for (int j = 0; j < nj; j++)
            {
                const double* J = d->J_coord[n];
                double x = J[j], y = J[nj + j], z = J[2 * nj + j], a = rad ? J[3 * nj + j] : 0.0;
                p64[jp0[n] + j] = make_double4(x, y, z, a);
                rel32(jp0[n] + j, x, y, z, a, c);
            }
        }

        struct Src { int pt0, npt, in_row, node; };
        // distinct source sets (point-space range), numbered in order of first use
        std::map<std::pair<int, int>, int> set_id;
        std::vector<Src> sets;
        auto shift = [&](int tn, int sn, JitSource& s) {
            s.sx = (float) (ctr[3 * tn] - ctr[3 * sn]);
            s.sy = (float) (ctr[3 * tn + 1] - ctr[3 * sn + 1]);
            s.sz = (float) (ctr[3 * tn + 2] - ctr[3 * sn + 2]);
        };
        const int TCH = 128;
        auto emit = [&](std::vector<JitTarget>& out, int tnode, int pt0, int npt, int out_row, int out_y1,
                        const std::vector<Src>& srcs) {
            int sb = (int) js.size();
            for (const Src& s : srcs)
            {
                JitSource j;
                j.pt0 = s.pt0; j.npt = s.npt; j.in_row = s.in_row;
                shift(tnode, s.node, j);
                auto ins = set_id.emplace(std::make_pair(s.pt0, s.npt), (int) sets.size());
                if (ins.second) sets.push_back(s);
                j.grp = ins.first->second;   // set number until the panel layout is known
                js.push_back(j);
            }
            int se = (int) js.size();
            for (int c0 = 0; c0 < npt; c0 += TCH)
            {
                JitTarget t;
                t.pt0 = pt0 + c0; t.npt = std::min(TCH, npt - c0);
                t.out_row = out_row + kd * c0; t.out_y1 = out_y1;
                t.src_beg = sb; t.src_end = se;
                out.push_back(t);
            }
        };
        // near field: every leaf against itself and its inadmissible partners
        std::vector<std::vector<Src>> near(n_node), farJ(n_node), farL(n_node);
        auto pts_src = [&](int n) { return Src{d->pt_cluster[2 * n], npt_of(d, n), mc[2 * n], n}; };
        auto J_src = [&](int n) { return Src{jp0[n], d->J_n[n], N + y0r[n], n}; };
        for (int i = 0; i < d->n_leaf_node; i++)
        {
            int n = d->leaf_nodes[i];
            near[n].push_back(pts_src(n));
        }
        for (int i = 0; i < d->n_r_inadm_pair; i++)
        {
            int a = d->r_inadm_pairs[2 * i], b = d->r_inadm_pairs[2 * i + 1];
            near[a].push_back(pts_src(b));
            near[b].push_back(pts_src(a));
        }
        for (int i = 0; i < d->n_r_adm_pair; i++)
        {
            int a = d->r_adm_pairs[2 * i], b = d->r_adm_pairs[2 * i + 1];
            int la = lvl[a], lb = lvl[b];
            if (la >= lb) REQ(y0r[a] >= 0 && d->U_ncol[a] == kd * d->J_n[a], "node %d: skeleton size mismatch", a);
            if (lb >= la) REQ(y0r[b] >= 0 && d->U_ncol[b] == kd * d->J_n[b], "node %d: skeleton size mismatch", b);
            if (la == lb) { farJ[a].push_back(J_src(b)); farJ[b].push_back(J_src(a)); }
            else if (la > lb) { farJ[a].push_back(pts_src(b)); farL[b].push_back(J_src(a)); }
            else { farL[a].push_back(J_src(b)); farJ[b].push_back(pts_src(a)); }
        }
        for (int i = 0; i < d->n_leaf_node; i++)
        {
            int n = d->leaf_nodes[i];
            int s = alloc(kd * npt_of(d, n));
            asms[n].push_back(s);
            emit(jtN, n, d->pt_cluster[2 * n], npt_of(d, n), s, 0, near[n]);
        }
        for (int n = 0; n < n_node; n++)
        {
            if (!farJ[n].empty() && d->J_n[n] > 0)
            {
                has_y1[n] = 1;
                emit(jtF, n, jp0[n], d->J_n[n], y0r[n], 1, farJ[n]);
            }
            if (!farL[n].empty())
            {
                int s = alloc(kd * npt_of(d, n));
                asms[n].push_back(s);
                emit(jtF, n, d->pt_cluster[2 * n], npt_of(d, n), s, 0, farL[n]);
            }
        }

        // ---- pair plan for the FP32 tensor-core path of scalar kernels: every unordered
        // pair (same-level skeleton sets, and inadmissible leaf pairs) is evaluated once
        // and applied both ways; its owner accumulates its side over all its partners,
        // each partner's side goes to a slot of its own.  Diagonal leaf blocks and the
        // level-mismatched pairs stay one-sided.  Slots are disjoint from the one-sided
        // plan's, so both plans share the partial space.
        if (kd == 1)
        {
            im->has_pair = 1;
            pair_y1.assign(n_node, {});
            pair_asm.assign(n_node, {});
            std::vector<double> load(n_node, 0.0);
            std::vector<std::vector<int>> fpart(n_node), npart(n_node);
            auto choose = [&](int a, int b, double w) {
                int o = (load[a] <= load[b]) ? a : b;
                load[o] += w;
                return o;
            };
            for (int i = 0; i < d->n_r_adm_pair; i++)
            {
                int a = d->r_adm_pairs[2 * i], b = d->r_adm_pairs[2 * i + 1];
                if (lvl[a] != lvl[b] || d->J_n[a] == 0 || d->J_n[b] == 0) continue;
                int o = choose(a, b, (double) d->J_n[a] * d->J_n[b]);
                fpart[o].push_back(o == a ? b : a);
            }
            for (int i = 0; i < d->n_r_inadm_pair; i++)
            {
                int a = d->r_inadm_pairs[2 * i], b = d->r_inadm_pairs[2 * i + 1];
                int o = choose(a, b, (double) npt_of(d, a) * npt_of(d, b));
                npart[o].push_back(o == a ? b : a);
            }
            // Work units: a chunk of <= 128 points of the owner a (one CTA's rows) and a
            // run of its partners whose work na * sum(nb) stays under a cap sized for
            // about 12 units per SM (148 SMs x 3 CTAs x 4 waves), so the largest owners
            // do not leave a tail.  Every unit has its own slot for a's side and one per
            // partner for b's side.
            const int PCH = kPairOwnerChunk;
            double w_total = 0.0;
            for (int n = 0; n < n_node; n++)
            {
                for (int b : fpart[n]) w_total += (double) d->J_n[n] * d->J_n[b];
                for (int b : npart[n]) w_total += (double) npt_of(d, n) * npt_of(d, b);
            }
            const double w_cap = std::max(w_total / (148.0 * 3 * 4), 128.0 * 512.0);
            auto emit_owner = [&](std::vector<PairOwner>& out, int a, bool isJ, const std::vector<int>& parts,
                                  std::vector<std::vector<std::pair<int, int>>>& lists) {
                const int na_all = isJ ? d->J_n[a] : npt_of(d, a);
                const int pa = isJ ? jp0[a] : d->pt_cluster[2 * a];
                const int in_a = isJ ? N + y0r[a] : mc[2 * a];
                for (int c0 = 0; c0 < na_all; c0 += PCH)
                {
                    const int na = std::min(PCH, na_all - c0);
                    size_t k = 0;
                    while (k < parts.size())
                    {
                        PairOwner ow;
                        ow.na = na; ow.pa = pa + c0; ow.in_a = in_a + c0;
                        ow.out_a = alloc(na);
                        lists[a].push_back({ow.out_a, c0});
                        ow.p_beg = (int) hp.partners.size();
                        double w = 0.0;
                        do {
                            const int b = parts[k++];
                            PairPartner pp;
                            pp.pb = isJ ? jp0[b] : d->pt_cluster[2 * b];
                            pp.nb = isJ ? d->J_n[b] : npt_of(d, b);
                            pp.in_b = isJ ? N + y0r[b] : mc[2 * b];
                            pp.out_b = alloc(pp.nb);
                            lists[b].push_back({pp.out_b, -1});
                            pp.sx = (float) (ctr[3 * a] - ctr[3 * b]);
                            pp.sy = (float) (ctr[3 * a + 1] - ctr[3 * b + 1]);
                            pp.sz = (float) (ctr[3 * a + 2] - ctr[3 * b + 2]);
                            hp.partners.push_back(pp);
                            w += (double) na * pp.nb;
                        } while (k < parts.size() && w < w_cap);
                        ow.p_end = (int) hp.partners.size();
                        out.push_back(ow);
                    }
                }
            };
            for (int n = 0; n < n_node; n++)
                if (!fpart[n].empty()) emit_owner(hp.owF, n, true, fpart[n], pair_y1);
            for (int n = 0; n < n_node; n++)
                if (!npart[n].empty()) emit_owner(hp.owN, n, false, npart[n], pair_asm);
            for (int i = 0; i < d->n_leaf_node; i++)
            {
                int n = d->leaf_nodes[i];
                int s = alloc(npt_of(d, n));
                pair_asm[n].push_back({s, -1});
                emit(hp.jtN2, n, d->pt_cluster[2 * n], npt_of(d, n), s, 0, std::vector<Src>{pts_src(n)});
            }
            for (int n = 0; n < n_node; n++)
            {
                std::vector<Src> left;
                for (const Src& sr : farJ[n])
                    if (sr.pt0 < d->n_point) left.push_back(sr);   // leaf points of a coarser node
                if (!left.empty() && d->J_n[n] > 0)
                {
                    int s = alloc(d->U_ncol[n]);
                    pair_y1[n].push_back({s, -1});
                    emit(hp.jtF2, n, jp0[n], d->J_n[n], s, 0, left);
                }
                if (!farL[n].empty())
                {
                    int s = alloc(npt_of(d, n));
                    pair_asm[n].push_back({s, -1});
                    emit(hp.jtF2, n, d->pt_cluster[2 * n], npt_of(d, n), s, 0, farL[n]);
                }
            }
            auto owner_work = [&](std::vector<PairOwner>& v) {
                std::vector<std::pair<double, int>> w(v.size());
                for (size_t i = 0; i < v.size(); i++)
                {
                    double sb = 0;
                    for (int k = v[i].p_beg; k < v[i].p_end; k++) sb += hp.partners[k].nb;
                    w[i] = {-(double) v[i].na * sb, (int) i};
                }
                std::stable_sort(w.begin(), w.end());
                std::vector<PairOwner> o(v.size());
                for (size_t i = 0; i < v.size(); i++) o[i] = v[w[i].second];
                v.swap(o);
            };
            owner_work(hp.owF);
            owner_work(hp.owN);
        }

        // ---- source panels: point sets first, then skeleton sets; each set padded to
        // whole groups of 8 points
        std::vector<int> first_grp(sets.size(), 0);
        for (int pass = 0; pass < 2; pass++)
        {
            for (size_t k = 0; k < sets.size(); k++)
            {
                const Src& sr = sets[k];
                if ((sr.pt0 >= d->n_point) != (pass == 1)) continue;
                first_grp[k] = (int) hp.pg.size();
                for (int j = 0; j < sr.npt; j += 8)
                    hp.pg.push_back(PanelGroup{sr.pt0 + j, sr.in_row + j, std::min(8, sr.npt - j), 0});
            }
            if (pass == 0) hp.pg_pts = (int) hp.pg.size();
        }
        REQ(hp.pg.size() < (1u << 28), "too many source panel groups");
        for (JitSource& j : js) j.grp = first_grp[j.grp];

        // ---- source tiles (128 points) of every target chunk (chunks of one target set share them)
        std::map<std::pair<int, int>, std::pair<int, int>> tile_range;
        for (std::vector<JitTarget>* v : {&jtN, &jtF, &hp.jtN2, &hp.jtF2})
            for (JitTarget& t : *v)
            {
                auto ins = tile_range.emplace(std::make_pair(t.src_beg, t.src_end), std::make_pair(0, 0));
                if (ins.second)
                {
                    ins.first->second.first = (int) hp.tiles.size();
                    for (int k = t.src_beg; k < t.src_end; k++)
                        for (int j0 = 0; j0 < js[k].npt; j0 += 128)
                        {
                            const int nj = std::min(128, js[k].npt - j0);
                            hp.tiles.push_back(TileRec{js[k].grp + j0 / 8, (nj + 7) / 8, nj, 0, js[k].sx, js[k].sy, js[k].sz, 0.f});
                        }
                    ins.first->second.second = (int) hp.tiles.size();
                    REQ(hp.tiles.size() < (1u << 30), "too many source tiles");
                }
                t.tile_beg = ins.first->second.first;
                t.tile_end = ins.first->second.second;
            }
    }

    // ---- JIT targets, largest work first (shorter tail of the launch)
    auto by_work = [&](std::vector<JitTarget>& v) {
        std::vector<std::pair<double, int>> w(v.size());
        for (size_t i = 0; i < v.size(); i++)
        {
            double srcpts = 0;
            for (int k = v[i].src_beg; k < v[i].src_end; k++) srcpts += js[k].npt;
            w[i] = {-(double) v[i].npt * srcpts, (int) i};
        }
        std::stable_sort(w.begin(), w.end());
        std::vector<JitTarget> out(v.size());
        for (size_t i = 0; i < v.size(); i++) out[i] = v[w[i].second];
        v.swap(out);
    };
    by_work(jtN);
    by_work(jtF);
    by_work(hp.jtN2);
    by_work(hp.jtF2);

    // ---- y1 sums (AOT)
    std::vector<Y1Task>& y1t = hp.y1t;
    std::vector<int>& y1_slots = hp.y1_slots;
    for (int n = 0; n < n_node; n++)
    {
        if (y1s[n].empty()) continue;
        Y1Task t;
        t.row = y0r[n]; t.nrow = d->U_ncol[n];
        t.slot_beg = (int) y1_slots.size();
        for (int s : y1s[n]) y1_slots.push_back(s);
        t.slot_end = (int) y1_slots.size();
        y1t.push_back(t);
    }

    // ---- downward tasks, levels min_adm .. max_level
    std::vector<DownTask>& dn = hp.dn;
    std::vector<char> done(n_node, 0);
    im->dn_beg.clear();
    for (int L = min_adm; L <= d->max_level; L++)
    {
        im->dn_beg.push_back((int) dn.size());
        for (int j = 0; j < d->level_n_node[L]; j++)
        {
            int n = d->level_nodes[(size_t) L * d->n_leaf_node + j];
            int nr = d->U_nrow[n], nc = d->U_ncol[n];
            if (nr == 0 || nc == 0) continue;
            bool push = parent[n] >= 0 && lvl[parent[n]] >= min_adm && done[parent[n]];
            if (!has_y1[n] && !push) continue;
            done[n] = 1;
            bool leaf = d->n_child[n] == 0;
            int dst = leaf ? alloc(nr) : y0r[d->children[n * d->max_child]];
            if (leaf) asms[n].push_back(dst);
            if (leaf && !pair_asm.empty()) pair_asm[n].push_back({dst, -1});
            const int RD = 64;       // downward tasks: one 64-row chunk of U each
            for (int r0 = 0; r0 < nr; r0 += RD)
            {
                DownTask t;
                t.ld = (nc + 3) & ~3;
                t.u_off = u_off[n] + (long long) r0 * t.ld;
                t.nrow = std::min(RD, nr - r0); t.ncol = nc;
                t.y1_row = has_y1[n] ? y0r[n] : -1;
                t.push_row = push ? y0r[n] : -1;
                t.dst_ps = leaf ? 1 : 0;
                t.dst_row = dst + r0;
                dn.push_back(t);
            }
        }
    }
    im->dn_beg.push_back((int) dn.size());

    // ---- assembly, one task per leaf
    std::vector<AsmTask>& at = hp.at;
    std::vector<int>& at_slots = hp.at_slots;
    for (int i = 0; i < d->n_leaf_node; i++)
    {
        int n = d->leaf_nodes[i];
        AsmTask t;
        t.row0 = mc[2 * n]; t.nrow = kd * npt_of(d, n);
        t.slot_beg = (int) at_slots.size();
        for (int s : asms[n]) at_slots.push_back(s);
        t.slot_end = (int) at_slots.size();
        at.push_back(t);
    }
    if (im->has_pair)
    {
        // one sum per 128-row piece of a node: the owner units' slots of that piece and
        // the same piece of every full-size slot, in the order the slots were made
        auto pieces = [&](const std::vector<std::pair<int, int>>& ent, int rows, std::vector<int>& slots, auto&& add) {
            for (int c0 = 0; c0 < rows; c0 += kPairOwnerChunk)
            {
                const int beg = (int) slots.size();
                for (const auto& e : ent)
                    if (e.second < 0) slots.push_back(e.first + c0);
                    else if (e.second == c0) slots.push_back(e.first);
                add(c0, std::min(kPairOwnerChunk, rows - c0), beg, (int) slots.size());
            }
        };
        for (int n = 0; n < n_node; n++)
        {
            if (!has_y1[n]) continue;
            pieces(pair_y1[n], d->U_ncol[n], hp.y1_slots2, [&](int c0, int len, int b, int e) {
                hp.y1t2.push_back(Y1Task{y0r[n] + c0, len, b, e});
            });
        }
        for (int i = 0; i < d->n_leaf_node; i++)
        {
            int n = d->leaf_nodes[i];
            pieces(pair_asm[n], kd * npt_of(d, n), hp.at_slots2, [&](int c0, int len, int b, int e) {
                hp.at2.push_back(AsmTask{mc[2 * n] + c0, len, b, e});
            });
        }
        im->n_asm2 = (int) hp.at2.size();
        im->n_owN = (int) hp.owN.size(); im->n_owF = (int) hp.owF.size();
        im->n_jtN2 = (int) hp.jtN2.size(); im->n_jtF2 = (int) hp.jtF2.size(); im->n_y12 = (int) hp.y1t2.size();
    }
    REQ(ps < (1LL << 31), "partial space too large");
    im->ps_rows = ps;

    // ---- statistics of the algorithm (per right-hand side)
    double ub = 0, bb = 0, db = 0, fwd = 0, mid = 0, bwd = 0, den = 0, pB = 0, pD = 0;
    for (int n = 0; n < n_node; n++)
    {
        double nr = d->U_nrow[n], nc = d->U_ncol[n];
        if (nr == 0 || nc == 0) continue;
        ub += nr * nc;
        fwd += nr * nc + nr + nc;
    }
    bwd = fwd;
    for (int i = 0; i < d->n_r_adm_pair; i++)
    {
        int a = d->r_adm_pairs[2 * i], b = d->r_adm_pairs[2 * i + 1];
        double na = lvl[a] >= lvl[b] ? d->J_n ? d->J_n[a] : d->U_ncol[a] / kd : npt_of(d, a);
        double nb = lvl[b] >= lvl[a] ? d->J_n ? d->J_n[b] : d->U_ncol[b] / kd : npt_of(d, b);
        pB += na * nb;
        if (!d->BD_JIT)
        {
            double nr = d->B_nrow[i], nc = d->B_ncol[i];
            bb += nr * nc;
            mid += nr * nc + 2 * (nr + nc);
        }
    }
    for (int i = 0; i < d->n_D; i++)
    {
        int n0, n1;
        if (i < d->n_leaf_node) n0 = n1 = d->leaf_nodes[i];
        else { n0 = d->r_inadm_pairs[2 * (i - d->n_leaf_node)]; n1 = d->r_inadm_pairs[2 * (i - d->n_leaf_node) + 1]; }
        pD += (double) npt_of(d, n0) * npt_of(d, n1);
        double nr = kd * npt_of(d, n0), nc = kd * npt_of(d, n1);
        db += nr * nc;
        den += nr * nc + (i < d->n_leaf_node ? 1 : 2) * (nr + nc);
    }
    im->st.bytes_U = 2.0 * ub;       // element counts here, scaled by the element size at query time
    im->st.bytes_B = bb;
    im->st.bytes_D = d->BD_JIT ? 0.0 : db;
    im->st.ref_mv_bytes = 8.0 * (fwd + mid + bwd + (d->BD_JIT ? 0.0 : den));
    im->st.jit_pairs_B = pB;
    im->st.jit_pairs_D = pD;
    im->st.n_tasks_B = d->BD_JIT ? (long long) jtF.size() : (long long) blkB.size();
    im->st.n_tasks_D = d->BD_JIT ? (long long) jtN.size() : (long long) blkD.size();

    hp.fw.assign(d->fwd_pmt_idx, d->fwd_pmt_idx + N);
    hp.bw.assign(d->bwd_pmt_idx, d->bwd_pmt_idx + N);
    im->n_dn = (int) dn.size(); im->n_y1 = (int) y1t.size(); im->n_blkB = (int) blkB.size();
    im->n_blkD = (int) blkD.size(); im->n_jtN = (int) jtN.size(); im->n_jtF = (int) jtF.size(); im->n_asm = (int) at.size();
    if (!d->BD_JIT)
    {
        im->B_elems = d->n_B > 0 ? d->B_ptr[d->n_B] : 0;
        im->D_elems = d->D_ptr[d->n_D];
    }
    return H2GPU_OK;
}

// ------------------------------------------------- stored blocks generated on the device

// Point arena and generation tasks of the stored blocks (H2GPU_BLOCKS_GENERATE).  Point
// space as in JIT mode: the sorted points, then the skeleton points of every node.
// Block i of B pairs (n0, n1) = r_adm_pairs[i]: rows are the skeleton points of n0 when
// its level is not coarser than n1's, else the points of n0; columns likewise
// (src/H2Pack_build.c:818-860).  D: the diagonal blocks of the leaves in leaf_nodes
// order, then the inadmissible pairs, points against points (:1063-1110).
struct GenPlan {
    std::vector<double4> pts;
    std::vector<GenTask> tB, tD;
};

int build_gen(const h2gpu_desc* d, GenPlan& g)
{
    const int kd = d->krnl_dim, n_node = d->n_node;
    const int* lvl = d->node_level;
    std::vector<int> jp0(n_node, 0);
    long long np = d->n_point;
    for (int n = 0; n < n_node; n++) { jp0[n] = (int) np; np += d->J_n[n]; }
    REQ(np < (1LL << 31), "too many points");
    g.pts.resize(np);
    const bool rad = d->xpt_dim >= 4;
    for (int p = 0; p < d->n_point; p++)
        g.pts[p] = make_double4(d->coord[p], d->coord[(size_t) d->n_point + p], d->coord[2 * (size_t) d->n_point + p],
                                rad ? d->coord[3 * (size_t) d->n_point + p] : 0.0);
    for (int n = 0; n < n_node; n++)
    {
        const int nj = d->J_n[n];
        if (nj > 0) REQ(d->J_coord[n] != nullptr, "node %d: skeleton coordinates missing", n);
        const double* J = d->J_coord[n];
        for (int j = 0; j < nj; j++)
            g.pts[jp0[n] + j] = make_double4(J[j], J[nj + j], J[2 * nj + j], rad ? J[3 * nj + j] : 0.0);
    }
    const int GR = 16;   // row points per task
    std::vector<long long> off32B, off32D;
    pack_f32(d->n_B, d->B_nrow, d->B_ncol, off32B);
    pack_f32(d->n_D, d->D_nrow, d->D_ncol, off32D);
    auto emit = [&](std::vector<GenTask>& out, size_t off, int rp0, int nrp, int cp0, int ncp, int nrow, int ncol,
                    const char* what, int i) {
        REQ(nrow == kd * nrp && ncol == kd * ncp, "%s block %d is %dx%d, its points give %dx%d", what, i, nrow, ncol,
            kd * nrp, kd * ncp);
        const size_t total = what[0] == 'B' ? d->B_ptr[d->n_B] : d->D_ptr[d->n_D];
        REQ(off + (size_t) nrow * ncol <= total, "%s block %d lies outside the packed arena", what, i);
        for (int r0 = 0; r0 < nrp; r0 += GR)
        {
            GenTask t;
            t.a_off = (long long) off + (long long) kd * r0 * (long long) ncol;
            t.a32 = (what[0] == 'B' ? off32B[i] : off32D[i]) + (long long) kd * r0 * (long long) f32_ld(ncol);
            t.row_pt0 = rp0 + r0;
            t.nrp = std::min(GR, nrp - r0);
            t.col_pt0 = cp0;
            t.ncp = ncp;
            out.push_back(t);
        }
        return H2GPU_OK;
    };
    for (int i = 0; i < d->n_B; i++)
    {
        const int n0 = d->r_adm_pairs[2 * i], n1 = d->r_adm_pairs[2 * i + 1];
        const bool s0 = lvl[n0] >= lvl[n1], s1 = lvl[n1] >= lvl[n0];
        const int rp0 = s0 ? jp0[n0] : d->pt_cluster[2 * n0], nrp = s0 ? d->J_n[n0] : npt_of(d, n0);
        const int cp0 = s1 ? jp0[n1] : d->pt_cluster[2 * n1], ncp = s1 ? d->J_n[n1] : npt_of(d, n1);
        TRY(emit(g.tB, d->B_ptr[i], rp0, nrp, cp0, ncp, d->B_nrow[i], d->B_ncol[i], "B", i));
    }
    for (int i = 0; i < d->n_D; i++)
    {
        int n0, n1;
        if (i < d->n_leaf_node) n0 = n1 = d->leaf_nodes[i];
        else { n0 = d->r_inadm_pairs[2 * (i - d->n_leaf_node)]; n1 = d->r_inadm_pairs[2 * (i - d->n_leaf_node) + 1]; }
        TRY(emit(g.tD, d->D_ptr[i], d->pt_cluster[2 * n0], npt_of(d, n0), d->pt_cluster[2 * n1], npt_of(d, n1),
                 d->D_nrow[i], d->D_ncol[i], "D", i));
    }
    return H2GPU_OK;
}

// ------------------------------------------------------------------ plan self-check

// rows [beg, beg + n) of a space counted in cnt; false when they do not fit
bool mark_rows(std::vector<int>& cnt, long long beg, long long n)
{
    if (n < 0 || beg < 0 || beg + n > (long long) cnt.size()) return false;
    for (long long r = beg; r < beg + n; r++) cnt[r]++;
    return true;
}

// Invariants of a built plan (h2gpu_plan_check); everything is recomputed from the
// descriptor where it can be, so that the check does not restate the builder.
int check_plan(const h2gpu_image* im, const h2gpu_desc* d, const HostPlan& hp, long long* counts)
{
    const int kd = d->krnl_dim, N = kd * d->n_point, n_node = d->n_node;
    const long long Y0 = im->y0_rows, PSR = im->ps_rows;
    const int* lvl = d->node_level;

    // ---- upward: per node (keyed by its U offset) every column swept once
    std::map<long long, std::vector<int>> ucols;
    std::map<long long, std::pair<int, int>> ushape;   // U offset -> (rows, row stride)
    for (const UpTask& t : hp.up)
    {
        REQ(t.nrow >= 1 && t.ld >= 1 && t.nc >= 1 && t.nc <= 64 && t.c0 >= 0 && t.c0 % 64 == 0 && t.c0 + t.nc <= t.ld,
            "plan: upward task with a bad column tile");
        REQ(t.u_off % 4 == 0 && t.ld % 4 == 0, "plan: U not aligned for 16-byte rows");
        auto ins = ushape.emplace(t.u_off, std::make_pair(t.nrow, t.ld));
        REQ(ins.first->second == std::make_pair(t.nrow, t.ld), "plan: upward tasks of one node disagree on its U");
        std::vector<int>& c = ucols[t.u_off];
        if (c.empty()) c.assign(t.ld, 0);
        for (int j = t.c0; j < t.c0 + t.nc; j++) c[j]++;
        REQ(t.out_row >= N && (long long) t.out_row + t.c0 + t.nc <= N + Y0, "plan: upward output outside y0");
        REQ(t.in_row >= 0 && (long long) t.in_row + t.nrow <= N + Y0, "plan: upward input outside the input space");
        REQ(t.in_row >= N || (long long) t.in_row + t.nrow <= N, "plan: upward input straddles x and y0");
    }
    long long u_total = 0;
    std::map<long long, int> ucount;                   // U offset -> columns (the rest is padding)
    for (const auto& kv : ucols)
    {
        int nc = 0;
        while (nc < (int) kv.second.size() && kv.second[nc] == 1) nc++;
        for (int j = nc; j < (int) kv.second.size(); j++)
            REQ(kv.second[j] == 0 && j - nc < 3, "plan: a column of U is swept %d times upward", kv.second[j]);
        ucount[kv.first] = nc;
        u_total += (long long) ushape[kv.first].first * ushape[kv.first].second;
    }
    REQ(u_total == (long long) im->U_elems, "plan: upward tasks cover %lld of %lld U elements", u_total,
        (long long) im->U_elems);

    // ---- downward: inside a node's U, disjoint; push-down rows written once and read only when written
    std::vector<int> push(Y0, 0);
    std::vector<std::pair<long long, long long>> spans;
    for (const DownTask& t : hp.dn)
    {
        REQ(t.nrow >= 1 && t.nrow <= 64 && t.ncol >= 1, "plan: downward task with a bad shape");
        auto it = ushape.upper_bound(t.u_off);
        REQ(it != ushape.begin(), "plan: downward task before the U arena");
        --it;
        const long long base = it->first;
        const int nr = it->second.first, ld = it->second.second;
        REQ(t.ld == ld && ucount[base] == t.ncol && (t.u_off - base) % ld == 0 && (t.u_off - base) / ld + t.nrow <= nr,
            "plan: downward task outside its node's U");
        spans.push_back({t.u_off, t.u_off + (long long) t.nrow * t.ld});
        REQ(t.y1_row < 0 || (long long) t.y1_row + t.ncol <= Y0, "plan: downward y1 rows outside y0");
        REQ(t.push_row < 0 || (long long) t.push_row + t.ncol <= Y0, "plan: downward push rows outside y0");
        if (!t.dst_ps) REQ(mark_rows(push, t.dst_row, t.nrow), "plan: push-down rows outside y0");
    }
    std::sort(spans.begin(), spans.end());
    for (size_t i = 1; i < spans.size(); i++) REQ(spans[i].first >= spans[i - 1].second, "plan: two downward tasks share rows of U");
    for (int v : push) REQ(v <= 1, "plan: a push-down row is written %d times", v);
    for (const DownTask& t : hp.dn)
        if (t.push_row >= 0)
            for (int r = 0; r < t.ncol; r++) REQ(push[t.push_row + r] == 1, "plan: a push-down row is read but never written");

    // ---- partial space, y1 rows and assembly of one plan
    auto check_space = [&](const char* plan, const std::vector<std::pair<long long, long long>>& prod,
                           const std::vector<std::pair<long long, long long>>& y1w, const std::vector<AsmTask>& at,
                           const std::vector<int>& at_slots, const std::vector<Y1Task>& y1t,
                           const std::vector<int>& y1_slots) -> int {
        std::vector<int> w(PSR, 0), r(PSR, 0), y1(Y0, 0), out(N, 0);
        for (const auto& p : prod) REQ(mark_rows(w, p.first, p.second), "plan (%s): a slot lies outside the partial space", plan);
        for (const AsmTask& t : at)
        {
            REQ(mark_rows(out, t.row0, t.nrow), "plan (%s): assembly rows outside the output", plan);
            for (int k = t.slot_beg; k < t.slot_end; k++)
                REQ(mark_rows(r, at_slots[k], t.nrow), "plan (%s): an assembly slot lies outside the partial space", plan);
        }
        for (const Y1Task& t : y1t)
        {
            REQ(mark_rows(y1, t.row, t.nrow), "plan (%s): y1 sum rows outside y0", plan);
            for (int k = t.slot_beg; k < t.slot_end; k++)
                REQ(mark_rows(r, y1_slots[k], t.nrow), "plan (%s): a y1 slot lies outside the partial space", plan);
        }
        for (const auto& p : y1w) REQ(mark_rows(y1, p.first, p.second), "plan (%s): y1 rows outside y0", plan);
        for (long long i = 0; i < PSR; i++)
            REQ(w[i] == r[i] && w[i] <= 1, "plan (%s): partial row %lld written %d times, summed %d times", plan, i, w[i], r[i]);
        for (int v : out) REQ(v == 1, "plan (%s): an output row is assembled %d times", plan, v);
        for (int v : y1) REQ(v <= 1, "plan (%s): a y1 row is written %d times", plan, v);
        for (const DownTask& t : hp.dn)
            if (t.y1_row >= 0)
                for (int k = 0; k < t.ncol; k++) REQ(y1[t.y1_row + k] == 1, "plan (%s): a y1 row is read but never written", plan);
        return H2GPU_OK;
    };
    std::vector<std::pair<long long, long long>> down_ps;
    for (const DownTask& t : hp.dn)
        if (t.dst_ps) down_ps.push_back({t.dst_row, t.nrow});
    std::vector<std::pair<long long, long long>> prod = down_ps, y1w;
    for (const std::vector<BlkTask>* v : {&hp.blkB, &hp.blkD})
        for (const BlkTask& t : *v)
        {
            REQ(t.nrow >= 1 && t.ncol >= 1, "plan: stored-block task with a bad shape");
            const long long elems = (long long) (v == &hp.blkB ? im->B_elems : im->D_elems);
            REQ(t.a_off >= 0 && t.a_off + (long long) t.nrow * t.ncol <= elems, "plan: stored-block task outside its arena");
            const long long elems32 = (long long) (v == &hp.blkB ? im->B32_elems : im->D32_elems);
            REQ(t.ld32 == f32_ld(t.ncol) && t.a32 >= 0 && t.a32 % 4 == 0 && t.a32 + (long long) t.nrow * t.ld32 <= elems32,
                "plan: stored-block task outside its FP32 arena");
            REQ(t.in0_row >= 0 && (long long) t.in0_row + t.ncol <= N + Y0, "plan: stored-block input outside the input space");
            REQ(t.in1_row >= 0 && (long long) t.in1_row + t.nrow <= N + Y0, "plan: stored-block input outside the input space");
            if (t.out0_row >= 0) prod.push_back({t.out0_row, t.nrow});
            if (t.out1_row >= 0) prod.push_back({t.out1_row, t.ncol});
        }
    // the one-RHS kernel gives the leading blk1_small tasks of a list one warp each
    for (int li = 0; li < 2; li++)
    {
        const std::vector<BlkTask>& ts = li == 0 ? hp.blkB : hp.blkD;
        for (int pi = 0; pi < 2; pi++)
        {
            const int ns = im->blk1_small[li][pi];
            REQ(ns >= 0 && ns <= (int) ts.size(), "plan: bad count of one-warp stored-block tasks");
            for (int i = 0; i < ns; i++)
                REQ(blk1_fits(ts[i].nrow, ts[i].ncol, pi == 0 ? 8 : 4), "plan: one-warp stored-block task too large");
        }
    }
    for (const std::vector<JitTarget>* v : {&hp.jtN, &hp.jtF})
        for (const JitTarget& t : *v) (t.out_y1 ? y1w : prod).push_back({t.out_row, (long long) kd * t.npt});
    TRY(check_space("one-sided", prod, y1w, hp.at, hp.at_slots, hp.y1t, hp.y1_slots));

    // ---- stored blocks: the tasks of every B / D block cover its rows once, at its width
    if (!d->BD_JIT)
    {
        auto cover_blocks = [&](const char* which, const std::vector<BlkTask>& tasks, int nb, const int* nrow,
                                const int* ncol, const size_t* ptr) -> int {
            std::vector<std::vector<char>> rows(nb);
            for (const BlkTask& t : tasks)
            {
                const size_t* it = std::upper_bound(ptr, ptr + nb + 1, (size_t) t.a_off);
                const int i = (int) (it - ptr) - 1;
                REQ(i >= 0 && i < nb && ncol[i] == t.ncol && ((long long) t.a_off - (long long) ptr[i]) % t.ncol == 0,
                    "plan: a %s task does not start on a row of its block", which);
                const long long r0 = ((long long) t.a_off - (long long) ptr[i]) / t.ncol;
                REQ(r0 + t.nrow <= nrow[i], "plan: a %s task runs past its block", which);
                if (rows[i].empty()) rows[i].assign(nrow[i], 0);
                for (long long r = r0; r < r0 + t.nrow; r++) REQ(++rows[i][r] == 1, "plan: a row of %s block %d is covered twice", which, i);
            }
            for (int i = 0; i < nb; i++)
                if (nrow[i] > 0 && ncol[i] > 0)
                    REQ(!rows[i].empty() && std::count(rows[i].begin(), rows[i].end(), 1) == nrow[i],
                        "plan: %s block %d is not covered by its tasks", which, i);
            return H2GPU_OK;
        };
        TRY(cover_blocks("B", hp.blkB, d->n_B, d->B_nrow, d->B_ncol, d->B_ptr));
        TRY(cover_blocks("D", hp.blkD, d->n_D, d->D_nrow, d->D_ncol, d->D_ptr));
        // ---- units of the 64-wide passes: every 64-row chunk (pass 0) and every 64-column
        //      tile (pass 1) of every task that has the product, once each
        long long w0 = 0;
        const int* nw = im->n_wide;
        REQ((long long) hp.wide.size() == (long long) nw[0] + nw[1] + nw[2] + nw[3], "plan: wide unit counts");
        for (int part = 0; part < 4; part++)
        {
            const std::vector<BlkTask>& ts = part < 2 ? hp.blkB : hp.blkD;
            const int pass = part & 1;
            std::vector<std::vector<char>> seen(ts.size());
            for (long long k = w0; k < w0 + nw[part]; k++)
            {
                const WideUnit u = hp.wide[k];
                REQ(u.task >= 0 && u.task < (int) ts.size(), "plan: a wide unit names no task");
                const BlkTask& t = ts[u.task];
                const int ext = pass == 0 ? t.nrow : t.ncol;
                REQ((pass == 0 ? t.out0_row : t.out1_row) >= 0, "plan: a wide unit of a product its task lacks");
                REQ(u.off >= 0 && u.off < ext && u.off % 64 == 0, "plan: a wide unit starts off its 64-grid");
                if (seen[u.task].empty()) seen[u.task].assign((ext + 63) / 64, 0);
                REQ(++seen[u.task][u.off / 64] == 1, "plan: a wide unit repeats");
            }
            for (size_t i = 0; i < ts.size(); i++)
                if ((pass == 0 ? ts[i].out0_row : ts[i].out1_row) >= 0)
                    REQ(!seen[i].empty() && std::count(seen[i].begin(), seen[i].end(), 1) == (long long) seen[i].size(),
                        "plan: a task's %s is not covered by wide units", pass == 0 ? "rows" : "columns");
            w0 += nw[part];
        }
    }

    long long pairs_plan = 0;
    if (d->BD_JIT)
    {
        // ---- (target, source) point pairs against H2Pack's pair lists
        std::vector<long long> jp0(n_node, 0);
        long long np = d->n_point;
        for (int n = 0; n < n_node; n++) { jp0[n] = np; np += d->J_n[n]; }
        auto npt = [&](int n) { return (long long) npt_of(d, n); };
        long long near_o = 0, far_o = 0, near_u = 0, far_u = 0;   // ordered / unordered (pair plan) counts
        for (int i = 0; i < d->n_leaf_node; i++) { const long long p = npt(d->leaf_nodes[i]); near_o += p * p; near_u += p * p; }
        for (int i = 0; i < d->n_r_inadm_pair; i++)
        {
            const long long q = npt(d->r_inadm_pairs[2 * i]) * npt(d->r_inadm_pairs[2 * i + 1]);
            near_o += 2 * q; near_u += q;
        }
        for (int i = 0; i < d->n_r_adm_pair; i++)
        {
            const int a = d->r_adm_pairs[2 * i], b = d->r_adm_pairs[2 * i + 1];
            const long long q = lvl[a] == lvl[b] ? (long long) d->J_n[a] * d->J_n[b]
                              : lvl[a] > lvl[b] ? (long long) d->J_n[a] * npt(b) : (long long) d->J_n[b] * npt(a);
            far_o += 2 * q;
            far_u += lvl[a] == lvl[b] ? q : 2 * q;
        }
        auto pairs_of = [&](const std::vector<JitTarget>& v) {
            long long s = 0;
            for (const JitTarget& t : v)
            {
                long long ns = 0;
                for (int k = t.src_beg; k < t.src_end; k++) ns += hp.js[k].npt;
                s += (long long) t.npt * ns;
            }
            return s;
        };
        REQ(pairs_of(hp.jtN) == near_o, "plan: near field evaluates %lld point pairs, the pair lists imply %lld",
            pairs_of(hp.jtN), near_o);
        REQ(pairs_of(hp.jtF) == far_o, "plan: far field evaluates %lld point pairs, the pair lists imply %lld",
            pairs_of(hp.jtF), far_o);
        pairs_plan = near_o + far_o;

        // ---- each target's source sets are exactly the ones its node's pair lists name
        {
            std::map<long long, int> leaf_at, jset_at;   // first point of a leaf's points / a skeleton -> node
            for (int i = 0; i < d->n_leaf_node; i++) leaf_at[d->pt_cluster[2 * d->leaf_nodes[i]]] = d->leaf_nodes[i];
            for (int n = 0; n < n_node; n++)
                if (d->J_n[n] > 0) jset_at[jp0[n]] = n;
            // a set as (node, skeleton?) from its first point; -1 when it is neither
            auto set_key = [&](long long pt0, int npt_) -> std::pair<int, int> {
                if (pt0 < d->n_point)
                {
                    auto it = leaf_at.find(pt0);
                    return (it != leaf_at.end() && npt(it->second) == npt_) ? std::make_pair(it->second, 0) : std::make_pair(-1, 0);
                }
                auto it = jset_at.find(pt0);
                return (it != jset_at.end() && d->J_n[it->second] == npt_) ? std::make_pair(it->second, 1) : std::make_pair(-1, 1);
            };
            // expected sources of every (node, skeleton?) target set
            std::map<std::pair<int, int>, std::vector<std::pair<int, int>>> near_src, far_src;
            for (int i = 0; i < d->n_leaf_node; i++)
            {
                const int n = d->leaf_nodes[i];
                near_src[{n, 0}].push_back({n, 0});
            }
            for (int i = 0; i < d->n_r_inadm_pair; i++)
            {
                const int a = d->r_inadm_pairs[2 * i], b = d->r_inadm_pairs[2 * i + 1];
                near_src[{a, 0}].push_back({b, 0});
                near_src[{b, 0}].push_back({a, 0});
            }
            for (int i = 0; i < d->n_r_adm_pair; i++)
            {
                const int a = d->r_adm_pairs[2 * i], b = d->r_adm_pairs[2 * i + 1];
                // empty skeletons contribute nothing and are left out of the expected lists
                auto add = [&](int t, int ts, int u, int us) {
                    if (!us || d->J_n[u] > 0) far_src[{t, ts}].push_back({u, us});
                };
                if (lvl[a] == lvl[b]) { add(a, 1, b, 1); add(b, 1, a, 1); }
                else if (lvl[a] > lvl[b]) { add(a, 1, b, 0); add(b, 0, a, 1); }
                else { add(a, 0, b, 1); add(b, 1, a, 0); }
            }
            auto match = [&](const char* field, const std::vector<JitTarget>& v,
                             std::map<std::pair<int, int>, std::vector<std::pair<int, int>>>& want) -> int {
                std::map<std::pair<int, int>, long long> rows;   // target set -> points covered by its chunks
                for (const JitTarget& t : v)
                {
                    // the chunk's set: the leaf or skeleton set holding its first point
                    std::pair<int, int> key{-1, 0};
                    if (t.pt0 < d->n_point)
                    {
                        auto it = leaf_at.upper_bound(t.pt0);
                        if (it != leaf_at.begin()) key = {std::prev(it)->second, 0};
                    } else {
                        auto it = jset_at.upper_bound(t.pt0);
                        if (it != jset_at.begin()) key = {std::prev(it)->second, 1};
                    }
                    REQ(key.first >= 0, "plan (%s): a target chunk belongs to no point set", field);
                    rows[key] += t.npt;
                    std::vector<std::pair<int, int>> got;
                    for (int k = t.src_beg; k < t.src_end; k++)
                    {
                        if (hp.js[k].npt == 0) continue;
                        const auto sk = set_key(hp.js[k].pt0, hp.js[k].npt);
                        REQ(sk.first >= 0, "plan (%s): a source is not a whole point set", field);
                        got.push_back(sk);
                    }
                    std::vector<std::pair<int, int>> exp = want[key];
                    std::sort(got.begin(), got.end());
                    std::sort(exp.begin(), exp.end());
                    REQ(got == exp, "plan (%s): node %d's sources differ from its pair lists", field, key.first);
                }
                for (const auto& kv : want)
                {
                    if (kv.second.empty()) continue;
                    const long long full = kv.first.second ? d->J_n[kv.first.first] : npt(kv.first.first);
                    if (full == 0) continue;
                    REQ(rows[kv.first] == full, "plan (%s): node %d's targets cover %lld of %lld points", field,
                        kv.first.first, rows[kv.first], full);
                }
                return H2GPU_OK;
            };
            TRY(match("near", hp.jtN, near_src));
            TRY(match("far", hp.jtF, far_src));
        }

        // ---- sources, tiles and panel groups
        for (const JitSource& s : hp.js)
        {
            // an empty skeleton (rank 0) is a source of no points: nothing to check
            REQ(s.npt >= 0 && s.pt0 >= 0 && (long long) s.pt0 + s.npt <= np, "plan: JIT source outside the point space");
            if (s.npt == 0) continue;
            if (s.pt0 < d->n_point) REQ(s.in_row == kd * s.pt0, "plan: JIT source input row does not match its points");
            else REQ(s.in_row >= N && (long long) s.in_row + (long long) kd * s.npt <= N + Y0, "plan: JIT source input outside y0");
            if (kd == 1)
                for (int j = 0; j < s.npt; j += 8)
                {
                    const int g = s.grp + j / 8;
                    REQ(g >= 0 && g < (int) hp.pg.size(), "plan: panel group outside the panels");
                    const PanelGroup& G = hp.pg[g];
                    REQ(G.pt0 == s.pt0 + j && G.row0 == s.in_row + j && G.nvalid == std::min(8, s.npt - j),
                        "plan: panel groups do not cover a source set in order");
                }
        }
        for (const std::vector<JitTarget>* v : {&hp.jtN, &hp.jtF, &hp.jtN2, &hp.jtF2})
            for (const JitTarget& t : *v)
            {
                REQ(t.npt >= 1 && t.npt <= 128, "plan: JIT target chunk of %d points", t.npt);
                REQ(t.pt0 >= 0 && (long long) t.pt0 + t.npt <= np, "plan: JIT target outside the point space");
                REQ(t.src_beg >= 0 && t.src_beg <= t.src_end && t.src_end <= (int) hp.js.size(), "plan: JIT target sources out of range");
                int k = t.tile_beg;
                for (int si = t.src_beg; si < t.src_end; si++)
                    for (int j0 = 0; j0 < hp.js[si].npt; j0 += 128, k++)
                    {
                        REQ(k < t.tile_end && k < (int) hp.tiles.size(), "plan: a target has too few source tiles");
                        const TileRec& T = hp.tiles[k];
                        const int nj = std::min(128, hp.js[si].npt - j0);
                        REQ(T.nj == nj && T.ng == (nj + 7) / 8 && T.gb == hp.js[si].grp + j0 / 8,
                            "plan: source tiles do not cover a source set in order");
                    }
                REQ(k == t.tile_end, "plan: a target has too many source tiles");
            }

        // ---- pair plan: every unordered pair owned once, both sides summed once
        if (im->has_pair)
        {
            std::map<long long, int> set_of;   // first point of a set -> node (leaf point sets, skeleton sets)
            for (int i = 0; i < d->n_leaf_node; i++) set_of[d->pt_cluster[2 * d->leaf_nodes[i]]] = d->leaf_nodes[i];
            for (int n = 0; n < n_node; n++)
                if (d->J_n[n] > 0) set_of[jp0[n]] = n;
            auto node_at = [&](long long p) {
                auto it = set_of.upper_bound(p);
                return it == set_of.begin() ? -1 : std::prev(it)->second;
            };
            std::map<std::pair<int, int>, long long> cover;   // (owner, partner) -> owner points covered
            long long pairs_u = 0;
            std::vector<std::pair<long long, long long>> prod2 = down_ps;
            for (const std::vector<PairOwner>* v : {&hp.owN, &hp.owF})
                for (const PairOwner& o : *v)
                {
                    const int a = node_at(o.pa);
                    REQ(a >= 0 && o.na >= 1 && o.na <= kPairOwnerChunk && o.p_beg <= o.p_end &&
                            o.p_end <= (int) hp.partners.size(), "plan: bad pair owner");
                    REQ(o.pa + o.na <= np && o.in_a >= 0 && (long long) o.in_a + o.na <= N + Y0, "plan: pair owner out of range");
                    prod2.push_back({o.out_a, o.na});
                    for (int k = o.p_beg; k < o.p_end; k++)
                    {
                        const PairPartner& pp = hp.partners[k];
                        const int b = node_at(pp.pb);
                        REQ(b >= 0, "plan: pair partner is not a point set");
                        REQ(pp.nb >= 1 && pp.pb + pp.nb <= np && pp.in_b >= 0 && (long long) pp.in_b + pp.nb <= N + Y0,
                            "plan: pair partner out of range");
                        cover[{a, b}] += o.na;
                        pairs_u += (long long) o.na * pp.nb;
                        prod2.push_back({pp.out_b, pp.nb});
                    }
                }
            std::map<std::pair<int, int>, long long> want;   // unordered pairs the pair plan must own
            for (int i = 0; i < d->n_r_inadm_pair; i++)
            {
                const int a = d->r_inadm_pairs[2 * i], b = d->r_inadm_pairs[2 * i + 1];
                want[{std::min(a, b), std::max(a, b)}] = 0;
            }
            for (int i = 0; i < d->n_r_adm_pair; i++)
            {
                const int a = d->r_adm_pairs[2 * i], b = d->r_adm_pairs[2 * i + 1];
                if (lvl[a] == lvl[b] && d->J_n[a] > 0 && d->J_n[b] > 0) want[{std::min(a, b), std::max(a, b)}] = 0;
            }
            for (const auto& kv : cover)
            {
                const int a = kv.first.first, b = kv.first.second;
                auto it = want.find({std::min(a, b), std::max(a, b)});
                REQ(it != want.end(), "plan: the pair plan owns nodes %d and %d, which are not a pair", a, b);
                REQ(cover.count({b, a}) == 0, "plan: the pair of nodes %d and %d is owned both ways", a, b);
                it->second++;
            }
            for (const auto& kv : want) REQ(kv.second == 1, "plan: the pair of nodes %d and %d is not owned", kv.first.first, kv.first.second);
            for (const std::vector<JitTarget>* v : {&hp.jtN2, &hp.jtF2})
                for (const JitTarget& t : *v) prod2.push_back({t.out_row, (long long) t.npt});
            pairs_u += pairs_of(hp.jtN2) + pairs_of(hp.jtF2);
            REQ(pairs_u == near_u + far_u, "plan: the pair plan evaluates %lld point pairs, the pair lists imply %lld",
                pairs_u, near_u + far_u);
            TRY(check_space("pair", prod2, {}, hp.at2, hp.at_slots2, hp.y1t2, hp.y1_slots2));
        }
    }
    if (counts)
    {
        counts[0] = (long long) hp.up.size();
        counts[1] = (long long) hp.dn.size();
        counts[2] = (long long) (hp.blkB.size() + hp.blkD.size());
        counts[3] = (long long) (hp.jtN.size() + hp.jtF.size());
        counts[4] = (long long) hp.tiles.size();
        counts[5] = (long long) hp.pg.size();
        counts[6] = PSR;
        counts[7] = pairs_plan;
    }
    return H2GPU_OK;
}


KParam kparam_of(const h2gpu_image* im);

int upload_plan(h2gpu_image* im, const h2gpu_desc* d, HostPlan& hp)
{
    TRY(upload(hp.U, &im->d_U64, im->bytes));
    TRY(upload(hp.up, &im->d_up, im->bytes));
    TRY(upload(hp.dn, &im->d_dn, im->bytes));
    TRY(upload(hp.y1t, &im->d_y1t, im->bytes));
    TRY(upload(hp.y1_slots, &im->d_y1_slots, im->bytes));
    TRY(upload(hp.blkB, &im->d_blkB, im->bytes));
    TRY(upload(hp.blkD, &im->d_blkD, im->bytes));
    TRY(upload(hp.wide, &im->d_wide, im->bytes));
    TRY(upload(hp.jtN, &im->d_jtN, im->bytes));
    TRY(upload(hp.jtF, &im->d_jtF, im->bytes));
    TRY(upload(hp.js, &im->d_js, im->bytes));
    TRY(upload(hp.at, &im->d_asm, im->bytes));
    TRY(upload(hp.at_slots, &im->d_asm_slots, im->bytes));
    TRY(upload(hp.fw, &im->d_fwd, im->bytes));
    TRY(upload(hp.bw, &im->d_bwd, im->bytes));
    TRY(upload(hp.p64, &im->d_pts64, im->bytes));
    TRY(upload(hp.p32, &im->d_pts32, im->bytes));
    TRY(upload(hp.p32lo, &im->d_pts32lo, im->bytes));
    TRY(upload(hp.owN, &im->d_owN, im->bytes));
    TRY(upload(hp.owF, &im->d_owF, im->bytes));
    TRY(upload(hp.partners, &im->d_pp, im->bytes));
    TRY(upload(hp.jtN2, &im->d_jtN2, im->bytes));
    TRY(upload(hp.jtF2, &im->d_jtF2, im->bytes));
    TRY(upload(hp.y1t2, &im->d_y1t2, im->bytes));
    TRY(upload(hp.y1_slots2, &im->d_y1_slots2, im->bytes));
    TRY(upload(hp.at2, &im->d_asm2, im->bytes));
    TRY(upload(hp.at_slots2, &im->d_asm_slots2, im->bytes));
    TRY(upload(hp.pg, &im->d_pg, im->bytes));
    TRY(upload(hp.tiles, &im->d_tiles, im->bytes));
    im->n_pg = (int) hp.pg.size();
    im->n_pg_pts = hp.pg_pts;
    if (im->n_pg > 0 && d->krnl_dim == 1)
    {
        // the point half of the panels is static
        CK(cudaMalloc(&im->d_ppts, sizeof(float4) * 8 * (size_t) im->n_pg));
        im->bytes += sizeof(float4) * 8 * (size_t) im->n_pg;
        CK(launch_panel_pts(im->d_pg, im->n_pg, im->d_pts32, kparam_of(im).sigma, im->d_ppts, im->stream));
        if (im->d_pts32lo)
        {
            CK(cudaMalloc(&im->d_pplo, sizeof(float4) * 6 * (size_t) im->n_pg));
            im->bytes += sizeof(float4) * 6 * (size_t) im->n_pg;
            CK(launch_panel_lo(im->d_pg, im->n_pg, im->d_pts32lo, im->d_pplo, im->stream));
        }
        CK(cudaStreamSynchronize(im->stream));
    }
    if (!d->BD_JIT && !im->gen)
    {
        if (im->B_elems)
        {
            CK(cudaMalloc(&im->d_B64, 8 * im->B_elems));
            CK(cudaMemcpy(im->d_B64, d->B_data, 8 * im->B_elems, cudaMemcpyHostToDevice));
            im->bytes += 8 * im->B_elems;
        }
        CK(cudaMalloc(&im->d_D64, 8 * im->D_elems));
        CK(cudaMemcpy(im->d_D64, d->D_data, 8 * im->D_elems, cudaMemcpyHostToDevice));
        im->bytes += 8 * im->D_elems;
    }
    return H2GPU_OK;
}

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, size_t n)
{
    for (size_t i = blockIdx.x * (size_t) blockDim.x + threadIdx.x; i < n; i += (size_t) gridDim.x * blockDim.x)
        b[i] = (float) a[i];
}

// FP32 copy of a stored-block arena in the padded layout: one CTA per block task (the
// tasks of a list cover every block row once), padding written as zeros
__global__ void k_blk_to_f32(const BlkTask* __restrict__ tasks, const double* __restrict__ a, float* __restrict__ b)
{
    const BlkTask t = tasks[blockIdx.x];
    const long long n = (long long) t.nrow * t.ld32;
    for (long long i = threadIdx.x; i < n; i += blockDim.x)
    {
        const int r = (int) (i / t.ld32), c = (int) (i % t.ld32);
        b[t.a32 + i] = c < t.ncol ? (float) a[t.a_off + (long long) r * t.ncol + c] : 0.f;
    }
}

int make_f32_blocks(h2gpu_image* im, const BlkTask* tasks, int n, const double* src, float** dst, size_t n32)
{
    if (n32 == 0 || *dst) return H2GPU_OK;
    CK(cudaMalloc(dst, 4 * n32));
    if (n > 0) k_blk_to_f32<<<n, 256, 0, im->stream>>>(tasks, src, *dst);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(im->stream));
    im->bytes += 4 * n32;
    return H2GPU_OK;
}

int make_f32(h2gpu_image* im, const double* src, float** dst, size_t n)
{
    if (n == 0 || *dst) return H2GPU_OK;
    CK(cudaMalloc(dst, 4 * n));
    k_to_f32<<<148 * 8, 256, 0, im->stream>>>(src, *dst, n);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(im->stream));
    im->bytes += 4 * n;
    return H2GPU_OK;
}

int ensure_work(h2gpu_image* im, int NV)
{
    if (im->NVb >= NV) return H2GPU_OK;
    for (double** p : {&im->d_XS, &im->d_PS, &im->d_Y1, &im->d_PUSH})
        if (*p) { cudaFree(*p); *p = nullptr; }
    if (im->d_XS3) { cudaFree(im->d_XS3); im->d_XS3 = nullptr; }
    im->NVb = 0;          // no buffers until all four are allocated
    im->work_bytes = 0;
    size_t xs = ((size_t) im->N + im->y0_rows) * NV, ps = (size_t) im->ps_rows * NV, y1 = (size_t) im->y0_rows * NV;
    CK(cudaMalloc(&im->d_XS, 8 * std::max<size_t>(xs, 1)));
    CK(cudaMalloc(&im->d_PS, 8 * std::max<size_t>(ps, 1)));
    CK(cudaMalloc(&im->d_Y1, 8 * std::max<size_t>(y1, 1)));
    CK(cudaMalloc(&im->d_PUSH, 8 * std::max<size_t>(y1, 1)));
    size_t xs3 = 0;
    if (NV == 64 && !im->BD_JIT)
    {
        // the 64-wide block passes read their inputs as BF16 pieces (3 x 2 bytes per value)
        xs3 = 3 * ((size_t) im->N + im->y0_rows) * 64;
        CK(cudaMalloc(&im->d_XS3, 2 * xs3));
    }
    im->work_bytes = 8 * (xs + ps + 2 * y1) + 2 * xs3;
    im->NVb = NV;
    return H2GPU_OK;
}

int panel_width(int n_vec, int max_nv)
{
    int w = 1;
    while (w < n_vec && w < max_nv) w <<= 1;
    return w;
}

// Widest panel of right-hand sides the image's kernels take: 64 for mixed stored-block
// images (the wide tcgen05 block kernel: one read of every block per 64 right-hand
// sides), 8 for RPY JIT images, 16 otherwise; never above the image's max_n_vec.
int panel_cap(const h2gpu_image* im)
{
    if (im->BD_JIT && im->kd == 3) return std::min(im->max_nv, 8);
    if (!im->BD_JIT && im->precision == H2GPU_PREC_MIXED) return std::min(im->max_nv, 64);
    return std::min(im->max_nv, 16);
}

KParam kparam_from(int kernel_id, const double* kp, int n_kp)
{
    KParam k{0.0, 0.0, 1.f, 0.f};
    const float log2e = 1.4426950408889634f;
    switch (kernel_id)
    {
        case H2GPU_KRNL_COULOMB: k.p0 = n_kp > 0 ? kp[0] : 0.0; break;
        case H2GPU_KRNL_GAUSSIAN: k.p0 = kp[0]; k.sigma = (float) k.p0 * log2e; break;
        case H2GPU_KRNL_MATERN32:
        {
            k.p0 = kp[0];
            k.c0 = -1.7320508075688772 * kp[0];
            const float q1 = (float) k.c0 * log2e;
            k.sigma = q1 * q1;
            break;
        }
        case H2GPU_KRNL_RPY: k.p0 = kp[0]; k.c0 = 1.0 / (6.0 * M_PI * kp[0]); break;
    }
    return k;
}

KParam kparam_of(const h2gpu_image* im) { return kparam_from(im->kernel_id, im->kp, im->n_kp); }

// The tcgen05 stored-block kernel (mixed precision, normal mode) reports through the
// status word.
bool uses_status(const h2gpu_image* im, int NV)
{
    return im->d_status && im->h_status && (im->blk_tc == 2 || NV > 16) && !im->BD_JIT &&
           im->precision == H2GPU_PREC_MIXED;
}

// FP32 sweeps on the tensor cores when the image's kernel variant is a tensor-core one.
int sweep_tc(const h2gpu_image* im) { return im->BD_JIT ? im->jit_tc : im->blk_tc; }

// The tensor-core JIT kernel (FP32 scalar kernels, panels of 8 / 16) reads its sources
// from the panels; they are refilled from XS for every panel of right-hand sides.
bool panels_used(const h2gpu_image* im, int NV)
{
    return im->BD_JIT && im->kd == 1 && im->jit_tc && im->d_pin && (NV == 8 || NV == 16);
}

// One panel of NV right-hand sides: X (original order, strides x_rs, x_cs) -> Y.
int run_panel(h2gpu_image* im, int NV, int nv, const double* X, long long x_rs, long long x_cs, double* Y,
              long long y_rs, long long y_cs, cudaStream_t s, bool timed)
{
    const bool f32 = im->precision == H2GPU_PREC_MIXED;
    cudaEvent_t* e = im->ev.e;
    if (im->has_pair && im->jit_pair && f32 && im->jit_tc && (NV == 8 || NV == 16))
    {
        // each unordered JIT pair evaluated once, applied both ways (tensor cores)
        const KParam kp = kparam_of(im);
        if (timed) CK(cudaEventRecord(e[0], s));
        CK(launch_gather(NV, X, x_rs, x_cs, nv, im->d_fwd, im->N, im->d_XS, s));
        if (timed) CK(cudaEventRecord(e[1], s));
        CK(launch_panel_in(NV, im->d_pg, 0, im->n_pg_pts, im->d_XS, im->d_pin, s));
        CK(launch_jit(im->kernel_id, 1, NV, im->d_jtN2, im->n_jtN2, im->d_js, im->d_pts32, kp, 1, 1, im->d_XS,
                      im->d_PS, im->d_Y1, s, 0, im->d_ppts, im->d_pin, im->d_tiles, im->d_pts32lo, im->d_pplo));
        CK(launch_pair(im->kernel_id, NV, im->d_owN, im->n_owN, im->d_pp, im->d_pts32, kp, im->d_XS, im->d_PS, s, 0,
                       im->d_pts32lo));
        if (timed) CK(cudaEventRecord(e[2], s));
        for (size_t L = 0; L + 1 < im->up_beg.size(); L++)
        {
            int b = im->up_beg[L], n = im->up_beg[L + 1] - b;
            CK(launch_up<float>(NV, im->d_up + b, n, im->d_U32, im->d_XS, s, sweep_tc(im)));
        }
        if (timed) CK(cudaEventRecord(e[3], s));
        CK(launch_pair(im->kernel_id, NV, im->d_owF, im->n_owF, im->d_pp, im->d_pts32, kp, im->d_XS, im->d_PS, s,
                       im->far_diff ? 0 : 1, im->d_pts32lo));
        CK(launch_panel_in(NV, im->d_pg, im->n_pg_pts, im->n_pg - im->n_pg_pts, im->d_XS, im->d_pin, s));
        CK(launch_jit(im->kernel_id, 1, NV, im->d_jtF2, im->n_jtF2, im->d_js, im->d_pts32, kp, 1, 1, im->d_XS,
                      im->d_PS, im->d_Y1, s, im->far_diff ? 0 : 1, im->d_ppts, im->d_pin, im->d_tiles, im->d_pts32lo,
                      im->d_pplo));
        CK(launch_y1sum(NV, im->d_y1t2, im->n_y12, im->d_y1_slots2, im->d_PS, im->d_Y1, s));
        if (timed) CK(cudaEventRecord(e[4], s));
        for (size_t L = 0; L + 1 < im->dn_beg.size(); L++)
        {
            int b = im->dn_beg[L], n = im->dn_beg[L + 1] - b;
            CK(launch_down<float>(NV, im->d_dn + b, n, im->d_U32, im->d_Y1, im->d_PS, im->d_PUSH, s, sweep_tc(im)));
        }
        if (timed) CK(cudaEventRecord(e[5], s));
        CK(launch_asm(NV, im->d_asm2, im->n_asm2, im->d_asm_slots2, im->d_PS, im->d_fwd, Y, y_rs, y_cs, nv, s));
        if (timed) CK(cudaEventRecord(e[6], s));
        im->st.n_launches += 9 + (long long) (im->up_beg.size() - 1) + (long long) (im->dn_beg.size() - 1);
        return H2GPU_OK;
    }
    const bool wide = f32 && !im->BD_JIT && NV == 64;   // two GEMM passes per block list
    const long long xs_rows = (long long) im->N + im->y0_rows;
    if (timed) CK(cudaEventRecord(e[0], s));
    CK(launch_gather(NV, X, x_rs, x_cs, nv, im->d_fwd, im->N, im->d_XS, s));
    if (wide) CK(launch_split3(im->d_XS, 0, im->N, xs_rows, im->d_XS3, s));
    // D phase first: it needs only x (in the graph-free stream order it simply runs before the upward sweep)
    if (timed) CK(cudaEventRecord(e[1], s));
    if (!im->BD_JIT)
    {
        if (wide)
        {
            const int* nw = im->n_wide;
            CK(launch_blk_wide(0, im->d_blkD, im->d_wide + nw[0] + nw[1], nw[2], im->d_D32, im->d_XS3, xs_rows,
                               im->d_PS, s, im->d_status));
            CK(launch_blk_wide(1, im->d_blkD, im->d_wide + nw[0] + nw[1] + nw[2], nw[3], im->d_D32, im->d_XS3,
                               xs_rows, im->d_PS, s, im->d_status));
            im->st.n_launches += 2;   // the second pass and the split of the inputs
        }
        else if (f32) CK(launch_blk<float>(NV, im->d_blkD, im->n_blkD, im->d_D32, im->d_XS, im->d_PS, s, im->blk_tc, im->d_status,
                                           im->blk1_small[1][1]));
        else CK(launch_blk<double>(NV, im->d_blkD, im->n_blkD, im->d_D64, im->d_XS, im->d_PS, s, 0, nullptr,
                                   im->blk1_small[1][0]));
    } else {
        const bool panels = f32 && panels_used(im, NV);
        if (panels) CK(launch_panel_in(NV, im->d_pg, 0, im->n_pg_pts, im->d_XS, im->d_pin, s));
        CK(launch_jit(im->kernel_id, f32, NV, im->d_jtN, im->n_jtN, im->d_js, f32 ? (const void*) im->d_pts32 : (const void*) im->d_pts64,
                      kparam_of(im), f32 ? 1 : 0, im->jit_tc, im->d_XS, im->d_PS, im->d_Y1, s, 0, im->d_ppts, im->d_pin, im->d_tiles,
                      im->d_pts32lo, im->d_pplo));
        im->st.n_launches += panels ? 1 : 0;
    }
    if (timed) CK(cudaEventRecord(e[2], s));
    for (size_t L = 0; L + 1 < im->up_beg.size(); L++)
    {
        int b = im->up_beg[L], n = im->up_beg[L + 1] - b;
        if (f32) CK(launch_up<float>(NV, im->d_up + b, n, im->d_U32, im->d_XS, s, sweep_tc(im)));
        else CK(launch_up<double>(NV, im->d_up + b, n, im->d_U64, im->d_XS, s));
    }
    if (timed) CK(cudaEventRecord(e[3], s));
    if (!im->BD_JIT)
    {
        if (wide)
        {
            const int* nw = im->n_wide;
            CK(launch_split3(im->d_XS, im->N, im->y0_rows, xs_rows, im->d_XS3, s));   // the skeleton rows y0
            CK(launch_blk_wide(0, im->d_blkB, im->d_wide, nw[0], im->d_B32, im->d_XS3, xs_rows, im->d_PS, s,
                               im->d_status));
            CK(launch_blk_wide(1, im->d_blkB, im->d_wide + nw[0], nw[1], im->d_B32, im->d_XS3, xs_rows, im->d_PS, s,
                               im->d_status));
            im->st.n_launches += 2;   // the second pass and the split of the inputs
        }
        else if (f32) CK(launch_blk<float>(NV, im->d_blkB, im->n_blkB, im->d_B32, im->d_XS, im->d_PS, s, im->blk_tc, im->d_status,
                                           im->blk1_small[0][1]));
        else CK(launch_blk<double>(NV, im->d_blkB, im->n_blkB, im->d_B64, im->d_XS, im->d_PS, s, 0, nullptr,
                                   im->blk1_small[0][0]));
        CK(launch_y1sum(NV, im->d_y1t, im->n_y1, im->d_y1_slots, im->d_PS, im->d_Y1, s));
    } else {
        const bool panels = f32 && panels_used(im, NV);
        if (panels) CK(launch_panel_in(NV, im->d_pg, im->n_pg_pts, im->n_pg - im->n_pg_pts, im->d_XS, im->d_pin, s));
        CK(launch_jit(im->kernel_id, f32, NV, im->d_jtF, im->n_jtF, im->d_js, f32 ? (const void*) im->d_pts32 : (const void*) im->d_pts64,
                      kparam_of(im), f32 ? 1 : 0, im->jit_tc, im->d_XS, im->d_PS, im->d_Y1, s, im->far_diff ? 0 : 1,
                      im->d_ppts, im->d_pin, im->d_tiles, im->d_pts32lo, im->d_pplo));
        im->st.n_launches += panels ? 1 : 0;
    }
    if (timed) CK(cudaEventRecord(e[4], s));
    for (size_t L = 0; L + 1 < im->dn_beg.size(); L++)
    {
        int b = im->dn_beg[L], n = im->dn_beg[L + 1] - b;
        if (f32) CK(launch_down<float>(NV, im->d_dn + b, n, im->d_U32, im->d_Y1, im->d_PS, im->d_PUSH, s, sweep_tc(im)));
        else CK(launch_down<double>(NV, im->d_dn + b, n, im->d_U64, im->d_Y1, im->d_PS, im->d_PUSH, s));
    }
    if (timed) CK(cudaEventRecord(e[5], s));
    CK(launch_asm(NV, im->d_asm, im->n_asm, im->d_asm_slots, im->d_PS, im->d_fwd, Y, y_rs, y_cs, nv, s));
    if (timed && uses_status(im, NV))
        CK(cudaMemcpyAsync(im->h_status, im->d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (timed) CK(cudaEventRecord(e[6], s));
    im->st.n_launches += 4 + (long long) (im->up_beg.size() - 1) + (long long) (im->dn_beg.size() - 1)
                         + (im->BD_JIT ? 0 : 1);
    return H2GPU_OK;
}

// Bounded waits inside the tcgen05 block kernel set the image's status word when they
// expire; a timed panel copies it back (pinned) before its last event, and a
// synchronised apply reports it (and clears it) as H2GPU_ERR_DEVICE.
int check_status(h2gpu_image* im)
{
    if (!im->d_status || !im->h_status) return H2GPU_OK;
    if (*(volatile int*) im->h_status != 0)
    {
        *im->h_status = 0;
        CK(cudaMemset(im->d_status, 0, sizeof(int)));
        return fail(H2GPU_ERR_DEVICE, "tcgen05 block kernel: a bounded wait on the MMA completion expired");
    }
    return H2GPU_OK;
}

// Fill the stored-block arenas on the device (H2GPU_BLOCKS_GENERATE): FP64 for an FP64
// image, FP32 only for a mixed one.  The point arena and the task lists are freed again.
int generate_blocks(h2gpu_image* im, const GenPlan& g)
{
    const int fp32 = im->precision == H2GPU_PREC_MIXED;
    const size_t es = fp32 ? 4 : 8;
    double4* pts = nullptr;
    GenTask* tasks = nullptr;
    size_t dummy = 0;
    int st = H2GPU_OK;
    do {
        if ((st = upload(g.pts, &pts, dummy)) != H2GPU_OK) break;
        std::vector<GenTask> all(g.tB);
        all.insert(all.end(), g.tD.begin(), g.tD.end());
        if ((st = upload(all, &tasks, dummy)) != H2GPU_OK) break;
        void* B = nullptr;
        void* D = nullptr;
        const size_t nB = fp32 ? im->B32_elems : im->B_elems, nD = fp32 ? im->D32_elems : im->D_elems;
        cudaError_t e = cudaSuccess;
        if (nB) e = cudaMalloc(&B, es * nB);
        if (e == cudaSuccess) e = cudaMalloc(&D, es * std::max<size_t>(nD, 1));
        if (e != cudaSuccess)
        {
            if (B) cudaFree(B);
            st = fail(H2GPU_ERR_NOMEM, "stored-block arenas of %.1f GB do not fit on the device", 1e-9 * es * (nB + nD));
            break;
        }
        if (fp32) { im->d_B32 = (float*) B; im->d_D32 = (float*) D; im->f32_only = 1; }
        else { im->d_B64 = (double*) B; im->d_D64 = (double*) D; }
        im->bytes += es * (nB + nD);
        // the FP32 rows' padding stays zero (the kernels read it through 16-byte loads)
        if (fp32 && nB) e = cudaMemsetAsync(B, 0, es * nB, im->stream);
        if (fp32 && nD && e == cudaSuccess) e = cudaMemsetAsync(D, 0, es * nD, im->stream);
        const KParam kp = kparam_of(im);
        // one launch per block kind, in slices that keep the grid inside its limits
        const int tB = (int) g.tB.size(), tD = (int) g.tD.size();
        const int slice = 1 << 24;
        for (int b = 0; b < tB && e == cudaSuccess; b += slice)
            e = launch_gen(im->kernel_id, im->kd, fp32, tasks + b, std::min(slice, tB - b), pts, kp, B, im->stream);
        for (int b = 0; b < tD && e == cudaSuccess; b += slice)
            e = launch_gen(im->kernel_id, im->kd, fp32, tasks + tB + b, std::min(slice, tD - b), pts, kp, D, im->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(im->stream);
        if (e != cudaSuccess) st = fail(H2GPU_ERR_CUDA, "stored-block generation failed: %s", cudaGetErrorString(e));
    } while (0);
    if (pts) cudaFree(pts);
    if (tasks) cudaFree(tasks);
    return st;
}

int prepare(h2gpu_image* im, int NV)
{
    CK(cudaSetDevice(im->device));
    if (im->f32_only && im->precision != H2GPU_PREC_MIXED)
        return fail(H2GPU_ERR_STATE, "this image holds its stored blocks in FP32 only (generated for mixed "
                                     "precision); create it in FP64 for FP64 applies");
    if (im->precision == H2GPU_PREC_MIXED)
    {
        TRY(make_f32(im, im->d_U64, &im->d_U32, im->U_elems));
        TRY(make_f32_blocks(im, im->d_blkB, im->n_blkB, im->d_B64, &im->d_B32, im->B32_elems));
        TRY(make_f32_blocks(im, im->d_blkD, im->n_blkD, im->d_D64, &im->d_D32, im->D32_elems));
        if (im->d_ppts && !im->d_pin)
        {
            const size_t b = sizeof(uint4) * 64 * (size_t) im->n_pg;   // panels of up to 16 right-hand sides
            CK(cudaMalloc(&im->d_pin, b));
            im->bytes += b;
        }
    }
    return ensure_work(im, NV);
}

// Apply to n_vec columns of a device matrix (strides in elements), panel by panel.
int apply_device(h2gpu_image* im, int n_vec, const double* X, long long x_rs, long long x_cs, double* Y,
                 long long y_rs, long long y_cs, cudaStream_t s)
{
    // JIT tensor kernels keep 3 x NV accumulators per target: panels of at most 8 there
    int NV = panel_width(n_vec, panel_cap(im));
    if (im->tuned_nv > 0) NV = std::min(NV, im->tuned_nv);
    int pst = prepare(im, NV);
    if (pst == H2GPU_ERR_NOMEM && NV > 16)
    {
        // the work space of a wide panel does not fit: panels of 16
        cudaGetLastError();
        NV = 16;
        pst = prepare(im, NV);
    }
    TRY(pst);
    float ph[5] = {0, 0, 0, 0, 0};
    for (int c0 = 0; c0 < n_vec; c0 += NV)
    {
        int nv = std::min(NV, n_vec - c0);
        TRY(run_panel(im, NV, nv, X + c0 * x_cs, x_rs, x_cs, Y + c0 * y_cs, y_rs, y_cs, s, true));
        CK(cudaEventSynchronize(im->ev.e[6]));
        TRY(check_status(im));
        float t[6];
        for (int k = 0; k < 6; k++) CK(cudaEventElapsedTime(&t[k], im->ev.e[k], im->ev.e[k + 1]));
        ph[0] += t[0] + t[2];   // gather + upward
        ph[1] += t[3];          // B
        ph[2] += t[4];          // downward
        ph[3] += t[1];          // D
        ph[4] += t[5];          // assemble
    }
    for (int k = 0; k < 5; k++) { im->st.ms_phase[k] += ph[k]; im->st.ms_total += ph[k]; }
    im->st.n_matvec += n_vec;
    return H2GPU_OK;
}

// Apply without events or host synchronisation (the CG engine), in the given precision.
int apply_quiet(h2gpu_image* im, int precision, int n_vec, const double* X, int ldx, double* Y, int ldy,
                cudaStream_t s)
{
    const int saved = im->precision;
    im->precision = precision;
    int NV = panel_width(n_vec, panel_cap(im));
    if (im->tuned_nv > 0) NV = std::min(NV, im->tuned_nv);
    int st = prepare(im, NV);
    for (int c0 = 0; st == H2GPU_OK && c0 < n_vec; c0 += NV)
        st = run_panel(im, NV, std::min(NV, n_vec - c0), X + c0, ldx, 1, Y + c0, ldy, 1, s, false);
    im->precision = saved;
    if (st == H2GPU_OK) im->st.n_matvec += n_vec;
    return st;
}

int ensure_io(h2gpu_image* im, size_t elems)
{
    if (im->io_elems >= elems) return H2GPU_OK;
    if (im->d_io) cudaFree(im->d_io);
    im->d_io = nullptr;
    im->io_elems = 0;
    CK(cudaMalloc(&im->d_io, 8 * elems));
    im->io_elems = elems;
    return H2GPU_OK;
}

}  // namespace

// ===================================================================== C ABI

H2G_API int h2gpu_abi_version(void) { return H2GPU_ABI_VERSION; }

H2G_API const char* h2gpu_last_error(void) { return g_err.c_str(); }

H2G_API void h2gpu_default_options(h2gpu_options* opt)
{
    if (!opt) return;
    opt->precision = H2GPU_PREC_FP64;
    opt->max_n_vec = 64;
    opt->device = -1;
    opt->blocks = H2GPU_BLOCKS_GIVEN;
}

H2G_API int h2gpu_image_create(const h2gpu_desc* desc, const h2gpu_options* opt, h2gpu_image** out)
{
    if (!out) return fail(H2GPU_ERR_INVALID, "out is NULL");
    *out = nullptr;
    h2gpu_options o;
    h2gpu_default_options(&o);
    if (opt) o = *opt;
    REQ(o.precision == H2GPU_PREC_FP64 || o.precision == H2GPU_PREC_MIXED, "unknown precision %d", o.precision);
    REQ(o.blocks == H2GPU_BLOCKS_GIVEN || o.blocks == H2GPU_BLOCKS_GENERATE, "unknown blocks option %d", o.blocks);
    const bool gen = o.blocks == H2GPU_BLOCKS_GENERATE;
    // generated blocks: the representation is applied as a stored-block (AOT) one whose
    // B / D arenas the device fills; the descriptor's own B_data / D_data are not read
    h2gpu_desc dg;
    if (gen && desc)
    {
        dg = *desc;
        dg.BD_JIT = 0;
        dg.B_data = nullptr;
        dg.D_data = nullptr;
        desc = &dg;
    }
    TRY(validate(desc, gen));
    h2gpu_image* im = new h2gpu_image();
    im->gen = gen;
    {
        const char* e = getenv("H2G_JIT_TC");
        im->jit_tc = !(e && e[0] == '0');
        e = getenv("H2G_JIT_PAIR");
        im->jit_pair = (e && e[0] == '1');
        e = getenv("H2G_BLK_TC");
        im->blk_tc = !(e && e[0] == '0');
    }
    HostPlan hp;
    GenPlan gp;
    int pst = build_plan(im, desc, hp);   // all structural checks happen here, before any CUDA call
    if (pst == H2GPU_OK && gen) pst = build_gen(desc, gp);
    if (pst == H2GPU_OK)
    {
        // the plan self-check of h2gpu_plan_check, on request (the test suite sets it)
        const char* e = getenv("H2G_PLAN_CHECK");
        if (e && e[0] == '1') pst = check_plan(im, desc, hp, nullptr);
    }
    if (pst != H2GPU_OK) { delete im; return pst; }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
    {
        delete im;
        return fail(H2GPU_ERR_CUDA, "no CUDA device available (%s); the H2 apply path has no CPU fallback",
                    cudaGetErrorString(e));
    }
    im->precision = o.precision;
    im->max_nv = (o.max_n_vec >= 1 && o.max_n_vec <= 64) ? o.max_n_vec : 64;
    if (o.device >= 0) im->device = o.device;
    else cudaGetDevice(&im->device);
    int st = H2GPU_OK;
    do {
        if (cudaSetDevice(im->device) != cudaSuccess) { st = fail(H2GPU_ERR_CUDA, "cudaSetDevice(%d) failed", im->device); break; }
        if (cudaStreamCreateWithFlags(&im->stream, cudaStreamNonBlocking) != cudaSuccess) { st = fail(H2GPU_ERR_CUDA, "stream creation failed"); break; }
        for (auto& ev : im->ev.e)
            if (cudaEventCreate(&ev) != cudaSuccess) { st = fail(H2GPU_ERR_CUDA, "event creation failed"); break; }
        if (st != H2GPU_OK) break;
        st = upload_plan(im, desc, hp);
        if (st == H2GPU_OK && gen) st = generate_blocks(im, gp);
        if (st == H2GPU_OK && (cudaMalloc(&im->d_status, sizeof(int)) != cudaSuccess ||
                               cudaMemset(im->d_status, 0, sizeof(int)) != cudaSuccess ||
                               cudaHostAlloc(&im->h_status, sizeof(int), cudaHostAllocDefault) != cudaSuccess))
            st = fail(H2GPU_ERR_NOMEM, "status word allocation failed");
        if (st == H2GPU_OK) *im->h_status = 0;
    } while (0);
    if (st != H2GPU_OK)
    {
        free_all(im);
        delete im;
        return st;
    }
    *out = im;
    return H2GPU_OK;
}

H2G_API int h2gpu_image_destroy(h2gpu_image* im)
{
    if (!im) return H2GPU_OK;
    {
        std::lock_guard<std::mutex> lk(im->mu);
        cudaSetDevice(im->device);
        if (im->stream) cudaStreamSynchronize(im->stream);
        free_all(im);
    }
    delete im;
    return H2GPU_OK;
}

H2G_API int h2gpu_set_precision(h2gpu_image* im, int precision)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    REQ(precision == H2GPU_PREC_FP64 || precision == H2GPU_PREC_MIXED, "unknown precision %d", precision);
    std::lock_guard<std::mutex> lk(im->mu);
    if (im->f32_only && precision != H2GPU_PREC_MIXED)
        return fail(H2GPU_ERR_STATE, "this image holds its stored blocks in FP32 only (generated for mixed "
                                     "precision); create it in FP64 for FP64 applies");
    im->precision = precision;
    return H2GPU_OK;
}

H2G_API int h2gpu_matmul_device(h2gpu_image* im, int n_vec, const double* dX, int ldx, double* dY, int ldy,
                                void* stream)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    REQ(n_vec >= 1 && ldx >= n_vec && ldy >= n_vec && dX && dY, "bad matmul_device arguments");
    std::lock_guard<std::mutex> lk(im->mu);
    cudaStream_t s = stream ? (cudaStream_t) stream : im->stream;
    TRY(apply_device(im, n_vec, dX, ldx, 1, dY, ldy, 1, s));
    return H2GPU_OK;
}

H2G_API int h2gpu_matmul(h2gpu_image* im, int layout, int n_vec, const double* X, int ldx, double* Y, int ldy)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    REQ(X && Y && n_vec >= 1, "bad matmul arguments");
    REQ(layout == H2GPU_ROW_MAJOR || layout == H2GPU_COL_MAJOR, "bad layout %d", layout);
    const long long N = 0;
    (void) N;
    std::lock_guard<std::mutex> lk(im->mu);
    const size_t n = (size_t) im->N;
    if (layout == H2GPU_ROW_MAJOR) REQ(ldx >= n_vec && ldy >= n_vec, "row-major leading dimension < n_vec");
    else REQ((size_t) ldx >= n && (size_t) ldy >= n, "column-major leading dimension < krnl_mat_size");
    CK(cudaSetDevice(im->device));
    TRY(ensure_io(im, 2 * n * n_vec));
    double* dX = im->d_io;
    double* dY = im->d_io + n * n_vec;
    cudaStream_t s = im->stream;
    if (layout == H2GPU_ROW_MAJOR)
    {
        CK(cudaMemcpy2DAsync(dX, 8 * (size_t) n_vec, X, 8 * (size_t) ldx, 8 * (size_t) n_vec, n, cudaMemcpyHostToDevice, s));
        TRY(apply_device(im, n_vec, dX, n_vec, 1, dY, n_vec, 1, s));
        CK(cudaMemcpy2DAsync(Y, 8 * (size_t) ldy, dY, 8 * (size_t) n_vec, 8 * (size_t) n_vec, n, cudaMemcpyDeviceToHost, s));
    } else {
        CK(cudaMemcpy2DAsync(dX, 8 * n, X, 8 * (size_t) ldx, 8 * n, n_vec, cudaMemcpyHostToDevice, s));
        TRY(apply_device(im, n_vec, dX, 1, (long long) n, dY, 1, (long long) n, s));
        CK(cudaMemcpy2DAsync(Y, 8 * (size_t) ldy, dY, 8 * n, 8 * n, n_vec, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    return H2GPU_OK;
}

H2G_API int h2gpu_matvec(h2gpu_image* im, const double* x, double* y)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    return h2gpu_matmul(im, H2GPU_COL_MAJOR, 1, x, im->N, y, im->N);
}

namespace h2gpu {
cudaError_t launch_permute(const double* X, long long x_rs, long long x_cs, const int* idx, int n, int nv, double* Y,
                           long long y_rs, long long y_cs, cudaStream_t st);
}

H2G_API int h2gpu_permute_matrix_rows(h2gpu_image* im, int forward, int layout, int n_vec, const double* X, int ldx,
                                      double* PX, int ldp)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    REQ(X && PX && n_vec >= 1, "bad permute arguments");
    REQ(layout == H2GPU_ROW_MAJOR || layout == H2GPU_COL_MAJOR, "bad layout %d", layout);
    std::lock_guard<std::mutex> lk(im->mu);
    const size_t n = (size_t) im->N;
    if (layout == H2GPU_ROW_MAJOR) REQ(ldx >= n_vec && ldp >= n_vec, "row-major leading dimension < n_vec");
    else REQ((size_t) ldx >= n && (size_t) ldp >= n, "column-major leading dimension < krnl_mat_size");
    CK(cudaSetDevice(im->device));
    TRY(ensure_io(im, 2 * n * n_vec));
    double* dX = im->d_io;
    double* dY = im->d_io + n * n_vec;
    cudaStream_t s = im->stream;
    const int* idx = forward ? im->d_fwd : im->d_bwd;
    if (layout == H2GPU_ROW_MAJOR)
    {
        CK(cudaMemcpy2DAsync(dX, 8 * (size_t) n_vec, X, 8 * (size_t) ldx, 8 * (size_t) n_vec, n, cudaMemcpyHostToDevice, s));
        CK(launch_permute(dX, n_vec, 1, idx, (int) n, n_vec, dY, n_vec, 1, s));
        CK(cudaMemcpy2DAsync(PX, 8 * (size_t) ldp, dY, 8 * (size_t) n_vec, 8 * (size_t) n_vec, n, cudaMemcpyDeviceToHost, s));
    } else {
        CK(cudaMemcpy2DAsync(dX, 8 * n, X, 8 * (size_t) ldx, 8 * n, n_vec, cudaMemcpyHostToDevice, s));
        CK(launch_permute(dX, 1, (long long) n, idx, (int) n, n_vec, dY, 1, (long long) n, s));
        CK(cudaMemcpy2DAsync(PX, 8 * (size_t) ldp, dY, 8 * n, 8 * n, n_vec, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    return H2GPU_OK;
}

H2G_API int h2gpu_permute_vector(h2gpu_image* im, int forward, const double* x, double* px)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    return h2gpu_permute_matrix_rows(im, forward, H2GPU_COL_MAJOR, 1, x, im->N, px, im->N);
}


H2G_API int h2gpu_get_blocks(h2gpu_image* im, int which, double* host, size_t n_elems)
{
    if (!im || !host) return fail(H2GPU_ERR_INVALID, "NULL argument");
    REQ(which == 0 || which == 1, "which must be 0 (B) or 1 (D)");
    std::lock_guard<std::mutex> lk(im->mu);
    const size_t n = which == 0 ? im->B_elems : im->D_elems;
    REQ(n_elems == n, "the image holds %zu elements of %s, not %zu", n, which == 0 ? "B" : "D", n_elems);
    if (n == 0) return H2GPU_OK;
    const double* d64 = which == 0 ? im->d_B64 : im->d_D64;
    const float* d32 = which == 0 ? im->d_B32 : im->d_D32;
    if (!d64 && !d32) return fail(H2GPU_ERR_STATE, "the image stores no blocks (JIT image)");
    CK(cudaSetDevice(im->device));
    if (d64)
    {
        CK(cudaMemcpy(host, d64, 8 * n, cudaMemcpyDeviceToHost));
        return H2GPU_OK;
    }
    // the FP32 arena (padded rows, blocks in order) in runs of whole blocks of up to 64 M
    // elements: copied to the host, widened and unpadded into H2Pack's packing
    const std::vector<h2gpu_image::BlkMap>& bm = im->bmap[which];
    const size_t cap = std::max<size_t>((size_t) 1 << 26, [&] {
        size_t m = 0;
        for (const auto& b : bm) m = std::max(m, (size_t) b.nrow * f32_ld(b.ncol));
        return m;
    }());
    std::vector<float> tmp(cap);
    int st = H2GPU_OK;
    for (size_t i0 = 0; i0 < bm.size() && st == H2GPU_OK;)
    {
        size_t i1 = i0, m = 0;
        while (i1 < bm.size() && m + (size_t) bm[i1].nrow * f32_ld(bm[i1].ncol) <= cap)
            m += (size_t) bm[i1].nrow * f32_ld(bm[i1].ncol), i1++;
        cudaError_t e = cudaMemcpy(tmp.data(), d32 + bm[i0].off32, 4 * m, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) { st = fail(H2GPU_ERR_CUDA, "block copy failed: %s", cudaGetErrorString(e)); break; }
        for (size_t i = i0; i < i1; i++)
        {
            const auto& b = bm[i];
            const int ld = f32_ld(b.ncol);
            const float* srow = tmp.data() + (b.off32 - bm[i0].off32);
            for (int r = 0; r < b.nrow; r++)
                for (int c = 0; c < b.ncol; c++) host[b.off64 + (long long) r * b.ncol + c] = srow[(long long) r * ld + c];
        }
        i0 = i1;
    }
    return st;
}

H2G_API int h2gpu_get_stats(h2gpu_image* im, h2gpu_stats* st)
{
    if (!im || !st) return fail(H2GPU_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(im->mu);
    *st = im->st;
    const double es = im->precision == H2GPU_PREC_MIXED ? 4.0 : 8.0;
    st->bytes_U = im->st.bytes_U * es;
    st->bytes_B = im->st.bytes_B * es;
    st->bytes_D = im->st.bytes_D * es;
    st->device_bytes = (long long) (im->bytes + im->work_bytes + 8 * im->io_elems);
    return H2GPU_OK;
}

H2G_API int h2gpu_reset_stats(h2gpu_image* im)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    std::lock_guard<std::mutex> lk(im->mu);
    im->st.n_matvec = 0;
    im->st.ms_total = 0;
    for (double& m : im->st.ms_phase) m = 0;
    return H2GPU_OK;
}

H2G_API int h2gpu_plan_check(const h2gpu_desc* desc, long long* counts)
{
    TRY(validate(desc));
    h2gpu_image* im = new h2gpu_image();   // plan fields only: no stream, event or allocation is made
    HostPlan hp;
    int st = build_plan(im, desc, hp);
    if (st == H2GPU_OK) st = check_plan(im, desc, hp, counts);
    delete im;
    return st;
}

H2G_API size_t h2gpu_image_bytes(const h2gpu_image* im)
{
    return im ? im->bytes + im->work_bytes + 8 * im->io_elems : 0;
}

H2G_API int h2gpu_measure_peaks(int device, double* fp32_tflops, double* mufu_tops)
{
    if (!fp32_tflops || !mufu_tops) return fail(H2GPU_ERR_INVALID, "NULL output");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(H2GPU_ERR_CUDA, "no CUDA device available");
    if (device < 0) CK(cudaGetDevice(&device));
    CK(cudaSetDevice(device));
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    float* out = nullptr;
    CK(cudaMalloc(&out, sizeof(float) * 148 * 64));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int st = H2GPU_OK;
    const int blocks = sms * 8, iters = 1 << 14;
    double res[2] = {0, 0};
    for (int which = 0; which < 2 && st == H2GPU_OK; which++)
    {
        float best = 1e30f;
        for (int rep = 0; rep < 4 && st == H2GPU_OK; rep++)      // first one warms up
        {
            cudaEventRecord(e0, 0);
            cudaError_t e = launch_peak(which, blocks, iters, out, 0);
            cudaEventRecord(e1, 0);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            if (e != cudaSuccess) { st = fail(H2GPU_ERR_CUDA, "peak kernel: %s", cudaGetErrorString(e)); break; }
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) best = std::min(best, ms);
        }
        const double ops = (double) blocks * 256 * iters * 8;      // chain steps
        res[which] = which == 0 ? ops * 4 / (best * 1e-3) / 1e12   // FFMA2: 2 FMA = 4 flop
                                : ops / (best * 1e-3) / 1e12;      // ex2 operations
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *fp32_tflops = res[0];
    *mufu_tops = res[1];
    return st;
}

H2G_API int h2gpu_direct_sum(int kernel_id, const double* krnl_param, int n_krnl_param, int xpt_dim, int krnl_dim,
                             const double* src_coord, int n_src, const double* src_val, const double* trg_coord,
                             int n_trg, double* trg_val)
{
    REQ(kernel_id >= H2GPU_KRNL_COULOMB && kernel_id <= H2GPU_KRNL_RPY, "bad kernel id %d", kernel_id);
    REQ((kernel_id == H2GPU_KRNL_RPY) == (krnl_dim == 3), "kernel id does not match krnl_dim");
    REQ(xpt_dim >= 3 && xpt_dim <= 4 && (kernel_id != H2GPU_KRNL_RPY || xpt_dim == 4), "bad xpt_dim");
    REQ(n_src > 0 && n_trg > 0 && src_coord && src_val && trg_coord && trg_val, "bad direct-sum arguments");
    REQ(kernel_id == H2GPU_KRNL_COULOMB || (krnl_param && n_krnl_param >= 1), "kernel needs a parameter");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(H2GPU_ERR_CUDA, "no CUDA device available for the direct sum");
    h2gpu_image tmp;
    tmp.kernel_id = kernel_id;
    tmp.n_kp = n_krnl_param;
    for (int i = 0; i < n_krnl_param && i < 4; i++) tmp.kp[i] = krnl_param[i];
    KParam kp = kparam_of(&tmp);
    auto pack = [&](const double* c, int n) {
        std::vector<double4> p(n);
        for (int i = 0; i < n; i++)
            p[i] = make_double4(c[i], c[(size_t) n + i], c[2 * (size_t) n + i], xpt_dim >= 4 ? c[3 * (size_t) n + i] : 0.0);
        return p;
    };
    std::vector<double4> hs = pack(src_coord, n_src), ht = pack(trg_coord, n_trg);
    double4 *ds = nullptr, *dt = nullptr;
    double *dv = nullptr, *dout = nullptr;
    int st = H2GPU_OK;
    do {
        if (cudaMalloc(&ds, sizeof(double4) * n_src) != cudaSuccess || cudaMalloc(&dt, sizeof(double4) * n_trg) != cudaSuccess ||
            cudaMalloc(&dv, 8 * (size_t) n_src * krnl_dim) != cudaSuccess ||
            cudaMalloc(&dout, 8 * (size_t) n_trg * krnl_dim) != cudaSuccess)
        { st = fail(H2GPU_ERR_NOMEM, "direct sum: device allocation failed"); break; }
        cudaMemcpy(ds, hs.data(), sizeof(double4) * n_src, cudaMemcpyHostToDevice);
        cudaMemcpy(dt, ht.data(), sizeof(double4) * n_trg, cudaMemcpyHostToDevice);
        cudaMemcpy(dv, src_val, 8 * (size_t) n_src * krnl_dim, cudaMemcpyHostToDevice);
        cudaError_t e = launch_direct(kernel_id, dt, n_trg, ds, n_src, dv, kp, dout, 0);
        if (e == cudaSuccess) e = cudaMemcpy(trg_val, dout, 8 * (size_t) n_trg * krnl_dim, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = fail(H2GPU_ERR_CUDA, "direct sum: %s", cudaGetErrorString(e));
    } while (0);
    cudaFree(ds); cudaFree(dt); cudaFree(dv); cudaFree(dout);
    return st;
}

// ============================================== construction: interpolative decompositions

H2G_API int h2gpu_id_batch(int kernel_id, const double* krnl_param, int n_krnl_param, double reltol, int n_blk,
                           const int* ncand, int npp, const double* cand, const double* prox, int* rank, int* perm,
                           double** E, long long* e_off)
{
    // E == NULL: skeletons only (no interpolation matrices, e_off unused)
    const int want_e = E != nullptr;
    if ((want_e && !e_off) || !rank || (n_blk > 0 && (!ncand || !cand || !perm)) || (npp > 0 && !prox) || n_blk < 0 ||
        npp < 0)
        return fail(H2GPU_ERR_INVALID, "bad h2gpu_id_batch arguments");
    if (want_e) *E = nullptr;
    REQ(kernel_id == H2GPU_KRNL_COULOMB || kernel_id == H2GPU_KRNL_GAUSSIAN || kernel_id == H2GPU_KRNL_MATERN32,
        "interpolative decompositions on the GPU take the scalar kernels (id %d)", kernel_id);
    REQ(kernel_id == H2GPU_KRNL_COULOMB || (n_krnl_param >= 1 && krnl_param), "kernel parameter missing");
    REQ(reltol > 0.0, "reltol must be positive");
    int max_nc = 0;
    for (int b = 0; b < n_blk; b++)
    {
        REQ(ncand[b] >= 0, "block %d: negative size", b);
        max_nc = std::max(max_nc, ncand[b]);
    }
    // Blocks decomposed alone by the grid-wide QR: those whose work space exceeds the
    // shared memory of one CTA, and large blocks (>= 2^20 entries) of a level with too
    // few of them to fill the GPU one CTA each (one SM would stream each one's trailing
    // matrix per pivot step).
    auto big = [&](int b) { return (long long) ncand[b] * npp >= (1LL << 20); };
    int n_big = 0;
    for (int b = 0; b < n_blk; b++) n_big += big(b);
    auto solo = [&](int b) {
        return id_qr_smem_bytes(ncand[b], npp) > 200 * 1024 || (big(b) && n_big < 64);
    };
    if (npp == 0 || max_nc == 0)
    {
        // no proxy points (levels without admissible pairs) or no candidates: rank 0
        long long o = 0;
        if (want_e) e_off[0] = 0;
        for (int b = 0; b < n_blk; b++)
        {
            rank[b] = 0;
            for (int j = 0; j < ncand[b]; j++) perm[o + j] = j;
            o += ncand[b];
            if (want_e) e_off[b + 1] = 0;
        }
        if (!want_e) return H2GPU_OK;
        *E = (double*) malloc(8);
        return *E ? H2GPU_OK : fail(H2GPU_ERR_NOMEM, "host buffer of the interpolation matrices");
    }
    int caller_dev = 0;
    CK(cudaGetDevice(&caller_dev));
    const KParam kp = kparam_from(kernel_id, krnl_param, n_krnl_param);
    // chunks of blocks whose workspaces (ncand x npp doubles each) stay within 4 GB
    std::vector<long long> coff(n_blk + 1, 0);
    for (int b = 0; b < n_blk; b++) coff[b + 1] = coff[b] + ncand[b];
    std::vector<int> rk(n_blk, 0);
    double* d_prox = nullptr;
    int st = H2GPU_OK;
    auto cuda_fail = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess && st == H2GPU_OK)
            st = fail(e == cudaErrorMemoryAllocation ? H2GPU_ERR_NOMEM : H2GPU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
        return e != cudaSuccess;
    };
    if (npp > 0 && !cuda_fail(cudaMalloc(&d_prox, 8 * 3 * (size_t) npp), "proxy upload"))
        cuda_fail(cudaMemcpy(d_prox, prox, 8 * 3 * (size_t) npp, cudaMemcpyHostToDevice), "proxy upload");
    std::vector<std::vector<double>> Eb(n_blk);
    const long long budget = 4LL << 27;   // doubles (4 GB)
    for (int b0 = 0; b0 < n_blk && st == H2GPU_OK;)
    {
        int b1 = b0;
        long long w = 0;
        const bool alone = solo(b0) && ncand[b0] > 0;
        if (alone)
            b1 = b0 + 1;
        else
            while (b1 < n_blk && (b1 == b0 || (w + (long long) ncand[b1] * npp <= budget && !solo(b1))))
                w += (long long) ncand[b1++] * npp;
        std::vector<IdBlock> blks(b1 - b0);
        std::vector<double> cc(3 * (size_t) (coff[b1] - coff[b0]));
        long long wo = 0;
        int mx = 0;
        for (int b = b0; b < b1; b++)
        {
            IdBlock& B = blks[b - b0];
            B.ncand = ncand[b]; B.npp = npp;
            B.cand_off = 3 * (coff[b] - coff[b0]); B.prox_off = 0; B.w_off = wo; B.perm_off = coff[b] - coff[b0];
            wo += (long long) ncand[b] * npp;
            mx = std::max(mx, ncand[b]);
            memcpy(&cc[B.cand_off], cand + 3 * coff[b], 8 * 3 * (size_t) ncand[b]);
        }
        if (mx == 0)   // only blocks without candidates: rank 0
        {
            for (int b = b0; b < b1; b++) rk[b] = 0;
            b0 = b1;
            continue;
        }
        IdBlock* d_blk = nullptr;
        double *d_cand = nullptr, *d_W = nullptr;
        int *d_rank = nullptr, *d_perm = nullptr;
        void* d_work = nullptr;
        const size_t nperm = (size_t) (coff[b1] - coff[b0]);
        auto decompose = [&]() {
            if (!alone)
                return launch_id(kernel_id, d_blk, (int) blks.size(), mx, npp, d_cand, d_prox, kp, d_W, reltol, d_rank,
                                 d_perm, 0, want_e);
            int sms = 0;
            cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, caller_dev);
            if (e == cudaSuccess) e = cudaMalloc(&d_work, qr_grid_work_bytes(npp, mx));
            if (e == cudaSuccess) e = launch_id_eval(kernel_id, d_blk, 1, mx, d_cand, d_prox, kp, d_W, 0);
            if (e == cudaSuccess) e = launch_qr_grid(d_W, npp, mx, reltol, d_work, d_rank, d_perm, sms, want_e, 0);
            return e;
        };
        if (!cuda_fail(cudaMalloc(&d_blk, sizeof(IdBlock) * blks.size()), "work space") &&
            !cuda_fail(cudaMalloc(&d_cand, 8 * std::max<size_t>(cc.size(), 1)), "work space") &&
            !cuda_fail(cudaMalloc(&d_W, 8 * (size_t) std::max<long long>(wo, 1)), "work space") &&
            !cuda_fail(cudaMalloc(&d_rank, 4 * blks.size()), "work space") &&
            !cuda_fail(cudaMalloc(&d_perm, 4 * std::max<size_t>(nperm, 1)), "work space") &&
            !cuda_fail(cudaMemcpy(d_blk, blks.data(), sizeof(IdBlock) * blks.size(), cudaMemcpyHostToDevice), "upload") &&
            !cuda_fail(cc.empty() ? cudaSuccess : cudaMemcpy(d_cand, cc.data(), 8 * cc.size(), cudaMemcpyHostToDevice), "upload") &&
            !cuda_fail(decompose(), "interpolative decomposition") &&
            !cuda_fail(cudaMemcpy(rk.data() + b0, d_rank, 4 * blks.size(), cudaMemcpyDeviceToHost), "download") &&
            !cuda_fail(nperm ? cudaMemcpy(perm + coff[b0], d_perm, 4 * nperm, cudaMemcpyDeviceToHost) : cudaSuccess, "download"))
        {
            // E of block b: columns r .. n-1 of R (column stride npp), rows 0 .. r-1
            for (int b = b0; b < b1 && st == H2GPU_OK && want_e; b++)
            {
                const int r = rk[b], n = ncand[b];
                if (r == 0 || r == n) continue;
                Eb[b].resize((size_t) r * (n - r));
                cuda_fail(cudaMemcpy2D(Eb[b].data(), 8 * (size_t) r, d_W + blks[b - b0].w_off + (long long) r * npp,
                                       8 * (size_t) npp, 8 * (size_t) r, (size_t) (n - r), cudaMemcpyDeviceToHost),
                          "download");
            }
        }
        for (void* p : {(void*) d_blk, (void*) d_cand, (void*) d_W, (void*) d_rank, (void*) d_perm, d_work})
            if (p) cudaFree(p);
        b0 = b1;
    }
    if (d_prox) cudaFree(d_prox);
    cudaSetDevice(caller_dev);
    if (st != H2GPU_OK) return st;
    for (int b = 0; b < n_blk; b++) rank[b] = rk[b];
    if (!want_e) return H2GPU_OK;
    e_off[0] = 0;
    for (int b = 0; b < n_blk; b++) e_off[b + 1] = e_off[b] + (long long) rk[b] * (ncand[b] - rk[b]);
    double* out = (double*) malloc(8 * (size_t) std::max<long long>(e_off[n_blk], 1));
    if (!out) return fail(H2GPU_ERR_NOMEM, "host buffer of the interpolation matrices");
    for (int b = 0; b < n_blk; b++)
        if (!Eb[b].empty()) memcpy(out + e_off[b], Eb[b].data(), 8 * Eb[b].size());
    *E = out;
    return H2GPU_OK;
}

H2G_API void h2gpu_free(void* p) { free(p); }

H2G_API int h2gpu_pp_sketch_id(int kernel_id, const double* krnl_param, int n_krnl_param, double reltol, int nx,
                               const double* X0, int ny, const double* Y0, const int* st_rowptr, const int* st_col,
                               const double* st_val, int* rank, int* perm)
{
    if (nx <= 0 || ny <= 0 || !X0 || !Y0 || !st_rowptr || !st_col || !st_val || !rank || !perm)
        return fail(H2GPU_ERR_INVALID, "bad h2gpu_pp_sketch_id arguments");
    REQ(kernel_id == H2GPU_KRNL_COULOMB || kernel_id == H2GPU_KRNL_GAUSSIAN || kernel_id == H2GPU_KRNL_MATERN32,
        "proxy points on the GPU take the scalar kernels (id %d)", kernel_id);
    REQ(kernel_id == H2GPU_KRNL_COULOMB || (n_krnl_param >= 1 && krnl_param), "kernel parameter missing");
    REQ(reltol > 0.0, "reltol must be positive");
    const long long nnz = st_rowptr[nx];
    REQ(st_rowptr[0] == 0 && nnz >= 0, "bad CSR row pointer");
    for (int c = 0; c < nx; c++) REQ(st_rowptr[c + 1] >= st_rowptr[c], "bad CSR row pointer");
    for (long long p = 0; p < nnz; p++) REQ(st_col[p] >= 0 && st_col[p] < ny, "CSR column %lld out of range", p);
    int caller_dev = 0;
    CK(cudaGetDevice(&caller_dev));
    struct DeviceRestore {
        int dev;
        ~DeviceRestore() { cudaSetDevice(dev); }
    } restore{caller_dev};
    const KParam kp = kparam_from(kernel_id, krnl_param, n_krnl_param);
    double *dX = nullptr, *dY = nullptr, *dv = nullptr, *dW = nullptr;
    int *drp = nullptr, *dc = nullptr, *drank = nullptr, *dperm = nullptr;
    void* dwork = nullptr;
    int sms = 0;
    cudaError_t e = cudaSuccess;
    auto step = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    step(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, caller_dev));
    step(cudaMalloc(&dX, 8 * 3 * (size_t) nx));
    step(cudaMalloc(&dY, 8 * 3 * (size_t) ny));
    step(cudaMalloc(&drp, 4 * (size_t) (nx + 1)));
    step(cudaMalloc(&dc, 4 * (size_t) std::max<long long>(nnz, 1)));
    step(cudaMalloc(&dv, 8 * (size_t) std::max<long long>(nnz, 1)));
    step(cudaMalloc(&dW, 8 * (size_t) nx * nx));
    step(cudaMalloc(&drank, 4));
    step(cudaMalloc(&dperm, 4 * (size_t) nx));
    step(cudaMalloc(&dwork, qr_grid_work_bytes(nx, nx)));
    if (e == cudaSuccess)
    {
        step(cudaMemcpy(dX, X0, 8 * 3 * (size_t) nx, cudaMemcpyHostToDevice));
        step(cudaMemcpy(dY, Y0, 8 * 3 * (size_t) ny, cudaMemcpyHostToDevice));
        step(cudaMemcpy(drp, st_rowptr, 4 * (size_t) (nx + 1), cudaMemcpyHostToDevice));
        if (nnz > 0) step(cudaMemcpy(dc, st_col, 4 * (size_t) nnz, cudaMemcpyHostToDevice));
        if (nnz > 0) step(cudaMemcpy(dv, st_val, 8 * (size_t) nnz, cudaMemcpyHostToDevice));
        step(launch_pp_sketch(kernel_id, nx, dX, ny, dY, drp, dc, dv, kp, dW, 0));
        // one nx x nx matrix: the pivoted QR spread over the whole GPU
        step(launch_qr_grid(dW, nx, nx, reltol, dwork, drank, dperm, sms, 0, 0));
        step(cudaMemcpy(rank, drank, 4, cudaMemcpyDeviceToHost));
        step(cudaMemcpy(perm, dperm, 4 * (size_t) nx, cudaMemcpyDeviceToHost));
    }
    for (void* p : {(void*) dX, (void*) dY, (void*) drp, (void*) dc, (void*) dv, (void*) dW, (void*) drank,
                    (void*) dperm, dwork})
        if (p) cudaFree(p);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? H2GPU_ERR_NOMEM : H2GPU_ERR_CUDA, "proxy-point sketch: %s",
                    cudaGetErrorString(e));
    return H2GPU_OK;
}

// ================================================== apply without allocation
//
// h2gpu_matvec_device_noalloc: y = A x for one device-resident vector, with every
// work buffer (input space, partial sums, y1 sums, push-down) taken from the fixed
// device array below instead of cudaMalloc.  For callers that cannot allocate device
// memory at apply time: code whose device memory is owned entirely by another
// allocator (a framework's caching allocator or a pool reserved up front, where a
// direct cudaMalloc fails or fragments memory), and code that must not stall, since
// cudaMalloc / cudaFree synchronize the device.  The image itself is created
// beforehand, at set-up, where allocation is allowed.
//
// Limit: the work buffers of one right-hand side must fit in
// H2GPU_NOALLOC_SCRATCH_DOUBLES doubles (16 MiB); larger images are rejected with
// H2GPU_ERR_INVALID.  The array is a static device symbol, so every GPU that loads
// the library holds these 16 MiB until the process exits.  Every call shares it and
// it keeps the last call's contents: nothing needs clearing (each value read within a
// call is written earlier in the same call), but calls that overlap on the GPU
// (different streams, or different host threads on the same device) race on it.
// The first call on a device looks up the array's device address with that device
// current (cudaGetSymbolAddress), so that first call should come before any stream
// capture.  A mixed-precision image applies FP32 copies of U/B/D that its first
// allocating apply (h2gpu_matvec, h2gpu_matmul, h2gpu_matmul_device) creates; until
// then this entry point refuses it with H2GPU_ERR_STATE.  The caller's current device
// is left as it was.

#define H2GPU_NOALLOC_SCRATCH_DOUBLES (2u * 1024u * 1024u)

static __device__ __align__(256) double g_noalloc_scratch[H2GPU_NOALLOC_SCRATCH_DOUBLES];

namespace {

std::mutex g_noalloc_mu;
double* g_noalloc_addr[64] = {};

// Device address of the scratch array for `dev` (the current device), looked up once.
int noalloc_scratch(int dev, double** out)
{
    if (dev < 0 || dev >= 64) return fail(H2GPU_ERR_INVALID, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (g_noalloc_addr[dev] == nullptr)
    {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            return fail(H2GPU_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed: %s", cudaGetErrorString(e));
        g_noalloc_addr[dev] = (double*) p;
    }
    *out = g_noalloc_addr[dev];
    return H2GPU_OK;
}

}  // namespace

H2G_API int h2gpu_matvec_device_noalloc(h2gpu_image* im, const double* d_x, double* d_y, void* stream)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    REQ(d_x && d_y, "device vectors are NULL");
    std::lock_guard<std::mutex> lk(im->mu);
    // the caller's current device is restored on every return
    int caller_dev = -1;
    CK(cudaGetDevice(&caller_dev));
    struct DeviceRestore {
        int dev;
        ~DeviceRestore() { cudaSetDevice(dev); }
    } restore{caller_dev};
    CK(cudaSetDevice(im->device));
    if (im->precision == H2GPU_PREC_MIXED &&
        ((im->U_elems && !im->d_U32) || (im->B_elems && !im->d_B32) || (im->D_elems && !im->d_D32)))
        return fail(H2GPU_ERR_STATE, "the FP32 copies of this image are created by its first allocating apply "
                                     "in mixed precision; run one h2gpu_matmul_device call first or use FP64");
    const unsigned long long xs = (unsigned long long) im->N + im->y0_rows, ps = im->ps_rows, y1 = im->y0_rows;
    const unsigned long long need = xs + ps + 2 * y1;
    if (need > H2GPU_NOALLOC_SCRATCH_DOUBLES)
        return fail(H2GPU_ERR_INVALID, "image needs %llu doubles of work space per right-hand side; the "
                                       "no-allocation apply is limited to %u (16 MiB)", need,
                    (unsigned) H2GPU_NOALLOC_SCRATCH_DOUBLES);
    double* base = nullptr;
    TRY(noalloc_scratch(im->device, &base));
    cudaStream_t s = stream ? (cudaStream_t) stream : im->stream;
    // run the regular panel sequence on the scratch buffers
    double* keep[4] = {im->d_XS, im->d_PS, im->d_Y1, im->d_PUSH};
    im->d_XS = base;
    im->d_PS = base + xs;
    im->d_Y1 = base + xs + ps;
    im->d_PUSH = base + xs + ps + y1;
    int st = run_panel(im, 1, 1, d_x, 1, 0, d_y, 1, 0, s, false);
    im->d_XS = keep[0]; im->d_PS = keep[1]; im->d_Y1 = keep[2]; im->d_PUSH = keep[3];
    if (st == H2GPU_OK) im->st.n_matvec += 1;
    return st;
}

// ============================================================ batched images
//
// A batch of independent H2 representations (same kernel, precision and mode) is
// applied as one: their descriptors are merged into one forest -- node, point and
// block indices offset, per-level node lists concatenated, B/D blocks re-packed
// diagonal blocks first -- so every phase is one launch per tree level over all
// matrices of the batch (flattened cross-matrix work lists).  The caller stacks the
// matrices' vectors in batch order.

namespace {

struct MergedDesc {
    h2gpu_desc d{};
    std::vector<int> n_child, children, node_level, pt_cluster, mat_cluster, level_n_node, level_nodes, leaf_nodes,
        U_nrow, U_ncol, U_ld, r_adm, r_inadm, B_nrow, B_ncol, D_nrow, D_ncol, J_n, fwd, bwd;
    std::vector<size_t> B_ptr, D_ptr;
    std::vector<double> B_data, D_data, coord;
    std::vector<const double*> U, J;
};

int merge_descs(const h2gpu_desc* ds, int n, MergedDesc& m)
{
    REQ(ds && n >= 1, "empty batch");
    const h2gpu_desc& a = ds[0];
    int n_point = 0, n_node = 0, n_leaf = 0, max_level = 0, min_adm = 1 << 30, nadm = 0, ninadm = 0;
    for (int i = 0; i < n; i++)
    {
        TRY(validate(&ds[i]));
        const h2gpu_desc& d = ds[i];
        REQ(d.krnl_dim == a.krnl_dim && d.xpt_dim == a.xpt_dim && d.BD_JIT == a.BD_JIT && d.kernel_id == a.kernel_id &&
                d.n_krnl_param == a.n_krnl_param,
            "batch member %d differs in kernel, dimension or mode", i);
        for (int k = 0; k < d.n_krnl_param; k++) REQ(d.krnl_param[k] == a.krnl_param[k], "batch member %d: kernel parameter differs", i);
        n_point += d.n_point; n_node += d.n_node; n_leaf += d.n_leaf_node;
        max_level = std::max(max_level, d.max_level);
        min_adm = std::min(min_adm, d.min_adm_level);
        nadm += d.n_r_adm_pair; ninadm += d.n_r_inadm_pair;
    }
    const int kd = a.krnl_dim, L = max_level + 1;
    REQ((long long) kd * n_point < (1LL << 30), "batch too large for 32-bit row indices");
    m.level_n_node.assign(L, 0);
    m.level_nodes.assign((size_t) L * n_leaf, 0);
    std::vector<int> lfill(L, 0);
    int no = 0, po = 0;
    size_t bo = 0;
    // first pass: node-indexed arrays, pairs, coordinates
    m.coord.assign((size_t) a.xpt_dim * n_point, 0.0);
    for (int i = 0; i < n; i++)
    {
        const h2gpu_desc& d = ds[i];
        for (int v = 0; v < d.n_node; v++)
        {
            m.n_child.push_back(d.n_child[v]);
            for (int k = 0; k < d.max_child; k++)
                m.children.push_back(k < d.n_child[v] ? d.children[v * d.max_child + k] + no : -1);
            m.node_level.push_back(d.node_level[v]);
            m.pt_cluster.push_back(d.pt_cluster[2 * v] + po);
            m.pt_cluster.push_back(d.pt_cluster[2 * v + 1] + po);
            m.mat_cluster.push_back(d.mat_cluster[2 * v] + kd * po);
            m.mat_cluster.push_back(d.mat_cluster[2 * v + 1] + kd * po);
            m.U_nrow.push_back(d.U_nrow[v]); m.U_ncol.push_back(d.U_ncol[v]); m.U_ld.push_back(d.U_ld[v]);
            m.U.push_back(d.U[v]);
            m.J_n.push_back(d.J_n ? d.J_n[v] : 0);
            m.J.push_back(d.J_coord ? d.J_coord[v] : nullptr);
        }
        for (int l = 0; l <= d.max_level; l++)
            for (int j = 0; j < d.level_n_node[l]; j++)
                m.level_nodes[(size_t) l * n_leaf + lfill[l]++] = d.level_nodes[(size_t) l * d.n_leaf_node + j] + no;
        for (int j = 0; j < d.n_leaf_node; j++) m.leaf_nodes.push_back(d.leaf_nodes[j] + no);
        for (int j = 0; j < 2 * d.n_r_adm_pair; j++) m.r_adm.push_back(d.r_adm_pairs[j] + no);
        for (int j = 0; j < 2 * d.n_r_inadm_pair; j++) m.r_inadm.push_back(d.r_inadm_pairs[j] + no);
        if (d.coord)
            for (int k = 0; k < a.xpt_dim; k++)
                memcpy(&m.coord[(size_t) k * n_point + po], d.coord + (size_t) k * d.n_point, 8 * (size_t) d.n_point);
        for (int j = 0; j < kd * d.n_point; j++)
        {
            m.fwd.push_back(d.fwd_pmt_idx[j] + kd * po);
            m.bwd.push_back(d.bwd_pmt_idx[j] + kd * po);
        }
        no += d.n_node; po += d.n_point;
    }
    for (int l = 0; l < L; l++) m.level_n_node[l] = lfill[l];
    // B / D blocks: B in member order; D diagonal blocks of all members first, then the others
    if (!a.BD_JIT)
    {
        m.B_ptr.push_back(0);
        for (int i = 0; i < n; i++)
        {
            const h2gpu_desc& d = ds[i];
            for (int j = 0; j < d.n_B; j++)
            {
                m.B_nrow.push_back(d.B_nrow[j]); m.B_ncol.push_back(d.B_ncol[j]);
                size_t sz = d.B_ptr[j + 1] - d.B_ptr[j];
                m.B_data.insert(m.B_data.end(), d.B_data + d.B_ptr[j], d.B_data + d.B_ptr[j] + sz);
                bo += sz;
                m.B_ptr.push_back(bo);
            }
        }
        m.D_ptr.push_back(0);
        size_t dofs = 0;
        for (int pass = 0; pass < 2; pass++)
            for (int i = 0; i < n; i++)
            {
                const h2gpu_desc& d = ds[i];
                int j0 = pass == 0 ? 0 : d.n_leaf_node, j1 = pass == 0 ? d.n_leaf_node : d.n_D;
                for (int j = j0; j < j1; j++)
                {
                    m.D_nrow.push_back(d.D_nrow[j]); m.D_ncol.push_back(d.D_ncol[j]);
                    size_t sz = d.D_ptr[j + 1] - d.D_ptr[j];
                    m.D_data.insert(m.D_data.end(), d.D_data + d.D_ptr[j], d.D_data + d.D_ptr[j] + sz);
                    dofs += sz;
                    m.D_ptr.push_back(dofs);
                }
            }
    } else {
        m.B_ptr.assign(1, 0);
        m.D_ptr.assign(1, 0);
    }
    h2gpu_desc& d = m.d;
    d.n_point = n_point; d.pt_dim = a.pt_dim; d.xpt_dim = a.xpt_dim; d.krnl_dim = kd;
    d.n_node = n_node; d.n_leaf_node = n_leaf; d.max_child = a.max_child; d.max_level = max_level;
    d.min_adm_level = min_adm; d.BD_JIT = a.BD_JIT;
    d.n_child = m.n_child.data(); d.children = m.children.data(); d.node_level = m.node_level.data();
    d.pt_cluster = m.pt_cluster.data(); d.mat_cluster = m.mat_cluster.data();
    d.level_n_node = m.level_n_node.data(); d.level_nodes = m.level_nodes.data(); d.leaf_nodes = m.leaf_nodes.data();
    d.U_nrow = m.U_nrow.data(); d.U_ncol = m.U_ncol.data(); d.U_ld = m.U_ld.data(); d.U = m.U.data();
    d.n_r_adm_pair = nadm; d.r_adm_pairs = m.r_adm.data();
    d.n_r_inadm_pair = ninadm; d.r_inadm_pairs = m.r_inadm.data();
    d.n_B = a.BD_JIT ? nadm : (int) m.B_nrow.size();
    d.B_nrow = m.B_nrow.data(); d.B_ncol = m.B_ncol.data(); d.B_ptr = m.B_ptr.data();
    d.B_data = m.B_data.empty() ? nullptr : m.B_data.data();
    d.n_D = n_leaf + ninadm;
    d.D_nrow = m.D_nrow.data(); d.D_ncol = m.D_ncol.data(); d.D_ptr = m.D_ptr.data();
    d.D_data = m.D_data.empty() ? nullptr : m.D_data.data();
    d.coord = m.coord.data(); d.J_n = m.J_n.data(); d.J_coord = m.J.data();
    d.fwd_pmt_idx = m.fwd.data(); d.bwd_pmt_idx = m.bwd.data();
    d.kernel_id = a.kernel_id; d.n_krnl_param = a.n_krnl_param;
    for (int k = 0; k < 4; k++) d.krnl_param[k] = a.krnl_param[k];
    return H2GPU_OK;
}

}  // namespace

H2G_API int h2gpu_batch_plan_check(const h2gpu_desc* descs, int n_desc, long long* counts)
{
    MergedDesc m;
    TRY(merge_descs(descs, n_desc, m));
    return h2gpu_plan_check(&m.d, counts);
}

H2G_API int h2gpu_batch_create(const h2gpu_desc* descs, int n_desc, const h2gpu_options* opt, h2gpu_image** out)
{
    if (!out) return fail(H2GPU_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (opt && opt->blocks != H2GPU_BLOCKS_GIVEN)
        return fail(H2GPU_ERR_UNSUPPORTED, "batched images take their blocks as given");
    MergedDesc m;
    TRY(merge_descs(descs, n_desc, m));
    TRY(h2gpu_image_create(&m.d, opt, out));
    (*out)->n_images = n_desc;
    return H2GPU_OK;
}

// ================================================================ CUDA graph

H2G_API int h2gpu_graph_capture(h2gpu_image* im, int n_vec, const double* dX, int ldx, double* dY, int ldy)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    REQ(n_vec >= 1 && ldx >= n_vec && ldy >= n_vec && dX && dY, "bad graph_capture arguments");
    std::lock_guard<std::mutex> lk(im->mu);
    int NV = panel_width(n_vec, panel_cap(im));
    if (im->tuned_nv > 0) NV = std::min(NV, im->tuned_nv);
    TRY(prepare(im, NV));
    if (im->graph_exec) { cudaGraphExecDestroy(im->graph_exec); im->graph_exec = nullptr; }
    if (im->graph) { cudaGraphDestroy(im->graph); im->graph = nullptr; }
    cudaStream_t s = im->stream;
    // one eager pass first so that every kernel attribute is set outside the capture
    for (int c0 = 0; c0 < n_vec; c0 += NV)
        TRY(run_panel(im, NV, std::min(NV, n_vec - c0), dX + c0, ldx, 1, dY + c0, ldy, 1, s, false));
    CK(cudaStreamSynchronize(s));
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    int st = H2GPU_OK;
    for (int c0 = 0; c0 < n_vec && st == H2GPU_OK; c0 += NV)
        st = run_panel(im, NV, std::min(NV, n_vec - c0), dX + c0, ldx, 1, dY + c0, ldy, 1, s, false);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (st != H2GPU_OK) { if (g) cudaGraphDestroy(g); return st; }
    if (e != cudaSuccess) return fail(H2GPU_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&im->graph_exec, g, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return fail(H2GPU_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e)); }
    im->graph = g;
    im->st.n_matvec += 0;
    return H2GPU_OK;
}

H2G_API int h2gpu_graph_launch(h2gpu_image* im, void* stream)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    std::lock_guard<std::mutex> lk(im->mu);
    if (!im->graph_exec) return fail(H2GPU_ERR_STATE, "no graph captured (call h2gpu_graph_capture first)");
    CK(cudaGraphLaunch(im->graph_exec, stream ? (cudaStream_t) stream : im->stream));
    return H2GPU_OK;
}

static void set_variant(h2gpu_image* im, int variant)
{
    im->jit_tc = variant != H2GPU_JIT_SIMT;
    im->jit_pair = variant == H2GPU_JIT_PAIR;
    im->blk_tc = variant == H2GPU_JIT_SIMT ? 0 : (variant == H2GPU_BLK_TCGEN05 ? 2 : 1);
}

H2G_API int h2gpu_set_jit_variant(h2gpu_image* im, int variant)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    REQ(variant == H2GPU_JIT_SIMT || variant == H2GPU_JIT_TC || variant == H2GPU_JIT_PAIR ||
            variant == H2GPU_BLK_TCGEN05, "unknown kernel variant %d", variant);
    if (variant == H2GPU_JIT_PAIR && !im->has_pair)
        return fail(H2GPU_ERR_UNSUPPORTED, "the pair variant needs a JIT image of a scalar kernel");
    if (variant == H2GPU_BLK_TCGEN05 && im->BD_JIT)
        return fail(H2GPU_ERR_UNSUPPORTED, "the tcgen05 variant applies to stored-block images");
    std::lock_guard<std::mutex> lk(im->mu);
    set_variant(im, variant);
    return H2GPU_OK;
}

// ================================================================= autotuner
//
// Times the apply of n_vec device-resident right-hand sides under each candidate
// (panel width among 4, 8, 16 not above n_vec's panel; for FP32 JIT images the
// CUDA-core, tensor-core and pair tensor-core kernels) and keeps the fastest.

H2G_API int h2gpu_autotune(h2gpu_image* im, int n_vec, const double* dX, int ldx, double* dY, int ldy, int* best_nv,
                           int* best_variant)
{
    if (!im) return fail(H2GPU_ERR_INVALID, "image is NULL");
    REQ(n_vec >= 1 && ldx >= n_vec && ldy >= n_vec && dX && dY, "bad autotune arguments");
    std::lock_guard<std::mutex> lk(im->mu);
    const int full = panel_width(n_vec, panel_cap(im));
    std::vector<int> nvs;
    for (int w = 1; w <= full; w <<= 1)
        if (w == full || w >= 4) nvs.push_back(w);
    auto variant = [&]() {
        if (!im->BD_JIT) return im->blk_tc == 2 ? H2GPU_BLK_TCGEN05 : (im->blk_tc ? H2GPU_JIT_TC : H2GPU_JIT_SIMT);
        return im->jit_tc ? (im->jit_pair ? H2GPU_JIT_PAIR : H2GPU_JIT_TC) : H2GPU_JIT_SIMT;
    };
    std::vector<int> vars = {variant()};
    if (im->precision == H2GPU_PREC_MIXED && (!im->BD_JIT || im->kd == 1))
    {
        vars = {H2GPU_JIT_TC, H2GPU_JIT_SIMT};
        if (im->BD_JIT && im->has_pair) vars.push_back(H2GPU_JIT_PAIR);
        if (!im->BD_JIT) vars.push_back(H2GPU_BLK_TCGEN05);
    }
    float best = 1e30f;
    int bnv = full, bvar = variant();
    cudaEvent_t* e = im->ev.e;
    for (int nv : nvs)
        for (int var : vars)
        {
            // wide panels (32 / 64) have one kernel whatever the variant: time them once
            if (nv >= 32 && var != vars[0]) continue;
            if (nv < 32 && (var == H2GPU_JIT_PAIR || var == H2GPU_BLK_TCGEN05) && nv != 8 && nv != 16) continue;
            // the tensor-core kernels exist for panels of 8 and 16; narrower panels run
            // the CUDA-core kernel whatever the variant, so time that once
            if (nv < 32 && var == H2GPU_JIT_TC && nv != 8 && nv != 16 && vars.size() > 1) continue;
            set_variant(im, var);
            TRY(prepare(im, nv));
            float ms = 0;
            for (int rep = 0; rep < 2; rep++)
            {
                CK(cudaEventRecord(e[7], im->stream));
                for (int c0 = 0; c0 < n_vec; c0 += nv)
                    TRY(run_panel(im, nv, std::min(nv, n_vec - c0), dX + c0, ldx, 1, dY + c0, ldy, 1, im->stream, false));
                CK(cudaEventRecord(e[6], im->stream));
                CK(cudaEventSynchronize(e[6]));
                CK(cudaEventElapsedTime(&ms, e[7], e[6]));
            }
            if (ms < best) { best = ms; bnv = nv; bvar = var; }
        }
    im->tuned_nv = bnv;
    set_variant(im, bvar);
    TRY(check_status(im));
    if (best_nv) *best_nv = bnv;
    if (best_variant) *best_variant = bvar;
    return H2GPU_OK;
}

// ------------------------------------------------ hooks for the CG engine (h2gpu_solve.cu)

namespace h2gpu {

int set_error(int code, const char* msg) { return fail(code, "%s", msg); }

int image_apply_quiet(h2gpu_image* im, int precision, int n_vec, const double* dX, int ldx, double* dY, int ldy)
{
    std::lock_guard<std::mutex> lk(im->mu);
    if (cudaSetDevice(im->device) != cudaSuccess) return fail(H2GPU_ERR_CUDA, "cudaSetDevice failed");
    return apply_quiet(im, precision, n_vec, dX, ldx, dY, ldy, im->stream);
}

int image_info(const h2gpu_image* im, int* N, int* device, int* precision, void** stream)
{
    *N = im->N;
    *device = im->device;
    *precision = im->precision;
    *stream = (void*) im->stream;
    return H2GPU_OK;
}

}  // namespace h2gpu
