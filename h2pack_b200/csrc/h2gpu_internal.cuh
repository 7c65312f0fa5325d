// h2gpu_internal.cuh -- device-side data layout and task records of the H2 apply engine.
//
// Vector spaces.  Every vector space is a matrix of `rows` x NV (row-major, the
// right-hand sides of one row contiguous, NV = panel width):
//   XS   input space:   rows [0, N)        the forward-permuted input (N = krnl_mat_size)
//                       rows [N, N+Y0)     y0 = U^T x of every node, laid out so that the
//                                          children of a node are contiguous in child order
//                                          (the upward input of a non-leaf node is then one slice)
//   PS   partial space: disjoint slots written by the block tasks; every output row is
//                       the sum of its slots in a fixed order (deterministic, no atomics)
//   PUSH downward push: rows indexed like the y0 region; a non-leaf node writes
//                       U_node * y1_node there and each child reads its own slice
// This replaces the reference's per-thread y copies and y1 rows (src/H2Pack_matvec.c:234-300,
// :1191-1263) and the H2P_dense_mat y0/y1 arrays (src/H2Pack_typedef.h:171-172).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace h2gpu {

// Upward task, one tile of <= 64 columns of a node's U:
//   XS[out_row + c][v] = sum_r U[r][c] * XS[in_row + r][v],  c0 <= c < c0 + nc
// (H2P_matvec_fwd_transform, src/H2Pack_matvec.c:126-156)
// U arena: every node's U row-major with its row stride rounded up to a multiple of 4
// elements (zero padding) and its offset a multiple of 4, so that 16-byte loads of FP32
// rows are aligned.
struct UpTask {
    long long u_off;   // element offset of the node's U in the U arena (row-major)
    int nrow, ld;      // rows of U, row stride (columns of U rounded up to a multiple of 4)
    int c0, nc;        // column tile
    int in_row;        // leaf: first row of its x slice; non-leaf: y0 row of its first child
    int out_row;       // y0 row of the node
};

// Downward task (a chunk of <= 64 rows of U):  t = U[rows] * y1t,
//   y1t[c][v] = Y1[y1_row + c][v] + PUSH[push_row + c][v]   (absent terms are zero)
// (H2P_matvec_bwd_transform, src/H2Pack_matvec.c:806-841)
struct DownTask {
    long long u_off;          // element offset of the chunk's first row of U
    int nrow, ncol;
    int ld;                   // row stride of U (as UpTask::ld)
    int y1_row;               // -1: the node has no admissible-pair contributions
    int push_row;             // -1: no push-down from the parent
    int dst_ps;               // 1: destination is a PS slot (leaf), 0: PUSH rows (children)
    int dst_row;
};

// Sum of a node's y1 slots into Y1 (rows indexed like the y0 region)
struct Y1Task {
    int row, nrow;
    int slot_beg, slot_end;
};

// Stored block (AOT) chunk: PS[out0_row + r] = A[r, :] * XS[in0_row : +ncol]  (r < nrow)
//                           PS[out1_row + c] = A[:, c]^T * XS[in1_row : +nrow]
// One read of the block feeds both products, as CBLAS_BI_GEMV does
// (src/H2Pack_matvec.c:26-65, used at :333-379 and :929-932).
// Stored-block arenas: the FP64 arena keeps H2Pack's packing (B_ptr / D_ptr, rows of
// ncol elements); the FP32 arena pads every row to a multiple of 4 elements with zeros
// and starts every block on a 16-byte boundary, so FP32 rows take 16-byte loads.
__host__ __device__ inline int f32_ld(int ncol) { return (ncol + 3) & ~3; }

struct BlkTask {
    long long a_off;   // element offset of the chunk's first row in the FP64 arena
    int nrow, ncol;    // rows in this chunk, columns (= the FP64 row stride)
    int in0_row, in1_row;
    int out0_row, out1_row;   // -1: product not needed
    long long a32;     // element offset of the chunk's first row in the FP32 arena
    int ld32;          // FP32 row stride, f32_ld(ncol)
    int pad;
};

// Stored-block tasks of one right-hand side (k_blk1) small enough for one warp: at most
// 256 columns, 512 rows and 128 KB of block values.  The plan puts them first in each
// block-task list (those within the FP64 limit, then those within the FP32 limit only).
constexpr int kBlk1WarpCols = 256, kBlk1WarpRows = 512;
constexpr long long kBlk1WarpBytes = 128 * 1024;
__host__ __device__ inline bool blk1_fits(int nrow, int ncol, int elem_bytes)
{
    return ncol <= kBlk1WarpCols && nrow <= kBlk1WarpRows && (long long) nrow * ncol * elem_bytes <= kBlk1WarpBytes;
}

// Unit of the wide-panel stored-block passes: one 64-row chunk of a task (pass 0,
// A V over all column tiles) or one 64-column tile of a task (pass 1, A^T W over all of
// the task's rows).
struct WideUnit {
    int task;          // index into the block-task list
    int off;           // first row (pass 0) or first column (pass 1) of the unit
};

// JIT target: a set of points whose outputs accumulate over a list of source sets
// (owner computes; each (target, source) kernel block is evaluated by its owner).
struct JitTarget {
    int pt0, npt;      // point-space range of this chunk of targets
    int out_row;       // row of the chunk's first output row (PS, or Y1 when out_y1)
    int out_y1;        // 1: outputs are the node's y1 rows
    int src_beg, src_end;
    int tile_beg, tile_end;   // its source tiles (FP32 tensor-core path)
};

struct JitSource {
    int pt0, npt;      // point-space range of the source set
    int in_row;        // XS row of the input of the first source point
    float sx, sy, sz;  // center(target set) - center(source set), for re-centred FP32 evaluation
    int grp;           // first 8-point group of the set in the source panels (FP32 tensor-core path)
};

// Source panels (FP32 tensor-core JIT path): every source set is cut into groups of 8
// points, padded at its end.  Per group, the points in the pairs the m16n8k8 B fragment
// holds them (static) and the inputs split into TF32 hi / lo in A-fragment order
// (refilled from XS for every panel of right-hand sides).
// One tile (up to 128 points) of a source set for a target (FP32 tensor-core JIT path):
// the tiles of all the target's source sets in order, so the kernel walks one array.
struct TileRec {
    int gb;            // first panel group of the tile
    int ng;            // groups in the tile (1..16)
    int nj;            // points in the tile (1..128)
    int pad0;
    float sx, sy, sz;  // center(target set) - center(source set)
    float pad1;
};

struct PanelGroup {
    int pt0;           // point-space index of the group's first point
    int row0;          // XS row of its input
    int nvalid;        // points of the set in this group (1..8)
    int pad;
};

// JIT pair tasks (FP32 tensor-core path): every unordered pair of point sets (a, b)
// is evaluated once and applied both ways.  One record per chunk of <= 256 points of
// an owner set a, with the list of its partners b.
struct PairOwner {
    int pa, na;          // point-space range of a
    int in_a;            // XS row of y0 / x of a's first point
    int out_a;           // PS row of a's first output row (sum over all partners)
    int p_beg, p_end;    // partner range
};
struct PairPartner {
    int pb, nb;          // point-space range of b
    int in_b;            // XS row of b's input
    int out_b;           // PS row of b's output slot (its pair with this owner only)
    float sx, sy, sz;    // center(a) - center(b)
};

// Generation of stored blocks on the device (H2P_build_B_AOT, src/H2Pack_build.c:789-889;
// H2P_build_D_AOT, :1034-1140): rows [kd*r0, kd*(r0 + nr)) of one block,
// A[kd i + a][kd j + b] = K_ab(row point i, column point j), packed row-major with
// ld = kd * ncp at the block's offset in H2Pack's B / D packing.
struct GenTask {
    long long a_off;   // element offset of the task's first row in the FP64 arena (ld = kd * ncp)
    int row_pt0;       // point-space index of the task's first row point
    int nrp;           // row points in this task (<= 16)
    int col_pt0;       // point-space index of the block's first column point
    int ncp;           // column points of the block
    long long a32;     // ... in the FP32 arena (ld = f32_ld(kd * ncp))
};

// One block of a batch of interpolative decompositions (construction of U): the
// kernel matrix of ncand candidate points against npp proxy points, its candidate and
// proxy coordinates (dim-major, 3 x n) and its workspace (ncand x npp, row-major)
struct IdBlock {
    int ncand, npp;
    long long cand_off, prox_off, w_off, perm_off;
};

// Final assembly of a leaf: Y[fwd[row0 + r]][v] = sum_s PS[slot_s + r][v]
struct AsmTask {
    int row0, nrow;
    int slot_beg, slot_end;
};

// Kernel parameters as the device sees them
struct KParam {
    double p0;         // Coulomb: value on r == 0; Gaussian: l; Matern: l; RPY: eta
    double c0;         // derived constant (Matern: -sqrt(3) l; RPY: 1 / (6 pi eta))
    float sigma;       // FP32 far field: the scale of r^2 its kernel form takes (ScalarFar)
    float pad;
};

}  // namespace h2gpu
