"""H2 matrices stored on disk in H2Pack's file format, read straight into a device image.

H2Pack stores a constructed H2 (or HSS) matrix as three files (H2P_store_to_file,
src/H2Pack_file_IO.c:17-218, with the JSON encoding of examples/meta_txt_to_json.py):

* a metadata JSON: matrix size and symmetry, the partition tree (``nodes_row``: index,
  level, cluster head / tail, children), the basis matrices' shapes
  (``basis_matrices_row``), the admissible blocks (``B_matrices``: node_row, node_col,
  num_row, num_col, is_part_adm) and the inadmissible blocks (``D_matrices``, the leaf
  diagonal blocks first);
* an auxiliary JSON: point and kernel dimensions, HSS flag, minimum admissible level,
  the points in the caller's order (``point_coordinate``), H2Pack's sorting of them
  (``permutation_array``: sorted position -> caller index) and every node's skeleton
  point indices (into the sorted points);
* a binary file of FP64 values: every U (node order, row-major), then every B block, then
  every D block, each row-major with its stated shape.

:func:`read_h2` turns the three files into an :class:`H2File` whose ``desc`` is an
``h2gpu_desc`` over numpy buffers (the binary file is memory-mapped, so U/B/D are copied
once, by ``h2gpu_image_create``, from the page cache to the device).  The reader follows
the format, not H2Pack's reader: permutation indices, level lists, skeleton coordinates
and block offsets are rebuilt as H2P_read_from_file does (src/H2Pack_file_IO.c:220-560).

RPY extension.  H2Pack refuses to store matrices whose points carry more than their
space dimension (src/H2Pack_file_IO.c:22-26), so the RPY kernel's radii cannot be
stored.  :func:`write_h2` writes one more auxiliary field, ``point_radius`` (the radius
of every point, caller's order); :func:`read_h2` uses it when present (xpt_dim = 4).
Files without it are H2Pack's own format unchanged.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from . import _abi

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class H2File:
    """An H2 representation read from disk; ``desc`` stays valid while this object lives."""

    def __init__(self, arrays: dict, U: list, J: list, B: np.ndarray, D: np.ndarray, info: dict):
        self.a = arrays
        self.info = info
        self._U = U
        self._J = J
        self._B = B
        self._D = D
        n_node = arrays["n_node"]
        d = _abi.Desc()
        for k in ("n_point", "pt_dim", "xpt_dim", "krnl_dim", "n_node", "n_leaf_node", "max_child", "max_level",
                  "min_adm_level", "BD_JIT", "n_r_adm_pair", "n_r_inadm_pair", "n_B", "n_D", "kernel_id",
                  "n_krnl_param"):
            setattr(d, k, int(arrays[k]))
        for k in ("n_child", "children", "node_level", "pt_cluster", "mat_cluster", "level_n_node", "level_nodes",
                  "leaf_nodes", "U_nrow", "U_ncol", "U_ld", "r_adm_pairs", "r_inadm_pairs", "B_nrow", "B_ncol",
                  "D_nrow", "D_ncol", "J_n", "fwd_pmt_idx", "bwd_pmt_idx"):
            arr = np.ascontiguousarray(arrays[k], dtype=np.int32)
            arrays[k] = arr
            setattr(d, k, arr.ctypes.data_as(_ip))
        for k in ("B_ptr", "D_ptr"):
            arr = np.ascontiguousarray(arrays[k], dtype=np.uint64)
            arrays[k] = arr
            setattr(d, k, arr.ctypes.data_as(C.POINTER(C.c_size_t)))
        if B.size:
            d.B_data = B.ctypes.data_as(_dp)
        if D.size:
            d.D_data = D.ctypes.data_as(_dp)
        arrays["coord"] = np.ascontiguousarray(arrays["coord"], dtype=np.float64)
        d.coord = arrays["coord"].ctypes.data_as(_dp)
        self._Up = (_dp * n_node)()
        self._Jp = (_dp * n_node)()
        for i in range(n_node):
            if U[i] is not None and U[i].size:
                self._Up[i] = U[i].ctypes.data_as(_dp)
            if J[i] is not None and J[i].size:
                self._Jp[i] = J[i].ctypes.data_as(_dp)
        d.U = C.cast(self._Up, C.POINTER(_dp))
        d.J_coord = C.cast(self._Jp, C.POINTER(_dp))
        for i, v in enumerate(arrays["krnl_param"][:4]):
            d.krnl_param[i] = float(v)
        self.desc = d

    @property
    def N(self) -> int:
        return int(self.a["krnl_dim"]) * int(self.a["n_point"])


def read_h2(meta_json: str, aux_json: str, binary: str, kernel=None, param=()) -> H2File:
    """Read an H2 / HSS matrix stored in H2Pack's format.  ``kernel`` / ``param`` name the
    kernel function (its identity is not part of the format); it is needed for JIT use
    and for generating blocks, not for applying the stored U/B/D."""
    with open(meta_json) as f:
        meta = json.load(f)
    with open(aux_json) as f:
        aux = json.load(f)
    if int(meta["is_symmetric"]) != 1:
        raise ValueError("only symmetric H2 matrices are stored by H2Pack")
    pt_dim, kd, n_point = int(aux["dim_point"]), int(aux["dim_kernel"]), int(aux["num_point"])
    n_node = int(meta["num_node_row"])
    max_level = int(meta["num_level_row"]) - 1
    max_child = 1 << pt_dim
    nodes = meta["nodes_row"]
    n_child = np.zeros(n_node, np.int32)
    children = np.full((n_node, max_child), -1, np.int32)
    node_level = np.zeros(n_node, np.int32)
    pt_cluster = np.zeros((n_node, 2), np.int32)
    for nd in nodes:
        i = int(nd["index"])
        node_level[i] = int(nd["level"])
        pt_cluster[i] = (int(nd["cluster_head"]), int(nd["cluster_tail"]))
        n_child[i] = int(nd["num_children"])
        children[i, :n_child[i]] = [int(c) for c in nd["children"]]
    n_leaf = int((n_child == 0).sum())
    mat_cluster = np.stack([kd * pt_cluster[:, 0], kd * (pt_cluster[:, 1] + 1) - 1], axis=1)
    level_n_node = np.zeros(max_level + 1, np.int32)
    level_nodes = np.zeros((max_level + 1, n_leaf), np.int32)
    for i in range(n_node):              # nodes of a level in index order
        L = node_level[i]
        level_nodes[L, level_n_node[L]] = i
        level_n_node[L] += 1

    # binary: U (node order), B, D
    data = np.memmap(binary, dtype=np.float64, mode="r") if os.path.getsize(binary) else np.zeros(0)
    off = 0
    U_nrow = np.zeros(n_node, np.int32)
    U_ncol = np.zeros(n_node, np.int32)
    U = [None] * n_node
    for e in meta["basis_matrices_row"]:
        i, nr, nc = int(e["node"]), int(e["num_row"]), int(e["num_col"])
        U_nrow[i], U_ncol[i] = nr, nc
        U[i] = np.ascontiguousarray(data[off:off + nr * nc]) if nr * nc else None
        off += nr * nc
    Bm = meta["B_matrices"]
    n_B = len(Bm)
    r_adm = np.array([(int(e["node_row"]), int(e["node_col"])) for e in Bm], np.int32).reshape(-1, 2)
    B_nrow = np.array([int(e["num_row"]) for e in Bm], np.int32)
    B_ncol = np.array([int(e["num_col"]) for e in Bm], np.int32)
    B_ptr = np.zeros(n_B + 1, np.uint64)
    B_ptr[1:] = np.cumsum(B_nrow.astype(np.uint64) * B_ncol.astype(np.uint64))
    nBe = int(B_ptr[-1])
    B = data[off:off + nBe]
    off += nBe
    Dm = meta["D_matrices"]
    n_D = len(Dm)
    leaf_nodes = np.array([int(e["node_row"]) for e in Dm[:n_leaf]], np.int32)
    r_inadm = np.array([(int(e["node_row"]), int(e["node_col"])) for e in Dm[n_leaf:]], np.int32).reshape(-1, 2)
    D_nrow = np.array([int(e["num_row"]) for e in Dm], np.int32)
    D_ncol = np.array([int(e["num_col"]) for e in Dm], np.int32)
    D_ptr = np.zeros(n_D + 1, np.uint64)
    D_ptr[1:] = np.cumsum(D_nrow.astype(np.uint64) * D_ncol.astype(np.uint64))
    nDe = int(D_ptr[-1])
    D = data[off:off + nDe]
    off += nDe
    if off != data.size:
        raise ValueError(f"binary file holds {data.size} values, the metadata describes {off}")

    # points: sorted coordinates (dim-major), permutation indices, skeleton coordinates
    coord0 = np.asarray(aux["point_coordinate"], np.float64).reshape(n_point, pt_dim)
    perm = np.asarray(aux["permutation_array"], np.int64)
    radius = aux.get("point_radius")
    xpt_dim = pt_dim + (1 if radius is not None else 0)
    coord = np.empty((xpt_dim, n_point))
    coord[:pt_dim] = coord0[perm].T
    if radius is not None:
        coord[pt_dim] = np.asarray(radius, np.float64)[perm]
    fwd = (perm[:, None] * kd + np.arange(kd)[None, :]).ravel().astype(np.int32)
    bwd = np.empty_like(fwd)
    bwd[fwd] = np.arange(kd * n_point, dtype=np.int32)
    J_n = np.zeros(n_node, np.int32)
    J = [None] * n_node
    for e in aux.get("skeleton_points", []):
        i, idx = int(e["node"]), np.asarray(e["skeleton_point_indices"], np.int64)
        J_n[i] = idx.size
        J[i] = np.ascontiguousarray(coord[:, idx]) if idx.size else None

    kid = _abi.KERNEL_IDS[kernel] if isinstance(kernel, str) else int(kernel or 0)
    kp = np.zeros(4)
    kp[:len(param)] = param
    arrays = dict(n_point=n_point, pt_dim=pt_dim, xpt_dim=xpt_dim, krnl_dim=kd, n_node=n_node, n_leaf_node=n_leaf,
                  max_child=max_child, max_level=max_level, min_adm_level=int(aux["min_adm_level"]), BD_JIT=0,
                  n_child=n_child, children=children.ravel(), node_level=node_level, pt_cluster=pt_cluster.ravel(),
                  mat_cluster=mat_cluster.ravel(), level_n_node=level_n_node, level_nodes=level_nodes.ravel(),
                  leaf_nodes=leaf_nodes, U_nrow=U_nrow, U_ncol=U_ncol, U_ld=U_ncol.copy(),
                  n_r_adm_pair=n_B, r_adm_pairs=r_adm.ravel(), n_r_inadm_pair=len(r_inadm),
                  r_inadm_pairs=r_inadm.ravel(), n_B=n_B, B_nrow=B_nrow, B_ncol=B_ncol, B_ptr=B_ptr,
                  n_D=n_D, D_nrow=D_nrow, D_ncol=D_ncol, D_ptr=D_ptr, coord=coord, J_n=J_n,
                  fwd_pmt_idx=fwd, bwd_pmt_idx=bwd, kernel_id=kid, n_krnl_param=len(param), krnl_param=kp)
    info = {"is_HSS": int(aux.get("is_HSS", 0)), "max_leaf_points": int(aux.get("max_leaf_points", 0)),
            "QR_stop_tol": float(aux.get("QR_stop_tol", 0.0)), "has_partial_adm_blocks":
            int(meta.get("has_partial_adm_blocks", 0))}
    return H2File(arrays, U, J, B, D, info)


def _ints(p, n):
    return np.ctypeslib.as_array(p, shape=(n,)).copy() if n else np.zeros(0, np.int32)


def write_h2(desc: _abi.Desc, meta_json: str, aux_json: str, binary: str, max_leaf_points: int = 0,
             qr_stop_tol: float = 0.0, is_hss: bool = False):
    """Store a stored-block (AOT) representation in H2Pack's format; the radii of RPY
    points go into the extra auxiliary field ``point_radius``."""
    d = desc
    if d.BD_JIT or not d.D_data:
        raise ValueError("only representations with stored B / D blocks can be written")
    n_node, n_point, kd, pt, xd = d.n_node, d.n_point, d.krnl_dim, d.pt_dim, d.xpt_dim
    n_child = _ints(d.n_child, n_node)
    children = _ints(d.children, n_node * d.max_child).reshape(n_node, d.max_child)
    level = _ints(d.node_level, n_node)
    pc = _ints(d.pt_cluster, 2 * n_node).reshape(n_node, 2)
    U_nrow, U_ncol, U_ld = _ints(d.U_nrow, n_node), _ints(d.U_ncol, n_node), _ints(d.U_ld, n_node)
    adm = _ints(d.r_adm_pairs, 2 * d.n_r_adm_pair).reshape(-1, 2)
    inadm = _ints(d.r_inadm_pairs, 2 * d.n_r_inadm_pair).reshape(-1, 2)
    B_nrow, B_ncol = _ints(d.B_nrow, d.n_B), _ints(d.B_ncol, d.n_B)
    D_nrow, D_ncol = _ints(d.D_nrow, d.n_D), _ints(d.D_ncol, d.n_D)
    leaf = _ints(d.leaf_nodes, d.n_leaf_node)
    J_n = _ints(d.J_n, n_node) if d.J_n else np.zeros(n_node, np.int32)
    coord = np.ctypeslib.as_array(d.coord, shape=(xd * n_point,)).reshape(xd, n_point)
    fwd = _ints(d.fwd_pmt_idx, kd * n_point)
    perm = fwd[::kd] // kd                       # sorted position -> caller index
    nB = int(d.B_ptr[d.n_B]) if d.n_B else 0
    nD = int(d.D_ptr[d.n_D])
    # skeleton point indices: positions of the skeleton coordinates among the sorted points
    key = {tuple(coord[:pt, i]): i for i in range(n_point)}
    skel = []
    for i in range(n_node):
        idx = []
        if J_n[i] and d.J_coord and d.J_coord[i]:
            Jc = np.ctypeslib.as_array(d.J_coord[i], shape=(xd * int(J_n[i]),)).reshape(xd, -1)
            idx = [key[tuple(Jc[:pt, j])] for j in range(Jc.shape[1])]
        skel.append({"node": i, "num_skeleton_point": len(idx), "skeleton_point_indices": idx})
    meta = {
        "nrow_matrix": kd * n_point, "ncol_matrix": kd * n_point, "is_symmetric": 1,
        "num_node_row": n_node, "num_node_col": n_node, "root_node_row": int(np.argmin(level)),
        "root_node_col": int(np.argmin(level)), "num_level_row": d.max_level + 1, "num_level_col": d.max_level + 1,
        "num_inadmissible_blocks": d.n_D, "num_admissible_blocks": d.n_B,
        "has_partial_adm_blocks": int(any(level[a] != level[b] for a, b in adm)),
        "nodes_row": [{"index": i, "level": int(level[i]), "cluster_head": int(pc[i, 0]),
                       "cluster_tail": int(pc[i, 1]), "num_children": int(n_child[i]),
                       "children": [int(c) for c in children[i, :n_child[i]]]} for i in range(n_node)],
        "basis_matrices_row": [{"node": i, "num_row": int(U_nrow[i]), "num_col": int(U_ncol[i])}
                               for i in range(n_node)],
        "B_matrices": [{"node_row": int(a), "node_col": int(b), "num_row": int(B_nrow[k]),
                        "num_col": int(B_ncol[k]), "is_part_adm": int(level[a] != level[b])}
                       for k, (a, b) in enumerate(adm)],
        "D_matrices": [{"node_row": int(n), "node_col": int(n), "num_row": int(D_nrow[k]), "num_col": int(D_ncol[k])}
                       for k, n in enumerate(leaf)] +
                      [{"node_row": int(a), "node_col": int(b), "num_row": int(D_nrow[len(leaf) + k]),
                        "num_col": int(D_ncol[len(leaf) + k])} for k, (a, b) in enumerate(inadm)],
    }
    coord0 = np.empty((n_point, pt))
    coord0[perm] = coord[:pt].T
    aux = {"dim_point": pt, "dim_kernel": kd, "num_point": n_point, "is_HSS": int(is_hss),
           "min_adm_level": d.min_adm_level, "max_leaf_points": int(max_leaf_points), "QR_stop_tol": float(qr_stop_tol),
           "has_skeleton_points": 1, "point_coordinate": coord0.ravel().tolist(),
           "permutation_array": perm.tolist(), "skeleton_points": skel}
    if xd > pt:
        rad = np.empty(n_point)
        rad[perm] = coord[pt]
        aux["point_radius"] = rad.tolist()
    with open(meta_json, "w") as f:
        json.dump(meta, f)
    with open(aux_json, "w") as f:
        json.dump(aux, f)
    with open(binary, "wb") as f:
        for i in range(n_node):
            nr, nc, ld = int(U_nrow[i]), int(U_ncol[i]), int(U_ld[i])
            if nr * nc:
                u = np.ctypeslib.as_array(d.U[i], shape=(nr * ld,)).reshape(nr, ld)[:, :nc]
                f.write(np.ascontiguousarray(u).tobytes())
        if nB:
            f.write(np.ctypeslib.as_array(d.B_data, shape=(nB,)).tobytes())
        f.write(np.ctypeslib.as_array(d.D_data, shape=(nD,)).tobytes())
