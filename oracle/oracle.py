"""Parity oracle for the H2 apply path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only as the checker.  It wraps two libraries built by
``oracle/Makefile`` into ``oracle/_ref``:

* ``libh2ref.so``   -- the reference H2Pack compiled unchanged from its sources
  (construction + CPU ``H2P_matvec`` / ``H2P_matmul``), the ground truth;
* ``libh2oracle.so`` -- ``h2_oracle.c``, a plain-C restatement of the apply
  path over the flat ``h2gpu_desc`` view, pinned to ``libh2ref.so`` by
  ``tests/test_oracle_pin.py``, and of the HSS ULV solves over ``h2gpu_ulv_desc``,
  pinned by ``tests/test_ulv.py``.

It also runs the reference's own column-pivoted QR (``ref_pivot_qr``) as the checker
of the construction's interpolative decompositions.

It also converts a descriptor to and from plain numpy arrays, which is the
format of the golden fixtures in ``tests/golden``.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(_HERE))
from h2pack_b200 import _abi  # noqa: E402  (ctypes structs only)

REF_DIR = os.path.join(_HERE, "_ref")
LIBH2REF = os.path.join(REF_DIR, "libh2ref.so")
LIBH2ORACLE = os.path.join(REF_DIR, "libh2oracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

REF_SYMBOLS = dict(_abi.BUILDER_SYMBOLS)
REF_SYMBOLS.update({
    "H2P_matvec": (None, [C.c_void_p, _dp, _dp]),
    "H2P_matmul": (None, [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int]),
    "H2P_print_statistic": (None, [C.c_void_p]),
    "H2P_partial_pivot_QR": (None, [C.c_void_p, C.c_int, C.c_double, C.c_int, _ip, _ip, C.c_int, _dp]),
    "H2P_HSS_ULV_Cholesky_factorize": (None, [C.c_void_p, C.c_double]),
    "H2P_HSS_ULV_LU_factorize": (None, [C.c_void_p, C.c_double]),
    "H2P_HSS_ULV_Cholesky_solve": (None, [C.c_void_p, C.c_int, _dp, _dp]),
    "H2P_HSS_ULV_LU_solve": (None, [C.c_void_p, C.c_int, _dp, _dp]),
    "h2pb_describe_ulv": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(_abi.UlvDesc), C.POINTER(C.c_void_p)]),
    "h2pb_free": (None, [C.c_void_p]),
})
ORACLE_SYMBOLS = {
    "h2o_eval": (None, [C.c_int, _dp, C.c_int, _dp, C.c_int, C.c_int, _dp, C.c_int, C.c_int, _dp, C.c_int]),
    "h2o_matvec": (C.c_int, [C.POINTER(_abi.Desc), _dp, _dp]),
    "h2o_matmul": (C.c_int, [C.POINTER(_abi.Desc), C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int]),
    "h2o_direct_sum": (None, [C.c_int, _dp, C.c_int, C.c_int, C.c_int, _dp, C.c_int, C.c_int, _dp,
                              _dp, C.c_int, C.c_int, _dp]),
    "h2o_ulv_solve": (C.c_int, [C.POINTER(_abi.UlvDesc), C.c_int, _dp, _dp]),
}

_libs: dict = {}


def _lib(path, table):
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library {path} is not built; run `make -C oracle`")
        _libs[path] = _abi.bind(C.CDLL(path, mode=C.RTLD_LOCAL), table)
    return _libs[path]


def have_ref() -> bool:
    return os.path.exists(LIBH2REF)


def libref():
    return _lib(LIBH2REF, REF_SYMBOLS)


def liboracle():
    return _lib(LIBH2ORACLE, ORACLE_SYMBOLS)


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


# ------------------------------------------------- interpolative decompositions
class _DenseMat(C.Structure):
    """H2Pack's H2P_dense_mat (src/H2Pack_aux_structs.h:150-157)."""
    _fields_ = [("nrow", C.c_int), ("ncol", C.c_int), ("ld", C.c_int), ("size", C.c_int), ("data", _dp)]


def ref_pivot_qr(cols: np.ndarray, reltol: float, n_thread: int = 1):
    """H2Pack's own column-pivoted Householder QR (H2P_partial_pivot_QR,
    src/H2Pack_ID_compress.c:51-189, relative-norm stop as H2P_ID_compress calls it)
    run from ``libh2ref.so`` on a matrix given as ``cols`` (n x m: row j is column j of
    the m x n matrix decomposed).  Returns (R as n x m, column j of R in row j; the
    permutation; the rank)."""
    R = np.ascontiguousarray(cols, dtype=np.float64).copy()
    n, m = R.shape
    A = _DenseMat(m, n, m, m * n, dptr(R))
    perm = np.zeros(max(n, 1), dtype=np.int32)
    r = C.c_int(0)
    buf = np.zeros(max(n, 1))
    libref().H2P_partial_pivot_QR(C.byref(A), min(m, n), float(reltol), 1, iptr(perm), C.byref(r), int(n_thread),
                                  dptr(buf))
    return R, perm[:n], r.value


def ref_interp(R: np.ndarray, r: int) -> np.ndarray:
    """E = R11^-1 R12 of a pivoted QR (the interpolation part of H2P_ID_compress,
    src/H2Pack_ID_compress.c:491-576), r x (n - r), from ``ref_pivot_qr``'s R."""
    Rt = R.T   # m x n
    n = Rt.shape[1]
    if r == 0 or r == n:
        return np.zeros((r, n - r))
    import scipy.linalg
    return scipy.linalg.solve_triangular(Rt[:r, :r], Rt[:r, r:], lower=False)


# ----------------------------------------------------------------- kernels

def kernel_eval(kernel_id, param, cA, cB):
    """FP64 kernel block K(cA, cB) of the restatement; cA, cB are (xpt_dim, n) arrays."""
    cA = np.ascontiguousarray(cA, dtype=np.float64)
    cB = np.ascontiguousarray(cB, dtype=np.float64)
    kd = 3 if kernel_id == _abi.KRNL_RPY else 1
    nA, nB = cA.shape[1], cB.shape[1]
    mat = np.zeros((nA * kd, nB * kd))
    p = np.zeros(4)
    p[:len(param)] = param
    liboracle().h2o_eval(kernel_id, dptr(p), len(param), dptr(cA), nA, nA, dptr(cB), nB, nB, dptr(mat), nB * kd)
    return mat


def direct_sum(kernel_id, param, src_coord, src_val, trg_coord):
    """FP64 direct sum y_t = sum_s K(t, s) v_s (restatement of examples/direct_nbody.h)."""
    src = np.ascontiguousarray(src_coord, dtype=np.float64)
    trg = np.ascontiguousarray(trg_coord, dtype=np.float64)
    val = np.ascontiguousarray(src_val, dtype=np.float64)
    kd = 3 if kernel_id == _abi.KRNL_RPY else 1
    out = np.zeros(trg.shape[1] * kd)
    p = np.zeros(4)
    p[:len(param)] = param
    liboracle().h2o_direct_sum(kernel_id, dptr(p), len(param), src.shape[0], kd,
                               dptr(src), src.shape[1], src.shape[1], dptr(val),
                               dptr(trg), trg.shape[1], trg.shape[1], dptr(out))
    return out


# -------------------------------------------------------- descriptor arrays

_INT_FIELDS = ["n_child", "children", "node_level", "pt_cluster", "mat_cluster", "level_n_node",
               "level_nodes", "leaf_nodes", "U_nrow", "U_ncol", "U_ld", "r_adm_pairs", "r_inadm_pairs",
               "B_nrow", "B_ncol", "D_nrow", "D_ncol", "J_n", "fwd_pmt_idx", "bwd_pmt_idx"]
_SCALARS = ["n_point", "pt_dim", "xpt_dim", "krnl_dim", "n_node", "n_leaf_node", "max_child", "max_level",
            "min_adm_level", "BD_JIT", "n_r_adm_pair", "n_r_inadm_pair", "n_B", "n_D", "kernel_id",
            "n_krnl_param"]


def desc_to_arrays(d: _abi.Desc) -> dict:
    """Copy a descriptor into plain numpy arrays (U and J_coord packed densely)."""
    s = {k: int(getattr(d, k)) for k in _SCALARS}
    n_node, nl, L = s["n_node"], s["n_leaf_node"], s["max_level"] + 1
    sizes = {
        "n_child": n_node, "children": n_node * s["max_child"], "node_level": n_node,
        "pt_cluster": 2 * n_node, "mat_cluster": 2 * n_node, "level_n_node": L, "level_nodes": L * nl,
        "leaf_nodes": nl, "U_nrow": n_node, "U_ncol": n_node, "U_ld": n_node,
        "r_adm_pairs": 2 * s["n_r_adm_pair"], "r_inadm_pairs": 2 * s["n_r_inadm_pair"],
        "B_nrow": s["n_B"], "B_ncol": s["n_B"], "D_nrow": s["n_D"], "D_ncol": s["n_D"], "J_n": n_node,
        "fwd_pmt_idx": s["krnl_dim"] * s["n_point"], "bwd_pmt_idx": s["krnl_dim"] * s["n_point"],
    }
    out = dict(s)
    for k in _INT_FIELDS:
        n = sizes[k]
        out[k] = np.ctypeslib.as_array(getattr(d, k), shape=(n,)).copy() if n > 0 else np.zeros(0, np.int32)
    out["krnl_param"] = np.array(list(d.krnl_param), dtype=np.float64)
    B_ptr = np.ctypeslib.as_array(d.B_ptr, shape=(s["n_B"] + 1,)).astype(np.int64) if s["n_B"] > 0 else np.zeros(1, np.int64)
    D_ptr = np.ctypeslib.as_array(d.D_ptr, shape=(s["n_D"] + 1,)).astype(np.int64)
    out["B_ptr"], out["D_ptr"] = B_ptr, D_ptr
    if not s["BD_JIT"]:
        out["B_data"] = np.ctypeslib.as_array(d.B_data, shape=(int(B_ptr[-1]),)).copy() if B_ptr[-1] > 0 else np.zeros(0)
        out["D_data"] = np.ctypeslib.as_array(d.D_data, shape=(int(D_ptr[-1]),)).copy()
    out["coord"] = np.ctypeslib.as_array(d.coord, shape=(s["xpt_dim"] * s["n_point"],)).copy()
    # U packed densely (ld = ncol), J_coord packed (xpt_dim x J_n each)
    U_off = np.zeros(n_node + 1, np.int64)
    J_off = np.zeros(n_node + 1, np.int64)
    Us, Js = [], []
    for i in range(n_node):
        nr, nc, ld = out["U_nrow"][i], out["U_ncol"][i], out["U_ld"][i]
        if nr > 0 and nc > 0:
            u = np.ctypeslib.as_array(d.U[i], shape=(nr * ld,)).reshape(nr, ld)[:, :nc].copy()
            Us.append(u.ravel())
        U_off[i + 1] = U_off[i] + nr * nc
        nj = out["J_n"][i]
        if nj > 0:
            Js.append(np.ctypeslib.as_array(d.J_coord[i], shape=(s["xpt_dim"] * nj,)).copy())
        J_off[i + 1] = J_off[i] + s["xpt_dim"] * nj
    out["U_ld"] = out["U_ncol"].copy()
    out["U_data"] = np.concatenate(Us) if Us else np.zeros(0)
    out["U_off"] = U_off
    out["J_data"] = np.concatenate(Js) if Js else np.zeros(0)
    out["J_off"] = J_off
    return out


class DescHolder:
    """A Desc whose arrays live in numpy buffers held by this object."""

    def __init__(self, arrays: dict):
        self.a = {k: (np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v) for k, v in arrays.items()}
        a = self.a
        d = _abi.Desc()
        for k in _SCALARS:
            setattr(d, k, int(a[k]))
        for k in _INT_FIELDS:
            arr = np.ascontiguousarray(a[k], dtype=np.int32)
            a[k] = arr
            setattr(d, k, iptr(arr))
        n_node = int(a["n_node"])
        for k in ("B_ptr", "D_ptr"):
            arr = np.ascontiguousarray(a[k], dtype=np.uint64)
            a[k + "_u"] = arr
            setattr(d, k, arr.ctypes.data_as(C.POINTER(C.c_size_t)))
        for k in ("B_data", "D_data"):
            if k in a and a[k].size > 0:
                a[k] = np.ascontiguousarray(a[k], dtype=np.float64)
                setattr(d, k, dptr(a[k]))
        a["coord"] = np.ascontiguousarray(a["coord"], dtype=np.float64)
        d.coord = dptr(a["coord"])
        a["U_data"] = np.ascontiguousarray(a["U_data"], dtype=np.float64)
        a["J_data"] = np.ascontiguousarray(a["J_data"], dtype=np.float64)
        self._Uptr = (_dp * n_node)()
        self._Jptr = (_dp * n_node)()
        base_u = a["U_data"].ctypes.data
        base_j = a["J_data"].ctypes.data
        for i in range(n_node):
            if a["U_off"][i + 1] > a["U_off"][i]:
                self._Uptr[i] = C.cast(base_u + 8 * int(a["U_off"][i]), _dp)
            if a["J_off"][i + 1] > a["J_off"][i]:
                self._Jptr[i] = C.cast(base_j + 8 * int(a["J_off"][i]), _dp)
        d.U = C.cast(self._Uptr, C.POINTER(_dp))
        d.J_coord = C.cast(self._Jptr, C.POINTER(_dp))
        for i, v in enumerate(a["krnl_param"][:4]):
            d.krnl_param[i] = float(v)
        self.desc = d

    @property
    def N(self):
        return int(self.a["krnl_dim"]) * int(self.a["n_point"])


# --------------------------------------------------------- restated apply

def matvec(desc: _abi.Desc, x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x)
    st = liboracle().h2o_matvec(C.byref(desc), dptr(x), dptr(y))
    if st != 0:
        raise RuntimeError(f"h2o_matvec status {st}")
    return y


def matmul(desc: _abi.Desc, X: np.ndarray, layout: int = _abi.ROW_MAJOR) -> np.ndarray:
    """X is (N, n_vec); layout selects how it is handed to the C routine."""
    N, nv = X.shape
    if layout == _abi.ROW_MAJOR:
        Xc = np.ascontiguousarray(X, dtype=np.float64)
        Y = np.zeros((N, nv))
        st = liboracle().h2o_matmul(C.byref(desc), layout, nv, dptr(Xc), nv, dptr(Y), nv)
        res = Y
    else:
        Xc = np.ascontiguousarray(X.T, dtype=np.float64)
        Y = np.zeros((nv, N))
        st = liboracle().h2o_matmul(C.byref(desc), layout, nv, dptr(Xc), N, dptr(Y), N)
        res = Y.T
    if st != 0:
        raise RuntimeError(f"h2o_matmul status {st}")
    return res


# ------------------------------------------------------------ PCG restated

def pcg(apply, b: np.ndarray, tol: float, max_iter: int, x0: np.ndarray | None = None):
    """Left-preconditioned CG with the identity preconditioner, restated step by step from
    examples/PCG/pcg.c:11-152 (r = b - A x; rho = r'z; p = z + (rho/rho0) p, p = z at the
    first iteration; alpha = rho / p'Ap; stop when ||r|| <= tol ||b|| or max_iter).
    ``apply`` maps a vector to A x (e.g. H2Pack's CPU H2P_matvec plus mu x, the wrapper of
    examples/SPDHSS-H2/pcg_tests.c:13-20).  Returns (x, flag, relres, iters, res_history),
    flag 0 when converged as pcg.c:131; relres is the recursive residual as pcg.c:132."""
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    r = b - apply(x)
    b2 = float(np.sqrt(b @ b))
    rn = float(np.sqrt(r @ r))
    stop = b2 * tol
    it, rho = 0, 1.0
    p = np.zeros_like(b)
    hist = []
    while it < max_iter and rn > stop:
        z = r                                  # invMx == NULL: z = r (pcg.c:71-72)
        rho0, rho = rho, float(r @ z)
        beta = rho / rho0
        p = z.copy() if it == 0 else z + beta * p
        s = apply(p)
        alpha = rho / float(p @ s)
        x = x + alpha * p
        r = r - alpha * s
        rn = float(np.sqrt(r @ r))
        hist.append(rn)
        it += 1
    return x, (0 if rn <= stop else 1), rn / b2, it, np.array(hist)


# -------------------------------------------------- the reference library

class RefH2:
    """An H2 representation built and applied by the reference library itself."""

    def __init__(self, kernel: str, param, coord: np.ndarray, reltol: float, max_leaf_points: int = 0,
                 max_leaf_size: float = 0.0, BD_JIT: int = 0, proxy: str = "surface",
                 pp_fname: str | None = None, n_thread: int = 0, use_bimv: bool = True, hss: bool = False):
        lib = libref()
        self.lib = lib
        self.kernel_id = _abi.KERNEL_IDS[kernel]
        self.param = np.array(list(param) + [0.0] * (4 - len(param)), dtype=np.float64)
        self.n_param = len(param)
        self.coord = np.ascontiguousarray(coord, dtype=np.float64)
        n_point = self.coord.shape[1]
        h = lib.h2pb_build(self.kernel_id, dptr(self.param), self.n_param, n_point, dptr(self.coord),
                           float(reltol), int(max_leaf_points), float(max_leaf_size), int(BD_JIT),
                           0 if proxy == "id" else 1, pp_fname.encode() if pp_fname else None,
                           1 if use_bimv else 0, int(n_thread), 1 if hss else 0)
        if not h:
            raise RuntimeError("h2pb_build failed")
        self.handle = h
        self.h2pack = lib.h2pb_h2pack(h)
        info = (C.c_longlong * 16)()
        lib.h2pb_info(self.h2pack, info)
        self.info = dict(zip(["n_point", "krnl_dim", "xpt_dim", "n_node", "n_leaf_node", "max_level",
                              "min_adm_level", "n_r_adm_pair", "n_r_inadm_pair", "n_B", "n_D", "BD_JIT",
                              "krnl_mat_size", "max_leaf_points", "n_thread", "mm_max_n_vec"], list(info)))
        self.N = self.info["krnl_mat_size"]
        self.build_seconds = lib.h2pb_build_seconds(h)

    def describe(self) -> _abi.Desc:
        d = _abi.Desc()
        st = self.lib.h2pb_describe(self.handle, C.byref(d))
        if st != 0:
            raise RuntimeError(f"h2pb_describe status {st}")
        return d

    def ulv_factorize(self, shift: float = 0.0, lu: bool = False):
        """The reference's HSS ULV factorization (src/H2Pack_HSS_ULV.c:601 / :16)."""
        _abi.blas_one_thread(self.lib)
        (self.lib.H2P_HSS_ULV_LU_factorize if lu else self.lib.H2P_HSS_ULV_Cholesky_factorize)(self.h2pack, shift)
        self._ulv_lu = bool(lu)

    def ulv_solve_oracle(self, b: np.ndarray, op: int = 3) -> np.ndarray:
        """The restatement's ULV solve (h2_oracle.c, h2o_ulv_solve) on this handle's
        factors, through the plain h2gpu_ulv_desc view."""
        d = _abi.UlvDesc()
        buf = C.c_void_p()
        st = self.lib.h2pb_describe_ulv(self.h2pack, int(self._ulv_lu), C.byref(d), C.byref(buf))
        if st != 0:
            raise RuntimeError(f"h2pb_describe_ulv status {st}")
        try:
            b = np.ascontiguousarray(b, dtype=np.float64)
            x = np.empty(self.N)
            if liboracle().h2o_ulv_solve(C.byref(d), int(op), dptr(b), dptr(x)) != 0:
                raise RuntimeError("h2o_ulv_solve failed")
            return x
        finally:
            self.lib.h2pb_free(buf)

    def ulv_solve(self, b: np.ndarray, op: int = 3) -> np.ndarray:
        """The reference's ULV solve on the CPU (src/H2Pack_HSS_ULV.c:981 / :429)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty(self.N)
        _abi.blas_one_thread(self.lib)
        (self.lib.H2P_HSS_ULV_LU_solve if self._ulv_lu else self.lib.H2P_HSS_ULV_Cholesky_solve)(
            self.h2pack, int(op), dptr(b), dptr(x))
        return x

    def matvec(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.N)
        self.lib.H2P_matvec(self.h2pack, dptr(x), dptr(y))
        return y

    def matmul(self, X: np.ndarray, layout: int = _abi.ROW_MAJOR) -> np.ndarray:
        N, nv = X.shape
        if layout == _abi.ROW_MAJOR:
            Xc = np.ascontiguousarray(X, dtype=np.float64)
            Y = np.zeros((N, nv))
            self.lib.H2P_matmul(self.h2pack, layout, nv, dptr(Xc), nv, dptr(Y), nv)
            return Y
        Xc = np.ascontiguousarray(X.T, dtype=np.float64)
        Y = np.zeros((nv, N))
        self.lib.H2P_matmul(self.h2pack, layout, nv, dptr(Xc), N, dptr(Y), N)
        return Y.T

    def counters(self):
        ms = (C.c_double * 11)()
        tm = (C.c_double * 11)()
        jf = (C.c_double * 2)()
        nmv = C.c_longlong()
        self.lib.h2pb_counters(self.h2pack, ms, tm, jf, C.byref(nmv))
        return {"mat_size": list(ms), "timers": list(tm), "JIT_flops": list(jf), "n_matvec": nmv.value}

    def reset_timers(self):
        self.lib.h2pb_reset_timers(self.h2pack)

    def close(self):
        if self.handle:
            self.lib.h2pb_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
