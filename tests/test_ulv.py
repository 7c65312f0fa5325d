"""HSS ULV solves on the GPU (H2P_HSS_ULV_Cholesky_solve / H2P_HSS_ULV_LU_solve).

The factorizations stay H2Pack's own (src/H2Pack_HSS_ULV.c:601, :16); the solves
(:981-1159, :429-599) run on the device, one launch per tree level.  Checks:

- CPU: the reference library's own factorization and solve of (A + shift I) invert the
  HSS operator, and the restatement in oracle/h2_oracle.c reproduces the reference's
  solve on the same factors (pins the checker); without a device the GPU solve refuses
  (no CPU path); malformed factors are refused on the host.
- GPU: the device solve of every op (1, 2, 3) agrees with H2Pack's solve on the same
  handle's factors (its own code, compiled into the library under the name
  H2P_HSS_ULV_*_solve_host); op 3 inverts the shifted HSS operator; the drop-in entry
  point gives the same bits as the status form; a new factorization of the handle
  (another shift, LU after Cholesky) is picked up by the next solve.

Ops 1 and 2 alone depend on the factorization's own choices (Householder signs, ranks),
so the comparison is on the same factors: two separate builds from the same points can
differ by a pivot tie in an interpolative decomposition (one skeleton point in 28,274
for the Gaussian case at N = 12,000).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import KERNEL_PARAMS, make_points, rel
from h2pack_b200 import _abi
from h2pack_b200.h2pack import H2Matrix
from oracle import oracle

# FP64 solves with the same factors: rounding of the per-node products and triangular
# solves, amplified by the condition of the shifted HSS matrix (~1e2 .. 1e4 here)
TOL = 1e-11

CASES = [("gaussian", False, 1e-2), ("matern32", False, 1e-1), ("gaussian", True, 1e-2), ("coulomb", True, 1.0)]


def _build(kernel, n, seed):
    P = make_points(kernel, n, seed)
    return H2Matrix(kernel, P, KERNEL_PARAMS[kernel], 1e-6, BD_JIT=1, max_leaf_points=100, hss=True), P


def _build_ref(kernel, P):
    return oracle.RefH2(kernel, KERNEL_PARAMS[kernel], P, 1e-6, BD_JIT=1, max_leaf_points=100, hss=True)


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _oracle_solve(H, lu, b, op):
    """h2o_ulv_solve (oracle/h2_oracle.c) on the factors of the drop-in's handle H."""
    from h2pack_b200 import _abi
    d = _abi.UlvDesc()
    buf = C.c_void_p()
    assert H.lib.h2pb_describe_ulv(H.h2pack, int(lu), C.byref(d), C.byref(buf)) == 0
    try:
        x = np.empty(H.N)
        assert oracle.liboracle().h2o_ulv_solve(C.byref(d), int(op), _dp(b), _dp(x)) == 0
        return x
    finally:
        H.lib.h2pb_free(buf)


def test_reference_ulv_inverts_the_hss_operator():
    R = _build_ref("gaussian", make_points("gaussian", 3000, 61))
    try:
        R.ulv_factorize(1e-2)
        b = np.random.default_rng(1).standard_normal(R.N)
        x = R.ulv_solve(b, 3)
        assert rel(R.matvec(x) + 1e-2 * x, b) < 1e-9
    finally:
        R.close()


@pytest.mark.parametrize("kernel,lu,shift", [("gaussian", False, 1e-2), ("gaussian", True, 1e-2),
                                              ("matern32", False, 1e-1), ("coulomb", True, 1.0),
                                              ("rpy", False, 1e-1), ("rpy", True, 1e-1)])
def test_oracle_ulv_solve_pinned_to_reference(kernel, lu, shift):
    """The restatement (oracle/h2_oracle.c, h2o_ulv_solve) over the plain descriptor of
    the reference library's own factors gives the reference's solve, every op."""
    R = _build_ref(kernel, make_points(kernel, 2000 if kernel == "rpy" else 6000, 66))
    try:
        R.ulv_factorize(shift, lu=lu)
        rng = np.random.default_rng(9)
        for op in (1, 2, 3):
            b = rng.standard_normal(R.N)
            assert rel(R.ulv_solve_oracle(b, op), R.ulv_solve(b, op)) < 1e-12, op
    finally:
        R.close()


def test_gpu_solve_has_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present (GPU tests cover the solve)")
    H, _ = _build("gaussian", 2000, 62)
    try:
        H.ulv_factorize(1e-2)
        # H2Pack's factors pass every host check of h2gpu_ulv_create; only the device is missing
        with pytest.raises(RuntimeError, match="no CUDA device"):
            H.ulv_solve(np.ones(H.N))
        # an LU solve on a Cholesky-factored handle: no LU factors to upload
        b, x = np.ones(H.N), np.empty(H.N)
        st = H.lib.H2P_gpu_ULV_solve(H.h2pack, 1, 3, _dp(b), _dp(x))
        assert st != 0 and "LU factors" in H.lib.H2P_gpu_last_error().decode()
    finally:
        H.close()


def test_solve_refuses_handles_without_factors():
    """The status form names what is missing, as the reference's messages do
    (src/H2Pack_HSS_ULV.c:983-992); no device is touched."""
    from h2pack_b200 import _abi
    P = make_points("gaussian", 2000, 65)
    b = np.ones(2000)
    x = np.empty(2000)
    for hss, msg in ((False, "HSS mode"), (True, "no ULV factorization")):
        H = H2Matrix("gaussian", P, [1.0], 1e-6, BD_JIT=1, max_leaf_points=100, hss=hss)
        try:
            st = H.lib.H2P_gpu_ULV_solve(H.h2pack, 0, 3, _dp(b), _dp(x))
            assert _abi.STATUS_NAMES[st] == "STATE"
            assert msg in H.lib.H2P_gpu_last_error().decode()
            st = H.lib.H2P_gpu_ULV_solve(H.h2pack, 0, 4, _dp(b), _dp(x))
            assert st != 0
        finally:
            H.close()


def _tiny_desc(lu=0, **bad):
    """Factors of a two-level tree by hand: root 0 over leaves 1 and 2 (two points each,
    one Householder vector each), for the host-side checks of h2gpu_ulv_create."""
    from h2pack_b200 import _abi
    keep = []

    def ia(v):
        a = np.ascontiguousarray(v, dtype=np.int32)
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_int))

    def da(v):
        a = np.ascontiguousarray(v, dtype=np.float64)
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_double))

    idx = bad.get("idx", [[0, 2], [0, 1], [2, 3]])
    m = [len(i) for i in idx]
    Ls = bad.get("Ls", [0, 1, 1])
    q_ncol = bad.get("q_ncol", [0, 1, 1])
    Q = [None] + [da([[1.0], [0.5], [1.2]]) for _ in range(2)]   # (m + 1) x 1: vector, tau
    L = [da(np.eye(mm) * 2.0) for mm in m]
    p = bad.get("p", [[0, 1], [0], [0]])
    d = _abi.UlvDesc()
    d.lu = lu
    d.n_node, d.max_level, d.n_leaf_node, d.krnl_mat_size = 3, 1, 2, 4
    d.level_n_node = ia(bad.get("level_n_node", [1, 2]))
    d.level_nodes = ia(bad.get("level_nodes", [0, -1, 1, 2]))
    d.fwd_pmt_idx = ia(bad.get("fwd", [0, 1, 2, 3]))
    d.bwd_pmt_idx = ia([0, 1, 2, 3])
    d.Ls, d.m, d.q_ncol, d.l_ld = ia(Ls), ia(m), ia(q_ncol), ia(m)
    d.idx = (C.POINTER(C.c_int) * 3)(*[ia(i) for i in idx])
    d.Q = (C.POINTER(C.c_double) * 3)(*[q if q is not None else C.POINTER(C.c_double)() for q in Q])
    d.L = (C.POINTER(C.c_double) * 3)(*L)
    d.p = (C.POINTER(C.c_int) * 3)(*[ia(x) for x in p]) if lu else None
    d.device = -1
    d._keep = keep
    return d


@pytest.mark.parametrize("bad,lu,status", [
    ({"idx": [[0, 2], [0, 9], [2, 3]]}, 0, "INVALID"),            # index outside the vector
    ({"fwd": [0, 1, 2, 7]}, 0, "INVALID"),                        # permutation entry
    ({"level_n_node": [2, 1], "level_nodes": [0, 1, 2, -1]}, 0, "INVALID"),   # level 0 not the root alone
    ({"level_nodes": [0, -1, 1, 1]}, 0, "INVALID"),               # a node twice
    ({"Ls": [0, 3, 1]}, 0, "INVALID"),                            # Ls > m
    ({"q_ncol": [0, 3, 1]}, 0, "UNSUPPORTED"),                    # more reflectors than rows
    ({"p": [[0, 1], [4], [0]]}, 1, "INVALID"),                    # LU pivot out of range
])
def test_ulv_create_checks_factors_on_the_host(bad, lu, status):
    """h2gpu_ulv_create range-checks every index the kernels use before any device
    work, so malformed factors are refused with a status (no GPU needed)."""
    from h2pack_b200 import _abi
    lib = _abi.libh2gpu()
    out = C.c_void_p()
    st = lib.h2gpu_ulv_create(C.byref(_tiny_desc(lu, **bad)), C.byref(out))
    assert _abi.STATUS_NAMES[st] == status, lib.h2gpu_last_error()
    assert not out.value


def test_ulv_create_valid_factors_need_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from h2pack_b200 import _abi
    lib = _abi.libh2gpu()
    out = C.c_void_p()
    for lu in (0, 1):
        st = lib.h2gpu_ulv_create(C.byref(_tiny_desc(lu)), C.byref(out))
        assert _abi.STATUS_NAMES[st] == "CUDA" and not out.value


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,lu,shift", CASES)
def test_gpu_ulv_solve_matches_h2pack(kernel, lu, shift):
    H, _ = _build(kernel, 12000, 63)
    try:
        H.ulv_factorize(shift, lu=lu)
        host = H.lib.H2P_HSS_ULV_LU_solve_host if lu else H.lib.H2P_HSS_ULV_Cholesky_solve_host
        dropin = H.lib.H2P_HSS_ULV_LU_solve if lu else H.lib.H2P_HSS_ULV_Cholesky_solve
        rng = np.random.default_rng(7)
        for op in (1, 2, 3):
            b = rng.standard_normal(H.N)
            x = H.ulv_solve(b, op)
            xh = np.empty(H.N)
            _abi.blas_one_thread(H.lib)
            host(H.h2pack, op, _dp(b), _dp(xh))          # H2Pack's solve, same factors
            assert rel(x, xh) < TOL, (op, rel(x, xh))
            # the restatement (each of the two within TOL of H2Pack's solve)
            assert rel(x, _oracle_solve(H, lu, b, op)) < 2 * TOL, op
            xd = np.empty(H.N)
            dropin(H.h2pack, op, _dp(b), _dp(xd))        # the replaced entry point
            assert np.array_equal(xd, x)
        # op 3 inverts the shifted HSS operator
        b = rng.standard_normal(H.N)
        x = H.ulv_solve(b, 3)
        assert rel(H.matvec(x) + shift * x, b) < 1e-8
    finally:
        H.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,lu,shift", [("gaussian", False, 1e-2), ("rpy", False, 1e-1), ("rpy", True, 1e-1)])
def test_gpu_ulv_solve_on_reference_handles(kernel, lu, shift):
    """A handle built and factorized by the reference library itself, solved by the
    drop-in on the GPU (the struct layout is H2Pack's): every op against the reference
    library's own CPU solve of the same factors, the RPY tensor kernel (3 rows per
    point) included."""
    from h2pack_b200 import _abi
    lib = _abi.libh2pack_gpu()
    R = _build_ref(kernel, make_points(kernel, 2000 if kernel == "rpy" else 6000, 69))
    try:
        R.ulv_factorize(shift, lu=lu)
        rng = np.random.default_rng(11)
        for op in (1, 2, 3):
            b = rng.standard_normal(R.N)
            x = np.empty(R.N)
            assert lib.H2P_gpu_ULV_solve(R.h2pack, int(lu), op, _dp(b), _dp(x)) == 0, lib.H2P_gpu_last_error()
            assert rel(x, R.ulv_solve(b, op)) < TOL, op
    finally:
        lib.H2P_gpu_ULV_release(R.h2pack)    # the reference's H2P_destroy does not know the drop-in
        R.close()


@pytest.mark.gpu
def test_gpu_ulv_follows_refactorization():
    H, _ = _build("gaussian", 8000, 64)
    try:
        b = np.random.default_rng(8).standard_normal(H.N)
        for shift, lu in ((1e-2, False), (1.0, False), (1e-1, True)):
            H.ulv_factorize(shift, lu=lu)
            x = H.ulv_solve(b, 3)
            assert rel(H.matvec(x) + shift * x, b) < 1e-8, (shift, lu)
    finally:
        H.close()


@pytest.mark.gpu
def test_gpu_two_factorizations_alive():
    """Two handles' factors on the device at once, the second with smaller nodes: the
    first still solves, bit for bit as before (the solve kernels' shared-memory limit is
    a process-wide setting that a later, smaller factorization must not lower)."""
    A, _ = _build("gaussian", 12000, 67)
    B, _ = _build("gaussian", 1500, 68)
    try:
        A.ulv_factorize(1e-2)
        B.ulv_factorize(1e-2)
        rng = np.random.default_rng(10)
        ba, bb = rng.standard_normal(A.N), rng.standard_normal(B.N)
        xa = A.ulv_solve(ba)
        xb = B.ulv_solve(bb)
        assert np.array_equal(A.ulv_solve(ba), xa)
        assert rel(A.matvec(xa) + 1e-2 * xa, ba) < 1e-8
        assert rel(B.matvec(xb) + 1e-2 * xb, bb) < 1e-8
    finally:
        A.close()
        B.close()
