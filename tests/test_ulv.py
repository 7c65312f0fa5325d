"""HSS ULV solves on the GPU (H2P_HSS_ULV_Cholesky_solve / H2P_HSS_ULV_LU_solve).

The factorizations stay H2Pack's own (src/H2Pack_HSS_ULV.c:601, :16); the solves
(:981-1159, :429-599) run on the device, one launch per tree level.  Checks:

- CPU: the reference library's own factorization and solve of (A + shift I) invert the
  HSS operator (pins the checker); without a device the GPU solve refuses (no CPU path).
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


def test_reference_ulv_inverts_the_hss_operator():
    R = _build_ref("gaussian", make_points("gaussian", 3000, 61))
    try:
        R.ulv_factorize(1e-2)
        b = np.random.default_rng(1).standard_normal(R.N)
        x = R.ulv_solve(b, 3)
        assert rel(R.matvec(x) + 1e-2 * x, b) < 1e-9
    finally:
        R.close()


def test_gpu_solve_has_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present (GPU tests cover the solve)")
    H, _ = _build("gaussian", 2000, 62)
    try:
        H.ulv_factorize(1e-2)
        with pytest.raises(RuntimeError):
            H.ulv_solve(np.ones(H.N))
    finally:
        H.close()


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
            host(H.h2pack, op, _dp(b), _dp(xh))          # H2Pack's solve, same factors
            assert rel(x, xh) < TOL, (op, rel(x, xh))
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
