"""The C restatement of the apply path (oracle/h2_oracle.c) against the reference
library built from H2Pack's sources (oracle/_ref/libh2ref.so): same H2Pack handle,
same inputs.  This pins the oracle before it judges the GPU engine."""
import numpy as np
import pytest

from conftest import KERNEL_PARAMS, build_kwargs, make_points, rel
from oracle import oracle as O
from h2pack_b200 import _abi

pytestmark = pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built (needs the H2Pack sources)")

CASES = [(k, jit, hss) for k in ("coulomb", "gaussian", "matern32", "rpy") for jit in (0, 1) for hss in (0, 1)]


@pytest.mark.parametrize("kernel,jit,hss", CASES)
def test_restatement_matches_reference(kernel, jit, hss):
    """H2 and HSS mode (HSS: its own pair lists and minimum admissible level,
    src/H2Pack_matvec.c:101, :308, :773, :904)."""
    n = 1500 if kernel == "rpy" else 3000
    coord = make_points(kernel, n, seed=11)
    R = O.RefH2(kernel, KERNEL_PARAMS[kernel], coord, 1e-6, BD_JIT=jit, hss=bool(hss), **build_kwargs(kernel))
    try:
        rng = np.random.default_rng(3)
        x = rng.random(R.N) - 0.5
        d = R.describe()
        assert rel(O.matvec(d, x), R.matvec(x)) < 1e-13
        X = rng.standard_normal((R.N, 3))
        Yr = R.matmul(X)
        assert rel(O.matmul(d, X), Yr) < 1e-13
        assert rel(O.matmul(d, X, _abi.COL_MAJOR), Yr) < 1e-13
        # the reference's own matvec <-> matmul consistency (extra/test_H2_matmul.h:48-83)
        assert rel(R.matmul(X, _abi.COL_MAJOR)[:, 1], R.matvec(X[:, 1])) < 1e-13
    finally:
        R.close()


def test_direct_sum_restatement_matches_kernel_blocks():
    rng = np.random.default_rng(5)
    src = make_points("matern32", 300, seed=1)
    trg = src[:, :40]
    v = rng.standard_normal(300)
    K = O.kernel_eval(_abi.KRNL_MATERN32, [1.0], trg, src)
    assert rel(O.direct_sum(_abi.KRNL_MATERN32, [1.0], src, v, trg), K @ v) < 1e-14


def test_coulomb_diagonal_value():
    c = make_points("coulomb", 5, seed=2)
    K0 = O.kernel_eval(_abi.KRNL_COULOMB, [], c, c)
    K7 = O.kernel_eval(_abi.KRNL_COULOMB, [7.0], c, c)
    assert np.all(np.diag(K0) == 0.0) and np.all(np.diag(K7) == 7.0)


def test_rpy_branches_symmetric():
    """RPY 3x3 blocks are symmetric; the three distance branches of
    src/H2Pack_3D_kernels.h:917-935 are all exercised."""
    a = np.array([[0.0, 0.5, 1.5, 4.0], [0, 0, 0, 0], [0, 0, 0, 0], [1.0, 0.3, 1.0, 1.0]])
    K = O.kernel_eval(_abi.KRNL_RPY, [1.0 / (6 * np.pi)], a, a)
    assert np.allclose(K, K.T, atol=1e-15)
    # r = 0 with equal radii: C / a on the diagonal
    assert abs(K[0, 0] - 1.0) < 1e-15
