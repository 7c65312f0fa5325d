"""Source panels of the tensor-core JIT kernel: edge shapes.

The FP32 tensor-core JIT path cuts every source set into groups of 8 points (the last
group padded with far-away points and zero inputs) and walks each target chunk's
source tiles of up to 128 points.  These cases put the padding and the tile edges
everywhere: leaves of a few points (every group partial), leaves just past a multiple
of 8, and leaves wider than one 128-point target chunk (chunks whose last warps hold
no targets).  The mixed result must stay as close to the FP64 GPU result as on the
regular shapes, for panels of 8 and 16 right-hand sides and for the pair variant
(including owner sets of more than 128 points, which the pair plan walks in pieces
of 128 and sums piece by piece).
"""
import numpy as np
import pytest

from conftest import KERNEL_PARAMS, make_points, rel
from h2pack_b200.h2pack import H2Matrix

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel", ["coulomb", "gaussian", "matern32"])
@pytest.mark.parametrize("leaf", [3, 9, 300])
def test_mixed_close_on_edge_shapes(kernel, leaf):
    n = 1500 if leaf < 100 else 6000
    H = H2Matrix(kernel, make_points(kernel, n, 31 + leaf), KERNEL_PARAMS[kernel], 1e-6, BD_JIT=1,
                 max_leaf_points=leaf)
    try:
        rng = np.random.default_rng(leaf)
        for nv in (8, 16):
            X = rng.standard_normal((H.N, nv))
            H.set_precision("fp64")
            Y64 = H.matmul(X)
            H.set_precision("mixed")
            Ym = H.matmul(X)
            assert rel(Ym, Y64) < 2e-6, (kernel, leaf, nv, rel(Ym, Y64))
            # the same columns in a wider panel: the right-hand sides are independent
            if nv == 8:
                Yw = H.matmul(np.hstack([X, X]))
                assert rel(Yw[:, :8], Ym) < 1e-12 and rel(Yw[:, 8:], Ym) < 1e-12
    finally:
        H.close()


@pytest.mark.parametrize("leaf", [5, 200])
def test_pair_variant_on_edge_shapes(leaf):
    H = H2Matrix("matern32", make_points("matern32", 3000, 77), [1.0], 1e-6, BD_JIT=1, max_leaf_points=leaf,
                 precision="mixed")
    try:
        X = np.random.default_rng(3).standard_normal((H.N, 16))
        img = H.image()
        Ytc = H.matmul(X)
        img.set_jit_variant("pair")
        Ypair = H.matmul(X)
        img.set_jit_variant("tc")
        H.set_precision("fp64")
        Y64 = H.matmul(X)
        assert rel(Ytc, Y64) < 2e-6
        assert rel(Ypair, Y64) < 2e-6
    finally:
        H.close()


@pytest.mark.parametrize("kernel,n,leaf", [("coulomb", 20000, 400), ("gaussian", 8000, 200)])
def test_pair_variant_on_sets_wider_than_a_unit(kernel, n, leaf):
    H = H2Matrix(kernel, make_points(kernel, n, 5), KERNEL_PARAMS[kernel], 1e-6, BD_JIT=1, max_leaf_points=leaf,
                 precision="mixed")
    try:
        d = H.describe()
        widest = max(max(d.J_n[i] for i in range(d.n_node)),
                     max(d.pt_cluster[2 * i + 1] - d.pt_cluster[2 * i] + 1 for i in range(d.n_node)))
        assert widest > 128
        X = np.random.default_rng(7).standard_normal((H.N, 16))
        img = H.image()
        img.set_jit_variant("pair")
        Ypair = H.matmul(X)
        img.set_jit_variant("tc")
        Ytc = H.matmul(X)
        H.set_precision("fp64")
        Y64 = H.matmul(X)
        assert rel(Ytc, Y64) < 2e-6
        assert rel(Ypair, Y64) < 2e-6, rel(Ypair, Y64)
    finally:
        H.close()
