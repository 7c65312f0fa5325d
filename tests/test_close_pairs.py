"""Coulomb's FP32 near field with nearly coincident points.

1/r is singular at r = 0.  A distance formed from FP32 coordinates re-centred on a box
of size L carries an absolute error near eps * L, i.e. a relative error eps * L / r:
about 1e-3 for a pair 1e-4 * L apart, passed on to every row such a pair dominates.
The FP32 Coulomb near field therefore forms differences from hi + lo coordinates
(frame shifts exactly representable, TwoSum of a target coordinate and its shift), so
r keeps FP32 relative accuracy at any distance.  Planted pairs 1e-2 .. 1e-6 apart must
come out of the mixed apply within 2e-6 of the FP64 apply on their own rows, for every
FP32 near-field kernel: CUDA cores (panels of 1 and 8), tensor cores per target, and
tensor cores per unordered pair.  Coincident points keep the kernel's r = 0 value.
"""
import numpy as np
import pytest

from conftest import make_points, rel
from h2pack_b200.h2pack import H2Matrix

pytestmark = pytest.mark.gpu

DIST = [1e-2, 1e-3, 1e-4, 1e-5, 1e-6, 0.0, 3e-4, 3e-6]


def planted(n, seed):
    """Uniform points with len(DIST) pairs moved to the given distances; returns the
    coordinates and the row indices of the moved pairs."""
    P = make_points("coulomb", n, seed)
    rng = np.random.default_rng(seed)
    idx = rng.choice(n, 2 * len(DIST), replace=False)
    for k, d in enumerate(DIST):
        a, b = idx[2 * k], idx[2 * k + 1]
        u = rng.standard_normal(3)
        P[:, b] = P[:, a] + d * u / np.linalg.norm(u)
    return P, idx


@pytest.mark.parametrize("variant,nv", [("simt", 1), ("simt", 8), ("tc", 8), ("tc", 16), ("pair", 8), ("pair", 16)])
def test_close_pairs_mixed_rows(variant, nv):
    P, rows = planted(6000, 11)
    H = H2Matrix("coulomb", P, [], 1e-6, BD_JIT=1, max_leaf_points=200)
    try:
        X = np.random.default_rng(nv).standard_normal((H.N, nv))
        H.set_precision("fp64")
        Y64 = H.matmul(X)
        H.set_precision("mixed")
        H.image().set_jit_variant(variant)
        Ym = H.matmul(X)
        errs = [rel(Ym[r], Y64[r]) for r in rows]
        assert max(errs) < 2e-6, (variant, nv, errs)
        assert rel(Ym, Y64) < 2e-6
    finally:
        H.close()
