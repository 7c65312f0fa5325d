"""Host-only self-check of the apply plan (h2gpu_plan_check): no GPU needed.

The plan is what h2gpu_image_create uploads: the upward / downward tasks, the
partial-space slots and the sums that read them, and for JIT images the (target,
source) point pairs with their source tiles and panel groups, plus the pair plan that
evaluates every unordered pair once.  The library checks these invariants itself.
The tests below check two further things:

- The number of point pairs the plan evaluates matches H2Pack's pair lists. The count
  is recomputed here in Python from the descriptor: near field each leaf with itself
  and its inadmissible partners; far field the admissible pairs, skeleton or leaf
  points as the node levels say (src/H2Pack_matvec.c:586-764, :1002-1145).
- The plan's sizes (tasks, slots) fit the representation.

The shapes cover the golden fixtures and freshly built trees whose point and skeleton
sets are wider than one 128-point pair-plan unit.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import KERNEL_PARAMS, make_points
from oracle import oracle as O
from h2pack_b200 import _abi
from h2pack_b200.h2pack import H2Matrix
from test_host_validation import arrays
import os

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def plan_check(desc):
    lib = _abi.libh2gpu()
    cnt = (C.c_longlong * 8)()
    st = lib.h2gpu_plan_check(C.byref(desc), cnt)
    assert st == _abi.H2GPU_OK, lib.h2gpu_last_error().decode()
    return list(cnt)


def pairs_from_lists(d):
    """Ordered (target point, source point) pairs of one JIT apply, from the pair lists."""
    npt = lambda n: d.pt_cluster[2 * n + 1] - d.pt_cluster[2 * n] + 1
    lvl = lambda n: d.node_level[n]
    s = sum(npt(d.leaf_nodes[i]) ** 2 for i in range(d.n_leaf_node))
    s += sum(2 * npt(d.r_inadm_pairs[2 * i]) * npt(d.r_inadm_pairs[2 * i + 1]) for i in range(d.n_r_inadm_pair))
    for i in range(d.n_r_adm_pair):
        a, b = d.r_adm_pairs[2 * i], d.r_adm_pairs[2 * i + 1]
        if lvl(a) == lvl(b):
            s += 2 * d.J_n[a] * d.J_n[b]
        elif lvl(a) > lvl(b):
            s += 2 * d.J_n[a] * npt(b)
        else:
            s += 2 * d.J_n[b] * npt(a)
    return s


def check(d):
    c = plan_check(d)
    n_up, n_dn, n_blk, n_jt, n_tiles, n_pg, ps_rows, pairs = c
    assert ps_rows > 0
    if d.n_r_adm_pair > 0:
        assert n_up > 0 and n_dn > 0
    if d.BD_JIT:
        assert n_blk == 0 and n_jt > 0 and n_tiles > 0
        assert pairs == pairs_from_lists(d)
        if d.krnl_dim == 1:
            assert n_pg > 0
    else:
        assert n_blk >= d.n_B + d.n_D - d.n_leaf_node and n_jt == 0 and pairs == 0
    return c


@pytest.mark.parametrize("name", ["coulomb_aot", "rpy_aot", "coulomb_jit", "gaussian_jit", "matern32_jit", "rpy_jit"])
def test_plan_of_golden_fixtures(name):
    h = O.DescHolder(arrays(os.path.join(GOLDEN, name + ".npz")))
    check(h.desc)


@pytest.mark.parametrize("kernel,n,leaf,jit", [
    ("coulomb", 20000, 400, 1),     # leaves and skeletons wider than 128 points
    ("gaussian", 8000, 200, 1),
    ("matern32", 6000, 300, 1),
    ("matern32", 1500, 3, 1),       # leaves of a few points: every panel group partial
    ("rpy", 3000, 100, 1),
    ("coulomb", 8000, 200, 0),
    ("rpy", 3000, 100, 0),
])
def test_plan_of_built_trees(kernel, n, leaf, jit):
    H = H2Matrix(kernel, make_points(kernel, n, 5), KERNEL_PARAMS[kernel], 1e-6, BD_JIT=jit, max_leaf_points=leaf)
    try:
        check(H.describe())
    finally:
        H.close()


def batch_plan_check(descs):
    lib = _abi.libh2gpu()
    arr = (_abi.Desc * len(descs))(*descs)
    cnt = (C.c_longlong * 8)()
    st = lib.h2gpu_batch_plan_check(arr, len(descs), cnt)
    assert st == _abi.H2GPU_OK, lib.h2gpu_last_error().decode()
    return list(cnt)


@pytest.mark.parametrize("kernel,jit", [("coulomb", 1), ("matern32", 1), ("rpy", 1), ("coulomb", 0), ("rpy", 0)])
def test_batched_plan_is_the_union_of_its_members(kernel, jit):
    """Members of different depths (and so different min_adm / max_level) merged into
    one image: the merged plan passes the self-check, and its tasks, tiles, panel
    groups and evaluated point pairs are the sums of the members' own (nothing is
    lost or paired across members)."""
    shapes = [(1500, 100), (6000, 60), (3000, 300)]
    Hs = [H2Matrix(kernel, make_points(kernel, n, 40 + i), KERNEL_PARAMS[kernel], 1e-6, BD_JIT=jit,
                   max_leaf_points=leaf) for i, (n, leaf) in enumerate(shapes)]
    try:
        ds = [H.describe() for H in Hs]
        assert len({(d.max_level, d.min_adm_level) for d in ds}) > 1
        own = [check(d) for d in ds]
        merged = batch_plan_check(ds)
        for k in (0, 1, 2, 3, 4, 5, 7):   # all but the partial-space size (pair units depend on the total work)
            assert merged[k] == sum(c[k] for c in own), k
    finally:
        for H in Hs:
            H.close()


def test_python_wrapper():
    from h2pack_b200 import plan_check as pc
    H = H2Matrix("gaussian", make_points("gaussian", 4000, 3), KERNEL_PARAMS["gaussian"], 1e-6, BD_JIT=1,
                 max_leaf_points=100)
    try:
        c = H.plan_check()
        assert list(c.values()) == plan_check(H.describe())
        assert c["jit_point_pairs"] == pairs_from_lists(H.describe())
        assert pc([H.describe(), H.describe()])["jit_point_pairs"] == 2 * c["jit_point_pairs"]
    finally:
        H.close()


def test_descriptors_of_one_handle_stay_valid():
    """Several descriptors of one handle are all usable at once: each describe() call
    owns its arrays until the handle is destroyed (a batch listing a matrix twice, or
    a descriptor kept across a later describe, read no freed memory)."""
    H = H2Matrix("coulomb", make_points("coulomb", 3000, 5), [], 1e-6, BD_JIT=0, max_leaf_points=100)
    try:
        d1 = H.describe()
        d2 = H.describe()
        d3 = H.describe()
        addr = [C.cast(d.U_nrow, C.c_void_p).value for d in (d1, d2, d3)]
        assert len(set(addr)) == 3           # storage of their own
        c1 = plan_check(d1)
        assert plan_check(d2) == c1 and plan_check(d3) == c1
        merged = batch_plan_check([d1, d2, d3])
        assert merged[2] == 3 * c1[2]       # stored-block tasks of three copies
        assert plan_check(d1) == c1          # the oldest is still intact
    finally:
        H.close()
