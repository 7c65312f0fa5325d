"""Projection matrices of the construction on the GPU (H2P_gpu_build_uj).

H2Pack builds U and the skeleton sets J with an interpolative decomposition per node
(H2P_build_H2_UJ_proxy, src/H2Pack_build.c:32-270; H2P_ID_compress,
src/H2Pack_ID_compress.c:491-576).  The GPU path computes the same decompositions on
the device, one batch per tree level.  Pivot choices can differ where two column norms
tie to rounding, so the checks are structural and by accuracy:

- the partition and pair lists are unchanged, the skeleton sizes agree with H2Pack's
  to a few percent;
- every leaf's U holds the identity at its skeleton rows (U = P [I; E^T]);
- the FP64 apply of the GPU-built matrix is as accurate against the FP64 direct sum as
  the CPU-built one (within the construction tolerance);
- without a usable device the switch falls back to H2Pack's code (CPU test).
"""
import numpy as np
import pytest

from conftest import KERNEL_PARAMS, make_points, rel
from h2pack_b200 import direct_sum
from h2pack_b200.h2pack import H2Matrix


def _skeleton_sizes(H):
    d = H.describe()
    return np.array([d.J_n[i] for i in range(d.n_node)])


def test_switch_falls_back_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: the GPU path runs (GPU tests)")
    P = make_points("coulomb", 3000, 5)
    a = H2Matrix("coulomb", P, [], 1e-6, BD_JIT=1, max_leaf_points=100)
    n0 = a.lib.H2P_gpu_build_uj_count()
    b = H2Matrix("coulomb", P, [], 1e-6, BD_JIT=1, max_leaf_points=100, build_uj_gpu=True)
    try:
        assert b.lib.H2P_gpu_build_uj_count() == n0      # fell back to H2Pack's code
        assert np.array_equal(_skeleton_sizes(a), _skeleton_sizes(b))
    finally:
        a.close()
        b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["coulomb", "gaussian", "matern32"])
@pytest.mark.parametrize("jit", [1, 0])
def test_gpu_uj_as_accurate_as_h2pack(kernel, jit):
    P = make_points(kernel, 8000, 41)
    par = KERNEL_PARAMS[kernel]
    Hc = H2Matrix(kernel, P, par, 1e-6, BD_JIT=jit, max_leaf_points=200)
    n0 = Hc.lib.H2P_gpu_build_uj_count()
    Hg = H2Matrix(kernel, P, par, 1e-6, BD_JIT=jit, max_leaf_points=200, build_uj_gpu=True)
    try:
        assert Hg.lib.H2P_gpu_build_uj_count() == n0 + 1   # the device path ran (no fallback)
        for k in ("n_node", "max_level", "n_r_adm_pair", "n_r_inadm_pair", "krnl_mat_size"):
            assert Hc.info[k] == Hg.info[k], k
        sc, sg = _skeleton_sizes(Hc), _skeleton_sizes(Hg)
        assert abs(int(sg.sum()) - int(sc.sum())) <= 0.05 * sc.sum(), (sc.sum(), sg.sum())
        # leaves: U holds the identity at the skeleton rows
        d = Hg.describe()
        n = d.n_point
        coord = np.ctypeslib.as_array(d.coord, shape=(3 * n,)).reshape(3, n)
        for i in range(min(d.n_leaf_node, 16)):
            node = d.leaf_nodes[i]
            r, c = d.U_nrow[node], d.U_ncol[node]
            if c == 0:
                continue
            U = np.ctypeslib.as_array(d.U[node], shape=(r * d.U_ld[node],)).reshape(r, d.U_ld[node])[:, :c]
            s, e = d.pt_cluster[2 * node], d.pt_cluster[2 * node + 1]
            jc = np.ctypeslib.as_array(d.J_coord[node], shape=(3 * c,)).reshape(3, c)
            pts = coord[:, s:e + 1]
            rows = [int(np.argmin(((pts - jc[:, [k]]) ** 2).sum(0))) for k in range(c)]
            assert np.array_equal(U[rows], np.eye(c)), node
        rng = np.random.default_rng(3)
        x = rng.random(Hc.N) - 0.5
        rows = rng.choice(Hc.N, 2000, replace=False)
        yd = direct_sum(kernel, par, P, x, P[:, rows])
        ec = rel(Hc.matvec(x)[rows], yd)
        eg = rel(Hg.matvec(x)[rows], yd)
        assert eg <= max(3.0 * ec, 1e-6), (ec, eg)
    finally:
        Hc.close()
        Hg.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["gaussian", "matern32"])
def test_gpu_proxy_points_as_accurate_as_h2pack(kernel):
    """Numerical proxy points (H2P_generate_proxy_point_ID_file, generated afresh: no
    cache file) selected on the device give the construction H2Pack's accuracy."""
    P = make_points(kernel, 6000, 43)
    par = KERNEL_PARAMS[kernel]
    Hc = H2Matrix(kernel, P, par, 1e-6, BD_JIT=1, max_leaf_points=200, proxy="id")
    n0 = Hc.lib.H2P_gpu_build_pp_count()
    Hg = H2Matrix(kernel, P, par, 1e-6, BD_JIT=1, max_leaf_points=200, proxy="id", build_pp_gpu=True)
    try:
        assert Hg.lib.H2P_gpu_build_pp_count() > n0     # levels selected on the device
        sc, sg = _skeleton_sizes(Hc), _skeleton_sizes(Hg)
        assert abs(int(sg.sum()) - int(sc.sum())) <= 0.10 * sc.sum(), (sc.sum(), sg.sum())
        rng = np.random.default_rng(4)
        x = rng.random(Hc.N) - 0.5
        rows = rng.choice(Hc.N, 2000, replace=False)
        yd = direct_sum(kernel, par, P, x, P[:, rows])
        ec = rel(Hc.matvec(x)[rows], yd)
        eg = rel(Hg.matvec(x)[rows], yd)
        assert eg <= max(3.0 * ec, 1e-6), (ec, eg)
    finally:
        Hc.close()
        Hg.close()
