"""H2 matrices in H2Pack's on-disk format (h2pack_b200/h2file.py).

* A file written by H2Pack itself (H2P_store_to_file + H2Pack's JSON encoding, fixture
  made by tests/golden/make_golden.py) is read into a descriptor that passes the plan
  self-check; the C restatement of the apply on it reproduces H2Pack's own outputs on the
  stored matrix (CPU), and so does the GPU image (FP64, 1e-12).
* write_h2 -> read_h2 round trips every array exactly, for H2 and HSS handles and, with
  the extra point_radius field, for RPY (which H2Pack's own writer refuses).
"""
import os

import numpy as np
import pytest

from conftest import KERNEL_PARAMS, build_kwargs, make_points, rel
from oracle import oracle as O
from h2pack_b200 import plan_check
from h2pack_b200.h2file import read_h2, write_h2

FIX = os.path.join(os.path.dirname(__file__), "golden", "h2file_coulomb")


def fixture_file():
    f = read_h2(os.path.join(FIX, "meta.json"), os.path.join(FIX, "aux.json"), os.path.join(FIX, "h2.bin"), "coulomb")
    return f, np.load(os.path.join(FIX, "io.npz"))


def test_reads_a_file_written_by_h2pack():
    f, z = fixture_file()
    assert plan_check(f.desc)["block_tasks"] > 0
    assert rel(O.matvec(f.desc, z["x"]), z["y_ref"]) < 1e-14
    assert rel(O.matmul(f.desc, z["X"]), z["Y_ref"]) < 1e-14
    # the caller's point order is restored from the file's permutation
    coord = np.ascontiguousarray(z["coord_in"])
    perm = f.a["fwd_pmt_idx"]
    assert np.array_equal(f.a["coord"][:, :], coord[:, perm])


@pytest.mark.parametrize("kernel,hss", [("coulomb", False), ("gaussian", True), ("rpy", False), ("rpy", True)])
def test_write_read_round_trip(kernel, hss, tmp_path):
    R = O.RefH2(kernel, KERNEL_PARAMS[kernel], make_points(kernel, 1500, 71), 1e-6, BD_JIT=0, hss=hss,
                **build_kwargs(kernel))
    try:
        d = R.describe()
        paths = [str(tmp_path / n) for n in ("m.json", "a.json", "h.bin")]
        write_h2(d, *paths, is_hss=hss)
        f = read_h2(*paths, kernel, KERNEL_PARAMS[kernel])
        ref = O.desc_to_arrays(d)
        for k in ("n_child", "node_level", "pt_cluster", "mat_cluster", "leaf_nodes", "U_nrow", "U_ncol",
                  "r_adm_pairs", "r_inadm_pairs", "B_nrow", "B_ncol", "D_nrow", "D_ncol", "J_n", "fwd_pmt_idx",
                  "bwd_pmt_idx"):
            assert np.array_equal(np.asarray(f.a[k]).ravel(), np.asarray(ref[k]).ravel()), k
        assert np.array_equal(f.a["coord"], ref["coord"].reshape(f.a["coord"].shape))
        assert f.a["min_adm_level"] == d.min_adm_level
        x = np.random.default_rng(72).standard_normal(R.N)
        assert rel(O.matvec(f.desc, x), R.matvec(x)) < 1e-14
    finally:
        R.close()


@pytest.mark.gpu
def test_file_applied_on_the_gpu(tmp_path):
    from h2pack_b200 import Image
    f, z = fixture_file()
    img = Image(f.desc)
    try:
        assert rel(img.matvec(z["x"]), z["y_ref"]) < 1e-12
        assert rel(img.matmul(z["X"]), z["Y_ref"]) < 1e-12
    finally:
        img.close()
    # an RPY matrix through the extended format
    R = O.RefH2("rpy", KERNEL_PARAMS["rpy"], make_points("rpy", 1500, 73), 1e-8, BD_JIT=0, **build_kwargs("rpy"))
    try:
        paths = [str(tmp_path / n) for n in ("m.json", "a.json", "h.bin")]
        write_h2(R.describe(), *paths)
        g = read_h2(*paths, "rpy", KERNEL_PARAMS["rpy"])
        img = Image(g.desc, "mixed")
        X = np.random.default_rng(74).standard_normal((R.N, 64))
        Yr = R.matmul(X)
        assert rel(img.matmul(X), Yr) < 2e-6
        img.set_precision("fp64")
        assert rel(img.matmul(X), Yr) < 1e-12
        img.close()
    finally:
        R.close()
