"""GPU drop-in against the reference on the same H2 representation.

The H2Pack handle is built by H2Pack's construction; the reference's CPU
H2P_matvec / H2P_matmul (oracle/_ref/libh2ref.so) and the GPU drop-in
(libH2Pack_gpu.so -> libh2gpu.so) are applied to the same handle and inputs.
Bar for the plain FP64 path: relative 2-norm difference <= 1e-12.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import KERNEL_PARAMS, build_kwargs, make_points, rel
from oracle import oracle as O
from h2pack_b200 import _abi
from h2pack_b200.h2pack import H2Matrix, direct_sum

pytestmark = pytest.mark.gpu
TOL64 = 1e-12
KERNELS = ["coulomb", "gaussian", "matern32", "rpy"]


def ref_matvec(h2pack, x):
    y = np.zeros_like(x)
    O.libref().H2P_matvec(h2pack, O.dptr(x), O.dptr(y))
    return y


def ref_matmul(h2pack, X):
    N, nv = X.shape
    Xc = np.ascontiguousarray(X)
    Y = np.zeros((N, nv))
    O.libref().H2P_matmul(h2pack, _abi.ROW_MAJOR, nv, O.dptr(Xc), nv, O.dptr(Y), nv)
    return Y


def build(kernel, n, jit, seed=7, **kw):
    coord = make_points(kernel, n, seed)
    args = build_kwargs(kernel)
    args.update(kw)
    return H2Matrix(kernel, coord, KERNEL_PARAMS[kernel], args.pop("reltol", 1e-6), BD_JIT=jit, **args)


@pytest.fixture(scope="module", params=[(k, j) for k in KERNELS for j in (0, 1)],
                ids=[f"{k}-{'jit' if j else 'aot'}" for k in KERNELS for j in (0, 1)])
def h2(request):
    kernel, jit = request.param
    n = 2500 if kernel == "rpy" else 6000
    H = build(kernel, n, jit)
    yield H
    H.close()


def test_matvec_fp64_matches_reference(h2):
    rng = np.random.default_rng(1)
    x = rng.random(h2.N) - 0.5
    assert rel(h2.matvec(x), ref_matvec(h2.h2pack, x)) < TOL64


@pytest.mark.parametrize("nv", [2, 3, 16, 21])
def test_matmul_fp64_matches_reference(h2, nv):
    rng = np.random.default_rng(nv)
    X = rng.standard_normal((h2.N, nv))
    Yr = ref_matmul(h2.h2pack, X)
    assert rel(h2.matmul(X), Yr) < TOL64
    assert rel(h2.matmul(X, _abi.COL_MAJOR), Yr) < TOL64


def test_matvec_matmul_consistent(h2):
    """extra/test_H2_matmul.h:48-83: matmul columns equal separate matvecs."""
    rng = np.random.default_rng(2)
    X = rng.standard_normal((h2.N, 5))
    Y = h2.matmul(X)
    for j in range(5):
        assert rel(Y[:, j], h2.matvec(X[:, j])) < 1e-13


def test_deterministic(h2):
    rng = np.random.default_rng(3)
    X = rng.standard_normal((h2.N, 4))
    assert np.array_equal(h2.matmul(X), h2.matmul(X))


@pytest.mark.parametrize("nv", [8, 16])
def test_mixed_precision_close(h2, nv):
    rng = np.random.default_rng(4)
    X = rng.standard_normal((h2.N, nv))
    Y64 = h2.matmul(X)
    h2.set_precision("mixed")
    try:
        Ym = h2.matmul(X)
    finally:
        h2.set_precision("fp64")
    assert rel(Ym, Y64) < 2e-6


def test_counters_updated(h2):
    before = h2.counters()["n_matvec"]
    h2.matmul(np.ones((h2.N, 3)))
    assert h2.counters()["n_matvec"] == before + 3


def test_error_vs_direct_sum_within_reltol():
    """The representation's error against the FP64 direct sum (examples/example_H2.c:131-141)."""
    H = build("coulomb", 8000, 0, seed=21)
    try:
        rng = np.random.default_rng(5)
        x = rng.random(H.N) - 0.5
        y = H.matvec(x)
        rows = rng.choice(H.N, 500, replace=False)
        coord = H.coord
        yd = direct_sum("coulomb", [], coord, x, coord[:, rows])
        assert rel(y[rows], yd) < 1e-5
    finally:
        H.close()


@pytest.mark.parametrize("kernel", KERNELS)
def test_direct_sum_matches_oracle(kernel):
    rng = np.random.default_rng(6)
    src = make_points(kernel, 1200, seed=8)
    kd = 3 if kernel == "rpy" else 1
    v = rng.standard_normal(1200 * kd)
    trg = src[:, rng.choice(1200, 200, replace=False)]
    p = KERNEL_PARAMS[kernel]
    assert rel(direct_sum(kernel, p, src, v, trg), O.direct_sum(_abi.KERNEL_IDS[kernel], p, src, v, trg)) < 1e-13


def test_reference_built_handle_through_dropin():
    """A JIT handle built by the reference library itself, applied by the drop-in with
    no extra call: the kernel is identified from the handle's own kernel function."""
    coord = make_points("matern32", 5000, 13)
    R = O.RefH2("matern32", [1.0], coord, 1e-6, BD_JIT=1, max_leaf_points=100)
    lib = _abi.libh2pack_gpu()
    try:
        x = np.random.default_rng(9).standard_normal(R.N)
        y = np.zeros(R.N)
        assert lib.H2P_gpu_matvec(R.h2pack, O.dptr(x), O.dptr(y)) == 0
        assert rel(y, R.matvec(x)) < TOL64
        # the void H2Pack signature on the same handle
        y2 = np.zeros(R.N)
        lib.H2P_matvec(R.h2pack, O.dptr(x), O.dptr(y2))
        assert np.array_equal(y, y2)
        # an explicit kernel id gives the same image
        p = np.array([1.0, 0, 0, 0])
        assert lib.H2P_gpu_set_kernel(R.h2pack, _abi.KRNL_MATERN32, O.dptr(p), 1) == 0
        y3 = np.zeros(R.N)
        assert lib.H2P_gpu_matvec(R.h2pack, O.dptr(x), O.dptr(y3)) == 0
        assert np.array_equal(y, y3)
    finally:
        lib.H2P_gpu_release(R.h2pack)
        R.close()


def test_jit_handle_with_a_wrong_explicit_kernel_differs():
    """H2P_gpu_set_kernel overrides the identification (a Gaussian handle declared
    Matern-3/2 is evaluated as Matern-3/2, so its result no longer matches)."""
    coord = make_points("gaussian", 1500, 14)
    R = O.RefH2("gaussian", [1.0], coord, 1e-6, BD_JIT=1, max_leaf_points=100)
    lib = _abi.libh2pack_gpu()
    try:
        x = np.ones(R.N)
        y = np.zeros(R.N)
        assert lib.H2P_gpu_matvec(R.h2pack, O.dptr(x), O.dptr(y)) == 0
        assert rel(y, R.matvec(x)) < TOL64
        p = np.array([1.0, 0, 0, 0])
        assert lib.H2P_gpu_set_kernel(R.h2pack, _abi.KRNL_MATERN32, O.dptr(p), 1) == 0
        assert lib.H2P_gpu_matvec(R.h2pack, O.dptr(x), O.dptr(y)) == 0
        assert rel(y, R.matvec(x)) > 1e-3
    finally:
        lib.H2P_gpu_release(R.h2pack)
        R.close()


def test_permutations_match_reference_semantics():
    H = build("gaussian", 3000, 1, seed=15)
    try:
        lib = H.lib
        x = np.arange(H.N, dtype=np.float64)
        px = np.zeros(H.N)
        lib.H2P_permute_vector_forward(H.h2pack, O.dptr(x), O.dptr(px))
        d = O.desc_to_arrays(H.describe())
        assert np.array_equal(px, x[d["fwd_pmt_idx"]])
        back = np.zeros(H.N)
        lib.H2P_permute_vector_backward(H.h2pack, O.dptr(px), O.dptr(back))
        assert np.array_equal(back, x)
    finally:
        H.close()


def test_small_problem_without_admissible_pairs():
    H = build("coulomb", 300, 0, seed=16, max_leaf_points=64)
    try:
        assert H.info["n_r_adm_pair"] == 0
        x = np.random.default_rng(1).standard_normal(H.N)
        assert rel(H.matvec(x), ref_matvec(H.h2pack, x)) < TOL64
    finally:
        H.close()


def test_zero_input_gives_zero():
    H = build("matern32", 2000, 1, seed=17)
    try:
        assert np.all(H.matvec(np.zeros(H.N)) == 0.0)
    finally:
        H.close()


def test_device_resident_matmul():
    import torch
    from h2pack_b200.h2pack import Image
    H = build("matern32", 4000, 1, seed=18)
    try:
        img = Image(H.describe())
        X = torch.randn(H.N, 16, dtype=torch.float64, device="cuda")
        Y = img.matmul_device(X)
        torch.cuda.synchronize()
        assert rel(Y.cpu().numpy(), ref_matmul(H.h2pack, X.cpu().numpy())) < TOL64
        img.close()
    finally:
        H.close()


@pytest.mark.parametrize("kernel", ["coulomb", "gaussian", "matern32", "rpy"])
@pytest.mark.parametrize("jit", [0, 1])
def test_hss_mode_matches_reference(kernel, jit):
    """HSS-mode handles (H2P_run_HSS) through the drop-in: the same phases over the HSS
    pair lists and minimum admissible level (src/H2Pack_matvec.c:101, :308, :773, :904),
    FP64 within 1e-12 of the reference's HSS H2P_matvec / H2P_matmul, mixed within 2e-6."""
    coord = make_points(kernel, 2500 if kernel == "rpy" else 5000, 61)
    R = O.RefH2(kernel, KERNEL_PARAMS[kernel], coord, 1e-6, BD_JIT=jit, hss=True, **build_kwargs(kernel))
    lib = _abi.libh2pack_gpu()
    try:
        rng = np.random.default_rng(62)
        x = rng.standard_normal(R.N)
        y = np.zeros(R.N)
        assert lib.H2P_gpu_matvec(R.h2pack, O.dptr(x), O.dptr(y)) == 0
        assert rel(y, R.matvec(x)) < TOL64
        X = rng.standard_normal((R.N, 16))
        Y = np.zeros_like(X)
        assert lib.H2P_gpu_matmul(R.h2pack, _abi.ROW_MAJOR, 16, O.dptr(X), 16, O.dptr(Y), 16) == 0
        Yr = R.matmul(X)
        assert rel(Y, Yr) < TOL64
        assert lib.H2P_gpu_set_precision(R.h2pack, _abi.PREC_MIXED) == 0
        assert lib.H2P_gpu_matmul(R.h2pack, _abi.ROW_MAJOR, 16, O.dptr(X), 16, O.dptr(Y), 16) == 0
        assert rel(Y, Yr) < 2e-6
    finally:
        lib.H2P_gpu_release(R.h2pack)
        R.close()
