"""Host-side behaviour of the H2Pack drop-in that needs no GPU.

Kernel identification: a JIT-mode H2Pack handle holds its kernel only as a function
pointer and a parameter pointer (src/H2Pack_typedef.h:160, :193).  The drop-in calls
that function on probe points and matches Coulomb, Gaussian, Matern-3/2 and RPY with
the handle's own parameter (H2P_gpu_kernel_of).  Handles built by the drop-in's own
construction library and by the reference library are both identified.
"""
import numpy as np
import pytest

from conftest import KERNEL_PARAMS, build_kwargs, make_points
from oracle import oracle as O
from h2pack_b200 import _abi
from h2pack_b200.h2pack import H2Matrix, kernel_of


@pytest.mark.parametrize("kernel", ["coulomb", "gaussian", "matern32", "rpy"])
@pytest.mark.parametrize("jit", [0, 1])
def test_kernel_identified_from_handle(kernel, jit):
    H = H2Matrix(kernel, make_points(kernel, 1500, 3), KERNEL_PARAMS[kernel], 1e-6, BD_JIT=jit,
                 **build_kwargs(kernel))
    try:
        name, p = H.kernel_of()
        assert name == kernel
        assert p == pytest.approx(KERNEL_PARAMS[kernel], rel=0, abs=0)
    finally:
        H.close()


@pytest.mark.parametrize("kernel,param", [("gaussian", [0.37]), ("matern32", [2.5]), ("coulomb", [3.0]),
                                          ("rpy", [0.25])])
def test_reference_library_handle_identified(kernel, param):
    """Handles built by the reference library (its own static kernel functions), other
    parameters; Coulomb with a parameter uses it as the value at r = 0."""
    R = O.RefH2(kernel, param, make_points(kernel, 1200, 4), 1e-6, BD_JIT=1, **build_kwargs(kernel))
    lib = _abi.libh2pack_gpu()
    try:
        name, p = kernel_of(lib, R.h2pack)
        assert name == kernel and p == param
    finally:
        lib.H2P_gpu_release(R.h2pack)
        R.close()


def test_explicit_kernel_overrides_identification():
    H = H2Matrix("gaussian", make_points("gaussian", 1200, 5), [1.0], 1e-6, BD_JIT=1, max_leaf_points=100)
    try:
        p = np.array([0.5, 0, 0, 0])
        assert H.lib.H2P_gpu_set_kernel(H.h2pack, _abi.KRNL_MATERN32, p.ctypes.data_as(_abi._dp), 1) == 0
        assert H.kernel_of() == ("matern32", [0.5])
    finally:
        H.close()
