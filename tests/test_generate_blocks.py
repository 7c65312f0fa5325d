"""Stored B / D blocks generated on the GPU (h2gpu_options.blocks = H2GPU_BLOCKS_GENERATE).

The generated arenas are compared entry by entry with what H2Pack's own construction
stores (H2P_build_B_AOT, src/H2Pack_build.c:789-889; H2P_build_D_AOT, :1034-1140) for
the same handle: FP64 to a few ulps (the same formulas; the exponential may round its
last bit differently), FP32 to the rounding of those values.  Images with generated
blocks apply like images with uploaded ones, and a handle constructed in JIT mode
(no stored blocks on the host) is applied in stored-block mode on the GPU and matches
the reference's own JIT H2P_matmul on that handle.
"""
import numpy as np
import pytest

from conftest import KERNEL_PARAMS, build_kwargs, make_points, rel
from oracle import oracle as O
from h2pack_b200 import Image, _abi
from h2pack_b200.h2pack import H2Matrix

pytestmark = pytest.mark.gpu
KERNELS = ["coulomb", "gaussian", "matern32", "rpy"]


def ref_handle(kernel, n, seed, jit=0):
    return O.RefH2(kernel, KERNEL_PARAMS[kernel], make_points(kernel, n, seed),
                   1e-8 if kernel == "rpy" else 1e-6, BD_JIT=jit, **build_kwargs(kernel))


def host_blocks(d, which):
    n = int((d.B_ptr if which == "B" else d.D_ptr)[d.n_B if which == "B" else d.n_D])
    return np.ctypeslib.as_array(d.B_data if which == "B" else d.D_data, shape=(n,)).copy()


@pytest.mark.parametrize("kernel", KERNELS)
def test_generated_blocks_equal_h2pack_build(kernel):
    R = ref_handle(kernel, 3000 if kernel != "rpy" else 1500, 40)
    d = R.describe()
    img64 = Image(d, "fp64", blocks="generate")
    img32 = Image(d, "mixed", blocks="generate")
    try:
        for which in ("B", "D"):
            ref = host_blocks(d, which)
            if ref.size == 0:
                continue
            g64 = img64.blocks(which, ref.size)
            scale = np.abs(ref).max()
            assert np.max(np.abs(g64 - ref)) <= 1e-14 * scale, which
            # FP32 arena: the FP64 values rounded to FP32
            g32 = img32.blocks(which, ref.size)
            assert np.array_equal(g32, g64.astype(np.float32).astype(np.float64)), which
        x = np.random.default_rng(41).standard_normal((R.N, 5))
        y_ref = R.matmul(x)
        assert rel(img64.matmul(x), y_ref) < 1e-12
        assert rel(img32.matmul(x), y_ref) < 2e-6
    finally:
        img64.close()
        img32.close()
        R.close()


@pytest.mark.parametrize("kernel", KERNELS)
def test_jit_handle_applied_with_generated_blocks(kernel):
    """Construction in JIT mode (U, skeletons, pair lists and block metadata only), blocks
    generated on the GPU: the stored-block apply equals the reference's JIT apply."""
    R = ref_handle(kernel, 4000 if kernel != "rpy" else 2000, 42, jit=1)
    d = R.describe()
    assert d.B_data is None or not bool(d.B_data)
    img = Image(d, "fp64", blocks="generate")
    mix = Image(d, "mixed", blocks="generate")
    try:
        st = img.stats()
        assert st["bytes_B"] > 0 and st["n_tasks_B"] > 0      # applied as stored blocks
        x = np.random.default_rng(43).standard_normal((R.N, 16))
        y_ref = R.matmul(x)
        assert rel(img.matmul(x), y_ref) < 1e-12
        assert rel(mix.matmul(x), y_ref) < 2e-6
        # an FP32-only image refuses FP64 applies
        with pytest.raises(RuntimeError, match="STATE"):
            mix.set_precision("fp64")
    finally:
        img.close()
        mix.close()
        R.close()


def test_generated_and_uploaded_images_agree_on_device():
    """Device-resident applies of an image with uploaded blocks and one with generated
    blocks of the same handle agree to rounding."""
    import torch
    R = ref_handle("coulomb", 2500, 44)
    d = R.describe()
    a = Image(d, "fp64")
    b = Image(d, "fp64", blocks="generate")
    try:
        x = torch.randn(R.N, 8, dtype=torch.float64, device="cuda")
        ya = a.matmul_device(x)
        yb = b.matmul_device(x)
        torch.cuda.synchronize()
        assert rel(yb.cpu().numpy(), ya.cpu().numpy()) < 1e-14
    finally:
        a.close()
        b.close()
        R.close()
