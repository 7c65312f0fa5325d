"""Wide right-hand-side panels of mixed stored-block images (tcgen05 kernel k_blk_bf3w).

A mixed-precision image with stored blocks applies up to 64 right-hand sides per pass,
so a 64-column matmul reads every B / D block once (H2P_matmul applies each block to up
to mm_max_n_vec right-hand sides per read, src/H2Pack_matmul.c:497).  The results are
checked against H2Pack's own FP64 H2P_matmul on the same handle (relative 2-norm within
the FP32-storage tolerance 2e-6 used for every mixed stored-block test) and against the
same image restricted to panels of 16.
"""
import numpy as np
import pytest

from conftest import KERNEL_PARAMS, build_kwargs, make_points, rel
from oracle import oracle as O
from h2pack_b200 import Image, _abi

pytestmark = pytest.mark.gpu
TOL_MIXED = 2e-6


def ref(kernel, n, seed, reltol=None, jit=0):
    return O.RefH2(kernel, KERNEL_PARAMS[kernel], make_points(kernel, n, seed),
                   reltol or (1e-8 if kernel == "rpy" else 1e-6), BD_JIT=jit, **build_kwargs(kernel))


@pytest.mark.parametrize("kernel,n", [("rpy", 3000), ("coulomb", 6000), ("gaussian", 5000)])
@pytest.mark.parametrize("nvec", [64, 20, 33])
def test_wide_panels_match_reference(kernel, n, nvec):
    R = ref(kernel, n, 50)
    d = R.describe()
    img = Image(d, "mixed")
    narrow = Image(d, "mixed", max_n_vec=16)
    try:
        X = np.random.default_rng(51).standard_normal((R.N, nvec))
        Y_ref = R.matmul(X)
        Y = img.matmul(X)
        assert rel(Y, Y_ref) < TOL_MIXED
        Yn = narrow.matmul(X)
        assert rel(Y, Yn) < TOL_MIXED
        # column-major storage through the same wide path
        Yc = img.matmul(X, layout=_abi.COL_MAJOR)
        assert np.array_equal(Yc, Y)
    finally:
        img.close()
        narrow.close()
        R.close()


def test_one_pass_for_64_columns():
    """64 right-hand sides take one pass over the phases (the 64-wide block products run
    as two launches per block list instead of one, plus one split of the input rows per
    list), the narrow image four passes."""
    R = ref("rpy", 2500, 52)
    d = R.describe()
    img = Image(d, "mixed")
    narrow = Image(d, "mixed", max_n_vec=16)
    try:
        X = np.random.default_rng(53).standard_normal((R.N, 64))

        def launches(im, cols):
            s0 = im.stats()["n_launches"]
            im.matmul(X[:, :cols])
            return im.stats()["n_launches"] - s0
        assert launches(img, 64) == launches(img, 16) + 4
        assert launches(narrow, 64) == 4 * launches(narrow, 16)
        st = img.stats()
        assert st["bytes_B"] > 0
    finally:
        img.close()
        narrow.close()
        R.close()


def test_wide_panels_with_generated_blocks_and_device_apply():
    """JIT-mode construction, FP32 blocks generated on the device, 64 device-resident
    right-hand sides: equals the reference's JIT H2P_matmul within the mixed tolerance,
    and repeated applies are bitwise identical."""
    import torch
    R = ref("rpy", 3000, 54, jit=1)
    img = Image(R.describe(), "mixed", blocks="generate")
    try:
        X = torch.randn(R.N, 64, dtype=torch.float64, device="cuda")
        Y1 = img.matmul_device(X)
        Y2 = img.matmul_device(X)
        torch.cuda.synchronize()
        assert torch.equal(Y1, Y2)
        Y_ref = R.matmul(X.cpu().numpy())
        assert rel(Y1.cpu().numpy(), Y_ref) < TOL_MIXED
    finally:
        img.close()
        R.close()
