"""The no-allocation apply (h2gpu_matvec_device_noalloc) against the regular device
apply (h2gpu_matmul_device) of the same image.

The no-allocation entry point is for callers that cannot allocate device memory when
they apply the matrix (device memory owned by another allocator, or code that must not
stall on cudaMalloc/cudaFree, which synchronize the device).  Its work buffers live in a
fixed 16 MiB device array of the library; it must give the same result as the regular
path on two calls in a row (the array keeps the previous call's contents), and reject
images that need more work space.  This file is collected last on purpose.
"""
import os

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def image_from(name, precision="fp64"):
    from oracle import oracle as O
    from h2pack_b200 import Image
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    keep = ("x", "y_ref", "X", "Y_ref", "coord_in", "reltol")
    h = O.DescHolder({k: (int(z[k]) if z[k].ndim == 0 else z[k]) for k in z.files if k not in keep})
    return Image(h.desc, precision=precision), h


@pytest.mark.parametrize("name,precision", [("coulomb_aot", "fp64"), ("matern32_jit", "fp64"),
                                            ("rpy_jit", "fp64"), ("gaussian_jit", "mixed")])
def test_noalloc_matches_regular_apply_twice(name, precision):
    import torch
    img, _h = image_from(name, precision)
    try:
        g = torch.Generator(device="cuda").manual_seed(5)
        x = torch.randn(img.N, 1, dtype=torch.float64, device="cuda", generator=g)
        y_ref = img.matmul_device(x)            # regular path (allocates its work buffers)
        torch.cuda.synchronize()
        y_ref = y_ref[:, 0].cpu().numpy()
        x0 = x[:, 0].contiguous()
        ys = [torch.full((img.N,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
        torch.cuda.synchronize()
        free_before = None
        for y in ys:                            # the scratch keeps the previous call's contents
            img.matvec_device_noalloc(x0, y)
            torch.cuda.synchronize()
            if free_before is None:
                # the first call on the device may load the library's device module (and
                # with it the scratch array); later calls allocate nothing on the device
                free_before = torch.cuda.mem_get_info()[0]
            else:
                assert torch.cuda.mem_get_info()[0] == free_before
            assert rel(y.cpu().numpy(), y_ref) < 1e-12
    finally:
        img.close()


def test_noalloc_rejects_images_beyond_the_limit():
    import torch
    from conftest import make_points
    from h2pack_b200 import H2Matrix
    H = H2Matrix("coulomb", make_points("coulomb", 40000, 3), [], 1e-6, BD_JIT=0, max_leaf_points=300)
    try:
        img = H.image()
        x = torch.zeros(H.N, dtype=torch.float64, device="cuda")
        y = torch.zeros_like(x)
        with pytest.raises(RuntimeError, match="limited to"):
            img.matvec_device_noalloc(x, y)
    finally:
        H.close()


def test_noalloc_refuses_mixed_image_before_its_first_apply():
    """A mixed-precision image holds FP32 copies of U/B/D only after one allocating
    apply; before that the no-allocation entry point refuses it (status STATE) and
    leaves the caller's current device unchanged."""
    import torch
    img, _h = image_from("coulomb_aot", "mixed")
    try:
        x = torch.randn(img.N, dtype=torch.float64, device="cuda")
        y = torch.zeros_like(x)
        dev = torch.cuda.current_device()
        with pytest.raises(RuntimeError, match="STATE"):
            img.matvec_device_noalloc(x, y)
        assert torch.cuda.current_device() == dev
        img.matmul_device(x[:, None].contiguous())     # makes the FP32 copies
        img.matvec_device_noalloc(x, y)
        torch.cuda.synchronize()
        assert torch.isfinite(y).all()
    finally:
        img.close()
