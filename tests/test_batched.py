"""Batched form: many independent representations in one image (flattened
cross-matrix task lists, one launch per phase per tree level), CUDA-graph replay
and the autotuner.  Each member's result in the batch must equal its result alone."""
import glob
import os

import numpy as np
import pytest

from conftest import rel
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def holder(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    keep = ("x", "y_ref", "X", "Y_ref", "coord_in", "reltol")
    return O.DescHolder({k: (int(z[k]) if z[k].ndim == 0 else z[k]) for k in z.files if k not in keep}), z


def test_batch_of_mismatched_kernels_is_rejected():
    from h2pack_b200 import Image
    a, _ = holder("coulomb_jit")
    b, _ = holder("gaussian_jit")
    with pytest.raises(RuntimeError, match="INVALID"):
        Image.batch([a.desc, b.desc])


@pytest.mark.gpu
@pytest.mark.parametrize("names,precision", [
    (["coulomb_aot", "coulomb_aot"], "fp64"),
    (["matern32_jit", "matern32_jit"], "fp64"),
    (["matern32_jit", "matern32_jit"], "mixed"),
])
def test_batch_equals_members_alone(names, precision):
    import torch
    from h2pack_b200 import Image
    hs = [holder(n) for n in names]
    batch = Image.batch([h.desc for h, _ in hs], precision=precision)
    alone = [Image(h.desc, precision=precision) for h, _ in hs]
    try:
        g = torch.Generator(device="cuda").manual_seed(1)
        X = torch.randn(batch.N, 8, dtype=torch.float64, device="cuda", generator=g)
        Yb = batch.matmul_device(X).cpu().numpy()
        off = 0
        for img in alone:
            n = img.N
            Ya = img.matmul_device(X[off:off + n].contiguous()).cpu().numpy()
            assert rel(Yb[off:off + n], Ya) < 1e-14
            off += n
    finally:
        batch.close()
        for img in alone:
            img.close()


@pytest.mark.gpu
def test_batch_fp64_matches_reference_outputs():
    from h2pack_b200 import Image
    hs = [holder(n) for n in ("gaussian_jit", "gaussian_jit")]
    batch = Image.batch([h.desc for h, _ in hs])
    try:
        X = np.concatenate([z["X"] for _, z in hs])
        Y = batch.matmul(X)
        off = 0
        for _, z in hs:
            n = z["X"].shape[0]
            assert rel(Y[off:off + n], z["Y_ref"]) < 1e-12
            off += n
    finally:
        batch.close()


@pytest.mark.gpu
def test_graph_replay_and_autotune_match_eager():
    import torch
    from h2pack_b200 import Image
    h, z = holder("matern32_jit")
    img = Image(h.desc, precision="mixed")
    try:
        X = torch.randn(img.N, 16, dtype=torch.float64, device="cuda")
        Y0 = img.matmul_device(X).clone()
        nv, tc = img.autotune(X, torch.empty_like(X))
        assert nv in (4, 8, 16)
        Y1 = torch.zeros_like(X)
        img.graph_capture(X, Y1)
        Y1.zero_()
        img.graph_launch()
        torch.cuda.synchronize()
        assert rel(Y1.cpu().numpy(), Y0.cpu().numpy()) < 2e-6
        X.copy_(torch.randn_like(X))          # the graph reads the same buffer: new inputs, new outputs
        img.graph_launch()
        Y2 = img.matmul_device(X)
        torch.cuda.synchronize()
        assert rel(Y1.cpu().numpy(), Y2.cpu().numpy()) < 2e-6
    finally:
        img.close()
