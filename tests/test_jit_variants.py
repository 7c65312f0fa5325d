"""The FP32 kernel variants against the FP64 apply of the same image: for JIT images
CUDA cores, tensor cores per target and tensor cores per unordered pair; for stored
blocks CUDA cores, warp-level tensor-core MMAs and tcgen05 (TMEM accumulators).

The reference evaluates every JIT block from both sides with one bi-matvec
(src/H2Pack_matvec.c:170-236, H2P_matvec_fwd_transform/intmd_mult_JIT); the pair
variant does the same per unordered pair on the GPU.  Bar: relative 2-norm error of
the mixed apply <= 2e-6, bitwise repeatable.
"""
import numpy as np
import pytest

from conftest import rel
from test_batched import holder

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["matern32_jit", "coulomb_jit", "gaussian_jit", "coulomb_aot", "rpy_aot"])
@pytest.mark.parametrize("nv", [8, 16, 5])
def test_variants_match_fp64(name, nv):
    import torch
    from h2pack_b200 import Image
    h, _ = holder(name)
    img = Image(h.desc, precision="fp64")
    try:
        X = torch.randn(img.N, nv, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(nv))
        Y64 = img.matmul_device(X).cpu().numpy()
        img.set_precision("mixed")
        outs = {}
        for var in (("simt", "tc", "pair") if name.endswith("jit") else ("simt", "tc", "tcgen05")):
            img.set_jit_variant(var)
            Ya = img.matmul_device(X).cpu().numpy()
            Yb = img.matmul_device(X).cpu().numpy()
            assert np.array_equal(Ya, Yb), var
            assert rel(Ya, Y64) < 2e-6, var
            outs[var] = Ya
        # the variants differ only by FP32 rounding
        assert rel(outs["simt"], outs["tc"]) < 2e-6
    finally:
        img.close()


@pytest.mark.parametrize("name", ["rpy_jit", "coulomb_aot"])
def test_pair_variant_refused(name):
    from h2pack_b200 import Image
    h, _ = holder(name)
    img = Image(h.desc, precision="mixed")
    try:
        with pytest.raises(RuntimeError):
            img.set_jit_variant("pair")
        img.set_jit_variant("tc")
    finally:
        img.close()


def test_tcgen05_variant_refused_for_jit_images():
    from h2pack_b200 import Image
    h, _ = holder("matern32_jit")
    img = Image(h.desc, precision="mixed")
    try:
        with pytest.raises(RuntimeError):
            img.set_jit_variant("tcgen05")
    finally:
        img.close()
