"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the
reference library): the oracle restatement on CPU, and the GPU engine through the
C ABI, must reproduce H2Pack's own H2P_matvec / H2P_matmul outputs."""
import glob
import os

import numpy as np
import pytest

from conftest import rel
from oracle import oracle as O
from h2pack_b200 import _abi

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
IDS = [os.path.basename(p)[:-4] for p in GOLDEN]


def load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def holder(f):
    keys = [k for k in f if k not in ("x", "y_ref", "X", "Y_ref", "coord_in", "reltol")]
    a = {k: (int(f[k]) if f[k].ndim == 0 else f[k]) for k in keys}
    return O.DescHolder(a)


def test_fixtures_present():
    assert len(GOLDEN) >= 6


@pytest.mark.parametrize("path", GOLDEN, ids=IDS)
def test_oracle_reproduces_reference(path):
    f = load(path)
    h = holder(f)
    assert rel(O.matvec(h.desc, f["x"]), f["y_ref"]) < 1e-13
    assert rel(O.matmul(h.desc, f["X"]), f["Y_ref"]) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN, ids=IDS)
def test_gpu_fp64_reproduces_reference(path):
    from h2pack_b200 import Image
    f = load(path)
    h = holder(f)
    img = Image(h.desc, precision="fp64")
    try:
        assert rel(img.matvec(f["x"]), f["y_ref"]) < 1e-12
        assert rel(img.matmul(f["X"]), f["Y_ref"]) < 1e-12
        assert rel(img.matmul(f["X"], _abi.COL_MAJOR), f["Y_ref"]) < 1e-12
    finally:
        img.close()


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN, ids=IDS)
def test_gpu_mixed_close_to_reference(path):
    from h2pack_b200 import Image
    f = load(path)
    h = holder(f)
    img = Image(h.desc, precision="mixed")
    try:
        # FP32 blocks / FP32 re-centred evaluation, FP64 sums across blocks
        assert rel(img.matvec(f["x"]), f["y_ref"]) < 2e-6
        assert rel(img.matmul(f["X"]), f["Y_ref"]) < 2e-6
    finally:
        img.close()
