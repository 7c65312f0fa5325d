"""Host-side checks of the descriptor: malformed representations are rejected with
H2GPU_ERR_INVALID before anything touches a GPU (the fault injection of this path is
on the host).  Runs without a GPU."""
import copy
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from h2pack_b200 import _abi
from h2pack_b200.h2pack import Image

FIX = os.path.join(os.path.dirname(__file__), "golden", "coulomb_aot.npz")
FIXJ = os.path.join(os.path.dirname(__file__), "golden", "matern32_jit.npz")


def arrays(path):
    z = np.load(path)
    return {k: (int(z[k]) if z[k].ndim == 0 else z[k].copy()) for k in z.files
            if k not in ("x", "y_ref", "X", "Y_ref", "coord_in", "reltol")}


def status_of(a):
    h = O.DescHolder(a)
    try:
        img = Image(h.desc)
        img.close()
        return 0
    except RuntimeError as e:
        msg = str(e)
        assert "status" in msg
        return int(msg.split("status ")[1].split(" ")[0])


def corrupt(path, fn):
    a = arrays(path)
    fn(a)
    return status_of(a)


@pytest.mark.parametrize("name,fn", [
    ("negative U size", lambda a: a["U_ncol"].__setitem__(5, -3)),
    ("adm pair out of range", lambda a: a["r_adm_pairs"].__setitem__(0, 10 ** 6)),
    ("inadm pair not leaf", lambda a: a["r_inadm_pairs"].__setitem__(0, int(np.flatnonzero(a["n_child"] > 0)[0]))),
    ("bad permutation", lambda a: a["fwd_pmt_idx"].__setitem__(1, a["fwd_pmt_idx"][0])),
    ("pt_cluster past n_point", lambda a: a["pt_cluster"].__setitem__(1, 10 ** 7)),
    ("mat_cluster mismatch", lambda a: a["mat_cluster"].__setitem__(0, 3)),
    ("wrong B shape", lambda a: a["B_nrow"].__setitem__(0, a["B_nrow"][0] + 1)),
    ("bad level list", lambda a: a["level_nodes"].__setitem__(0, -7)),
])
def test_malformed_descriptor_rejected(name, fn):
    assert corrupt(FIX, fn) == -1, name


def test_jit_without_kernel_id_rejected():
    def fn(a):
        a["kernel_id"] = 0
    assert corrupt(FIXJ, fn) == -1


def test_jit_skeleton_mismatch_rejected():
    def fn(a):
        n = int(np.flatnonzero(a["J_n"] > 0)[0])
        a["J_n"][n] += 1
        a["J_off"][n + 1:] += a["xpt_dim"]
        a["J_data"] = np.concatenate([a["J_data"], np.zeros(a["xpt_dim"])])
    assert corrupt(FIXJ, fn) == -1


def test_no_gpu_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert status_of(arrays(FIX)) == -3
