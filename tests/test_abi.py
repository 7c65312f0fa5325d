"""The C-ABI libraries load and export every symbol include/*.h declares (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT
from h2pack_b200 import _abi


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b(h2gpu_[a-z_]+|H2P_[A-Za-z_]+)\s*\(", txt)
    return sorted(set(names))


def test_h2gpu_exports_every_declared_symbol():
    lib = C.CDLL(_abi.LIBH2GPU)
    names = declared("h2gpu.h")
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_abi.H2GPU_SYMBOLS)


def test_dropin_exports_every_declared_symbol():
    _abi.libh2gpu()
    lib = C.CDLL(_abi.LIBH2PACK_GPU)
    names = declared("h2p_dropin.h")
    for n in names:
        assert hasattr(lib, n), n
    assert "H2P_matvec" in names and "H2P_matmul" in names


def test_abi_version():
    assert _abi.libh2gpu().h2gpu_abi_version() == 2


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    monkeypatch.setattr(_abi, "LIBH2GPU", str(tmp_path / "libh2gpu.so"))
    monkeypatch.setattr(_abi, "_cache", {})
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _abi.libh2gpu()


def test_cg_engine_argument_checks_without_gpu():
    """The CG engine refuses bad handles and arguments before any CUDA call."""
    lib = _abi.libh2gpu()
    h = C.c_void_p()
    assert lib.h2gpu_cg_create(None, 1e-2, 0, C.byref(h)) == _abi.H2GPU_OK - 1
    assert lib.h2gpu_cg_admit(None, 0, _abi.CG_PCG, None, 1e-6, 10) == _abi.H2GPU_OK - 1
    assert lib.h2gpu_cg_step(None, 1) == _abi.H2GPU_OK - 1
    assert lib.h2gpu_cg_check(None) == _abi.H2GPU_OK - 1
    assert lib.h2gpu_cg_take(None, 0, None) == _abi.H2GPU_OK - 1
    assert lib.h2gpu_cg_destroy(None) == _abi.H2GPU_OK
    assert b"NULL" in lib.h2gpu_last_error()
