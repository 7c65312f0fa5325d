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
    assert _abi.libh2gpu().h2gpu_abi_version() == 1


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    monkeypatch.setattr(_abi, "LIBH2GPU", str(tmp_path / "libh2gpu.so"))
    monkeypatch.setattr(_abi, "_cache", {})
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _abi.libh2gpu()
