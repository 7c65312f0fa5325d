"""The pipe-peak micro-benchmark behind the JIT roofline (h2gpu_measure_peaks): FP32 FMA
and MUFU throughput of the device, in plausible ranges of a B200 (148 SMs, <= 1.965 GHz:
nominal 74.4 TFLOP/s FP32 and 4.65 10^12 MUFU ops/s)."""
import ctypes as C

import pytest

from h2pack_b200 import _abi

pytestmark = pytest.mark.gpu


def test_measured_peaks_are_plausible():
    lib = _abi.libh2gpu()
    f, m = C.c_double(), C.c_double()
    assert lib.h2gpu_measure_peaks(-1, C.byref(f), C.byref(m)) == 0
    assert 20.0 < f.value < 160.0, f.value
    assert 1.0 < m.value < 20.0, m.value
