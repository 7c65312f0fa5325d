import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# every image the tests create first passes the host-side plan self-check
# (h2gpu_plan_check: slots written and summed once, tasks inside their arrays, ...)
os.environ.setdefault("H2G_PLAN_CHECK", "1")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def make_points(kernel: str, n: int, seed: int):
    """Points uniform in [0, n^(1/3)]^3; RPY: radius row of 1 in a cube sized for volume fraction 0.1."""
    rng = np.random.default_rng(seed)
    if kernel == "rpy":
        L = (n * 4.0 * np.pi / 3.0 / 0.1) ** (1.0 / 3.0)
        return np.vstack([rng.random((3, n)) * L, np.ones((1, n))])
    return rng.random((3, n)) * n ** (1.0 / 3.0)


KERNEL_PARAMS = {"coulomb": [], "gaussian": [1.0], "matern32": [1.0], "rpy": [1.0 / (6.0 * np.pi)]}


def build_kwargs(kernel: str):
    """Leaf settings of the reference drivers (examples/example_H2_RPY.c:55-64 for RPY)."""
    if kernel == "rpy":
        return dict(max_leaf_points=100, max_leaf_size=4.0)
    return dict(max_leaf_points=100, max_leaf_size=0.0)
