"""Generate the golden fixtures of tests/golden from the reference H2Pack library.

Each fixture is an H2 representation built by H2Pack's construction (through
oracle/_ref/libh2ref.so, compiled from H2Pack's sources), flattened to plain
arrays, plus seeded inputs and the outputs of H2Pack's own CPU H2P_matvec and
H2P_matmul on that representation.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from conftest import KERNEL_PARAMS, make_points  # noqa: E402
from oracle import oracle as O  # noqa: E402

FIXTURES = [
    # name, kernel, n, BD_JIT, max_leaf_points, max_leaf_size, reltol
    ("coulomb_jit", "coulomb", 1600, 1, 64, 0.0, 1e-6),
    ("gaussian_jit", "gaussian", 1600, 1, 64, 0.0, 1e-6),
    ("matern32_jit", "matern32", 1600, 1, 64, 0.0, 1e-6),
    ("rpy_jit", "rpy", 700, 1, 48, 4.0, 1e-6),
    ("coulomb_aot", "coulomb", 500, 0, 40, 0.0, 1e-6),
    ("rpy_aot", "rpy", 200, 0, 32, 4.0, 1e-8),
]


def main():
    for name, kernel, n, jit, mlp, mls, tol in FIXTURES:
        coord = make_points(kernel, n, seed=1234)
        R = O.RefH2(kernel, KERNEL_PARAMS[kernel], coord, tol, max_leaf_points=mlp, max_leaf_size=mls,
                    BD_JIT=jit, proxy="surface")
        rng = np.random.default_rng(99)
        x = rng.random(R.N) - 0.5
        X = rng.standard_normal((R.N, 3))
        y = R.matvec(x)
        Y = R.matmul(X)
        arrays = O.desc_to_arrays(R.describe())
        out = {k: np.asarray(v) for k, v in arrays.items()}
        out.update(x=x, y_ref=y, X=X, Y_ref=Y, coord_in=coord, reltol=np.array(tol))
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(name, R.info["n_node"], R.info["n_leaf_node"], os.path.getsize(path) // 1024, "KiB")
        R.close()


if __name__ == "__main__":
    main()
