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


H2FILE_DIR = os.path.join(HERE, "h2file_coulomb")
REF_EXAMPLES = os.environ.get("H2PACK_EXAMPLES", "/root/reference/examples")


def make_h2file():
    """An H2 matrix stored by H2Pack itself (H2P_store_to_file, src/H2Pack_file_IO.c:17-218,
    whose JSON encoding is done by H2Pack's examples/meta_txt_to_json.py, run here from the
    H2Pack tree in a scratch directory), plus inputs and H2Pack's own H2P_matvec /
    H2P_matmul outputs on the stored representation."""
    import ctypes as C
    import shutil
    import tempfile
    coord = make_points("coulomb", 400, seed=4321)
    R = O.RefH2("coulomb", [], coord, 1e-6, max_leaf_points=40, BD_JIT=0, proxy="surface")
    os.makedirs(H2FILE_DIR, exist_ok=True)
    lib = O.libref()
    lib.H2P_store_to_file.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p]
    lib.H2P_store_to_file.restype = None
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        shutil.copy(os.path.join(REF_EXAMPLES, "meta_txt_to_json.py"), tmp)
        os.chmod(os.path.join(tmp, "meta_txt_to_json.py"), 0o755)
        os.chdir(tmp)
        try:
            lib.H2P_store_to_file(R.h2pack, b"meta.json", b"aux.json", b"h2.bin")
        finally:
            os.chdir(cwd)
        for f in ("meta.json", "aux.json", "h2.bin"):
            shutil.copy(os.path.join(tmp, f), os.path.join(H2FILE_DIR, f))
    rng = np.random.default_rng(98)
    x = rng.random(R.N) - 0.5
    X = rng.standard_normal((R.N, 4))
    np.savez_compressed(os.path.join(H2FILE_DIR, "io.npz"), x=x, y_ref=R.matvec(x), X=X, Y_ref=R.matmul(X),
                        coord_in=coord)
    print("h2file_coulomb", R.info["n_node"], sum(os.path.getsize(os.path.join(H2FILE_DIR, f)) for f in
                                                 os.listdir(H2FILE_DIR)) // 1024, "KiB")
    R.close()


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
    if len(sys.argv) > 1 and sys.argv[1] == "h2file":
        make_h2file()
    else:
        main()
        make_h2file()
