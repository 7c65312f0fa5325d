"""The H2Pack drop-in under H2Pack's own programs and under concurrent callers (GPU).

* The reference's example drivers (examples/example_H2.c: Coulomb, JIT mode, N = 40,000,
  numerical proxy points; examples/example_H2_RPY.c: RPY, JIT mode, N = 20,000), compiled
  unchanged against the drop-in library by oracle/Makefile, run with "0" on stdin (do not
  store the matrix) and print their error against their own direct N-body sum; it must
  stay within the construction tolerance 1e-6 that the programs print beside it.
* H2Pack's own extra/test_HSS_scalar.c (HSS build, matvec, ULV LU factorization and
  solve) runs unchanged on the drop-in; its errors stay within the spread of its CPU build.
* examples/SPDHSS-H2/example_regularHSS.c (PCG on an H2 operator preconditioned by the
  HSS ULV solve) runs unchanged on the drop-in and converges as its CPU build does.
* Two handles applied from two host threads at once give the results they give alone.
* A handle whose arrays change in place (same addresses and sizes) is re-uploaded.
* H2P_destroy releases the handle's device image.
"""
import os
import re
import subprocess
import threading

import numpy as np
import pytest

from conftest import ROOT, make_points, rel
from oracle import oracle as O
from h2pack_b200 import _abi
from h2pack_b200.h2pack import H2Matrix

pytestmark = pytest.mark.gpu
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
# The HSS programs run H2Pack's ULV factorization, which calls BLAS / LAPACK inside
# OpenMP loops after H2P_build has set the BLAS to n_thread threads; with the pthreads
# OpenBLAS here those nested calls race.  One OpenMP thread (n_thread = 1) avoids the
# nesting; the GPU parts are unaffected.
_ONE_THREAD = {"OMP_NUM_THREADS": "1", "OPENBLAS_NUM_THREADS": "1"}


@pytest.mark.parametrize("program", ["example_H2_gpu", "example_H2_RPY_gpu"])
def test_reference_example_runs_unchanged_on_the_dropin(program, tmp_path):
    exe = os.path.join(REF_BIN, program)
    assert os.path.exists(exe), f"{exe} is built by oracle/Makefile (make -C oracle examples)"
    env = dict(os.environ, OMP_NUM_THREADS=str(min(os.cpu_count() or 8, 32)))
    r = subprocess.run([exe], input="0\n", capture_output=True, text=True, cwd=tmp_path, env=env, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    m = re.search(r"validation points: \|\|y_\{H2\} - y\|\|_2 / \|\|y\|\|_2 = ([0-9.eE+-]+)", r.stdout)
    t = re.search(r"relative error threshold is ([0-9.eE+-]+)", r.stdout)
    assert m and t, r.stdout[-2000:]
    err, tol = float(m.group(1)), float(t.group(1))
    print(f"{program}: error {err:.3e} (threshold {tol:.0e})")
    assert err <= tol


def test_reference_hss_test_program_runs_unchanged_on_the_dropin(tmp_path):
    """H2Pack's own extra/test_HSS_scalar.c (Gaussian kernel, N = 8,000, JIT mode): an
    HSS build, H2P_matvec against its direct N-body sum, then H2P_HSS_ULV_LU_factorize
    with shift 0 and H2P_HSS_ULV_LU_solve of A x0, compiled unchanged against the
    drop-in by oracle/Makefile, so that the apply and the ULV solve run on the GPU.  The
    program draws its points from the clock; the bounds cover the spread of its CPU
    build (oracle/_ref/test_HSS_scalar_cpu) over four runs at this size: HSS error
    1.3e-5 .. 8.5e-5, solve error 1.1e-11 .. 7.7e-11."""
    exe = os.path.join(REF_BIN, "test_HSS_scalar_gpu")
    assert os.path.exists(exe), f"{exe} is built by oracle/Makefile (make -C oracle examples)"
    env = dict(os.environ, **_ONE_THREAD)
    args = ["3", "8000", "1e-6", "1", "1", str(tmp_path / "pp_gaussian.dat")]
    r = subprocess.run([exe, *args], capture_output=True, text=True, cwd=tmp_path, env=env, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    m = re.search(r"validation points: \|\|y_\{HSS\} - y\|\|_2 / \|\|y\|\|_2 = ([0-9.eE+-]+)", r.stdout)
    u = re.search(r"H2P_HSS_ULV_LU_solve relerr = ([0-9.eE+-]+)", r.stdout)
    assert m and u, r.stdout[-2000:]
    err, solve_err = float(m.group(1)), float(u.group(1))
    print(f"test_HSS_scalar on the drop-in: HSS error {err:.3e}, ULV LU solve error {solve_err:.3e}")
    assert err < 1e-3
    assert solve_err < 1e-8


def test_reference_hss_preconditioned_pcg_runs_unchanged_on_the_dropin(tmp_path):
    """H2Pack's examples/SPDHSS-H2/example_regularHSS.c (Gaussian l = 0.1, shift 1,
    N = 8,000, JIT mode): an H2 matrix applied by H2P_matvec, a rank-100 HSS matrix,
    H2P_HSS_ULV_Cholesky_factorize, and PCG on the shifted H2 operator preconditioned by
    H2P_HSS_ULV_Cholesky_solve (pcg_tests.c:41-45), compiled unchanged against the
    drop-in: both the operator and the preconditioner run on the GPU.  Its CPU build
    (oracle/_ref/example_regularHSS_cpu) converged in 4 or 5 iterations to a relative
    residual of 2.5e-5 .. 6.6e-5 in four runs (points drawn from the clock)."""
    exe = os.path.join(REF_BIN, "example_regularHSS_gpu")
    assert os.path.exists(exe), f"{exe} is built by oracle/Makefile (make -C oracle examples)"
    env = dict(os.environ, **_ONE_THREAD)
    args = ["3", "8000", "1e-6", "1", "1", "random", "0.1", "1.0"]
    r = subprocess.run([exe, *args], capture_output=True, text=True, cwd=tmp_path, env=env, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    if "The constructed HSS matrix is non-SPD" in r.stdout:
        pytest.skip("this random point set gave a non-SPD rank-100 HSS matrix (the program skips PCG)")
    assert "The constructed HSS matrix is SPD" in r.stdout, r.stdout[-2000:]
    it = re.search(r"PCG: Converged in (\d+) iterations", r.stdout)
    rr = re.search(r"PCG stopped after \d+ iterations, relres = ([0-9.eE+-]+)", r.stdout)
    assert it and rr, r.stdout[-2000:]
    print(f"example_regularHSS on the drop-in: {it.group(1)} iterations, relres {rr.group(1)}")
    assert int(it.group(1)) <= 10
    assert float(rr.group(1)) < 1e-4


def test_two_handles_from_two_threads():
    Ha = H2Matrix("matern32", make_points("matern32", 20000, 21), [1.0], 1e-6, BD_JIT=1, max_leaf_points=200)
    Hb = H2Matrix("coulomb", make_points("coulomb", 15000, 22), [], 1e-6, BD_JIT=0, max_leaf_points=200)
    try:
        rng = np.random.default_rng(23)
        xa, xb = rng.standard_normal((Ha.N, 4)), rng.standard_normal(Hb.N)
        ya, yb = Ha.matmul(xa), Hb.matvec(xb)          # alone
        out, errs = {}, []

        def run(name, f):
            try:
                out[name] = [f() for _ in range(6)]
            except Exception as e:  # pragma: no cover - reported below
                errs.append(e)

        ts = [threading.Thread(target=run, args=("a", lambda: Ha.matmul(xa))),
              threading.Thread(target=run, args=("b", lambda: Hb.matvec(xb)))]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        assert not errs, errs
        assert all(np.array_equal(y, ya) for y in out["a"])
        assert all(np.array_equal(y, yb) for y in out["b"])
    finally:
        Ha.close()
        Hb.close()


def test_handle_changed_in_place_is_reuploaded():
    """The D blocks of a stored-block handle are scaled in place (same addresses and
    sizes): the next apply sees the new values."""
    R = O.RefH2("coulomb", [], make_points("coulomb", 4000, 24), 1e-6, BD_JIT=0, max_leaf_points=100)
    lib = _abi.libh2pack_gpu()
    try:
        x = np.random.default_rng(25).standard_normal(R.N)
        y0 = np.zeros(R.N)
        assert lib.H2P_gpu_matvec(R.h2pack, O.dptr(x), O.dptr(y0)) == 0
        d = R.describe()
        nD = int(d.D_ptr[d.n_D])
        D = np.ctypeslib.as_array(d.D_data, shape=(nD,))
        D *= 2.0
        y1 = np.zeros(R.N)
        assert lib.H2P_gpu_matvec(R.h2pack, O.dptr(x), O.dptr(y1)) == 0
        assert rel(y1, R.matvec(x)) < 1e-12           # the reference applies the changed blocks
        assert rel(y1, y0) > 1e-3
    finally:
        lib.H2P_gpu_release(R.h2pack)
        R.close()


def test_h2p_destroy_releases_the_device_image():
    import torch
    H = H2Matrix("coulomb", make_points("coulomb", 30000, 26), [], 1e-6, BD_JIT=0, max_leaf_points=200)
    H.matvec(np.ones(H.N))
    torch.cuda.synchronize()
    free_with = torch.cuda.mem_get_info()[0]
    img_bytes = H.lib.H2P_gpu_image(H.h2pack) and _abi.libh2gpu().h2gpu_image_bytes(H.lib.H2P_gpu_image(H.h2pack))
    assert img_bytes > 50 << 20
    # H2Pack's own destroy through the handle pointer, without H2P_gpu_release first
    H.lib.h2pb_destroy(H.handle)
    H.handle = None
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] >= free_with + img_bytes // 2
