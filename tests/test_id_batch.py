"""Interpolative decompositions of the construction on the GPU against H2Pack's own QR.

``h2gpu_id_batch`` decomposes a batch of kernel matrices K(candidates, proxy points)^T
by a column-pivoted Householder QR (one CTA per block; one large block, or a block
whose work space does not fit one CTA's shared memory, over the whole GPU).
``h2gpu_pp_sketch_id`` decomposes the proxy-point sketch K(X0, Y0) S.  Both must choose
what H2Pack's H2P_partial_pivot_QR (src/H2Pack_ID_compress.c:51-189) chooses on the same
matrix: the same rank and pivot order, and E = R11^-1 R12 (src/H2Pack_ID_compress.c:
540-560) to FP64 rounding.  The reference QR runs from the library compiled from
H2Pack's sources.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import KERNEL_PARAMS
from h2pack_b200 import _abi

from oracle import oracle

# E entries: FP64 back substitutions of a pivoted R11 (condition ~ 1 / reltol)
E_TOL = 1e-7


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _param(kernel):
    p = np.zeros(4)
    par = KERNEL_PARAMS[kernel]
    p[:len(par)] = par
    return p, len(par)


def _shell(rng, n, r0, r1):
    d = rng.standard_normal((3, n))
    d /= np.linalg.norm(d, axis=0)
    return d * rng.uniform(r0, r1, n)


def _gpu_id_batch(kernel, blocks, prox, reltol):
    lib = _abi.libh2gpu()
    p, n_p = _param(kernel)
    nc = np.array([b.shape[1] for b in blocks], dtype=np.int32)
    cand = np.concatenate([b.reshape(-1) for b in blocks]) if blocks else np.zeros(1)
    cand = np.ascontiguousarray(cand, dtype=np.float64)
    prox = np.ascontiguousarray(prox, dtype=np.float64)
    rank = np.zeros(len(blocks), dtype=np.int32)
    perm = np.zeros(max(int(nc.sum()), 1), dtype=np.int32)
    E = C.POINTER(C.c_double)()
    e_off = (C.c_longlong * (len(blocks) + 1))()
    st = lib.h2gpu_id_batch(_abi.KERNEL_IDS[kernel], _dp(p), n_p, reltol, len(blocks), _ip(nc), prox.shape[1],
                            _dp(cand), _dp(prox), _ip(rank), _ip(perm), C.byref(E), e_off)
    assert st == 0, lib.h2gpu_last_error()
    out, o = [], 0
    for b, n in enumerate(nc):
        r = int(rank[b])
        ne = int(e_off[b + 1] - e_off[b])
        assert ne == r * (n - r)
        Eb = np.ctypeslib.as_array(E, shape=(max(int(e_off[len(blocks)]), 1),))[e_off[b]:e_off[b] + ne].copy()
        out.append((r, perm[o:o + n].copy(), Eb.reshape(n - r, r).T if ne else np.zeros((r, n - r))))
        o += n
    lib.h2gpu_free(E)
    return out


def _check_block(kernel, cand, prox, reltol, got):
    K = oracle.kernel_eval(_abi.KERNEL_IDS[kernel], KERNEL_PARAMS[kernel], cand, prox)   # ncand x npp
    R, perm_ref, r_ref = oracle.ref_pivot_qr(K, reltol, n_thread=os.cpu_count() or 1)
    r, perm, E = got
    assert r == r_ref, (r, r_ref)
    assert np.array_equal(perm, perm_ref)
    E_ref = oracle.ref_interp(R, r_ref)
    if E_ref.size:
        assert np.abs(E - E_ref).max() <= E_TOL * max(1.0, np.abs(E_ref).max()), np.abs(E - E_ref).max()


def test_reference_qr_gives_an_interpolative_decomposition():
    """The oracle wrapper of H2Pack's QR (CPU): the non-skeleton columns are E times the
    skeleton ones to the tolerance, R11 is upper triangular."""
    rng = np.random.default_rng(10)
    cand, prox = rng.uniform(-0.5, 0.5, (3, 300)), _shell(rng, 400, 1.5, 2.5)
    K = oracle.kernel_eval(_abi.KRNL_GAUSSIAN, [1.0], cand, prox)   # column j of K^T = candidate j
    R, perm, r = oracle.ref_pivot_qr(K, 1e-8)
    assert 0 < r < 300 and sorted(perm.tolist()) == list(range(300))
    E = oracle.ref_interp(R, r)
    At = K.T
    err = np.linalg.norm(At[:, perm[r:]] - At[:, perm[:r]] @ E) / np.linalg.norm(At)
    assert err < 1e-7, err
    assert np.allclose(np.tril(R.T[:r, :r], -1), 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["coulomb", "gaussian", "matern32"])
def test_id_batch_matches_h2pack_qr(kernel):
    """A level-like batch: small blocks (one CTA each), an empty block, and one block of
    1.2M entries (decomposed alone over the whole GPU)."""
    rng = np.random.default_rng(11)
    prox = _shell(rng, 1000, 1.5, 2.5)
    blocks = [rng.uniform(-0.5, 0.5, (3, n)) for n in (80, 200, 0, 150, 1200)]
    reltol = 1e-6
    got = _gpu_id_batch(kernel, blocks, prox, reltol)
    for b, g in zip(blocks, got):
        if b.shape[1]:
            _check_block(kernel, b, prox, reltol, g)
        else:
            assert g[0] == 0


@pytest.mark.gpu
def test_id_batch_wide_block_beyond_shared_memory():
    """20,000 candidates x 60 proxy points: the QR work space exceeds one CTA's shared
    memory, so the block goes to the grid-wide QR."""
    rng = np.random.default_rng(12)
    prox = _shell(rng, 60, 1.5, 2.5)
    blocks = [rng.uniform(-0.5, 0.5, (3, 100)), rng.uniform(-0.5, 0.5, (3, 20000))]
    got = _gpu_id_batch("gaussian", blocks, prox, 1e-8)
    for b, g in zip(blocks, got):
        _check_block("gaussian", b, prox, 1e-8, g)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["gaussian", "matern32"])
def test_pp_sketch_id_matches_h2pack_qr(kernel):
    """The proxy-point sketch W = K(X0, Y0) S (S sparse, given as S^T in CSR) and the
    decomposition of its rows: H2Pack's rank and pivots."""
    rng = np.random.default_rng(13)
    nx, ny, nnz_row = 1000, 2000, 32
    X0 = rng.uniform(-0.5, 0.5, (3, nx))
    Y0 = _shell(rng, ny, 1.5, 2.5)
    rowptr = np.arange(0, (nx + 1) * nnz_row, nnz_row, dtype=np.int32)
    col = np.concatenate([rng.choice(ny, nnz_row, replace=False) for _ in range(nx)]).astype(np.int32)
    val = rng.choice([-1.0, 1.0], nx * nnz_row)
    reltol = 1e-8
    lib = _abi.libh2gpu()
    p, n_p = _param(kernel)
    rank = np.zeros(1, dtype=np.int32)
    perm = np.zeros(nx, dtype=np.int32)
    Xc, Yc = np.ascontiguousarray(X0), np.ascontiguousarray(Y0)
    st = lib.h2gpu_pp_sketch_id(_abi.KERNEL_IDS[kernel], _dp(p), n_p, reltol, nx, _dp(Xc), ny, _dp(Yc), _ip(rowptr),
                                _ip(col), _dp(val), _ip(rank), _ip(perm))
    assert st == 0, lib.h2gpu_last_error()
    K = oracle.kernel_eval(_abi.KERNEL_IDS[kernel], KERNEL_PARAMS[kernel], X0, Y0)   # nx x ny
    S = np.zeros((ny, nx))
    for c in range(nx):
        S[col[rowptr[c]:rowptr[c + 1]], c] = val[rowptr[c]:rowptr[c + 1]]
    W = K @ S
    R, perm_ref, r_ref = oracle.ref_pivot_qr(W, reltol, n_thread=os.cpu_count() or 1)
    r = int(rank[0])
    assert r == r_ref
    assert sorted(perm.tolist()) == list(range(nx))
    if not np.array_equal(perm, perm_ref):
        # Late pivots can swap where two downdated column norms tie to rounding: the
        # downdate cn^2 - c0^2 loses digits as (|R_00| / |R_ii|)^2, and H2Pack's own QR
        # on this Matern sketch with one ulp of noise on the input diverges at step 181
        # of 345 (|R_ii| / |R_00| = 1.3e-6).  So: the same pivots while
        # |R_ii| >= 1e-5 |R_00|, and rows that approximate the sketch as well as H2Pack's.
        d = int(np.argmax(perm != perm_ref))
        dg = np.abs(np.diag(R.T[:r_ref, :r_ref]))
        assert dg[d] < 1e-5 * dg[0], (d, r, dg[d] / dg[0])

        def id_residual(skel):
            At = W.T
            B = At[:, skel]
            X, *_ = np.linalg.lstsq(B, At, rcond=None)
            return np.linalg.norm(At - B @ X) / np.linalg.norm(At)

        e_gpu, e_ref = id_residual(perm[:r]), id_residual(perm_ref[:r])
        assert e_gpu <= 2.0 * e_ref + 1e-15, (d, r, e_gpu, e_ref)
