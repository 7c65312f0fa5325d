"""Host-side API of the B200 H2 apply engine.

Two layers, mirroring how H2Pack is used:

* :class:`H2Matrix` -- an H2 representation built by H2Pack's own construction
  (``H2P_init -> H2P_partition_points -> proxy points -> H2P_build``, through
  ``libH2Pack_gpu.so``) and applied with H2Pack's entry points ``H2P_matvec`` /
  ``H2P_matmul``, which in that library run on the GPU.  This is the drop-in:
  the calls and their argument meaning are H2Pack's (src/H2Pack_matvec.h:17,
  src/H2Pack_matmul.h:25-28), with host arrays in the caller's point order.
* :class:`Image` -- the engine's C ABI (include/h2gpu.h) on a plain-pointer
  descriptor, including the device-resident apply on torch CUDA tensors.

There is no CPU fallback: every apply goes through ``libh2gpu.so``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi

_dp = C.POINTER(C.c_double)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _stream_arg(stream=None):
    """cudaStream_t for the C ABI: the given torch stream, else torch's current stream.
    torch's default stream has handle 0, which the ABI reads as "the image's own stream";
    it is passed as cudaStreamLegacy so that work is ordered with torch's default stream."""
    import torch
    h = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    return C.c_void_p(h if h else 0x1)


def _kernel_id(kernel) -> int:
    return _abi.KERNEL_IDS[kernel] if isinstance(kernel, str) else int(kernel)


def _prec(p) -> int:
    if isinstance(p, str):
        return {"fp64": _abi.PREC_FP64, "mixed": _abi.PREC_MIXED}[p]
    return int(p)


class Image:
    """Device image of one H2 representation (h2gpu_image_create)."""

    def __init__(self, desc: _abi.Desc, precision="fp64", max_n_vec: int = 64, device: int = -1,
                 blocks: str = "given"):
        """blocks: "given" (stored blocks uploaded from the descriptor, or evaluated on the
        fly for a JIT descriptor) or "generate" (stored B / D blocks generated on the
        device from the kernel and the points, as H2P_build_B_AOT / H2P_build_D_AOT do)."""
        self.lib = _abi.libh2gpu()
        opt = _abi.Options(_prec(precision), int(max_n_vec), int(device),
                           {"given": _abi.BLOCKS_GIVEN, "generate": _abi.BLOCKS_GENERATE}[blocks])
        h = C.c_void_p()
        _abi.check(self.lib.h2gpu_image_create(C.byref(desc), C.byref(opt), C.byref(h)), self.lib, "h2gpu_image_create")
        self.handle = h
        self.N = int(desc.krnl_dim) * int(desc.n_point)

    @classmethod
    def batch(cls, descs, precision="fp64", max_n_vec: int = 64, device: int = -1) -> "Image":
        """One image for many representations (h2gpu_batch_create); vectors are stacked in order."""
        lib = _abi.libh2gpu()
        arr = (_abi.Desc * len(descs))(*descs)
        opt = _abi.Options(_prec(precision), int(max_n_vec), int(device), _abi.BLOCKS_GIVEN)
        h = C.c_void_p()
        _abi.check(lib.h2gpu_batch_create(arr, len(descs), C.byref(opt), C.byref(h)), lib, "h2gpu_batch_create")
        img = cls.__new__(cls)
        img.lib = lib
        img.handle = h
        img.N = sum(int(d.krnl_dim) * int(d.n_point) for d in descs)
        img.sizes = [int(d.krnl_dim) * int(d.n_point) for d in descs]
        return img

    def set_precision(self, precision):
        _abi.check(self.lib.h2gpu_set_precision(self.handle, _prec(precision)), self.lib, "h2gpu_set_precision")

    def graph_capture(self, X, Y):
        """Capture the device apply X -> Y (torch CUDA float64, row-major) in a CUDA graph."""
        st = self.lib.h2gpu_graph_capture(self.handle, X.shape[1], C.c_void_p(X.data_ptr()), X.stride(0),
                                          C.c_void_p(Y.data_ptr()), Y.stride(0))
        _abi.check(st, self.lib, "h2gpu_graph_capture")

    def graph_launch(self, stream=None):
        s = _stream_arg(stream)
        _abi.check(self.lib.h2gpu_graph_launch(self.handle, s), self.lib, "h2gpu_graph_launch")

    def set_jit_variant(self, variant: str):
        """FP32 kernel variant: "simt", "tc" (default) or "pair" (JIT images), "tcgen05"
        (stored-block images)."""
        code = {"simt": _abi.JIT_SIMT, "tc": _abi.JIT_TC, "pair": _abi.JIT_PAIR, "tcgen05": _abi.BLK_TCGEN05}[variant]
        _abi.check(self.lib.h2gpu_set_jit_variant(self.handle, code), self.lib, "h2gpu_set_jit_variant")

    def autotune(self, X, Y):
        """Pick the panel width and JIT kernel variant that apply X fastest; returns
        (nv, variant) with variant one of "simt", "tc", "pair"."""
        nv, var = C.c_int(), C.c_int()
        st = self.lib.h2gpu_autotune(self.handle, X.shape[1], C.c_void_p(X.data_ptr()), X.stride(0),
                                     C.c_void_p(Y.data_ptr()), Y.stride(0), C.byref(nv), C.byref(var))
        _abi.check(st, self.lib, "h2gpu_autotune")
        return nv.value, ("simt", "tc", "pair", "tcgen05")[var.value]

    def matvec(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.N)
        _abi.check(self.lib.h2gpu_matvec(self.handle, _dptr(x), _dptr(y)), self.lib, "h2gpu_matvec")
        return y

    def matmul(self, X: np.ndarray, layout: int = _abi.ROW_MAJOR) -> np.ndarray:
        """Y = A X for X of shape (N, n_vec); layout picks the storage handed to the ABI."""
        N, nv = X.shape
        if layout == _abi.ROW_MAJOR:
            Xc = np.ascontiguousarray(X, dtype=np.float64)
            Y = np.empty((N, nv))
            st = self.lib.h2gpu_matmul(self.handle, layout, nv, _dptr(Xc), nv, _dptr(Y), nv)
            res = Y
        else:
            Xc = np.ascontiguousarray(X.T, dtype=np.float64)
            Y = np.empty((nv, N))
            st = self.lib.h2gpu_matmul(self.handle, layout, nv, _dptr(Xc), N, _dptr(Y), N)
            res = Y.T
        _abi.check(st, self.lib, "h2gpu_matmul")
        return res

    def matmul_device(self, X, Y=None, stream=None):
        """Device-resident apply on torch CUDA tensors of shape (N, n_vec), float64, row-major."""
        import torch
        assert X.is_cuda and X.dtype == torch.float64 and X.dim() == 2 and X.stride(1) == 1
        if Y is None:
            Y = torch.empty_like(X)
        s = _stream_arg(stream)
        st = self.lib.h2gpu_matmul_device(self.handle, X.shape[1], C.c_void_p(X.data_ptr()), X.stride(0),
                                          C.c_void_p(Y.data_ptr()), Y.stride(0), s)
        _abi.check(st, self.lib, "h2gpu_matmul_device")
        return Y

    def matvec_device_noalloc(self, x, y, stream=None):
        """y = A x on torch CUDA float64 vectors of length N, with no device allocation
        (h2gpu_matvec_device_noalloc: work buffers in the library's fixed device array)."""
        import torch
        assert x.is_cuda and y.is_cuda and x.dtype == torch.float64 and y.dtype == torch.float64
        assert x.numel() == self.N and y.numel() == self.N and x.is_contiguous() and y.is_contiguous()
        s = _stream_arg(stream)
        st = self.lib.h2gpu_matvec_device_noalloc(self.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), s)
        _abi.check(st, self.lib, "h2gpu_matvec_device_noalloc")
        return y

    def permute(self, x: np.ndarray, forward: bool = True) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        _abi.check(self.lib.h2gpu_permute_vector(self.handle, 1 if forward else 0, _dptr(x), _dptr(y)),
                   self.lib, "h2gpu_permute_vector")
        return y

    def blocks(self, which: str, n_elems: int) -> np.ndarray:
        """The image's stored B or D blocks (which = "B" / "D") in H2Pack's packing, as FP64."""
        out = np.empty(int(n_elems))
        _abi.check(self.lib.h2gpu_get_blocks(self.handle, 0 if which == "B" else 1, _dptr(out), out.size),
                   self.lib, "h2gpu_get_blocks")
        return out

    def stats(self) -> dict:
        s = _abi.Stats()
        _abi.check(self.lib.h2gpu_get_stats(self.handle, C.byref(s)), self.lib, "h2gpu_get_stats")
        out = {k: getattr(s, k) for k, _ in _abi.Stats._fields_}
        out["ms_phase"] = list(s.ms_phase)
        return out

    def reset_stats(self):
        self.lib.h2gpu_reset_stats(self.handle)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.h2gpu_image_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


PLAN_COUNT_NAMES = ("up_tasks", "down_tasks", "block_tasks", "jit_targets", "source_tiles", "panel_groups",
                    "partial_rows", "jit_point_pairs")


def plan_check(descs) -> dict:
    """Host-only self-check of the apply plan (h2gpu_plan_check; no GPU needed) of one
    descriptor, or of the merged representation of a list of them
    (h2gpu_batch_plan_check).  Returns the plan's sizes; raises RuntimeError naming the
    first violated invariant."""
    lib = _abi.libh2gpu()
    cnt = (C.c_longlong * len(PLAN_COUNT_NAMES))()
    if isinstance(descs, (list, tuple)):
        arr = (_abi.Desc * len(descs))(*descs)
        _abi.check(lib.h2gpu_batch_plan_check(arr, len(descs), cnt), lib, "h2gpu_batch_plan_check")
    else:
        _abi.check(lib.h2gpu_plan_check(C.byref(descs), cnt), lib, "h2gpu_plan_check")
    return dict(zip(PLAN_COUNT_NAMES, list(cnt)))


def direct_sum(kernel, param, src_coord, src_val, trg_coord) -> np.ndarray:
    """FP64 direct sum on the GPU: y_t = sum_s K(x_t, x_s) v_s (examples/direct_nbody.h)."""
    lib = _abi.libh2gpu()
    kid = _kernel_id(kernel)
    kd = 3 if kid == _abi.KRNL_RPY else 1
    src = np.ascontiguousarray(src_coord, dtype=np.float64)
    trg = np.ascontiguousarray(trg_coord, dtype=np.float64)
    val = np.ascontiguousarray(src_val, dtype=np.float64)
    p = np.zeros(4)
    p[:len(param)] = param
    out = np.empty(trg.shape[1] * kd)
    st = lib.h2gpu_direct_sum(kid, _dptr(p), len(param), src.shape[0], kd, _dptr(src), src.shape[1], _dptr(val),
                              _dptr(trg), trg.shape[1], _dptr(out))
    _abi.check(st, lib, "h2gpu_direct_sum")
    return out


def kernel_of(lib, h2pack):
    """Kernel of an H2Pack handle as the drop-in identifies it from the handle's kernel
    function and parameter (H2P_gpu_kernel_of): (name, parameters)."""
    kid, n = C.c_int(), C.c_int()
    p = np.zeros(4)
    st = lib.H2P_gpu_kernel_of(C.c_void_p(h2pack) if isinstance(h2pack, int) else h2pack, C.byref(kid), _dptr(p),
                               C.byref(n))
    if st != 0:
        m = lib.H2P_gpu_last_error()
        raise RuntimeError(f"H2P_gpu_kernel_of failed with status {st}: {m.decode() if m else ''}")
    names = {v: k for k, v in _abi.KERNEL_IDS.items()}
    return names[kid.value], list(p[:n.value])


class H2Matrix:
    """An H2 matrix built by H2Pack's construction and applied by the GPU drop-in.

    ``proxy`` selects the proxy points: ``"id"`` numerical (H2P_generate_proxy_point_ID_file,
    cached in ``pp_fname``) or ``"surface"`` (H2P_generate_proxy_point_surface).
    """

    def __init__(self, kernel, coord: np.ndarray, param=(), reltol: float = 1e-6, BD_JIT: int = 0,
                 max_leaf_points: int = 0, max_leaf_size: float = 0.0, proxy: str = "surface",
                 pp_fname: str | None = None, precision="fp64", n_thread: int = 0, hss: bool = False,
                 build_uj_gpu: bool = False, build_pp_gpu: bool = False):
        self.lib = _abi.libh2pack_gpu()
        self.kernel_id = _kernel_id(kernel)
        self.param = np.zeros(4)
        self.param[:len(param)] = param
        self.n_param = len(param)
        self.coord = np.ascontiguousarray(coord, dtype=np.float64)
        n_point = self.coord.shape[1]
        # projection matrices U / J of the construction on the GPU (scalar kernels) or by
        # H2Pack's own CPU code
        self.lib.H2P_gpu_build_uj(1 if build_uj_gpu else 0)
        self.lib.H2P_gpu_build_pp(1 if build_pp_gpu else 0)
        h = self.lib.h2pb_build(self.kernel_id, _dptr(self.param), self.n_param, n_point, _dptr(self.coord),
                                float(reltol), int(max_leaf_points), float(max_leaf_size), int(BD_JIT),
                                0 if proxy == "id" else 1, pp_fname.encode() if pp_fname else None, 1, int(n_thread),
                                1 if hss else 0)
        if not h:
            raise RuntimeError("H2Pack construction (h2pb_build) failed")
        self.handle = h
        self._hss = bool(hss)
        self.h2pack = self.lib.h2pb_h2pack(h)
        info = (C.c_longlong * 16)()
        self.lib.h2pb_info(self.h2pack, info)
        self.info = dict(zip(["n_point", "krnl_dim", "xpt_dim", "n_node", "n_leaf_node", "max_level",
                              "min_adm_level", "n_r_adm_pair", "n_r_inadm_pair", "n_B", "n_D", "BD_JIT",
                              "krnl_mat_size", "max_leaf_points", "n_thread", "mm_max_n_vec"], list(info)))
        self.N = self.info["krnl_mat_size"]
        self.build_seconds = self.lib.h2pb_build_seconds(h)
        # JIT handles: the drop-in identifies the kernel from the handle's own kernel
        # function and parameter, as it does for any H2Pack program
        self.set_precision(precision)

    def _check(self, st, what):
        if st != 0:
            m = self.lib.H2P_gpu_last_error()
            raise RuntimeError(f"{what} failed with status {st}: {m.decode() if m else ''}")

    def set_precision(self, precision):
        self._check(self.lib.H2P_gpu_set_precision(self.h2pack, _prec(precision)), "H2P_gpu_set_precision")

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """y = A x through H2Pack's H2P_matvec signature (status-returning form)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.N)
        self._check(self.lib.H2P_gpu_matvec(self.h2pack, _dptr(x), _dptr(y)), "H2P_matvec")
        return y

    def matmul(self, X: np.ndarray, layout: int = _abi.ROW_MAJOR) -> np.ndarray:
        N, nv = X.shape
        if layout == _abi.ROW_MAJOR:
            Xc = np.ascontiguousarray(X, dtype=np.float64)
            Y = np.empty((N, nv))
            st = self.lib.H2P_gpu_matmul(self.h2pack, layout, nv, _dptr(Xc), nv, _dptr(Y), nv)
            res = Y
        else:
            Xc = np.ascontiguousarray(X.T, dtype=np.float64)
            Y = np.empty((nv, N))
            st = self.lib.H2P_gpu_matmul(self.h2pack, layout, nv, _dptr(Xc), N, _dptr(Y), N)
            res = Y.T
        self._check(st, "H2P_matmul")
        return res

    def matmul_raw(self, layout: int, n_vec: int, X_ptr: int, ldx: int, Y_ptr: int, ldy: int):
        """H2P_matmul on caller-owned host memory (e.g. pinned torch tensors)."""
        st = self.lib.H2P_gpu_matmul(self.h2pack, layout, n_vec, C.cast(X_ptr, _dp), ldx, C.cast(Y_ptr, _dp), ldy)
        self._check(st, "H2P_matmul")

    def ulv_factorize(self, shift: float = 0.0, lu: bool = False):
        """H2Pack's own ULV factorization of an HSS-mode matrix (plus shift on the
        diagonal): H2P_HSS_ULV_Cholesky_factorize, or H2P_HSS_ULV_LU_factorize with lu
        (src/H2Pack_HSS_ULV.c:601, :16).  Runs on the host; the solves run on the GPU."""
        if not self._hss:
            raise RuntimeError("the ULV factorization needs a matrix built with hss=True")
        fn = self.lib.H2P_HSS_ULV_LU_factorize if lu else self.lib.H2P_HSS_ULV_Cholesky_factorize
        _abi.blas_one_thread(self.lib)
        fn(self.h2pack, float(shift))
        self._ulv_lu = bool(lu)

    def ulv_solve(self, b: np.ndarray, op: int = 3) -> np.ndarray:
        """x = the ULV solve of b on the GPU (H2P_HSS_ULV_Cholesky_solve / _LU_solve,
        op 1, 2 or 3 as H2Pack's)."""
        if not hasattr(self, "_ulv_lu"):
            raise RuntimeError("call ulv_factorize first")
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty(self.N)
        self._check(self.lib.H2P_gpu_ULV_solve(self.h2pack, int(self._ulv_lu), int(op), _dptr(b), _dptr(x)),
                    "H2P_HSS_ULV_solve")
        return x

    def image(self) -> Image:
        """A non-owning Image view of the handle's device image."""
        ptr = self.lib.H2P_gpu_image(self.h2pack)
        if not ptr:
            self._check(-5, "H2P_gpu_image")
        img = Image.__new__(Image)
        img.lib = _abi.libh2gpu()
        img.handle = None          # not owned: released with the H2Matrix
        img._view = C.c_void_p(ptr)
        img.N = self.N
        return _ImageView(img._view, self.N)

    def kernel_of(self):
        """The kernel the drop-in sees in this handle (H2P_gpu_kernel_of): (name, param list)."""
        return kernel_of(self.lib, self.h2pack)

    def describe(self) -> _abi.Desc:
        d = _abi.Desc()
        self._check(self.lib.h2pb_describe(self.handle, C.byref(d)), "h2pb_describe")
        return d

    def plan_check(self) -> dict:
        """The host-only plan self-check of this matrix's representation (no GPU needed)."""
        return plan_check(self.describe())

    def sorted_coord(self) -> np.ndarray:
        xd = self.info["xpt_dim"]
        p = self.lib.h2pb_coord(self.h2pack)
        return np.ctypeslib.as_array(p, shape=(xd * self.info["n_point"],)).reshape(xd, -1).copy()

    def counters(self) -> dict:
        ms = (C.c_double * 11)()
        tm = (C.c_double * 11)()
        jf = (C.c_double * 2)()
        nmv = C.c_longlong()
        self.lib.h2pb_counters(self.h2pack, ms, tm, jf, C.byref(nmv))
        return {"mat_size": list(ms), "timers": list(tm), "JIT_flops": list(jf), "n_matvec": nmv.value}

    def close(self):
        if getattr(self, "handle", None):
            self.lib.H2P_gpu_release(self.h2pack)
            self.lib.h2pb_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _ImageView(Image):
    """Image methods on an image owned by someone else (the drop-in registry)."""

    def __init__(self, handle, N):  # noqa: D401 - thin view
        self.lib = _abi.libh2gpu()
        self.handle = handle
        self.N = N

    def close(self):
        self.handle = None
