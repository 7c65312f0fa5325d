"""ctypes mirror of include/h2gpu.h and loaders for the package's shared libraries.

The engine is the C ABI in ``lib/libh2gpu.so`` (CUDA, sm_100a).  The drop-in
``lib/libH2Pack_gpu.so`` is H2Pack's own construction code linked with the GPU
versions of ``H2P_matvec`` / ``H2P_matmul``.  Loading fails loudly when a library
is missing: there is no CPU fallback for the apply path.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "lib")
LIBH2GPU = os.path.join(LIB_DIR, "libh2gpu.so")
LIBH2PACK_GPU = os.path.join(LIB_DIR, "libH2Pack_gpu.so")

H2GPU_OK = 0
BLOCKS_GIVEN, BLOCKS_GENERATE = 0, 1
STATUS_NAMES = {0: "OK", -1: "INVALID", -2: "UNSUPPORTED", -3: "CUDA", -4: "NOMEM", -5: "STATE", -6: "DEVICE"}

KRNL_COULOMB, KRNL_GAUSSIAN, KRNL_MATERN32, KRNL_RPY = 1, 2, 3, 4
KERNEL_IDS = {"coulomb": KRNL_COULOMB, "gaussian": KRNL_GAUSSIAN, "matern32": KRNL_MATERN32, "rpy": KRNL_RPY}
PREC_FP64, PREC_MIXED = 0, 1
JIT_SIMT, JIT_TC, JIT_PAIR, BLK_TCGEN05 = 0, 1, 2, 3
CG_FREE, CG_RUN, CG_CHECK, CG_DONE = 0, 1, 2, 3
CG_MATVEC, CG_PCG = 0, 1
ROW_MAJOR, COL_MAJOR = 101, 102

_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)
_szp = C.POINTER(C.c_size_t)
_dpp = C.POINTER(C.POINTER(C.c_double))


class Desc(C.Structure):
    """struct h2gpu_desc"""
    _fields_ = [
        ("n_point", C.c_int), ("pt_dim", C.c_int), ("xpt_dim", C.c_int), ("krnl_dim", C.c_int),
        ("n_node", C.c_int), ("n_leaf_node", C.c_int), ("max_child", C.c_int), ("max_level", C.c_int),
        ("min_adm_level", C.c_int), ("BD_JIT", C.c_int),
        ("n_child", _ip), ("children", _ip), ("node_level", _ip), ("pt_cluster", _ip),
        ("mat_cluster", _ip), ("level_n_node", _ip), ("level_nodes", _ip), ("leaf_nodes", _ip),
        ("U_nrow", _ip), ("U_ncol", _ip), ("U_ld", _ip), ("U", _dpp),
        ("n_r_adm_pair", C.c_int), ("r_adm_pairs", _ip),
        ("n_r_inadm_pair", C.c_int), ("r_inadm_pairs", _ip),
        ("n_B", C.c_int), ("B_nrow", _ip), ("B_ncol", _ip), ("B_ptr", _szp), ("B_data", _dp),
        ("n_D", C.c_int), ("D_nrow", _ip), ("D_ncol", _ip), ("D_ptr", _szp), ("D_data", _dp),
        ("coord", _dp), ("J_n", _ip), ("J_coord", _dpp),
        ("fwd_pmt_idx", _ip), ("bwd_pmt_idx", _ip),
        ("kernel_id", C.c_int), ("n_krnl_param", C.c_int), ("krnl_param", C.c_double * 4),
    ]


class Options(C.Structure):
    """struct h2gpu_options"""
    _fields_ = [("precision", C.c_int), ("max_n_vec", C.c_int), ("device", C.c_int), ("blocks", C.c_int)]


class Stats(C.Structure):
    """struct h2gpu_stats"""
    _fields_ = [
        ("n_matvec", C.c_longlong), ("ms_total", C.c_double), ("ms_phase", C.c_double * 5),
        ("bytes_U", C.c_double), ("bytes_B", C.c_double), ("bytes_D", C.c_double),
        ("ref_mv_bytes", C.c_double), ("jit_pairs_B", C.c_double), ("jit_pairs_D", C.c_double),
        ("n_tasks_B", C.c_longlong), ("n_tasks_D", C.c_longlong), ("device_bytes", C.c_longlong),
        ("n_launches", C.c_longlong),
    ]


_pp_i = C.POINTER(C.POINTER(C.c_int))
_pp_d = C.POINTER(C.POINTER(C.c_double))


class UlvDesc(C.Structure):
    """struct h2gpu_ulv_desc"""
    _fields_ = [
        ("lu", C.c_int), ("n_node", C.c_int), ("max_level", C.c_int), ("n_leaf_node", C.c_int),
        ("krnl_mat_size", C.c_int), ("level_n_node", _ip), ("level_nodes", _ip), ("fwd_pmt_idx", _ip),
        ("bwd_pmt_idx", _ip), ("Ls", _ip), ("m", _ip), ("q_ncol", _ip), ("l_ld", _ip), ("idx", _pp_i),
        ("Q", _pp_d), ("L", _pp_d), ("p", _pp_i), ("device", C.c_int),
    ]


# Every symbol include/h2gpu.h declares, with its ctypes signature.
H2GPU_SYMBOLS = {
    "h2gpu_abi_version": (C.c_int, []),
    "h2gpu_last_error": (C.c_char_p, []),
    "h2gpu_default_options": (None, [C.POINTER(Options)]),
    "h2gpu_image_create": (C.c_int, [C.POINTER(Desc), C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "h2gpu_image_destroy": (C.c_int, [C.c_void_p]),
    "h2gpu_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "h2gpu_matvec": (C.c_int, [C.c_void_p, _dp, _dp]),
    "h2gpu_matmul": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int]),
    "h2gpu_matmul_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "h2gpu_permute_vector": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp]),
    "h2gpu_permute_matrix_rows": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int]),
    "h2gpu_matvec_device_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "h2gpu_set_jit_variant": (C.c_int, [C.c_void_p, C.c_int]),
    "h2gpu_cg_create": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.POINTER(C.c_void_p)]),
    "h2gpu_cg_destroy": (C.c_int, [C.c_void_p]),
    "h2gpu_cg_admit": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_double, C.c_int]),
    "h2gpu_cg_step": (C.c_int, [C.c_void_p, C.c_int]),
    "h2gpu_cg_check": (C.c_int, [C.c_void_p]),
    "h2gpu_cg_sync": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp]),
    "h2gpu_cg_query": (C.c_int, [C.c_void_p]),
    "h2gpu_cg_cancel": (C.c_int, [C.c_void_p, C.c_int]),
    "h2gpu_cg_take": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "h2gpu_cg_history": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int]),
    "h2gpu_batch_create": (C.c_int, [C.POINTER(Desc), C.c_int, C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "h2gpu_graph_capture": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "h2gpu_graph_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "h2gpu_autotune": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                 C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "h2gpu_get_blocks": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_size_t]),
    "h2gpu_get_stats": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "h2gpu_reset_stats": (C.c_int, [C.c_void_p]),
    "h2gpu_image_bytes": (C.c_size_t, [C.c_void_p]),
    "h2gpu_plan_check": (C.c_int, [C.POINTER(Desc), C.POINTER(C.c_longlong)]),
    "h2gpu_batch_plan_check": (C.c_int, [C.POINTER(Desc), C.c_int, C.POINTER(C.c_longlong)]),
    "h2gpu_measure_peaks": (C.c_int, [C.c_int, _dp, _dp]),
    "h2gpu_direct_sum": (C.c_int, [C.c_int, _dp, C.c_int, C.c_int, C.c_int, _dp, C.c_int, _dp, _dp, C.c_int, _dp]),
    "h2gpu_id_batch": (C.c_int, [C.c_int, _dp, C.c_int, C.c_double, C.c_int, _ip, C.c_int, _dp, _dp, _ip, _ip,
                                 C.POINTER(_dp), C.POINTER(C.c_longlong)]),
    "h2gpu_free": (None, [C.c_void_p]),
    "h2gpu_pp_sketch_id": (C.c_int, [C.c_int, _dp, C.c_int, C.c_double, C.c_int, _dp, C.c_int, _dp, _ip, _ip, _dp,
                                     _ip, _ip]),
    "h2gpu_ulv_create": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "h2gpu_ulv_destroy": (C.c_int, [C.c_void_p]),
    "h2gpu_ulv_solve": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp]),
    "h2gpu_ulv_solve_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "h2gpu_ulv_bytes": (C.c_size_t, [C.c_void_p]),
}

# Entry points of the drop-in library (include/h2p_dropin.h) and of the construction driver.
H2PACK_GPU_SYMBOLS = {
    "H2P_matvec": (None, [C.c_void_p, _dp, _dp]),
    "H2P_matmul": (None, [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int]),
    "H2P_permute_vector_forward": (None, [C.c_void_p, _dp, _dp]),
    "H2P_permute_vector_backward": (None, [C.c_void_p, _dp, _dp]),
    "H2P_permute_matrix_row_forward": (None, [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int]),
    "H2P_permute_matrix_row_backward": (None, [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int]),
    "H2P_gpu_set_kernel": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_int]),
    "H2P_gpu_kernel_of": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), _dp, C.POINTER(C.c_int)]),
    "H2P_gpu_build_uj": (None, [C.c_int]),
    "H2P_gpu_build_uj_count": (C.c_int, []),
    "H2P_gpu_build_pp": (None, [C.c_int]),
    "H2P_gpu_build_pp_count": (C.c_int, []),
    "H2P_destroy": (None, [C.POINTER(C.c_void_p)]),
    "H2P_gpu_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "H2P_gpu_matvec": (C.c_int, [C.c_void_p, _dp, _dp]),
    "H2P_gpu_matmul": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_int]),
    "H2P_gpu_image": (C.c_void_p, [C.c_void_p]),
    "H2P_gpu_release": (C.c_int, [C.c_void_p]),
    "H2P_gpu_last_error": (C.c_char_p, []),
    "H2P_HSS_ULV_Cholesky_solve": (None, [C.c_void_p, C.c_int, _dp, _dp]),
    "H2P_HSS_ULV_LU_solve": (None, [C.c_void_p, C.c_int, _dp, _dp]),
    "H2P_gpu_ULV_solve": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, _dp]),
    "H2P_gpu_ULV_release": (C.c_int, [C.c_void_p]),
    # H2Pack's own ULV code inside the library: the factorizations, and its CPU solves
    # under their aliased names
    "H2P_HSS_ULV_Cholesky_factorize": (None, [C.c_void_p, C.c_double]),
    "H2P_HSS_ULV_LU_factorize": (None, [C.c_void_p, C.c_double]),
    "H2P_HSS_ULV_Cholesky_solve_host": (None, [C.c_void_p, C.c_int, _dp, _dp]),
    "H2P_HSS_ULV_LU_solve_host": (None, [C.c_void_p, C.c_int, _dp, _dp]),
}

BUILDER_SYMBOLS = {
    "h2pb_build": (C.c_void_p, [C.c_int, _dp, C.c_int, C.c_int, _dp, C.c_double, C.c_int, C.c_double,
                                C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_int]),
    "h2pb_h2pack": (C.c_void_p, [C.c_void_p]),
    "h2pb_build_seconds": (C.c_double, [C.c_void_p]),
    "h2pb_destroy": (None, [C.c_void_p]),
    "h2pb_info": (None, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "h2pb_counters": (None, [C.c_void_p, _dp, _dp, _dp, C.POINTER(C.c_longlong)]),
    "h2pb_reset_timers": (None, [C.c_void_p]),
    "h2pb_coord": (_dp, [C.c_void_p]),
    "h2pb_coord_idx": (_ip, [C.c_void_p]),
    "h2pb_describe": (C.c_int, [C.c_void_p, C.POINTER(Desc)]),
    "h2pb_describe_ulv": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "h2pb_free": (None, [C.c_void_p]),
}


def bind(lib: C.CDLL, table: dict) -> C.CDLL:
    for name, (res, args) in table.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_cache: dict = {}


def _load(path: str, tables) -> C.CDLL:
    if path in _cache:
        return _cache[path]
    if not os.path.exists(path):
        raise RuntimeError(
            f"{os.path.basename(path)} is not built ({path}); run __graft_entry__.build() "
            "or `make -C h2pack_b200`.  There is no CPU fallback for the H2 apply path.")
    lib = C.CDLL(path, mode=C.RTLD_LOCAL)
    for t in tables:
        bind(lib, t)
    _cache[path] = lib
    return lib


def libh2gpu() -> C.CDLL:
    """The CUDA engine (C ABI of include/h2gpu.h)."""
    return _load(LIBH2GPU, [H2GPU_SYMBOLS])


def libh2pack_gpu() -> C.CDLL:
    """H2Pack construction + GPU drop-in H2P_matvec/H2P_matmul (include/h2p_dropin.h)."""
    libh2gpu()  # resolve the engine first so the drop-in finds it
    return _load(LIBH2PACK_GPU, [H2PACK_GPU_SYMBOLS, BUILDER_SYMBOLS])


def blas_one_thread(lib: C.CDLL) -> None:
    """Pin the OpenBLAS that H2Pack's code in `lib` calls to one thread.  H2Pack's ULV
    factorizations and solves call BLAS / LAPACK from inside their OpenMP loops
    (src/H2Pack_HSS_ULV.c), and its construction leaves the BLAS at n_thread threads
    (src/H2Pack_build.c:269, :644); with a pthreads OpenBLAS, such nested calls from
    several OpenMP threads race.  One BLAS thread per OpenMP thread is how H2Pack's own
    construction loops call it."""
    f = getattr(lib, "openblas_set_num_threads", None)
    if f is not None:
        f.argtypes = [C.c_int]
        f.restype = None
        f(1)


def check(status: int, lib: C.CDLL | None = None, what: str = "") -> None:
    if status != H2GPU_OK:
        msg = ""
        try:
            lib = lib or libh2gpu()
            m = lib.h2gpu_last_error()
            msg = m.decode() if m else ""
        except Exception:  # pragma: no cover - message lookup only
            pass
        raise RuntimeError(f"{what} failed with status {status} ({STATUS_NAMES.get(status, '?')}): {msg}")
