"""ctypes binding of the in-tree shared library libfap_b200.so.

The library is the product: every solve runs there (sm_100a kernels behind
the C ABI of include/fap_b200.h and include/fap_host.h).  There is no Python
or CPU fallback -- if the library is missing or cannot be loaded, importing
the functions that need it raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfap_b200.so")

FAP_OK = 0
FAP_ERR_INVALID = -1
FAP_ERR_CUDA = -2
FAP_ERR_NOMEM = -3
FAP_ERR_STATE = -4
FAP_ERR_NOT_CONVERGED = -5
FAP_ERR_RANGE = -6
FAP_ERR_IO = -7
FAP_ERR_PARTITION = -8
FAP_ERR_DEVICE = -9

FAP_DTYPE_AUTO = -1
FAP_DTYPE_I32 = 0
FAP_DTYPE_F32 = 1
FAP_MODE_PLAIN = 0
FAP_MODE_BATCHED = 1
FAP_NOALLOC_FLOYD_MAX = 1024
FAP_INF_I32 = 100000000
FAP_INF_F32 = 1e8

_ERR_NAMES = {
    FAP_ERR_INVALID: "invalid argument", FAP_ERR_CUDA: "CUDA error", FAP_ERR_NOMEM: "out of memory",
    FAP_ERR_STATE: "bad call order", FAP_ERR_NOT_CONVERGED: "SSSP did not converge",
    FAP_ERR_RANGE: "weights out of int32 range", FAP_ERR_IO: "graph file error",
    FAP_ERR_PARTITION: "partition error", FAP_ERR_DEVICE: "device-side error",
}


class FapError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code} {_ERR_NAMES.get(code, 'error')}] {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()

P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64
INT = ctypes.c_int
DBL = ctypes.c_double
PP = ctypes.POINTER(ctypes.c_void_p)

# name: (restype, argtypes)
_SIGS = {
    "fap_last_error": (ctypes.c_char_p, []),
    "fap_version": (INT, []),
    "fap_ctx_create": (INT, [INT, PP]),
    "fap_ctx_destroy": (INT, [P]),
    "fap_ctx_set_stream": (INT, [P, P]),
    "fap_ctx_get_stream": (INT, [P, PP]),
    "fap_ctx_sync": (INT, [P]),
    "fap_graph_create": (INT, [P, I32, I64, P, P, P, INT, PP]),
    "fap_graph_destroy": (INT, [P]),
    "fap_graph_dtype": (INT, [P]),
    "fap_graph_set_parts": (INT, [P, I32, P, P, P, P, P]),
    "fap_graph_reserve": (INT, [P, I64]),
    "fap_solve": (INT, [P, P, I32, INT]),
    "fap_graph_check": (INT, [P]),
    "fap_graph_block": (INT, [P, I32, PP, ctypes.POINTER(I64), ctypes.POINTER(I64)]),
    "fap_graph_copy_block": (INT, [P, I32, P, INT]),
    "fap_graph_copy_block_async": (INT, [P, I32, P, INT, I32]),
    "fap_graph_copy_wait": (INT, [P, I32]),
    "fap_graph_block_checksums": (INT, [P, I32, P]),
    "fap_graph_path_block": (INT, [P, I32, PP, ctypes.POINTER(I64), ctypes.POINTER(I64)]),
    "fap_graph_copy_path_block": (INT, [P, I32, P]),
    "fap_graph_sssp_rows": (INT, [P, P, I32, P]),
    "fap_queue_order_check": (INT, [P, I32, INT]),
    "fap_graph_set_param": (INT, [P, ctypes.c_char_p, DBL]),
    "fap_graph_last_timing": (INT, [P, P]),
    "fap_graph_last_launches": (INT, [P, ctypes.POINTER(I64)]),
    "fap_graph_last_stage1": (INT, [P]),
    "fap_graph_stage1_name": (ctypes.c_char_p, [P]),
    "fap_op_sssp": (INT, [P, INT, I32, I64, P, P, P, P, I32, P, I64]),
    "fap_op_floyd": (INT, [P, INT, I32, P, I64]),
    "fap_op_minplus": (INT, [P, INT, I32, I32, I32, P, I64, P, I64, P, I64]),
    "fap_measure_relax_peak": (INT, [P, INT, ctypes.POINTER(DBL)]),
    "fap_graph_tune_sssp": (INT, [P, P, I32, I32, ctypes.POINTER(DBL), P]),
    "fap_graph_mean_weight": (DBL, [P]),
    "fap_graph_release": (INT, [P]),
    "fap_graph_device_bytes": (INT, [P, ctypes.POINTER(I64)]),
    "fap_graph_resident": (INT, [P, I32]),
    "fap_graph_rows_async": (INT, [P, P, I32, P]),
    "fap_graph_cache_build": (INT, [P]),
    "fap_graph_cache_rebuild": (INT, [P]),
    "fap_graph_cache_timing": (INT, [P, P]),
    "fap_graph_cache_release": (INT, [P]),
    "fap_graph_cache_bytes": (INT, [P, ctypes.POINTER(I64), ctypes.POINTER(INT)]),
    "fap_server_create": (INT, [INT, DBL, I64, PP]),
    "fap_server_destroy": (INT, [P]),
    "fap_server_add_graph": (INT, [P, I32, I64, P, P, P, INT, I32, P, P, P, P, P, ctypes.POINTER(I32)]),
    "fap_server_submit": (INT, [P, I32, INT, P, I32, P, P, ctypes.POINTER(I64)]),
    "fap_server_wait": (INT, [P, I64, DBL, ctypes.POINTER(INT)]),
    "fap_server_request_info": (INT, [P, I64, P]),
    "fap_server_forget": (INT, [P, I64]),
    "fap_server_drain": (INT, [P]),
    "fap_server_stats": (INT, [P, P, I32]),
    "fap_server_reset_stats": (INT, [P]),
    "fap_server_set_option": (INT, [P, ctypes.c_char_p, DBL]),
    "fap_graph_checksums_async": (INT, [P, I32, P]),
    "fap_graph_status_async": (INT, [P, P]),
    "fap_status_code": (INT, [I32]),
    "fap_server_last_error": (ctypes.c_char_p, []),
    "fap_floyd_noalloc": (INT, [INT, I32, P, I64, P]),
    "fap_floyd_noalloc_last_error": (ctypes.c_char_p, []),
    "fap_floyd_noalloc_status": (INT, []),
    "fap_graph_pack16_tiles": (INT, [P, ctypes.POINTER(I64), ctypes.POINTER(I64)]),
    "fap_graph_expand16_tiles": (INT, [P, ctypes.POINTER(I64), ctypes.POINTER(I64)]),
    "fap_graph_shard_begin": (INT, [P, P, I32, P, I64, ctypes.POINTER(I64)]),
    "fap_graph_shard_finish": (INT, [P, P, I32, P, I64]),
    "fap_legacy_last_status": (INT, []),
    "fap_host_last_error": (ctypes.c_char_p, []),
    "fap_host_from_mtx": (INT, [ctypes.c_char_p, INT, INT, INT, PP]),
    "fap_host_from_csr": (INT, [I32, I64, P, P, P, INT, INT, PP]),
    "fap_host_save": (INT, [P, ctypes.c_char_p]),
    "fap_host_load": (INT, [ctypes.c_char_p, PP]),
    "fap_host_flags": (INT, [P, P, P]),
    "fap_host_destroy": (INT, [P]),
    "fap_host_set_partition": (INT, [P, P]),
    "fap_host_set_options": (INT, [P, INT, INT, INT]),
    "fap_host_set_max_resident_rows": (INT, [P, I64]),
    "fap_host_precondition": (INT, [P]),
    "fap_host_is_split": (INT, [P]),
    "fap_host_dtype": (INT, [P]),
    "fap_host_sizes": (INT, [P, P]),
    "fap_host_csr": (INT, [P, P, P, P]),
    "fap_host_graph_id": (INT, [P, P]),
    "fap_host_mapping": (INT, [P, P]),
    "fap_host_parts": (INT, [P, P, P, P]),
    "fap_host_solve": (INT, [P, INT]),
    "fap_host_solve_subgraph": (INT, [P, INT, INT]),
    "fap_host_current_subgraph": (INT, [P]),
    "fap_host_subgraph_distance": (INT, [P, INT, P]),
    "fap_host_all_distance": (INT, [P, P]),
    "fap_host_distance_from_one_point": (INT, [P, INT, P]),
    "fap_host_distance_p2p": (INT, [P, INT, INT, ctypes.POINTER(ctypes.c_float)]),
    "fap_host_subgraph_path": (INT, [P, INT, P]),
    "fap_host_all_path": (INT, [P, P]),
    "fap_host_path_from_one_point": (INT, [P, INT, P]),
    "fap_host_path_p2p": (INT, [P, INT, INT, P, I32, ctypes.POINTER(I32)]),
    "fap_host_check_result": (INT, [P, INT, ctypes.POINTER(INT)]),
    "fap_host_device_graph": (P, [P]),
}

# C++-linkage legacy entry points (fap/kernel/cuda/cuda_kernel.h of the
# reference); looked up by their mangled names.
LEGACY_SYMBOLS = {
    "handle_boundry_Nvidia_GPU": "_Z25handle_boundry_Nvidia_GPUPfiiiPiS0_S0_S_S0_i",
    "floyd_GPU_Nvidia_path": "_Z21floyd_GPU_Nvidia_pathiPfPi",
    "minplus_NVIDIA_path": "_Z19minplus_NVIDIA_pathPfS_PiS_S0_iii",
    "floyd_NVIDIA_GPU": "_Z16floyd_NVIDIA_GPUiPf",
    "floyd_path_A_Nvidia": "_Z19floyd_path_A_NvidiaPfPiiiS_S0_",
    "floyd_path_B_Nvidia": "_Z19floyd_path_B_NvidiaPfPiiiS_S0_",
    "floyd_min_plus_Nvidia": "_Z21floyd_min_plus_NvidiaPfS_PiS_S0_iii",
    "minplus_NVIDIA_GPU": "_Z18minplus_NVIDIA_GPUPfS_S_iii",
}


def lib():
    """Load libfap_b200.so (building it first when a toolchain is present and
    the file is missing).  Raises if it cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    L = lib()
    msgs = [m.decode() for m in (L.fap_last_error(), L.fap_host_last_error(),
                                 L.fap_server_last_error()) if m]
    return " | ".join(msgs) or "unknown error"


def check(rc: int, what: str = "") -> None:
    if rc != FAP_OK:
        raise FapError(rc, f"{what}: {last_error()}" if what else last_error())


def ptr(a) -> ctypes.c_void_p:
    """Address of a numpy array, a torch tensor or an int."""
    if a is None:
        return ctypes.c_void_p(0)
    if isinstance(a, int):
        return ctypes.c_void_p(a)
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)
