"""ctypes binding of libfmm.so (the C ABI declared in include/fmm.h).

The library is built in-tree by ``python -m fast_matmul_b200.build``.  There
is no fallback: if the library is missing or a call fails, an exception
says so.
"""

from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
# FMM_LIBRARY selects another build of the engine, e.g. libfmm_checked.so
# (device-side checks, see fmm_debug_check_flags); the default is libfmm.so.
LIB_PATH = os.environ.get("FMM_LIBRARY") or os.path.join(_HERE, "libfmm.so")

_lock = threading.Lock()
_lib = None

c_double_p = ctypes.POINTER(ctypes.c_double)

FMM_OK = 0
STATUS_NAMES = {
    0: "FMM_OK",
    1: "FMM_ERR_INVALID_ARGUMENT",
    2: "FMM_ERR_UNKNOWN_ALGORITHM",
    3: "FMM_ERR_OUT_OF_MEMORY",
    4: "FMM_ERR_CUDA",
    5: "FMM_ERR_NOT_SUPPORTED",
    6: "FMM_ERR_WORKSPACE_TOO_SMALL",
    7: "FMM_ERR_TIMEOUT",
}

SCHEDULES = {"auto": 0, "dfs": 1, "bfs": 2, "hybrid": 3}
PRECISIONS = {"fp64": 0, "split_bf16": 1, "split_int8": 2}
GEMM_TILES = {"auto": 0, "large": 1, "small": 2}


class FmmError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, str(status)), message))
        self.status = status


class Options(ctypes.Structure):
    _fields_ = [
        ("schedule", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("split_slices", ctypes.c_int),
        ("dfs_levels", ctypes.c_int),
        ("workspace_limit", ctypes.c_size_t),
        ("gemm_tile", ctypes.c_int),
    ]


class Profile(ctypes.Structure):
    _fields_ = [
        ("form_launches", ctypes.c_int64), ("gemm_launches", ctypes.c_int64),
        ("peel_launches", ctypes.c_int64), ("combine_launches", ctypes.c_int64),
        ("form_ms", ctypes.c_double), ("gemm_ms", ctypes.c_double),
        ("peel_ms", ctypes.c_double), ("combine_ms", ctypes.c_double),
        ("form_bytes", ctypes.c_double), ("combine_bytes", ctypes.c_double),
        ("gemm_flops", ctypes.c_double), ("peel_flops", ctypes.c_double),
        ("split_ms", ctypes.c_double), ("split_bf16_flops", ctypes.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


FMM_ALG_AUTO = -1
FMM_ALG_CLASSICAL = -2


class BatchItem(ctypes.Structure):
    _fields_ = [
        ("alg", ctypes.c_int), ("num_steps", ctypes.c_int),
        ("A", ctypes.c_void_p), ("lda", ctypes.c_int64),
        ("B", ctypes.c_void_p), ("ldb", ctypes.c_int64),
        ("C", ctypes.c_void_p), ("ldc", ctypes.c_int64),
        ("m", ctypes.c_int64), ("k", ctypes.c_int64), ("n", ctypes.c_int64),
        ("x", ctypes.c_double), ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
        ("precision", ctypes.c_int), ("split_slices", ctypes.c_int),
        ("gemm_tile", ctypes.c_int),
    ]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("workspace_bytes", ctypes.c_size_t), ("max_inflight", ctypes.c_int),
                ("max_batch", ctypes.c_int)]


class Request(ctypes.Structure):
    _fields_ = [
        ("alg", ctypes.c_int), ("num_steps", ctypes.c_int), ("precision", ctypes.c_int),
        ("A", ctypes.c_void_p), ("lda", ctypes.c_int64),
        ("B", ctypes.c_void_p), ("ldb", ctypes.c_int64),
        ("C", ctypes.c_void_p), ("ldc", ctypes.c_int64),
        ("m", ctypes.c_int64), ("k", ctypes.c_int64), ("n", ctypes.c_int64),
        ("x", ctypes.c_double), ("alpha", ctypes.c_double), ("beta", ctypes.c_double),
        ("split_slices", ctypes.c_int),
    ]


class RequestInfo(ctypes.Structure):
    _fields_ = [("done", ctypes.c_int), ("status", ctypes.c_int), ("submit_ms", ctypes.c_double),
                ("launch_ms", ctypes.c_double), ("done_ms", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("launches", ctypes.c_int64),
                ("batches", ctypes.c_int64), ("max_batch_seen", ctypes.c_int64),
                ("workspace_peak", ctypes.c_size_t)]


# name -> (restype, argtypes); every function declared in include/fmm.h
SIGNATURES = {
    "fmm_options_init": (None, [ctypes.POINTER(Options)]),
    "fmm_handle_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]),
    "fmm_handle_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fmm_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "fmm_set_workspace_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t]),
    "fmm_release_workspace": (ctypes.c_int, [ctypes.c_void_p]),
    "fmm_debug_check_flags": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint)]),
    "fmm_debug_fill_workspace": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]),
    "fmm_last_error": (ctypes.c_char_p, []),
    "fmm_num_algorithms": (ctypes.c_int, []),
    "fmm_algorithm_name": (ctypes.c_char_p, [ctypes.c_int]),
    "fmm_algorithm_header": (ctypes.c_char_p, [ctypes.c_int]),
    "fmm_algorithm_lookup": (ctypes.c_int, [ctypes.c_char_p]),
    "fmm_algorithm_info": (ctypes.c_int, [ctypes.c_int] + [ctypes.POINTER(ctypes.c_int)] * 5),
    "fmm_fast_matmul": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
                                        ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                        ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.POINTER(Options)]),
    "fmm_fast_matmul_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
                                             ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                             ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                             ctypes.POINTER(Options), c_double_p]),
    "fmm_fast_matmul_host_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
                                                   ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                                   ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                                   ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                   ctypes.POINTER(Options)]),
    "fmm_host_sync": (ctypes.c_int, [ctypes.c_void_p]),
    "fmm_workspace_query": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
                                            ctypes.c_int64, ctypes.c_int, ctypes.POINTER(Options),
                                            ctypes.POINTER(ctypes.c_size_t)]),
    "fmm_dgemm": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                  ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                  ctypes.c_int64, ctypes.c_int64, ctypes.c_double, ctypes.c_double]),
    "fmm_dgemm_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                       ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                       ctypes.c_int64, ctypes.c_int64, ctypes.c_double, ctypes.c_double]),
    "fmm_dgemm_split_bf16": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                             ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                             ctypes.c_int64, ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_int]),
    "fmm_dgemm_split_int8": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                             ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                             ctypes.c_int64, ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_int]),
    "fmm_fill_uniform": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                         ctypes.c_int64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_double,
                                         ctypes.c_double]),
    "fmm_max_relative_diff": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                              ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, c_double_p,
                                              c_double_p]),
    "fmm_diagonal_scaling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                             ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "fmm_scaling_postprocess": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                                ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]),
    "fmm_diagonal_scaling_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                                  ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "fmm_scaling_postprocess_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                                     ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                                                     ctypes.c_void_p]),
    "fmm_fast_matmul_f32": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
                                            ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                            ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_float, ctypes.c_float,
                                            ctypes.POINTER(Options)]),
    "fmm_sgemm": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                 ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                 ctypes.c_float, ctypes.c_float, ctypes.POINTER(Options)]),
    "fmm_fast_matmul_f32_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
                                                 ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                                 ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                                 ctypes.c_double, ctypes.c_float, ctypes.c_float,
                                                 ctypes.POINTER(Options), c_double_p]),
    "fmm_sgemm_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                      ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                      ctypes.c_int64, ctypes.c_int64, ctypes.c_float, ctypes.c_float,
                                      ctypes.POINTER(Options)]),
    "fmm_diagonal_scaling_f32": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                                 ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                                 ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "fmm_scaling_postprocess_f32": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                                    ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                                                    ctypes.c_void_p]),
    "fmm_diagonal_scaling_f32_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                                      ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                                      ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                                      ctypes.c_void_p, ctypes.c_void_p]),
    "fmm_scaling_postprocess_f32_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                                         ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                                                         ctypes.c_void_p]),
    "fmm_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "fmm_kernel_launch_count": (ctypes.c_int64, [ctypes.c_void_p]),
    "fmm_selftest_wait_timeout": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]),
    "fmm_fast_matmul_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                                ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                                ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
    "fmm_fast_matmul_batched": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchItem), ctypes.c_int]),
    "fmm_autotune_tile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                          ctypes.POINTER(ctypes.c_int)]),
    "fmm_autotune_choice": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                            ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "fmm_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int]),
    "fmm_autotune_export": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t,
                                            ctypes.POINTER(ctypes.c_size_t)]),
    "fmm_autotune_import": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p]),
    "fmm_plan_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
                                        ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                        ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.POINTER(Options),
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "fmm_plan_create_batched": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchItem), ctypes.c_int,
                                                ctypes.POINTER(ctypes.c_void_p)]),
    "fmm_plan_execute": (ctypes.c_int, [ctypes.c_void_p]),
    "fmm_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fmm_plan_kernel_count": (ctypes.c_int64, [ctypes.c_void_p]),
    "fmm_server_create": (ctypes.c_int, [ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "fmm_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)]),
    "fmm_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double,
                                        ctypes.POINTER(RequestInfo)]),
    "fmm_server_drain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "fmm_server_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerStats)]),
    "fmm_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fmm_profile_enable": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "fmm_profile_reset": (ctypes.c_int, [ctypes.c_void_p]),
    "fmm_profile_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Profile)]),
}


def lib() -> ctypes.CDLL:
    """The loaded engine library; raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError("%s is missing: build it with `python -m fast_matmul_b200.build`" % LIB_PATH)
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
        return _lib


def check(status: int) -> None:
    if status != FMM_OK:
        msg = lib().fmm_last_error()
        raise FmmError(status, msg.decode() if msg else "")
