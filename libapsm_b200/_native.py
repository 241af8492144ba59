"""ctypes binding of libapsm_b200.so (the C ABI of include/apsm_b200.h).

The library is built in-tree by ``python -m libapsm_b200.build``.  There is no
fallback: if the shared library is missing or fails to load, every detector
call raises.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libapsm_b200.so"

APSM_OK = 0
APSM_ERR_INVALID_ARGUMENT = 1
APSM_ERR_INVALID_CONFIG = 2
APSM_ERR_CUDA = 3
APSM_ERR_OUT_OF_MEMORY = 4
APSM_ERR_UNSUPPORTED = 5
APSM_ERR_NO_DEVICE = 6
APSM_ERR_TIMEOUT = 7
APSM_ERR_DEADLINE = 8
APSM_ERR_CANCELLED = 9
APSM_FAULT_LANE_ALLOC = 1
APSM_FAULT_DROP_REQUEST = 2

STATUS_NAMES = {
    APSM_OK: "APSM_OK",
    APSM_ERR_INVALID_ARGUMENT: "APSM_ERR_INVALID_ARGUMENT",
    APSM_ERR_INVALID_CONFIG: "APSM_ERR_INVALID_CONFIG",
    APSM_ERR_CUDA: "APSM_ERR_CUDA",
    APSM_ERR_OUT_OF_MEMORY: "APSM_ERR_OUT_OF_MEMORY",
    APSM_ERR_UNSUPPORTED: "APSM_ERR_UNSUPPORTED",
    APSM_ERR_NO_DEVICE: "APSM_ERR_NO_DEVICE",
    APSM_ERR_TIMEOUT: "APSM_ERR_TIMEOUT",
    APSM_ERR_DEADLINE: "APSM_ERR_DEADLINE",
    APSM_ERR_CANCELLED: "APSM_ERR_CANCELLED",
}

# (name, restype, argtypes) of every exported entry point
_P = ctypes.c_void_p
_F = ctypes.POINTER(ctypes.c_float)
_U32 = ctypes.c_uint32
SIGNATURES = [
    ("apsm_version", ctypes.c_char_p, []),
    ("apsm_create", ctypes.c_int, [ctypes.c_char_p, _U32, _U32, ctypes.POINTER(_P), ctypes.c_char_p, ctypes.c_size_t]),
    ("apsm_destroy", None, [_P]),
    ("apsm_train", ctypes.c_int, [_P, _P, _P, _U32, _F]),
    ("apsm_train_history", ctypes.c_int, [_P, _P, _P, _U32, _P, _P, _U32, _U32, ctypes.c_float, _P, _U32,
                                          ctypes.POINTER(_U32), _F]),
    ("apsm_train_steps", _U32, [_P, _U32]),
    ("apsm_norm_ratio", ctypes.c_int, [_P, _U32, _F]),
    ("apsm_gaussian_variance", ctypes.c_int, [_P, _F]),
    ("apsm_detect", ctypes.c_int, [_P, _P, _U32, _P, _F]),
    ("apsm_reset", ctypes.c_int, [_P]),
    ("apsm_train_device", ctypes.c_int, [_P, _P, _P, _U32, _P]),
    ("apsm_detect_device", ctypes.c_int, [_P, _P, _U32, _P, _P]),
    ("apsm_detect_device_noalloc", ctypes.c_int, [_P, _P, _U32, _P, _P]),
    ("apsm_stream", _P, [_P]),
    ("apsm_synchronize", ctypes.c_int, [_P]),
    ("apsm_rows", _U32, [_P]),
    ("apsm_get_state", ctypes.c_int, [_P, _P, _P, _P]),
    ("apsm_copy_state", ctypes.c_int, [_P, _P]),
    ("apsm_last_kernel_ms", ctypes.c_int, [_P, _F, _F]),
    ("apsm_last_error", ctypes.c_char_p, [_P]),
    ("apsm_set_wait_limit_ns", None, [ctypes.c_uint64]),
    ("apsm_wait_limit_ns", ctypes.c_uint64, []),
    ("apsm_measure_ex2_rate", ctypes.c_int, [ctypes.POINTER(ctypes.c_double), _F]),
    # detector pool (batched many-detector form)
    ("apsm_pool_create", ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint64, _U32, ctypes.POINTER(_P), ctypes.c_char_p,
                                        ctypes.c_size_t]),
    ("apsm_pool_destroy", None, [_P]),
    ("apsm_pool_add", ctypes.c_int, [_P, _U32, ctypes.POINTER(_U32)]),
    ("apsm_pool_remove", ctypes.c_int, [_P, _U32]),
    ("apsm_pool_reset", ctypes.c_int, [_P, _U32]),
    ("apsm_pool_run", ctypes.c_int, [_P, _U32, _P, _U32, ctypes.c_int]),
    ("apsm_pool_wait", ctypes.c_int, [_P, _U32]),
    ("apsm_pool_reserve", ctypes.c_int, [_P, _U32, _P, _U32, ctypes.c_int]),
    ("apsm_pool_autotune", ctypes.c_int, [_P, _U32, _P, _U32, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]),
    ("apsm_pool_query", ctypes.c_int, [_P, _U32]),
    ("apsm_pool_stream", _P, [_P, _U32]),
    ("apsm_pool_job_bytes", ctypes.c_uint64, [_P, _P]),
    ("apsm_pool_budget", ctypes.c_uint64, [_P]),
    ("apsm_pool_bytes_in_use", ctypes.c_uint64, [_P]),
    ("apsm_pool_last_ms", ctypes.c_int, [_P, _U32, _F, _F]),
    ("apsm_pool_get_state", ctypes.c_int, [_P, _U32, ctypes.POINTER(_U32), _P, _P]),
    ("apsm_pool_last_error", ctypes.c_char_p, [_P]),
    ("apsm_pool_last_launches", ctypes.c_int, [_P, _U32]),
    ("apsm_pool_last_sweep_ms", ctypes.c_int, [_P, _U32, _F]),
    ("apsm_pool_set_timing", ctypes.c_int, [_P, ctypes.c_int]),
    ("apsm_pool_check_job", ctypes.c_int, [_P, _P]),
    ("apsm_pool_inject_fault", ctypes.c_int, [_P, ctypes.c_int, _U32]),
    # request server (continuous batching over a pool)
    ("apsm_server_create", ctypes.c_int, [_P, _U32, _U32, ctypes.POINTER(_P)]),
    ("apsm_server_destroy", None, [_P]),
    ("apsm_server_submit", ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_uint64)]),
    ("apsm_server_submit_deadline", ctypes.c_int, [_P, _P, ctypes.c_double, ctypes.POINTER(ctypes.c_uint64)]),
    ("apsm_server_set_deadline", ctypes.c_int, [_P, ctypes.c_double]),
    ("apsm_server_cancel", ctypes.c_int, [_P, ctypes.c_uint64]),
    ("apsm_server_counts", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64),
                                          ctypes.POINTER(ctypes.c_uint64)]),
    ("apsm_server_inject_fault", ctypes.c_int, [_P, ctypes.c_int, _U32]),
    ("apsm_server_poll", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int)]),
    ("apsm_server_wait", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_double]),
    ("apsm_server_times", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    ("apsm_server_release", ctypes.c_int, [_P, ctypes.c_uint64]),
    ("apsm_server_stats", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    ("apsm_server_clock", ctypes.c_double, []),
]

_lib = None
_lock = threading.Lock()


def load() -> ctypes.CDLL:
    """Load (once) and return the native library; raises if it is missing."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"native library {LIB_PATH} is missing; build it with `python -m libapsm_b200.build`"
            )
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib
