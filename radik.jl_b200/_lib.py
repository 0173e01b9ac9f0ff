"""ctypes binding of libradik_b200.so (the C ABI in include/radik.h).

There is no CPU fallback: if the library is missing or cannot be loaded the
import of the binding raises, and every entry point reports CUDA errors as
RadiKError.
"""
from __future__ import annotations

import ctypes
import pathlib
import threading

_PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = _PKG / "libradik_b200.so"

RADIK_LARGEST = 0x1
RADIK_ASCEND = 0x2
RADIK_WITHSCALE = 0x4
RADIK_WITHIDXIN = 0x8
RADIK_WITHPACKING = 0x10
RADIK_ASYNC = 0x100
RADIK_PLAIN = 0x200

STATUS = {
    0: "RADIK_OK", 1: "RADIK_ERR_INVALID", 2: "RADIK_ERR_OOM", 3: "RADIK_ERR_WS_TOO_SMALL",
    4: "RADIK_ERR_CUDA", 5: "RADIK_ERR_DEVICE", 6: "RADIK_ERR_TIMEOUT", 7: "RADIK_ERR_CAPTURE",
}

# Every symbol include/radik.h declares (checked by the CPU test suite).
EXPORTS = (
    "radik_ws_create", "radik_ws_destroy", "radik_ws_bytes", "radik_ws_error", "radik_ws_prepare",
    "radik_ws_plan_info", "radik_ws_autotune",
    "radik_topk_radix_select", "radik_topk", "radik_topk_host", "radik_topk_noalloc",
    "radik_count_bin_ex", "radik_count_bin", "radik_select_bin", "radik_filter",
    "radik_last_error", "radik_status_string", "radik_version", "radik_alloc_count",
    "radik_tune_save", "radik_tune_load", "radik_tune_clear",
    "radik_server_create", "radik_server_destroy", "radik_server_submit", "radik_server_wait",
    "radik_server_get_stats", "radik_server_get_latencies", "radik_server_get_batches", "radik_server_reset_stats",
)


class PlanInfo(ctypes.Structure):
    """radik_plan_info (include/radik.h)."""
    _fields_ = [(n, ctypes.c_int) for n in (
        "path", "block_threads", "grid", "smem_bytes", "candidate_capacity", "segments", "sample_jobs",
        "kernels_per_call")]


class ServerConfig(ctypes.Structure):
    """radik_server_config (include/radik.h)."""
    _fields_ = [("slots", ctypes.c_int), ("device", ctypes.c_int), ("mem_cap_bytes", ctypes.c_int64),
                ("max_batch_rows", ctypes.c_int64)]


class ServerStats(ctypes.Structure):
    """radik_server_stats (include/radik.h)."""
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("rows", ctypes.c_uint64), ("elements", ctypes.c_double), ("p50_us", ctypes.c_double),
                ("p99_us", ctypes.c_double), ("mean_us", ctypes.c_double), ("mem_in_flight", ctypes.c_int64),
                ("mem_pool", ctypes.c_int64)]


class ServerBatch(ctypes.Structure):
    """radik_server_batch (include/radik.h)."""
    _fields_ = [("k", ctypes.c_int64), ("rows", ctypes.c_int64), ("max_row_len", ctypes.c_int64),
                ("elements", ctypes.c_double), ("gpu_us", ctypes.c_double), ("launch_us", ctypes.c_double)]


class RadiKError(Exception):
    """Raised for invalid arguments and engine failures (Julia's ErrorException)."""

    def __init__(self, msg: str, status: int | None = None):
        super().__init__(msg)
        self.status = status


_lock = threading.Lock()
_lib: ctypes.CDLL | None = None


def _declare(L: ctypes.CDLL) -> None:
    P, I, I64, U32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_uint32
    PP = ctypes.POINTER(ctypes.c_void_p)
    L.radik_ws_create.argtypes = [I64, I64, I, PP]
    L.radik_ws_destroy.argtypes = [P]
    L.radik_ws_bytes.argtypes = [P, ctypes.POINTER(ctypes.c_size_t)]
    L.radik_ws_error.argtypes = [P, ctypes.POINTER(U32)]
    L.radik_ws_prepare.argtypes = [P, P, I64, I64, U32, I]
    L.radik_ws_plan_info.argtypes = [P, ctypes.POINTER(PlanInfo)]
    L.radik_ws_autotune.argtypes = [P, P, P, I, P, P, P, I64, I64, U32, P, I, ctypes.POINTER(PlanInfo),
                                    ctypes.POINTER(ctypes.c_double)]
    L.radik_topk_radix_select.argtypes = [P, P, I, P, P, P, P, I64, I64, U32, P]
    L.radik_topk.argtypes = [P, P, I, P, I64, P, I64, P, I64, I64, I, I, P]
    L.radik_topk_host.argtypes = [P, P, I, P, I64, P, I64, P, I64, I64, I, I, P, P]
    L.radik_topk_noalloc.argtypes = [P, P, I, P, P, P, I64, I64, U32, P]
    L.radik_count_bin_ex.argtypes = [P, P, P, I64, I, I, I, I, P]
    L.radik_count_bin.argtypes = [P, P, P, I64, I64, I, I, P]
    L.radik_select_bin.argtypes = [P, P, P, P, I64, I64, I, P]
    L.radik_filter.argtypes = [P, P, I, P, P, P, P, P, P, I64, I64, I, I, P]
    L.radik_server_create.argtypes = [ctypes.POINTER(ServerConfig), PP]
    L.radik_server_destroy.argtypes = [P]
    L.radik_server_submit.argtypes = [P, P, I64, I64, I64, U32, P, P, I, ctypes.POINTER(ctypes.c_uint64)]
    L.radik_server_wait.argtypes = [P, ctypes.c_uint64, I64]
    L.radik_server_get_stats.argtypes = [P, ctypes.POINTER(ServerStats)]
    L.radik_server_get_latencies.argtypes = [P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_double),
                                             I64, ctypes.POINTER(I64)]
    L.radik_server_get_batches.argtypes = [P, ctypes.POINTER(ServerBatch), I64, ctypes.POINTER(I64)]
    L.radik_server_reset_stats.argtypes = [P]
    L.radik_alloc_count.argtypes = [ctypes.POINTER(ctypes.c_uint64)]
    L.radik_tune_save.argtypes = [ctypes.c_char_p]
    L.radik_tune_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(I64)]
    L.radik_tune_clear.argtypes = []
    L.radik_last_error.restype = ctypes.c_char_p
    L.radik_status_string.restype = ctypes.c_char_p
    L.radik_status_string.argtypes = [I]
    L.radik_version.restype = ctypes.c_char_p
    for name in EXPORTS:
        if name not in ("radik_last_error", "radik_status_string", "radik_version"):
            getattr(L, name).restype = I


def load(path: pathlib.Path | str | None = None) -> ctypes.CDLL:
    """Load the engine library (no GPU is needed to load it)."""
    global _lib
    with _lock:
        if _lib is None:
            p = pathlib.Path(path) if path else LIB_PATH
            if not p.exists():
                raise RadiKError(
                    f"{p} is missing: build it with `python radik.jl_b200/build.py` "
                    "(the engine has no CPU fallback)")
            L = ctypes.CDLL(str(p))
            _declare(L)
            _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        L = load()
        msg = L.radik_last_error().decode(errors="replace")
        raise RadiKError(msg or STATUS.get(rc, f"status {rc}"), rc)
