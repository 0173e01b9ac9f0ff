"""ctypes front end of the CPU oracle (oracle/radik_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker.  The product path
(radik.jl_b200) never imports this module.

The C file restates RadiK.jl's top-k path; see its header for the reference
citations and the three documented semantic choices where the reference's own
result is ill-defined.
"""
from __future__ import annotations

import ctypes
import os
import pathlib
import subprocess

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
_SO = _HERE / "_build" / "libradik_oracle.so"
_lib = None


def build() -> pathlib.Path:
    """Compile the oracle with its Makefile (gcc, OpenMP) if it is stale."""
    src = _HERE / "radik_oracle.c"
    if not _SO.exists() or _SO.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _SO


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(_SO))
        P, I64, I32, U32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_uint32
        L.ro_key.argtypes = [ctypes.c_float]
        L.ro_key.restype = U32
        L.ro_get_bin_id.argtypes = [ctypes.c_float, I32, I32]
        L.ro_get_bin_id.restype = U32
        L.ro_sample_scaler.argtypes = [P, I64, I32]
        L.ro_sample_scaler.restype = ctypes.c_float
        L.ro_apply_scaling.argtypes = [ctypes.c_float, ctypes.c_float, I32, I32]
        L.ro_apply_scaling.restype = ctypes.c_float
        L.ro_count_bin_ex.argtypes = [P, P, I64, I32, I32, I64, I32, I32, P]
        L.ro_count_bin.argtypes = [P, P, I64, I64, I32, I32, I64, P]
        L.ro_select_bin.argtypes = [P, I64, I64, I32, P, P, P]
        L.ro_select_candidate.argtypes = [P, P, I64, I64, P, I32, I32, P, P]
        L.ro_select_candidate_ex.argtypes = [P, P, I64, P, I32, I32, I32, I32, I64, P, P]
        L.ro_filter.argtypes = [P, P, I64, P, P, I64, I64, I32, I32, P, I32, P, P, I32, P]
        L.ro_topk.argtypes = [P, P, I64, I64, I32, I32, I32, P, I32, P, P, I32, I32]
        L.ro_topk.restype = I32
        L.ro_max_threads.restype = I32
        _lib = L
    return _lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def key(v: float) -> int:
    return int(lib().ro_key(ctypes.c_float(v)))


def get_bin_id(v: float, left: int, right: int) -> int:
    return int(lib().ro_get_bin_id(ctypes.c_float(v), left, right))


def apply_scaling(v: float, scaler: float, withscale: bool, largest: bool) -> float:
    return float(lib().ro_apply_scaling(ctypes.c_float(v), ctypes.c_float(scaler),
                                        int(withscale), int(largest)))


def offsets(task_lens) -> np.ndarray:
    off = np.zeros(len(task_lens) + 1, dtype=np.int64)
    np.cumsum(np.asarray(task_lens, dtype=np.int64), out=off[1:])
    return off


def count_bin_ex(data, task_lens, left, right, withscale=False, largest=True):
    data = np.ascontiguousarray(data, dtype=np.float32)
    off = offsets(task_lens)
    bins = 1 << (32 - right)
    hist = np.zeros((len(task_lens), bins), dtype=np.int32)
    lib().ro_count_bin_ex(_p(data), _p(off), len(task_lens), left, right, bins,
                          int(withscale), int(largest), _p(hist))
    return hist


def count_bin(padded, task_lens, stride, left, right):
    padded = np.ascontiguousarray(padded, dtype=np.float32)
    tl = np.ascontiguousarray(task_lens, dtype=np.int32)
    bins = 1 << (32 - right)
    hist = np.zeros((len(tl), bins), dtype=np.int32)
    lib().ro_count_bin(_p(padded), _p(tl), int(stride), len(tl), left, right, bins, _p(hist))
    return hist


def select_bin(hist, k_values, largest, bin_ids=None, counts=None):
    """Returns (bin_ids 1-based, residual k_values, counts); untouched entries
    keep their input values (the reference writes nothing when k is out of
    range)."""
    hist = np.ascontiguousarray(hist, dtype=np.int32)
    T, bins = hist.shape
    kv = np.array(k_values, dtype=np.int32)
    bi = np.zeros(T, np.int32) if bin_ids is None else np.array(bin_ids, np.int32)
    ct = np.zeros(T, np.int32) if counts is None else np.array(counts, np.int32)
    lib().ro_select_bin(_p(hist), T, bins, int(largest), _p(bi), _p(kv), _p(ct))
    return bi, kv, ct


def select_candidate(padded, task_lens, stride, bin_ids, left, right):
    padded = np.ascontiguousarray(padded, dtype=np.float32)
    tl = np.ascontiguousarray(task_lens, dtype=np.int32)
    bi = np.ascontiguousarray(bin_ids, dtype=np.int32)
    out = np.zeros_like(padded)
    cnt = np.zeros(len(tl), np.int32)
    lib().ro_select_candidate(_p(padded), _p(tl), int(stride), len(tl), _p(bi), left, right,
                              _p(out), _p(cnt))
    return [out[t * stride: t * stride + cnt[t]] for t in range(len(tl))]


def select_candidate_ex(data, task_lens, bin_ids, left, right, withscale=False, largest=True):
    data = np.ascontiguousarray(data, dtype=np.float32)
    off = offsets(task_lens)
    stride = max(1, int(max(task_lens)) if len(task_lens) else 1)
    bi = np.ascontiguousarray(bin_ids, dtype=np.int32)
    out = np.zeros(len(task_lens) * stride, np.float32)
    cnt = np.zeros(len(task_lens), np.int32)
    lib().ro_select_candidate_ex(_p(data), _p(off), len(task_lens), _p(bi), left, right,
                                 int(withscale), int(largest), stride, _p(out), _p(cnt))
    return [out[t * stride: t * stride + cnt[t]] for t in range(len(task_lens))]


def filter_(data, task_lens, kth, boundary, k, withscale=False, largest=True,
            idx_in=None, idx_dtype=np.int32):
    """Reference filter primitive; returns per-task lists of (values, indices)
    and the updated boundary counters."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    off = offsets(task_lens)
    T = len(task_lens)
    kth = np.ascontiguousarray(kth, dtype=np.float32)
    bnd = np.array(boundary, dtype=np.int32)
    idx_in_a = None if idx_in is None else np.ascontiguousarray(idx_in)
    ib = 0 if idx_in_a is None else idx_in_a.dtype.itemsize
    out_dtype = np.dtype(idx_dtype) if idx_in_a is None else idx_in_a.dtype
    width = max(int(k), int(max(task_lens)) if T else 0, 1)
    vo = np.zeros(T * width, np.float32)
    io = np.zeros(T * width, out_dtype)
    cnt = np.zeros(T, np.int32)
    lib().ro_filter(_p(data), _p(off), T, _p(kth), _p(bnd), int(k), int(width), int(withscale),
                    int(largest), _p(idx_in_a), ib, _p(vo), _p(io), out_dtype.itemsize, _p(cnt))
    res = [(vo[t * width: t * width + cnt[t]], io[t * width: t * width + cnt[t]]) for t in range(T)]
    return res, bnd


def topk(data, task_lens, k, largest=True, rev=False, withscale=False, indices=None,
         idx_dtype=np.int32, threads=0):
    """Exact batched top-k.  Returns (values[T, k], indices[T, k]) with task
    rows (the Julia API's column-major [k, T])."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    off = offsets(task_lens)
    T = len(task_lens)
    idx_a = None if indices is None else np.ascontiguousarray(indices)
    out_dtype = np.dtype(idx_dtype) if idx_a is None else idx_a.dtype
    vo = np.zeros((T, k), np.float32)
    io = np.zeros((T, k), out_dtype)
    rc = lib().ro_topk(_p(data), _p(off), T, int(k), int(largest), int(not rev), int(withscale),
                       _p(idx_a), 0 if idx_a is None else idx_a.dtype.itemsize,
                       _p(vo), _p(io), out_dtype.itemsize, int(threads))
    if rc != 0:
        raise RuntimeError(f"oracle ro_topk failed with {rc}")
    return vo, io


def max_threads() -> int:
    return int(lib().ro_max_threads())


def env_threads() -> int:
    return int(os.environ.get("OMP_NUM_THREADS", "0") or 0)
