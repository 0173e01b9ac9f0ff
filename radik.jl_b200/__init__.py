"""radik.jl_b200 -- Python host side of the B200 exact Float32 radix top-k.

This module mirrors RadiK.jl's public API (src/RadiK.jl:19-22 exports
``topk_radix_select!``, ``topk``, ``topk!``, ``RadiKWorkspace``) over the C ABI
of libradik_b200.so (include/radik.h).  Device arrays are CUDA torch tensors
(torch is used only for device memory and streams); every computation runs in
the library's sm_100a kernels and there is no CPU fallback.

Layout: Julia's column-major ``[k, num_tasks]`` outputs are torch tensors of
shape ``(num_tasks, k)`` (the same memory), the input is the concatenation of
all tasks.  Julia's ``!`` suffix becomes a trailing underscore:

    topk(data, k; indices, largest, rev)                -> topk(data, k, ...)
    topk(data, task_lens, k; ...)                       -> topk(data, task_lens, k, ...)
    topk!(val_out, idx_out, data, [task_lens,] k; ...)  -> topk_(val_out, idx_out, data, [task_lens,] k, ...)
    topk_radix_select!(val_out, idx_out, ws, val_in, idx_in, task_lens, k,
                       Val(LARGEST), Val(ASCEND), Val(WITHSCALE), Val(WITHIDXIN), ...)
                                                        -> topk_radix_select_(...)
    RadiKWorkspace(backend, n, num_tasks, I=Int32)      -> RadiKWorkspace(backend, n, num_tasks, I=torch.int32)
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from ._lib import (RADIK_ASCEND, RADIK_ASYNC, RADIK_LARGEST, RADIK_PLAIN, RADIK_WITHIDXIN,
                   RADIK_WITHPACKING, RADIK_WITHSCALE, RadiKError, check, load)

__all__ = ["topk", "topk_", "topk_radix_select_", "RadiKWorkspace", "RadiKError", "topk_host",
           "count_bin_ex", "count_bin", "select_bin", "filter_", "version", "Server",
           "tune_save", "tune_load", "tune_clear"]


def _torch():
    import torch  # deferred: the library loads without torch
    return torch


def version() -> str:
    return load().radik_version().decode()


def tune_save(path) -> None:
    """Write the process-wide tuning table (the autotuner's choices by batch
    shape, from every workspace) to a text file (radik_tune_save)."""
    check(load().radik_tune_save(str(path).encode()))


def tune_load(path) -> int:
    """Merge a tuning table written by tune_save; returns the entries read.
    Workspaces then use those choices for matching batch shapes without
    autotuning (radik_tune_load)."""
    n = ctypes.c_int64()
    check(load().radik_tune_load(str(path).encode(), ctypes.byref(n)))
    return int(n.value)


def tune_clear() -> None:
    """Forget every remembered tuning choice of the process (workspaces keep
    their own)."""
    check(load().radik_tune_clear())


def _ptr(t) -> ctypes.c_void_p | None:
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(stream) -> ctypes.c_void_p:
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def _lens_array(task_lens) -> np.ndarray:
    """task_lens as a contiguous int64 array: free for such an array, a
    conversion (tens of microseconds for a thousand tasks) for a list."""
    if isinstance(task_lens, np.ndarray) and task_lens.dtype == np.int64 and task_lens.ndim == 1 \
            and task_lens.flags.c_contiguous:
        return task_lens
    return np.ascontiguousarray(np.asarray(task_lens, dtype=np.int64).reshape(-1))


def _check_cuda(t, what: str):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise RadiKError(f"{what} must be a CUDA tensor (the engine has no CPU path)")
    if not t.is_contiguous():
        raise RadiKError(f"{what} must be contiguous")


def _check_float32(data):
    torch = _torch()
    if data.dtype != torch.float32:
        # src/algorithm.jl:492-494
        raise RadiKError(f"RadiK.jl only supports Float32 input data. Got {data.dtype}. "
                         "Convert with: data.to(torch.float32)")


def _check_io(val_out, idx_out, val_in, idx_in, lens: np.ndarray, k: int, withidxin: bool) -> None:
    """Buffer sizes against the batch, then placement: the kernels write
    len(lens) * k entries of each output and read sum(lens) input elements
    (and indices) on the current device, so a short buffer or a tensor on
    another GPU must be refused here, not turned into a device fault.
    Sizes are checked first (they need no GPU)."""
    T, total = len(lens), int(lens.sum()) if len(lens) else 0
    need = T * int(k)
    for name, t, n in (("val_out", val_out, need), ("idx_out", idx_out, need), ("val_in", val_in, total),
                       ("idx_in", idx_in if withidxin else None, total)):
        if t is not None and t.numel() < n:
            what = f"{T} tasks x k = {k}" if name in ("val_out", "idx_out") else f"sum(task_lens) = {total}"
            raise RadiKError(f"{name} holds {t.numel()} elements; {what} needs {n}")
    if withidxin and idx_in is None:
        raise RadiKError("withidxin needs idx_in")
    tensors = [("val_out", val_out), ("idx_out", idx_out), ("val_in", val_in)]
    if withidxin:
        tensors.append(("idx_in", idx_in))
    for name, t in tensors:
        _check_cuda(t, name)
    dev = _torch().cuda.current_device()
    for name, t in tensors:
        if t.device.index != dev:
            raise RadiKError(f"{name} is on cuda:{t.device.index} but the current device is cuda:{dev}; "
                             "the kernels run on the current device")


def _idx_bytes(dtype) -> int:
    torch = _torch()
    if dtype == torch.int32:
        return 4
    if dtype == torch.int64:
        return 8
    raise RadiKError(f"index type must be Int32 or Int64, got {dtype}")


class RadiKWorkspace:
    """Device workspace, RadiKWorkspace(backend, n, num_tasks, I) in
    src/algorithm.jl:58-83.  ``n`` bounds the longest task and ``num_tasks``
    the batch of every call that uses it (src/algorithm.jl:156-160).  The
    engine sizes its buffers from the calls it serves; ``I`` is kept for API
    parity (4- or 8-byte integers)."""

    def __init__(self, backend, n: int, num_tasks: int, I=None):
        torch = _torch()
        self.backend = backend
        self.n = int(n)
        self.num_tasks = int(num_tasks)
        self.I = torch.int32 if I is None else I
        self.device = torch.device("cuda", torch.cuda.current_device()) if backend in (None, "cuda") else \
            torch.device(backend)
        L = load()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(L.radik_ws_create(self.n, self.num_tasks, _idx_bytes(self.I), ctypes.byref(h)))
        self._h = h

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def nbytes(self) -> int:
        b = ctypes.c_size_t()
        check(load().radik_ws_bytes(self._h, ctypes.byref(b)))
        return int(b.value)

    def error_bits(self) -> int:
        b = ctypes.c_uint32()
        check(load().radik_ws_error(self._h, ctypes.byref(b)))
        return int(b.value)

    def prepare(self, task_lens, k: int, *, largest=True, ascend=True, withscale=False,
                withidxin=False, idx_dtype=None, plain=False) -> None:
        """Build the launch plan for a batch shape ahead of CUDA-graph capture."""
        torch = _torch()
        lens = _lens_array(task_lens)
        flags = _flags(largest, ascend, withscale, withidxin, plain)
        ib = _idx_bytes(idx_dtype if idx_dtype is not None else torch.int32)
        check(load().radik_ws_prepare(self._h, lens.ctypes.data_as(ctypes.c_void_p), len(lens), int(k),
                                      flags, ib))

    def plan_info(self) -> dict:
        """The plan the workspace holds (kernel form, grid, launches per call)."""
        from ._lib import PlanInfo
        info = PlanInfo()
        check(load().radik_ws_plan_info(self._h, ctypes.byref(info)))
        return {n: getattr(info, n) for n, _ in PlanInfo._fields_}

    def autotune(self, val_out, idx_out, val_in, idx_in, task_lens, k: int, largest: bool = True,
                 ascend: bool = True, withscale: bool = False, withidxin: bool = False, *, reps: int = 5,
                 stream=None, plain: bool = False) -> dict:
        """Time the candidate configurations on this batch -- of the fused
        path, or with plain=True the multi-pass path's digit schedules -- and
        keep the fastest for its shape, here and in the process-wide tuning
        table (radik_ws_autotune); returns the chosen plan with its time per
        call ("ms")."""
        from ._lib import PlanInfo
        lens = _lens_array(task_lens)
        _check_io(val_out, idx_out, val_in, idx_in, lens, k, withidxin)
        info = PlanInfo()
        ms = ctypes.c_double()
        flags = _flags(largest, ascend, withscale, withidxin, plain=plain)
        check(load().radik_ws_autotune(self._h, _ptr(val_out), _ptr(idx_out), _idx_bytes(idx_out.dtype), _ptr(val_in),
                                       _ptr(idx_in) if withidxin else None, lens.ctypes.data_as(ctypes.c_void_p),
                                       len(lens), int(k), flags, _stream(stream), int(reps), ctypes.byref(info),
                                       ctypes.byref(ms)))
        out = {n: getattr(info, n) for n, _ in PlanInfo._fields_}
        out["ms"] = ms.value
        return out

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            load().radik_ws_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _flags(largest, ascend, withscale, withidxin, plain=False, sync=True) -> int:
    f = RADIK_WITHPACKING
    f |= RADIK_LARGEST if largest else 0
    f |= RADIK_ASCEND if ascend else 0
    f |= RADIK_WITHSCALE if withscale else 0
    f |= RADIK_WITHIDXIN if withidxin else 0
    f |= RADIK_PLAIN if plain else 0
    f |= 0 if sync else RADIK_ASYNC
    return f


def topk_radix_select_(val_out, idx_out, ws: RadiKWorkspace, val_in, idx_in, task_lens, k: int,
                       largest: bool = True, ascend: bool = True, withscale: bool = False,
                       withidxin: bool = False, withpacking: bool = True, vload_size_bytes: int = 32,
                       *, stream=None, plain: bool = False, sync: bool = True):
    """topk_radix_select!(val_out, idx_out, ws, val_in, idx_in, task_lens, k,
    Val(LARGEST), Val(ASCEND), Val(WITHSCALE), Val(WITHIDXIN), Val(WITHPACKING),
    Val(VLOAD_SIZE_BYTES)) -- src/algorithm.jl:162-368.

    Writes the k selected values/indices of every task into val_out/idx_out
    ((num_tasks, k) tensors), sorted ascending when ``ascend``.  Synchronous
    like the reference unless ``sync=False``.  ``withpacking`` and
    ``vload_size_bytes`` are accepted for parity (loads are 128-bit)."""
    _check_float32(val_in)
    lens = _lens_array(task_lens)
    _check_io(val_out, idx_out, val_in, idx_in, lens, k, withidxin)
    if withidxin and idx_in.dtype != idx_out.dtype:
        raise RadiKError("idx_in and idx_out must have the same element type")
    L = load()
    flags = _flags(largest, ascend, withscale, withidxin, plain, sync)
    check(L.radik_topk_radix_select(_ptr(val_out), _ptr(idx_out), _idx_bytes(idx_out.dtype), ws.handle,
                                    _ptr(val_in), _ptr(idx_in) if withidxin else None,
                                    lens.ctypes.data_as(ctypes.c_void_p), len(lens), int(k), flags,
                                    _stream(stream)))
    return val_out, idx_out


def topk_radix_select_noalloc_(val_out, idx_out, val_in, idx_in, task_lens, k: int, largest: bool = True,
                               ascend: bool = True, withscale: bool = False, withidxin: bool = False,
                               *, stream=None):
    """``topk_radix_select_`` without a workspace (no counterpart in the
    reference): the engine's scratch is a static 8 MiB device array, so the
    call allocates no device memory -- for callers inside a memory pool's
    out-of-memory path or under a hard memory cap.  k <= 4096 and the batch's
    scratch must fit in 8 MiB, else RadiKError.  Calls that overlap in time
    on one device race; the first call on a device does set-up and must come
    before any stream capture."""
    _check_float32(val_in)
    lens = _lens_array(task_lens)
    _check_io(val_out, idx_out, val_in, idx_in, lens, k, withidxin)
    if withidxin and idx_in.dtype != idx_out.dtype:
        raise RadiKError("idx_in and idx_out must have the same element type")
    L = load()
    flags = _flags(largest, ascend, withscale, withidxin)
    check(L.radik_topk_noalloc(_ptr(val_out), _ptr(idx_out), _idx_bytes(idx_out.dtype), _ptr(val_in),
                               _ptr(idx_in) if withidxin else None, lens.ctypes.data_as(ctypes.c_void_p),
                               len(lens), int(k), flags, _stream(stream)))
    return val_out, idx_out


def _split_args(task_lens_or_k, k, data):
    if k is None:
        return [int(data.numel())], int(task_lens_or_k), True
    return list(np.asarray(task_lens_or_k, dtype=np.int64).reshape(-1)), int(k), False


def topk_(val_out, idx_out, data, task_lens_or_k, k=None, *, indices=None, largest=True, rev=False,
          stream=None, plain=False):
    """topk!(val_out, idx_out, data, [task_lens,] k; indices, largest, rev) --
    src/algorithm.jl:477-526.  Validates sizes, uses a fresh workspace for the
    call (as the reference does, :503) and returns when the results are
    complete.  ``rev=False`` sorts the selected values ascending (:520)."""
    _check_float32(data)
    task_lens, k, single = _split_args(task_lens_or_k, k, data)
    T = len(task_lens)
    expected = (k,) if (single and val_out.dim() == 1) else (T, k)
    # src/algorithm.jl:497-501
    if tuple(val_out.shape) != expected:
        raise RadiKError(f"val_out must have size {expected}, got {tuple(val_out.shape)}")
    if tuple(idx_out.shape) != expected:
        raise RadiKError(f"idx_out must have size {expected}, got {tuple(idx_out.shape)}")
    # src/algorithm.jl:506-510
    if indices is not None and indices.numel() > 0 and indices.numel() != data.numel():
        raise RadiKError("indices length must equal data length. "
                         f"Got {indices.numel()} vs {data.numel()}")
    with_idx = indices is not None and indices.numel() > 0
    ws = RadiKWorkspace("cuda", max(task_lens) if T else 0, T)
    try:
        topk_radix_select_(val_out, idx_out, ws, data, indices if with_idx else None, task_lens, k,
                           largest, not rev, False, with_idx, True, stream=stream, plain=plain)
    finally:
        ws.close()
    return None


def topk(data, task_lens_or_k, k=None, *, indices=None, largest=True, rev=False, stream=None,
         plain=False):
    """topk(data, k; ...) -> (values[k], indices[k]) and topk(data, task_lens, k; ...)
    -> (values[T, k], indices[T, k]) -- src/algorithm.jl:528-559.  The index
    type follows ``indices`` (default Int32)."""
    torch = _torch()
    _check_float32(data)
    task_lens, kk, single = _split_args(task_lens_or_k, k, data)
    T = len(task_lens)
    idx_dtype = torch.int32 if indices is None else indices.dtype
    val_out = torch.zeros((T, kk), dtype=torch.float32, device=data.device)
    idx_out = torch.zeros((T, kk), dtype=idx_dtype, device=data.device)
    topk_(val_out, idx_out, data, task_lens, kk, indices=indices, largest=largest, rev=rev,
          stream=stream, plain=plain)
    if single:
        return val_out[0], idx_out[0]
    return val_out, idx_out


def topk_host(data: np.ndarray, task_lens: Sequence[int], k: int, *, indices: np.ndarray | None = None,
              largest=True, rev=False, ws: RadiKWorkspace | None = None, stream=None,
              out: tuple[np.ndarray, np.ndarray] | None = None):
    """Top-k of HOST (numpy) buffers through radik_topk_host: copies in,
    selects on the GPU, copies the (T, k) results back."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    lens = _lens_array(task_lens)
    T = len(lens)
    idx_dtype = np.int32 if indices is None else np.asarray(indices).dtype
    if out is None:
        vo = np.zeros((T, k), np.float32)
        io = np.zeros((T, k), idx_dtype)
    else:
        vo, io = out
    own = ws is None
    if own:
        ws = RadiKWorkspace("cuda", int(lens.max()) if T else 0, T)
    try:
        ind = None if indices is None else np.ascontiguousarray(indices)
        check(load().radik_topk_host(vo.ctypes.data_as(ctypes.c_void_p), io.ctypes.data_as(ctypes.c_void_p),
                                     io.dtype.itemsize, data.ctypes.data_as(ctypes.c_void_p), data.size,
                                     None if ind is None else ind.ctypes.data_as(ctypes.c_void_p),
                                     0 if ind is None else ind.size, lens.ctypes.data_as(ctypes.c_void_p), T,
                                     int(k), int(bool(largest)), int(bool(rev)), ws.handle, _stream(stream)))
    finally:
        if own:
            ws.close()
    return vo, io


# ---- stage entry points (the reference kernels' contracts) -----------------

def count_bin_ex(data, task_lens, left: int, right: int, withscale=False, largest=True, stream=None):
    """count_bin_ex_kernel! (src/kernels/count_bin.jl:78-203) -> int32 (T, 2^(32-right))."""
    torch = _torch()
    _check_cuda(data, "data")
    lens = _lens_array(task_lens)
    hist = torch.zeros((len(lens), 1 << (32 - right)), dtype=torch.int32, device=data.device)
    check(load().radik_count_bin_ex(_ptr(hist), _ptr(data), lens.ctypes.data_as(ctypes.c_void_p), len(lens),
                                    left, right, int(withscale), int(largest), _stream(stream)))
    return hist


def count_bin(padded, task_lens, stride: int, left: int, right: int, stream=None):
    """count_bin_kernel! (src/kernels/count_bin.jl:20-59) on the padded layout."""
    torch = _torch()
    _check_cuda(padded, "data")
    lens = _lens_array(task_lens)
    hist = torch.zeros((len(lens), 1 << (32 - right)), dtype=torch.int32, device=padded.device)
    check(load().radik_count_bin(_ptr(hist), _ptr(padded), lens.ctypes.data_as(ctypes.c_void_p), int(stride),
                                 len(lens), left, right, _stream(stream)))
    return hist


def select_bin(hist, k_values, largest: bool, bin_ids=None, counts=None, stream=None):
    """select_bin_kernel! (src/kernels/select_bin.jl:268-348) -> (bin_ids 1-based,
    residual k_values, counts); entries stay unchanged when k is out of range."""
    torch = _torch()
    _check_cuda(hist, "hist")
    T, hl = hist.shape
    kv = torch.as_tensor(np.asarray(k_values, np.int32), device=hist.device).clone()
    bi = torch.zeros(T, dtype=torch.int32, device=hist.device) if bin_ids is None else \
        torch.as_tensor(np.asarray(bin_ids, np.int32), device=hist.device).clone()
    ct = torch.zeros(T, dtype=torch.int32, device=hist.device) if counts is None else \
        torch.as_tensor(np.asarray(counts, np.int32), device=hist.device).clone()
    check(load().radik_select_bin(_ptr(bi), _ptr(kv), _ptr(ct), _ptr(hist.contiguous()), T, hl, int(largest),
                                  _stream(stream)))
    return bi, kv, ct


def filter_(data, task_lens, kth, boundary, k: int, withscale=False, largest=True, idx_in=None,
            idx_dtype=None, stream=None):
    """filter_kernel! / filter_general_kernel! (src/kernels/filter.jl:172-621).
    Returns per-task (values, indices) in emission order and the counters."""
    torch = _torch()
    _check_cuda(data, "data")
    lens = _lens_array(task_lens)
    T = len(lens)
    dev = data.device
    idt = idx_in.dtype if idx_in is not None else (idx_dtype or torch.int32)
    width = max(int(k), 1)
    vo = torch.zeros((T, width), dtype=torch.float32, device=dev)
    io = torch.zeros((T, width), dtype=idt, device=dev)
    cnt = torch.zeros(T, dtype=torch.int32, device=dev)
    bnd = torch.as_tensor(np.asarray(boundary, np.int32), device=dev).clone()
    kt = torch.as_tensor(np.asarray(kth, np.float32), device=dev).clone()
    check(load().radik_filter(_ptr(vo), _ptr(io), _idx_bytes(idt), _ptr(cnt), _ptr(bnd), _ptr(data),
                              _ptr(idx_in), _ptr(kt), lens.ctypes.data_as(ctypes.c_void_p), T, int(k),
                              int(withscale), int(largest), _stream(stream)))
    c = cnt.cpu().numpy()
    v, i = vo.cpu().numpy(), io.cpu().numpy()
    return [(v[t, :c[t]], i[t, :c[t]]) for t in range(T)], bnd.cpu().numpy()


class Server:
    """Request server over the C ABI (radik_server_*, include/radik.h):
    continuous batching of top-k requests on a pool of ``slots`` streams
    with device-resident workspaces, admission by memory (``mem_cap_bytes``
    covers the inputs and outputs of the requests in flight plus the pool)
    and latency statistics.  No counterpart in the reference, which serves
    one call at a time."""

    def __init__(self, slots: int = 4, mem_cap_bytes: int = 32 << 30, max_batch_rows: int = 4096, device=None):
        torch = _torch()
        from ._lib import ServerConfig
        dev = torch.cuda.current_device() if device is None else int(device)
        cfg = ServerConfig(int(slots), dev, int(mem_cap_bytes), int(max_batch_rows))
        h = ctypes.c_void_p()
        with torch.cuda.device(dev):
            check(load().radik_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._keep = {}  # ticket -> tensors that must outlive the request

    def submit(self, data, k: int, *, largest: bool = True, rev: bool = False, withscale: bool = False,
               val_out=None, idx_out=None, idx_dtype=None) -> int:
        """Queue ``data`` ((rows, row_len) CUDA Float32, row-major): the k best
        of every row, sorted ascending unless ``rev`` (ASCEND = !rev as in
        topk!).  Returns a ticket; outputs are (rows, k) tensors."""
        torch = _torch()
        _check_cuda(data, "data")
        _check_float32(data)
        if data.dim() == 1:
            data = data.view(1, -1)
        rows, row_len = data.shape
        it = idx_dtype or torch.int32
        if val_out is None:
            val_out = torch.empty((rows, k), dtype=torch.float32, device=data.device)
        if idx_out is None:
            idx_out = torch.empty((rows, k), dtype=it, device=data.device)
        flags = _flags(largest, not rev, withscale, False)
        t = ctypes.c_uint64()
        check(load().radik_server_submit(self._h, _ptr(data), rows, row_len, int(k), flags, _ptr(val_out),
                                         _ptr(idx_out), _idx_bytes(idx_out.dtype), ctypes.byref(t)))
        self._keep[t.value] = (data, val_out, idx_out)
        return t.value

    def wait(self, ticket: int, timeout_s: float | None = None):
        """Block until the request completes; returns its (values, indices)."""
        us = -1 if timeout_s is None else int(timeout_s * 1e6)
        rc = load().radik_server_wait(self._h, ctypes.c_uint64(ticket), us)
        if rc == 6:  # RADIK_ERR_TIMEOUT
            raise TimeoutError(f"request {ticket} not complete")
        keep = self._keep.pop(ticket, None)
        check(rc)
        return keep[1], keep[2]

    def stats(self) -> dict:
        from ._lib import ServerStats
        st = ServerStats()
        check(load().radik_server_get_stats(self._h, ctypes.byref(st)))
        return {n: getattr(st, n) for n, _ in ServerStats._fields_}

    def latencies(self) -> dict:
        """Submission-to-completion latency (us) of every request completed
        since the last reset_stats, by ticket."""
        L = load()
        n = ctypes.c_int64()
        check(L.radik_server_get_latencies(self._h, None, None, 0, ctypes.byref(n)))
        cap = int(n.value)
        tk = (ctypes.c_uint64 * max(cap, 1))()
        lat = (ctypes.c_double * max(cap, 1))()
        check(L.radik_server_get_latencies(self._h, tk, lat, cap, ctypes.byref(n)))
        return {int(tk[i]): float(lat[i]) for i in range(min(cap, int(n.value)))}

    def batches(self) -> list[dict]:
        """The launched batches completed since the last reset_stats: k,
        rows, longest row, elements, device time and host launch time (us)."""
        from ._lib import ServerBatch
        L = load()
        n = ctypes.c_int64()
        check(L.radik_server_get_batches(self._h, None, 0, ctypes.byref(n)))
        cap = int(n.value)
        arr = (ServerBatch * max(cap, 1))()
        check(L.radik_server_get_batches(self._h, arr, cap, ctypes.byref(n)))
        return [{f: getattr(arr[i], f) for f, _ in ServerBatch._fields_} for i in range(min(cap, int(n.value)))]

    def reset_stats(self) -> None:
        check(load().radik_server_reset_stats(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            load().radik_server_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
