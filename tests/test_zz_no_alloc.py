"""radik_topk_noalloc (static device scratch, no workspace) against the
workspace entry point radik_topk_radix_select and against the oracle on the
same inputs.

The comparison tolerance is zero: the selection is exact, so values must
agree bit for bit and indices exactly.  Each case makes two calls in a row
through the allocation-free entry point, so state left in the static scratch
by one call must not leak into the next.  That a call allocates nothing is
checked with the library's own count of its CUDA allocations
(radik_alloc_count, which sees a cudaMalloc inside the library that torch's
allocator counters cannot) and with the device's free memory
(cudaMemGetInfo) before and after it.  This file is collected last so that
it runs both alone and after every other GPU test."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VALUE_ATOL = 0.0  # exact selection: no floating-point tolerance
SCRATCH_BYTES = 8 << 20


def _outputs(torch, T, k, idx_dtype):
    dev = torch.device("cuda")
    return (torch.full((T, k), 7.0, dtype=torch.float32, device=dev),
            torch.full((T, k), 7, dtype=idx_dtype, device=dev))


def _with_workspace(radik, torch, x, lens, k, idx, largest, ascend, idx_dtype):
    vo, io = _outputs(torch, len(lens), k, idx_dtype)
    ws = radik.RadiKWorkspace("cuda", max(lens), len(lens), idx_dtype)
    radik.topk_radix_select_(vo, io, ws, x, idx, lens, k, largest, ascend, False, idx is not None)
    ws.close()
    return vo, io


def _alloc_count(radik):
    n = ctypes.c_uint64()
    assert radik._lib.load().radik_alloc_count(ctypes.byref(n)) == 0
    return n.value


def _no_alloc(radik, torch, x, lens, k, idx, largest, ascend, idx_dtype):
    vo, io = _outputs(torch, len(lens), k, idx_dtype)
    torch.cuda.synchronize()
    count0 = _alloc_count(radik)
    free0 = torch.cuda.mem_get_info()[0]
    torch0 = (torch.cuda.memory_allocated(), torch.cuda.memory_reserved())
    radik.topk_radix_select_noalloc_(vo, io, x, idx, lens, k, largest, ascend, False, idx is not None)
    assert _alloc_count(radik) == count0, "the library allocated during the call"
    assert torch.cuda.mem_get_info()[0] == free0, "device free memory changed during the call"
    assert (torch.cuda.memory_allocated(), torch.cuda.memory_reserved()) == torch0
    return vo, io


def _assert_same(a, b):
    av, ai = (t.cpu().numpy() for t in a)
    bv, bi = (t.cpu().numpy() for t in b)
    assert np.allclose(av, bv, rtol=0.0, atol=VALUE_ATOL, equal_nan=True)
    assert np.array_equal(av.view(np.uint32), bv.view(np.uint32))
    assert np.array_equal(ai, bi)


def _assert_oracle(oracle, got, xs, lens, k, largest, ascend, ind):
    ov, oi = oracle.topk(xs, list(lens), k, largest=largest, rev=not ascend, indices=ind)
    gv, gi = (t.cpu().numpy() for t in got)
    assert np.array_equal(gv.view(np.uint32), ov.reshape(gv.shape).view(np.uint32))
    assert np.array_equal(gi.astype(np.int64), oi.reshape(gi.shape).astype(np.int64))


def _case(radik, oracle, torch, rng, lens, k, *, largest, ascend, custom_idx, idx_dtype):
    N = int(sum(lens))
    xs = rng.standard_normal(N).astype(np.float32)
    x = torch.from_numpy(xs).cuda()
    idx, ind = None, None
    if custom_idx:
        ind = rng.permutation(N).astype(np.int64 if idx_dtype == torch.int64 else np.int32)
        idx = torch.from_numpy(ind).cuda()
    ref = _with_workspace(radik, torch, x, lens, k, idx, largest, ascend, idx_dtype)
    # a first call warms the kernels up (their code may load lazily on first use)
    _no_alloc_unchecked(radik, torch, x, lens, k, idx, largest, ascend, idx_dtype)
    got = _no_alloc(radik, torch, x, lens, k, idx, largest, ascend, idx_dtype)
    _assert_same(got, ref)
    _assert_oracle(oracle, got, xs, lens, k, largest, ascend, ind)


def _no_alloc_unchecked(radik, torch, x, lens, k, idx, largest, ascend, idx_dtype):
    vo, io = _outputs(torch, len(lens), k, idx_dtype)
    radik.topk_radix_select_noalloc_(vo, io, x, idx, lens, k, largest, ascend, False, idx is not None)
    return vo, io


def test_no_alloc_matches_workspace_entry_two_calls_in_a_row(radik, oracle, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(101)
    lens = [int(v) for v in np.clip(rng.lognormal(np.log(4000), 1.2, size=40), 1, 300_000)]
    lens[5] = 0
    # first call: uneven batch, custom Int64 indices, largest, ascending
    _case(radik, oracle, torch, rng, lens, 64, largest=True, ascend=True, custom_idx=True, idx_dtype=torch.int64)
    # second call, straight after: another shape, automatic Int32 indices
    _case(radik, oracle, torch, rng, [70_000, 3, 12_345], 500, largest=False, ascend=False, custom_idx=False,
          idx_dtype=torch.int32)


def test_no_alloc_multi_segment_two_calls_in_a_row(radik, oracle, torch_cuda, monkeypatch):
    """Tasks split across blocks use the candidate regions, the sampled
    threshold and the retry launch, all inside the static scratch."""
    monkeypatch.setenv("RADIK_SEG", "16384")
    torch = torch_cuda
    rng = np.random.default_rng(103)
    for _ in range(2):
        _case(radik, oracle, torch, rng, [1 << 20], 256, largest=True, ascend=True, custom_idx=False,
              idx_dtype=torch.int32)
    # planted large values where the sampler reads force the retry launch
    n = 1 << 20
    xs = rng.random(n, dtype=np.float32)
    for m in range(64):
        xs[m * 16384:m * 16384 + 512] = 100.0 + rng.random(512, dtype=np.float32)
    x = torch.from_numpy(xs).cuda()
    for _ in range(2):
        ref = _with_workspace(radik, torch, x, [n], 1000, None, True, True, torch.int32)
        got = _no_alloc(radik, torch, x, [n], 1000, None, True, True, torch.int32)
        _assert_same(got, ref)
        _assert_oracle(oracle, got, xs, [n], 1000, True, True, None)


def test_no_alloc_rejects_oversize_and_recovers(radik, oracle, torch_cuda):
    torch = torch_cuda
    x = torch.rand(300_000, device="cuda")
    vo, io = _outputs(torch, 1, 4097, torch.int32)
    with pytest.raises(radik.RadiKError, match="k <= 4096"):
        radik.topk_radix_select_noalloc_(vo, io, x, None, [300_000], 4097)
    # 300k one-element tasks: per-task state and descriptors exceed 8 MiB
    lens = [1] * 300_000
    vo, io = _outputs(torch, len(lens), 1, torch.int32)
    with pytest.raises(radik.RadiKError, match="bytes of scratch") as ei:
        radik.topk_radix_select_noalloc_(vo, io, x, None, lens, 1)
    assert ei.value.status == 3
    # asynchronous and multi-pass requests are refused
    L = radik._lib.load()
    lens_np = np.array([300_000], dtype=np.int64)
    for bad in (radik._lib.RADIK_ASYNC, radik._lib.RADIK_PLAIN):
        rc = L.radik_topk_noalloc(ctypes.c_void_p(vo.data_ptr()), ctypes.c_void_p(io.data_ptr()), 4,
                                  ctypes.c_void_p(x.data_ptr()), None,
                                  lens_np.ctypes.data_as(ctypes.c_void_p), 1, 1,
                                  radik._lib.RADIK_LARGEST | bad, None)
        assert rc == 1
    # a valid call straight after the refusals is still exact
    rng = np.random.default_rng(107)
    _case(radik, oracle, torch, rng, [300_000, 5], 100, largest=True, ascend=True, custom_idx=False,
          idx_dtype=torch.int32)
