"""Parity at the benchmark workloads' full sizes: the three batch
configurations bench.py measures, at their real sizes and distributions,
through the C ABI, compared bit for bit with the oracle (values) and
exactly (indices).

* uniform batch: 1024 tasks x 65,536 U(0,1), k = 256, largest;
* adversarial single task: 2^28 elements (heavy ties, one crowded top
  bin), k = 4096, smallest, descending output;
* uneven batch: 4096 lognormal task lengths (about 2.5e8 elements), custom
  Int32 indices (a permutation), k = 64, largest.

The C oracle takes a few seconds on each.  Size-independent properties are
checked as well (sorted rows, values at their indices, the k-th value's rank
counts), so that a failure says which part broke."""
from __future__ import annotations

import pathlib
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _bench():
    sys.path.insert(0, str(ROOT))
    import bench
    return bench


def _run(radik, torch, x_np, lens, k, largest, rev, ind_np=None):
    dev = torch.device("cuda")
    x = torch.from_numpy(x_np).to(dev)
    T = len(lens)
    vo = torch.empty((T, k), dtype=torch.float32, device=dev)
    io = torch.empty((T, k), dtype=torch.int32, device=dev)
    ws = radik.RadiKWorkspace("cuda", max(lens), T)
    ind = None if ind_np is None else torch.from_numpy(ind_np).to(dev)
    radik.topk_radix_select_(vo, io, ws, x, ind, lens, k, largest, not rev, False, ind is not None)
    assert ws.error_bits() == 0
    ws.close()
    return x, vo, io


def _properties(torch, x, lens, vo, io, k, largest, rev, ind=None):
    """Rows sorted in the requested order; every value is the input at its
    index; exactly the k best by (value, lowest position) were taken."""
    T = len(lens)
    starts = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.int64)
    v = vo
    d = v[:, 1:] - v[:, :-1]
    ascend = not rev
    assert bool(((d >= 0) if ascend else (d <= 0)).all()), "rows not sorted"
    if ind is None:
        pos = io.to(torch.int64) - 1 + torch.from_numpy(starts).to(x.device)[:, None]
    else:
        inv = torch.empty_like(ind, dtype=torch.int64)
        inv[ind.to(torch.int64)] = torch.arange(ind.numel(), device=ind.device)
        pos = inv[io.to(torch.int64)]
    assert bool((x[pos] == v).all()), "values are not the input at their indices"
    # the k-th best value of each task and its rank counts
    kth = v.min(dim=1).values if largest else v.max(dim=1).values
    tid = torch.repeat_interleave(torch.arange(T, device=x.device), torch.tensor(lens, device=x.device))
    kk = kth[tid]
    better = (x > kk) if largest else (x < kk)
    n_better = torch.zeros(T, dtype=torch.int64, device=x.device).index_add_(0, tid, better.to(torch.int64))
    n_equal = torch.zeros(T, dtype=torch.int64, device=x.device).index_add_(0, tid, (x == kk).to(torch.int64))
    assert bool((n_better < k).all()) and bool((n_better + n_equal >= k).all()), "not the k best"


def _compare(oracle, v, i, ov, oi):
    assert np.array_equal(v.cpu().numpy().view(np.uint32), ov.view(np.uint32)), "values differ from the oracle"
    assert np.array_equal(i.cpu().numpy().astype(np.int64), oi.astype(np.int64)), "indices differ from the oracle"


def test_uniform_batch_full_size(oracle, radik, torch_cuda):
    bench = _bench()
    lens = bench.task_lens_of("uniform_batch")
    x_np = bench.make_input_np("uniform_batch", sum(lens))
    x, vo, io = _run(radik, torch_cuda, x_np, lens, 256, True, False)
    _properties(torch_cuda, x, lens, vo, io, 256, True, False)
    ov, oi = oracle.topk(x_np, lens, 256, largest=True, rev=False)
    _compare(oracle, vo, io, ov, oi)


def test_adversarial_single_full_size(oracle, radik, torch_cuda):
    bench = _bench()
    n = 1 << 28
    x_np = bench.make_input_np("adversarial_single", n)
    x, vo, io = _run(radik, torch_cuda, x_np, [n], 4096, False, True)
    _properties(torch_cuda, x, [n], vo, io, 4096, False, True)
    del x
    ov, oi = oracle.topk(x_np, [n], 4096, largest=False, rev=True)
    _compare(oracle, vo, io, ov, oi)


def test_uneven_batch_full_size(oracle, radik, torch_cuda):
    bench = _bench()
    lens = bench.task_lens_of("uneven_batch")
    N = sum(lens)
    x_np = bench.make_input_np("uneven_batch", N)
    ind_np = np.random.default_rng(5).permutation(N).astype(np.int32)
    x, vo, io = _run(radik, torch_cuda, x_np, lens, 64, True, False, ind_np)
    _properties(torch_cuda, x, lens, vo, io, 64, True, False, torch_cuda.from_numpy(ind_np).cuda())
    del x
    ov, oi = oracle.topk(x_np, lens, 64, largest=True, rev=False, indices=ind_np, idx_dtype=np.int32)
    _compare(oracle, vo, io, ov, oi)


def test_adversarial_single_full_size_largest(oracle, radik, torch_cuda):
    """The adversarial task's stress variant: the k largest (ascending),
    where 40 % of the elements crowd one narrow band just above 1.0."""
    bench = _bench()
    n = 1 << 28
    x_np = bench.make_input_np("adversarial_single", n)
    x, vo, io = _run(radik, torch_cuda, x_np, [n], 4096, True, False)
    _properties(torch_cuda, x, [n], vo, io, 4096, True, False)
    del x
    ov, oi = oracle.topk(x_np, [n], 4096, largest=True, rev=False)
    _compare(oracle, vo, io, ov, oi)
