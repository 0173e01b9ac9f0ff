"""The multi-GPU paths of radik.jl_b200/multi.py with the engine's own top-k,
on one GPU, against the oracle.

* Single-task split: a task is cut into G contiguous slices (the ranks'
  shares, multi.split_task); each slice's exact top k with global positions
  comes from the engine, and multi.merge_candidates -- the step that runs
  after the all-gather -- selects the task's result, again with the engine.
  G slices are computed one after another on this GPU, which is what G
  ranks compute side by side; no kernel waits for another.
* distributed_topk_single and distributed_topk_batch themselves, over a
  one-rank NCCL process group (the collective is a no-op copy), so their
  engine calls and index mapping run as in a real job.
Values must match the oracle bit for bit and indices exactly, ties included:
the merge orders candidates by global position, so ties at the k-th value
resolve to the lowest positions as on one device."""
from __future__ import annotations

import importlib
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _multi(radik):
    return importlib.import_module("radik_b200.multi")


def _data(rng, n):
    x = rng.standard_normal(n).astype(np.float32)
    x[::97] = 1.5   # ties around the k-th value
    x[5::1013] = -2.25
    return x


def _same(got, want):
    gv, gi = got
    ov, oi = want
    gv = gv.reshape(-1).cpu().numpy()
    gi = gi.reshape(-1).cpu().numpy().astype(np.int64)
    assert np.array_equal(gv.view(np.uint32), ov.reshape(-1).view(np.uint32))
    assert np.array_equal(gi, oi.reshape(-1).astype(np.int64))


@pytest.mark.parametrize("G", [2, 3, 8])
def test_split_task_merge_with_engine_equals_one_device(radik, oracle, torch_cuda, G):
    torch = torch_cuda
    multi = _multi(radik)
    rng = np.random.default_rng(40 + G)
    n = (1 << 20) + 12_345
    x = _data(rng, n)
    xd = torch.from_numpy(x).cuda()
    for k, largest, rev in [(1, True, False), (100, True, False), (1000, False, True), (4096, True, True)]:
        parts_v, parts_i = [], []
        for s0, s1 in multi.split_task(n, G):
            pos = torch.arange(s0 + 1, s1 + 1, dtype=torch.int64, device="cuda")
            lv, li = multi._engine_topk(xd[s0:s1], [s1 - s0], k, pos, largest, rev)
            parts_v.append(lv.reshape(-1)[:k])
            parts_i.append(li.reshape(-1)[:k].to(torch.int64))
        got = multi.merge_candidates(torch.cat(parts_v), torch.cat(parts_i), k, largest=largest, rev=rev,
                                     topk_fn=multi._engine_topk)
        _same(got, oracle.topk(x, [n], k, largest=largest, rev=rev))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_distributed_functions_on_a_one_rank_group(radik, oracle, torch_cuda):
    torch = torch_cuda
    import torch.distributed as dist
    multi = _multi(radik)
    rng = np.random.default_rng(77)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1)
    try:
        n = 300_001
        x = _data(rng, n)
        xd = torch.from_numpy(x).cuda()
        for k, largest, rev in [(64, True, False), (777, False, False)]:
            got = multi.distributed_topk_single(xd, 0, k, largest=largest, rev=rev)
            _same(got, oracle.topk(x, [n], k, largest=largest, rev=rev))
        # custom indices of the whole task
        ci = rng.permutation(n).astype(np.int64)
        v, i = multi.distributed_topk_single(xd, 0, 50, custom_indices=torch.from_numpy(ci).cuda())
        ov, oi = oracle.topk(x, [n], 50, indices=ci, idx_dtype=np.int64)
        _same((v, i), (ov, oi))

        lens = [3000, 5, 0, 70_000, 1, 12_345, 999, 40_000]
        xb = _data(rng, sum(lens))
        xbd = torch.from_numpy(xb).cuda()
        ov, oi = oracle.topk(xb, lens, 64)
        (t0, t1), parts = multi.distributed_topk_batch(xbd, lens, 64, gather=True)
        assert (t0, t1) == (0, len(lens))
        (_, res), = parts
        _same(res, (ov, oi))
        (t0, t1), (v, i) = multi.distributed_topk_batch(xbd, lens, 64, local=True)
        _same((v, i), (ov, oi))
    finally:
        dist.destroy_process_group()
