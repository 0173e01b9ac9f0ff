"""Multi-rank paths (radik.jl_b200/multi.py) as world-size-2 gloo process
groups on the CPU: the per-rank top-k is the CPU restatement (oracle), so
these tests check the distributed logic -- task sharding, the single-task
split, the all-gather and the final merge with its tie order -- against the
single-process result."""
from __future__ import annotations

import importlib.util
import os
import pathlib
import socket
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _load_multi():
    """multi.py as the engine package's submodule, the way users import it
    (its engine top-k resolves through the package)."""
    if "radik_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location("radik_b200", ROOT / "radik.jl_b200" / "__init__.py",
                                                      submodule_search_locations=[str(ROOT / "radik.jl_b200")])
        pkg = importlib.util.module_from_spec(spec)
        sys.modules["radik_b200"] = pkg
        spec.loader.exec_module(pkg)
    return importlib.import_module("radik_b200.multi")


def _load_oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    return oracle


def _oracle_fn(values, task_lens, k, indices, largest, rev):
    oracle = _load_oracle()
    v = values.cpu().numpy().astype(np.float32)
    idx = None if indices is None else indices.cpu().numpy().astype(np.int64)
    ov, oi = oracle.topk(v, list(task_lens), k, largest=largest, rev=rev, indices=idx,
                         idx_dtype=np.int64 if idx is not None else np.int32)
    return torch.from_numpy(np.ascontiguousarray(ov)), torch.from_numpy(np.ascontiguousarray(oi).astype(np.int64))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, case, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        multi = _load_multi()
        kind, seed, n_or_lens, k, largest, rev = case
        rng = np.random.default_rng(seed)
        if kind == "single":
            n = n_or_lens
            x = rng.standard_normal(n).astype(np.float32)
            x[::97] = 1.5  # ties at the boundary of the k best
            s0, s1 = multi.split_task(n, world)[rank]
            v, i = multi.distributed_topk_single(torch.from_numpy(x[s0:s1].copy()), s0, k, largest=largest, rev=rev,
                                                 topk_fn=_oracle_fn)
            q.put((rank, v.numpy(), i.numpy()))
        else:
            lens = n_or_lens
            x = rng.standard_normal(sum(lens)).astype(np.float32)
            _, parts = multi.distributed_topk_batch(torch.from_numpy(x), lens, k, largest=largest, rev=rev,
                                                   topk_fn=_oracle_fn, gather=True)
            # numpy, not tensors: the queue must not hold shared-memory handles of an exiting process
            parts = [(rng_, None if res is None else (res[0].numpy(), res[1].numpy())) for rng_, res in parts]
            q.put((rank, parts, None))
    finally:
        dist.destroy_process_group()


def _run(case, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(out, key=lambda t: t[0])


def test_shard_and_split_geometry():
    multi = _load_multi()
    lens = [5, 100, 0, 7, 3000, 1, 1]
    for world in (1, 2, 3, 8):
        ranges = multi.shard_tasks(lens, world)
        assert ranges[0][0] == 0 and ranges[-1][1] == len(lens)
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        sl = multi.split_task(10_003, world)
        assert sl[0][0] == 0 and sl[-1][1] == 10_003
        assert all(a[1] == b[0] for a, b in zip(sl, sl[1:]))
        assert all(s[0] % 4 == 0 for s in sl)
        for r in range(world):
            t0, t1, lo, hi = multi.local_shard(lens, world, r)
            assert (t0, t1) == ranges[r] and lo == sum(lens[:t0]) and hi == sum(lens[:t1])


def test_engine_topk_needs_the_package():
    """Loaded on its own, outside the package, the module refuses to guess
    where the engine is."""
    spec = importlib.util.spec_from_file_location("lone_multi", ROOT / "radik.jl_b200" / "multi.py")
    lone = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(lone)
    with pytest.raises(RuntimeError, match="submodule of the engine package"):
        lone._engine_topk(torch.zeros(4), [4], 1, None, True, False)
    assert _load_multi()._engine().__name__ == "radik_b200"


@pytest.mark.parametrize("k,largest,rev", [(1, True, False), (100, True, False), (257, False, True)])
def test_single_task_split_over_two_ranks_equals_one_device(oracle, k, largest, rev):
    n = 200_003
    case = ("single", k, n, k, largest, rev)
    out = _run(case)
    rng = np.random.default_rng(k)
    x = rng.standard_normal(n).astype(np.float32)
    x[::97] = 1.5
    ov, oi = oracle.topk(x, [n], k, largest=largest, rev=rev)
    for _, v, i in out:  # every rank holds the task's result
        assert np.array_equal(v.view(np.uint32), ov[0].view(np.uint32))
        assert np.array_equal(i.astype(np.int64), oi[0].astype(np.int64))


def test_task_sharding_over_two_ranks_equals_one_device(oracle):
    lens = [3000, 5, 0, 70_000, 1, 12_345, 999, 40_000]
    k = 64
    out = _run(("batch", 3, lens, k, True, False))
    rng = np.random.default_rng(3)
    x = rng.standard_normal(sum(lens)).astype(np.float32)
    ov, oi = oracle.topk(x, lens, k)
    parts = out[0][1]
    rows_v, rows_i = [], []
    for (t0, t1), res in parts:
        if res is not None:
            rows_v.append(res[0])
            rows_i.append(res[1])
    gv = np.concatenate(rows_v)
    gi = np.concatenate(rows_i)
    assert np.array_equal(gv.view(np.uint32), ov.view(np.uint32))
    assert np.array_equal(gi.astype(np.int64), oi.astype(np.int64))
