"""Multi-GPU top-k over torch.distributed (one process per GPU).

Tasks are independent, so a batch shards across ranks with no collective on
the data path: every rank takes a contiguous range of tasks (balanced by
element count), runs the engine on them and keeps its own rows of the
output.  A single task too large for one GPU is split into contiguous
slices: every rank computes the exact top k of its slice with global
positions, one all-gather moves the G * k (value, position) pairs, and a
final top k over those pairs -- ordered by global position, so that ties at
the k-th value resolve to the lowest positions exactly as on one device --
gives the task's result.

The per-rank computation is a function ``topk_fn(values, task_lens, k,
indices, largest, rev) -> (values[T, k], indices[T, k])`` with the
semantics of ``topk`` (indices 1-based positions inside each task, or the
given custom indices; padding 0 / -1): the engine on CUDA tensors by
default; the tests pass the CPU restatement.
"""
from __future__ import annotations

import importlib
import sys
from typing import Callable, Sequence

import numpy as np


def shard_tasks(task_lens: Sequence[int], world: int) -> list[tuple[int, int]]:
    """Contiguous task ranges [t0, t1) per rank, cut where the running
    element count crosses r * total / world."""
    lens = np.asarray(task_lens, dtype=np.int64)
    total = int(lens.sum())
    bounds = [0]
    csum = np.cumsum(lens)
    for r in range(1, world):
        target = total * r / world
        t = int(np.searchsorted(csum, target, side="left")) + 1 if total else 0
        t = min(max(t, bounds[-1]), len(lens))
        bounds.append(t)
    bounds.append(len(lens))
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def split_task(n: int, world: int) -> list[tuple[int, int]]:
    """Contiguous slices [s0, s1) of one task of n elements, one per rank,
    boundaries on multiples of 4 elements (16-byte aligned loads)."""
    out, start = [], 0
    for r in range(world):
        stop = n if r == world - 1 else min(n, ((n * (r + 1) // world) + 3) // 4 * 4)
        out.append((start, max(start, stop)))
        start = max(start, stop)
    return out


def _engine():
    """The engine package this module belongs to (loaded as its submodule)."""
    pkg = __name__.rpartition(".")[0]
    if not pkg or pkg not in sys.modules:
        raise RuntimeError("multi.py must be imported as a submodule of the engine package "
                           "(e.g. radik_b200.multi) to run the engine's top-k")
    return importlib.import_module(pkg)


def _engine_topk(values, task_lens, k, indices, largest, rev):
    return _engine().topk(values, list(task_lens), k, indices=indices, largest=largest, rev=rev)


def _world_rank(group):
    """(world size, rank); an uninitialised process group is one rank."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def merge_candidates(values, positions, k: int, *, largest: bool, rev: bool, topk_fn: Callable):
    """Exact top k of one task from gathered candidates: `values` and
    `positions` (global 1-based positions, -1 for padding) of equal length.
    Candidates are put in position order first, so the final selection's
    tie rule (lowest position in its input) is the task's own."""
    import torch
    keep = positions >= 0
    v = values[keep]
    p = positions[keep]
    order = torch.argsort(p, stable=True)
    v = v[order].contiguous()
    p = p[order].contiguous()
    return topk_fn(v, [int(v.numel())], k, p, largest, rev)


def distributed_topk_single(local_values, start: int, k: int, *, largest: bool = True, rev: bool = False,
                            topk_fn: Callable | None = None, group=None, custom_indices=None):
    """Top k of one task split across ranks.  `local_values` is this rank's
    contiguous slice, beginning at position `start` (0-based) of the task.
    Every rank returns the task's (values[k], indices[k]); indices are the
    task's 1-based positions, or custom_indices[position - 1] when a custom
    index array of the whole task is given."""
    import torch
    import torch.distributed as dist
    fn = topk_fn or _engine_topk
    n = int(local_values.numel())
    pos = torch.arange(start + 1, start + n + 1, dtype=torch.int64, device=local_values.device)
    lv, li = fn(local_values, [n], k, pos, largest, rev)
    lv = lv.reshape(-1)[:k].contiguous()
    li = li.reshape(-1)[:k].to(torch.int64).contiguous()
    world, _ = _world_rank(group)
    if world == 1:
        gv, gi = [lv], [li]
    else:
        gv = [torch.empty_like(lv) for _ in range(world)]
        gi = [torch.empty_like(li) for _ in range(world)]
        dist.all_gather(gv, lv, group=group)
        dist.all_gather(gi, li, group=group)
    v, i = merge_candidates(torch.cat(gv), torch.cat(gi), k, largest=largest, rev=rev, topk_fn=fn)
    v = v.reshape(-1)
    i = i.reshape(-1).to(torch.int64)
    if custom_indices is not None:
        ci = torch.as_tensor(custom_indices, device=i.device)
        i = torch.where(i > 0, ci[(i - 1).clamp(min=0)].to(torch.int64), i)
    return v, i


def local_shard(task_lens: Sequence[int], world: int, rank: int) -> tuple[int, int, int, int]:
    """This rank's task range [t0, t1) of shard_tasks and the element range
    [lo, hi) those tasks occupy in the concatenated batch."""
    t0, t1 = shard_tasks(task_lens, world)[rank]
    offs = np.concatenate([[0], np.cumsum(np.asarray(task_lens, dtype=np.int64))])
    return t0, t1, int(offs[t0]), int(offs[t1])


def distributed_topk_batch(values, task_lens: Sequence[int], k: int, *, largest: bool = True, rev: bool = False,
                           topk_fn: Callable | None = None, group=None, gather: bool = False,
                           local: bool = False):
    """Batched top k with the tasks sharded across ranks (no collective on
    the data path).  `values` holds the whole concatenated batch on every
    rank, or -- with local=True -- only this rank's tasks (its local_shard,
    from offset 0).  Returns this rank's task range and its rows; with
    gather=True every rank also receives all rows (one all_gather_object,
    for checking)."""
    import torch.distributed as dist
    fn = topk_fn or _engine_topk
    world, rank = _world_rank(group)
    t0, t1, lo, hi = local_shard(task_lens, world, rank)
    if local:
        lo, hi = 0, hi - lo
    lens = [int(x) for x in task_lens[t0:t1]]
    if t1 > t0:
        v, i = fn(values[lo:hi], lens, k, None, largest, rev)
    else:
        v, i = None, None
    if not gather:
        return (t0, t1), (v, i)
    if world == 1:
        return (t0, t1), [((t0, t1), None if v is None else (v.cpu(), i.cpu()))]
    parts = [None] * world
    dist.all_gather_object(parts, ((t0, t1), None if v is None else (v.cpu(), i.cpu())), group=group)
    return (t0, t1), parts
