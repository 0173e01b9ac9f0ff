"""GPU parity tests: the engine (through the C ABI) against the oracle.

Values must match bit for bit and, because both sides resolve ties at the k-th
value by lowest position, indices must match exactly too.  A relaxed check in
the reference's own terms (test/test_algorithm.jl:31-36: indices valid, unique
and addressing equal values) is applied as well."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import plain_topk

pytestmark = pytest.mark.gpu


def _run(radik, torch, data_np, lens, k, *, largest=True, rev=False, withscale=False, indices=None,
         plain=False, idx_dtype=None, offset=0):
    dev = torch.device("cuda")
    buf = torch.empty(len(data_np) + offset, dtype=torch.float32, device=dev)
    buf[offset:] = torch.from_numpy(np.ascontiguousarray(data_np))
    data = buf[offset:]
    T = len(lens)
    it = torch.int32 if (indices is None and idx_dtype is None) else (
        idx_dtype or torch.from_numpy(indices).dtype)
    vo = torch.full((T, k), 7.0, dtype=torch.float32, device=dev)
    io = torch.full((T, k), 7, dtype=it, device=dev)
    ws = radik.RadiKWorkspace("cuda", max(lens) if T else 0, T)
    idx_t = None if indices is None else torch.from_numpy(indices).to(dev)
    radik.topk_radix_select_(vo, io, ws, data, idx_t, lens, k, largest, not rev, withscale,
                             idx_t is not None, plain=plain)
    assert ws.error_bits() == 0
    ws.close()
    return vo.cpu().numpy(), io.cpu().numpy()


def _compare(oracle, radik, torch, data, lens, k, **kw):
    plain = kw.pop("plain", False)
    offset = kw.pop("offset", 0)
    gv, gi = _run(radik, torch, data, lens, k, plain=plain, offset=offset, **kw)
    ov, oi = oracle.topk(data, lens, k, largest=kw.get("largest", True), rev=kw.get("rev", False),
                         withscale=kw.get("withscale", False), indices=kw.get("indices"),
                         idx_dtype=np.int64 if kw.get("idx_dtype") is torch.int64 else np.int32)
    assert np.array_equal(gv.view(np.uint32), ov.view(np.uint32)), "values differ from the oracle"
    assert np.array_equal(gi.astype(np.int64), oi.astype(np.int64)), "indices differ from the oracle"
    return gv, gi


@pytest.mark.parametrize("plain", [False, True])
@pytest.mark.parametrize("n,k", [(1, 1), (7, 3), (100, 100), (100, 1), (4097, 16), (65536, 256),
                                 (65536, 4096), (1 << 20, 100), (300_001, 1000)])
@pytest.mark.parametrize("largest,rev", [(True, False), (False, True), (True, True), (False, False)])
def test_single_task_matches_oracle(oracle, radik, torch_cuda, plain, n, k, largest, rev):
    rng = np.random.default_rng(n * 31 + k + 2 * largest + rev)
    x = rng.random(n, dtype=np.float32)
    _compare(oracle, radik, torch_cuda, x, [n], k, largest=largest, rev=rev, plain=plain)


@pytest.mark.parametrize("plain", [False, True])
def test_uneven_batch_custom_indices(oracle, radik, torch_cuda, plain):
    rng = np.random.default_rng(5)
    lens = [int(v) for v in np.clip(rng.lognormal(np.log(3000), 1.5, size=96), 1, 400_000)]
    lens[3] = 0
    lens[10] = 5
    N = sum(lens)
    x = rng.standard_normal(N).astype(np.float32)
    for dt, npdt in ((torch_cuda.int32, np.int32), (torch_cuda.int64, np.int64)):
        ind = rng.permutation(N).astype(npdt)
        _compare(oracle, radik, torch_cuda, x, lens, 64, indices=ind, plain=plain)
    _compare(oracle, radik, torch_cuda, x, lens, 64, idx_dtype=torch_cuda.int64, plain=plain)


@pytest.mark.parametrize("k", [1, 37, 256, 4096])
def test_multi_segment_tasks(oracle, radik, torch_cuda, k, monkeypatch):
    """Force segmentation so several CTAs share one task (global threshold,
    candidate slots, last-segment merge)."""
    monkeypatch.setenv("RADIK_SEG", "16384")
    rng = np.random.default_rng(k)
    for n in (50_000, 1 << 20):
        x = rng.standard_normal(n).astype(np.float32)
        _compare(oracle, radik, torch_cuda, x, [n], k)
        _compare(oracle, radik, torch_cuda, x, [n], k, largest=False, rev=True)
    # ascending data: every element beats the running threshold
    x = np.arange(1 << 18, dtype=np.float32)
    _compare(oracle, radik, torch_cuda, x, [len(x)], k)
    _compare(oracle, radik, torch_cuda, x[::-1].copy(), [len(x)], k)
    # batch of long tasks
    lens = [70_000, 10, 200_000, 16_384, 16_385]
    x = rng.random(sum(lens), dtype=np.float32)
    _compare(oracle, radik, torch_cuda, x, lens, k)


@pytest.mark.parametrize("plain", [False, True])
def test_special_values_and_ties(oracle, radik, torch_cuda, plain):
    rng = np.random.default_rng(11)
    specials = np.array([0.0, -0.0, np.nan, np.inf, -np.inf, 1.0, -1.0,
                         np.finfo(np.float32).tiny, np.finfo(np.float32).max], np.float32)
    x = rng.choice(specials, size=20_000).astype(np.float32)
    for k in (1, 5, 100, 3000):
        for largest, rev in ((True, False), (False, True), (True, True)):
            _compare(oracle, radik, torch_cuda, x, [len(x)], k, largest=largest, rev=rev, plain=plain)
    # heavy ties: 5 distinct values over many tasks, all-equal task
    lens = [1000, 1, 64, 65, 5000, 2]
    y = rng.integers(0, 5, size=sum(lens)).astype(np.float32)
    y[1066:1066 + 5000] = 3.0
    for k in (1, 64, 500):
        _compare(oracle, radik, torch_cuda, y, lens, k, plain=plain)
        _compare(oracle, radik, torch_cuda, y, lens, k, largest=False, plain=plain)


@pytest.mark.parametrize("plain", [False, True])
def test_withscale(oracle, radik, torch_cuda, plain):
    rng = np.random.default_rng(13)
    lens = [5000, 1, 0, 30_000]
    x = (1.0 + rng.random(sum(lens), dtype=np.float32) * np.float32(2 ** -10)).astype(np.float32)
    x[7] = np.nan
    x[5001] = np.inf  # scaler of task 1 is Inf -> 0
    for largest in (True, False):
        _compare(oracle, radik, torch_cuda, x, lens, 50, largest=largest, withscale=True, plain=plain)


@pytest.mark.parametrize("plain", [False, True])
@pytest.mark.parametrize("k", [4097, 8192])
def test_large_k_radix_sort(oracle, radik, torch_cuda, plain, k):
    rng = np.random.default_rng(k)
    lens = [100_000, 5000, 20_000]
    x = rng.standard_normal(sum(lens)).astype(np.float32)
    _compare(oracle, radik, torch_cuda, x, lens, k, plain=plain)
    _compare(oracle, radik, torch_cuda, x, lens, k, largest=False, rev=True, plain=plain)


def test_k_beyond_shared_memory_uses_multipass(oracle, radik, torch_cuda):
    rng = np.random.default_rng(21)
    x = rng.random(200_000, dtype=np.float32)
    _compare(oracle, radik, torch_cuda, x, [len(x)], 40_000)


def test_unaligned_input_pointer(oracle, radik, torch_cuda):
    rng = np.random.default_rng(23)
    x = rng.random(100_003, dtype=np.float32)
    for off in (1, 2, 3):
        _compare(oracle, radik, torch_cuda, x, [50_001, 50_002], 33, offset=off)


def test_reference_relaxed_checks(radik, torch_cuda):
    """test/test_algorithm.jl:6-40 in its own terms."""
    rng = np.random.default_rng(42)
    n = 1 << 14
    for k in (16, 32, 64, 128, 256, 512, 1024, 2048, 4096):
        for largest in (True, False):
            for rev in (True, False):
                x = rng.random(n, dtype=np.float32)
                v, i = radik.topk(torch_cuda.from_numpy(x).cuda(), k, largest=largest, rev=rev)
                v, i = v.cpu().numpy(), i.cpu().numpy().astype(np.int64)
                part = np.sort(x)[::-1][:k] if largest else np.sort(x)[:k]
                exp = np.sort(part)[::-1] if rev else np.sort(part)
                assert np.array_equal(v, exp)
                assert np.all((1 <= i) & (i <= n)) and len(np.unique(i)) == k
                assert np.array_equal(x[i - 1], v)


def test_plain_numpy_crosscheck(radik, torch_cuda):
    rng = np.random.default_rng(3)
    lens = [3000, 0, 17, 100_000]
    x = rng.standard_normal(sum(lens)).astype(np.float32)
    gv, gi = _run(radik, torch_cuda, x, lens, 20, largest=False, rev=True)
    pv, pi = plain_topk(x, lens, 20, largest=False, rev=True)
    assert np.array_equal(gv.view(np.uint32), pv.view(np.uint32))
    assert np.array_equal(gi.astype(np.int64), pi.astype(np.int64))


def test_deterministic_alone_and_in_batch(radik, torch_cuda):
    """A task gives the same result alone and inside a batch, and repeated
    calls give identical bits."""
    rng = np.random.default_rng(9)
    lens = [40_000, 3, 70_000, 12_345]
    x = rng.integers(0, 50, size=sum(lens)).astype(np.float32)  # many ties
    bv, bi = _run(radik, torch_cuda, x, lens, 100)
    bv2, bi2 = _run(radik, torch_cuda, x, lens, 100)
    assert np.array_equal(bv, bv2) and np.array_equal(bi, bi2)
    off = 0
    for t, n in enumerate(lens):
        av, ai = _run(radik, torch_cuda, x[off:off + n], [n], 100)
        assert np.array_equal(av[0].view(np.uint32), bv[t].view(np.uint32))
        assert np.array_equal(ai[0], bi[t])
        off += n


def test_sampled_threshold_retry(oracle, radik, torch_cuda, monkeypatch):
    """Large values planted exactly where the multi-segment sampler reads
    (64 chunks of 512 at multiples of 16384 for n = 2^20 with 16384-element
    segments) make the seeded threshold too high; the retry launch must still
    return the exact answer."""
    monkeypatch.setenv("RADIK_SEG", "16384")
    n = 1 << 20
    rng = np.random.default_rng(31)
    x = rng.random(n, dtype=np.float32)
    for m in range(64):
        x[m * 16384:m * 16384 + 512] = 100.0 + rng.random(512, dtype=np.float32)
    for k in (256, 1000):
        _compare(oracle, radik, torch_cuda, x, [n], k)
        _compare(oracle, radik, torch_cuda, x, [n], k, largest=False)


def test_in_block_sample_redo(oracle, radik, torch_cuda):
    """Large values planted where the in-block sampler of a single-segment
    task reads (16 chunks of 64 at multiples of len/16) force the redo path."""
    n = 1 << 16
    rng = np.random.default_rng(37)
    x = rng.random(n, dtype=np.float32)
    for c in range(16):
        x[c * (n // 16):c * (n // 16) + 64] = 50.0 + rng.random(64, dtype=np.float32)
    lens = [n, n]
    data = np.concatenate([x, x[::-1].copy()])
    for k in (64, 256, 1024):
        _compare(oracle, radik, torch_cuda, data, lens, k)


KERNEL_FORMS = [
    {"RADIK_WS": "0"},
    {"RADIK_WS": "1", "RADIK_WST": "256", "RADIK_WSJ": "8", "RADIK_WSS": "16"},
    {"RADIK_WS": "1", "RADIK_WST": "256", "RADIK_WSJ": "4", "RADIK_WSS": "24"},
    {"RADIK_WS": "1", "RADIK_WST": "128", "RADIK_WSJ": "8", "RADIK_WSS": "8"},
    {"RADIK_WS": "1", "RADIK_WST": "128", "RADIK_WSJ": "8", "RADIK_WSS": "12", "RADIK_WS_SAMPLE": "4096"},
    {"RADIK_WS": "1", "RADIK_WST": "128", "RADIK_WSJ": "8", "RADIK_WSS": "8", "RADIK_DEFER": "1"},
    {"RADIK_WS": "1", "RADIK_WST": "64", "RADIK_WSJ": "8", "RADIK_WSS": "4"},
]


@pytest.mark.parametrize("form", KERNEL_FORMS, ids=["barrier", "ws-256-j8", "ws-256-j4", "ws-128-s8", "ws-128-s12",
                                                    "ws-128-s8-defer", "ws-64-s4-narrow"])
def test_many_items_per_block(oracle, radik, torch_cuda, monkeypatch, form):
    """A grid of 2-3 blocks works through every batch, so each block takes
    many work items in a row: ring stages, phases and item slots carry over
    from one item to the next, and a redo or a shrink in one item must not
    disturb the next."""
    for kk, vv in form.items():
        monkeypatch.setenv(kk, vv)
    monkeypatch.setenv("RADIK_GRID", "3")
    rng = np.random.default_rng(77)
    # sampled single-segment tasks (length >= 16384), several k
    lens = [65536] * 12 + [20000, 16384, 40000, 3, 0, 70001]
    x = rng.random(sum(lens), dtype=np.float32)
    for k in (1, 64, 256, 1000):
        _compare(oracle, radik, torch_cuda, x, lens, k)
    _compare(oracle, radik, torch_cuda, x, lens, 100, largest=False, rev=True)
    # 128 large values planted in sampled groups (32 chunks of 64 at multiples
    # of 2048 for length 65536): the sampled threshold passes only those, fewer
    # than k, so every other item takes the redo path
    y = rng.random(65536 * 8, dtype=np.float32)
    for t in range(0, 8, 2):
        for c in range(32):
            for off in (0, 4, 8, 12):
                y[t * 65536 + c * 2048 + off] = 10.0 + rng.random(dtype=np.float32)
    _compare(oracle, radik, torch_cuda, y, [65536] * 8, 256)
    # uneven batch with custom indices
    ulen = [int(v) for v in np.clip(rng.lognormal(np.log(5000), 1.3, size=60), 1, 200_000)]
    z = rng.standard_normal(sum(ulen)).astype(np.float32)
    ind = rng.permutation(sum(ulen)).astype(np.int32)
    _compare(oracle, radik, torch_cuda, z, ulen, 64, indices=ind)
    # multi-segment tasks (candidate regions, global thresholds, sampling)
    monkeypatch.setenv("RADIK_SEG", "16384")
    monkeypatch.setenv("RADIK_GRID", "2")
    w = rng.standard_normal(1 << 20).astype(np.float32)
    for k in (16, 256):
        _compare(oracle, radik, torch_cuda, w, [1 << 20], k)
        _compare(oracle, radik, torch_cuda, w, [300_000, 1 << 19, 5], k, largest=False)


@pytest.mark.parametrize("k", [256, 1000, 4096, 6000, 8192])
def test_flush_merge_and_rank_paths(oracle, radik, torch_cuda, monkeypatch, k):
    """A task split into 32 segments with a sampled threshold runs in flush
    mode; its merge selects in registers and leaves the row to the rank
    kernel when the candidates fit (up to 16384), else selects, sorts and
    writes in one block.  Both must give the exact answer with ties at the
    k-th value, NaN, custom indices and scaling."""
    monkeypatch.setenv("RADIK_SEG", "65536")
    n = 1 << 21 if k <= 1000 else 1 << 24  # the block sampler's rank stays within its limit
    rng = np.random.default_rng(k)
    x = rng.standard_normal(n).astype(np.float32)
    ws = radik.RadiKWorkspace("cuda", n, 1)
    ws.prepare([n], k)
    assert ws.plan_info()["sample_jobs"] > 0  # flush mode with the merge and rank kernels
    ws.close()
    _compare(oracle, radik, torch_cuda, x, [n], k)
    _compare(oracle, radik, torch_cuda, x, [n], k, largest=False, rev=True)
    q = np.round(x * 64.0).astype(np.float32) / 64.0  # about 500 distinct values: ties at the k-th one
    q[::1009] = np.nan
    _compare(oracle, radik, torch_cuda, q, [n], k, largest=False)
    _compare(oracle, radik, torch_cuda, q, [n], k, rev=True)
    ind = rng.permutation(n).astype(np.int64) * 5 - 7
    _compare(oracle, radik, torch_cuda, x, [n], k, indices=ind)
    _compare(oracle, radik, torch_cuda, x + 2.5, [n], k, withscale=True, largest=False)


@pytest.mark.parametrize("k", [1, 64, 256, 1000, 5000])
def test_deferred_finish(oracle, radik, torch_cuda, monkeypatch, k):
    """Single-segment tasks whose streaming block queues its candidates for
    a block with no streaming left to finish (RADIK_DEFER=1): exact results
    for every order, ties and NaN, scaling and custom indices, beside short
    tasks that are finished where they are streamed."""
    monkeypatch.setenv("RADIK_DEFER", "1")
    monkeypatch.setenv("RADIK_WS", "1")
    rng = np.random.default_rng(500 + k)
    lens = [65536] * 24 + [16384, 40000, 100, 0, 3, 200_000, 70_001, 4096, 5003]
    x = rng.standard_normal(sum(lens)).astype(np.float32)
    _compare(oracle, radik, torch_cuda, x, lens, k)
    _compare(oracle, radik, torch_cuda, x, lens, k, largest=False, rev=True)
    q = np.round(x * 8.0).astype(np.float32) / 8.0  # heavy ties
    q[::997] = np.nan
    _compare(oracle, radik, torch_cuda, q, lens, k, rev=True)
    _compare(oracle, radik, torch_cuda, q, lens, k, largest=False)
    ind = rng.permutation(sum(lens)).astype(np.int64) * 3 + 1
    _compare(oracle, radik, torch_cuda, x, lens, k, indices=ind)
    _compare(oracle, radik, torch_cuda, x + 5.0, lens, k, withscale=True)


@pytest.mark.parametrize("k", [1, 100, 1000, 4096])
def test_short_segments_single_task(oracle, radik, torch_cuda, monkeypatch, k):
    """The autotuner's short-segment plan (RADIK_SEG_MIN=4: 8192-element
    segments) on the 2^20-element N(0,1) task of seed 0: 128 segments, with a
    sampled threshold and the merge kernel where the segments' candidates
    would be many (128 k >= 8192) and the sample's rank fits (8 sampling
    blocks of 4096 elements: lam = k / 32, r = lam + max(3 sqrt(lam) + 6,
    5 sqrt(lam)) <= 256), else unsampled with every segment's k candidates."""
    monkeypatch.setenv("RADIK_SEG_MIN", "4")
    n = 1 << 20
    x = np.random.default_rng(0).standard_normal(n).astype(np.float32)
    ws = radik.RadiKWorkspace("cuda", n, 1)
    ws.prepare([n], k)
    info = ws.plan_info()
    ws.close()
    assert info["segments"] == 128
    lam = k * 8 * 8 * 512 / n
    r = int(np.ceil(lam + max(3 * np.sqrt(lam) + 6, 5 * np.sqrt(lam))))
    assert (info["sample_jobs"] > 0) == (128 * k >= 8192 and r <= 256)
    _compare(oracle, radik, torch_cuda, x, [n], k)
    _compare(oracle, radik, torch_cuda, x, [n], k, largest=False, rev=True)
    q = np.round(x * 32.0).astype(np.float32) / 32.0  # ties at the k-th value
    q[::1013] = np.nan
    _compare(oracle, radik, torch_cuda, q, [n], k, rev=True)
    _compare(oracle, radik, torch_cuda, x + 3.0, [n], k, withscale=True)
    # a batch of a few such tasks beside short ones
    lens = [n, 3 * n // 2, 20_000, 7]
    y = np.random.default_rng(k + 1).standard_normal(sum(lens)).astype(np.float32)
    ind = np.random.default_rng(k + 2).permutation(sum(lens)).astype(np.int32)
    _compare(oracle, radik, torch_cuda, y, lens, k, indices=ind)


def test_multipass_repeated_calls_stay_consistent(oracle, radik, torch_cuda):
    """The multi-pass path on a batch of many tasks, called repeatedly with
    one workspace: every call must leave the device error word clear (its
    rank search once let a slow warp read a residual rank that another
    thread had already updated) and match the oracle."""
    rng = np.random.default_rng(41)
    lens = [int(v) for v in np.clip(rng.lognormal(np.log(20000), 1.5, size=2048), 1, 400_000)]
    x = rng.standard_normal(sum(lens)).astype(np.float32)
    dev = torch_cuda.device("cuda")
    xt = torch_cuda.from_numpy(x).to(dev)
    T, k = len(lens), 64
    vo = torch_cuda.empty((T, k), dtype=torch_cuda.float32, device=dev)
    io = torch_cuda.empty((T, k), dtype=torch_cuda.int32, device=dev)
    ws = radik.RadiKWorkspace("cuda", max(lens), T)
    ov, oi = oracle.topk(x, lens, k)
    for _ in range(12):
        radik.topk_radix_select_(vo, io, ws, xt, None, lens, k, True, True, plain=True)
        assert ws.error_bits() == 0
        assert np.array_equal(vo.cpu().numpy().view(np.uint32), ov.view(np.uint32))
        assert np.array_equal(io.cpu().numpy().astype(np.int64), oi.astype(np.int64))
    ws.close()
