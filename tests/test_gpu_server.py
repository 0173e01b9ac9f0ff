"""Request server (radik_server_*): continuous batching must not change any
result.  Every request's values and indices -- served in the mix and served
alone -- are compared with the oracle (the CPU restatement of the
reference's top-k, the standard of test/test_algorithm.jl:6-40) and with the
same request computed alone by radik.topk; the tolerance is zero: the
selection is exact and ties are broken by position, so a row's result does
not depend on which other rows share its launch.  The request shapes include
the serving stream's own: rows of 32,768, 131,072 and 1,048,576 elements
with k from {1, 50, 1024, 8192}, N(0,1) logits with a Gumbel(0,1) tail on 1%
of entries."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VALUE_ATOL = 0.0


def _requests(torch, rng, n, lens=(1000, 32768, 70000), ks=(1, 50, 1024)):
    """(device data, k, largest, rev, host copy of the data) per request."""
    reqs = []
    for i in range(n):
        rows = int(rng.integers(1, 9))
        row_len = int(rng.choice(lens))
        k = int(rng.choice(ks))
        largest = bool(rng.integers(0, 2))
        rev = bool(rng.integers(0, 2))
        x = rng.standard_normal((rows, row_len)).astype(np.float32)
        tail = rng.random((rows, row_len)) < 0.01  # logits with a Gumbel tail on 1% of entries
        x[tail] += rng.gumbel(size=int(tail.sum())).astype(np.float32)
        if i % 7 == 0:  # ties and special values
            x[:, ::5] = 3.0
            x[0, 1] = np.nan
            x[0, 2] = -0.0
            x[0, 3] = np.inf
        reqs.append((torch.from_numpy(x).cuda(), k, largest, rev, x))
    return reqs


def _alone(radik, torch, data, k, largest, rev, host=None):
    rows, row_len = data.shape
    v, i = radik.topk(data.reshape(-1), [row_len] * rows, k, largest=largest, rev=rev)
    return v, i


def _oracle(oracle, host, k, largest, rev):
    rows, row_len = host.shape
    return oracle.topk(host.reshape(-1), [row_len] * rows, k, largest=largest, rev=rev)


def _same_as_oracle(got, want):
    gv, gi = (t.cpu().numpy() for t in got)
    ov, oi = want
    assert gv.shape == ov.shape
    assert np.array_equal(gv.view(np.uint32), ov.view(np.uint32))
    assert np.array_equal(gi.astype(np.int64), oi.astype(np.int64))


def _same(a, b):
    av, ai = (t.cpu().numpy() for t in a)
    bv, bi = (t.cpu().numpy() for t in b)
    assert av.shape == bv.shape
    assert np.allclose(av, bv, rtol=0.0, atol=VALUE_ATOL, equal_nan=True)
    assert np.array_equal(av.view(np.uint32), bv.view(np.uint32))
    assert np.array_equal(ai.astype(np.int64), bi.astype(np.int64))


def test_server_results_in_the_mix_equal_alone(radik, oracle, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(2024)
    reqs = _requests(torch, rng, 40)
    alone = [_alone(radik, torch, *r) for r in reqs]
    want = [_oracle(oracle, h, k, lg, rv) for _, k, lg, rv, h in reqs]
    with radik.Server(slots=3, mem_cap_bytes=2 << 30, max_batch_rows=64) as srv:
        tickets = [srv.submit(d, k, largest=lg, rev=rv) for d, k, lg, rv, _ in reqs]  # all in flight together
        mixed = [srv.wait(t, timeout_s=60) for t in tickets]
        # each request submitted alone to the server, one at a time
        solo = []
        for d, k, lg, rv, _ in reqs:
            solo.append(srv.wait(srv.submit(d, k, largest=lg, rev=rv), timeout_s=60))
        st = srv.stats()
        log = srv.batches()
    for a, w, m, s in zip(alone, want, mixed, solo):
        _same_as_oracle(m, w)
        _same_as_oracle(s, w)
        _same(m, a)
        _same(s, a)
    assert st["completed"] == 2 * len(reqs)
    assert st["batches"] < 2 * len(reqs)  # requests were packed together
    # the batch log: one entry per launched batch, rows and elements adding up to the requests'
    assert len(log) == st["batches"]
    assert sum(b["rows"] for b in log) == 2 * sum(r[0].shape[0] for r in reqs)
    assert sum(b["elements"] for b in log) == 2 * sum(r[0].numel() for r in reqs)
    assert all(b["gpu_us"] > 0 and b["launch_us"] > 0 and b["k"] in (1, 50, 1024) for b in log)
    assert 0 < st["p50_us"] <= st["p99_us"]


def test_server_large_k_and_rows_of_many_tasks(radik, oracle, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(7)
    hosts = [(rng.random((2, 200_000), dtype=np.float32), 8192, True, False),
             (rng.random((300, 4000), dtype=np.float32), 50, False, True),
             (rng.random((1, 1 << 21), dtype=np.float32), 1024, True, True)]
    reqs = [(torch.from_numpy(h).cuda(), k, lg, rv, h) for h, k, lg, rv in hosts]
    alone = [_alone(radik, torch, *r) for r in reqs]
    with radik.Server(slots=2, mem_cap_bytes=4 << 30) as srv:
        outs = [srv.wait(srv.submit(d, k, largest=lg, rev=rv), timeout_s=60) for d, k, lg, rv, _ in reqs]
    for (_, k, lg, rv, h), a, o in zip(reqs, alone, outs):
        _same_as_oracle(o, _oracle(oracle, h, k, lg, rv))
        _same(o, a)


def test_server_stream_shapes_against_the_oracle(radik, oracle, torch_cuda):
    """The serving stream's request shapes -- 1,048,576-element rows with
    k = 8192 and k = 1 among them -- submitted together (so rows of
    different requests share launches) and one at a time, every result
    against the oracle."""
    torch = torch_cuda
    rng = np.random.default_rng(44)
    shapes = [(2, 1 << 20, 8192, True, False), (3, 1 << 20, 1, True, False), (2, 1 << 20, 1024, True, True),
              (3, 131072, 8192, True, False), (4, 131072, 50, False, False), (5, 32768, 1, True, True),
              (2, 32768, 8192, True, False), (3, 1 << 20, 50, True, False)]
    reqs = []
    for rows, n, k, lg, rv in shapes:
        x = rng.standard_normal((rows, n)).astype(np.float32)
        tail = rng.random((rows, n)) < 0.01
        x[tail] += rng.gumbel(size=int(tail.sum())).astype(np.float32)
        reqs.append((torch.from_numpy(x).cuda(), k, lg, rv, x))
    want = [_oracle(oracle, h, k, lg, rv) for _, k, lg, rv, h in reqs]
    with radik.Server(slots=4, mem_cap_bytes=8 << 30, max_batch_rows=4096) as srv:
        tickets = [srv.submit(d, k, largest=lg, rev=rv) for d, k, lg, rv, _ in reqs]
        mixed = [srv.wait(t, timeout_s=120) for t in tickets]
        solo = [srv.wait(srv.submit(d, k, largest=lg, rev=rv), timeout_s=120) for d, k, lg, rv, _ in reqs]
    for w, m, s in zip(want, mixed, solo):
        _same_as_oracle(m, w)
        _same_as_oracle(s, w)


def test_server_admission_by_memory(radik, oracle, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(11)
    x = torch.from_numpy(rng.random((4, 65536), dtype=np.float32)).cuda()
    one = 4 * 65536 * 4 + 4 * 64 * 8
    # a cap that admits the workspace pool and about one request at a time
    with radik.Server(slots=4, mem_cap_bytes=64 << 20) as srv:
        tickets = [srv.submit(x, 64) for _ in range(12)]
        outs = [srv.wait(t, timeout_s=60) for t in tickets]
        st = srv.stats()
        assert st["completed"] == 12 and st["mem_in_flight"] == 0
    ref = _alone(radik, torch, x, 64, True, False)
    want = _oracle(oracle, x.cpu().numpy(), 64, True, False)
    for o in outs:
        _same(o, ref)
        _same_as_oracle(o, want)
    with radik.Server(slots=1, mem_cap_bytes=one - 1) as srv:
        with pytest.raises(radik.RadiKError, match="memory cap"):
            srv.submit(x, 64)
