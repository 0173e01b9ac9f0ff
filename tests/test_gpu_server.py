"""Request server (radik_server_*): continuous batching must not change any
result.  Each request's values and indices are compared with the same
request computed alone (radik.topk on its rows, and the request submitted
alone to the server); the tolerance is zero -- the selection is exact and
ties are broken by position, so a row's result does not depend on which
other rows share its launch."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VALUE_ATOL = 0.0


def _requests(torch, rng, n, lens=(1000, 32768, 70000), ks=(1, 50, 1024)):
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
        reqs.append((torch.from_numpy(x).cuda(), k, largest, rev))
    return reqs


def _alone(radik, torch, data, k, largest, rev):
    rows, row_len = data.shape
    v, i = radik.topk(data.reshape(-1), [row_len] * rows, k, largest=largest, rev=rev)
    return v, i


def _same(a, b):
    av, ai = (t.cpu().numpy() for t in a)
    bv, bi = (t.cpu().numpy() for t in b)
    assert av.shape == bv.shape
    assert np.allclose(av, bv, rtol=0.0, atol=VALUE_ATOL, equal_nan=True)
    assert np.array_equal(av.view(np.uint32), bv.view(np.uint32))
    assert np.array_equal(ai.astype(np.int64), bi.astype(np.int64))


def test_server_results_in_the_mix_equal_alone(radik, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(2024)
    reqs = _requests(torch, rng, 40)
    alone = [_alone(radik, torch, *r) for r in reqs]
    with radik.Server(slots=3, mem_cap_bytes=2 << 30, max_batch_rows=64) as srv:
        tickets = [srv.submit(d, k, largest=lg, rev=rv) for d, k, lg, rv in reqs]  # all in flight together
        mixed = [srv.wait(t, timeout_s=60) for t in tickets]
        # each request submitted alone to the server, one at a time
        solo = []
        for d, k, lg, rv in reqs:
            solo.append(srv.wait(srv.submit(d, k, largest=lg, rev=rv), timeout_s=60))
        st = srv.stats()
    for a, m, s in zip(alone, mixed, solo):
        _same(m, a)
        _same(s, a)
    assert st["completed"] == 2 * len(reqs)
    assert st["batches"] < 2 * len(reqs)  # requests were packed together
    assert 0 < st["p50_us"] <= st["p99_us"]


def test_server_large_k_and_rows_of_many_tasks(radik, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(7)
    reqs = [(torch.from_numpy(rng.random((2, 200_000), dtype=np.float32)).cuda(), 8192, True, False),
            (torch.from_numpy(rng.random((300, 4000), dtype=np.float32)).cuda(), 50, False, True),
            (torch.from_numpy(rng.random((1, 1 << 21), dtype=np.float32)).cuda(), 1024, True, True)]
    alone = [_alone(radik, torch, *r) for r in reqs]
    with radik.Server(slots=2, mem_cap_bytes=4 << 30) as srv:
        outs = [srv.wait(srv.submit(d, k, largest=lg, rev=rv), timeout_s=60) for d, k, lg, rv in reqs]
    for a, o in zip(alone, outs):
        _same(o, a)


def test_server_admission_by_memory(radik, torch_cuda):
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
    for o in outs:
        _same(o, ref)
    with radik.Server(slots=1, mem_cap_bytes=one - 1) as srv:
        with pytest.raises(radik.RadiKError, match="memory cap"):
            srv.submit(x, 64)
