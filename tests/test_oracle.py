"""CPU tests: the oracle against the reference's known answers (transcribed in
tests/golden/) and against an independent numpy top-k."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import expected_values, plain_topk, task_data


def _cases(golden, kind):
    return [c for c in golden if c["kind"] == kind]


def test_get_bin_id_order(oracle, golden):
    c = _cases(golden, "get_bin_id_order")[0]
    vals = [float(v) if not isinstance(v, str) else float(v.replace("inf", "Infinity")) for v in c["values"]]
    bins = [oracle.get_bin_id(v, c["left"], c["right"]) for v in vals]
    assert all(0 <= b < 256 for b in bins)
    assert bins[0] == c["first"] and bins[-1] == c["last"]
    assert all(b > a for a, b in zip(bins[1:], bins[:-1]))


def test_key_properties(oracle):
    # -0 < +0, NaN above +Inf (unsubstituted key), order preserved on a sweep
    assert oracle.key(-0.0) < oracle.key(0.0)
    assert oracle.key(float("nan")) > oracle.key(float("inf"))
    xs = np.sort(np.random.default_rng(0).standard_normal(2000).astype(np.float32))
    keys = [oracle.key(float(x)) for x in xs]
    assert all(b >= a for a, b in zip(keys, keys[1:]))


def test_apply_scaling(oracle):
    fmin = float(np.finfo(np.float32).tiny)
    fmax = float(np.finfo(np.float32).max)
    assert oracle.apply_scaling(float("nan"), 0.0, False, True) == fmin
    assert oracle.apply_scaling(float("nan"), 0.0, False, False) == fmax
    assert oracle.apply_scaling(5.0, 2.0, True, True) == 3.0
    assert oracle.apply_scaling(5.0, 2.0, False, True) == 5.0


@pytest.mark.parametrize("idx", range(8))
def test_select_bin_known_answers(oracle, golden, idx):
    cases = _cases(golden, "select_bin")
    if idx >= len(cases):
        pytest.skip()
    c = cases[idx]
    bi, kv, ct = oracle.select_bin(np.array(c["hist"], np.int32), c["k"], c["largest"])
    assert list(bi) == c["bin_ids"], c["cite"]
    assert list(kv) == c["k_values"], c["cite"]
    assert list(ct) == c["counts"], c["cite"]


def test_count_bin_known_answers(oracle, golden):
    for c in _cases(golden, "count_bin_ex"):
        tasks = [task_data(t) for t in c["tasks"]]
        h = oracle.count_bin_ex(np.concatenate(tasks), [len(t) for t in tasks], c["left"], c["right"],
                                c["withscale"], c["largest"])
        assert h.tolist() == c["hist"], c["cite"]
    for c in _cases(golden, "count_bin"):
        tasks = [task_data(t) for t in c["tasks"]]
        stride = max(len(t) for t in tasks)
        padded = np.zeros(len(tasks) * stride, np.float32)
        for i, t in enumerate(tasks):
            padded[i * stride:i * stride + len(t)] = t
        h = oracle.count_bin(padded, [len(t) for t in tasks], stride, c["left"], c["right"])
        assert h.tolist() == c["hist"], c["cite"]


def test_select_candidate_known_answers(oracle, golden):
    for c in _cases(golden, "select_candidate"):
        tasks = [task_data(t) for t in c["tasks"]]
        stride = max(len(t) for t in tasks)
        padded = np.concatenate(tasks)
        out = oracle.select_candidate(padded, [len(t) for t in tasks], stride, c["bin_ids"], c["left"], c["right"])
        for o, e in zip(out, c["expected"]):
            assert sorted(o.tolist()) == sorted(e), c["cite"]
        out2 = oracle.select_candidate_ex(padded, [len(t) for t in tasks], c["bin_ids"], c["left"], c["right"])
        for o, e in zip(out2, c["expected"]):
            assert sorted(o.tolist()) == sorted(e), c["cite"]


def test_filter_known_answers(oracle, golden):
    n = 0
    for c in _cases(golden, "filter"):
        data = np.concatenate([task_data(t) for t in c["tasks"]])
        res, _ = oracle.filter_([*data], [len(data)], c["kth"], c["boundary"], c["k"], c["withscale"],
                                c["largest"])
        vals = res[0][0]
        assert len(vals) == c["count"], c["cite"]
        assert sorted(vals.tolist()) == sorted(expected_values(c["expected"]).tolist()), c["cite"]
        n += 1
    for c in _cases(golden, "filter_multi"):
        idx_in = np.array(c["idx_in"], np.int32) if "idx_in" in c else None
        res, _ = oracle.filter_(c["data"], c["task_lens"], c["kth"], c["boundary"], c["k"], c["withscale"],
                                c["largest"], idx_in=idx_in)
        for t, (v, i) in enumerate(res):
            assert len(v) == c["counts"][t], c["cite"]
            assert sorted(v.tolist()) == sorted(c["expected"][t]), c["cite"]
            if "expected_idx" in c:
                assert sorted(i.tolist()) == sorted(c["expected_idx"][t]), c["cite"]
        n += 1
    assert n >= 15


def _check_against_plain(oracle, data, lens, k, **kw):
    ov, oi = oracle.topk(data, lens, k, idx_dtype=np.int64, **kw)
    pv, pi = plain_topk(data, lens, k, **kw)
    assert np.array_equal(ov.view(np.uint32), pv.view(np.uint32))
    assert np.array_equal(oi, pi)


@pytest.mark.parametrize("largest", [True, False])
@pytest.mark.parametrize("rev", [True, False])
@pytest.mark.parametrize("k", [1, 16, 100, 4096])
def test_oracle_topk_vs_plain(oracle, largest, rev, k):
    rng = np.random.default_rng(k * 4 + largest * 2 + rev)
    data = rng.random(1 << 14, dtype=np.float32)
    _check_against_plain(oracle, data, [len(data)], k, largest=largest, rev=rev)


def test_oracle_property_test_algorithm(oracle, golden):
    """test/test_algorithm.jl:6-40: values equal sort(partialsort(x, 1:k,
    rev=LARGEST), rev=REV); indices valid, unique and pointing to equal values."""
    c = _cases(golden, "topk_property")[0]
    rng = np.random.default_rng(42)
    for k in c["k"]:
        for largest in c["largest"]:
            for rev in c["rev"]:
                x = rng.random(c["n"], dtype=np.float32)
                v, i = oracle.topk(x, [len(x)], k, largest=largest, rev=rev)
                part = np.sort(x)[::-1][:k] if largest else np.sort(x)[:k]
                exp = np.sort(part)[::-1] if rev else np.sort(part)
                assert np.array_equal(v[0], exp)
                idx = i[0].astype(np.int64)
                assert np.all((1 <= idx) & (idx <= len(x)))
                assert len(np.unique(idx)) == k
                assert np.array_equal(x[idx - 1], v[0])


def test_oracle_edge_cases(oracle):
    rng = np.random.default_rng(7)
    # ties, +-0, NaN, inf, short and empty tasks, scaling
    x = np.array([0.0, -0.0, 1.0, 1.0, 1.0, np.nan, np.inf, -np.inf, 2.0, -0.0, 0.0, 1.0], np.float32)
    for k in (1, 3, 5, 8, 12, 20):
        for largest in (True, False):
            for rev in (True, False):
                _check_against_plain(oracle, x, [len(x)], k, largest=largest, rev=rev)
    lens = [0, 3, 100, 1, 64, 65, 1000]
    data = rng.integers(0, 5, size=sum(lens)).astype(np.float32)
    for k in (1, 4, 64):
        for largest in (True, False):
            _check_against_plain(oracle, data, lens, k, largest=largest)
            _check_against_plain(oracle, data, lens, k, largest=largest, withscale=True)
    y = rng.standard_normal(5000).astype(np.float32) * 1e-3 + 1.0
    _check_against_plain(oracle, y, [5000], 50, withscale=True)
    _check_against_plain(oracle, y, [5000], 50, withscale=True, largest=False)


def test_oracle_custom_indices(oracle, golden):
    c = _cases(golden, "topk_multitask_custom_idx")[0]
    lens = c["task_lens"]
    rng = np.random.default_rng(1)
    x = rng.random(sum(lens), dtype=np.float32)
    ind = np.arange(1, sum(lens) + 1, dtype=np.int32)
    v, i = oracle.topk(x, lens, c["k"], largest=c["largest"], rev=c["rev"], indices=ind)
    off = 0
    for t, n in enumerate(lens):
        part = np.sort(x[off:off + n])[::-1][:c["k"]]
        assert np.array_equal(v[t], np.sort(part))
        local = i[t].astype(np.int64) - off
        assert np.array_equal(x[off:off + n][local - 1], v[t])
        off += n


def test_oracle_threads_equivalent(oracle):
    rng = np.random.default_rng(3)
    lens = list(rng.integers(0, 3000, size=64))
    x = rng.standard_normal(int(sum(lens))).astype(np.float32)
    a = oracle.topk(x, lens, 37, threads=1)
    b = oracle.topk(x, lens, 37, threads=0)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_oracle_large_property():
    """Sanity of the numpy reference itself on a heavy-tie input."""
    x = np.repeat(np.arange(10, dtype=np.float32), 100)
    v, i = plain_topk(x, [len(x)], 150)
    assert math.isclose(float(v[0, 0]), 8.0) and np.all(v[0, 50:] == 9.0)
    # the 50 tied 8.0 values taken are the lowest positions among the 8.0s
    assert sorted(i[0, :50].tolist()) == list(range(801, 851))
