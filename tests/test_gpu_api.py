"""GPU tests of the reference-facing API (the Julia surface mirrored in
radik.jl_b200) and of the stage entry points against the reference's known
answers (tests/golden/)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import expected_values, task_data

pytestmark = pytest.mark.gpu


def _cases(golden, kind):
    return [c for c in golden if c["kind"] == kind]


def test_count_bin_known_answers(radik, torch_cuda, golden):
    for c in _cases(golden, "count_bin_ex"):
        tasks = [task_data(t) for t in c["tasks"]]
        d = torch_cuda.from_numpy(np.concatenate(tasks)).cuda()
        h = radik.count_bin_ex(d, [len(t) for t in tasks], c["left"], c["right"], c["withscale"], c["largest"])
        assert h.cpu().numpy().tolist() == c["hist"], c["cite"]
    for c in _cases(golden, "count_bin"):
        tasks = [task_data(t) for t in c["tasks"]]
        stride = max(len(t) for t in tasks)
        padded = np.zeros(len(tasks) * stride, np.float32)
        for i, t in enumerate(tasks):
            padded[i * stride:i * stride + len(t)] = t
        h = radik.count_bin(torch_cuda.from_numpy(padded).cuda(), [len(t) for t in tasks], stride,
                            c["left"], c["right"])
        assert h.cpu().numpy().tolist() == c["hist"], c["cite"]


def test_count_bin_ex_matches_oracle_with_nan(radik, torch_cuda, oracle):
    rng = np.random.default_rng(0)
    lens = [1000, 0, 77, 50_000]
    x = rng.standard_normal(sum(lens)).astype(np.float32)
    x[::97] = np.nan
    for right in (20, 24, 30):
        for ws in (False, True):
            for lg in (False, True):
                h = radik.count_bin_ex(torch_cuda.from_numpy(x).cuda(), lens, 0, right, ws, lg).cpu().numpy()
                assert np.array_equal(h, oracle.count_bin_ex(x, lens, 0, right, ws, lg))


def test_select_bin_known_answers(radik, torch_cuda, golden):
    for c in _cases(golden, "select_bin"):
        h = torch_cuda.tensor(np.array(c["hist"], np.int32)).cuda()
        bi, kv, ct = radik.select_bin(h, c["k"], c["largest"])
        assert bi.cpu().tolist() == c["bin_ids"], c["cite"]
        assert kv.cpu().tolist() == c["k_values"], c["cite"]
        assert ct.cpu().tolist() == c["counts"], c["cite"]


def test_select_bin_matches_oracle(radik, torch_cuda, oracle):
    rng = np.random.default_rng(1)
    h = rng.integers(0, 50, size=(40, 4096)).astype(np.int32)
    h[3] = 0
    k = rng.integers(1, 60_000, size=40).astype(np.int32)
    for largest in (True, False):
        g = radik.select_bin(torch_cuda.from_numpy(h).cuda(), k, largest)
        o = oracle.select_bin(h, k, largest)
        for a, b in zip(g, o):
            assert np.array_equal(a.cpu().numpy(), b)


def test_filter_known_answers(radik, torch_cuda, golden):
    for c in _cases(golden, "filter"):
        data = np.concatenate([task_data(t) for t in c["tasks"]])
        res, _ = radik.filter_(torch_cuda.from_numpy(data).cuda(), [len(data)], c["kth"], c["boundary"], c["k"],
                               c["withscale"], c["largest"])
        vals = res[0][0]
        assert len(vals) == c["count"], c["cite"]
        assert sorted(vals.tolist()) == sorted(expected_values(c["expected"]).tolist()), c["cite"]
    for c in _cases(golden, "filter_multi"):
        idx_in = torch_cuda.tensor(np.array(c["idx_in"], np.int32)).cuda() if "idx_in" in c else None
        d = torch_cuda.tensor(np.array(c["data"], np.float32)).cuda()
        res, _ = radik.filter_(d, c["task_lens"], c["kth"], c["boundary"], c["k"], c["withscale"], c["largest"],
                               idx_in=idx_in)
        for t, (v, i) in enumerate(res):
            assert len(v) == c["counts"][t], c["cite"]
            assert sorted(v.tolist()) == sorted(c["expected"][t]), c["cite"]
            if "expected_idx" in c:
                assert sorted(i.tolist()) == sorted(c["expected_idx"][t]), c["cite"]


def test_topk_overloads(radik, torch_cuda, golden):
    """test/test_algorithm.jl:98-112."""
    rng = np.random.default_rng(2)
    x = torch_cuda.from_numpy(rng.random(1000, dtype=np.float32)).cuda()
    v1, i1 = radik.topk(x, 100, largest=True, rev=False)
    ind = torch_cuda.arange(1, 1001, dtype=torch_cuda.int32, device="cuda")
    v2, i2 = radik.topk(x, 100, indices=ind, largest=True, rev=False)
    assert torch_cuda.equal(v1, v2) and torch_cuda.equal(i1, i2)
    exp = np.sort(np.sort(x.cpu().numpy())[::-1][:100])
    assert np.array_equal(v1.cpu().numpy(), exp)
    assert v1.shape == (100,) and i1.dtype == torch_cuda.int32


def test_topk_batch_sequential_indices(radik, torch_cuda):
    """test/test_algorithm.jl:114-150: per-task sequential custom indices give
    the automatic indices."""
    rng = np.random.default_rng(4)
    lens = [1000, 1500, 800]
    x = torch_cuda.from_numpy(rng.random(sum(lens), dtype=np.float32)).cuda()
    v1, i1 = radik.topk(x, lens, 50)
    ind = torch_cuda.from_numpy(np.concatenate([np.arange(1, n + 1, dtype=np.int32) for n in lens])).cuda()
    v2, i2 = radik.topk(x, lens, 50, indices=ind)
    assert torch_cuda.equal(v1, v2) and torch_cuda.equal(i1, i2)
    assert v1.shape == (3, 50)


def test_topk_inplace_and_errors(radik, torch_cuda):
    """test/test_algorithm.jl:152-162 and the validation of src/algorithm.jl:492-510."""
    x = torch_cuda.randn(1000, device="cuda")
    vo = torch_cuda.zeros((1, 50), device="cuda")
    io = torch_cuda.zeros((1, 50), dtype=torch_cuda.int32, device="cuda")
    with pytest.raises(radik.RadiKError, match="val_out must have size"):
        radik.topk_(vo, io, x, [1000], 100)
    with pytest.raises(radik.RadiKError, match="indices length must equal data length"):
        radik.topk(x, 100, indices=torch_cuda.arange(1, 501, dtype=torch_cuda.int32, device="cuda"))
    with pytest.raises(radik.RadiKError, match="only supports Float32"):
        radik.topk(x.double(), 10)
    vo = torch_cuda.zeros((1, 100), device="cuda")
    io = torch_cuda.zeros((1, 100), dtype=torch_cuda.int32, device="cuda")
    assert radik.topk_(vo, io, x, [1000], 100) is None
    assert np.array_equal(vo[0].cpu().numpy(), np.sort(np.sort(x.cpu().numpy())[-100:]))


def test_workspace_reuse_and_limits(radik, torch_cuda):
    ws = radik.RadiKWorkspace("cuda", 10_000, 4)
    vo = torch_cuda.zeros((4, 100), device="cuda")
    io = torch_cuda.zeros((4, 100), dtype=torch_cuda.int32, device="cuda")
    for _ in range(3):
        x = torch_cuda.randn(10_000, device="cuda")
        radik.topk_radix_select_(vo, io, ws, x, None, [5000, 2000, 2000, 1000], 100)
    with pytest.raises(radik.RadiKError, match="workspace requires"):
        radik.topk_radix_select_(vo, io, ws, torch_cuda.randn(20_000, device="cuda"), None,
                                 [15_000, 2000, 2000, 1000], 100)
    ws.close()


def test_host_buffer_entry_point(radik, torch_cuda, oracle):
    rng = np.random.default_rng(8)
    lens = [10_000, 5, 60_000]
    x = rng.standard_normal(sum(lens)).astype(np.float32)
    v, i = radik.topk_host(x, lens, 77, largest=False, rev=True)
    ov, oi = oracle.topk(x, lens, 77, largest=False, rev=True)
    assert np.array_equal(v, ov) and np.array_equal(i, oi)


def test_autotune_keeps_results_exact(oracle, radik, torch_cuda):
    """radik_ws_autotune times the candidate configurations on the batch and
    keeps the fastest for its shape; results stay identical to the oracle
    under the chosen configuration and on later calls."""
    torch = torch_cuda
    rng = np.random.default_rng(99)
    lens = [40_000] * 24 + [300_000, 7]
    k = 128
    h = rng.standard_normal(sum(lens)).astype(np.float32)
    x = torch.from_numpy(h).cuda()
    vo = torch.empty((len(lens), k), device="cuda")
    io = torch.empty((len(lens), k), dtype=torch.int32, device="cuda")
    ws = radik.RadiKWorkspace("cuda", max(lens), len(lens))
    info = ws.autotune(vo, io, x, None, lens, k, True, True, reps=2)
    assert info["ms"] > 0 and info["path"] in (0, 1) and info["grid"] > 0
    ov, oi = oracle.topk(h, lens, k)
    for _ in range(2):
        vo.fill_(7.0)
        radik.topk_radix_select_(vo, io, ws, x, None, lens, k, True, True)
        assert np.array_equal(vo.cpu().numpy().view(np.uint32), ov.view(np.uint32))
        assert np.array_equal(io.cpu().numpy().astype(np.int64), oi.astype(np.int64))
        assert ws.plan_info()["path"] == info["path"]
    ws.close()


def _tuned_lines(path):
    return [l.split() for l in path.read_text().splitlines() if l and not l.startswith("#")]


def test_tuning_table_shared_across_workspaces(oracle, radik, torch_cuda, tmp_path):
    """The autotuner's choice for a batch shape is kept process-wide: a new
    workspace meeting that shape uses it without timing; a saved and edited
    table, loaded back, decides the plan of the next workspace."""
    torch = torch_cuda
    radik.tune_clear()
    rng = np.random.default_rng(123)
    lens = [40_000] * 24 + [300_000, 7]
    k = 128
    h = rng.standard_normal(sum(lens)).astype(np.float32)
    x = torch.from_numpy(h).cuda()
    vo = torch.empty((len(lens), k), device="cuda")
    io = torch.empty((len(lens), k), dtype=torch.int32, device="cuda")
    ov, oi = oracle.topk(h, lens, k)
    ws = radik.RadiKWorkspace("cuda", max(lens), len(lens))
    info = ws.autotune(vo, io, x, None, lens, k, True, True, reps=2)
    ws.close()
    p = tmp_path / "tune.txt"
    radik.tune_save(p)
    rows = _tuned_lines(p)
    assert len(rows) == 1 and int(rows[0][1]) == len(lens) and int(rows[0][2]) == sum(lens) and int(rows[0][3]) == k

    def run_new():
        w = radik.RadiKWorkspace("cuda", max(lens), len(lens))
        vo.fill_(7.0)
        radik.topk_radix_select_(vo, io, w, x, None, lens, k, True, True)
        assert np.array_equal(vo.cpu().numpy().view(np.uint32), ov.view(np.uint32))
        assert np.array_equal(io.cpu().numpy().astype(np.int64), oi.astype(np.int64))
        plan = w.plan_info()
        w.close()
        return plan

    assert run_new()["path"] == info["path"]
    for form, path in ((0, 0), (1, 1)):
        rows[0][6] = str(form)  # the kernel form field
        p2 = tmp_path / f"tune_{form}.txt"
        p2.write_text(" ".join(rows[0]) + "\n")
        radik.tune_clear()
        assert radik.tune_load(p2) == 1
        assert run_new()["path"] == path
    radik.tune_clear()


def test_plain_path_digit_schedules(oracle, radik, torch_cuda, tmp_path):
    """The multi-pass path tunes its digit schedule (pass widths and count);
    every schedule gives the oracle's rows, ties and NaNs included."""
    torch = torch_cuda
    radik.tune_clear()
    rng = np.random.default_rng(321)
    lens = [100_000, 3, 0, 65_536, 250_000]
    k = 300
    h = rng.integers(-50, 50, sum(lens)).astype(np.float32)  # many ties
    h[::101] = np.nan
    x = torch.from_numpy(h).cuda()
    vo = torch.empty((len(lens), k), device="cuda")
    io = torch.empty((len(lens), k), dtype=torch.int64, device="cuda")
    for largest, ascend in ((True, False), (False, True)):
        ov, oi = oracle.topk(h, lens, k, largest=largest, rev=not ascend)
        ws = radik.RadiKWorkspace("cuda", max(lens), len(lens))
        info = ws.autotune(vo, io, x, None, lens, k, largest, ascend, reps=1, plain=True)
        assert info["path"] == 2
        ws.close()
        p = tmp_path / "plain.txt"
        radik.tune_save(p)
        rows = [r for r in _tuned_lines(p) if int(r[1]) == len(lens)]
        assert len(rows) == 1
        for sched in range(4):
            rows[0][14] = str(sched)
            p2 = tmp_path / f"plain_{sched}.txt"
            p2.write_text(" ".join(rows[0]) + "\n")
            radik.tune_clear()
            assert radik.tune_load(p2) == 1
            w = radik.RadiKWorkspace("cuda", max(lens), len(lens))
            vo.fill_(7.0)
            radik.topk_radix_select_(vo, io, w, x, None, lens, k, largest, ascend, plain=True)
            got_v = vo.cpu().numpy()
            assert np.array_equal(got_v.view(np.uint32), ov.view(np.uint32)), sched
            assert np.array_equal(io.cpu().numpy(), oi.astype(np.int64)), sched
            assert w.plan_info()["path"] == 2
            w.close()
        radik.tune_clear()
