"""Generate tests/golden/reference_known_answers.json.

The reference (RadiK.jl) is Julia and cannot run on this machine, so its golden
vectors are its own known-answer tests, transcribed here case by case with the
test file:line each one comes from (paths relative to the RadiK.jl project
root).  Where a reference test computes its expectation with a CPU loop
(test_count_bin.jl, test_select_candidate.jl), the expectation is recomputed
below with an independent numpy restatement of the same formula
(src/utils.jl:29-33, :62-71), so the fixture does not depend on the oracle it
is used to check.

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import pathlib

import numpy as np

OUT = pathlib.Path(__file__).resolve().parent / "reference_known_answers.json"
FLT_MIN = float(np.finfo(np.float32).tiny)


def np_key(x: np.ndarray) -> np.ndarray:
    b = np.atleast_1d(np.asarray(x, dtype=np.float32)).view(np.uint32)
    with np.errstate(over="ignore"):
        mask = ((~(b >> np.uint32(31))) + np.uint32(1)) | np.uint32(0x80000000)
    return b ^ mask


def np_bin(x, left, right):
    return ((np_key(x) << np.uint32(left)) & np.uint32(0xFFFFFFFF)) >> np.uint32(right)


def np_scale(x, scaler, withscale, largest):
    x = np.asarray(x, dtype=np.float32)
    p = np.where(np.isnan(x), np.float32(FLT_MIN if largest else np.finfo(np.float32).max), x)
    return (p - np.float32(scaler)).astype(np.float32) if withscale else p


def f32list(a):
    return [float(v) for v in np.asarray(a, dtype=np.float32)]


def main():
    cases = []

    # --- test/test_utils.jl:9-23 -------------------------------------------
    cases.append({
        "kind": "get_bin_id_order",
        "cite": "test/test_utils.jl:9-23",
        "values": ["inf", 100.0, 2.0, 1.0, 0.0, -1.0, -2.0, -100.0, "-inf"],
        "left": 0, "right": 24,
        "first": 255, "last": 0, "strictly_decreasing": True,
    })

    # --- test/test_select_bin.jl (kernel-level known answers) --------------
    def hist256(entries):
        h = [0] * 256
        for lo, hi, v in entries:
            for b in range(lo, hi + 1):
                h[b - 1] = v  # 1-based bins as in the Julia test
        return h

    h = hist256([(1, 1, 2), (2, 2, 8), (3, 3, 14), (4, 4, 3)])
    cases.append({"kind": "select_bin", "cite": "test/test_select_bin.jl:194-222",
                  "hist": [h], "k": [5], "largest": True,
                  "bin_ids": [3], "k_values": [2], "counts": [14]})
    cases.append({"kind": "select_bin", "cite": "test/test_select_bin.jl:224-252",
                  "hist": [h], "k": [5], "largest": False,
                  "bin_ids": [2], "k_values": [3], "counts": [8]})
    cases.append({"kind": "select_bin", "cite": "test/test_select_bin.jl:254-282",
                  "hist": [hist256([(1, 10, 1)])], "k": [5], "largest": True,
                  "bin_ids": [6], "k_values": [1], "counts": [1]})
    cases.append({"kind": "select_bin", "cite": "test/test_select_bin.jl:284-326",
                  "hist": [hist256([(1, 10, 1)]), hist256([(101, 110, 2)]),
                           hist256([(201, 206, 3)])],
                  "k": [5, 7, 8], "largest": True,
                  "bin_ids": [6, 107, 204], "k_values": [1, 1, 2], "counts": [1, 2, 3]})
    cases.append({"kind": "select_bin", "cite": "test/test_select_bin.jl:328-352",
                  "hist": [hist256([(1, 1, 5)])], "k": [3], "largest": True,
                  "bin_ids": [1], "k_values": [3], "counts": [5]})
    # find_bin_and_write! boundary cases (test/test_select_bin.jl:146-188),
    # restated on a 3-bin histogram handled by one thread.
    cases.append({"kind": "select_bin", "cite": "test/test_select_bin.jl:150-168",
                  "hist": [[5, 3, 2]], "k": [1], "largest": False,
                  "bin_ids": [1], "k_values": [1], "counts": [5]})
    cases.append({"kind": "select_bin", "cite": "test/test_select_bin.jl:170-187",
                  "hist": [[5, 3, 2]], "k": [10], "largest": False,
                  "bin_ids": [3], "k_values": [2], "counts": [2]})
    # k beyond the total: nothing written (test/test_select_bin.jl:122-144)
    cases.append({"kind": "select_bin", "cite": "test/test_select_bin.jl:122-144",
                  "hist": [[3, 5, 2, 8]], "k": [24], "largest": True,
                  "bin_ids": [0], "k_values": [24], "counts": [0]})

    # --- test/test_count_bin.jl:11-112 -------------------------------------
    scale = 10
    tasks = [np.arange(1, 20_000 * scale + 1, dtype=np.float32),
             np.arange(50 * scale, 80 * scale + 1, dtype=np.float32),
             np.arange(100 * scale, 200 * scale + 1, dtype=np.float32)]
    left, right = 0, 30
    bins = 1 << (32 - right)
    ex = []
    for t in tasks:
        s = np_scale(t, t[0], True, True)
        ex.append(np.bincount(np_bin(s, left, right).astype(np.int64), minlength=bins).tolist())
    plain = [np.bincount(np_bin(t, left, right).astype(np.int64), minlength=bins).tolist()
             for t in tasks]
    assert all(sum(h) == len(t) for h, t in zip(ex, tasks))
    cases.append({"kind": "count_bin_ex", "cite": "test/test_count_bin.jl:11-63",
                  "tasks": [{"range": [1, 20_000 * scale]}, {"range": [50 * scale, 80 * scale]},
                            {"range": [100 * scale, 200 * scale]}],
                  "left": left, "right": right, "withscale": True, "largest": True,
                  "hist": ex})
    cases.append({"kind": "count_bin", "cite": "test/test_count_bin.jl:65-111",
                  "tasks": [{"range": [1, 20_000 * scale]}, {"range": [50 * scale, 80 * scale]},
                            {"range": [100 * scale, 200 * scale]}],
                  "left": left, "right": right, "hist": plain})

    # --- test/test_select_candidate.jl -------------------------------------
    d = np.arange(1, 11, dtype=np.float32)
    tb = int(np_bin(np.float32(3.0), 0, 23)[0]) + 1
    cases.append({"kind": "select_candidate", "cite": "test/test_select_candidate.jl:12-48",
                  "tasks": [{"range": [1, 10]}], "left": 0, "right": 23, "bin_ids": [tb],
                  "expected": [[2.0, 3.0]]})
    d = np.arange(1, 31, dtype=np.float32)
    tb = int(np_bin(np.float32(15.0), 0, 20)[0]) + 1
    exp = f32list(d[np_bin(d, 0, 20) + 1 == tb])
    cases.append({"kind": "select_candidate", "cite": "test/test_select_candidate.jl:190-232",
                  "tasks": [{"range": [1, 30]}], "left": 0, "right": 20, "bin_ids": [tb],
                  "expected": [exp]})

    # --- test/test_filter.jl ------------------------------------------------
    def filt(cite, rng, K, kth, boundary, withscale, largest, count, expected,
             idx_in=None, expected_idx=None, kind="filter"):
        exp = list(expected)
        if len(exp) > 8 and exp == list(range(exp[0], exp[0] + len(exp))):
            exp = {"range": [exp[0], exp[-1]]}  # contiguous integer values
        c = {"kind": kind, "cite": cite, "tasks": rng, "k": K, "kth": kth,
             "boundary": boundary, "withscale": withscale, "largest": largest,
             "count": count, "expected": exp}
        if idx_in is not None:
            c["idx_in"] = idx_in
            c["expected_idx"] = expected_idx
        cases.append(c)

    r1000 = [{"range": [1, 1000]}]
    filt("test/test_filter.jl:8-49", r1000, 1000, [0.0], [0], False, True, 1000,
         list(range(1, 1001)), expected_idx=None)
    # largest, scaled kth = data[996] - data[1] = 995
    filt("test/test_filter.jl:51-95", r1000, 5, [995.0], [0], True, True, 4, [1000, 999, 998, 997])
    filt("test/test_filter.jl:97-116", r1000, 5, [995.0], [1], True, True, 5, [1000, 999, 998, 997, 996])
    filt("test/test_filter.jl:118-137", r1000, 5, [995.0], [0], False, True, 5, [1000, 999, 998, 997, 996])
    # smallest, scaled kth = data[5] - data[1] = 4
    filt("test/test_filter.jl:140-184", r1000, 5, [4.0], [0], True, False, 4, [1, 2, 3, 4])
    filt("test/test_filter.jl:186-205", r1000, 5, [4.0], [1], True, False, 5, [1, 2, 3, 4, 5])
    filt("test/test_filter.jl:207-226", r1000, 5, [4.0], [0], False, False, 3, [1, 2, 3])
    filt("test/test_filter.jl:228-247", r1000, 5, [4.0], [1], False, False, 4, [1, 2, 3, 4])
    # multi-task, K = 2, kth = 4th element of each task, boundary = K
    cases.append({"kind": "filter_multi", "cite": "test/test_filter.jl:254-319",
                  "data": [1, 2, 3, 4, 5, 10, 20, 30, 40, 50, 100, 200, 300, 400, 500],
                  "task_lens": [5, 5, 5], "k": 2, "kth": [4, 40, 400], "boundary": [2, 2, 2],
                  "withscale": False, "largest": True, "counts": [2, 2, 2],
                  "expected": [[5, 4], [50, 40], [500, 400]]})
    r2000 = [{"range": [1, 2000]}]
    filt("test/test_filter.jl:321-354", r2000, 2001, [500.0], [10], False, True, 2000,
         list(range(1, 2001)))
    filt("test/test_filter.jl:356-389", r2000, 1500, [500.0], [0], False, True, 1500,
         list(range(501, 2001)))
    r10k = [{"range": [1, 10000]}]
    # largest, scaled kth = data[8001] - data[1] = 8000
    filt("test/test_filter.jl:391-440", r10k, 2000, [8000.0], [0], True, True, 1999,
         list(range(8002, 10001)))
    filt("test/test_filter.jl:441-460", r10k, 2000, [8000.0], [1], True, True, 2000,
         list(range(8001, 10001)))
    # unscaled kth 8000 -> strictly greater 8001..10000 = 2000 values
    filt("test/test_filter.jl:461-479", r10k, 2000, [8000.0], [0], False, True, 2000,
         list(range(8001, 10001)))
    # smallest, scaled kth = data[2000] - data[1] = 1999
    filt("test/test_filter.jl:481-524", r10k, 2000, [1999.0], [0], True, False, 1999,
         list(range(1, 2000)))
    filt("test/test_filter.jl:526-545", r10k, 2000, [1999.0], [1], True, False, 2000,
         list(range(1, 2001)))
    filt("test/test_filter.jl:546-564", r10k, 2000, [1999.0], [0], False, False, 1998,
         list(range(1, 1999)))
    filt("test/test_filter.jl:566-584", r10k, 2000, [1999.0], [1], False, False, 1999,
         list(range(1, 2000)))
    # custom indices (WITHIDXIN)
    cases.append({"kind": "filter_multi", "cite": "test/test_filter.jl:705-781",
                  "data": [100, 85, 92, 78, 95, 88, 90, 82], "task_lens": [8], "k": 3,
                  "kth": [92], "boundary": [3], "withscale": False, "largest": True,
                  "idx_in": [10, 11, 12, 13, 14, 15, 16, 17], "counts": [3],
                  "expected": [[100, 95, 92]], "expected_idx": [[10, 14, 12]]})
    # edge cases
    cases.append({"kind": "filter_multi", "cite": "test/test_filter.jl:789-832",
                  "data": [1, 2, 3], "task_lens": [3], "k": 2, "kth": [100], "boundary": [0],
                  "withscale": False, "largest": True, "counts": [0], "expected": [[]]})
    cases.append({"kind": "filter_multi", "cite": "test/test_filter.jl:834-891",
                  "data": [50, 50, 50, 50, 50], "task_lens": [5], "k": 3, "kth": [50],
                  "boundary": [3], "withscale": False, "largest": True, "counts": [3],
                  "expected": [[50, 50, 50]]})

    # --- test/test_algorithm.jl (end-to-end properties) --------------------
    cases.append({"kind": "topk_property", "cite": "test/test_algorithm.jl:6-40",
                  "n": 1 << 14, "k": [16, 32, 64, 128, 256, 512, 1024, 2048, 4096],
                  "largest": [True, False], "rev": [True, False], "dist": "uniform01"})
    cases.append({"kind": "topk_multitask_custom_idx", "cite": "test/test_algorithm.jl:42-96",
                  "task_lens": [1000, 2000, 1500, 500, 5000], "k": 64, "largest": True,
                  "rev": False, "indices": "global_1_based"})
    cases.append({"kind": "topk_overloads", "cite": "test/test_algorithm.jl:98-112",
                  "n": 1000, "k": 100})
    cases.append({"kind": "topk_batch_seq_idx", "cite": "test/test_algorithm.jl:114-150",
                  "task_lens": [1000, 1500, 800], "k": 50})
    cases.append({"kind": "topk_errors", "cite": "test/test_algorithm.jl:152-162",
                  "n": 1000, "bad_out_rows": 50, "k": 100, "bad_indices_len": 500})

    OUT.write_text(json.dumps({"source": "RadiK.jl test/ (transcribed)", "cases": cases},
                              indent=1) + "\n")
    print(f"wrote {OUT} ({len(cases)} cases)")


if __name__ == "__main__":
    main()
