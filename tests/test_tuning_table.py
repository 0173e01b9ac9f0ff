"""The process-wide tuning table (radik_tune_save / radik_tune_load /
radik_tune_clear): host-only, so these run without a GPU."""
from __future__ import annotations

import pytest

LINE_A = "1234567890123 26 1260007 128 13 4 1 128 8 8 2048 3 -1 0 0"
LINE_B = "987654321 4096 80000000 64 29 8 -1 128 8 8 2048 3 -1 0 2"
LINE_C = "555 256 8388608 8192 3 4 0 128 8 8 2048 3 -1 0 0 512"  # with the barrier form's block size


def test_tuning_table_round_trip(radik, tmp_path):
    radik.tune_clear()
    src = tmp_path / "in.txt"
    src.write_text("# a comment\n" + LINE_A + "\nnot a line\n" + LINE_B + "\n" + LINE_C + "\n"
                   "5 1 1 1 1 4 1 128 8 8 2048 3 -1 0 9\n"  # schedule 9 does not exist: skipped
                   "6 1 1 1 1 4 0 128 8 8 2048 3 -1 0 0 384\n")  # no 384-thread barrier block: skipped
    assert radik.tune_load(src) == 3
    out = tmp_path / "out.txt"
    radik.tune_save(out)
    rows = [l for l in out.read_text().splitlines() if not l.startswith("#")]
    assert rows == [LINE_A, LINE_B, LINE_C]
    # loading the same shapes again replaces, not duplicates
    assert radik.tune_load(src) == 3
    radik.tune_save(out)
    assert [l for l in out.read_text().splitlines() if not l.startswith("#")] == [LINE_A, LINE_B, LINE_C]
    radik.tune_clear()
    radik.tune_save(out)
    assert [l for l in out.read_text().splitlines() if not l.startswith("#")] == []


def test_tuning_table_errors(radik, tmp_path):
    with pytest.raises(radik.RadiKError, match="cannot read"):
        radik.tune_load(tmp_path / "missing.txt")
    with pytest.raises(radik.RadiKError, match="cannot write"):
        radik.tune_save(tmp_path / "no_such_dir" / "t.txt")
