"""Shared test fixtures.

The package directory is ``radik.jl_b200`` (a dot in the name), so it is
loaded by path and registered as ``radik_b200``.  The oracle under oracle/ is
loaded only here, as the checker.
"""
from __future__ import annotations

import importlib.util
import json
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
PKG_DIR = ROOT / "radik.jl_b200"
GOLDEN = ROOT / "tests" / "golden" / "reference_known_answers.json"


def load_package():
    if "radik_b200" in sys.modules:
        return sys.modules["radik_b200"]
    spec = importlib.util.spec_from_file_location("radik_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["radik_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    try:
        import oracle  # noqa: E402
    finally:
        sys.path.pop(0)
    return oracle


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    return load_oracle()


@pytest.fixture(scope="session")
def golden():
    return json.loads(GOLDEN.read_text())["cases"]


@pytest.fixture(scope="session")
def radik():
    """The engine package with its library loaded; builds the library if it
    is missing (GPU tests only)."""
    build = importlib.util.spec_from_file_location("radik_b200_build", PKG_DIR / "build.py")
    bmod = importlib.util.module_from_spec(build)
    build.loader.exec_module(bmod)
    bmod.build()
    return load_package()


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def task_data(spec) -> np.ndarray:
    """Materialise a fixture task description ({"range": [a, b]} or a list)."""
    if isinstance(spec, dict) and "range" in spec:
        a, b = spec["range"]
        return np.arange(a, b + 1, dtype=np.float32)
    return np.asarray(spec, dtype=np.float32)


def expected_values(spec) -> np.ndarray:
    if isinstance(spec, dict) and "range" in spec:
        a, b = spec["range"]
        return np.arange(a, b + 1, dtype=np.float32)
    return np.asarray(spec, dtype=np.float32)


def plain_topk(data, task_lens, k, largest=True, rev=False, withscale=False, indices=None):
    """Independent numpy top-k (sort based) with the engine's tie and order
    rules, used to cross-check the oracle: NaN is the substitute value, keys
    order -0 < +0, ties at the k-th score go to the lowest positions, the
    output is sorted by value key (ascending unless rev) then position."""
    data = np.asarray(data, dtype=np.float32)
    T = len(task_lens)
    vo = np.zeros((T, k), np.float32)
    io = np.zeros((T, k), np.int64 if indices is None else np.asarray(indices).dtype)
    fmin, fmax = np.finfo(np.float32).tiny, np.finfo(np.float32).max
    off = 0
    for t, n in enumerate(task_lens):
        x = data[off:off + n]
        sub = np.where(np.isnan(x), np.float32(fmin if largest else fmax), x).astype(np.float32)
        s = sub
        if withscale and n > 0:
            sc = x[0] if np.isfinite(x[0]) else np.float32(0)
            s = (sub - np.float32(sc)).astype(np.float32)
        key = _np_key(s)
        score = key if largest else ~key
        pos = np.arange(n, dtype=np.int64)
        if n > k:
            order = np.lexsort((pos, -score.astype(np.int64)))
            win = order[:k]
        else:
            win = pos
        okey = _np_key(sub[win]).astype(np.int64)
        if rev:
            okey = -okey
        srt = win[np.lexsort((win, okey))]
        m = len(srt)
        vo[t, :m] = x[srt]
        io[t, :m] = (srt + 1) if indices is None else np.asarray(indices)[off + srt]
        vo[t, m:] = 0
        io[t, m:] = -1
        off += n
    return vo, io


def _np_key(x):
    b = np.asarray(x, dtype=np.float32).view(np.uint32)
    with np.errstate(over="ignore"):
        mask = ((~(b >> np.uint32(31))) + np.uint32(1)) | np.uint32(0x80000000)
    return (b ^ mask).astype(np.uint32)
