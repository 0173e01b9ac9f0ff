"""Host-side argument checks of the low-level entry points, on the CPU.

topk_radix_select_ and topk_radix_select_noalloc_ hand raw pointers to
kernels that write len(task_lens) * k entries of each output and read
sum(task_lens) input elements (and custom indices).  A buffer shorter than
that must be refused with RadiKError before any device call, because on the
GPU it would become an out-of-bounds write rather than a Python error.  The
size checks come before the CUDA-placement checks, so CPU tensors show them
here without a GPU."""
from __future__ import annotations

import pytest
import torch

from conftest import load_package

LENS = [100, 50]
K = 8


def _bufs(n_out=len(LENS) * K, n_in=sum(LENS), n_idx=None):
    vo = torch.zeros(n_out, dtype=torch.float32)
    io = torch.zeros(n_out, dtype=torch.int32)
    x = torch.zeros(n_in, dtype=torch.float32)
    ind = None if n_idx is None else torch.zeros(n_idx, dtype=torch.int32)
    return vo, io, x, ind


@pytest.mark.parametrize("entry", ["topk_radix_select_", "topk_radix_select_noalloc_"])
def test_short_output_is_refused(entry):
    pkg = load_package()
    vo, io, x, _ = _bufs()
    short = torch.zeros(len(LENS) * K - 1, dtype=torch.float32)
    call = getattr(pkg, entry)
    args = (None,) if entry == "topk_radix_select_" else ()
    with pytest.raises(pkg.RadiKError, match=r"val_out holds 15 elements; 2 tasks x k = 8 needs 16"):
        call(short, io, *args, x, None, LENS, K)
    with pytest.raises(pkg.RadiKError, match=r"idx_out holds 15 elements"):
        call(vo, torch.zeros(15, dtype=torch.int32), *args, x, None, LENS, K)


@pytest.mark.parametrize("entry", ["topk_radix_select_", "topk_radix_select_noalloc_"])
def test_short_input_and_indices_are_refused(entry):
    pkg = load_package()
    call = getattr(pkg, entry)
    args = (None,) if entry == "topk_radix_select_" else ()
    vo, io, x, _ = _bufs(n_in=sum(LENS) - 1)
    with pytest.raises(pkg.RadiKError, match=r"val_in holds 149 elements; sum\(task_lens\) = 150 needs 150"):
        call(vo, io, *args, x, None, LENS, K)
    vo, io, x, ind = _bufs(n_idx=sum(LENS) - 2)
    with pytest.raises(pkg.RadiKError, match=r"idx_in holds 148 elements"):
        call(vo, io, *args, x, ind, LENS, K, True, True, False, True)
    vo, io, x, _ = _bufs()
    with pytest.raises(pkg.RadiKError, match="withidxin needs idx_in"):
        call(vo, io, *args, x, None, LENS, K, True, True, False, True)


def test_full_sized_cpu_tensors_reach_the_placement_check():
    """Correct sizes pass the size checks; CPU tensors are then refused as
    not being CUDA tensors (the engine has no CPU path)."""
    pkg = load_package()
    vo, io, x, _ = _bufs()
    with pytest.raises(pkg.RadiKError, match="must be a CUDA tensor"):
        pkg.topk_radix_select_noalloc_(vo, io, x, None, LENS, K)
