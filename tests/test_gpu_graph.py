"""CUDA-graph capture of the batched form: after RadiKWorkspace.prepare a
call with sync=False enqueues only memsets and kernels, so it can be
captured once and replayed on new data in the same input buffer."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lens,k,largest", [([65536] * 64, 256, True), ([1 << 20], 100, False),
                                            ([5000, 1, 70000, 300_000], 64, True)])
def test_captured_call_replays_on_new_data(oracle, radik, torch_cuda, lens, k, largest):
    torch = torch_cuda
    T, N = len(lens), sum(lens)
    x = torch.empty(N, device="cuda")
    vo = torch.empty((T, k), device="cuda")
    io = torch.empty((T, k), dtype=torch.int32, device="cuda")
    ws = radik.RadiKWorkspace("cuda", max(lens), T)
    ws.prepare(lens, k, largest=largest, ascend=True)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):  # warm-up outside the capture
        x.uniform_()
        radik.topk_radix_select_(vo, io, ws, x, None, lens, k, largest, True, sync=False)
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        radik.topk_radix_select_(vo, io, ws, x, None, lens, k, largest, True, sync=False)
    rng = np.random.default_rng(k)
    for _ in range(3):
        h = rng.standard_normal(N).astype(np.float32)
        x.copy_(torch.from_numpy(h))
        g.replay()
        torch.cuda.synchronize()
        ov, oi = oracle.topk(h, lens, k, largest=largest, rev=False)
        assert np.array_equal(vo.cpu().numpy().view(np.uint32), ov.view(np.uint32))
        assert np.array_equal(io.cpu().numpy().astype(np.int64), oi.astype(np.int64))
    assert ws.error_bits() == 0
    del g
    ws.close()


def test_capture_without_prepared_plan_is_refused(radik, torch_cuda):
    torch = torch_cuda
    x = torch.rand(4096, device="cuda")
    vo = torch.empty((1, 8), device="cuda")
    io = torch.empty((1, 8), dtype=torch.int32, device="cuda")
    ws = radik.RadiKWorkspace("cuda", 4096, 1)
    g = torch.cuda.CUDAGraph()
    with pytest.raises(radik.RadiKError, match="prepare"):
        with torch.cuda.graph(g):
            radik.topk_radix_select_(vo, io, ws, x, None, [4096], 8, True, True, sync=False)
    ws.close()
