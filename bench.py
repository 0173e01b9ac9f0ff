"""Benchmark of the B200 exact Float32 radix top-k (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config uniform_batch|adversarial_single|uneven_batch|single_1m|
                              rows64_k8192|rows256_k8192|serving] [--tune-file PATH]

A step is one batched top-k over the configuration's synthetic input (seeded,
shapes and distributions of the workload; no dataset exists):
  uniform_batch       1024 tasks x 65,536 Float32 U(0,1) (seed 1), k=256,
                      largest, one topk_radix_select! into (1024, 256) outputs
  adversarial_single  one task of 2^28 Float32 (seed 2): 50% from 1024 distinct
                      N(0,1) values, 40% in [1, 1+2^-10), 10% N(0,100^2);
                      k=4096, largest=false, rev=true
  uneven_batch        4096 tasks, lengths lognormal(median 20,000, sigma 1.5)
                      clamped to [1, 4,194,304] (seed 3), N(0,1), custom Int32
                      indices (a permutation), k=64, largest
  single_1m           one task of 2^20 N(0,1) (seed 0), k=100, largest
  rows64_k8192        64 tasks x 2^20 N(0,1), k=8192, largest (the serving
                      stream's heaviest request shape)
  rows256_k8192       256 tasks x 32,768 N(0,1), k=8192, largest (its
                      costliest shape per element)
  serving             the request server on a Poisson stream of top-k requests
                      (see run_serving)
`value` is elements/s with the inputs already in HBM (timed with CUDA events
on the launching stream, max over ranks); `e2e` is the same metric through the
host-buffer public entry point (pinned host input copied in and results copied
back every step).  A plain run (uniform_batch on one GPU) also carries the
rest of the metric as sub-blocks measured in the same run: the
`adversarial_single` task against the HBM roofline and the `serving` stream's
p50 / p99 beside the plain per-call path (--no-extra leaves them out).
Multi-GPU runs give every GPU the per-GPU batch (weak scaling): the job's
tasks are sharded by element count (multi.local_shard), with no collective on
the data path.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
L2_BYTES = 126 * 1024 * 1024


def load_package():
    import importlib.util
    if "radik_b200" in sys.modules:
        return sys.modules["radik_b200"]
    pkg = ROOT / "radik.jl_b200"
    spec = importlib.util.spec_from_file_location("radik_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["radik_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle  # the CPU baseline only
    sys.path.pop(0)
    return oracle


# ---------------------------------------------------------------------------
# Workloads
# ---------------------------------------------------------------------------
CONFIGS = {
    "uniform_batch": dict(k=256, largest=True, rev=False, custom_idx=False),
    "adversarial_single": dict(k=4096, largest=False, rev=True, custom_idx=False),
    "uneven_batch": dict(k=64, largest=True, rev=False, custom_idx=True),
    # The reference's CPU-runnable case: one task of 2^20 N(0,1), seed 0.
    "single_1m": dict(k=100, largest=True, rev=False, custom_idx=False),
    # The serving stream's heaviest request shape: 64 rows of 2^20 N(0,1),
    # k = 8192 (sampled thresholds, the merge and rank kernels, radix sorts).
    "rows64_k8192": dict(k=8192, largest=True, rev=False, custom_idx=False),
    # The serving stream's costliest shape per element: 256 rows of 32,768
    # N(0,1), k = 8192 (a quarter of each row; the barrier form and its sort).
    "rows256_k8192": dict(k=8192, largest=True, rev=False, custom_idx=False),
}


def task_lens_of(name: str) -> list[int]:
    if name == "uniform_batch":
        return [65536] * 1024
    if name == "adversarial_single":
        return [1 << 28]
    if name == "single_1m":
        return [1 << 20]
    if name == "rows64_k8192":
        return [1 << 20] * 64
    if name == "rows256_k8192":
        return [1 << 15] * 256
    rng = np.random.default_rng(3)
    v = np.clip(np.round(rng.lognormal(np.log(20000), 1.5, size=4096)), 1, 4_194_304)
    return [int(x) for x in v]


def make_input_np(name: str, N: int, seed_offset: int = 0) -> np.ndarray:
    if name == "uniform_batch":
        return np.random.default_rng(1 + seed_offset).random(N, dtype=np.float32)
    if name == "adversarial_single":
        rng = np.random.default_rng(2 + seed_offset)
        pool = rng.standard_normal(1024).astype(np.float32)
        u = rng.random(N, dtype=np.float32)
        out = np.empty(N, np.float32)
        a = u < 0.5
        b = (u >= 0.5) & (u < 0.9)
        c = u >= 0.9
        out[a] = pool[rng.integers(0, 1024, size=int(a.sum()))]
        out[b] = (1.0 + rng.random(int(b.sum()), dtype=np.float32) * np.float32(2.0 ** -10)).astype(np.float32)
        out[c] = (rng.standard_normal(int(c.sum())).astype(np.float32) * np.float32(100.0))
        return out
    if name == "single_1m":
        return np.random.default_rng(seed_offset).standard_normal(N).astype(np.float32)
    return np.random.default_rng(3 + seed_offset).standard_normal(N).astype(np.float32)


def make_input_dev(torch, name: str, N: int, seed: int):
    """Same distributions generated on the device (fast for 2^28 elements)."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    if name == "uniform_batch":
        return torch.rand(N, device="cuda", generator=g)
    if name == "adversarial_single":
        pool = torch.randn(1024, device="cuda", generator=g)
        u = torch.rand(N, device="cuda", generator=g)
        a = pool[torch.randint(0, 1024, (N,), device="cuda", generator=g)]
        b = 1.0 + torch.rand(N, device="cuda", generator=g) * (2.0 ** -10)
        c = torch.randn(N, device="cuda", generator=g) * 100.0
        return torch.where(u < 0.5, a, torch.where(u < 0.9, b, c)).contiguous()
    return torch.randn(N, device="cuda", generator=g)


# ---------------------------------------------------------------------------
# Clocks (sampled during the timed region)
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic(config: str):
    p = ROOT / "profiles" / "traffic.json"
    try:
        d = json.loads(p.read_text())
        v = d.get(config)
        return v if isinstance(v, (int, float)) else None
    except (OSError, ValueError):
        return None


# ---------------------------------------------------------------------------
# Arms
# ---------------------------------------------------------------------------
def run_reference(args, rank: int, world: int):
    """CPU arm: the oracle port of the reference algorithm on all host
    threads, over a bounded sample of the same workload per step."""
    if rank != 0:
        return
    oracle = load_oracle()
    if args.config == "serving":
        run_reference_serving(args, oracle, world)
        return
    cfg = CONFIGS[args.config]
    lens = task_lens_of(args.config)
    threads = oracle.max_threads()
    if args.config == "uniform_batch":
        sample_lens = lens[:64]
        sample = f"64 of the 1024 tasks ({64 * 65536} elements) per step"
    elif args.config == "adversarial_single":
        sample_lens = [1 << 22]
        sample = "a 2^22-element prefix task of the same mixture per step"
    elif args.config == "single_1m":
        sample_lens = lens
        sample = "the whole 2^20-element task per step"
    elif args.config == "rows64_k8192":
        sample_lens = lens[:4]
        sample = "4 of the 64 rows per step"
    elif args.config == "rows256_k8192":
        sample_lens = lens[:32]
        sample = "32 of the 256 rows per step"
    else:
        sample_lens = lens[:256]
        sample = "the first 256 of the 4096 tasks per step"
    N = int(sum(sample_lens))
    x = make_input_np(args.config, N)
    ind = np.arange(N, dtype=np.int32) if cfg["custom_idx"] else None
    for _ in range(args.warmup):
        oracle.topk(x, sample_lens, cfg["k"], largest=cfg["largest"], rev=cfg["rev"], indices=ind, threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.topk(x, sample_lens, cfg["k"], largest=cfg["largest"], rev=cfg["rev"], indices=ind, threads=threads)
    dt = (time.perf_counter() - t0) / max(args.steps, 1)
    value = N / dt
    line = {
        "impl": "reference", "metric": "elements/s", "value": value, "unit": "elements/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.config, "task_lens": "see bench.py", "k": cfg["k"],
                   "largest": cfg["largest"], "rev": cfg["rev"]},
        "cpu_baseline": {"value": value, "unit": "elements/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "RadiK.jl is Julia; no Julia toolchain on this machine, so the reference arm is the C "
                "restatement of its algorithm (oracle/) on the host cores",
    }
    print(json.dumps(line), flush=True)


def run_reference_serving(args, oracle, world):
    """CPU arm of the serving stream: the oracle port on the host cores,
    requests served one after another, on a bounded sample (the first 6
    requests of the stream, rows capped at 8)."""
    rng = np.random.default_rng(4)
    shapes = [(min(r, 8), l, k) for r, l, k in serving_requests(rng, 6)]
    threads = oracle.max_threads()
    data = np.random.default_rng(5).standard_normal(max(r * l for r, l, _ in shapes)).astype(np.float32)
    for r, l, k in shapes[:1]:
        oracle.topk(data[: r * l], [l] * r, min(k, l), largest=True, rev=False, threads=threads)
    steps = max(args.steps, 1)
    t0 = time.perf_counter()
    elems = 0
    for _ in range(steps):
        for r, l, k in shapes:
            oracle.topk(data[: r * l], [l] * r, min(k, l), largest=True, rev=False, threads=threads)
            elems += r * l
    dt = time.perf_counter() - t0
    value = elems / dt
    print(json.dumps({
        "impl": "reference", "metric": "elements/s", "value": value, "unit": "elements/s", "n_gpus": world,
        "steps": steps, "warmup": 1, "ms_per_step": dt * 1e3 / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "serving_stream"},
        "cpu_baseline": {"value": value, "unit": "elements/s", "cores": threads, "kind": "port",
                         "sample": "first 6 requests of the serving stream, rows capped at 8, served in order"},
        "e2e": {"value": value, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def cpu_baseline_quick(args, config: str) -> dict:
    """Bounded CPU sample (oracle port, all host threads) for the JSON line."""
    oracle = load_oracle()
    cfg = CONFIGS[config]
    lens = task_lens_of(config)
    if config == "uniform_batch":
        sl, sample = lens[:64], "64 of the 1024 tasks, 3 repetitions"
    elif config == "adversarial_single":
        sl, sample = [1 << 22], "one 2^22-element task of the same mixture, 3 repetitions"
    elif config == "single_1m":
        sl, sample = lens, "the whole 2^20-element task, 3 repetitions"
    elif config == "rows64_k8192":
        sl, sample = lens[:4], "4 of the 64 rows, 3 repetitions"
    elif config == "rows256_k8192":
        sl, sample = lens[:32], "32 of the 256 rows, 3 repetitions"
    else:
        sl, sample = lens[:256], "first 256 of the 4096 tasks, 3 repetitions"
    N = int(sum(sl))
    x = make_input_np(config, N)
    threads = oracle.max_threads()
    oracle.topk(x, sl, cfg["k"], largest=cfg["largest"], rev=cfg["rev"], threads=threads)
    t0 = time.perf_counter()
    for _ in range(3):
        oracle.topk(x, sl, cfg["k"], largest=cfg["largest"], rev=cfg["rev"], threads=threads)
    dt = (time.perf_counter() - t0) / 3
    return {"value": N / dt, "unit": "elements/s", "cores": threads, "kind": "port", "sample": sample,
            "select_sort": select_sort_baseline(x, sl, cfg["k"], cfg["largest"])}


def select_sort_baseline(x: np.ndarray, lens, k: int, largest: bool) -> dict:
    """A generic CPU top-k for scale: per task an introselect partition
    (numpy argpartition, the algorithm of std::nth_element) and a sort of the
    k selected, one thread.  Its ties at the k-th value are not the lowest
    positions, so it is a speed reference only, not a result to compare."""
    def once():
        a = 0
        for n in lens:
            n = int(n)
            v = x[a:a + n]
            kk = min(k, n)
            if kk < n:
                sel = np.argpartition(v, n - kk)[n - kk:] if largest else np.argpartition(v, kk - 1)[:kk]
            else:
                sel = np.arange(n)
            sel[np.argsort(v[sel], kind="stable")]
            a += n
    once()
    t0 = time.perf_counter()
    for _ in range(3):
        once()
    dt = (time.perf_counter() - t0) / 3
    return {"value": int(sum(lens)) / dt, "unit": "elements/s", "cores": 1,
            "method": "numpy argpartition (introselect) + sort of the k, per task"}


def load_multi():
    load_package()
    import importlib
    return importlib.import_module("radik_b200.multi")


def run_ours(args, rank: int, world: int, dist, config: str | None = None, *, e2e_on: bool = True,
             plain_on: bool = True, cpu_on: bool = True) -> dict | None:
    """One workload on this rank's GPU; returns rank 0's line (None elsewhere).

    The job's batch is `world` copies of the workload's per-GPU batch (weak
    scaling: per-GPU work is fixed as N grows), sharded over the ranks by
    element count with multi.local_shard -- the partition the multi-GPU
    module uses, with no collective on the data path.  Each rank builds only
    its own shard."""
    import torch
    radik = load_package()
    multi = load_multi()
    config = config or args.config
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    cfg = CONFIGS[config]
    job_lens = np.tile(np.asarray(task_lens_of(config), dtype=np.int64), world)
    t0, t1, _, _ = multi.local_shard(job_lens, world, rank)
    # Task lengths as an int64 array, as a caller that reuses a batch shape
    # keeps them (a Python list is converted on every call).
    lens = np.ascontiguousarray(job_lens[t0:t1])
    T, k, N = len(lens), cfg["k"], int(lens.sum())
    # Inputs: enough rotating copies that the bytes touched between two reads
    # of the same buffer exceed the L2 several times.
    nbuf = max(2, int(np.ceil(3 * L2_BYTES / (4 * N))) + 1)
    xs = [make_input_dev(torch, config, N, seed=1000 * rank + i + 1) for i in range(nbuf)]
    ind = None
    if cfg["custom_idx"]:
        g = torch.Generator(device="cuda")
        g.manual_seed(7 + rank)
        ind = torch.randperm(N, device="cuda", generator=g).to(torch.int32)
    vo = torch.empty((T, k), dtype=torch.float32, device="cuda")
    io = torch.empty((T, k), dtype=torch.int32, device="cuda")
    ws = radik.RadiKWorkspace("cuda", max(lens), T)
    stream = torch.cuda.current_stream()
    # Pick the fastest configuration for this batch shape (untimed set-up);
    # it also prepares the plan.  With --tune-file, a table saved by an
    # earlier run decides instead (same plan under a profiler), or this run's
    # choice is saved there.
    main_run = config is None or config == args.config
    tune_file = pathlib.Path(args.tune_file) if (getattr(args, "tune_file", None) and main_run) else None
    if tune_file is not None and tune_file.exists():
        radik.tune_load(tune_file)
        tuned = {"ms": None, "loaded_from": str(tune_file)}
    else:
        tuned = ws.autotune(vo, io, xs[0], ind, lens, k, cfg["largest"], not cfg["rev"], False, ind is not None,
                            reps=10, stream=stream)
        if tune_file is not None and rank == 0:
            radik.tune_save(tune_file)

    def step(i):
        radik.topk_radix_select_(vo, io, ws, xs[i % nbuf], ind, lens, k, cfg["largest"], not cfg["rev"],
                                 False, ind is not None, sync=False, stream=stream)

    def barrier():
        if dist is not None:
            dist.barrier()

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if ws.error_bits():
        raise RuntimeError("device error during warm-up")
    plan = ws.plan_info()

    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # Per-step events made before the timed region: creating them inside it
    # costs host time that would show as gaps between the steps.
    per = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    # The timed steps run back to back with nothing between them (an event
    # between two calls would stop the next call's first kernel from being
    # launched programmatically behind the previous call's last).
    ev0.record(stream)
    for i in range(args.steps):
        step(i)
    ev1.record(stream)
    torch.cuda.synchronize()
    # The same K steps again, each bracketed by its own events: the launch
    # durations of the roofline below.
    for i in range(args.steps):
        a, b = per[i]
        a.record(stream)
        step(args.steps + i)
        b.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    total_ms = ev0.elapsed_time(ev1)
    launch_ms = [a.elapsed_time(b) for a, b in per]
    if ws.error_bits():
        raise RuntimeError("device error during the timed steps")
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    n_job = int(job_lens.sum())
    value = n_job / (ms_per_step * 1e-3)

    # Roofline of the dominant kernel (the fused single-read kernel is the
    # only kernel of a step): algorithmic bytes = one read of the input +
    # the (value, index) outputs (+ the gathered custom indices).
    idx_b = 4
    alg_bytes = 4 * N + (4 + idx_b) * T * k + (idx_b * T * k if ind is not None else 0)
    avg_launch_s = statistics.mean(launch_ms) * 1e-3
    peak, peak_kind = measured_peak_hbm()
    achieved = alg_bytes / avg_launch_s / 1e9
    kernel = {0: "fused_topk_kernel", 1: "fused_ws_kernel", 2: "multi-pass kernels"}[plan["path"]]
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": profile_traffic(config), "peak_source": peak_kind,
                "kernel": kernel, "algorithmic_bytes_per_launch": alg_bytes,
                "timing": "CUDA events around each of a second pass of the K steps (the launch's kernels)"}

    # The same step captured once in a CUDA graph and replayed (the plan was
    # prepared, so the call enqueues only memsets and kernels).
    graph = None
    try:
        side = torch.cuda.Stream()
        side.wait_stream(stream)
        with torch.cuda.stream(side):
            step(0)
        stream.wait_stream(side)
        torch.cuda.synchronize()
        graphs = []
        for b in range(nbuf):  # one graph per rotating input buffer
            cg = torch.cuda.CUDAGraph()
            with torch.cuda.graph(cg):
                radik.topk_radix_select_(vo, io, ws, xs[b], ind, lens, k, cfg["largest"], not cfg["rev"], False,
                                         ind is not None, sync=False)
            graphs.append(cg)
        for i in range(3):
            graphs[i % nbuf].replay()
        torch.cuda.synchronize()
        ga, gb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ga.record(stream)
        for i in range(args.steps):
            graphs[i % nbuf].replay()
        gb.record(stream)
        torch.cuda.synchronize()
        gms = ga.elapsed_time(gb) / args.steps
        graph = {"ms_per_step": gms, "value": n_job / (gms * 1e-3),
                 "note": f"the call captured once per input buffer ({nbuf}) and replayed in rotation"}
        del graphs
    except Exception as exc:  # report, do not fail the benchmark
        graph = {"error": repr(exc)[:200]}

    # End to end through the host-buffer entry point (pinned host memory).
    e2e = None
    if e2e_on and not args.no_e2e:
        hx = torch.empty(N, dtype=torch.float32, pin_memory=True)
        hx.copy_(xs[0].cpu())
        hx_np = hx.numpy()
        hv = torch.empty((T, k), dtype=torch.float32, pin_memory=True).numpy()
        hi = torch.empty((T, k), dtype=torch.int32, pin_memory=True).numpy()
        hind = None
        if ind is not None:
            hind_t = torch.empty(N, dtype=torch.int32, pin_memory=True)
            hind_t.copy_(ind.cpu())
            hind = hind_t.numpy()
        ws_e = radik.RadiKWorkspace("cuda", max(lens), T)
        e_steps = max(2, min(args.steps, 10))
        for _ in range(2):
            radik.topk_host(hx_np, lens, k, indices=hind, largest=cfg["largest"], rev=cfg["rev"], ws=ws_e,
                            out=(hv, hi))
        barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(e_steps):
            radik.topk_host(hx_np, lens, k, indices=hind, largest=cfg["largest"], rev=cfg["rev"], ws=ws_e,
                            out=(hv, hi), stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        e_ms = torch.tensor([a.elapsed_time(b) / e_steps], dtype=torch.float64, device="cuda")
        if dist is not None:
            dist.all_reduce(e_ms, op=dist.ReduceOp.MAX)
        h2d = 4 * N + (4 * N if hind is not None else 0)
        e2e = {"value": n_job / (float(e_ms.item()) * 1e-3), "unit": "elements/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": (4 + idx_b) * T * k,
               "steps": e_steps, "ms_per_step": float(e_ms.item())}
        ws_e.close()

    # Plain per-call path: the reference's launch structure (multi-pass
    # histogram / select / compact passes with host reads between passes) on
    # the same batch, with a workspace reused across calls ("reused_ws"), and
    # as topk! runs it with a fresh workspace allocated per call (src/algorithm.jl:503).
    plain = None
    if plain_on and not args.no_plain and rank == 0:
        ws_p = radik.RadiKWorkspace("cuda", max(lens), T)
        for i in range(2):
            radik.topk_radix_select_(vo, io, ws_p, xs[i % nbuf], ind, lens, k, cfg["largest"], not cfg["rev"],
                                     False, ind is not None, plain=True)
        torch.cuda.synchronize()
        ncall = 5
        t0 = time.perf_counter()
        for i in range(ncall):
            radik.topk_radix_select_(vo, io, ws_p, xs[i % nbuf], ind, lens, k, cfg["largest"], not cfg["rev"],
                                     False, ind is not None, plain=True)
        torch.cuda.synchronize()
        pdt = (time.perf_counter() - t0) / ncall
        ws_p.close()
        t0 = time.perf_counter()
        radik.topk_(vo, io, xs[0], lens, k, indices=ind, largest=cfg["largest"], rev=cfg["rev"], plain=True)
        torch.cuda.synchronize()
        fdt = time.perf_counter() - t0
        plain = {"value": N / pdt, "unit": "elements/s", "ms_per_call": pdt * 1e3,
                 "path": "multi-pass launch structure per call, workspace reused, host syncs between passes",
                 "fresh_workspace": {"value": N / fdt, "ms_per_call": fdt * 1e3,
                                     "path": "topk! shape: workspace allocated and freed in the call"}}

    cpu = cpu_baseline_quick(args, config) if (cpu_on and rank == 0 and world == 1 and not args.no_cpu) else None
    ws.close()
    del xs
    torch.cuda.empty_cache()
    if rank != 0:
        return None
    return {
        "metric": "elements/s", "value": value, "unit": "elements/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": config, "tasks_per_gpu": T, "elements_per_gpu": N, "job_elements": n_job, "k": k,
                   "largest": cfg["largest"], "rev": cfg["rev"], "custom_indices": ind is not None,
                   "l2": f"inputs larger than L2: {nbuf} rotating input buffers of {4 * N} bytes",
                   "parallelism": f"{world} GPU(s): the job's {len(job_lens)} tasks sharded by element count "
                                  "(multi.local_shard), no collective on the data path"},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
        "gpu_launches": plan["kernels_per_call"] * args.steps, "plan": plan, "autotune_ms": tuned["ms"],
        "plain_per_call": plain,
        "graph_replay": graph,
    }


# ---------------------------------------------------------------------------
# Serving stream (request server, continuous batching)
# ---------------------------------------------------------------------------
SERVING_LOADS = (1000, 5000, 20000, 50000)  # offered requests per second
SERVING_REQUESTS = 1000                     # requests per offered load and repeat
SERVING_REPEATS = 3                         # repeats per load (the spread of p50 / p99 is reported)


def serving_requests(rng, n):
    """Request shapes of the serving stream: rows U{1..512}, row length from
    {32768, 131072, 1048576}, k from {1, 50, 1024, 8192}."""
    rows = rng.integers(1, 513, size=n)
    lens = rng.choice([32768, 131072, 1048576], size=n)
    ks = rng.choice([1, 50, 1024, 8192], size=n)
    return [(int(r), int(l), int(k)) for r, l, k in zip(rows, lens, ks)]


def _pct(xs, q):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(round(q * (len(xs) - 1))))] if xs else None


def _spread(vals):
    return {"median": statistics.median(vals), "min": min(vals), "max": max(vals)}


def run_serving(args, rank: int, world: int, dist, *, requests: int = SERVING_REQUESTS,
                repeats: int = SERVING_REPEATS) -> dict | None:
    """Poisson arrivals (seed 4) at each offered load; every request is a
    [rows, row_len] slice of a device-resident pool of N(0,1) logits with a
    Gumbel(0,1) tail on 1% of entries, k largest per row.  The server packs
    requests into fused launches on 4 slots under a 32 GB admission cap.
    Reported per load and repeat: achieved requests/s and elements/s,
    p50/p99 latency from submission to completion; beside it the same
    arrival schedule served one request at a time by the plain per-call path
    (the reference's launch structure, workspace reused).  Per load, the
    median and range over the repeats, and the served latency by request
    shape (row length x k) over all repeats."""
    import torch
    radik = load_package()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    g = torch.Generator(device="cuda")
    g.manual_seed(4 + rank)
    pool_n = 1 << 29  # 2 GiB of logits: the largest request (512 x 2^20) fits
    pool = torch.randn(pool_n, device="cuda", generator=g)
    tail = torch.rand(pool_n, device="cuda", generator=g) < 0.01
    u = torch.rand(pool_n, device="cuda", generator=g).clamp_(1e-12, 1.0)
    pool += torch.where(tail, -torch.log(-torch.log(u)), torch.zeros_like(u))
    del tail, u
    rng = np.random.default_rng(4)
    loads = []
    clocks = ClockSampler(local)
    clocks.start()
    ws = radik.RadiKWorkspace("cuda", 1 << 20, 512)
    with radik.Server(slots=4, mem_cap_bytes=32 << 30, max_batch_rows=4096) as srv:
        # warm the slots' workspaces on every shape class
        for r, l, k in [(4, 32768, 1), (4, 131072, 50), (2, 1048576, 1024), (2, 131072, 8192)]:
            srv.wait(srv.submit(pool[: r * l].view(r, l), k), timeout_s=120)
        for load in SERVING_LOADS:
            reps = []
            by_shape = {}
            by_k = {}
            for _ in range(repeats):
                shapes = serving_requests(rng, requests)
                gaps = rng.exponential(1.0 / load, size=len(shapes))
                offs = [int(rng.integers(0, (pool_n - r * l) // 4 + 1)) * 4 for r, l, _ in shapes]
                outs = [(torch.empty((r, k), device="cuda"), torch.empty((r, k), dtype=torch.int32, device="cuda"))
                        for r, _, k in shapes]
                torch.cuda.synchronize()
                srv.reset_stats()
                t0 = time.perf_counter()
                due = t0
                tickets = []
                for (r, l, k), off, gap, (vo, io) in zip(shapes, offs, gaps, outs):
                    due += gap
                    while time.perf_counter() < due:
                        pass
                    tickets.append(srv.submit(pool[off: off + r * l].view(r, l), k, val_out=vo, idx_out=io))
                for t in tickets:
                    srv.wait(t, timeout_s=300)
                dt = time.perf_counter() - t0
                st = srv.stats()
                lat = srv.latencies()
                for bt in srv.batches():
                    agg = by_k.setdefault(int(bt["k"]), {"batches": 0, "rows": 0, "elements": 0.0, "gpu_us": 0.0,
                                                         "launch_us": 0.0})
                    agg["batches"] += 1
                    agg["rows"] += int(bt["rows"])
                    agg["elements"] += bt["elements"]
                    agg["gpu_us"] += bt["gpu_us"]
                    agg["launch_us"] += bt["launch_us"]
                for t, (r, l, k) in zip(tickets, shapes):
                    by_shape.setdefault(f"{l}x{k}", []).append(lat[t])
                elems = sum(r * l for r, l, _ in shapes)
                # plain per-call path on the same schedule, one request at a time
                plat = []
                t1 = time.perf_counter()
                due = t1
                for (r, l, k), off, gap, (vo, io) in zip(shapes, offs, gaps, outs):
                    due += gap
                    while time.perf_counter() < due:
                        pass
                    radik.topk_radix_select_(vo, io, ws, pool[off: off + r * l], None, [l] * r, k, True, True,
                                             plain=True)
                    plat.append((time.perf_counter() - due) * 1e6)
                pdt = time.perf_counter() - t1
                del outs
                reps.append({
                    "served": {"req_s": len(shapes) / dt, "elements_s": elems / dt, "p50_us": st["p50_us"],
                               "p99_us": st["p99_us"], "batches": st["batches"]},
                    "plain_per_call": {"req_s": len(shapes) / pdt, "elements_s": elems / pdt,
                                       "p50_us": _pct(plat, 0.50), "p99_us": _pct(plat, 0.99)},
                })
            loads.append({
                "offered_req_s": load, "requests_per_repeat": requests, "repeats": reps,
                "served": {key: _spread([r["served"][key] for r in reps])
                           for key in ("req_s", "elements_s", "p50_us", "p99_us")},
                "plain_per_call": {key: _spread([r["plain_per_call"][key] for r in reps])
                                   for key in ("req_s", "elements_s", "p50_us", "p99_us")},
                "served_by_shape": {key: {"n": len(v), "p50_us": _pct(v, 0.5), "p99_us": _pct(v, 0.99)}
                                    for key, v in sorted(by_shape.items())},
                # launched batches by k over all repeats: device time (each batch timed on its slot's
                # stream; slots overlap) and the worker's host time to launch them
                "batches_by_k": {str(kk): dict(v, device_elements_s=v["elements"] / max(v["gpu_us"], 1e-9) * 1e6,
                                               launch_us_mean=v["launch_us"] / max(v["batches"], 1))
                                 for kk, v in sorted(by_k.items())},
            })
    ws.close()
    clk = clocks.stop()
    del pool
    torch.cuda.empty_cache()
    if rank != 0:
        return None
    best = max(loads, key=lambda x: x["served"]["elements_s"]["median"])
    return {
        "metric": "elements/s", "value": best["served"]["elements_s"]["median"] * world, "unit": "elements/s",
        "n_gpus": world, "steps": len(SERVING_LOADS) * requests * repeats, "warmup": 4,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "serving_stream", "loads_req_s": list(SERVING_LOADS),
                   "requests_per_load": requests, "repeats": repeats, "slots": 4, "mem_cap_bytes": 32 << 30,
                   "rows": "U{1..512}", "row_len": [32768, 131072, 1048576], "k": [1, 50, 1024, 8192],
                   "arrivals": "Poisson, seed 4", "parallelism": f"replicas x{world}"},
        "loads": loads, "clocks": clk,
        # each packed batch launches at least one kernel (sampling, merge and retry add more)
        "gpu_launches": int(sum(r["served"]["batches"] for x in loads for r in x["repeats"])),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="uniform_batch", choices=sorted(CONFIGS) + ["serving"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true",
                    help="uniform_batch on one GPU without the adversarial_single and serving sub-blocks")
    ap.add_argument("--tune-file", default=None,
                    help="tuning table: loaded instead of autotuning when it exists, else written after it")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        if args.config == "serving":
            line = run_serving(args, rank, world, dist)
        else:
            line = run_ours(args, rank, world, dist)
            if line is not None and args.config == "uniform_batch" and world == 1 and not args.no_extra:
                # The rest of the metric, measured in the same run: the 2^28
                # adversarial task against the HBM roofline, and the serving
                # stream's p50 / p99 against the plain per-call path.
                adv = run_ours(args, rank, world, dist, "adversarial_single", e2e_on=False, plain_on=False,
                               cpu_on=False)
                line["adversarial_single"] = {key: adv[key] for key in (
                    "value", "unit", "ms_per_step", "steps", "config", "roofline", "graph_replay", "plan",
                    "clocks", "gpu_launches")}
                srv = run_serving(args, rank, world, dist)
                line["serving"] = {key: srv[key] for key in ("value", "unit", "config", "loads", "clocks",
                                                            "gpu_launches")}
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
