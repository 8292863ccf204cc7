#!/usr/bin/env python3
"""Benchmark of the per-trial Monte Carlo path on B200.

Workload (a "step"): one batch of 2^20 trials of the plain GPU configuration
N = 2^20 keys (ell_i 20), t = 1024 items, k = 3, B = 1536 buckets, max 500
kicks, BGH25 random walk, affine distinct inputs, seed 2, BT = 20.  Step s on
rank r evaluates batch r + s*N_ranks, so every step is new work.

Prints one JSON line (rank 0).  `value` is whole-job trials/s from CUDA
events around the engine launches on device-resident inputs; `e2e` is the same
metric through the C ABI call cmc_launch with host buffers (batch key in,
sorted failure offsets out, copies inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "pbc-based-dmpf-monte-carlo-test_b200"

# Single-configuration workloads (one launch per step over one batch's trials).
WORKLOADS = {
    "config2": dict(workload="plain GPU: N=2^20 keys, t=1024, k=3, B=1536, kick=500, bgh25, "
                             "affine inputs, seed 2, batches of 2^20 trials",
                    mode="bgh25", input_mode="affine", pnum=1024, ell_i=20, k=3, buckets=1536,
                    kick=500, seed=2, bt=20, trials=1 << 20),
    "config1": dict(workload="plain method: N=2^16 keys, t=64, k=3, B=96, kick=100, bgh25, "
                             "affine inputs, seed 1, batches of 2^16 trials",
                    mode="bgh25", input_mode="affine", pnum=64, ell_i=16, k=3, buckets=96,
                    kick=100, seed=1, bt=16, trials=1 << 16),
    "config4": dict(workload="large table: N=2^28 keys, t=16384, k=3, B=24576, kick=1000, bgh25, "
                             "affine inputs, seed 4, batches of 2^24 trials (first 2^16 of each "
                             "per step)",
                    mode="bgh25", input_mode="affine", pnum=16384, ell_i=28, k=3, buckets=24576,
                    kick=1000, seed=4, bt=24, trials=1 << 16),
}
WORKLOAD = WORKLOADS["config2"]
METRIC = "trials/s per B200 (bit-exact failures)"
AES_BYTES_PER_BLOCK = 640      # 160 table lookups x 4 bytes
SMEM_BYTES_PER_CLK_PER_SM = 128


def load_pkg():
    import importlib.util
    spec = importlib.util.spec_from_file_location("cmc_b200", PKG_DIR / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cmc_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def algorithmic_blocks(p) -> float:
    """A = 2 + min(8*2^h, ceil(8*k*t*c)) AES blocks per trial, c = 2^(2h)/D."""
    c = (2.0 ** (2 * p.half_bits)) / p.domain
    return 2 + min(8 * 2 ** p.half_bits, math.ceil(8 * p.k * p.pnum * c))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def read_peaks() -> dict:
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        return {}


def read_traffic(name: str = "config2") -> float | None:
    """DRAM bytes per engine launch from the committed ncu summary, if any."""
    f = ROOT / "profiles" / f"engine_{name}_traffic.txt"
    try:
        for line in f.read_text().splitlines():
            if line.startswith("dram_bytes_per_launch"):
                return float(line.split("=")[1])
    except (OSError, ValueError, IndexError):
        pass
    return None


# ------------------------------------------------------------- CPU baseline --

def reference_lib():
    path = ROOT / "oracle" / "_ref" / "libcmcref.so"
    if not path.exists():
        return None
    lib = ctypes.CDLL(str(path))
    u32, u64 = ctypes.c_uint32, ctypes.c_uint64
    lib.ref_batch_launch.argtypes = [ctypes.c_char_p, ctypes.c_char_p, u32, u32, u32, u32, u64,
                                     u64, u32, ctypes.c_int, ctypes.POINTER(u32),
                                     ctypes.POINTER(ctypes.c_int)]
    lib.ref_batch_launch.restype = u32
    lib.ref_has_aesni.restype = ctypes.c_int
    return lib if lib.ref_has_aesni() else None


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_run(n_trials: int, batch: int, threads: int, w: dict = WORKLOAD):
    """Trials [0, n) of `batch` on the CPU: the reference's own cpu_batch_launch
    (oracle/_ref) when built here, else the oracle restatement.  Returns
    (seconds, kind, sorted failing offsets)."""
    lib = reference_lib()
    out = (ctypes.c_uint32 * max(n_trials, 1))()
    t0 = time.perf_counter()
    if lib is not None:
        used = ctypes.c_int()
        n = lib.ref_batch_launch(w["mode"].encode(), w["input_mode"].encode(), w["pnum"],
                                 w["ell_i"], w["buckets"], w["kick"], w["seed"], batch, n_trials,
                                 threads, out, ctypes.byref(used))
        failures = list(out[:n])
        kind = "reference"
    else:
        sys.path.insert(0, str(ROOT / "tests"))
        from oracle_binding import Oracle
        o = Oracle()
        p = o.params(w["mode"], w["pnum"], w["ell_i"], w["k"], w["buckets"], w["kick"],
                     w["input_mode"])
        failures = o.batch(p, w["seed"], batch, 0, n_trials, threads)
        kind = "port"
    return time.perf_counter() - t0, kind, failures


def cpu_sample_size(threads: int, target_seconds: float,
                    w: dict = WORKLOAD) -> tuple[int, float, str, list]:
    """Grow the sample until one run takes about target_seconds (cap 2^20);
    returns (trials, seconds, kind, failures) of the last run."""
    n = max(256, threads * 16) if w["pnum"] < 4096 else threads * 2
    while True:
        secs, kind, failures = cpu_run(n, 0, threads, w)
        if secs >= target_seconds * 0.5 or n >= 1 << 20:
            return n, secs, kind, failures
        n = int(min(1 << 20, max(2 * n, n * target_seconds / max(secs, 1e-3))))


def cpu_baseline(target_seconds: float = 10.0, w: dict = WORKLOAD) -> tuple[dict, int, list]:
    """The timed CPU sample: its JSON object, its size n and its failing offsets
    (the first n trials of batch 0)."""
    threads = host_threads()
    n, secs, kind, failures = cpu_sample_size(threads, target_seconds, w)
    return {"value": n / secs, "unit": "trials/s", "cores": threads, "kind": kind,
            "sample": f"first {n} trials of batch 0 of the bench workload "
                      f"({'reference cpu_batch_launch, AES-NI' if kind == 'reference' else 'oracle port'}, "
                      f"{threads} threads, {secs:.1f} s)"}, n, failures


def parity_check(ctx, cmc, w: dict, n: int, cpu_failures: list, kind: str) -> dict:
    """The GPU on the CPU sample's trials (batch 0, offsets 0..n-1): both
    failure lists, compared offset by offset."""
    p = cmc.parameters(w["mode"], w["pnum"], w["ell_i"], w["k"], w["buckets"], w["kick"],
                       w["input_mode"])
    gpu = ctx.launch(p, cmc.batch_key(w["seed"], 0), 0, n)
    return {"trials": n, "batch": 0, "cpu": kind, "cpu_failures": len(cpu_failures),
            "gpu_failures": len(gpu), "equal": gpu == cpu_failures}


def stressed_parity(ctx, cmc, w: dict, trials: int = 1 << 18) -> dict:
    """The bench shape with fewer buckets (B = 1250 for t = 1024) and half the
    eviction limit, where about 1 % of trials fail: the reference's CPU code
    and the GPU on the same trials, failure lists compared."""
    ws = dict(w, buckets=int(w["buckets"] * 1250 // 1536), kick=max(1, w["kick"] // 2))
    secs, kind, failures = cpu_run(trials, 0, host_threads(), ws)
    out = parity_check(ctx, cmc, ws, trials, failures, kind)
    out["shape"] = f"t={ws['pnum']}, N=2^{ws['ell_i']}, k={ws['k']}, B={ws['buckets']}, " \
                   f"kick={ws['kick']}, seed {ws['seed']}"
    out["cpu_seconds"] = secs
    return out


# ------------------------------------------------------------- replicas --

def batch_of(step: int, rank: int, world: int) -> int:
    """Batch id of rank `rank`'s step: ranks interleave, so every rank runs
    disjoint batches of the same experiment (replicas, no collective on the
    data path; the reference's workers claim batch ids the same way,
    cuckoo_bench.cu:976)."""
    return rank + world * step


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The slowest rank's time: whole-job throughput is set by it."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference_arm(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    threads = host_threads()
    w = WORKLOADS.get(args.workload, WORKLOAD)
    # bounded sample per step: about 2 s of CPU work each
    per_step, _, kind, _ = cpu_sample_size(threads, 2.0, w)
    for s in range(args.warmup):
        cpu_run(per_step, s, threads, w)
    total = 0.0
    for s in range(args.steps):
        secs, kind, _ = cpu_run(per_step, args.warmup + s, threads, w)
        total += secs
    value = per_step * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "trials/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded AES-CTR trial stream)",
        "config": {"workload": w["workload"], "trials_per_step": per_step,
                   "parallelism": f"{threads} host threads"},
        "cpu_baseline": {"value": value, "unit": "trials/s", "cores": threads, "kind": kind,
                         "sample": f"{per_step} trials per step, batches {args.warmup}.."
                                   f"{args.warmup + args.steps - 1}"},
        "e2e": {"value": value, "unit": "trials/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------- reference arm on the GPU --

def reference_gpu_lib():
    """The reference's own CUDA driver and kernels (oracle/_ref/librefgpu.so,
    built unmodified from its sources for sm_100a), or None."""
    path = ROOT / "oracle" / "_ref" / "librefgpu.so"
    if not path.exists():
        return None
    lib = ctypes.CDLL(str(path))
    u32, u64, P = ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER
    lib.ref_gpu_run.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p, u32, u32, u32, u32,
                                u64, u32, u32, ctypes.c_char_p, ctypes.c_char_p,
                                P(ctypes.c_double), P(u64), P(u64), ctypes.c_char_p, u32]
    lib.ref_gpu_run.restype = ctypes.c_int
    return lib


def reference_gpu_batch(lib, w: dict, seed: int, bt: int, layout: str = "auto"):
    """Batch 0 (2^bt trials) of the experiment through the reference's stock
    GPU worker, with B and the eviction limit of `w`.  Returns (seconds,
    sorted failing offsets, layout description)."""
    import tempfile
    with tempfile.TemporaryDirectory(prefix="cmc-refgpu-") as d:
        secs, done, failed = ctypes.c_double(), ctypes.c_uint64(), ctypes.c_uint64()
        info = ctypes.create_string_buffer(256)
        rc = lib.ref_gpu_run(0, w["mode"].encode(), w["input_mode"].encode(), w["pnum"],
                             w["ell_i"], w["buckets"], w["kick"], seed, bt, bt, layout.encode(),
                             d.encode(), ctypes.byref(secs), ctypes.byref(done),
                             ctypes.byref(failed), info, 256)
        if rc:
            raise RuntimeError(f"reference GPU run failed: {info.value.decode()}")
        rows = (Path(d) / "failures.csv").read_text().split()[1:]
        offsets = sorted(int(r.split(",")[1]) for r in rows)
    assert len(offsets) == failed.value and done.value == 1 << bt
    return secs.value, offsets, info.value.decode()


def failure_digest(lists) -> str:
    import hashlib
    h = hashlib.sha256()
    for f in lists:
        h.update(",".join(map(str, f)).encode() + b";")
    return h.hexdigest()[:16]


def run_reference_gpu_arm(args, rank: int, world: int) -> None:
    """The reference's own CUDA kernels (the plain one-configuration-per-launch
    GPU form) on this arm's workload: batch 0 of each step's experiment through
    its stock gpu_worker, timed like its work_elapsed_seconds."""
    if rank != 0:
        return
    lib = reference_gpu_lib()
    if lib is None:
        print(json.dumps({"impl": "reference", "ref_device": "gpu",
                          "unavailable": "oracle/_ref/librefgpu.so not built "
                                         "(make -C oracle refgpu REF=<reference dir>)"}))
        return
    if args.workload == "sweep":
        n = args.sweep_trials
        bt = n.bit_length() - 1
        assert n == 1 << bt, "--sweep-trials must be a power of two for the reference worker"
        sets = [s for s in sweep_sets() if s["k"] == 3]   # the reference hard-codes k = 3
        total, lists, per_set = 0.0, [], []
        for s in sets:
            secs, fails, info = reference_gpu_batch(lib, s, s["seed"], bt)
            total += secs
            lists.append(fails)
            per_set.append({"t": s["pnum"], "B": s["buckets"], "kick": s["kick"],
                            "trials_per_s": n / secs, "failures": len(fails), "plan": info})
        line = {"impl": "reference", "ref_device": "gpu",
                "metric": "sweep trials/s, k = 3 sets (bit-exact failures)",
                "value": n * len(sets) / total, "unit": "trials/s", "sets": len(sets),
                "trials_per_set": n, "seconds": total, "failures": sum(map(len, lists)),
                "failures_digest": failure_digest(lists), "per_set": per_set,
                "timing": "host wall clock around the reference's gpu_worker per set"}
        print(json.dumps(line), flush=True)
        return
    w = WORKLOADS.get(args.workload, WORKLOAD)
    bt = min(w["bt"], (w["trials"] - 1).bit_length())
    for _ in range(args.warmup):
        reference_gpu_batch(lib, w, w["seed"], bt)
    total, info, fails = 0.0, "", []
    for _ in range(args.steps):
        secs, fails, info = reference_gpu_batch(lib, w, w["seed"], bt)
        total += secs
    value = (1 << bt) * args.steps / total
    line = {"impl": "reference", "ref_device": "gpu", "metric": METRIC, "value": value,
            "unit": "trials/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "dtype": "u32", "data": "synthetic (seeded AES-CTR trial stream)",
            "config": {"workload": w["workload"], "trials_per_step": 1 << bt,
                       "batch": 0, "plan": info},
            "failures": len(fails), "failures_digest": failure_digest([fails]),
            "timing": "host wall clock around the reference's gpu_worker (its "
                      "work_elapsed_seconds): allocation, launches, per-launch read-back, "
                      "journal commit"}
    print(json.dumps(line), flush=True)


# ------------------------------------------------- other single-set workloads --

def workload_summary(cmc, ctx, w: dict, sms: int, max_mhz: float, steps: int = 4,
                     warmup: int = 3, name: str | None = None) -> dict:
    """A compact line for another single-configuration workload, measured after
    the main timed region: device-resident launches over batches warmup..,
    timed with CUDA events (L2 flushed between steps), the roofline fraction,
    e2e through cmc_launch with host buffers, and a bounded CPU sample of the
    reference's own code with its failure list compared on the GPU."""
    import torch
    p = cmc.parameters(w["mode"], w["pnum"], w["ell_i"], w["k"], w["buckets"], w["kick"],
                       w["input_mode"])
    n = min(w["trials"], 1 << w["bt"])
    stream = torch.cuda.Stream()
    d_out = torch.empty(n, dtype=torch.int32, device="cuda")
    d_n = torch.zeros(1, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    keys = [torch.tensor(cmc.batch_key(w["seed"], b), dtype=torch.int64).to(torch.int32).cuda()
            for b in range(warmup + steps)]
    for b in range(warmup):
        ctx.launch_device(p, keys[b].data_ptr(), 0, n, d_out.data_ptr(), d_n.data_ptr(),
                          stream.cuda_stream)
    torch.cuda.synchronize()
    ctx.check()
    total_ms, engine_ms = 0.0, []
    for b in range(warmup, warmup + steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.launch_device(p, keys[b].data_ptr(), 0, n, d_out.data_ptr(), d_n.data_ptr(),
                          stream.cuda_stream)
        e1.record(stream)
        engine_ms.append(ctx.last_engine_ms())
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    ctx.check()
    value = n * steps / (total_ms / 1e3)
    host_keys = [cmc.batch_key(w["seed"], warmup + steps + b) for b in range(2)]
    ctx.launch(p, host_keys[0], 0, n)
    t0 = time.perf_counter()
    ctx.launch(p, host_keys[1], 0, n)
    e2e = n / (time.perf_counter() - t0)
    blocks = algorithmic_blocks(p)
    achieved = blocks * AES_BYTES_PER_BLOCK * n / (statistics.mean(engine_ms) / 1e3) / 1e9
    peak = sms * SMEM_BYTES_PER_CLK_PER_SM * max_mhz * 1e6 / 1e9
    base, n_cpu, cpu_fails = cpu_baseline(5.0, w)
    return {"workload": w["workload"], "value": value, "unit": "trials/s",
            "steps": steps, "warmup": warmup, "ms_per_step": total_ms / steps,
            "e2e": {"value": e2e, "unit": "trials/s",
                    "timing": "host wall clock around one cmc_launch with host buffers"},
            "roofline": {"bound": "smem", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": read_traffic(name) if name else None},
            "plan": ctx.last_plan, "cpu_baseline": base,
            "parity": parity_check(ctx, cmc, w, n_cpu, cpu_fails, base["kind"])}


# ------------------------------------------------------------ sweep workload --

def sweep_sets(n_sets: int = 64, draw_seed: int = 3):
    """The mixed sweep: n_sets parameter sets drawn with draw_seed.  t is
    log-uniform over 16..4096, B = ceil(r t) with r in {1.25, 1.35, 1.5}, k in
    {2, 3, 4}, max kicks in {100, 500}, N = 2^24 (ell_i 24), BGH25, affine
    inputs.  Set i is its own experiment with seed draw_seed*1000 + i."""
    import numpy as np
    rng = np.random.default_rng(draw_seed)
    sets = []
    for i in range(n_sets):
        t = int(round(math.exp(rng.uniform(math.log(16), math.log(4096)))))
        r = float(rng.choice([1.25, 1.35, 1.5]))
        k = int(rng.choice([2, 3, 4]))
        kick = int(rng.choice([100, 500]))
        sets.append(dict(mode="bgh25", pnum=max(t, 3), ell_i=24, k=k, buckets=math.ceil(r * t),
                         kick=kick, input_mode="affine", seed=draw_seed * 1000 + i))
    return sets


def run_sweep_workload(args):
    cmc = load_pkg()
    ctx = cmc.Context(0)
    print(json.dumps(sweep_measure(cmc, ctx, args.sweep_trials)), flush=True)
    ctx.close()


def sweep_measure(cmc, ctx, n: int) -> dict:
    """Plain (one launch per parameter set) vs batched (all sets in one call)
    on the mixed sweep; both must give identical failures."""
    import torch
    sets = sweep_sets()
    params = [cmc.parameters(s["mode"], s["pnum"], s["ell_i"], s["k"], s["buckets"], s["kick"],
                             s["input_mode"]) for s in sets]
    jobs = [(p, s["seed"], 0, 0, n) for p, s in zip(params, sets)]
    total = n * len(sets)

    def plain():
        fails = []
        for p, s in zip(params, sets):
            fails.append(ctx.launch(p, cmc.batch_key(s["seed"], 0), 0, n))
        return fails

    def batched():
        counts, per_job = ctx.run_jobs(jobs)
        return [per_job[i] for i in range(len(jobs))]

    # warm-up (also the correctness check)
    ref = plain()
    got = batched()
    same = ref == got
    torch.cuda.synchronize()
    t0 = time.perf_counter(); plain(); t_plain = time.perf_counter() - t0
    batched()  # second call of this shape: captured into a CUDA graph; timed calls replay it
    t0 = time.perf_counter(); batched(); t_batched = time.perf_counter() - t0
    choice = ctx.autotune(jobs, sample_div=max(1, min(16, n // 1024)))
    batched()
    batched()
    t0 = time.perf_counter(); tuned = batched(); t_tuned = time.perf_counter() - t0
    graph_state = ctx.last_plan.rsplit("graph=", 1)[-1] if "graph=" in ctx.last_plan else "off"
    same = same and tuned == ref
    avg_blocks = sum(algorithmic_blocks(p) for p in params) / len(params)
    # the k = 3 sets alone: the sets the reference's kernels can run
    # (bench.py --impl reference --ref-device gpu --workload sweep times them)
    k3 = [i for i, st in enumerate(sets) if st["k"] == 3]
    k3_jobs = [jobs[i] for i in k3]
    ctx.run_jobs(k3_jobs)
    ctx.run_jobs(k3_jobs)
    t0 = time.perf_counter(); ctx.run_jobs(k3_jobs); t_k3 = time.perf_counter() - t0
    t0 = time.perf_counter()
    for i in k3:
        ctx.launch(params[i], cmc.batch_key(sets[i]["seed"], 0), 0, n)
    t_k3_plain = time.perf_counter() - t0
    line = {
        "metric": "sweep trials/s (64 mixed parameter sets, bit-exact failures)",
        "workload": f"sweep: 64 sets drawn with seed 3, {n} trials each (batch 0, offsets 0..{n - 1})",
        "plain_trials_per_s": total / t_plain, "batched_trials_per_s": total / t_batched,
        "batched_tuned_trials_per_s": total / t_tuned,
        "speedup_batched_vs_plain": t_plain / t_tuned,
        "identical_failures": same, "failures": sum(len(f) for f in ref),
        "batched_graph": graph_state,
        "mean_aes_blocks_per_trial": avg_blocks, "tuned_plan": choice,
        "k3_sets": {"sets": len(k3), "batched_trials_per_s": n * len(k3) / t_k3,
                    "plain_trials_per_s": n * len(k3) / t_k3_plain,
                    "failures": sum(len(ref[i]) for i in k3),
                    "failures_digest": failure_digest([ref[i] for i in k3])},
        "timing": "host wall clock around synchronous C-ABI calls (cmc_launch / cmc_run_jobs)",
    }
    return line


# ------------------------------------------------------------ serve workload --

def serve_jobs(n_jobs: int, rate: float, log2_budget: tuple[float, float], draw_seed: int = 5):
    """The served stream: Poisson arrivals at `rate` jobs/s; t = round(2^U[4,14]),
    B = ceil(r t) with r in {1.2, 1.3, 1.4, 1.5}, k in {2, 3}, max kicks 500,
    N = 2^24, budget = round(2^U[log2_budget]) trials; job i has seed
    draw_seed*100000 + i.  The budget range is a parameter because the full
    range (2^16..2^24) is about an hour of GPU work."""
    import numpy as np
    rng = np.random.default_rng(draw_seed)
    t_arr = 0.0
    jobs = []
    for i in range(n_jobs):
        t_arr += float(rng.exponential(1.0 / rate))
        t = int(round(2 ** rng.uniform(4, 14)))
        r = float(rng.choice([1.2, 1.3, 1.4, 1.5]))
        k = int(rng.choice([2, 3]))
        budget = int(round(2 ** rng.uniform(*log2_budget)))
        jobs.append(dict(arrival=t_arr, mode="bgh25", pnum=max(t, 3), ell_i=24, k=k,
                         buckets=math.ceil(r * t), kick=500, input_mode="affine",
                         seed=draw_seed * 100000 + i, trials=budget))
    return jobs


def rounded_budget(trials: int, bt_max: int = 20):
    et = max(1, (trials - 1).bit_length())
    bt = min(bt_max, et)
    per = 1 << bt
    return -(-trials // per) * per, bt


def run_serve_workload(args):
    cmc = load_pkg()
    ctx = cmc.Context(0)
    print(json.dumps(serve_measure(cmc, ctx, args)), flush=True)
    ctx.close()


def serve_measure(cmc, ctx, args) -> dict:
    """Served (continuous batching) vs plain (one launch per job, in arrival
    order) on the same job stream; job latency = completion - arrival."""
    lo, hi = (float(x) for x in args.serve_log2_budget.split(","))
    jobs = serve_jobs(args.serve_jobs, args.serve_rate, (lo, hi))
    params = [cmc.parameters(j["mode"], j["pnum"], j["ell_i"], j["k"], j["buckets"], j["kick"],
                             j["input_mode"]) for j in jobs]
    total_trials = sum(rounded_budget(j["trials"])[0] for j in jobs)

    # untimed warm-up of both arms (module loads, first pool allocations)
    warm = cmc.Server(ctx, max_jobs=64, mem_budget=8 << 30, batch_bits=20,
                      max_iteration_trials=1 << 23)
    for i in range(min(16, len(jobs))):
        warm.submit(params[i], jobs[i]["seed"] + 7, 256)
    while warm.pending():
        warm.step(args.serve_step_blocks)
    warm.close()
    for i in range(min(16, len(jobs))):
        ctx.run_jobs([(params[i], jobs[i]["seed"] + 7, 0, 0, 256)], cap=0)

    # served
    srv = cmc.Server(ctx, max_jobs=4096, mem_budget=8 << 30, batch_bits=20,
                     max_iteration_trials=1 << 23)
    srv.policy(args.serve_fifo_share)
    srv.set_option("resident", args.serve_resident)
    t0 = time.perf_counter()
    submitted, done_at, ids = 0, {}, {}
    while len(done_at) < len(jobs):
        now = time.perf_counter() - t0
        while submitted < len(jobs) and jobs[submitted]["arrival"] <= now:
            j = jobs[submitted]
            ids[srv.submit(params[submitted], j["seed"], j["trials"])] = submitted
            submitted += 1
        if srv.pending():
            for jid in srv.step(args.serve_step_blocks):
                done_at[ids[jid]] = time.perf_counter() - t0
        elif submitted < len(jobs):
            time.sleep(max(0.0, jobs[submitted]["arrival"] - (time.perf_counter() - t0)))
    served_span = time.perf_counter() - t0
    served_failed = [srv.status(jid)[1] for jid in sorted(ids, key=lambda x: ids[x])]
    served_stats = srv.stats()
    srv.close()
    lat_served = sorted(done_at[i] - jobs[i]["arrival"] for i in range(len(jobs)))

    # plain: each job alone, one launch covering its batches, arrival order
    t0 = time.perf_counter()
    lat_plain, plain_failed = [], []
    for i, j in enumerate(jobs):
        now = time.perf_counter() - t0
        if j["arrival"] > now:
            time.sleep(j["arrival"] - now)
        budget, bt = rounded_budget(j["trials"])
        per = 1 << bt
        entries = [(params[i], j["seed"], b, 0, per) for b in range(budget // per)]
        counts, _ = ctx.run_jobs(entries, cap=0)
        plain_failed.append(sum(counts))
        lat_plain.append(time.perf_counter() - t0 - j["arrival"])
    plain_span = time.perf_counter() - t0
    lat_plain.sort()

    def pct(v, q):
        return v[min(len(v) - 1, int(q * len(v)))]

    line = {
        "metric": "served stream: job latency p50/p99 (s) and trials/s, served vs plain",
        "workload": f"{len(jobs)} jobs, Poisson {args.serve_rate}/s, budgets 2^U[{lo},{hi}] "
                    f"(rounded up to whole batches), t = 2^U[4,14], N = 2^24, seed 5",
        "served": {"p50_s": pct(lat_served, 0.5), "p99_s": pct(lat_served, 0.99),
                   "trials_per_s": total_trials / served_span, "makespan_s": served_span,
                   "iterations": served_stats["iterations"],
                   "engine_busy_s": served_stats["busy_ms"] / 1e3},
        "plain": {"p50_s": pct(lat_plain, 0.5), "p99_s": pct(lat_plain, 0.99),
                  "trials_per_s": total_trials / plain_span, "makespan_s": plain_span},
        "identical_failure_counts": served_failed == plain_failed,
        "total_trials": total_trials, "step_blocks": args.serve_step_blocks,
        "fifo_share": args.serve_fifo_share, "resident": args.serve_resident,
        "timing": "host wall clock from each job's arrival to its completion",
    }
    return line


# ------------------------------------------------------------------ our arm --

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-device", choices=["cpu", "gpu"], default="cpu",
                    help="--impl reference: the reference's CPU path (default) or its own CUDA "
                         "kernels built for sm_100a (the plain GPU form)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload only: skip the sweep and serve objects")
    ap.add_argument("--trials", type=int, default=0,
                    help="trials per step (default: the workload's, 2^20 for config2); "
                         "smaller for profiling")
    ap.add_argument("--workload", choices=["config2", "config1", "config4", "sweep", "serve"],
                    default="config2")
    ap.add_argument("--serve-jobs", type=int, default=400)
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-log2-budget", default="10,16")
    ap.add_argument("--serve-step-blocks", type=int, default=400_000_000)
    ap.add_argument("--serve-fifo-share", type=float, default=0.95)
    ap.add_argument("--serve-resident", type=int, default=1, choices=[0, 1],
                    help="1: one resident engine launch per busy period; 0: one launch per iteration")
    ap.add_argument("--sweep-trials", type=int, default=1 << 16,
                    help="trials per parameter set for --workload sweep")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if args.ref_device == "gpu":
            run_reference_gpu_arm(args, rank, world)
        else:
            run_reference_arm(args, rank, world)
        return
    if args.workload == "sweep":
        if rank == 0:
            run_sweep_workload(args)
        return
    if args.workload == "serve":
        if rank == 0:
            run_serve_workload(args)
        return

    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    cmc = load_pkg()
    ctx = cmc.Context(local)
    w = WORKLOADS[args.workload]
    p = cmc.parameters(w["mode"], w["pnum"], w["ell_i"], w["k"], w["buckets"], w["kick"],
                       w["input_mode"])
    n = min(args.trials or w["trials"], 1 << w["bt"])
    # a dedicated stream: the legacy default stream's handle is NULL, which the
    # C ABI reads as "the context's own stream"
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    d_out = torch.empty(n, dtype=torch.int32, device="cuda")
    d_n = torch.zeros(1, dtype=torch.int32, device="cuda")
    keys = {}

    def key_of(batch):
        if batch not in keys:
            keys[batch] = torch.tensor(cmc.batch_key(w["seed"], batch), dtype=torch.int64) \
                .to(torch.int32).cuda()
        return keys[batch]

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    # warm-up (untimed)
    for s in range(args.warmup):
        ctx.launch_device(p, key_of(batch_of(s, rank, world)).data_ptr(), 0, n, d_out.data_ptr(),
                          d_n.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    ctx.check()

    # timed region: K steps, per-step events on the launching stream, L2 flushed between
    steps = list(range(args.warmup, args.warmup + args.steps))
    for s in steps:
        key_of(batch_of(s, rank, world))
    starts = [torch.cuda.Event(enable_timing=True) for _ in steps]
    ends = [torch.cuda.Event(enable_timing=True) for _ in steps]
    engine_ms = []
    failures = 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for i, s in enumerate(steps):
            flush.zero_()
            starts[i].record(stream)
            ctx.launch_device(p, key_of(batch_of(s, rank, world)).data_ptr(), 0, n, d_out.data_ptr(),
                              d_n.data_ptr(), stream.cuda_stream)
            ends[i].record(stream)
            engine_ms.append(ctx.last_engine_ms())
            failures += int(d_n.item())
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    ctx.check()
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    total_ms = sum(step_ms)
    launches = ctx.last_kernel_count * len(steps)
    max_ms = max_over_ranks(total_ms, world, "cuda")
    value = world * n * len(steps) / (max_ms / 1e3)

    # e2e: the C ABI call with host buffers, copies inside the timed region
    e2e_steps = list(range(args.warmup + args.steps, args.warmup + 2 * args.steps))
    host_keys = {s: cmc.batch_key(w["seed"], batch_of(s, rank, world)) for s in e2e_steps}
    ctx.launch(p, host_keys[e2e_steps[0]], 0, n)  # warm host path
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    d2h = 0
    for s in e2e_steps:
        fails = ctx.launch(p, host_keys[s], 0, n)
        d2h += 4 + 4 * len(fails)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world, "cuda")
    e2e_value = world * n * len(e2e_steps) / (e2e_ms / 1e3)

    if rank == 0:
        peaks = read_peaks()
        clk = clocks.summary()
        blocks = algorithmic_blocks(p)
        mean_engine_ms = statistics.mean(engine_ms)
        achieved = blocks * AES_BYTES_PER_BLOCK * n / (mean_engine_ms / 1e3) / 1e9
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        max_mhz = peaks.get("sm_max_mhz") or clk.get("sm_max_mhz") or 1965.0
        peak = sms * SMEM_BYTES_PER_CLK_PER_SM * max_mhz * 1e6 / 1e9
        traffic = read_traffic(args.workload)
        line = {
            "metric": METRIC, "value": value, "unit": "trials/s", "n_gpus": world,
            "steps": len(steps), "warmup": args.warmup, "ms_per_step": max_ms / len(steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded AES-CTR trial stream; no dataset)",
            "config": {"workload": w["workload"], "trials_per_step": n,
                       "parallelism": f"replicas x{world} (disjoint batches, no collective)",
                       "l2": "256 MiB buffer written between steps, outside the step events",
                       "plan": ctx.last_plan},
            "e2e": {"value": e2e_value, "unit": "trials/s", "h2d_bytes_per_step": 176,
                    "d2h_bytes_per_step": d2h // len(e2e_steps)},
            "gpu_launches": launches,
            "failures_in_timed_steps": failures,
            "roofline": {
                "bound": "smem", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "basis": f"A={blocks:.0f} AES blocks/trial x 640 B of T-table lookups; peak = "
                         f"{sms} SMs x 128 B/clk x {max_mhz:.0f} MHz (sm_max_mhz of "
                         f"MEASURED_PEAKS.json); engine kernel {mean_engine_ms:.2f} ms/launch",
            },
            "clocks": clk,
        }
        if not args.no_cpu_baseline and world == 1:
            base, n_cpu, cpu_fails = cpu_baseline(w=w)
            line["cpu_baseline"] = base
            line["parity"] = parity_check(ctx, cmc, w, n_cpu, cpu_fails, base["kind"])
            if args.workload == "config2":
                line["parity_stressed"] = stressed_parity(ctx, cmc, w)
        if world == 1 and args.workload == "config2" and not args.no_extras:
            # the batching and serving patterns, measured on the same box after
            # the timed region (own contexts; bounded to about a minute each)
            for name, fn in (("config1", lambda c: workload_summary(cmc, c, WORKLOADS["config1"], sms, max_mhz,
                                                                    name="config1")),
                             ("config4", lambda c: workload_summary(cmc, c, WORKLOADS["config4"], sms, max_mhz,
                                                                    name="config4")),
                             ("sweep", lambda c: sweep_measure(cmc, c, args.sweep_trials)),
                             ("serve", lambda c: serve_measure(cmc, c, args))):
                c2 = cmc.Context(local)
                try:
                    line[name] = fn(c2)
                finally:
                    c2.close()
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
