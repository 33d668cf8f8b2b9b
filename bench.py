#!/usr/bin/env python
"""KL-NMF benchmark: iterations/s of the B200 engine (and of the CPU reference arm).

One *step* is one convergence-test block of the reference loop
(src/NMF_GPU.c:544-709): ``niter_test_conv`` (=10) multiplicative iterations
(update_H + update_W), the EPS adjust, the classification and the
connectivity test -- run on the default workload, the 60000 x 5000, k = 32
planted Poisson matrix (V = 1.2 GB FP32, larger than L2, so no flush is
needed between steps).  ``value`` = iterations/s with V resident in HBM,
timed with CUDA events on the engine's stream; ``e2e`` = the same metric for a
whole solve through the C ABI from pinned host buffers (V upload, CPU_RANDOM
init, 500 iterations, W/H download).

``--impl reference`` times the CPU restatement of the reference's loop
(oracle/, OpenMP, all host threads) on a bounded row sample of the same
workload, scaled to the full matrix.

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
Under torchrun (N > 1) every rank runs an independent replica (weak scaling).
"""
from __future__ import annotations

import argparse
import csv
import importlib.util
import io
import json
import os
import shutil
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "bionmf-gpu_b200")

WORKLOADS = {
    # name: (n, m, k, generator, description)
    "C32": (60000, 5000, 32, "poisson", "60000x5000 k=32 planted Poisson(50*W0H0) counts, FP32"),
    "C64": (60000, 5000, 64, "poisson", "60000x5000 k=64 planted Poisson(50*W0H0) counts, FP32"),
    "B16": (20000, 1000, 16, "expr", "20000x1000 k=16 planted lognormal-noise matrix, 1% zeros, FP32"),
}


def _import_package():
    if "nmf_b200" in sys.modules:
        return sys.modules["nmf_b200"]
    spec = importlib.util.spec_from_file_location("nmf_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["nmf_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d.get("bf16_tflops", 1590.0)), "measured"
    return 6650.0, 1590.0, "fallback"


def ncu_traffic(kernel_key: str):
    """DRAM bytes per launch of the dominant kernel from a committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(kernel_key)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = [r for r in csv.reader(io.StringIO(self.out or "")) if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_V(workload, device, seed=20240501):
    pkg = _import_package()
    import nmf_b200.synth as synth
    import torch
    n, m, k, gen, _ = WORKLOADS[workload]
    if gen == "poisson":
        V, _ = synth.poisson_counts(n, m, k, seed, device=device)
        return V.contiguous()
    V, _ = synth.expression_like(n, m, k, seed, dirichlet=2.0, zero_frac=0.01)
    return torch.from_numpy(V).to(device)


_SAMPLES = {}


def cpu_port_rate(workload, budget_s=12.0, max_rows=None):
    """Oracle (plain OpenMP C restatement, FP32) iterations/s scaled to the full matrix."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    _import_package()
    import nmf_b200.synth as synth
    n, m, k, gen, _ = WORKLOADS[workload]
    rows = max_rows or max(500, min(n, int(1.5e7 // m)))  # ~15 M entries of the matrix
    key = (workload, rows)
    if key not in _SAMPLES:
        if gen == "poisson":
            V, _ = synth.poisson_counts(rows, m, k, 7)
        else:
            V, _ = synth.expression_like(rows, m, k, 7, dirichlet=2.0, zero_frac=0.01)
        _SAMPLES[key] = V
    V = _SAMPLES[key]
    W, H = oracle.init_random(3, rows, m, k)
    t0 = time.perf_counter()
    iters = 0
    while True:
        H = oracle.update_H(V, W, H)
        W = oracle.update_W(V, W, H)
        iters += 1
        el = time.perf_counter() - t0
        if el > budget_s or iters >= 200:
            break
    per_iter_full = el / iters * (n / rows)
    return {"value": 1.0 / per_iter_full, "unit": "iters/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{iters} FP32 iterations of the oracle on a {rows}x{m} row sample ({el:.1f} s), "
                      f"scaled by {n}/{rows} rows"}


def run_reference_arm(a, rank, world):
    if rank != 0:
        return
    n, m, k, _, desc = WORKLOADS[a.workload]
    rates = []
    per_step = min(a.cpu_budget, 150.0 / max(1, a.steps + a.warmup))
    for s in range(a.warmup + a.steps):
        r = cpu_port_rate(a.workload, budget_s=per_step)
        if s >= a.warmup:
            rates.append(r["value"])
    v = statistics.median(rates)
    r["value"] = v
    line = {"impl": "reference", "metric": "KL-NMF iterations/s", "value": v, "unit": "iters/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * a.iters_per_step / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": desc, "n": n, "m": m, "k": k,
                                             "iters_per_step": a.iters_per_step},
            "cpu_baseline": r, "e2e": {"value": v, "unit": "iters/s", "h2d_bytes_per_step": 0,
                                       "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_engine_arm(a, rank, world, local_rank):
    import torch
    pkg = _import_package()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n, m, k, _, desc = WORKLOADS[a.workload]
    V = make_V(a.workload, dev, seed=20240501 + rank)
    stream = torch.cuda.Stream(device=dev)
    e = pkg.NMF(n, m, k, arm=a.arm, device=local_rank)
    e.set_stream(stream.cuda_stream)
    e.set_V_device(V.data_ptr(), m)
    e.init_random(3)
    J = a.iters_per_step
    never = 2 ** 31
    for _ in range(a.warmup):
        e.run(J, J, never)
    e.synchronize()
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    l0 = e.launch_count()
    e.profile(True)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        for _ in range(a.steps):
            e.run(J, J, never)
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = e.launch_count() - l0
    prof = {c: e.profile_read(c) for c in range(4)}
    e.profile(False)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    iters_total = a.steps * J * world
    value = iters_total / (ms_max / 1e3)

    # roofline of the dominant kernel: V read once per launch (n*m*4 bytes).
    cls = 0 if prof[0][0] >= prof[1][0] else 1
    tot, cnt = prof[cls]
    avg_ms = tot / max(cnt, 1)
    bytes_per_launch = n * m * 4
    hbm, _, peak_kind = measured_peaks()
    achieved = bytes_per_launch / (avg_ms / 1e3) / 1e9
    kname = ("update_H" if cls == 0 else "update_W") + f"[{a.arm}]"
    traffic = ncu_traffic(f"{a.workload}:{kname}")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": traffic, "kernel": kname, "avg_launch_ms": avg_ms, "launches": cnt,
                "algorithmic_bytes_per_launch": bytes_per_launch, "peak_source": peak_kind,
                "half_iteration_ms": {"update_H": prof[2][0] / max(prof[2][1], 1),
                                      "update_W": prof[3][0] / max(prof[3][1], 1)}}

    # end-to-end through the C ABI from pinned host memory: a whole solve.
    e2e = None
    if not a.no_e2e:
        Vh = torch.empty((n, m), dtype=torch.float32, pin_memory=True)
        Vh.copy_(V)
        torch.cuda.synchronize()
        E = a.e2e_iters
        W_out = np.empty((n, k), np.float32)
        H_out = np.empty((m, k), np.float32)
        times = []
        for rep in range(2):
            b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            b0.record(stream)
            e._check(e._L.nmfb_set_V(e._h, pkg._fptr(Vh.numpy()), m))
            e.init_random(3)
            e.run(E, J, never)
            W_out[:] = e.W
            H_out[:] = e.H
            b1.record(stream)
            b1.synchronize()
            times.append(b0.elapsed_time(b1))
        e2e_ms = min(times)
        kp = 16 if k <= 16 else (k + 31) // 32 * 32
        e2e = {"value": E / (e2e_ms / 1e3), "unit": "iters/s", "h2d_bytes_per_step": n * m * 4 + (n + m) * kp * 4,
               "d2h_bytes_per_step": (n + m) * kp * 4, "iters_per_step": E, "ms_per_step": e2e_ms}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_port_rate(a.workload, budget_s=a.cpu_budget)
    e.close()
    if rank != 0:
        return
    line = {"metric": "KL-NMF iterations/s", "value": value, "unit": "iters/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "n": n, "m": m, "k": k, "arm": a.arm, "iters_per_step": J,
                       "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (V = %.2f GB)" % (n * m * 4 / 1e9)},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--arm", default="fused", choices=["fused", "plain", "fused_tf32"])
    ap.add_argument("--workload", default="C32", choices=list(WORKLOADS))
    ap.add_argument("--iters-per-step", type=int, default=10)
    ap.add_argument("--e2e-iters", type=int, default=500)
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    a = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference_arm(a, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_engine_arm(a, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
