#!/usr/bin/env python
"""KL-NMF benchmark: iterations/s of the B200 engine (and of the CPU reference arm).

One *step* is one convergence-test block of the reference loop
(src/NMF_GPU.c:544-709): ``niter_test_conv`` (=10) multiplicative iterations
(update_H + update_W), the EPS adjust, the classification and the
connectivity test -- run on the default workload, the 60000 x 5000, k = 32
planted Poisson matrix (V = 1.2 GB FP32, larger than L2, so no flush is
needed between steps).  ``value`` = iterations/s with V resident in HBM,
timed with CUDA events on the engine's stream (each test block replayed as a
CUDA graph); the roofline's kernel time comes from a separate pass with
per-launch events; ``e2e`` = the same metric for a
whole solve through the C ABI from pinned host buffers (V upload, CPU_RANDOM
init, 500 iterations, W/H download).

The same line carries ``plain_arm`` (the unfused FP32 arm on the same V:
iterations/s, roofline fraction, fused speed-up) and ``sweep`` (the
rank-selection sweep 5000 x 200, k = 2..10 x 50 restarts, as one persistent
launch: solves/s on the device and end to end, against the same solves run
one by one through the single-problem engine).

Further extras: ``workloads`` (the fused arm at 60000 x 5000 k = 64 and at
20000 x 1000 k = 16) and ``reference_cuda`` (the reference's own CUDA build,
oracle/_ref/NMF_GPU compiled from its sources, timed on the same GPU and the
same matrices: a baseline leg, like ``cpu_baseline``, never the product).

``--impl reference`` times the CPU restatement of the reference's loop
(oracle/, OpenMP, all host threads) on the same full matrix, each step the
engine's step (10 iterations + adjust + classification); nothing is scaled.

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
    # profiling size of C32 for multi-pass ncu captures (V = 320 MB, still larger than L2)
    "C32P": (16000, 5000, 32, "poisson", "16000x5000 k=32 planted Poisson(50*W0H0) counts, FP32"),
    # blockwise (out-of-core) mode: V in host memory, streamed in row blocks
    "S32": (250000, 20000, 32, "poisson", "250000x20000 k=32 planted Poisson counts, FP32, V in host memory (20 GB)"),
}

# Rank-selection sweep (one V, every (k, restart) pair solved to convergence).
SWEEP = {"n": 5000, "m": 200, "true_k": 5, "ks": list(range(2, 11)), "restarts": 50, "seed": 4,
         "desc": "5000x200 planted k=5, k=2..10 x 50 restarts, -i 2000 -j 10 -t 40"}


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


def arm_precision():
    """Measured error of every fused arm against FP64 (6000 x 500 submatrix), committed with the profiles."""
    p = os.path.join(ROOT, "profiles", "arm_precision.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


def ncu_traffic(kernel_key: str):
    """DRAM bytes per launch of the dominant kernel from a committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(kernel_key)


class ClockSampler:
    """SM clocks and throttle reasons of one GPU, sampled every 10 ms by an NVML
    thread (the GPU is found by its PCI bus id, so CUDA_VISIBLE_DEVICES
    renumbering does not matter); nvidia-smi every 100 ms where NVML is
    unavailable.  `mark(True/False)` brackets the timed region, whose samples
    are summarised separately from the whole window."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40}

    def __init__(self, index: int, period_s: float = 0.01):
        self.index = index
        self.period = period_s
        self.samples = []          # (t, sm_mhz, reasons bitmask)
        self.window = [None, None]
        self.proc = None
        self.thread = None
        self.max_mhz = None
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.index)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())

    def __enter__(self):
        import threading
        try:
            nv, h = self._nvml_handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop = threading.Event()

            def loop():
                while not self.stop.is_set():
                    try:
                        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((time.perf_counter(), float(sm), int(rs)))
                    except Exception:
                        pass
                    time.sleep(self.period)

            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            self.source = "nvml, 10 ms"
        except Exception:
            if shutil.which("nvidia-smi"):
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                              "--format=csv,noheader,nounits", "-lms", "100"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.source = "nvidia-smi, 100 ms"
        return self

    def mark(self, begin: bool):
        self.window[0 if begin else 1] = time.perf_counter()

    def __exit__(self, *exc):
        self.out = ""
        if self.thread:
            self.stop.set()
            self.thread.join(timeout=2)
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def _summ(self, rows):
        if not rows:
            return None
        sm = [r[1] for r in rows]
        reasons = sorted({name for r in rows for name, bit in self.REASONS.items() if r[2] & bit})
        return {"sm_mhz": statistics.median(sm), "sm_min_mhz": min(sm), "reasons": reasons, "samples": len(rows)}

    def summary(self):
        if self.thread:
            t0, t1 = self.window
            inside = [r for r in self.samples if t0 is not None and t1 is not None and t0 <= r[0] <= t1]
            whole = self._summ(self.samples) or {"sm_mhz": None, "reasons": ["no samples"], "samples": 0}
            timed = self._summ(inside)
            out = dict(whole)
            out["sm_max_mhz"] = self.max_mhz
            out["source"] = self.source
            out["scope"] = "warm-up, timed steps and the profiled pass of the headline workload"
            out["timed_region"] = timed
            return out
        rows = [r for r in csv.reader(io.StringIO(self.out or "")) if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": self.source}


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


def host_V(workload, seed=20240501):
    """The workload's V in host memory, generated as make_V does (on a GPU when
    one is present, so that every arm sees the same matrix)."""
    if workload in _SAMPLES:
        return _SAMPLES[workload]
    _import_package()
    import nmf_b200.synth as synth
    n, m, k, gen, _ = WORKLOADS[workload]
    V = None
    try:
        import torch
        if torch.cuda.is_available():
            V = make_V(workload, torch.device("cuda", 0), seed=seed).cpu().numpy()
            torch.cuda.empty_cache()
    except Exception:
        V = None
    if V is None:
        if gen == "poisson":
            V, _ = synth.poisson_counts(n, m, k, seed)
        else:
            V, _ = synth.expression_like(n, m, k, seed, dirichlet=2.0, zero_frac=0.01)
    _SAMPLES[workload] = V
    return V


def cpu_port_step(oracle, V, W, H, J):
    """One step of the CPU restatement: J iterations of update_H + update_W,
    the EPS adjust and the classification (the engine's step, on the CPU)."""
    for _ in range(J):
        H = oracle.update_H(V, W, H)
        W = oracle.update_W(V, W, H)
    H = oracle.adjust(H)
    W = oracle.adjust(W)
    oracle.classify(H)
    return W, H


def cpu_port_rate(workload, J=10, steps=1, warmup=0):
    """Oracle (plain OpenMP C restatement, FP32, all host threads) iterations/s
    on the workload's full matrix: `steps` timed steps of J iterations each."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    n, m, k, gen, _ = WORKLOADS[workload]
    V = host_V(workload)
    W, H = oracle.init_random(3, n, m, k)
    times = []
    for s in range(warmup + steps):
        t0 = time.perf_counter()
        W, H = cpu_port_step(oracle, V, W, H, J)
        if s >= warmup:
            times.append(time.perf_counter() - t0)
    el = sum(times)
    return {"value": J * len(times) / el, "unit": "iters/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{J * len(times)} FP32 iterations ({len(times)} steps of {J} + adjust + classification) "
                      f"of the oracle on the full {n}x{m} matrix, {el:.1f} s"}


# ---------------------------------------------------------------------------
# The reference's own CUDA build (oracle/_ref/NMF_GPU, compiled from the
# reference sources by `make -C oracle ref`) timed on the same GPU.  It is a
# baseline, never the measured product.
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "NMF_GPU")


def _ref_input_path(tmp, name):
    """The reference allocates strlen(filename) + strlen(ext) bytes for its
    output name "<filename>_W<ext>" (src/NMF_GPU.c:974), three bytes short;
    choose a path length whose malloc rounding leaves room for them."""
    base = os.path.join(tmp, name)
    while True:
        s = len(base) + 4
        chunk = max(32, (s + 8 + 15) & ~15)
        if chunk - 8 >= s + 3:
            return base
        base += "_"


def _write_nonnative(path, V):
    """Non-native binary matrix file: u32 0xEDB10EA1, u32 rows, u32 cols, LE float64 data."""
    import struct
    n, m = V.shape
    with open(path, "wb") as f:
        f.write(struct.pack("<III", 0xEDB10EA1, n, m))
        for r0 in range(0, n, 8192):
            f.write(np.ascontiguousarray(V[r0:r0 + 8192], dtype="<f8").tobytes())


def _ref_run(path, k, it, j, t, timeout=900):
    """One NMF_GPU run; returns (seconds of its own TIME=1 line, iterations, converged)."""
    import re
    cmd = [REF_BIN, path, "-b", "0", "-e", "0", "-k", str(k), "-i", str(it), "-j", str(j), "-t", str(t)]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    out = p.stdout + p.stderr
    if p.returncode != 0:
        raise RuntimeError(f"NMF_GPU exited {p.returncode}: {out[-400:]}")
    secs = float(re.search(r"GPU \+ classification \+ check_result time: ([0-9.eE+-]+)", out).group(1))
    mc = re.search(r"converged in (\d+) iterations", out)
    mp = re.search(r"NMF: (\d+) iterations performed", out)
    return secs, int(mc.group(1) if mc else mp.group(1)), bool(mc)


def reference_cuda_rates(pkg, dev, engine_rates, short=10, long=510):
    """Iterations/s of the reference's CUDA build (cuBLAS SGEMMs + its own
    kernels) on the same V and GPU: the difference of a `long`- and a
    `short`-iteration run of its TIME=1 wall clock (which starts before the V
    upload), so fixed costs cancel; plus its whole-run rate for `long`
    iterations (V upload included, like the engine's e2e).  Config A runs to
    convergence (-i 2000 -j 10 -t 40) and is compared on time to converge
    with a whole solve through the engine's C ABI."""
    import tempfile
    if not os.path.exists(REF_BIN):
        return {"unavailable": "oracle/_ref/NMF_GPU not built (make -C oracle ref needs the reference sources)"}
    out = {"binary": "oracle/_ref/NMF_GPU (reference sources, single precision, cuBLAS, CPU_RANDOM init)",
           "method": f"iters/s = {long - short} / (t(-i {long}) - t(-i {short})), t = its own TIME=1 line; "
                     f"-j 10 -t 1e9 keeps the adjust cadence"}
    with tempfile.TemporaryDirectory(dir="/tmp") as tmp:
        for wl in ("C32", "B16"):
            n, m, k, _, desc = WORKLOADS[wl]
            path = _ref_input_path(tmp, wl)
            _write_nonnative(path, host_V(wl))
            t_s, _, _ = _ref_run(path, k, short, 10, 10 ** 9)
            t_l, it_l, _ = _ref_run(path, k, long, 10, 10 ** 9)
            rate = (long - short) / (t_l - t_s)
            r = {"workload": desc, "value": rate, "unit": "iters/s", "run_seconds": {str(short): t_s, str(long): t_l},
                 "e2e": {"value": it_l / t_l, "unit": "iters/s"},
                 "roofline_frac_2nm4": 2.0 * n * m * 4 * rate / 1e9 / measured_peaks()[0]}
            if wl in engine_rates:
                r["engine_iters_per_s"] = engine_rates[wl]
                r["engine_speedup"] = engine_rates[wl] / rate
            out[wl] = r
            os.unlink(path)
        # config A: time to converge
        import nmf_b200.synth as synth
        Va, _ = synth.config_a(1)
        path = _ref_input_path(tmp, "A")
        _write_nonnative(path, Va)
        ref = [_ref_run(path, 3, 2000, 10, 40) for _ in range(3)]
        t_ref = min(r[0] for r in ref)
        eng = []
        for _ in range(4):
            with pkg.NMF(Va.shape[0], Va.shape[1], 3, device=dev.index or 0) as e:
                t0 = time.perf_counter()
                e.set_V(Va)
                e.init_random(3)
                it, conv = e.run(2000, 10, 40)
                e.distance()
                eng.append((time.perf_counter() - t0, it, conv))
        t_eng = min(x[0] for x in eng[1:])
        out["A"] = {"workload": "5000x38 k=3 planted, -i 2000 -j 10 -t 40 (time to converge, V upload included)",
                    "reference_seconds": t_ref, "reference_iterations": ref[0][1], "reference_converged": ref[0][2],
                    "engine_seconds": t_eng, "engine_iterations": eng[-1][1], "engine_converged": eng[-1][2],
                    "engine_speedup": t_ref / t_eng}
    return out


class L2Flush:
    """Writes a buffer larger than L2 (126 MB) between timed steps."""

    def __init__(self, dev):
        import torch
        self.buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MB

    def __call__(self, stream=None):
        import torch
        with torch.cuda.stream(stream) if stream is not None else _nullctx():
            self.buf.fill_(1.0)


class _nullctx:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def sweep_rates(dev, steps=2, warmup=1, seq_sample=2, flush=None):
    """Config-D sweep: batched solves/s (one persistent launch per sweep, device
    time, L2 flushed before each sweep), its end-to-end rate through the public
    API from host memory, and the rate of the same solves run one by one
    through the single-problem engine (a sample of seq_sample restarts per k)."""
    import torch
    pkg = _import_package()
    import nmf_b200.synth as synth
    V, _ = synth.config_d(SWEEP["seed"])
    n, m = V.shape
    ks, R = SWEEP["ks"], SWEEP["restarts"]
    ranks = np.repeat(np.array(ks, np.uint32), R)
    seeds = np.tile(np.arange(1, R + 1, dtype=np.uint32), len(ks))
    nprob = len(ranks)
    flush = flush or L2Flush(dev)
    # tile shapes per rank from the project's autotuner (timed short runs of a
    # full wave per rank; cached per (k, m, n) bucket)
    import nmf_b200.sweep as sweep
    t0 = time.perf_counter()
    tiles = sweep.autotune(V, ks, device=dev.index or 0)
    tune_s = time.perf_counter() - t0
    dev_ms, e2e_ms, iters, ctas = [], [], None, 1
    with pkg.Batch(n, m, ranks, device=dev.index or 0) as b:
        for p, k in enumerate(ranks):
            b.set_tiles(p, *tiles[int(k)])
        for s in range(warmup + steps):
            torch.cuda.synchronize()
            flush()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            b.set_V(V)
            b.init_random(seeds)
            it, conv = b.run(2000, 10, 40)
            ctas = b.cluster
            b.classification()
            coph = {k: b.consensus(k)[2] for k in ks}
            t1 = time.perf_counter()
            if s >= warmup:
                dev_ms.append(b.last_ms())
                e2e_ms.append(1e3 * (t1 - t0))
            iters = it
    # sequential: the same solves one at a time through the single-problem engine
    seq_t, seq_n = 0.0, 0
    for k in ks:
        for r in range(1, seq_sample + 1):
            with pkg.NMF(n, m, k, device=dev.index or 0) as e:
                e.set_V(V)
                e.init_random(r)
                e.synchronize()
                t0 = time.perf_counter()
                e.run(2000, 10, 40)
                seq_t += time.perf_counter() - t0
                seq_n += 1
    batched = nprob / (statistics.median(dev_ms) / 1e3)
    seq = seq_n / seq_t
    flops = float(sum(int(iters[p]) * 8.0 * n * m * int(ranks[p]) for p in range(nprob)))
    return {"workload": SWEEP["desc"], "solves": nprob, "value": batched, "unit": "solves/s",
            "device_ms": statistics.median(dev_ms), "e2e": {"value": nprob / (statistics.median(e2e_ms) / 1e3),
                                                             "unit": "solves/s", "ms": statistics.median(e2e_ms)},
            "sequential": {"value": seq, "unit": "solves/s", "sample": f"{seq_n} solves (k=2..10 x {seq_sample} seeds), "
                                                                      "single-problem engine, host-timed"},
            "speedup_vs_sequential": batched / seq, "tflops": flops / (statistics.median(dev_ms) / 1e3) / 1e12,
            "mean_iterations": float(np.mean(iters)), "ctas_per_problem": ctas,
            "tiles": {str(k): list(v) for k, v in sorted(tiles.items())}, "autotune_s": round(tune_s, 2), "cophenetic": {str(k): round(v, 6) for k, v in coph.items()},
            "l2": "256 MB buffer written before every sweep"}


def stream_rates(dev, iters=10):
    """Blockwise mode on the S32 workload: iterations/s with V read from
    page-locked host memory, one convergence-test block of `iters` iterations
    (update_W's pass over V also forms the next update_H's sum, except after
    the block's last update_W: iters + 1 passes), the achieved host-to-device
    rate and the measured copy peak of the link (one 1 GiB pinned copy)."""
    import torch
    pkg = _import_package()
    n, m, k, _, desc = WORKLOADS["S32"]
    Vd = make_V("S32", dev)
    Vh = torch.empty((n, m), dtype=torch.float32, pin_memory=True)
    Vh.copy_(Vd)
    del Vd
    torch.cuda.empty_cache()
    # link peak: 1 GiB pinned H2D copy, best of 3
    src = Vh.view(-1)[: 1 << 28]
    dst = torch.empty_like(src, device=dev)
    peak = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        e1.synchronize()
        peak = max(peak, src.numel() * 4 / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del dst
    stream = torch.cuda.Stream(device=dev)
    with pkg.NMF(n, m, k, device=dev.index or 0, stream_rows=0) as e:
        e.set_stream(stream.cuda_stream)
        e.set_V(Vh.numpy())
        e.init_random(3)
        e.run(1, 1, 2 ** 31)
        e.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        e.run(iters, iters, 2 ** 31)
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
    rate = iters / (ms / 1e3)
    passes = iters + 1
    h2d = float(passes) * n * m * 4 / (ms / 1e3) / 1e9
    return {"workload": desc, "value": rate, "unit": "iters/s", "h2d_gbs": h2d, "h2d_peak_gbs": peak,
            "frac_of_link": h2d / peak, "passes_per_iteration": passes / iters,
            "bytes_per_iteration": passes / iters * n * m * 4,
            "cbig_s_per_iter_at_this_rate": passes / iters * 250000 * 200000 * 4 / (h2d * 1e9),
            "note": "250000x200000 (200 GB) is larger than this host's 196 GB of RAM; the blockwise path is "
                    "link-bound and linear in bytes, so its per-iteration time is extrapolated"}


SERVE = {"requests": 2000, "pool": 32, "n": (1000, 50000), "m": (20, 2000), "k": (2, 20), "iters": 300,
         "budget_gb": 120.0, "workers": 32, "load": 0.8,
         # SMs each request's context sizes its launches for: the best of 0 (all), 74, 37, 24
         # and 16 on 400 requests of this mix (121 solves/s at 74 against 112 at 0)
         "sm_limit": 74,
         "desc": "requests n~U[1000,50000], m~logU[20,2000], k~U[2,20], planted Poisson V, 300-iteration cap "
                 "(-j 10 -t 40: no request can converge before 410 iterations), 120 GB budget"}


def serve_requests(dev, count, seed=11):
    """`count` requests over a pool of planted matrices generated on the device
    and handed to the server in host memory."""
    import torch
    _import_package()
    import nmf_b200.serve as serve
    import nmf_b200.synth as synth
    rng = np.random.default_rng(seed)
    pool = []
    for i in range(SERVE["pool"]):
        n = int(rng.integers(SERVE["n"][0], SERVE["n"][1] + 1))
        m = int(np.exp(rng.uniform(np.log(SERVE["m"][0]), np.log(SERVE["m"][1]))))
        kt = int(rng.integers(SERVE["k"][0], SERVE["k"][1] + 1))
        V, _ = synth.poisson_counts(n, m, min(kt, m), 1000 + i, device=dev)
        pool.append(V.cpu().numpy())
        del V
    torch.cuda.empty_cache()
    reqs = []
    for i in range(count):
        V = pool[int(rng.integers(0, len(pool)))]
        k = min(int(rng.integers(SERVE["k"][0], SERVE["k"][1] + 1)), V.shape[1])
        reqs.append(serve.Request(V, k, seed=1 + i, n_iters=SERVE["iters"], niter_test_conv=10, stop_threshold=40,
                                  rid=i))
    return reqs


def serve_rates(dev, count=None, seq_sample=40):
    """Serving loop on config E's 2000 requests: capacity (all requests queued
    at once), the sequential baseline (one request at a time, same engine, a
    sample), and an open-loop run of all requests with Poisson arrivals at
    SERVE['load'] of the measured capacity (p50 / p99 latency from arrival to
    result on the host); the device queue and a half-load point on the first
    requests only, to keep the line within minutes."""
    _import_package()
    import nmf_b200.serve as serve
    count = count or SERVE["requests"]
    reqs = serve_requests(dev, count)
    srv = serve.Server(budget_bytes=SERVE["budget_gb"] * 1e9, workers=SERVE["workers"], device=dev.index or 0,
                       sm_limit=SERVE["sm_limit"])
    srv.run(reqs[:8], open_loop=False)                       # warm-up (module loads, allocator pools)
    cap = srv.run(reqs, open_loop=False)
    # the device queue (persistent serving kernel) against contexts on the
    # requests it takes (m <= 256)
    qsrv = serve.Server(budget_bytes=SERVE["budget_gb"] * 1e9, workers=SERVE["workers"], device=dev.index or 0,
                        batched=True)
    small = [r for r in reqs[:300] if qsrv._queued(r)]
    qsrv.run(small[:8], open_loop=False)
    q_small = qsrv.run(small, open_loop=False)
    c_small = srv.run(small, open_loop=False)
    seq = srv.run_sequential(reqs[:seq_sample])
    open_runs = {}
    for load, part in ((SERVE["load"], reqs), (0.5, reqs[:300])):
        rate = load * cap.solves_per_s()
        arr = serve.poisson_arrivals(len(part), rate, seed=5)
        for r, t in zip(part, arr):
            r.arrival = float(t)
        st = srv.run(part, open_loop=True)
        open_runs[load] = (rate, st)
    rate, op = open_runs[SERVE["load"]]
    rate50, op50 = open_runs[0.5]
    return {"workload": SERVE["desc"], "requests": count, "value": cap.solves_per_s(), "unit": "solves/s",
            "sequential": {"value": seq.solves_per_s(), "unit": "solves/s", "sample": f"first {seq_sample} requests"},
            "speedup_vs_sequential": cap.solves_per_s() / seq.solves_per_s(),
            "device_queue": {"requests": len(small), "max_m": qsrv.max_m, "ctas_per_request": qsrv.ctas,
                             "value": q_small.solves_per_s(), "unit": "solves/s",
                             "contexts_same_requests": c_small.solves_per_s(),
                             "p50_s": q_small.latency_pct(50), "p99_s": q_small.latency_pct(99),
                             "note": "the requests with m <= 256, all queued at t = 0: persistent serving kernel "
                                     "vs per-request contexts"},
            "open_loop": {"requests": count, "arrival_rate": rate, "solves_s": op.solves_per_s(), "p50_s": op.latency_pct(50),
                          "p99_s": op.latency_pct(99), "peak_active": op.peak_active,
                          "peak_gb": op.peak_bytes / 1e9},
            "open_loop_half_load": {"requests": 300, "arrival_rate": rate50, "solves_s": op50.solves_per_s(),
                                    "p50_s": op50.latency_pct(50), "p99_s": op50.latency_pct(99)},
            "sequential_p50_s_per_request": float(np.median([r.done - r.admitted for r in seq.results])),
            "workers": SERVE["workers"], "sm_limit": SERVE["sm_limit"],
            "sequential_note": "one request at a time, each context sized for all SMs"}


SERVE_SMALL = {"requests": 400, "n": (500, 5000), "m": (20, 256), "k": (2, 10), "iters": 300,
               "desc": "requests n~U[500,5000], m~logU[20,256], k~U[2,10], planted Poisson V, 300-iteration cap, "
                       "all queued at t = 0"}


def serve_small_rates(dev, seq_sample=40):
    """Many small requests (the regime the device queue is for): the
    persistent serving kernel against per-request contexts (concurrent, 32
    workers) and one request at a time."""
    _import_package()
    import nmf_b200.serve as serve
    import nmf_b200.synth as synth
    rng = np.random.default_rng(23)
    reqs = []
    for i in range(SERVE_SMALL["requests"]):
        n = int(rng.integers(SERVE_SMALL["n"][0], SERVE_SMALL["n"][1] + 1))
        m = int(np.exp(rng.uniform(np.log(SERVE_SMALL["m"][0]), np.log(SERVE_SMALL["m"][1]))))
        k = min(int(rng.integers(SERVE_SMALL["k"][0], SERVE_SMALL["k"][1] + 1)), m)
        V, _ = synth.poisson_counts(n, m, k, 5000 + i)
        reqs.append(serve.Request(V, k, seed=1 + i, n_iters=SERVE_SMALL["iters"], niter_test_conv=10,
                                  stop_threshold=40, rid=i))
    q = serve.Server(budget_bytes=SERVE["budget_gb"] * 1e9, workers=SERVE["workers"], device=dev.index or 0,
                     batched=True)
    c = serve.Server(budget_bytes=SERVE["budget_gb"] * 1e9, workers=SERVE["workers"], device=dev.index or 0,
                     sm_limit=SERVE["sm_limit"])
    q.run(reqs[:8], open_loop=False)                  # each path warmed up right before its own run
    qs = q.run(reqs, open_loop=False)
    c.run(reqs[:8], open_loop=False)
    cs = c.run(reqs, open_loop=False)
    seq = c.run_sequential(reqs[:seq_sample])
    return {"workload": SERVE_SMALL["desc"], "requests": len(reqs), "unit": "solves/s",
            "device_queue": {"value": qs.solves_per_s(), "p50_s": qs.latency_pct(50), "p99_s": qs.latency_pct(99)},
            "contexts": {"value": cs.solves_per_s(), "p50_s": cs.latency_pct(50), "p99_s": cs.latency_pct(99)},
            "sequential": {"value": seq.solves_per_s(), "sample": f"first {seq_sample} requests"},
            "queue_vs_contexts": qs.solves_per_s() / cs.solves_per_s(),
            "queue_vs_sequential": qs.solves_per_s() / seq.solves_per_s()}


def run_reference_arm(a, rank, world):
    if rank != 0:
        return
    n, m, k, _, desc = WORKLOADS[a.workload]
    # every step is the engine's step (J iterations + adjust + classification)
    # on the same full matrix; nothing is sampled or scaled
    r = cpu_port_rate(a.workload, J=a.iters_per_step, steps=a.steps, warmup=a.warmup)
    v = r["value"]
    line = {"impl": "reference", "metric": "KL-NMF iterations/s", "value": v, "unit": "iters/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * a.iters_per_step / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": desc, "n": n, "m": m, "k": k,
                                             "iters_per_step": a.iters_per_step},
            "cpu_baseline": r, "e2e": {"value": v, "unit": "iters/s", "h2d_bytes_per_step": 0,
                                       "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def replica_rate(ms, units_per_rank, world, device="cpu"):
    """Whole-job rate of `world` independent replicas (one per GPU): each rank
    processed `units_per_rank` in its own device time `ms`; the job's time is
    the slowest rank's (all-reduce MAX over the process group).  Returns
    (ms_max, units per second of the whole job)."""
    import torch
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    return ms_max, units_per_rank * world / (ms_max / 1e3)


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
    clk = ClockSampler(local_rank).__enter__()
    for _ in range(a.warmup):
        e.run(J, J, never)
    e.synchronize()
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    l0 = e.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk.mark(True)
    ev0.record(stream)
    for _ in range(a.steps):
        e.run(J, J, never)
    ev1.record(stream)
    ev1.synchronize()
    clk.mark(False)
    ms = ev0.elapsed_time(ev1)
    launches = e.launch_count() - l0
    # kernel times for the roofline: a separate pass with per-launch CUDA events
    # (events between launches disable the graph replay, so they stay out of the
    # timed loop above)
    e.profile(True)
    for _ in range(max(2, a.steps // 4)):
        e.run(J, J, never)
    e.synchronize()
    prof = {c: e.profile_read(c) for c in range(4)}
    e.profile(False)
    clk.__exit__(None, None, None)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ms_max, value = replica_rate(ms, a.steps * J, world, dev)

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
        for rep in range(3):       # the first solve also pays one-time host allocations
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
        _SAMPLES[a.workload] = V.cpu().numpy()
        cpu = cpu_port_rate(a.workload, J=a.iters_per_step, steps=1)
    e.close()
    extras = {}
    if rank == 0 and world == 1 and not a.no_extras:
        def guarded(fn, *args):
            # an extra measurement that fails is reported, not fatal to the line
            try:
                return fn(*args)
            except Exception as exc:
                return {"error": f"{type(exc).__name__}: {exc}"}

        extras["plain_arm"] = plain_arm_rate(a, pkg, V, dev, stream, n, m, k, hbm)
        extras["plain_arm"]["fused_speedup"] = value / extras["plain_arm"]["value"]
        extras["arms"] = {arm: guarded(other_arm_rate, a, pkg, V, dev, stream, n, m, k, hbm, arm)
                          for arm in ("bf16x3", "split_bf16", "bf16", "fused_tf32")}
        # each arm's error against FP64 on the 6000 x 500 submatrix, as measured by
        # the committed parity test's case (profiles/arm_precision.json)
        prec = arm_precision()
        if prec:
            extras["precision_vs_fp64"] = {"fused": prec.get(f"k{k}:fused"), "source": "profiles/arm_precision.json"}
            for arm, entry in extras["arms"].items():
                if isinstance(entry, dict) and f"k{k}:{arm}" in prec:
                    entry["precision_vs_fp64"] = prec[f"k{k}:{arm}"]
                    entry["speedup_vs_fp32_arm"] = entry.get("value", 0.0) / value
        del V
        torch.cuda.empty_cache()
        extras["workloads"] = {wl: guarded(workload_rate, a, pkg, dev, wl, hbm) for wl in ("C64", "B16")}
        eng = {"C32": value}
        if isinstance(extras["workloads"].get("B16"), dict) and "value" in extras["workloads"]["B16"]:
            eng["B16"] = extras["workloads"]["B16"]["value"]
        extras["reference_cuda"] = guarded(reference_cuda_rates, pkg, dev, eng)
        extras["sweep"] = guarded(sweep_rates, dev)
        extras["streamed"] = guarded(stream_rates, dev)
        extras["serving"] = guarded(serve_rates, dev)
        extras["serving_small"] = guarded(serve_small_rates, dev)
    if rank != 0:
        return
    line = {"metric": "KL-NMF iterations/s", "value": value, "unit": "iters/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "n": n, "m": m, "k": k, "arm": a.arm, "iters_per_step": J,
                       "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (V = %.2f GB)" % (n * m * 4 / 1e9)},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk.summary()}
    line.update(extras)
    print(json.dumps(line), flush=True)


def workload_rate(a, pkg, dev, wl, hbm, steps=20, arm="fused"):
    """The fused arm on another workload: iterations/s (steps of J iterations,
    L2 flushed before every timed step: B16's V fits in L2) and the dominant
    kernel's HBM fraction."""
    import torch
    n, m, k, _, desc = WORKLOADS[wl]
    V = make_V(wl, dev)
    stream = torch.cuda.Stream(device=dev)
    flush = L2Flush(dev)
    e = pkg.NMF(n, m, k, arm=arm, device=dev.index or 0)
    try:
        e.set_stream(stream.cuda_stream)
        e.set_V_device(V.data_ptr(), m)
        e.init_random(3)
        J = a.iters_per_step
        for _ in range(3):
            e.run(J, J, 2 ** 31)
        e.synchronize()
        ms = 0.0
        for _ in range(steps):
            flush(stream)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            e.run(J, J, 2 ** 31)
            ev1.record(stream)
            ev1.synchronize()
            ms += ev0.elapsed_time(ev1)
        e.profile(True)
        e.run(J, J, 2 ** 31)
        e.synchronize()
        prof = {c: e.profile_read(c) for c in range(4)}
        e.profile(False)
    finally:
        e.close()
        del V, flush
        torch.cuda.empty_cache()
    cls = 0 if prof[0][0] >= prof[1][0] else 1
    kms = prof[cls][0] / max(prof[cls][1], 1)
    value = steps * J / (ms / 1e3)
    return {"workload": desc, "value": value, "unit": "iters/s", "steps": steps, "iters_per_step": J,
            "l2": "256 MB written before every timed step" + (" (V fits in L2: within a step it is re-read from L2)"
                                                              if n * m * 4 < 126e6 else ""),
            "roofline": {"kernel": ("update_H" if cls == 0 else "update_W") + f"[{arm}]", "avg_launch_ms": kms,
                         "achieved": n * m * 4 / (kms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                         "frac": n * m * 4 / (kms / 1e3) / 1e9 / hbm},
            "iteration_frac_2nm4": 2.0 * n * m * 4 * value / 1e9 / hbm}


def other_arm_rate(a, pkg, V, dev, stream, n, m, k, hbm, arm, steps=5):
    """Another fused arm on the same V: iterations/s and its main kernel's HBM fraction."""
    import torch
    e = pkg.NMF(n, m, k, arm=arm, device=dev.index or 0)
    try:
        e.set_stream(stream.cuda_stream)
        e.set_V_device(V.data_ptr(), m)
        e.init_random(3)
        J = a.iters_per_step
        for _ in range(3):
            e.run(J, J, 2 ** 31)
        e.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            e.run(J, J, 2 ** 31)
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        e.profile(True)
        e.run(J, J, 2 ** 31)
        e.synchronize()
        tot, cnt = e.profile_read(0)
        e.profile(False)
    finally:
        e.close()
    kms = tot / max(cnt, 1)
    return {"value": steps * J / (ms / 1e3), "unit": "iters/s", "update_H_kernel_ms": kms,
            "roofline_frac": n * m * 4 / (kms / 1e3) / 1e9 / hbm}


def plain_arm_rate(a, pkg, V, dev, stream, n, m, k, hbm, steps=2):
    """The unfused FP32 arm on the same V and GPU: iterations/s and its roofline fraction."""
    import torch
    e = pkg.NMF(n, m, k, arm="plain", device=dev.index or 0)
    try:
        e.set_stream(stream.cuda_stream)
        e.set_V_device(V.data_ptr(), m)
        e.init_random(3)
        J = a.iters_per_step
        e.run(J, J, 2 ** 31)
        e.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            e.run(J, J, 2 ** 31)
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        e.profile(True)
        e.run(J, J, 2 ** 31)
        e.synchronize()
        tot, cnt = e.profile_read(2)
        e.profile(False)
    finally:
        e.close()
    half_ms = tot / max(cnt, 1)
    achieved = n * m * 4 / (half_ms / 1e3) / 1e9
    return {"value": steps * J / (ms / 1e3), "unit": "iters/s", "update_H_ms": half_ms,
            "roofline_frac": achieved / hbm, "note": "whole update_H (5 kernels) against n*m*4 bytes"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--arm", default="fused", choices=["fused", "plain", "fused_tf32", "bf16", "split_bf16", "bf16x3"])
    ap.add_argument("--workload", default="C32", choices=list(WORKLOADS))
    ap.add_argument("--iters-per-step", type=int, default=10)
    ap.add_argument("--e2e-iters", type=int, default=500)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the plain-arm and sweep measurements")
    ap.add_argument("--batch-wave", type=int, default=0, metavar="K",
                    help="profiling case of the batched kernel: one wave (2 per SM) of rank-K problems of the "
                         "sweep matrix, 20 iterations, run twice; prints the device times")
    ap.add_argument("--batch-ctas", type=int, default=0, help="CTAs per problem for --batch-wave (0 = automatic)")
    a = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference_arm(a, rank, world)
        return
    if a.batch_wave:
        pkg = _import_package()
        import nmf_b200.synth as synth
        V, _ = synth.config_d(SWEEP["seed"])
        nprob = 296
        with pkg.Batch(V.shape[0], V.shape[1], [a.batch_wave] * nprob) as b:
            b.set_V(V)
            b.init_random(np.arange(1, nprob + 1, dtype=np.uint32))
            b.set_cluster(a.batch_ctas)
            for rep in range(2):
                b.run(20, 20, 1 << 30)
                print(json.dumps({"batch_wave_k": a.batch_wave, "problems": nprob, "iterations": 20,
                                  "ctas_per_problem": b.cluster, "device_ms": b.last_ms()}), flush=True)
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
