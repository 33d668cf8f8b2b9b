"""Serving loop: many independent NMF requests of different sizes on one GPU.

A request carries its own V (host memory), rank k, seed and stopping rules
(-i / -j / -t).  The server admits requests in arrival order while their
device memory (``context_bytes``, an upper bound of what the context
allocates) fits the HBM budget and a worker is free; each admitted request
gets its own context on its own CUDA stream, keeps V, W and H resident on the
device for its whole solve, and runs the reference's loop (``NMF.run``).  The
workers are host threads: the C ABI releases the interpreter lock, so the
contexts' kernels are queued concurrently and overlap on the device, and a
request that arrives while others run starts as soon as memory and a worker
free up (continuous admission; no request waits for a whole batch to drain).

Every kernel of a context sums in a fixed order that depends only on the
request's own sizes, so a request's result is the same alone and in any mix.
Context memory is stream-ordered (cudaMallocAsync), so creating and freeing
contexts does not stall the others.
"""
from __future__ import annotations

import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import NMF, NMFError, context_bytes  # noqa: F401


@dataclass
class Request:
    V: np.ndarray                 # n x m float32, host memory
    k: int
    seed: int = 1
    n_iters: int = 300
    niter_test_conv: int = 10
    stop_threshold: int = 40
    arrival: float = 0.0          # seconds after the start of the trace
    rid: int = 0


@dataclass
class Result:
    rid: int
    W: np.ndarray
    H: np.ndarray
    iterations: int
    converged: bool
    arrival: float                # trace time of arrival
    admitted: float               # trace time the context was created
    done: float                   # trace time the result was on the host

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class ServeStats:
    results: list = field(default_factory=list)
    wall_s: float = 0.0
    peak_bytes: int = 0
    peak_active: int = 0

    def solves_per_s(self) -> float:
        return len(self.results) / self.wall_s if self.wall_s > 0 else 0.0

    def latency_pct(self, q: float) -> float:
        lat = np.array([r.latency for r in self.results])
        return float(np.percentile(lat, q)) if lat.size else 0.0


class Server:
    """Admission by device-memory budget and worker count, FIFO order."""

    def __init__(self, budget_bytes: float = 120e9, workers: int = 16, arm: str = "fused", device: int = 0):
        self.budget = int(budget_bytes)
        self.workers = int(workers)
        self.arm = arm
        self.device = device

    def _arm_for(self, k: int) -> str:
        return self.arm if k <= 64 else "plain"

    def _solve(self, req: Request, t0: float, admitted: float) -> Result:
        n, m = req.V.shape
        with NMF(n, m, req.k, arm=self._arm_for(req.k), device=self.device) as e:
            e.set_V(req.V)
            e.init_random(req.seed)
            it, conv = e.run(req.n_iters, req.niter_test_conv, req.stop_threshold)
            W, H = e.W, e.H
        return Result(req.rid, W, H, it, conv, req.arrival, admitted, time.perf_counter() - t0)

    def run(self, requests: list[Request], open_loop: bool = True) -> ServeStats:
        """Serve `requests` (sorted by arrival).  open_loop: each request is
        released at its arrival time; otherwise all are available at t = 0."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        need = [context_bytes(r.V.shape[0], r.V.shape[1], r.k, self._arm_for(r.k), self.device) for r in reqs]
        for r, b in zip(reqs, need):
            if b > self.budget:
                raise NMFError(-3, f"request {r.rid} needs {b} bytes, more than the {self.budget}-byte budget")
        stats = ServeStats()
        lock = threading.Condition()
        state = {"bytes": 0, "active": 0}
        futures = []

        def finish(b):
            with lock:
                state["bytes"] -= b
                state["active"] -= 1
                lock.notify_all()

        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=self.workers) as pool:
            for r, b in zip(reqs, need):
                if open_loop:
                    wait = r.arrival - (time.perf_counter() - t0)
                    if wait > 0:
                        time.sleep(wait)
                with lock:
                    while state["bytes"] + b > self.budget or state["active"] >= self.workers:
                        lock.wait()
                    state["bytes"] += b
                    state["active"] += 1
                    stats.peak_bytes = max(stats.peak_bytes, state["bytes"])
                    stats.peak_active = max(stats.peak_active, state["active"])
                admitted = time.perf_counter() - t0
                if not open_loop:
                    r = Request(r.V, r.k, r.seed, r.n_iters, r.niter_test_conv, r.stop_threshold, 0.0, r.rid)

                def job(r=r, b=b, admitted=admitted):
                    try:
                        return self._solve(r, t0, admitted)
                    finally:
                        finish(b)

                futures.append(pool.submit(job))
            stats.results = [f.result() for f in futures]
        stats.wall_s = time.perf_counter() - t0
        return stats

    def run_sequential(self, requests: list[Request]) -> ServeStats:
        """The baseline: one request at a time, each through its own context."""
        stats = ServeStats()
        t0 = time.perf_counter()
        for r in sorted(requests, key=lambda r: r.arrival):
            res = self._solve(Request(r.V, r.k, r.seed, r.n_iters, r.niter_test_conv, r.stop_threshold, 0.0, r.rid),
                              t0, time.perf_counter() - t0)
            stats.results.append(res)
        stats.wall_s = time.perf_counter() - t0
        return stats


def poisson_arrivals(count: int, rate: float, seed: int = 0) -> np.ndarray:
    """Arrival times (s) of a Poisson process of `rate` requests per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=count))
