"""Serving loop: many independent NMF requests of different sizes on one GPU.

A request carries its own V (host memory), rank k, seed and stopping rules
(-i / -j / -t).  The server admits requests in arrival order while their
device memory fits the HBM budget, and runs each on one of two paths:

* requests whose H fits a CTA's shared memory (m <= max_m, k <= 20) go to the
  device queue (``Serve``, ``nmfb_serve_*``): the admission thread uploads V
  and queues the request, a persistent kernel's clusters of CTAs take queued
  requests as they free up and run the reference's loop on them, and a
  collector thread fetches finished ones.  Requests that arrive while others
  are on the GPU join the running kernel (continuous batching); no launch per
  iteration or per request;
* larger requests get their own context on their own CUDA stream (V, W, H
  resident for the whole solve, ``NMF.run``), driven by worker threads (the C
  ABI releases the interpreter lock, so the contexts' kernels overlap);
  ``sm_limit`` sizes each context's launches for that many SMs, so that
  several requests' kernels share the GPU side by side.

Both paths sum in a fixed order that depends only on the request's own sizes,
so a request's result is the same alone and in any mix.  Device memory of
both paths is stream-ordered, so admitting and retiring requests does not
stall the others.
"""
from __future__ import annotations

import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import NMF, NMFError, Serve, context_bytes  # noqa: F401


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
    """Admission by device-memory budget (and, for the context path, worker
    count), FIFO order.  batched=True sends requests that fit (m <= max_m,
    k <= 20) to the device queue.  It is off by default: on one GPU the
    persistent serving CTAs (two per SM) and the fused kernels of the context
    path cannot share an SM, so in a mixed stream each path waits for the
    other's SMs (measured: a mix served both ways ran slower than with
    contexts alone)."""

    def __init__(self, budget_bytes: float = 120e9, workers: int = 16, arm: str = "fused", device: int = 0,
                 batched: bool = False, max_m: int = 256, ctas: int = 4, sm_limit: int = 0):
        self.budget = int(budget_bytes)
        self.workers = int(workers)
        self.arm = arm
        self.device = device
        self.batched = batched
        self.max_m = int(max_m)
        self.ctas = int(ctas)
        self.sm_limit = int(sm_limit)   # SMs each context sizes its launches for (0: all)

    def _arm_for(self, k: int) -> str:
        return self.arm if k <= 64 else "plain"

    def _queued(self, r: Request) -> bool:
        return self.batched and r.V.shape[1] <= self.max_m and 2 <= r.k <= 20

    def _bytes(self, r: Request) -> int:
        n, m = r.V.shape
        if self._queued(r):
            return Serve.request_bytes(n, m, r.k)
        return context_bytes(n, m, r.k, self._arm_for(r.k), self.device)

    def _solve(self, req: Request, t0: float, admitted: float, sm_limit: int | None = None) -> Result:
        n, m = req.V.shape
        sm_limit = self.sm_limit if sm_limit is None else sm_limit
        with NMF(n, m, req.k, arm=self._arm_for(req.k), device=self.device) as e:
            if sm_limit:
                e.set_sm_limit(sm_limit)
            e.set_V(req.V)
            e.init_random(req.seed)
            it, conv = e.run(req.n_iters, req.niter_test_conv, req.stop_threshold)
            W, H = e.W, e.H
        return Result(req.rid, W, H, it, conv, req.arrival, admitted, time.perf_counter() - t0)

    def run(self, requests: list[Request], open_loop: bool = True) -> ServeStats:
        """Serve `requests` (sorted by arrival).  open_loop: each request is
        released at its arrival time; otherwise all are available at t = 0."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        need = [self._bytes(r) for r in reqs]
        for r, b in zip(reqs, need):
            if b > self.budget:
                raise NMFError(-3, f"request {r.rid} needs {b} bytes, more than the {self.budget}-byte budget")
        stats = ServeStats()
        lock = threading.Condition()
        state = {"bytes": 0, "active": 0, "workers": 0, "admitting": True}
        futures, pending, queued_results = [], {}, []
        q = Serve(max_m=self.max_m, ctas=self.ctas, device=self.device) if self.batched else None

        def finish(b, worker):
            with lock:
                state["bytes"] -= b
                state["active"] -= 1
                if worker:
                    state["workers"] -= 1
                lock.notify_all()

        t0 = time.perf_counter()

        errors = []

        def collect():
            try:
                collect_loop()
            except BaseException as exc:   # surfaced by the admission loop and after the join
                with lock:
                    errors.append(exc)
                    lock.notify_all()

        def collect_loop():
            # fetch finished queued requests until admission is over and none is pending
            while True:
                with lock:
                    if not state["admitting"] and not pending:
                        return
                    items = list(pending.items())
                got = False
                for ticket, (r, b, admitted) in items:
                    if q.poll(ticket):
                        W, H, _, it, conv = q.fetch(ticket)
                        queued_results.append(Result(r.rid, W, H, it, conv, r.arrival, admitted,
                                                     time.perf_counter() - t0))
                        with lock:
                            del pending[ticket]
                        finish(b, False)
                        got = True
                if not got:
                    time.sleep(1e-4)

        collector = threading.Thread(target=collect, daemon=True) if q else None
        if collector:
            collector.start()
        try:
            with ThreadPoolExecutor(max_workers=self.workers) as pool:
                for r, b in zip(reqs, need):
                    if open_loop:
                        wait = r.arrival - (time.perf_counter() - t0)
                        if wait > 0:
                            time.sleep(wait)
                    queued = q is not None and self._queued(r)
                    with lock:
                        while not errors and (state["bytes"] + b > self.budget or
                                              (not queued and state["workers"] >= self.workers)):
                            lock.wait()
                        if errors:
                            raise errors[0]
                        state["bytes"] += b
                        state["active"] += 1
                        if not queued:
                            state["workers"] += 1
                        stats.peak_bytes = max(stats.peak_bytes, state["bytes"])
                        stats.peak_active = max(stats.peak_active, state["active"])
                    admitted = time.perf_counter() - t0
                    if not open_loop:
                        r = Request(r.V, r.k, r.seed, r.n_iters, r.niter_test_conv, r.stop_threshold, 0.0, r.rid)
                    if queued:
                        ticket = q.submit(r.V, r.k, r.seed, r.n_iters, r.niter_test_conv, r.stop_threshold)
                        with lock:
                            pending[ticket] = (r, b, admitted)
                        continue

                    def job(r=r, b=b, admitted=admitted):
                        try:
                            return self._solve(r, t0, admitted)
                        finally:
                            finish(b, True)

                    futures.append(pool.submit(job))
                with lock:
                    state["admitting"] = False
                stats.results = [f.result() for f in futures]
            if collector:
                collector.join()
            if errors:
                raise errors[0]
            stats.results += queued_results
        finally:
            with lock:
                state["admitting"] = False
                if collector and collector.is_alive():
                    pending.clear()
            if q:
                q.close()
        stats.wall_s = time.perf_counter() - t0
        return stats

    def run_sequential(self, requests: list[Request]) -> ServeStats:
        """The baseline: one request at a time, each through its own context
        sized for the whole device (sm_limit does not apply)."""
        stats = ServeStats()
        t0 = time.perf_counter()
        for r in sorted(requests, key=lambda r: r.arrival):
            res = self._solve(Request(r.V, r.k, r.seed, r.n_iters, r.niter_test_conv, r.stop_threshold, 0.0, r.rid),
                              t0, time.perf_counter() - t0, sm_limit=0)
            stats.results.append(res)
        stats.wall_s = time.perf_counter() - t0
        return stats


def poisson_arrivals(count: int, rate: float, seed: int = 0) -> np.ndarray:
    """Arrival times (s) of a Poisson process of `rate` requests per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=count))
