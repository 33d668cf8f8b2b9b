"""Rank-selection sweeps on the batched engine, and its tile autotuner.

``rank_sweep`` runs every (rank, restart) pair of a sweep as one batch
(one persistent launch), then reduces each rank's restarts to an exact integer
consensus matrix and its cophenetic correlation -- the consensus method of
Brunet et al. (PNAS 2004) that the reference's user guide points to for
choosing the factorization rank (doc/user_guide.txt.md:367).

``autotune`` picks the batched kernel's tile shapes (wt rows of W per
update_H tile, jt columns of V per update_W tile) per (k, m) bucket by timing
short fixed-iteration runs of a full wave of problems on the device, and caches
the choice for the process.  Tile shapes change only the grouping of FP32
partial sums, never the method.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import Batch, NMFError  # noqa: F401

WT_CANDIDATES = (16, 32, 64)
JT_CANDIDATES = (16, 32, 64)

_TUNED: dict[tuple[int, int, int], tuple[int, int]] = {}


def _bucket(n: int, m: int, k: int) -> tuple[int, int, int]:
    """(k, m rounded up to a power of two, n rounded up to a power of two)."""
    return (int(k), 1 << max(0, math.ceil(math.log2(max(m, 1)))), 1 << max(0, math.ceil(math.log2(max(n, 1)))))


def autotune(V: np.ndarray, ranks, waves: int = 1, iters: int = 20, sm_count: int = 148, device: int = 0,
             verbose: bool = False) -> dict[int, tuple[int, int]]:
    """Choose (wt, jt) for every distinct rank in ``ranks`` on matrix V.

    For each rank, a batch of ``2 * sm_count * waves`` problems of that rank is
    timed for ``iters`` iterations (no convergence test) under every candidate
    shape; the fastest shape wins.  Results are cached per (k, m, n) bucket.
    """
    V = np.ascontiguousarray(V, np.float32)
    n, m = V.shape
    out: dict[int, tuple[int, int]] = {}
    for k in sorted(set(int(r) for r in ranks)):
        key = _bucket(n, m, k)
        if key in _TUNED:
            out[k] = _TUNED[key]
            continue
        nprob = 2 * sm_count * waves
        best, best_ms = None, float("inf")
        with Batch(n, m, [k] * nprob, device=device) as b:
            b.set_V(V)
            b.init_random(np.arange(1, nprob + 1, dtype=np.uint32))
            for wt in WT_CANDIDATES:
                for jt in JT_CANDIDATES:
                    try:
                        for p in range(nprob):
                            b.set_tiles(p, wt, jt)
                    except NMFError:
                        continue            # shape does not fit shared memory
                    b.run(iters, iters, 1 << 30)   # warm-up
                    b.run(iters, iters, 1 << 30)
                    ms = b.last_ms()
                    if verbose:
                        print(f"autotune k={k} m={m}: wt={wt} jt={jt}: {ms:.3f} ms")
                    if ms < best_ms:
                        best, best_ms = (wt, jt), ms
        if best is None:
            raise NMFError(-1, f"no tile shape fits k={k}, m={m}")
        _TUNED[key] = best
        out[k] = best
    return out


@dataclass
class SweepResult:
    ranks: np.ndarray               # per problem
    seeds: np.ndarray               # per problem
    iterations: np.ndarray          # per problem
    converged: np.ndarray           # per problem
    labels: np.ndarray              # nprob x m
    consensus: dict = field(default_factory=dict)    # k -> m x m uint32 counts
    cophenetic: dict = field(default_factory=dict)   # k -> float
    device_ms: float = 0.0          # persistent launch, CUDA events


def rank_sweep(V: np.ndarray, ks=range(2, 11), restarts: int = 50, seed0: int = 1, n_iters: int = 2000,
               niter_test_conv: int = 10, stop_threshold: int = 40, tiles: dict | None = None,
               tune: bool = False, device: int = 0) -> SweepResult:
    """Factorise V for every k in ``ks`` from ``restarts`` CPU_RANDOM seeds each
    (seed of restart r = seed0 + r), all in one batch, with the reference's
    stopping rules; then consensus and cophenetic correlation per k."""
    V = np.ascontiguousarray(V, np.float32)
    n, m = V.shape
    ks = [int(k) for k in ks]
    ranks = np.repeat(np.array(ks, np.uint32), restarts)
    seeds = np.tile(np.arange(seed0, seed0 + restarts, dtype=np.uint32), len(ks))
    if tiles is None and tune:
        tiles = autotune(V, ks, device=device)
    with Batch(n, m, ranks, device=device) as b:
        b.set_V(V)
        if tiles:
            for p, k in enumerate(ranks):
                if int(k) in tiles:
                    b.set_tiles(p, *tiles[int(k)])
        b.init_random(seeds)
        it, conv = b.run(n_iters, niter_test_conv, stop_threshold)
        res = SweepResult(ranks, seeds, it, conv, b.classification(), device_ms=b.last_ms())
        for k in ks:
            C, nruns, coph = b.consensus(k)
            res.consensus[k] = C
            res.cophenetic[k] = coph
    return res
