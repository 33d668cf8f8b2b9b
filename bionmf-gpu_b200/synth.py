"""Seeded planted-factor matrices for the KL-NMF workloads.

The reference ships one example matrix (5000 x 38 expression data) and no
generator for the workloads it is measured on, so these seeded generators
stand in for them with the same shapes and value distributions:

* ``expression_like`` -- V = (W0 . H0) * lognormal(0, sigma), floored: W0 is
  lognormal(0, 1) with 5 % of the entries of every column boosted x10, H0 has
  one dominant factor (1.0) per sample and the others uniform in [0, 0.1].
* ``poisson_counts``  -- V = Poisson(scale * W0 . H0) as float32.

Both return float32 arrays (row-major n x m) and the planted class of every
sample (column).  ``numpy`` is used below ~50 M entries; the large variants
generate on a CUDA device through torch when one is given.
"""
from __future__ import annotations

import numpy as np


def class_sizes(m: int, k: int, rng: np.random.Generator, dirichlet: float | None = None,
                sizes=None) -> np.ndarray:
    if sizes is not None:
        s = np.asarray(sizes, dtype=np.int64)
        assert s.sum() == m and s.size == k
        return s
    if dirichlet is None:
        base = np.full(k, m // k, dtype=np.int64)
        base[: m - base.sum()] += 1
        return base
    p = rng.dirichlet(np.full(k, dirichlet))
    s = np.maximum(1, np.floor(p * m).astype(np.int64))
    while s.sum() > m:
        s[np.argmax(s)] -= 1
    while s.sum() < m:
        s[np.argmin(s)] += 1
    return s


def planted_factors(n: int, m: int, k: int, seed: int, *, sizes=None, dirichlet=None,
                    boost_frac=0.05, boost=10.0, off=0.1):
    """W0 (n x k), H0 (k x m) and the planted class of each sample."""
    rng = np.random.default_rng(seed)
    W0 = rng.lognormal(0.0, 1.0, size=(n, k)).astype(np.float64)
    nb = max(1, int(round(boost_frac * n)))
    for c in range(k):
        rows = rng.choice(n, size=nb, replace=False)
        W0[rows, c] *= boost
    cs = class_sizes(m, k, rng, dirichlet=dirichlet, sizes=sizes)
    labels = np.repeat(np.arange(k), cs)
    rng.shuffle(labels)
    H0 = rng.uniform(0.0, off, size=(k, m))
    H0[labels, np.arange(m)] = 1.0
    return W0, H0, labels.astype(np.uint32), rng


def expression_like(n: int, m: int, k: int, seed: int, *, sigma=0.2, floor=1e-9, sizes=None,
                    dirichlet=None, zero_frac=0.0):
    """Planted V = (W0 H0) * lognormal(0, sigma), floored at `floor` (float32)."""
    W0, H0, labels, rng = planted_factors(n, m, k, seed, sizes=sizes, dirichlet=dirichlet)
    V = (W0 @ H0) * rng.lognormal(0.0, sigma, size=(n, m))
    V = np.maximum(V, floor)
    if zero_frac > 0:
        nz = int(round(zero_frac * n * m))
        flat = rng.choice(n * m, size=nz, replace=False)
        V.reshape(-1)[flat] = 0.0
    return np.ascontiguousarray(V, dtype=np.float32), labels


def poisson_counts(n: int, m: int, k: int, seed: int, *, scale=50.0, sizes=None, dirichlet=None,
                   device=None):
    """Planted V = Poisson(scale * W0 H0) as float32; on `device` (torch) if given."""
    W0, H0, labels, _ = planted_factors(n, m, k, seed, sizes=sizes, dirichlet=dirichlet)
    if device is not None:
        import torch
        g = torch.Generator(device=device)
        g.manual_seed(seed)
        lam = (torch.from_numpy(W0).to(device=device, dtype=torch.float32)
               @ torch.from_numpy(H0).to(device=device, dtype=torch.float32)) * scale
        V = torch.poisson(lam, generator=g)
        return V, labels
    rng = np.random.default_rng(seed + 1)
    V = rng.poisson(scale * (W0 @ H0)).astype(np.float32)
    return V, labels


def config_a(seed: int = 1):
    """5000 x 38, k = 3; classes 12/13/13 (shape of the reference's example)."""
    return expression_like(5000, 38, 3, seed, sizes=[12, 13, 13])


def config_b(seed: int = 2):
    """20000 x 1000, k = 16; Dirichlet(2) class sizes; 1 % exact zeros."""
    return expression_like(20000, 1000, 16, seed, dirichlet=2.0, zero_frac=0.01)


def config_d(seed: int = 4):
    """5000 x 200 planted with true k = 5 (rank-selection sweep input)."""
    return expression_like(5000, 200, 5, seed)
