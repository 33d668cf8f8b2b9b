"""CPU tests of the oracle's consensus and cophenetic-correlation restatement.

The consensus counts are checked against a direct numpy evaluation; the
cophenetic correlation of average linkage is pinned against SciPy's published
implementation (scipy.cluster.hierarchy.linkage(method="average") + cophenet)
on distance matrices without ties, where the dendrogram is unique.
"""
from __future__ import annotations

import numpy as np
import pytest


def test_consensus_counts_match_numpy(oracle):
    rng = np.random.default_rng(5)
    labels = rng.integers(0, 4, size=(17, 60)).astype(np.uint32)
    C = oracle.consensus(labels)
    ref = (labels[:, :, None] == labels[:, None, :]).sum(axis=0)
    assert np.array_equal(C, ref)
    assert np.all(np.diag(C) == 17)


@pytest.mark.parametrize("m,seed", [(5, 1), (40, 2), (150, 3)])
def test_cophenetic_matches_scipy(oracle, m, seed):
    from scipy.cluster.hierarchy import cophenet, linkage
    from scipy.spatial.distance import squareform

    rng = np.random.default_rng(seed)
    X = rng.normal(size=(m, 3))
    D = np.sqrt(((X[:, None, :] - X[None, :, :]) ** 2).sum(-1))
    np.fill_diagonal(D, 0.0)
    cond = squareform(D, checks=False)
    ref, _ = cophenet(linkage(cond, method="average"), cond)
    assert abs(oracle.cophenetic_dist(D) - ref) < 1e-12


def test_cophenetic_of_perfect_consensus_is_one(oracle):
    # every run agrees on two classes -> D is 0 within and 1 across: dendrogram reproduces D exactly
    labels = np.tile(np.array([0] * 7 + [1] * 5, np.uint32), (10, 1))
    C = oracle.consensus(labels)
    assert abs(oracle.cophenetic(C, 10) - 1.0) < 1e-15
