"""CPU tests of the oracle: known answers, the reference's own semantics, and
the pin against fixtures produced by the reference's CUDA build."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import golden_cases, load_golden, maxnorm_rel


def test_init_random_matches_glibc(oracle):
    # src/NMF_routines.c:299-307: (float)random()/(float)RAND_MAX + FLT_MIN, W then H.
    libc = ctypes.CDLL("libc.so.6")
    libc.random.restype = ctypes.c_long
    libc.srandom(3)
    want = np.array([np.float32(libc.random()) / np.float32(2147483647) for _ in range(5 * 4 + 3 * 4)],
                    dtype=np.float32) + np.float32(np.finfo(np.float32).tiny)
    W, H = oracle.init_random(3, 5, 3, 4)
    got = np.concatenate([W.ravel(), H.ravel()])
    assert np.array_equal(got, want.astype(np.float32))


def test_difference_known_answers(oracle):
    a = np.array([0, 0, 1, 1], np.uint32)
    assert oracle.difference(a, a) == 0
    # relabelling does not change the partition
    assert oracle.difference(a, np.array([5, 5, 2, 2], np.uint32)) == 0
    # all-in-one vs two groups: pairs (0,2),(0,3),(1,2),(1,3) differ
    assert oracle.difference(a, np.zeros(4, np.uint32)) == 4
    assert oracle.difference(np.array([0, 1, 2], np.uint32), np.array([0, 0, 0], np.uint32)) == 3


def test_classify_tie_rule(oracle):
    k = 32
    H = np.zeros((4, k), np.float32)
    H[0, :] = 1.0                      # all equal -> lane 0 keeps its own column
    H[1, 8] = H[1, 16] = 2.0           # xor butterfly: lane 0 merges {0,16} before {8,24} -> 16
    H[2, 31] = 5.0                     # unique max
    H[3, 3] = H[3, 1] = 7.0            # {1,17,..} vs {3,..}: lane 0 side holds 1 first
    got = oracle.classify(H)
    assert list(got) == [0, 16, 31, 1]


def test_classify_wide_rank(oracle):
    # k > 96: block width next_pow2(ceil(ceil32(k)/3)) with a shared-memory tree.
    rng = np.random.default_rng(0)
    H = rng.random((50, 100)).astype(np.float32)
    got = oracle.classify(H)
    assert np.array_equal(got, H.argmax(axis=1).astype(np.uint32))  # no ties -> plain argmax
    # ties across the tree: columns 10 and 74 (10 + 64) equal and maximal.
    T = np.zeros((1, 100), np.float32)
    T[0, 10] = T[0, 74] = 3.0
    assert oracle.classify(T)[0] == 10


def test_adjust_semantics(oracle):
    A = np.array([[0.0, np.nan, 1e-40, 2.0]], np.float32)
    out = oracle.adjust(A)
    tiny = np.finfo(np.float32).tiny
    assert out[0, 0] == tiny and out[0, 1] == tiny and out[0, 2] == tiny and out[0, 3] == 2.0


def test_update_formulas_small(oracle):
    # Direct check of one H and one W update against numpy in float64.
    rng = np.random.default_rng(1)
    V = rng.random((7, 5)).astype(np.float32) + 0.1
    W = rng.random((7, 3)) + 0.1
    H = rng.random((5, 3)) + 0.1
    Q = V / (W @ H.T)
    H1 = H * (Q.T @ W) / W.sum(axis=0)
    got = oracle.update_H(V, W, H, prec="f64")
    assert np.allclose(got, H1, rtol=1e-13)
    Q = V / (W @ H1.T)
    W1 = W * (Q @ H1) / H1.sum(axis=0)
    assert np.allclose(oracle.update_W(V, W, H1, prec="f64"), W1, rtol=1e-13)


def test_fp32_tracks_fp64(oracle, synth):
    V, _ = synth.config_a(1)
    W, H = oracle.init_random(3, *V.shape, 3)
    W32, H32, _, _ = oracle.nmf(V, W, H, 50, 100, 40, prec="f32")
    W64, H64, _, _ = oracle.nmf(V, W, H, 50, 100, 40, prec="f64")
    assert maxnorm_rel(W32, W64) < 1e-4 and maxnorm_rel(H32, H64) < 1e-4


def test_loop_semantics_earliest_convergence(oracle, synth):
    # Stable classes from the first test: converges at the (t+2)-th test.
    V, _ = synth.config_a(1)
    W, H = oracle.init_random(3, *V.shape, 3)
    _, _, it, conv = oracle.nmf(V, W, H, 2000, 10, 40)
    assert conv and it == 420
    _, _, it, conv = oracle.nmf(V, W, H, 200, 10, 40)      # cap before convergence
    assert not conv and it == 200
    _, _, it, conv = oracle.nmf(V, W, H, 5, 10, 40)        # -j > -i: no test at all
    assert not conv and it == 5


CASES = golden_cases()


@pytest.mark.skipif(not CASES, reason="no reference fixtures")
@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_fixture(oracle, synth, case):
    g = load_golden(case)
    V = g["V"]
    n, m = V.shape
    k = int(g["k"])
    W0, H0 = oracle.init_random(int(g["seed"]), n, m, k)
    W, H, it, conv = oracle.nmf(V, W0, H0, int(g["n_iters"]), int(g["niter_test_conv"]), int(g["stop_threshold"]))
    assert it == int(g["iterations"])
    assert conv == bool(g["converged"])
    # Frobenius distance as printed by the reference (%g: 6 significant digits).
    a, b = oracle.dot_VWH(V, W, H)
    assert abs(np.sqrt(b / a) - float(g["distance"])) <= 1e-5 * float(g["distance"]) + 5e-7
    tol = 1e-4 if int(g["n_iters"]) <= 100 else 2e-3
    assert maxnorm_rel(W, g["W"]) < tol
    assert maxnorm_rel(H, g["H"]) < tol
    assert np.array_equal(oracle.classify(H), oracle.classify(g["H"]))
