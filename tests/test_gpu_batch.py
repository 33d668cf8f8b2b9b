"""GPU tests of the batched engine (many solves of one V in one persistent
launch) and of its consensus / cophenetic summaries, against the CPU oracle,
the reference's own fixture for config D, and the single-problem engine.

Tolerances as for the single-problem engine: 1e-4 (max|dX| / max|X|) after a
fixed iteration count; identical iteration counts and classifications for runs
to convergence, W/H within 2e-3; consensus counts exact; cophenetic correlation
within 1e-12 of the oracle evaluated on the same counts.  Problems split over
a cluster of CTAs meet the same bars and repeat bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_cases, load_golden, maxnorm_rel

pytestmark = pytest.mark.gpu


def test_fixed_iterations_every_rank_vs_fp64_oracle(pkg, oracle, synth):
    V, _ = synth.expression_like(1500, 90, 4, seed=31)
    n, m = V.shape
    ranks = [2, 3, 4, 7, 11, 16, 20]
    seeds = [5 + r for r in ranks]
    with pkg.Batch(n, m, ranks) as b:
        b.set_V(V)
        b.init_random(seeds)
        it, conv = b.run(40, 10, 1000)
        assert (it == 40).all() and not conv.any()
        for p, (k, s) in enumerate(zip(ranks, seeds)):
            W0, H0 = oracle.init_random(s, n, m, k)
            Wr, Hr, _, _ = oracle.nmf(V, W0, H0, 40, 10, 1000, prec="f64")
            assert maxnorm_rel(b.W(p), Wr) < 1e-4, k
            assert maxnorm_rel(b.H(p), Hr) < 1e-4, k
        labels = b.classification()
        for p in range(len(ranks)):
            assert np.array_equal(labels[p], oracle.classify(b.H(p)))


def test_remainder_iterations_and_tile_shapes(pkg, oracle, synth):
    # n_iters % niter_test_conv != 0 runs the remainder without adjust; tile shapes only regroup FP32 sums
    V, _ = synth.expression_like(700, 150, 5, seed=2, zero_frac=0.02)
    n, m = V.shape
    shapes = [(8, 4), (16, 8), (32, 16), (64, 32)]
    with pkg.Batch(n, m, [5] * len(shapes)) as b:
        b.set_V(V)
        b.init_random([9] * len(shapes))
        for p, (wt, jt) in enumerate(shapes):
            b.set_tiles(p, wt, jt)
        it, conv = b.run(27, 10, 1000)
        assert (it == 27).all()
        W0, H0 = oracle.init_random(9, n, m, 5)
        Wr, Hr, _, _ = oracle.nmf(V, W0, H0, 27, 10, 1000, prec="f64")
        for p in range(len(shapes)):
            assert maxnorm_rel(b.W(p), Wr) < 1e-4 and maxnorm_rel(b.H(p), Hr) < 1e-4


def test_convergence_matches_single_engine_and_oracle(pkg, oracle, synth):
    V, _ = synth.config_a(1)
    n, m = V.shape
    seeds = [3, 4, 5]
    with pkg.Batch(n, m, [3] * len(seeds)) as b:
        b.set_V(V)
        b.init_random(seeds)
        it, conv = b.run(2000, 10, 40)
        labels = b.classification()
        for p, s in enumerate(seeds):
            W0, H0 = oracle.init_random(s, n, m, 3)
            Wr, Hr, it_r, conv_r = oracle.nmf(V, W0, H0, 2000, 10, 40)
            assert (int(it[p]), bool(conv[p])) == (it_r, conv_r)
            assert np.array_equal(labels[p], oracle.classify(Hr))
            assert maxnorm_rel(b.W(p), Wr) < 2e-3 and maxnorm_rel(b.H(p), Hr) < 2e-3
            with pkg.NMF(n, m, 3) as e:
                e.set_V(V)
                e.init_random(s)
                assert e.run(2000, 10, 40) == (int(it[p]), bool(conv[p]))
                assert np.array_equal(e.classification(), labels[p])


@pytest.mark.skipif("D_k5_conv" not in golden_cases(), reason="no config-D fixture")
def test_reference_fixture_config_d(pkg, oracle):
    g = load_golden("D_k5_conv")
    V = g["V"]
    n, m = V.shape
    with pkg.Batch(n, m, [int(g["k"])]) as b:
        b.set_V(V)
        b.init_random([int(g["seed"])])
        it, conv = b.run(int(g["n_iters"]), int(g["niter_test_conv"]), int(g["stop_threshold"]))
        assert int(it[0]) == int(g["iterations"]) and bool(conv[0]) == bool(g["converged"])
        assert maxnorm_rel(b.W(0), g["W"]) < 2e-3 and maxnorm_rel(b.H(0), g["H"]) < 2e-3
        assert np.array_equal(b.classification()[0], oracle.classify(g["H"]))


def test_consensus_and_cophenetic_vs_oracle(pkg, oracle, synth):
    V, _ = synth.expression_like(800, 60, 3, seed=12)
    n, m = V.shape
    ks, restarts = [2, 3, 4], 6
    ranks = np.repeat(ks, restarts)
    seeds = np.tile(np.arange(1, restarts + 1), len(ks))
    with pkg.Batch(n, m, ranks) as b:
        b.set_V(V)
        b.init_random(seeds)
        b.run(300, 10, 40)
        labels = b.classification()
        for k in ks:
            C, nruns, coph = b.consensus(k)
            assert nruns == restarts
            ref = oracle.consensus(labels[ranks == k])
            assert np.array_equal(C, ref)
            assert abs(coph - oracle.cophenetic(ref, nruns)) < 1e-12
        with pytest.raises(pkg.NMFError):
            b.consensus(9)


def test_rank_sweep_recovers_planted_rank(pkg, synth):
    import nmf_b200.sweep as sweep

    V, _ = synth.config_d(4)
    res = sweep.rank_sweep(V, ks=range(2, 8), restarts=8, n_iters=600)
    assert set(res.cophenetic) == set(range(2, 8))
    assert res.consensus[5].dtype == np.uint32 and res.consensus[5].shape == (200, 200)
    # the planted rank is perfectly stable across restarts
    assert res.cophenetic[5] > 0.99
    assert res.device_ms > 0


def test_autotuner_tiles_keep_the_method(pkg, oracle, synth):
    # the tile autotuner picks (wt, jt) per rank from its candidates, caches the
    # choice, and a batch run with the chosen tiles matches the FP64 oracle
    import nmf_b200.sweep as sweep

    V, _ = synth.config_d(4)
    n, m = V.shape
    tiles = sweep.autotune(V, [3, 5], iters=10)
    assert set(tiles) == {3, 5}
    for wt, jt in tiles.values():
        assert wt in sweep.WT_CANDIDATES and jt in sweep.JT_CANDIDATES
    assert sweep.autotune(V, [5]) == {5: tiles[5]}       # cached per (k, m, n) bucket
    ranks = [3, 3, 5, 5]
    seeds = [1, 2, 1, 2]
    with pkg.Batch(n, m, ranks) as b:
        b.set_V(V)
        for p, k in enumerate(ranks):
            b.set_tiles(p, *tiles[k])
        b.init_random(seeds)
        it, conv = b.run(30, 10, 10 ** 9)
        assert (it == 30).all()
        for p, (k, sd) in enumerate(zip(ranks, seeds)):
            W0, H0 = oracle.init_random(sd, n, m, k)
            Wr, Hr, _, _ = oracle.nmf(V, W0, H0, 30, 10, 10 ** 9, prec="f64")
            assert maxnorm_rel(b.W(p), Wr) < 1e-4 and maxnorm_rel(b.H(p), Hr) < 1e-4


@pytest.mark.parametrize("ctas", [1, 2, 4, 8])
def test_cluster_split_problems(pkg, oracle, synth, ctas):
    # Each problem on a cluster of `ctas` CTAs (rows of W split, partial sums
    # added in rank order): fixed iterations within 1e-4 of the FP64 oracle;
    # runs to convergence with the iteration counts and labels of one CTA per
    # problem, W/H within 2e-3; two runs bit-identical.
    V, _ = synth.expression_like(1500, 90, 4, seed=31)
    n, m = V.shape
    ranks = [2, 3, 4, 7, 11, 20]
    seeds = [5 + r for r in ranks]
    with pkg.Batch(n, m, ranks) as b:
        b.set_cluster(ctas)
        b.set_V(V)
        b.init_random(seeds)
        it, conv = b.run(40, 10, 1000)
        assert b.cluster == ctas and (it == 40).all()
        for p, (k, s) in enumerate(zip(ranks, seeds)):
            W0, H0 = oracle.init_random(s, n, m, k)
            Wr, Hr, _, _ = oracle.nmf(V, W0, H0, 40, 10, 1000, prec="f64")
            assert maxnorm_rel(b.W(p), Wr) < 1e-4 and maxnorm_rel(b.H(p), Hr) < 1e-4, k
    V, _ = synth.config_d(4)
    n, m = V.shape
    ranks = [3, 5, 5, 8]
    seeds = [1, 2, 3, 4]
    out = {}
    for c in (1, ctas, ctas):
        with pkg.Batch(n, m, ranks) as b:
            b.set_cluster(c)
            b.set_V(V)
            b.init_random(seeds)
            it, conv = b.run(2000, 10, 40)
            out.setdefault(c, []).append((it, conv, b.classification(), [b.W(p) for p in range(4)],
                                          [b.H(p) for p in range(4)]))
    one, a, b2 = out[1][0], out[ctas][-2], out[ctas][-1]
    assert np.array_equal(a[0], one[0]) and np.array_equal(a[1], one[1]) and np.array_equal(a[2], one[2])
    for p in range(4):
        assert maxnorm_rel(a[3][p], one[3][p]) < 2e-3 and maxnorm_rel(a[4][p], one[4][p]) < 2e-3
        assert np.array_equal(a[3][p], b2[3][p]) and np.array_equal(a[4][p], b2[4][p])


def test_cluster_with_empty_slices(pkg, oracle, synth):
    # n = 6 rows over 8 CTAs: CTAs 6 and 7 own no rows and contribute zero partials
    V, _ = synth.expression_like(6, 40, 2, seed=3)
    n, m = V.shape
    with pkg.Batch(n, m, [2, 3]) as b:
        b.set_cluster(8)
        b.set_V(V)
        b.init_random([7, 8])
        it, _ = b.run(20, 10, 1000)
        assert (it == 20).all()
        for p, k in enumerate((2, 3)):
            W0, H0 = oracle.init_random(7 + p, n, m, k)
            Wr, Hr, _, _ = oracle.nmf(V, W0, H0, 20, 10, 1000, prec="f64")
            assert maxnorm_rel(b.W(p), Wr) < 1e-4 and maxnorm_rel(b.H(p), Hr) < 1e-4


def test_invalid_batches(pkg):
    with pytest.raises(pkg.NMFError) as ei:
        pkg.Batch(100, 50, [2, 21])
    assert ei.value.code == -1
    with pytest.raises(pkg.NMFError):
        pkg.Batch(100, 50, [1])
    with pkg.Batch(100, 50, [3]) as b:
        with pytest.raises(pkg.NMFError) as ei:
            b.run(10, 10, 1)              # V not set
        assert ei.value.code == -5
        with pytest.raises(pkg.NMFError):
            b.set_tiles(0, 12, 16)        # wt not a multiple of 8
        with pytest.raises(pkg.NMFError):
            b.set_cluster(3)              # not 0, 1, 2, 4 or 8
