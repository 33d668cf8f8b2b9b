"""GPU tests of the blockwise (out-of-core) mode: V stays in host memory and
is streamed through the device in row blocks (nmfb_create_streamed).

Tolerances: against the FP64 oracle as for the resident arms (1e-4 after a
fixed iteration count; identical iteration count and classification at
convergence); against the resident plain FP32 arm 1e-5 (only the order of the
FP32 partial sums differs); the block-wise FP64 objectives within 1e-9 relative
of the oracle's on the same factors.  Inside a run, update_W's pass over V also
forms the next update_H's sum (one pass per iteration); the same run done as
single update calls, one pass per half-iteration, must give identical factors.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import maxnorm_rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("block_rows", [100, 257, 0])
def test_streamed_fixed_iterations(pkg, oracle, synth, block_rows):
    V, _ = synth.expression_like(1111, 97, 7, seed=8, zero_frac=0.05)
    n, m = V.shape
    W0, H0 = oracle.init_random(3, n, m, 7)
    Wr, Hr, _, _ = oracle.nmf(V, W0, H0, 25, 10, 1000, prec="f64")
    with pkg.NMF(n, m, 7, stream_rows=block_rows) as s, pkg.NMF(n, m, 7, arm="plain") as r:
        for e in (s, r):
            e.set_V(V)
            e.init_random(3)
            assert e.run(25, 10, 1000) == (25, False)
        assert maxnorm_rel(s.W, Wr) < 1e-4 and maxnorm_rel(s.H, Hr) < 1e-4
        assert maxnorm_rel(s.W, r.W) < 1e-5 and maxnorm_rel(s.H, r.H) < 1e-5
        # the block-wise FP64 objectives equal the oracle's on the same factors
        a, b = s.dot_product_VWH()
        ra, rb = oracle.dot_VWH(V, s.W, s.H)
        assert abs(a - ra) <= 1e-9 * ra and abs(b - rb) <= 1e-9 * rb
        kl = oracle.kl_divergence(V, s.W, s.H)
        assert abs(s.kl_divergence() - kl) <= 1e-9 * abs(kl)


def test_streamed_convergence_matches_oracle(pkg, oracle, synth):
    V, _ = synth.config_a(1)
    n, m = V.shape
    W0, H0 = oracle.init_random(3, n, m, 3)
    Wr, Hr, it_r, conv_r = oracle.nmf(V, W0, H0, 2000, 10, 40)
    with pkg.NMF(n, m, 3, stream_rows=512) as e:
        e.set_V(V)
        e.init_random(3)
        assert e.run(2000, 10, 40) == (it_r, conv_r)
        assert np.array_equal(e.classification(), oracle.classify(Hr))
        assert maxnorm_rel(e.W, Wr) < 2e-3 and maxnorm_rel(e.H, Hr) < 2e-3


def test_streamed_single_updates_and_restrictions(pkg, oracle, synth):
    V, _ = synth.expression_like(700, 333, 33, seed=3)
    n, m = V.shape
    W0, H0 = oracle.init_random(3, n, m, 33)
    with pkg.NMF(n, m, 33, stream_rows=64) as e:
        e.set_V(V)
        e.init_random(3)
        e.update_H()
        H1 = oracle.update_H(V, W0, H0, prec="f64")
        assert maxnorm_rel(e.H, H1) < 1e-5
        e.update_W()
        assert maxnorm_rel(e.W, oracle.update_W(V, W0, H1, prec="f64")) < 1e-5
        with pytest.raises(pkg.NMFError) as ei:
            e.set_arm("fused")
        assert ei.value.code == -1
        with pytest.raises(pkg.NMFError) as ei:
            e.device_V()
        assert ei.value.code == -5
        # a second V replaces the first (re-registered host memory)
        V2 = np.ascontiguousarray(V[:, ::-1])
        e.set_V(V2)
        e.set_WH(W0, H0)
        e.update_H()
        assert maxnorm_rel(e.H, oracle.update_H(V2, W0, H0, prec="f64")) < 1e-5


def test_single_pass_equals_separate_passes(pkg, oracle, synth):
    # nmfb_run folds update_H's pass into the previous update_W's pass (except
    # after a test block's last update_W, whose EPS adjust of H follows); the
    # same updates as single calls (two passes per iteration) give the same
    # factors bit for bit: same kernels, same operands, same block order
    V, _ = synth.expression_like(900, 130, 6, seed=12, zero_frac=0.02)
    n, m = V.shape
    W0, H0 = oracle.init_random(5, n, m, 6)
    with pkg.NMF(n, m, 6, stream_rows=128) as a, pkg.NMF(n, m, 6, stream_rows=128) as b:
        for e in (a, b):
            e.set_V(V)
            e.set_WH(W0, H0)
        assert a.run(7, 10, 1000) == (7, False)       # no test block: no adjust, every W pass folded
        for _ in range(7):
            b.update_H()
            b.update_W()
        assert np.array_equal(a.W, b.W) and np.array_equal(a.H, b.H)
        Wr, Hr, _, _ = oracle.nmf(V, W0, H0, 7, 10, 1000, prec="f64")
        assert maxnorm_rel(a.W, Wr) < 1e-4 and maxnorm_rel(a.H, Hr) < 1e-4
