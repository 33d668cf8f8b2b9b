"""GPU tests of the reduced- and mixed-precision fused arms against the FP64
oracle (the precision comparison of the 60000 x 5000 workloads, at sizes the
oracle finishes in seconds).

Tolerances, from the operand rounding of each arm (u = unit roundoff):
  * bf16x3 (split-BF16 in both contractions, 16 significant bits per operand):
    one update within 1e-5 (max|dX| / max|X|); run to convergence: the same
    iteration count as the FP64 oracle and a final KL divergence within 1e-5
    relative -- the FP32 arm's bar;
  * split_bf16 (split-BF16 WH denominator, one BF16 product in the second
    contraction): one update within 4e-3 (u_bf16 = 2^-8 = 3.9e-3 bounds the
    rounding of R and Y); final KL within 1e-3;
  * bf16 (one BF16 product in both): one update within 8e-3 (2 u_bf16); final
    KL within 1e-3.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import maxnorm_rel

pytestmark = pytest.mark.gpu

SINGLE_TOL = {"bf16x3": 1e-5, "split_bf16": 4e-3, "bf16": 8e-3}
KL_TOL = {"bf16x3": 1e-5, "split_bf16": 1e-3, "bf16": 1e-3, "fused": 1e-5}


@pytest.mark.parametrize("arm", list(SINGLE_TOL))
@pytest.mark.parametrize("shape", [(300, 70, 5), (1000, 130, 16), (700, 333, 33), (257, 190, 64)])
def test_single_half_updates(pkg, oracle, synth, arm, shape):
    n, m, k = shape
    V, _ = synth.expression_like(n, m, k, seed=n + m)
    W0, H0 = oracle.init_random(3, n, m, k)
    H1 = oracle.update_H(V, W0, H0, prec="f64")
    W1 = oracle.update_W(V, W0, H1, prec="f64")
    with pkg.NMF(n, m, k, arm=arm) as e:
        e.set_V(V)
        e.init_random(3)
        e.update_H()
        assert maxnorm_rel(e.H, H1) < SINGLE_TOL[arm]
        e.update_W()
        assert maxnorm_rel(e.W, W1) < SINGLE_TOL[arm]


@pytest.fixture(scope="module")
def converged_case(oracle, synth):
    V, _ = synth.expression_like(3000, 400, 8, seed=21, zero_frac=0.01)
    n, m = V.shape
    W0, H0 = oracle.init_random(3, n, m, 8)
    W64, H64, it64, conv64 = oracle.nmf(V, W0, H0, 2000, 10, 40, prec="f64")
    kl64 = oracle.kl_divergence(V, W64.astype(np.float32), H64.astype(np.float32))
    return V, it64, conv64, kl64


@pytest.mark.parametrize("arm", list(KL_TOL))
def test_final_divergence_vs_fp64(pkg, converged_case, arm):
    V, it64, conv64, kl64 = converged_case
    n, m = V.shape
    with pkg.NMF(n, m, 8, arm=arm) as e:
        e.set_V(V)
        e.init_random(3)
        it, conv = e.run(2000, 10, 40)
        assert conv and conv64
        if arm in ("bf16x3", "fused"):
            assert it == it64
        assert abs(e.kl_divergence() - kl64) <= KL_TOL[arm] * kl64


def test_arm_switch_on_one_context(pkg, oracle, synth):
    # the same context moves between arms; every arm starts from the same factors
    V, _ = synth.expression_like(600, 120, 6, seed=4)
    n, m = V.shape
    W0, H0 = oracle.init_random(5, n, m, 6)
    H1 = oracle.update_H(V, W0, H0, prec="f64")
    with pkg.NMF(n, m, 6, arm="fused") as e:
        e.set_V(V)
        for arm in ("bf16x3", "split_bf16", "bf16", "fused", "bf16x3"):
            e.set_arm(arm)
            e.set_WH(W0, H0)
            e.update_H()
            tol = SINGLE_TOL.get(arm, 1e-5)
            assert maxnorm_rel(e.H, H1) < tol, arm
