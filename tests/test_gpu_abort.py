"""The fused kernels' bounded waits, made to run out on purpose.

Every device-side wait of the fused half-iteration kernels gives up after a
limit (1 s by default).  Here the limit is set to 1 ns through
nmfb_set_wait_limit, so the first wait that is not satisfied at once gives up:
its CTA stops its roles, drains the TMA loads and tensor-core work it has in
flight, frees its tensor memory and exits -- no fault, trap or hang.  The run
must report NMFB_ETIMEOUT, and the same context, with the default limit
restored and the factors re-initialised, must then produce the oracle's
result (the context stays usable).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import maxnorm_rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("arm", ["fused", "bf16x3"])
def test_wait_expiry_is_reported_and_context_recovers(pkg, oracle, synth, arm):
    V, _ = synth.expression_like(3000, 400, 8, seed=41)
    n, m = V.shape
    W0, H0 = oracle.init_random(3, n, m, 8)
    W64, H64, _, _ = oracle.nmf(V, W0, H0, 20, 10, 10 ** 9, prec="f64")
    with pkg.NMF(n, m, 8, arm=arm) as e:
        e.set_V(V)
        e.init_random(3)
        e.set_wait_limit(1)
        with pytest.raises(pkg.NMFError) as ei:
            e.run(20, 10, 10 ** 9)
        assert ei.value.code == -6 and "bounded wait" in str(ei.value)
        e.set_wait_limit(0)
        e.init_random(3)
        it, conv = e.run(20, 10, 10 ** 9)
        assert (it, conv) == (20, False)
        tol = 1e-4 if arm == "fused" else 1e-3
        assert maxnorm_rel(e.W, W64) < tol and maxnorm_rel(e.H, H64) < tol
        e.synchronize()                       # the error was reported once and cleared
