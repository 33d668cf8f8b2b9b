"""GPU tests of the serving loop: concurrent requests of different sizes,
admitted by a device-memory budget, give exactly the results they give alone
(every kernel sums in a fixed order that depends only on the request's own
sizes), and the budget is never exceeded."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(synth, count=10, seed=0):
    import nmf_b200.serve as serve

    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        n = int(rng.integers(300, 3000))
        m = int(np.exp(rng.uniform(np.log(20), np.log(600))))
        k = int(rng.integers(2, 21))
        k = min(k, m, n)
        V, _ = synth.expression_like(n, m, max(2, k // 2), seed=100 + i)
        reqs.append(serve.Request(V, k, seed=1 + i, n_iters=60, niter_test_conv=10, stop_threshold=3,
                                  arrival=0.002 * i, rid=i))
    return reqs


def test_results_same_alone_and_in_the_mix(pkg, synth):
    import nmf_b200.serve as serve

    reqs = _requests(synth)
    srv = serve.Server(budget_bytes=40e9, workers=6)
    alone = {r.rid: r for r in srv.run_sequential(reqs).results}
    mixed = srv.run(reqs, open_loop=True)
    assert len(mixed.results) == len(reqs)
    assert mixed.peak_active > 1                      # requests really overlapped
    for r in mixed.results:
        a = alone[r.rid]
        assert (r.iterations, r.converged) == (a.iterations, a.converged)
        assert np.array_equal(r.W, a.W) and np.array_equal(r.H, a.H)
        assert r.latency > 0


def test_admission_respects_the_budget(pkg, synth):
    import nmf_b200.serve as serve

    reqs = _requests(synth, count=8, seed=1)
    need = sorted(pkg.context_bytes(r.V.shape[0], r.V.shape[1], r.k) for r in reqs)
    budget = need[-1] + need[-2]                    # room for about two requests at a time
    st = serve.Server(budget_bytes=budget, workers=8).run(reqs, open_loop=False)
    assert len(st.results) == len(reqs)
    assert st.peak_bytes <= budget
    too_big = serve.Server(budget_bytes=need[0] - 1, workers=2)
    with pytest.raises(pkg.NMFError):
        too_big.run(reqs[:1])
