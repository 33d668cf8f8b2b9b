"""GPU tests of the serving loop: concurrent requests of different sizes,
admitted by a device-memory budget, give exactly the results they give alone
(every kernel sums in a fixed order that depends only on the request's own
sizes), and the budget is never exceeded.  Requests small enough for the
device queue (``Serve``: a persistent kernel fed while it runs) match the FP64
oracle within 1e-4 after a fixed iteration count, like the batched engine."""
from __future__ import annotations

import time

import numpy as np
import pytest

from conftest import maxnorm_rel

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


@pytest.mark.parametrize("batched", [True, False])
def test_results_same_alone_and_in_the_mix(pkg, synth, batched):
    import nmf_b200.serve as serve

    reqs = _requests(synth)
    srv = serve.Server(budget_bytes=40e9, workers=6, batched=batched)
    assert any(srv._queued(r) for r in reqs) == batched and any(not srv._queued(r) for r in reqs)
    alone = {}
    for r in reqs:                                    # each request alone through the same server
        alone[r.rid] = srv.run([r], open_loop=False).results[0]
    mixed = srv.run(reqs, open_loop=True)
    assert len(mixed.results) == len(reqs)
    assert mixed.peak_active > 1                      # requests really overlapped
    for r in mixed.results:
        a = alone[r.rid]
        assert (r.iterations, r.converged) == (a.iterations, a.converged)
        assert np.array_equal(r.W, a.W) and np.array_equal(r.H, a.H)
        assert r.latency > 0
    if not batched:                                   # the context path alone = one context at a time
        seq = {r.rid: r for r in srv.run_sequential(reqs).results}
        for r in mixed.results:
            assert np.array_equal(r.W, seq[r.rid].W) and np.array_equal(r.H, seq[r.rid].H)


def test_sm_limit_same_alone_and_in_the_mix(pkg, synth):
    """Contexts sized for 37 SMs: a request's result is the same alone and in
    the mix, and within FP32 summation-order noise of the whole-device run."""
    import nmf_b200.serve as serve

    reqs = _requests(synth, count=8, seed=2)
    srv = serve.Server(budget_bytes=40e9, workers=6, sm_limit=37)
    alone = {r.rid: srv.run([r], open_loop=False).results[0] for r in reqs}
    mixed = srv.run(reqs, open_loop=True)
    full = {r.rid: r for r in srv.run_sequential(reqs).results}
    assert mixed.peak_active > 1
    for r in mixed.results:
        a, f = alone[r.rid], full[r.rid]
        assert np.array_equal(r.W, a.W) and np.array_equal(r.H, a.H)
        assert maxnorm_rel(r.W, f.W) < 1e-4 and maxnorm_rel(r.H, f.H) < 1e-4


def test_admission_respects_the_budget(pkg, synth):
    import nmf_b200.serve as serve

    reqs = _requests(synth, count=8, seed=1)
    srv = serve.Server(budget_bytes=1, workers=8, batched=True)
    need = sorted(srv._bytes(r) for r in reqs)
    budget = need[-1] + need[-2]                    # room for about two requests at a time
    st = serve.Server(budget_bytes=budget, workers=8, batched=True).run(reqs, open_loop=False)
    assert len(st.results) == len(reqs)
    assert st.peak_bytes <= budget
    too_big = serve.Server(budget_bytes=srv._bytes(reqs[0]) - 1, workers=2, batched=True)
    with pytest.raises(pkg.NMFError):
        too_big.run(reqs[:1])


def test_queue_fixed_iterations_vs_fp64_oracle(pkg, oracle, synth):
    shapes = [(1500, 90, 4), (700, 150, 7), (2100, 40, 2), (300, 256, 20)]
    with pkg.Serve(max_m=256, ctas=4) as q:
        tickets = []
        for i, (n, m, k) in enumerate(shapes):
            V, _ = synth.expression_like(n, m, max(2, k // 2), seed=50 + i)
            tickets.append((q.submit(V, k, seed=3 + i, n_iters=40, niter_test_conv=10, stop_threshold=1000),
                            V, k, 3 + i))
        for t, V, k, s in tickets:
            q.wait(t)
            W, H, lab, it, conv = q.fetch(t)
            assert (it, conv) == (40, False)
            n, m = V.shape
            W0, H0 = oracle.init_random(s, n, m, k)
            Wr, Hr, _, _ = oracle.nmf(V, W0, H0, 40, 10, 1000, prec="f64")
            assert maxnorm_rel(W, Wr) < 1e-4 and maxnorm_rel(H, Hr) < 1e-4, (n, m, k)
            assert np.array_equal(lab, oracle.classify(H))


def test_queue_convergence_matches_batched_engine(pkg, synth):
    # the same solve through the device queue and through a batch with the
    # same cluster size and tile shapes: identical bits
    V, _ = synth.config_d(4)
    n, m = V.shape
    with pkg.Serve(max_m=256, ctas=4) as q:
        t = q.submit(V, 5, seed=2)
        q.wait(t)
        W, H, lab, it, conv = q.fetch(t)
    with pkg.Batch(n, m, [5]) as b:
        b.set_cluster(4)
        b.set_tiles(0, 16, 16)
        b.set_V(V)
        b.init_random([2])
        itb, convb = b.run(2000, 10, 40)
        assert (it, conv) == (int(itb[0]), bool(convb[0]))
        assert np.array_equal(W, b.W(0)) and np.array_equal(H, b.H(0))
        assert np.array_equal(lab, b.classification()[0])


def test_queue_relaunches_after_idle_and_rejects_misfits(pkg, synth):
    V, _ = synth.expression_like(800, 60, 3, seed=9)
    with pkg.Serve(max_m=128, max_k=10, capacity=2, ctas=2, idle_ms=5) as q:
        t1 = q.submit(V, 3, seed=4, n_iters=30)
        q.wait(t1)
        r1 = q.fetch(t1)
        time.sleep(0.05)                              # the kernel has left (5 ms without work)
        t2 = q.submit(V, 3, seed=4, n_iters=30)
        q.wait(t2)
        r2 = q.fetch(t2)
        assert np.array_equal(r1[0], r2[0]) and np.array_equal(r1[1], r2[1]) and r1[3] == r2[3] == 30
        W, _ = synth.expression_like(800, 200, 3, seed=9)
        with pytest.raises(pkg.NMFError) as ei:
            q.submit(W, 3)                            # m > max_m
        assert ei.value.code == -1
        with pytest.raises(pkg.NMFError):
            q.submit(V, 11)                           # k > max_k
        a, b = q.submit(V, 3, n_iters=20), q.submit(V, 3, n_iters=20)
        with pytest.raises(pkg.NMFError) as ei:
            q.submit(V, 3)                            # both slots queued or unfetched
        assert ei.value.code == -5
        for t in (a, b):
            q.wait(t)
            q.fetch(t)
