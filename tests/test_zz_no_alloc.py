"""GPU test of nmfb_update_H_noalloc, the update_H entry point that allocates
nothing (for callers whose device memory is owned by someone else: a framework
with its own caching allocator, a plugin host that hands out every buffer, a
loop that cannot take cudaFree's device-wide synchronisation).

The caller -- this test -- owns V, W and H as torch device tensors; the entry
point only borrows them and keeps its scratch in a fixed device array.  Its
result must match the context-based nmfb_update_H within the single-update
tolerance of the other GPU tests (max|dH| / max|H| <= 1e-5), on two calls in a
row, the second starting from the first's output; the first call is also
checked against the FP64 oracle's update_H.  Free device memory
(cudaMemGetInfo) is the same before and after the two calls: once the
library's module is loaded (the warm-up call), the entry point allocates
nothing.  The file is named to be collected last, and passes alone in a
fresh process as well.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import maxnorm_rel

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _call(pkg, V, W, H, stream):
    n, m = V.shape
    k = W.shape[1]
    pkg.update_H_noalloc(V.data_ptr(), V.stride(0), W.data_ptr(), W.stride(0), H.data_ptr(), H.stride(0),
                         n, m, k, stream)


@pytest.mark.parametrize("shape", [(1000, 130, 5), (4000, 700, 16), (2500, 333, 33), (3000, 257, 64)])
def test_noalloc_matches_update_H_twice(pkg, synth, oracle, shape):
    import torch

    n, m, k = shape
    V, _ = synth.expression_like(n, m, k, seed=7 * n + m)
    with pkg.NMF(n, m, k) as e:
        e.set_V(V)
        e.init_random(11)
        W0, H0 = e.W, e.H
        e.update_H()
        H1_ref = e.H
        e.update_H()
        H2_ref = e.H

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    dV = torch.from_numpy(np.ascontiguousarray(V, np.float32)).to(dev)
    dW = torch.from_numpy(W0).to(dev)
    dH = torch.from_numpy(H0).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    # warm-up on a throwaway copy of H: loads the library's device module (and
    # with it the fixed scratch array) if no earlier call has
    dH_warm = dH.clone()
    _call(pkg, dV, dW, dH_warm, stream)
    torch.cuda.synchronize(dev)
    del dH_warm
    free0, _ = torch.cuda.mem_get_info(dev)

    _call(pkg, dV, dW, dH, stream)
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    H1 = dH.cpu().numpy()
    assert np.isfinite(H1).all()
    assert maxnorm_rel(H1, H1_ref) < TOL
    assert maxnorm_rel(H1, oracle.update_H(V, W0, H0, prec="f64")) < TOL

    _call(pkg, dV, dW, dH, stream)
    torch.cuda.synchronize(dev)
    free2, _ = torch.cuda.mem_get_info(dev)
    H2 = dH.cpu().numpy()
    assert maxnorm_rel(H2, H2_ref) < TOL
    assert free0 == free1 == free2, (free0, free1, free2)
    # the inputs the caller lent are untouched
    assert np.array_equal(dW.cpu().numpy(), W0)
    assert np.array_equal(dV.cpu().numpy(), np.ascontiguousarray(V, np.float32))


def test_noalloc_rejects_sizes_beyond_scratch(pkg):
    import torch

    dev = torch.device("cuda", 0)
    n, k = 2, 64
    m = pkg.NOALLOC_MAX_MK // k + 1          # m * k just above the limit
    dV = torch.ones((n, m), device=dev)
    dW = torch.ones((n, k), device=dev)
    dH = torch.ones((m, k), device=dev)
    with pytest.raises(pkg.NMFError) as ei:
        _call(pkg, dV, dW, dH, None)
    assert ei.value.code == -7 and "scratch" in str(ei.value)
    assert bool((dH == 1).all())             # nothing was queued
    with pytest.raises(pkg.NMFError) as ei:  # rank beyond 64
        pkg.update_H_noalloc(dV.data_ptr(), m, dW.data_ptr(), 65, dH.data_ptr(), 65, n, 100, 65, None)
    assert ei.value.code == -1
