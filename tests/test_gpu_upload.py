"""GPU tests of nmfb_set_V's upload paths.  From pageable memory the rows are
packed at the device pitch into the library's page-locked staging buffers (at
most 8 MB each, filled in turn: several chunks here) with zero padding
columns; from page-locked memory V goes in one pitched DMA; nmfb_set_V_device
copies device to device.  All three must leave the same device matrix: the
same factors bit for bit after a fixed iteration count, and sum(V^2) equal to
the host's."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_pageable_pinned_and_device_sources_agree(pkg, synth):
    import torch

    n, m, k = 5000, 700, 8          # device pitch 704 floats: a 14 MB V, two staging chunks
    V, _ = synth.expression_like(n, m, 4, seed=31)
    # leave non-zero data in every column of the shared staging buffers first
    with pkg.NMF(n, 704, k) as e0:
        e0.set_V(np.full((n, 704), 3.0, np.float32))
    results = {}
    for path in ("pageable", "pinned", "device"):
        with pkg.NMF(n, m, k) as e:
            if path == "pageable":
                e.set_V(V)
            elif path == "pinned":
                Vp = torch.from_numpy(V).pin_memory()
                e._check(e._L.nmfb_set_V(e._h, pkg._fptr(Vp.numpy()), m))
            else:
                Vd = torch.from_numpy(V).cuda()
                torch.cuda.synchronize()
                e.set_V_device(Vd.data_ptr(), m)
                e.synchronize()
            e.init_random(5)
            e.run(20, 10, 1000)
            dot_v, _ = e.dot_product_VWH()
            results[path] = (e.W, e.H, dot_v)
    W0, H0, d0 = results["pageable"]
    for path in ("pinned", "device"):
        W, H, d = results[path]
        assert np.array_equal(W, W0) and np.array_equal(H, H0), path
        assert d == d0, path
    assert d0 == pytest.approx(float((V.astype(np.float64) ** 2).sum()), rel=1e-6)
