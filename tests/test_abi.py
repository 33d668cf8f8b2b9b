"""CPU tests of the C-ABI library: it loads without a GPU, exports every symbol
declared in include/nmfb200.h, and fails loudly (no CPU fallback) without a device."""
from __future__ import annotations

import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "nmfb200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nmfb_[A-Za-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("nmfb_create", "nmfb_update_H", "nmfb_update_W", "nmfb_get_classification", "nmfb_run",
              "nmfb_dot_product_VWH", "nmfb_init_random"):
        assert s in syms


def test_library_exports_every_declared_symbol(pkg):
    lib = ctypes.CDLL(pkg.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_no_cpu_fallback_without_device(pkg):
    if pkg.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.NMFError) as ei:
        pkg.NMF(100, 50, 4)
    assert ei.value.code in (-4, -2)


def test_argument_validation_before_device(pkg):
    # Rank checks happen before any device work (src/NMF_GPU.c:1121-1128).
    with pytest.raises(pkg.NMFError) as ei:
        pkg.NMF(10, 5, 6)
    assert ei.value.code == -1 and "factorization rank" in str(ei.value)
    with pytest.raises(pkg.NMFError) as ei:
        pkg.NMF(1, 5, 2)
    assert ei.value.code == -1


def test_context_bytes_accounts_for_each_arm(pkg):
    n, m, k = 20000, 1000, 16
    v = n * 1024 * 4
    fused = pkg.context_bytes(n, m, k, "fused")
    plain = pkg.context_bytes(n, m, k, "plain")
    bf16 = pkg.context_bytes(n, m, k, "bf16x3")
    streamed = pkg.context_bytes(n, m, k, "plain", stream_rows=1000)
    assert fused > v and plain - fused > v // 2 and bf16 > fused   # plain holds the n x m quotient
    assert streamed < plain - v               # neither V nor the n x m quotient on the device
    assert pkg.context_bytes(1, m, k) == 0    # invalid sizes
