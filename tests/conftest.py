"""Shared test plumbing.

Markers: ``gpu`` -- needs a B200 (sm_100); everything else runs on CPU.
The package directory is named ``bionmf-gpu_b200`` (not an identifier), so it
is imported here under the module name ``nmf_b200``.
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "bionmf-gpu_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def load_package():
    if "nmf_b200" in sys.modules:
        return sys.modules["nmf_b200"]
    spec = importlib.util.spec_from_file_location("nmf_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["nmf_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def synth():
    load_package()
    import nmf_b200.synth as s
    return s


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    o.build()
    return o


def golden_cases():
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_golden(name):
    """Load a reference-run fixture; regenerate V from its seeded generator
    when the fixture stores only the generator call and V's SHA-256."""
    import hashlib
    import json
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))
    if "V" not in g:
        load_package()
        import nmf_b200.synth as synth
        gen, kw = json.loads(str(g["generator"]))
        V, _ = getattr(synth, gen)(**kw)
        assert hashlib.sha256(np.ascontiguousarray(V, np.float32).tobytes()).hexdigest() == str(g["v_sha256"]), \
            f"{name}: regenerated V does not match the fixture's hash"
        g["V"] = V
    return g


def maxnorm_rel(a, b):
    """max |a - b| / max |b|: the relative error measure used for W and H."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())


def assert_labels_match(labels, H_ref, classify, margin=1e-3, min_checked=0.99):
    """Classification parity against a reference H: bit-exact on every sample
    whose two largest entries in H_ref differ by more than `margin` (relative);
    samples closer than that are ties at the factors' own tolerance and are
    not compared.  At least `min_checked` of the samples must be compared."""
    H_ref = np.asarray(H_ref, np.float64)
    srt = np.sort(H_ref, axis=1)
    top, second = srt[:, -1], srt[:, -2] if H_ref.shape[1] > 1 else np.zeros(H_ref.shape[0])
    sep = (top - second) > margin * np.abs(top)
    assert sep.mean() >= min_checked, f"only {sep.mean():.3f} of the samples are separated"
    ref = classify(H_ref)
    bad = np.nonzero((np.asarray(labels) != ref) & sep)[0]
    assert bad.size == 0, f"{bad.size} separated samples classified differently, e.g. {bad[:5]}"
