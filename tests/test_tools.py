"""CPU tests of the reference's two utilities as rebuilt here
(bionmf-gpu_b200/generate_matrix and file_converter, host/nmf_tools.c), and of
the matrix loader on the example matrix the reference ships.

generate_matrix must give, for a seed, the reference tool's matrix: entries
row by row, (float)random() / (float)RAND_MAX * max_value in single precision
from glibc's srandom(seed) (src/tools/generate_matrix.c:383-398) -- recomputed
here through ctypes calls of the same libc functions.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR, ROOT

GEN = os.path.join(PKG_DIR, "generate_matrix")
CONV = os.path.join(PKG_DIR, "file_converter")


@pytest.fixture(scope="module")
def mio(pkg):
    import nmf_b200.matrix_io as m
    return m


def _expected(seed, rows, cols, maxv):
    libc = ctypes.CDLL(None)
    libc.random.restype = ctypes.c_long
    libc.srandom(ctypes.c_uint(seed))
    num = np.array([libc.random() for _ in range(rows * cols)], dtype=np.float64).astype(np.float32)
    return ((num / np.float32(2147483647)) * np.float32(maxv)).reshape(rows, cols)


def _run(args, **env):
    e = dict(os.environ)
    e.update({k: str(v) for k, v in env.items()})
    return subprocess.run(args, capture_output=True, text=True, env=e, timeout=60)


@pytest.mark.parametrize("fmt,flag,ext", [("dat", ["-e", "0"], ".dat"), ("native", ["-e", "1"], ".native.dat"),
                                          ("txt", [], ".txt")])
def test_generate_matrix_matches_reference_formula(mio, tmp_path, fmt, flag, ext):
    out = str(tmp_path / f"g{ext}")
    r = _run([GEN, out, "7", "9"] + flag + ["3.5"], NMFB_SEED=5)
    assert r.returncode == 0, r.stderr
    V, name, hdr, lbl = mio.load(out, fmt)
    ref = _expected(5, 7, 9, 3.5)
    assert V.shape == (7, 9)
    if fmt == "txt":
        np.testing.assert_allclose(V, ref, rtol=1e-5)    # "%g": 6 significant digits
    else:
        assert np.array_equal(V, ref)
    assert name is None and hdr is None and lbl is None
    assert (V >= 0).all() and (V <= 3.5).all()


def test_generate_matrix_default_range_and_options_in_any_order(mio, tmp_path):
    out = str(tmp_path / "h.dat")
    # options before operands, and the solver's other letters ignored
    r = _run([GEN, "-e", "0", "-k", "4", out, "40", "3"], NMFB_SEED=9)
    assert r.returncode == 0, r.stderr
    V, *_ = mio.load(out, "dat")
    assert np.array_equal(V, _expected(9, 40, 3, 1.0))


@pytest.mark.parametrize("args", [["x.txt", "0", "5"], ["x.txt", "5"], ["x.txt", "4", "4", "-1"],
                                  ["x.txt", "4", "4", "1e39"], ["x.txt", "a", "4"], ["x.txt", "4", "4", "-e", "q"]])
def test_generate_matrix_rejects_bad_arguments(tmp_path, args):
    r = _run([GEN] + [str(tmp_path / a) if a == "x.txt" else a for a in args], NMFB_SEED=1)
    assert r.returncode == 1
    assert not os.path.exists(tmp_path / "x.txt")


def test_file_converter_round_trip_keeps_tags(mio, tmp_path):
    A = (np.random.default_rng(3).random((6, 4)) * 50 + 1).astype(np.float32)
    src = str(tmp_path / "m")
    hdr = [f"s{j}" for j in range(4)]
    lbl = [f"g{i}" for i in range(6)]
    mio.save(src, "txt", A, name="demo", headers=hdr, labels=lbl)
    # text -> non-native binary -> native binary -> text
    r = _run([CONV, src, "-e", "0"])
    assert r.returncode == 0, r.stderr
    r = _run([CONV, src + ".dat", "-b", "0", "-e", "1"])
    assert r.returncode == 0, r.stderr
    r = _run([CONV, src + ".dat.native.dat", "-b", "1"])
    assert r.returncode == 0, r.stderr
    for path, fmt in ((src + ".dat", "dat"), (src + ".dat.native.dat", "native"),
                      (src + ".dat.native.dat.txt", "txt")):
        B, name, h, l = mio.load(path, fmt)
        np.testing.assert_allclose(B, A, rtol=1e-5)
        assert (name, h, l) == ("demo", hdr, lbl), path


def test_file_converter_missing_input(tmp_path):
    r = _run([CONV, str(tmp_path / "absent.txt")])
    assert r.returncode == 1 and "absent" in r.stderr


def _reference_example():
    import importlib.util
    spec = importlib.util.spec_from_file_location("graft_entry", os.path.join(ROOT, "__graft_entry__.py"))
    g = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(g)
    ref = g.reference_path()
    p = os.path.join(ref, "test", "ALL_AML_data.txt") if ref else None
    return p if p and os.path.exists(p) else None


@pytest.mark.skipif(_reference_example() is None, reason="the reference's example matrix is not present")
def test_reference_example_matrix_loads_and_converts(mio, tmp_path):
    # test/ALL_AML_data.txt: a description token, 38 sample headers, then 5000
    # rows each led by a gene label (src/matrix_io/matrix_io.c:697, ASCII loader)
    path = _reference_example()
    V, name, hdr, lbl = mio.load(path, "txt")
    assert V.shape == (5000, 38)
    assert name == "Name"
    assert len(hdr) == 38 and hdr[0] == "ALL_19769_B-cell" and hdr[-1] == "AML_7"
    assert len(lbl) == 5000 and lbl[0] == "M12759_at"
    with open(path) as f:
        f.readline()
        first = f.readline().rstrip("\n").split("\t")
    assert np.array_equal(V[0], np.array(first[1:], dtype=np.float32))
    assert np.isfinite(V).all() and (V >= 0).all()
    # through the converter (as a user would before a binary run) and back
    local = str(tmp_path / "all_aml.txt")
    with open(path, "rb") as fi, open(local, "wb") as fo:
        fo.write(fi.read())
    r = _run([CONV, local, "-e", "0"])
    assert r.returncode == 0, r.stderr
    B, name2, hdr2, lbl2 = mio.load(local + ".dat", "dat")
    assert np.array_equal(B, V) and (name2, hdr2, lbl2) == (name, hdr, lbl)
