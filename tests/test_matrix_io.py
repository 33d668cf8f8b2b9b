"""CPU tests of the NMF-mGPU file formats (host/nmfio.c via nmf_b200.matrix_io)."""
from __future__ import annotations

import struct

import numpy as np
import pytest


@pytest.fixture(scope="module")
def mio(pkg):
    import nmf_b200.matrix_io as m
    return m


def _mat(rows=5, cols=4, seed=0):
    return (np.random.default_rng(seed).random((rows, cols)) * 100 + 0.5).astype(np.float32)


@pytest.mark.parametrize("fmt", ["txt", "dat", "native"])
def test_round_trip_untagged(mio, tmp_path, fmt):
    A = _mat()
    p = str(tmp_path / f"a.{fmt}")
    mio.save(p, fmt, A)
    B, name, hdr, lbl = mio.load(p, fmt)
    if fmt == "txt":
        assert np.allclose(A, B, rtol=1e-5)          # "%g" keeps 6 significant digits
    else:
        assert np.array_equal(A, B)
    assert name is None and hdr is None and lbl is None


@pytest.mark.parametrize("fmt", ["txt", "dat", "native"])
def test_round_trip_tagged(mio, tmp_path, fmt):
    A = _mat(3, 5)
    p = str(tmp_path / f"b.{fmt}")
    h = [f"sample {j}" for j in range(5)]
    l = [f"gene_{i}" for i in range(3)]
    mio.save(p, fmt, A, name="my matrix", headers=h, labels=l)
    B, name, hdr, lbl = mio.load(p, fmt)
    assert (name, hdr, lbl) == ("my matrix", h, l)
    assert np.allclose(A, B, rtol=1e-5)


def test_transposed_write(mio, tmp_path):
    A = _mat(6, 3)
    p = str(tmp_path / "t.dat")
    mio.save(p, "dat", A, transpose=True)
    B = mio.load(p, "dat")[0]
    assert np.array_equal(B, A.T)


def test_nonnative_binary_layout(mio, tmp_path):
    # u32 signature 0xEDB10EA1, u32 rows, u32 cols, float64 little-endian row-major.
    A = _mat(2, 3)
    p = str(tmp_path / "x.dat")
    mio.save(p, "dat", A)
    raw = open(p, "rb").read()
    assert raw[:12] == struct.pack("<III", 0xEDB10EA1, 2, 3)
    assert np.array_equal(np.frombuffer(raw[12:12 + 48], "<f8").reshape(2, 3), A.astype(np.float64))
    assert len(raw) == 12 + 48


def test_ascii_reference_layout(mio, tmp_path):
    # name + headers on line 1, labels in column 1 (the layout of the reference's example file).
    p = tmp_path / "e.txt"
    p.write_text("Name\tS1\tS2\tS3\ng1\t1\t2\t3\ng2\t4\t5\t6\r\n")
    V, name, hdr, lbl = mio.load(str(p), "txt")
    assert name == "Name" and hdr == ["S1", "S2", "S3"] and lbl == ["g1", "g2"]
    assert np.array_equal(V, np.array([[1, 2, 3], [4, 5, 6]], np.float32))


def test_ascii_space_separated_and_empty_entries(mio, tmp_path):
    p = tmp_path / "s.txt"
    p.write_text("1 2 3\n4  6\n")                    # empty entry reads as 0.0
    V = mio.load(str(p), "txt")[0]
    assert np.array_equal(V, np.array([[1, 2, 3], [4, 0, 6]], np.float32))


def test_numeric_labels_option(mio, tmp_path):
    p = tmp_path / "n.txt"
    p.write_text("10\t1\t2\n20\t3\t4\n")
    V, _, _, lbl = mio.load(str(p), "txt", numeric_labels=True)
    assert lbl == ["10", "20"] and np.array_equal(V, np.array([[1, 2], [3, 4]], np.float32))


@pytest.mark.parametrize("text,msg", [
    ("1\t-2\n3\t4\n", "negative"),
    ("1\t0\n3\t0\n", "empty"),
    ("1\t2\n0\t0\n", "empty"),
    ("1\t2\n", "not enough lines"),
    ("1\t2\n3\tx\n4\t5\n", "invalid numeric"),
    ("1\tnan\n3\t4\n", "invalid value"),
])
def test_validation_errors(mio, tmp_path, text, msg):
    p = tmp_path / "bad.txt"
    p.write_text(text)
    with pytest.raises(mio.MatrixIOError) as ei:
        mio.load(str(p), "txt")
    assert msg in str(ei.value)


def test_bad_signature(mio, tmp_path):
    p = tmp_path / "bad.dat"
    p.write_bytes(struct.pack("<III", 0x12345678, 2, 2) + b"\0" * 32)
    with pytest.raises(mio.MatrixIOError) as ei:
        mio.load(str(p), "dat")
    assert "signature" in str(ei.value)
