"""Matrix files of NMF-mGPU from Python (ctypes over libnmfio.so, host/nmfio.c).

``load(path, fmt)`` / ``save(path, fmt, A, transpose=False, name=, headers=, labels=)``
with fmt in {"txt", "dat", "native"}: ASCII text, "non-native" binary
(little-endian float64 with signature 0xEDB10EA1) and native binary.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
FORMATS = {"txt": 0, "dat": 1, "native": 2}


class _Tags(C.Structure):
    _fields_ = [("name", C.c_char_p), ("headers", C.POINTER(C.c_char_p)), ("labels", C.POINTER(C.c_char_p))]


class _Matrix(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("rows", C.c_uint32), ("cols", C.c_uint32), ("tags", _Tags)]


_lib = None


def _L():
    global _lib
    if _lib is None:
        L = C.CDLL(os.path.join(_HERE, "libnmfio.so"))
        L.nmfio_load.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(_Matrix)]
        L.nmfio_save.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.c_size_t,
                                 C.c_int, C.POINTER(_Tags)]
        L.nmfio_free.argtypes = [C.POINTER(_Matrix)]
        L.nmfio_error.restype = C.c_char_p
        _lib = L
    return _lib


class MatrixIOError(RuntimeError):
    pass


def load(path: str, fmt: str = "txt", numeric_headers: bool = False, numeric_labels: bool = False):
    """Returns (V float32 rows x cols, name, headers, labels)."""
    L = _L()
    m = _Matrix()
    if L.nmfio_load(path.encode(), FORMATS[fmt], int(numeric_headers), int(numeric_labels), C.byref(m)) != 0:
        raise MatrixIOError(L.nmfio_error().decode())
    try:
        V = np.ctypeslib.as_array(m.data, shape=(m.rows, m.cols)).copy()
        name = m.tags.name.decode() if m.tags.name else None
        headers = [m.tags.headers[j].decode() for j in range(m.cols)] if m.tags.headers else None
        labels = [m.tags.labels[i].decode() for i in range(m.rows)] if m.tags.labels else None
    finally:
        L.nmfio_free(C.byref(m))
    return V, name, headers, labels


def save(path: str, fmt: str, A, transpose: bool = False, name=None, headers=None, labels=None):
    L = _L()
    A = np.ascontiguousarray(A, np.float32)
    rows, cols = A.shape
    tags = None
    keep = []
    if name is not None or headers is not None or labels is not None:
        def arr(lst):
            if lst is None:
                return None
            a = (C.c_char_p * len(lst))(*[s.encode() for s in lst])
            keep.append(a)
            return C.cast(a, C.POINTER(C.c_char_p))
        tags = _Tags(name.encode() if name is not None else None, arr(headers), arr(labels))
    rc = L.nmfio_save(path.encode(), FORMATS[fmt], A.ctypes.data_as(C.POINTER(C.c_float)), rows, cols, cols,
                      int(transpose), C.byref(tags) if tags is not None else None)
    if rc != 0:
        raise MatrixIOError(L.nmfio_error().decode())
