"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()``
(as the checker) and by the CPU-baseline leg of ``bench.py``.  The product
path (the CUDA engine behind include/nmfb200.h) never imports this module.

The functions restate the reference's single-GPU loop; each C function cites
the reference file:line it follows (oracle/nmf_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

_u32 = C.c_uint32
_sz = C.c_size_t
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_up = C.POINTER(C.c_uint32)


def build() -> str:
    """Compile liboracle.so (gcc + OpenMP) if it is missing or stale."""
    src = [os.path.join(_HERE, f) for f in ("nmf_oracle.c", "nmf_oracle_core.inc", "nmf_oracle.h")]
    if not os.path.exists(_LIB) or any(os.path.getmtime(s) > os.path.getmtime(_LIB) for s in src):
        subprocess.run(["make", "-C", _HERE, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        L.oracle_init_random.argtypes = [_u32, _u32, _u32, _u32, _fp, _sz, _fp, _sz]
        for p, t in (("f32", _fp), ("f64", _dp)):
            getattr(L, f"oracle_update_H_{p}").argtypes = [_u32, _u32, _u32, _fp, _sz, t, _sz, t, _sz]
            getattr(L, f"oracle_update_W_{p}").argtypes = [_u32, _u32, _u32, _fp, _sz, t, _sz, t, _sz]
            getattr(L, f"oracle_adjust_{p}").argtypes = [t, _u32, _u32, _sz]
            getattr(L, f"oracle_classify_{p}").argtypes = [t, _u32, _u32, _sz, _up]
            f = getattr(L, f"oracle_nmf_{p}")
            f.argtypes = [_u32, _u32, _u32, _fp, _sz, t, _sz, t, _sz, _u32, _u32, _u32, C.POINTER(C.c_int)]
            f.restype = _u32
        L.oracle_difference.argtypes = [_up, _up, _u32]
        L.oracle_difference.restype = C.c_uint64
        L.oracle_dot_VWH.argtypes = [_u32, _u32, _u32, _fp, _sz, _fp, _sz, _fp, _sz, _dp, _dp]
        L.oracle_kl_divergence.argtypes = [_u32, _u32, _u32, _fp, _sz, _fp, _sz, _fp, _sz]
        L.oracle_consensus.argtypes = [_up, _u32, _u32, _up]
        L.oracle_cophenetic_dist.argtypes = [_dp, _u32]
        L.oracle_cophenetic_dist.restype = C.c_double
        L.oracle_cophenetic.argtypes = [_up, _u32, _u32]
        L.oracle_cophenetic.restype = C.c_double
        L.oracle_kl_divergence.restype = C.c_double
        L.oracle_num_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a


def init_random(seed: int, n: int, m: int, k: int):
    """W (n x k) and H (m x k) exactly as the reference's CPU_RANDOM init."""
    W = np.empty((n, k), np.float32)
    H = np.empty((m, k), np.float32)
    lib().oracle_init_random(seed, n, m, k, _p(W, C.c_float), k, _p(H, C.c_float), k)
    return W, H


def _dtype(prec):
    return (np.float32, C.c_float, "f32") if prec == "f32" else (np.float64, C.c_double, "f64")


def update_H(V, W, H, prec="f32"):
    dt, ct, sfx = _dtype(prec)
    V = _f32(V)
    W = np.ascontiguousarray(W, dt)
    H = np.array(H, dt, copy=True, order="C")
    n, m = V.shape
    k = W.shape[1]
    getattr(lib(), f"oracle_update_H_{sfx}")(n, m, k, _p(V, C.c_float), m, _p(W, ct), k, _p(H, ct), k)
    return H


def update_W(V, W, H, prec="f32"):
    dt, ct, sfx = _dtype(prec)
    V = _f32(V)
    W = np.array(W, dt, copy=True, order="C")
    H = np.ascontiguousarray(H, dt)
    n, m = V.shape
    k = W.shape[1]
    getattr(lib(), f"oracle_update_W_{sfx}")(n, m, k, _p(V, C.c_float), m, _p(W, ct), k, _p(H, ct), k)
    return W


def adjust(A, prec="f32"):
    dt, ct, sfx = _dtype(prec)
    A = np.array(A, dt, copy=True, order="C")
    getattr(lib(), f"oracle_adjust_{sfx}")(_p(A, ct), A.shape[0], A.shape[1], A.shape[1])
    return A


def classify(H, prec="f32"):
    dt, ct, sfx = _dtype(prec)
    H = np.ascontiguousarray(H, dt)
    out = np.empty(H.shape[0], np.uint32)
    getattr(lib(), f"oracle_classify_{sfx}")(_p(H, ct), H.shape[0], H.shape[1], H.shape[1], _p(out, C.c_uint32))
    return out


def difference(cls, last) -> int:
    cls = np.ascontiguousarray(cls, np.uint32)
    last = np.ascontiguousarray(last, np.uint32)
    return int(lib().oracle_difference(_p(cls, C.c_uint32), _p(last, C.c_uint32), cls.shape[0]))


def nmf(V, W, H, n_iters=2000, niter_test_conv=10, stop_threshold=40, prec="f32"):
    """Run the reference loop from (W, H).  Returns (W, H, iterations, converged)."""
    dt, ct, sfx = _dtype(prec)
    V = _f32(V)
    W = np.array(W, dt, copy=True, order="C")
    H = np.array(H, dt, copy=True, order="C")
    n, m = V.shape
    k = W.shape[1]
    conv = C.c_int(0)
    it = getattr(lib(), f"oracle_nmf_{sfx}")(n, m, k, _p(V, C.c_float), m, _p(W, ct), k, _p(H, ct), k,
                                             n_iters, niter_test_conv, stop_threshold, C.byref(conv))
    return W, H, int(it), bool(conv.value)


def dot_VWH(V, W, H):
    V = _f32(V)
    W = _f32(W)
    H = _f32(H)
    n, m = V.shape
    k = W.shape[1]
    a, b = C.c_double(), C.c_double()
    lib().oracle_dot_VWH(n, m, k, _p(V, C.c_float), m, _p(W, C.c_float), k, _p(H, C.c_float), k,
                         C.byref(a), C.byref(b))
    return a.value, b.value


def kl_divergence(V, W, H) -> float:
    V = _f32(V)
    W = _f32(W)
    H = _f32(H)
    n, m = V.shape
    k = W.shape[1]
    return float(lib().oracle_kl_divergence(n, m, k, _p(V, C.c_float), m, _p(W, C.c_float), k,
                                            _p(H, C.c_float), k))


def consensus(labels) -> np.ndarray:
    """labels: nruns x m classification vectors -> m x m uint32 co-clustering counts."""
    labels = np.ascontiguousarray(labels, np.uint32)
    nruns, m = labels.shape
    out = np.empty((m, m), np.uint32)
    lib().oracle_consensus(_p(labels, C.c_uint32), nruns, m, _p(out, C.c_uint32))
    return out


def cophenetic(counts, nruns: int) -> float:
    counts = np.ascontiguousarray(counts, np.uint32)
    return float(lib().oracle_cophenetic(_p(counts, C.c_uint32), counts.shape[0], nruns))


def cophenetic_dist(D) -> float:
    D = np.ascontiguousarray(D, np.float64)
    return float(lib().oracle_cophenetic_dist(_p(D, C.c_double), D.shape[0]))


def num_threads() -> int:
    return int(lib().oracle_num_threads())
