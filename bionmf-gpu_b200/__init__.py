"""nmf-b200: B200-native KL-NMF engine (drop-in for NMF-mGPU's single-GPU path).

Python host binding over the C ABI in ``include/nmfb200.h`` (``libnmfb200.so``,
built in-tree for sm_100a).  It mirrors the reference's entry points
(src/NMF_routines.c, src/NMF_GPU.c):

====================  ==========================================
reference             here
====================  ==========================================
init_V + upload       ``NMF(V, k)`` / ``NMF.set_V``
init_random (CPU)     ``NMF.init_random(seed)``
update_H / update_W   ``NMF.update_H()`` / ``NMF.update_W()``
matrix_adjust         ``NMF.adjust()``
get_classification    ``NMF.classification()``
nmf()                 ``NMF.run(n_iters, niter_test_conv, stop_threshold)``
dot_product_VWH       ``NMF.dot_product_VWH()``
====================  ==========================================

There is no CPU fallback: if the shared library is missing or no sm_100
device is present, constructing an ``NMF`` raises ``NMFError``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnmfb200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "nmfb200.h")

ARM_FUSED = 0
ARM_PLAIN = 1
ARM_FUSED_TF32 = 2
ARM_BF16 = 3
ARM_SPLIT_BF16 = 4
ARM_BF16X3 = 5
ARMS = {"fused": ARM_FUSED, "plain": ARM_PLAIN, "fused_tf32": ARM_FUSED_TF32, "bf16": ARM_BF16,
        "split_bf16": ARM_SPLIT_BF16, "bf16x3": ARM_BF16X3}

NMFB_OK = 0
_ERRNAMES = {-1: "EINVAL", -2: "ECUDA", -3: "ENOMEM", -4: "ENODEV", -5: "ESTATE", -6: "ETIMEOUT", -7: "ETOOBIG"}


class NMFError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libnmfb200.so and declare every exported function."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise NMFError(-4, f"{path} is missing: build it with __graft_entry__.build() (no CPU fallback)")
    L = C.CDLL(path)
    vp = C.c_void_p
    u32, sz, i32 = C.c_uint32, C.c_size_t, C.c_int
    fp = C.POINTER(C.c_float)
    sig = {
        "nmfb_version": ([], C.c_char_p),
        "nmfb_device_count": ([], i32),
        "nmfb_create": ([C.POINTER(vp), i32, u32, u32, u32, i32], i32),
        "nmfb_create_streamed": ([C.POINTER(vp), i32, u32, u32, u32, u32], i32),
        "nmfb_context_bytes": ([i32, u32, u32, u32, i32, u32], C.c_uint64),
        "nmfb_release_cached": ([i32], i32),
        "nmfb_destroy": ([vp], i32),
        "nmfb_last_error": ([vp], C.c_char_p),
        "nmfb_set_arm": ([vp, i32], i32),
        "nmfb_set_V": ([vp, fp, sz], i32),
        "nmfb_set_V_device": ([vp, vp, sz], i32),
        "nmfb_init_random": ([vp, u32], i32),
        "nmfb_set_WH": ([vp, fp, sz, fp, sz], i32),
        "nmfb_update_H": ([vp], i32),
        "nmfb_update_W": ([vp], i32),
        "nmfb_adjust": ([vp], i32),
        "nmfb_get_classification": ([vp, C.POINTER(u32)], i32),
        "nmfb_run": ([vp, u32, u32, u32, C.POINTER(u32), C.POINTER(i32)], i32),
        "nmfb_get_W": ([vp, fp, sz], i32),
        "nmfb_get_H": ([vp, fp, sz], i32),
        "nmfb_dot_product_VWH": ([vp, C.POINTER(C.c_double), C.POINTER(C.c_double)], i32),
        "nmfb_kl_divergence": ([vp, C.POINTER(C.c_double)], i32),
        "nmfb_device_factors": ([vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(u32)], i32),
        "nmfb_device_V": ([vp, C.POINTER(vp), C.POINTER(sz)], i32),
        "nmfb_set_stream": ([vp, vp], i32),
        "nmfb_profile": ([vp, i32], i32),
        "nmfb_profile_read": ([vp, i32, C.POINTER(C.c_double), C.POINTER(u32)], i32),
        "nmfb_synchronize": ([vp], i32),
        "nmfb_launch_count": ([vp], C.c_uint64),
        "nmfb_set_wait_limit": ([vp, C.c_uint64], i32),
        "nmfb_set_sm_limit": ([vp, u32], i32),
        "nmfb_update_H_noalloc": ([vp, sz, vp, sz, vp, sz, u32, u32, u32, vp], i32),
        "nmfb_batch_create": ([C.POINTER(vp), i32, u32, u32, u32, C.POINTER(u32)], i32),
        "nmfb_batch_destroy": ([vp], i32),
        "nmfb_batch_last_error": ([vp], C.c_char_p),
        "nmfb_batch_set_V": ([vp, fp, sz], i32),
        "nmfb_batch_init_random": ([vp, C.POINTER(u32)], i32),
        "nmfb_batch_set_WH": ([vp, u32, fp, sz, fp, sz], i32),
        "nmfb_batch_set_tiles": ([vp, u32, u32, u32], i32),
        "nmfb_batch_set_cluster": ([vp, u32], i32),
        "nmfb_batch_get_cluster": ([vp, C.POINTER(u32)], i32),
        "nmfb_batch_run": ([vp, u32, u32, u32, C.POINTER(u32), C.POINTER(i32)], i32),
        "nmfb_batch_last_ms": ([vp, C.POINTER(C.c_double)], i32),
        "nmfb_batch_get_classification": ([vp, C.POINTER(u32)], i32),
        "nmfb_batch_get_WH": ([vp, u32, fp, sz, fp, sz], i32),
        "nmfb_batch_consensus": ([vp, u32, C.POINTER(u32), C.POINTER(u32), C.POINTER(C.c_double)], i32),
        "nmfb_serve_create": ([C.POINTER(vp), i32, u32, u32, u32, u32, u32], i32),
        "nmfb_serve_destroy": ([vp], i32),
        "nmfb_serve_last_error": ([vp], C.c_char_p),
        "nmfb_serve_request_bytes": ([u32, u32, u32], C.c_uint64),
        "nmfb_serve_submit": ([vp, fp, sz, u32, u32, u32, u32, u32, u32, u32, C.POINTER(u32)], i32),
        "nmfb_serve_poll": ([vp, u32, C.POINTER(i32)], i32),
        "nmfb_serve_wait": ([vp, u32, C.c_double], i32),
        "nmfb_serve_fetch": ([vp, u32, fp, sz, fp, sz, C.POINTER(u32), C.POINTER(u32), C.POINTER(i32)], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def context_bytes(n: int, m: int, k: int, arm: str | int = "fused", device: int = 0, stream_rows: int = 0) -> int:
    """Upper bound of the device memory an NMF(n, m, k, arm) context allocates."""
    a = ARMS[arm] if isinstance(arm, str) else int(arm)
    return int(load_library().nmfb_context_bytes(device, n, m, k, a, stream_rows))


def device_count() -> int:
    return int(load_library().nmfb_device_count())


NOALLOC_SCRATCH_BYTES = 16 * 1024 * 1024
NOALLOC_MAX_MK = 4186112


def update_H_noalloc(V: int, ldv: int, W: int, ldw: int, H: int, ldh: int, n: int, m: int, k: int,
                     stream: int | None = None) -> None:
    """update_H on caller-owned device buffers, allocating nothing.

    For callers that must not allocate device memory (a framework whose caching
    allocator owns the HBM, a plugin host that hands out every buffer, a loop
    that cannot take cudaFree's device-wide synchronisation).  ``V``, ``W`` and
    ``H`` are device addresses (e.g. ``tensor.data_ptr()``) on the current
    device: V is n x m, W is n x k, H is m x k and is updated in place.  The
    work is queued on ``stream`` (a raw cudaStream_t handle; None = default
    stream) and this returns before it finishes.  Limits: k <= 64 and
    m * k <= NOALLOC_MAX_MK (NMFError ETOOBIG beyond).  Calls share one fixed
    16 MiB device scratch array, so calls that overlap on the GPU race; the
    first call on a device looks up that array and belongs before any stream
    capture.
    """
    rc = load_library().nmfb_update_H_noalloc(V, ldv, W, ldw, H, ldh, n, m, k, stream or None)
    if rc != NMFB_OK:
        why = {-1: "invalid pointer, rank or leading dimension",
               -7: f"m*k = {m * k} exceeds the fixed scratch (k <= 64, m*k <= {NOALLOC_MAX_MK})"}
        raise NMFError(rc, why.get(rc, "CUDA error or no sm_100 device"))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class NMF:
    """One factorisation V (n x m) ~ W (n x k) H (k x m) on one B200.

    H is exchanged as the reference stores it: m rows of k factors.
    """

    def __init__(self, n: int, m: int, k: int, arm: str | int = "fused", device: int = 0,
                 stream_rows: int | None = None):
        """stream_rows: if given, V stays in host memory and is streamed in
        blocks of that many rows (0 = automatic) -- the blockwise mode for
        matrices larger than device memory (plain FP32 arm)."""
        L = load_library()
        self._L = L
        self.n, self.m, self.k = int(n), int(m), int(k)
        self.arm = ARMS[arm] if isinstance(arm, str) else int(arm)
        self.streamed = stream_rows is not None
        self._V_keep = None
        h = C.c_void_p()
        if self.streamed:
            self.arm = ARM_PLAIN
            rc = L.nmfb_create_streamed(C.byref(h), device, self.n, self.m, self.k, int(stream_rows))
        else:
            rc = L.nmfb_create(C.byref(h), device, self.n, self.m, self.k, self.arm)
        self._h = h
        if rc != NMFB_OK:
            msg = L.nmfb_last_error(h).decode() if h else "allocation failed"
            L.nmfb_destroy(h)
            self._h = None
            raise NMFError(rc, msg)

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc: int):
        if rc != NMFB_OK:
            raise NMFError(rc, self._L.nmfb_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.nmfb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- reference entry points -------------------------------------------
    def set_arm(self, arm):
        self.arm = ARMS[arm] if isinstance(arm, str) else int(arm)
        self._check(self._L.nmfb_set_arm(self._h, self.arm))

    def set_V(self, V: np.ndarray):
        V = np.ascontiguousarray(V, dtype=np.float32)
        assert V.shape == (self.n, self.m), (V.shape, self.n, self.m)
        self._check(self._L.nmfb_set_V(self._h, _fptr(V), self.m))
        if self.streamed:
            self._V_keep = V          # a streamed context reads this host array on every iteration

    def set_V_device(self, ptr: int, ld: int):
        self._check(self._L.nmfb_set_V_device(self._h, C.c_void_p(ptr), ld))

    def init_random(self, seed: int):
        self._check(self._L.nmfb_init_random(self._h, seed))

    def set_WH(self, W: np.ndarray, H: np.ndarray):
        W = np.ascontiguousarray(W, np.float32)
        H = np.ascontiguousarray(H, np.float32)
        assert W.shape == (self.n, self.k) and H.shape == (self.m, self.k)
        self._check(self._L.nmfb_set_WH(self._h, _fptr(W), self.k, _fptr(H), self.k))

    def update_H(self):
        self._check(self._L.nmfb_update_H(self._h))

    def update_W(self):
        self._check(self._L.nmfb_update_W(self._h))

    def adjust(self):
        self._check(self._L.nmfb_adjust(self._h))

    def classification(self) -> np.ndarray:
        out = np.empty(self.m, np.uint32)
        self._check(self._L.nmfb_get_classification(self._h, out.ctypes.data_as(C.POINTER(C.c_uint32))))
        return out

    def run(self, n_iters=2000, niter_test_conv=10, stop_threshold=40):
        it = C.c_uint32()
        conv = C.c_int()
        self._check(self._L.nmfb_run(self._h, n_iters, niter_test_conv, stop_threshold, C.byref(it), C.byref(conv)))
        return int(it.value), bool(conv.value)

    @property
    def W(self) -> np.ndarray:
        out = np.empty((self.n, self.k), np.float32)
        self._check(self._L.nmfb_get_W(self._h, _fptr(out), self.k))
        return out

    @property
    def H(self) -> np.ndarray:
        out = np.empty((self.m, self.k), np.float32)
        self._check(self._L.nmfb_get_H(self._h, _fptr(out), self.k))
        return out

    def dot_product_VWH(self):
        a, b = C.c_double(), C.c_double()
        self._check(self._L.nmfb_dot_product_VWH(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def distance(self) -> float:
        """The reference's final line: sqrt(||V-WH||^2) / sqrt(||V||^2)."""
        a, b = self.dot_product_VWH()
        return float(np.sqrt(b) / np.sqrt(a))

    def kl_divergence(self) -> float:
        d = C.c_double()
        self._check(self._L.nmfb_kl_divergence(self._h, C.byref(d)))
        return d.value

    def device_factors(self):
        w, h, ld = C.c_void_p(), C.c_void_p(), C.c_uint32()
        self._check(self._L.nmfb_device_factors(self._h, C.byref(w), C.byref(h), C.byref(ld)))
        return w.value, h.value, ld.value

    def device_V(self):
        v, ld = C.c_void_p(), C.c_size_t()
        self._check(self._L.nmfb_device_V(self._h, C.byref(v), C.byref(ld)))
        return v.value, ld.value

    def set_stream(self, stream_handle: int | None):
        """Queue work on an external CUDA stream (``torch.cuda.Stream().cuda_stream``)."""
        self._check(self._L.nmfb_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    def profile(self, enable: bool = True):
        self._check(self._L.nmfb_profile(self._h, 1 if enable else 0))

    def profile_read(self, cls: int):
        """(total_ms, launches) of kernel class cls: 0/1 = update_H/W main kernel, 2/3 = whole update."""
        ms, cnt = C.c_double(), C.c_uint32()
        self._check(self._L.nmfb_profile_read(self._h, cls, C.byref(ms), C.byref(cnt)))
        return ms.value, int(cnt.value)

    def synchronize(self):
        self._check(self._L.nmfb_synchronize(self._h))

    def launch_count(self) -> int:
        return int(self._L.nmfb_launch_count(self._h))

    def set_wait_limit(self, ns: int):
        """Limit of the fused kernels' bounded device waits in ns (0: default, 1 s)."""
        self._check(self._L.nmfb_set_wait_limit(self._h, int(ns)))

    def set_sm_limit(self, sms: int):
        """Size this context's launches for `sms` SMs (0: the whole device), so
        that several contexts' kernels can share the GPU side by side."""
        self._check(self._L.nmfb_set_sm_limit(self._h, int(sms)))


def _uptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


class Batch:
    """Many independent solves of one V (n x m): problem p has rank ranks[p].

    All problems run the reference's loop in one persistent launch
    (``run``); ``consensus(k)`` summarises the restarts of rank k.
    """

    def __init__(self, n: int, m: int, ranks, device: int = 0):
        self._L = load_library()
        self.n, self.m = int(n), int(m)
        self.ranks = np.ascontiguousarray(ranks, np.uint32)
        self.nprob = int(self.ranks.shape[0])
        self._h = C.c_void_p()
        rc = self._L.nmfb_batch_create(C.byref(self._h), device, self.n, self.m, self.nprob, _uptr(self.ranks))
        if rc != NMFB_OK:
            msg = self._L.nmfb_batch_last_error(self._h).decode() if self._h.value else "batch creation failed"
            self._L.nmfb_batch_destroy(self._h)
            self._h = C.c_void_p()
            raise NMFError(rc, msg)

    def _check(self, rc: int):
        if rc != NMFB_OK:
            raise NMFError(rc, self._L.nmfb_batch_last_error(self._h).decode())

    def close(self):
        if self._h is not None and self._h.value:
            self._L.nmfb_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_V(self, V: np.ndarray):
        V = np.ascontiguousarray(V, np.float32)
        assert V.shape == (self.n, self.m)
        self._check(self._L.nmfb_batch_set_V(self._h, _fptr(V), self.m))

    def init_random(self, seeds):
        seeds = np.ascontiguousarray(seeds, np.uint32)
        assert seeds.shape == (self.nprob,)
        self._check(self._L.nmfb_batch_init_random(self._h, _uptr(seeds)))

    def set_WH(self, p: int, W: np.ndarray, H: np.ndarray):
        W = np.ascontiguousarray(W, np.float32)
        H = np.ascontiguousarray(H, np.float32)
        k = int(self.ranks[p])
        assert W.shape == (self.n, k) and H.shape == (self.m, k)
        self._check(self._L.nmfb_batch_set_WH(self._h, p, _fptr(W), k, _fptr(H), k))

    def set_tiles(self, p: int, wt: int, jt: int):
        self._check(self._L.nmfb_batch_set_tiles(self._h, p, wt, jt))

    def set_cluster(self, ctas: int):
        """CTAs per problem (1, 2, 4, 8; 0 = automatic); see nmfb_batch_set_cluster."""
        self._check(self._L.nmfb_batch_set_cluster(self._h, ctas))

    @property
    def cluster(self) -> int:
        """CTAs per problem of the last run."""
        c = C.c_uint32()
        self._check(self._L.nmfb_batch_get_cluster(self._h, C.byref(c)))
        return int(c.value)

    def run(self, n_iters=2000, niter_test_conv=10, stop_threshold=40):
        """Returns (iterations, converged) arrays, one entry per problem."""
        it = np.zeros(self.nprob, np.uint32)
        cv = np.zeros(self.nprob, np.int32)
        self._check(self._L.nmfb_batch_run(self._h, n_iters, niter_test_conv, stop_threshold, _uptr(it),
                                           cv.ctypes.data_as(C.POINTER(C.c_int))))
        return it, cv.astype(bool)

    def last_ms(self) -> float:
        ms = C.c_double()
        self._check(self._L.nmfb_batch_last_ms(self._h, C.byref(ms)))
        return ms.value

    def classification(self) -> np.ndarray:
        out = np.empty((self.nprob, self.m), np.uint32)
        self._check(self._L.nmfb_batch_get_classification(self._h, _uptr(out)))
        return out

    def W(self, p: int) -> np.ndarray:
        k = int(self.ranks[p])
        out = np.empty((self.n, k), np.float32)
        self._check(self._L.nmfb_batch_get_WH(self._h, p, _fptr(out), k, None, k))
        return out

    def H(self, p: int) -> np.ndarray:
        k = int(self.ranks[p])
        out = np.empty((self.m, k), np.float32)
        self._check(self._L.nmfb_batch_get_WH(self._h, p, None, k, _fptr(out), k))
        return out

    def consensus(self, k: int, cophenetic: bool = True):
        """(counts m x m uint32, nruns, cophenetic correlation or None) of the rank-k problems."""
        counts = np.empty((self.m, self.m), np.uint32)
        nruns = C.c_uint32()
        coph = C.c_double()
        self._check(self._L.nmfb_batch_consensus(self._h, k, _uptr(counts), C.byref(nruns),
                                                 C.byref(coph) if cophenetic else None))
        return counts, int(nruns.value), (coph.value if cophenetic else None)


class Serve:
    """Device-side request queue feeding a persistent kernel (``nmfb_serve_*``).

    ``submit`` uploads a request (V: n x m float32, m <= max_m; rank k <= max_k)
    and returns a ticket at once; clusters of ``ctas`` CTAs take requests in
    submission order as they free up.  ``poll`` / ``wait`` / ``fetch`` collect
    a finished request's (W, H, labels, iterations, converged).
    """

    def __init__(self, max_m: int = 256, max_k: int = 20, capacity: int = 4096, ctas: int = 4,
                 idle_ms: int = 50, device: int = 0):
        self._L = load_library()
        self.max_m, self.max_k = int(max_m), int(max_k)
        self._shapes = {}
        self._h = C.c_void_p()
        rc = self._L.nmfb_serve_create(C.byref(self._h), device, self.max_m, self.max_k, capacity, ctas, idle_ms)
        if rc != NMFB_OK:
            msg = self._L.nmfb_serve_last_error(self._h).decode() if self._h.value else "server creation failed"
            self._L.nmfb_serve_destroy(self._h)
            self._h = C.c_void_p()
            raise NMFError(rc, msg)

    def _check(self, rc: int):
        if rc != NMFB_OK:
            raise NMFError(rc, self._L.nmfb_serve_last_error(self._h).decode())

    def close(self):
        if self._h is not None and self._h.value:
            self._L.nmfb_serve_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def request_bytes(n: int, m: int, k: int) -> int:
        return int(load_library().nmfb_serve_request_bytes(n, m, k))

    def fits(self, m: int, k: int) -> bool:
        return m <= self.max_m and 2 <= k <= self.max_k

    def submit(self, V: np.ndarray, k: int, seed: int = 1, n_iters: int = 2000, niter_test_conv: int = 10,
               stop_threshold: int = 40) -> int:
        V = np.ascontiguousarray(V, np.float32)
        n, m = V.shape
        t = C.c_uint32()
        self._check(self._L.nmfb_serve_submit(self._h, _fptr(V), m, n, m, k, seed, n_iters, niter_test_conv,
                                              stop_threshold, C.byref(t)))
        self._shapes[int(t.value)] = (n, m, int(k))
        return int(t.value)

    def poll(self, ticket: int) -> bool:
        d = C.c_int()
        self._check(self._L.nmfb_serve_poll(self._h, ticket, C.byref(d)))
        return bool(d.value)

    def wait(self, ticket: int, timeout: float = 600.0):
        self._check(self._L.nmfb_serve_wait(self._h, ticket, timeout))

    def fetch(self, ticket: int):
        """(W, H, labels, iterations, converged) of a finished request."""
        n, m, k = self._shapes.pop(ticket)
        W = np.empty((n, k), np.float32)
        H = np.empty((m, k), np.float32)
        lab = np.empty(m, np.uint32)
        it, conv = C.c_uint32(), C.c_int()
        rc = self._L.nmfb_serve_fetch(self._h, ticket, _fptr(W), k, _fptr(H), k, _uptr(lab), C.byref(it),
                                      C.byref(conv))
        if rc != NMFB_OK:
            self._shapes[ticket] = (n, m, k)
            self._check(rc)
        return W, H, lab, int(it.value), bool(conv.value)


def nmf_gpu(V: np.ndarray, k: int = 2, n_iters: int = 2000, niter_test_conv: int = 10, stop_threshold: int = 40,
            seed: int = 3, arm: str = "fused", device: int = 0):
    """One call equivalent of ``NMF_GPU <file> -k K -i I -j J -t T`` (CPU_RANDOM init).

    Returns (W, H, iterations, converged, distance)."""
    V = np.ascontiguousarray(V, np.float32)
    with NMF(V.shape[0], V.shape[1], k, arm=arm, device=device) as e:
        e.set_V(V)
        e.init_random(seed)
        it, conv = e.run(n_iters, niter_test_conv, stop_threshold)
        return e.W, e.H, it, conv, e.distance()
