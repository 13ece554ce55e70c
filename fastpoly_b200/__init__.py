"""fastpoly_b200 - the fastpoly NTT hot path on one B200.

Python mirror of the reference's polynomial API (``fpx::poly::conv / inv / log /
exp / sqrt / pow / divmod / div / mod`` and ``NttPlan<M>::forward / inverse``;
include/fastpoly/poly.hpp, detail/poly/*.hpp, ntt.hpp) over the C ABI in
``include/fpx_b200.h``, implemented by the in-tree CUDA library
``fastpoly_b200/libfpx_b200.so``.  There is no CPU fallback: if the library is
missing or no GPU is present, constructing a ``Context`` raises.

Arrays are canonical residues (numpy ``uint32``) unless ``repr=MONTGOMERY``
selects the reference's Montgomery limbs.  Errors mirror the reference's
exceptions: ``DomainError`` (fpx::poly::domain_error), ``NttSizeError``
(fpx::ntt_size_error), ``LengthError`` (std::length_error).
"""
from __future__ import annotations

import ctypes as C
import mmap
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfpx_b200.so")

OK, EDOMAIN, ESIZE, ELENGTH, ENOMEM, ETIMEDOUT, ECUDA, EINVAL, EUNSUPPORTED, EPENDING = range(10)
CANONICAL, MONTGOMERY = 0, 1
SIZE_MAX = 2**64 - 1


class FpxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[fpx status {code}] {msg}")
        self.code = code


class DomainError(FpxError):
    """fpx::poly::domain_error (include/fastpoly/detail/poly/base.hpp:26-30)."""


class NttSizeError(FpxError):
    """fpx::ntt_size_error (include/fastpoly/ntt.hpp:59-70)."""


class LengthError(FpxError):
    """std::length_error from conv (convolution.hpp:20-21)."""


_ERRORS = {EDOMAIN: DomainError, ESIZE: NttSizeError, ELENGTH: LengthError}

_u32p = C.POINTER(C.c_uint32)
_szp = C.POINTER(C.c_size_t)
_lib = None


def load_library(path: str = LIB_PATH):
    """Loads the CUDA library (fails loudly when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"fastpoly_b200 CUDA library not built: {path} (run python -m fastpoly_b200.build)")
    L = C.CDLL(path)
    vp, u32, sz, u64, i32 = C.c_void_p, C.c_uint32, C.c_size_t, C.c_uint64, C.c_int
    L.fpx_ctx_create.argtypes = [i32, sz, C.POINTER(vp)]
    L.fpx_ctx_destroy.argtypes = [vp]
    L.fpx_ctx_set_stream.argtypes = [vp, vp]
    L.fpx_ctx_stream.argtypes = [vp]
    L.fpx_ctx_stream.restype = vp
    L.fpx_ctx_synchronize.argtypes = [vp]
    L.fpx_last_error_message.argtypes = [vp]
    L.fpx_last_error_message.restype = C.c_char_p
    L.fpx_pool_stats.argtypes = [vp, vp]
    L.fpx_release_pool.argtypes = [vp]
    L.fpx_host_alloc.argtypes = [sz, C.POINTER(vp)]
    L.fpx_host_free.argtypes = [vp]
    L.fpx_ctx_set_crt_block.argtypes = [vp, sz]
    L.fpx_ntt_max_log.argtypes = [u32]
    L.fpx_profile.argtypes = [vp, i32]
    L.fpx_profile_report.argtypes = [vp, C.c_char_p, sz, _szp]
    L.fpx_launch_count.argtypes = [vp]
    L.fpx_launch_count.restype = u64
    for f in ("fpx_ntt_forward", "fpx_ntt_inverse"):
        getattr(L, f).argtypes = [vp, u32, _u32p, u32, i32]
    for f in ("fpx_ntt_forward_device", "fpx_ntt_inverse_device"):
        getattr(L, f).argtypes = [vp, u32, vp, u32]
    L.fpx_conv.argtypes = [vp, u32, _u32p, sz, _u32p, sz, sz, _u32p, _szp, i32]
    L.fpx_conv_device.argtypes = [vp, u32, vp, sz, vp, sz, sz, vp, _szp]
    for f in ("fpx_inv", "fpx_log", "fpx_exp", "fpx_sqrt"):
        getattr(L, f).argtypes = [vp, u32, _u32p, sz, sz, _u32p, i32]
    for f in ("fpx_inv_device", "fpx_log_device", "fpx_exp_device", "fpx_sqrt_device"):
        getattr(L, f).argtypes = [vp, u32, vp, sz, sz, vp]
    L.fpx_pow.argtypes = [vp, u32, _u32p, sz, u64, sz, _u32p, i32]
    L.fpx_pow_device.argtypes = [vp, u32, vp, sz, u64, sz, vp]
    L.fpx_divmod.argtypes = [vp, u32, _u32p, sz, _u32p, sz, _u32p, _szp, _u32p, _szp, i32]
    L.fpx_div.argtypes = [vp, u32, _u32p, sz, _u32p, sz, _u32p, _szp, i32]
    L.fpx_mod.argtypes = [vp, u32, _u32p, sz, _u32p, sz, _u32p, _szp, i32]
    L.fpx_measure_imad_rate.argtypes = [i32, C.POINTER(C.c_double)]
    L.fpx_measure_butterfly_rate.argtypes = [i32, C.POINTER(C.c_double)]
    L.fpx_batch_submit.argtypes = [vp, vp, sz]
    L.fpx_batch_wait.argtypes = [vp]
    L.fpx_batch_run.argtypes = [vp, vp, sz, i32]
    L.fpx_serve_start.argtypes = [i32, vp, C.POINTER(vp)]
    L.fpx_serve_submit.argtypes = [vp, vp, C.POINTER(u64)]
    L.fpx_serve_poll.argtypes = [vp, u64, i32, C.POINTER(u64)]
    L.fpx_serve_stats_get.argtypes = [vp, vp]
    L.fpx_serve_stop.argtypes = [vp]
    L.fpx_serve_plan_bytes.argtypes = [vp]
    L.fpx_serve_plan_bytes.restype = sz
    L.fpx_col_shape_candidates.argtypes = [vp, i32, i32, vp, i32, C.POINTER(i32)]
    L.fpx_col_shape_get.argtypes = [vp, i32, i32, vp]
    L.fpx_col_shape_set.argtypes = [vp, i32, i32, vp]
    _lib = L
    return L


OP_CONV, OP_INV, OP_LOG, OP_EXP, OP_SQRT, OP_POW, OP_DIVMOD = range(7)
_OPS = {"conv": OP_CONV, "inv": OP_INV, "log": OP_LOG, "exp": OP_EXP, "sqrt": OP_SQRT, "pow": OP_POW,
        "divmod": OP_DIVMOD}


class ColShape(C.Structure):
    """struct fpx_col_shape (include/fpx_b200.h): tile shape of a column pass."""
    _fields_ = [("lw1", C.c_int), ("lw2", C.c_int), ("split", C.c_int)]

    def astuple(self):
        return (self.lw1, self.lw2, self.split)


COL_FWD1, COL_FWD2, COL_INV = 0, 1, 2


class Job(C.Structure):
    """struct fpx_job (include/fpx_b200.h): one operation of a batch."""
    _fields_ = [("op", C.c_int), ("p", C.c_uint32), ("a", C.c_void_p), ("la", C.c_size_t), ("b", C.c_void_p),
                ("lb", C.c_size_t), ("k", C.c_uint64), ("n", C.c_size_t), ("out", C.c_void_p),
                ("out2", C.c_void_p), ("out_len", C.c_size_t), ("out2_len", C.c_size_t), ("status", C.c_int)]


# The same layout as a numpy record: a batch's job array is filled column-wise.
_JOB_DTYPE = np.dtype({"names": [n for n, _ in Job._fields_],
                       "formats": [np.int32, np.uint32, np.uint64, np.uint64, np.uint64, np.uint64, np.uint64,
                                   np.uint64, np.uint64, np.uint64, np.uint64, np.uint64, np.int32],
                       "offsets": [getattr(Job, n).offset for n, _ in Job._fields_],
                       "itemsize": C.sizeof(Job)})


def _host_u32(x, keep: list):
    """x as a C-contiguous uint32 array (converted only when it is not one)."""
    if isinstance(x, np.ndarray) and x.dtype == np.uint32 and x.flags.c_contiguous:
        return x
    a = _arr(x)
    keep.append(a)
    return a


class ServeConfig(C.Structure):
    """struct fpx_serve_config."""
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("max_batch_jobs", C.c_size_t), ("workers", C.c_int),
                ("repr", C.c_int)]


class ServeStats(C.Structure):
    """struct fpx_serve_stats."""
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("batches", C.c_uint64),
                ("max_batch_jobs_seen", C.c_uint64), ("max_batch_bytes_seen", C.c_uint64),
                ("oversize_requests", C.c_uint64), ("max_in_flight_bytes", C.c_uint64),
                ("device_pool_bytes", C.c_uint64), ("device_allocations", C.c_uint64),
                ("pool_flushes", C.c_uint64), ("device_alloc_ns", C.c_uint64),
                ("device_alloc_ns_max", C.c_uint64), ("host_allocs", C.c_uint64),
                ("host_alloc_ns", C.c_uint64), ("host_alloc_ns_max", C.c_uint64)]


def make_job(spec, keep: list) -> tuple:
    """Fills a Job from a tuple spec (see Context.batch) with host buffers; returns
    (job, out, out2).  Arrays the job points into are appended to `keep`."""
    op, p = _OPS[spec[0]], int(spec[1])
    a = _arr(spec[2])
    b = np.zeros(0, np.uint32)
    k, n = 0, 0
    o2 = None
    if op == OP_CONV:
        b = _arr(spec[3])
        n = SIZE_MAX if len(spec) < 5 or spec[4] is None else int(spec[4])
        cap = min(a.size, n) + min(b.size, n) - 1 if a.size and b.size and n else 0
        o1 = np.empty(max(min(cap, n), 1), np.uint32)
    elif op == OP_POW:
        k, n = int(spec[3]), int(spec[4])
        o1 = np.empty(max(n, 1), np.uint32)
    elif op == OP_DIVMOD:
        b = _arr(spec[3])
        o1, o2 = np.empty(max(a.size, 1), np.uint32), np.empty(max(b.size, 1), np.uint32)
    else:
        n = int(spec[3])
        o1 = np.empty(max(n, 1), np.uint32)
    j = Job()
    j.op, j.p, j.la, j.lb, j.k, j.n = op, p, a.size, b.size, k, n
    j.a = a.ctypes.data if a.size else None
    j.b = b.ctypes.data if b.size else None
    j.out = o1.ctypes.data
    j.out2 = o2.ctypes.data if o2 is not None else None
    keep += [a, b, o1, o2]
    return j, o1, o2


def job_result(j, o1, o2, what=""):
    """The result of a finished Job: the array ((q, r) for divmod) or the exception the single call raises."""
    if j.status != OK:
        return _ERRORS.get(j.status, FpxError)(j.status, what)
    if j.op == OP_DIVMOD:
        return o1[: j.out_len], o2[: j.out2_len]
    return o1[: j.out_len]


class Server:
    """The request loop (fpx_serve_*): HBM-budget admission, continuous micro-batching."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, max_batch_jobs: int = 0, workers: int = 0,
                 repr: int = CANONICAL):
        self._L = load_library()
        cfg = ServeConfig(hbm_budget_bytes, max_batch_jobs, workers, repr)
        h = C.c_void_p()
        rc = self._L.fpx_serve_start(device, C.byref(cfg), C.byref(h))
        if rc != OK:
            raise FpxError(rc, "fpx_serve_start failed")
        self._h = h
        self._live = {}

    def submit(self, spec) -> int:
        """Queues one request (tuple spec as in Context.batch); returns its ticket."""
        keep = []
        j, o1, o2 = make_job(spec, keep)
        t = C.c_uint64(0)
        rc = self._L.fpx_serve_submit(self._h, C.byref(j), C.byref(t))
        if rc != OK:
            raise FpxError(rc, "fpx_serve_submit failed")
        self._live[t.value] = (j, o1, o2, keep, spec[0])
        return t.value

    def poll(self, ticket: int, wait: bool = True):
        """None while pending; else (result, latency_seconds)."""
        lat = C.c_uint64(0)
        rc = self._L.fpx_serve_poll(self._h, ticket, 1 if wait else 0, C.byref(lat))
        if rc == EPENDING:
            return None
        j, o1, o2, keep, op = self._live.pop(ticket)
        return job_result(j, o1, o2, f"served {op}"), lat.value * 1e-9

    def stats(self) -> dict:
        st = ServeStats()
        self._L.fpx_serve_stats_get(self._h, C.byref(st))
        return {k: getattr(st, k) for k, _ in ServeStats._fields_}

    def plan_bytes(self, spec) -> int:
        keep = []
        j, _, _ = make_job(spec, keep)
        return int(self._L.fpx_serve_plan_bytes(C.byref(j)))

    def stop(self):
        if getattr(self, "_h", None):
            self._L.fpx_serve_stop(self._h)
            self._h = None

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


class PoolStats(C.Structure):
    _fields_ = [("cached_bytes", C.c_size_t), ("cached_blocks", C.c_size_t), ("in_use_bytes", C.c_size_t),
                ("system_allocations", C.c_size_t), ("cache_hits", C.c_size_t), ("limit_bytes", C.c_size_t)]


def _arr(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


_JOBS_EXT = None


def _jobs_ext():
    """The C helper that fills batch job records (fastpoly_b200/_fpx_jobs, built
    with the library)."""
    global _JOBS_EXT
    if _JOBS_EXT is None:
        try:
            from . import _fpx_jobs
        except ImportError as e:
            raise ImportError("fastpoly_b200/_fpx_jobs is not built: run python -m fastpoly_b200.build") from e
        _JOBS_EXT = _fpx_jobs
    return _JOBS_EXT


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_u32p) if a.size else None


def _dptr(t) -> int:
    """Device pointer of a torch tensor (or an int address)."""
    return t if isinstance(t, int) else t.data_ptr()


# Batch output buffers of at least this many words are reused across calls.
_OUT_KEEP_WORDS = 1 << 20


def _pinned_words(lib, words: int):
    """A uint32 array in page-locked host memory (fpx_host_alloc), freed when the
    array and every view of it are gone; None if none can be had."""
    import weakref
    ptr = C.c_void_p()
    if lib.fpx_host_alloc(words * 4, C.byref(ptr)) != OK or not ptr.value:
        return None
    raw = (C.c_char * (words * 4)).from_address(ptr.value)
    arr = np.frombuffer(raw, np.uint32)
    weakref.finalize(arr, lib.fpx_host_free, ptr.value)
    return arr


class Context:
    """One device, one stream, one device-memory pool and plan cache (fpx_ctx)."""

    def __init__(self, device: int = 0, pool_limit_bytes: int = 0):
        self._L = load_library()
        h = C.c_void_p()
        rc = self._L.fpx_ctx_create(device, pool_limit_bytes, C.byref(h))
        if rc != OK:
            raise FpxError(rc, f"fpx_ctx_create(device={device}) failed")
        self._h = h
        self.device = device
        self._outbufs = []  # batch output buffers kept for reuse (at most two)

    # -- plumbing --------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._L.fpx_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != OK:
            msg = (self._L.fpx_last_error_message(self._h) or b"").decode()
            raise _ERRORS.get(rc, FpxError)(rc, f"{what}: {msg}")

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream=None):
        """Queue device-pointer work on a cudaStream_t (int handle or torch stream)."""
        s = getattr(stream, "cuda_stream", stream)
        self._check(self._L.fpx_ctx_set_stream(self._h, s), "set_stream")

    @property
    def stream(self) -> int:
        return self._L.fpx_ctx_stream(self._h) or 0

    def synchronize(self):
        self._check(self._L.fpx_ctx_synchronize(self._h), "synchronize")

    def pool_stats(self) -> dict:
        st = PoolStats()
        self._check(self._L.fpx_pool_stats(self._h, C.byref(st)), "pool_stats")
        return {k: getattr(st, k) for k, _ in PoolStats._fields_}

    def profile(self, enable: bool = True):
        """Start (and clear) or stop per-kernel CUDA-event timing on the context's stream."""
        self._check(self._L.fpx_profile(self._h, 1 if enable else 0), "profile")

    def profile_report(self) -> dict:
        """{kernel: (launches, total_ms)} for the launches recorded since profile(True)."""
        import json
        need = C.c_size_t(0)
        self._check(self._L.fpx_profile_report(self._h, None, 0, C.byref(need)), "profile_report")
        buf = C.create_string_buffer(need.value + 16)
        self._check(self._L.fpx_profile_report(self._h, buf, len(buf), C.byref(need)), "profile_report")
        return {k: (int(v[0]), float(v[1])) for k, v in json.loads(buf.value.decode()).items()}

    def launch_count(self) -> int:
        return int(self._L.fpx_launch_count(self._h))

    def release_pool(self):
        self._check(self._L.fpx_release_pool(self._h), "release_pool")

    def set_crt_block(self, terms: int = 0):
        """Terms per block of the block-pair CRT product (0: the default 2^23)."""
        self._check(self._L.fpx_ctx_set_crt_block(self._h, terms), "set_crt_block")

    # -- column-pass tile shapes (the tuner's choice per transform size) ----------
    def col_shape_candidates(self, log_n: int, kind: int) -> list:
        """Compiled (lw1, lw2, split) shapes of one column pass, the default first."""
        arr = (ColShape * 8)()
        cnt = C.c_int(0)
        self._check(self._L.fpx_col_shape_candidates(self._h, log_n, kind, arr, 8, C.byref(cnt)),
                    "col_shape_candidates")
        return [arr[i].astuple() for i in range(min(cnt.value, 8))]

    def col_shape(self, log_n: int, kind: int) -> tuple:
        """The shape in use (tuned on first use of the size)."""
        sh = ColShape()
        self._check(self._L.fpx_col_shape_get(self._h, log_n, kind, C.byref(sh)), "col_shape_get")
        return sh.astuple()

    def set_col_shape(self, log_n: int, kind: int, shape) -> None:
        sh = ColShape(*shape)
        self._check(self._L.fpx_col_shape_set(self._h, log_n, kind, C.byref(sh)), "col_shape_set")

    # -- transforms (NttPlan<M>::forward / inverse) ------------------------------
    def ntt_forward(self, p: int, x, repr: int = CANONICAL) -> np.ndarray:
        x = _arr(x).copy()
        self._check(self._L.fpx_ntt_forward(self._h, p, _ptr(x), x.size, repr), "ntt_forward")
        return x

    def ntt_inverse(self, p: int, x, repr: int = CANONICAL) -> np.ndarray:
        x = _arr(x).copy()
        self._check(self._L.fpx_ntt_inverse(self._h, p, _ptr(x), x.size, repr), "ntt_inverse")
        return x

    def ntt_forward_device(self, p: int, d_x, n: int):
        self._check(self._L.fpx_ntt_forward_device(self._h, p, _dptr(d_x), n), "ntt_forward_device")

    def ntt_inverse_device(self, p: int, d_x, n: int):
        self._check(self._L.fpx_ntt_inverse_device(self._h, p, _dptr(d_x), n), "ntt_inverse_device")

    # -- fpx::poly ---------------------------------------------------------------
    def conv(self, p: int, a, b, n: int | None = None, repr: int = CANONICAL, out: np.ndarray | None = None):
        """fpx::poly::conv(a, b[, n]); `out` may be a preallocated (e.g. pinned) uint32 array."""
        a, b = _arr(a), _arr(b)
        lim = SIZE_MAX if n is None else n
        cap = min(a.size + b.size - 1, lim) if a.size and b.size and lim else 0
        if out is None:
            out = np.empty(max(cap, 1), dtype=np.uint32)
        elif out.dtype != np.uint32 or not out.flags.c_contiguous or out.size < cap:
            raise ValueError("out must be a contiguous uint32 array with room for the product")
        got = C.c_size_t(0)
        pb = _ptr(a) if b is a else _ptr(b)
        self._check(self._L.fpx_conv(self._h, p, _ptr(a), a.size, pb, b.size, C.c_size_t(lim), _ptr(out),
                                     C.byref(got), repr), "conv")
        return out[: got.value]

    def conv_device(self, p: int, d_a, la: int, d_b, lb: int, n: int | None, d_out) -> int:
        got = C.c_size_t(0)
        lim = SIZE_MAX if n is None else n
        self._check(self._L.fpx_conv_device(self._h, p, _dptr(d_a), la, _dptr(d_b), lb, C.c_size_t(lim),
                                            _dptr(d_out), C.byref(got)), "conv_device")
        return got.value

    def _series(self, fn, what, p, a, n, repr):
        a = _arr(a)
        out = np.empty(max(n, 1), dtype=np.uint32)
        self._check(fn(self._h, p, _ptr(a), a.size, n, _ptr(out), repr), what)
        return out[:n]

    def inv(self, p, a, n, repr=CANONICAL):
        return self._series(self._L.fpx_inv, "inv", p, a, n, repr)

    def log(self, p, a, n, repr=CANONICAL):
        return self._series(self._L.fpx_log, "log", p, a, n, repr)

    def exp(self, p, a, n, repr=CANONICAL):
        return self._series(self._L.fpx_exp, "exp", p, a, n, repr)

    def sqrt(self, p, a, n, repr=CANONICAL):
        return self._series(self._L.fpx_sqrt, "sqrt", p, a, n, repr)

    def pow(self, p, a, k, n, repr=CANONICAL):
        a = _arr(a)
        out = np.empty(max(n, 1), dtype=np.uint32)
        self._check(self._L.fpx_pow(self._h, p, _ptr(a), a.size, C.c_uint64(k), n, _ptr(out), repr), "pow")
        return out[:n]

    def _series_dev(self, fn, what, p, d_a, la, n, d_out):
        self._check(fn(self._h, p, _dptr(d_a), la, n, _dptr(d_out)), what)

    def inv_device(self, p, d_a, la, n, d_out):
        self._series_dev(self._L.fpx_inv_device, "inv_device", p, d_a, la, n, d_out)

    def log_device(self, p, d_a, la, n, d_out):
        self._series_dev(self._L.fpx_log_device, "log_device", p, d_a, la, n, d_out)

    def exp_device(self, p, d_a, la, n, d_out):
        self._series_dev(self._L.fpx_exp_device, "exp_device", p, d_a, la, n, d_out)

    def sqrt_device(self, p, d_a, la, n, d_out):
        self._series_dev(self._L.fpx_sqrt_device, "sqrt_device", p, d_a, la, n, d_out)

    def pow_device(self, p, d_a, la, k, n, d_out):
        self._check(self._L.fpx_pow_device(self._h, p, _dptr(d_a), la, C.c_uint64(k), n, _dptr(d_out)), "pow_device")

    def divmod(self, p, a, b, repr=CANONICAL):
        a, b = _arr(a), _arr(b)
        q = np.empty(max(a.size, 1), dtype=np.uint32)
        r = np.empty(max(b.size, 1), dtype=np.uint32)
        lq, lr = C.c_size_t(0), C.c_size_t(0)
        self._check(self._L.fpx_divmod(self._h, p, _ptr(a), a.size, _ptr(b), b.size, _ptr(q), C.byref(lq), _ptr(r),
                                       C.byref(lr), repr), "divmod")
        return q[: lq.value], r[: lr.value]

    def div(self, p, a, b, repr=CANONICAL):
        a, b = _arr(a), _arr(b)
        q = np.empty(max(a.size, 1), dtype=np.uint32)
        lq = C.c_size_t(0)
        self._check(self._L.fpx_div(self._h, p, _ptr(a), a.size, _ptr(b), b.size, _ptr(q), C.byref(lq), repr), "div")
        return q[: lq.value]

    def mod(self, p, a, b, repr=CANONICAL):
        a, b = _arr(a), _arr(b)
        r = np.empty(max(b.size, 1), dtype=np.uint32)
        lr = C.c_size_t(0)
        self._check(self._L.fpx_mod(self._h, p, _ptr(a), a.size, _ptr(b), b.size, _ptr(r), C.byref(lr), repr), "mod")
        return r[: lr.value]


    # -- batches -------------------------------------------------------------------
    def batch(self, jobs, repr: int = CANONICAL) -> list:
        """Runs many operations in one call (fpx_batch_run, host buffers).

        Each job is a tuple: ("conv", p, a, b[, n]), ("inv" | "log" | "exp" | "sqrt", p, a, n),
        ("pow", p, a, k, n) or ("divmod", p, a, b).  Returns one entry per job: the
        result array ((q, r) for divmod; views into one output buffer), or the
        exception the single-job call would raise for that job (not raised).
        Large output buffers (page-locked, so results arrive by DMA in place) are
        kept by the context and used again by a later call only once no result
        of the call that had them is referenced: keep a result (or a copy), not
        a raw pointer into it.
        """
        m = len(jobs)
        arr = np.zeros(max(m, 1), dtype=_JOB_DTYPE)
        caps = np.empty(2 * max(m, 1), np.int64)
        keep = _jobs_ext().fill(jobs, arr.ctypes.data, caps.ctypes.data, _OPS, _arr)
        cap1, cap2 = caps[:m], caps[m: 2 * m]
        off1 = np.zeros(m, np.int64)
        if m:
            np.cumsum((cap1 + cap2)[:-1], out=off1[1:])
        off2 = off1 + cap1
        out = self._out_buffer(max(int((cap1 + cap2).sum()), 1))
        base = np.uint64(out.__array_interface__["data"][0])
        v = arr[:m]
        v["out"] = base + np.uint64(4) * off1.astype(np.uint64)
        v["out2"] = np.where(cap2 > 0, base + np.uint64(4) * off2.astype(np.uint64), np.uint64(0))
        rc = self._L.fpx_batch_run(self._h, arr.ctypes.data, m, repr)
        if rc not in (OK, EDOMAIN, ESIZE, ELENGTH, EINVAL):
            self._check(rc, "batch")
        del keep  # the converted inputs are no longer read
        st, ol, ol2 = v["status"].tolist(), v["out_len"].tolist(), v["out2_len"].tolist()
        o1s, o2s, ops = off1.tolist(), off2.tolist(), v["op"].tolist()
        res = []
        for i in range(m):
            if st[i] != OK:
                res.append(_ERRORS.get(st[i], FpxError)(st[i], f"batch job {i} ({jobs[i][0]})"))
            elif ops[i] == OP_DIVMOD:
                res.append((out[o1s[i]: o1s[i] + ol[i]], out[o2s[i]: o2s[i] + ol2[i]]))
            else:
                res.append(out[o1s[i]: o1s[i] + ol[i]])
        return res

    def _out_buffer(self, words: int) -> np.ndarray:
        """Output buffer of a batch.  Large ones are page-locked (fpx_host_alloc:
        the batch's results are copied straight into them, with no host-side
        unpacking), kept (at most two) and handed out again once no result of the
        call that had them is referenced any more.  When both kept buffers are
        still referenced, the call gets an ordinary buffer (transparent huge pages
        requested): pinning hundreds of MB costs more than the page faults."""
        if words < _OUT_KEEP_WORDS:
            return np.empty(words, np.uint32)
        for b in self._outbufs:
            # references: the list, the loop variable, the argument (a result view adds one)
            if b.size >= words and sys.getrefcount(b) == 3:
                return b[:words]
        free = [i for i, b in enumerate(self._outbufs) if sys.getrefcount(b) == 3]
        keep = len(self._outbufs) < 2 or bool(free)
        buf = _pinned_words(self._L, words) if keep else None
        if buf is None:
            m = mmap.mmap(-1, words * 4)
            if hasattr(m, "madvise") and hasattr(mmap, "MADV_HUGEPAGE"):
                try:
                    m.madvise(mmap.MADV_HUGEPAGE)
                except OSError:
                    pass
            buf = np.frombuffer(m, np.uint32)
        if keep:
            if len(self._outbufs) < 2:
                self._outbufs.append(buf)
            else:
                self._outbufs[free[0]] = buf
        return buf

    def batch_submit(self, jobs) -> int:
        """fpx_batch_submit on a ctypes array of Job with device pointers; returns the call's status
        (per-job statuses and lengths are written into the array)."""
        return self._L.fpx_batch_submit(self._h, C.cast(jobs, C.c_void_p), len(jobs))

    def batch_wait(self):
        self._check(self._L.fpx_batch_wait(self._h), "batch_wait")


def measure_imad_rate(device: int = 0) -> float:
    """Measured thread-level 32-bit multiply instructions per second of the GPU."""
    r = C.c_double(0)
    rc = load_library().fpx_measure_imad_rate(device, C.byref(r))
    if rc != OK:
        raise FpxError(rc, "fpx_measure_imad_rate failed")
    return r.value


def measure_butterfly_rate(device: int = 0) -> float:
    """Measured lazy DIF butterflies per second (all SMs), the transforms' compute ceiling."""
    r = C.c_double(0)
    rc = load_library().fpx_measure_butterfly_rate(device, C.byref(r))
    if rc != OK:
        raise FpxError(rc, "fpx_measure_butterfly_rate failed")
    return r.value


def ntt_max_log(p: int) -> int:
    return load_library().fpx_ntt_max_log(p)


__all__ = ["Context", "DomainError", "NttSizeError", "LengthError", "FpxError", "CANONICAL", "MONTGOMERY",
           "load_library", "ntt_max_log", "LIB_PATH", "Job", "Server", "make_job", "job_result", "OP_CONV", "OP_INV", "OP_LOG", "OP_EXP", "OP_SQRT",
           "OP_POW", "OP_DIVMOD"]
