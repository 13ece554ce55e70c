"""Python bindings for the parity oracle -- TEST INFRASTRUCTURE ONLY.

Two checkers live here:

* ``Oracle``: the plain-C restatement of fastpoly's algorithms
  (``oracle/fpx_oracle.c``, built to ``oracle/build/libfpx_oracle.so``).
* ``Reference``: the unmodified reference headers (xcx0902/fastpoly) behind a
  C shim (``oracle/ref_driver.cpp``, built to ``oracle/_ref/``).  Present only
  where the reference could be compiled; callers must handle ``None``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module.  The product library never does.

All arrays are canonical residues (numpy ``uint32``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "libfpx_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

OK, EDOMAIN, ESIZE, ELENGTH, ENOMEM = 0, 1, 2, 3, 4


class OracleError(Exception):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: status {code}")
        self.code = code


class DomainError(OracleError):
    """Mirrors fpx::poly::domain_error conditions."""


def _raise(code: int, what: str):
    if code == OK:
        return
    if code == EDOMAIN:
        raise DomainError(code, what)
    raise OracleError(code, what)


_u32p = C.POINTER(C.c_uint32)
_szp = C.POINTER(C.c_size_t)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_u32p) if a.size else None


def _arr(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def build(quiet: bool = True) -> None:
    """Compile the oracle (and the reference shim when the reference checkout,
    FPX_REFERENCE in oracle/Makefile, is present)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "oracle", "ref-if-present"], check=True, stdout=out)


class Oracle:
    """ctypes front end of the C restatement."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        self._L = L
        u32, sz, u64 = C.c_uint32, C.c_size_t, C.c_uint64
        L.fpo_conv.argtypes = [u32, _u32p, sz, _u32p, sz, sz, _u32p, _szp]
        L.fpo_crt_convolution.argtypes = [u32, _u32p, sz, _u32p, sz, sz, sz, _u32p]
        for f in ("fpo_inv", "fpo_log", "fpo_exp", "fpo_sqrt"):
            getattr(L, f).argtypes = [u32, _u32p, sz, sz, _u32p]
        L.fpo_pow.argtypes = [u32, _u32p, sz, u64, sz, _u32p]
        L.fpo_divmod.argtypes = [u32, _u32p, sz, _u32p, sz, _u32p, _szp, _u32p, _szp]
        L.fpo_ntt_forward.argtypes = [u32, _u32p, u32]
        L.fpo_ntt_inverse.argtypes = [u32, _u32p, u32]
        L.fpo_inv_series.argtypes = [u32, sz, _u32p]
        L.fpo_mt19937_64.argtypes = [u64, C.POINTER(C.c_uint64), sz]
        L.fpo_checksum_mont.argtypes = [u32, _u32p, sz]
        L.fpo_checksum_mont.restype = u64
        L.fpo_to_mont.argtypes = [u32, u32]
        L.fpo_to_mont.restype = u32
        L.fpo_sqrt_mod.argtypes = [u32, u32, _u32p]
        L.fpo_primitive_root.argtypes = [u32]
        L.fpo_primitive_root.restype = u32
        L.fpo_ntt_max_log.argtypes = [u32]
        L.fpo_crt_prime_count.argtypes = [u32, sz]
        L.fpo_crt_prime_count.restype = sz

    # -- generators and checksums ------------------------------------------
    def mt19937_64(self, seed: int, count: int) -> np.ndarray:
        out = np.empty(count, dtype=np.uint64)
        self._L.fpo_mt19937_64(seed, out.ctypes.data_as(C.POINTER(C.c_uint64)), count)
        return out

    def checksum(self, p: int, vals) -> int:
        v = _arr(vals)
        return int(self._L.fpo_checksum_mont(p, _ptr(v), v.size))

    def to_mont(self, p: int, v: int) -> int:
        return int(self._L.fpo_to_mont(p, v))

    def primitive_root(self, p: int) -> int:
        return int(self._L.fpo_primitive_root(p))

    def ntt_max_log(self, p: int) -> int:
        return int(self._L.fpo_ntt_max_log(p))

    def crt_prime_count(self, p: int, terms: int) -> int:
        return int(self._L.fpo_crt_prime_count(p, terms))

    def sqrt_mod(self, x: int, p: int):
        out = C.c_uint32(0)
        ok = self._L.fpo_sqrt_mod(x, p, C.byref(out))
        return int(out.value) if ok else None

    # -- operations ---------------------------------------------------------
    def conv(self, p, a, b, n=None) -> np.ndarray:
        a, b = _arr(a), _arr(b)
        lim = (2**64 - 1) if n is None else n
        cap = max(0, min(a.size + b.size - 1, lim)) if a.size and b.size else 0
        out = np.zeros(max(cap, 1), dtype=np.uint32)
        ln = C.c_size_t(0)
        _raise(self._L.fpo_conv(p, _ptr(a), a.size, _ptr(b), b.size, C.c_size_t(lim), _ptr(out), C.byref(ln)), "conv")
        return out[: ln.value].copy()

    def crt_convolution(self, p, a, b, outn, block) -> np.ndarray:
        a, b = _arr(a), _arr(b)
        out = np.zeros(max(outn, 1), dtype=np.uint32)
        _raise(self._L.fpo_crt_convolution(p, _ptr(a), a.size, _ptr(b), b.size, outn, block, _ptr(out)), "crt")
        return out[:outn].copy()

    def _series(self, fn, p, a, n) -> np.ndarray:
        a = _arr(a)
        out = np.zeros(max(n, 1), dtype=np.uint32)
        _raise(fn(p, _ptr(a), a.size, n, _ptr(out)), fn.__name__)
        return out[:n].copy()

    def inv(self, p, a, n):
        return self._series(self._L.fpo_inv, p, a, n)

    def log(self, p, a, n):
        return self._series(self._L.fpo_log, p, a, n)

    def exp(self, p, a, n):
        return self._series(self._L.fpo_exp, p, a, n)

    def sqrt(self, p, a, n):
        return self._series(self._L.fpo_sqrt, p, a, n)

    def pow(self, p, a, k, n):
        a = _arr(a)
        out = np.zeros(max(n, 1), dtype=np.uint32)
        _raise(self._L.fpo_pow(p, _ptr(a), a.size, C.c_uint64(k), n, _ptr(out)), "pow")
        return out[:n].copy()

    def divmod(self, p, a, b):
        a, b = _arr(a), _arr(b)
        q = np.zeros(max(a.size, 1), dtype=np.uint32)
        r = np.zeros(max(a.size, 1), dtype=np.uint32)
        lq, lr = C.c_size_t(0), C.c_size_t(0)
        _raise(self._L.fpo_divmod(p, _ptr(a), a.size, _ptr(b), b.size, _ptr(q), C.byref(lq), _ptr(r), C.byref(lr)),
               "divmod")
        return q[: lq.value].copy(), r[: lr.value].copy()

    def ntt_forward(self, p, x) -> np.ndarray:
        x = _arr(x).copy()
        _raise(self._L.fpo_ntt_forward(p, _ptr(x), x.size), "ntt_forward")
        return x

    def ntt_inverse(self, p, x) -> np.ndarray:
        x = _arr(x).copy()
        _raise(self._L.fpo_ntt_inverse(p, _ptr(x), x.size), "ntt_inverse")
        return x

    def inv_series(self, p, n) -> np.ndarray:
        out = np.zeros(n + 1, dtype=np.uint32)
        _raise(self._L.fpo_inv_series(p, n, _ptr(out)), "inv_series")
        return out

    # -- the reference bench's synthetic inputs (bench/bench.cpp:216-220) ----
    def bench_rnd(self, p: int, seed: int, *counts: int):
        """Consecutive draws of rng() % p from std::mt19937_64(seed)."""
        raw = self.mt19937_64(seed, sum(counts))
        vals = (raw % np.uint64(p)).astype(np.uint32)
        out, pos = [], 0
        for c in counts:
            out.append(vals[pos: pos + c].copy())
            pos += c
        return out


# --------------------------------------------------------------------------
# The reference itself (oracle/_ref).
# --------------------------------------------------------------------------
OP_CONV, OP_INV, OP_LOG, OP_EXP, OP_SQRT, OP_POW, OP_DIVMOD, OP_NTT_FWD, OP_NTT_INV, OP_CRT64 = range(10)


def _cpu_has(flag: str) -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return flag in line.split()
    except OSError:
        pass
    return False


def reference_library_path():
    """Best reference build for this host CPU, or None if none was built."""
    cands = []
    if _cpu_has("avx512f") and _cpu_has("avx512vl"):
        cands.append("libfpx_ref_avx512.so")
    if _cpu_has("avx2"):
        cands.append("libfpx_ref_avx2.so")
    for c in cands:
        path = os.path.join(REF_DIR, c)
        if os.path.exists(path):
            return path
    return None


class Reference:
    """The reference library itself, compiled from its headers (oracle/_ref)."""

    def __init__(self, path: str):
        L = C.CDLL(path)
        self._L = L
        self.path = path
        sz = C.c_size_t
        L.fpr_run.argtypes = [C.c_int, C.c_uint32, _u32p, sz, _u32p, sz, sz, C.c_uint64,
                              _u32p, _szp, _u32p, _szp, C.c_int, C.c_int, C.POINTER(C.c_double)]
        L.fpr_moduli.argtypes = [_u32p, sz]
        L.fpr_moduli.restype = sz
        L.fpr_simd_backend.restype = C.c_char_p
        self.backend = L.fpr_simd_backend().decode()
        buf = np.zeros(64, dtype=np.uint32)
        k = L.fpr_moduli(_ptr(buf), 64)
        self.moduli = [int(x) for x in buf[:k]]

    @classmethod
    def load(cls):
        path = reference_library_path()
        return cls(path) if path else None

    def run(self, op, p, a=(), b=(), n=None, k=0, cap=None, reps=1, threads=1):
        """Run one reference operation; returns (out1, out2, per-rep seconds)."""
        a, b = _arr(a), _arr(b)
        nn = (2**64 - 1) if n is None else n
        if cap is None:
            cap = max(a.size + b.size, (n or 0), 1)
        o1 = np.zeros(cap, dtype=np.uint32)
        o2 = np.zeros(cap, dtype=np.uint32)
        l1, l2 = C.c_size_t(0), C.c_size_t(0)
        times = np.zeros(max(reps, 1), dtype=np.float64)
        rc = self._L.fpr_run(op, p, _ptr(a), a.size, _ptr(b), b.size, C.c_size_t(nn), C.c_uint64(k),
                             _ptr(o1), C.byref(l1), _ptr(o2), C.byref(l2), reps, threads,
                             times.ctypes.data_as(C.POINTER(C.c_double)))
        _raise(rc, f"reference op {op}")
        return o1[: l1.value].copy(), o2[: l2.value].copy(), times

    def conv(self, p, a, b, n=None):
        return self.run(OP_CONV, p, a, b, n=n)[0]

    def inv(self, p, a, n):
        return self.run(OP_INV, p, a, n=n)[0]

    def log(self, p, a, n):
        return self.run(OP_LOG, p, a, n=n)[0]

    def exp(self, p, a, n):
        return self.run(OP_EXP, p, a, n=n)[0]

    def sqrt(self, p, a, n):
        return self.run(OP_SQRT, p, a, n=n)[0]

    def pow(self, p, a, k, n):
        return self.run(OP_POW, p, a, n=n, k=k)[0]

    def divmod(self, p, a, b):
        q, r, _ = self.run(OP_DIVMOD, p, a, b)
        return q, r

    def ntt_forward(self, p, x):
        return self.run(OP_NTT_FWD, p, x)[0]

    def ntt_inverse(self, p, x):
        return self.run(OP_NTT_INV, p, x)[0]

    def crt_convolution64(self, p, a, b, outn):
        return self.run(OP_CRT64, p, a, b, n=outn)[0]
