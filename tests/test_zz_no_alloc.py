"""fpx_conv_noalloc: the convolution entry point that allocates no device memory.

It exists for callers that cannot allocate when they need a product: code whose
device memory is owned by a host framework's allocator (often reserved in full
at start-up), or latency-critical loops that cannot take cudaMalloc's implicit
device synchronisation.  Its scratch lives in a static device array, so this
test checks it through the C ABI against the ordinary allocating entry point
(fpx_conv_device) on calls in a row -- different sizes, primes and a square,
so no call may see an earlier call's tables or transform buffers -- and that
sizes beyond the array or the prime's roots of unity are refused with
FPX_ESIZE and unusable moduli with FPX_EINVAL.  The test allocates its
own inputs and outputs; the entry point under test allocates nothing.
Exact equality: the results are integers modulo p.
"""
import ctypes as C

import numpy as np
import pytest

import fastpoly_b200 as F

pytestmark = pytest.mark.gpu


def _entry():
    lib = F.load_library()
    fn = lib.fpx_conv_noalloc
    fn.argtypes = [C.c_uint32, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p,
                   C.POINTER(C.c_size_t), C.c_void_p]
    fn.restype = C.c_int
    return fn


def _dev(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).cuda()


def test_conv_noalloc_matches_allocating_entry_point():
    import torch

    noalloc = _entry()
    ctx = F.Context(0)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(2024)
    # two calls in a row: a two-pass size (2^19-point transform) and a one-CTA size on another prime
    cases = [(998244353, 300000, 200001, None), (167772161, 3000, 2500, 4000)]
    for p, la, lb, n in cases:
        a = rng.integers(0, p, la, dtype=np.uint64).astype(np.uint32)
        b = rng.integers(0, p, lb, dtype=np.uint64).astype(np.uint32)
        da, db = _dev(torch, a), _dev(torch, b)
        outn = la + lb - 1 if n is None else min(n, la + lb - 1)
        want_t = torch.empty(outn, dtype=torch.int32, device="cuda")
        got_t = torch.full((outn,), -1, dtype=torch.int32, device="cuda")
        lim = F.SIZE_MAX if n is None else n
        want_len = ctx.conv_device(p, da, la, db, lb, n, want_t)
        ctx.synchronize()
        got_len = C.c_size_t(0)
        rc = noalloc(p, da.data_ptr(), la, db.data_ptr(), lb, lim, got_t.data_ptr(), C.byref(got_len), stream)
        torch.cuda.synchronize()
        assert rc == F.OK
        assert got_len.value == want_len == outn
        assert torch.equal(got_t, want_t), f"p={p} {la}x{lb}"

    # a square (both operands the same buffer), a one-CTA size below 2^13 points
    # and the two-pass size again: each call rebuilds only the tables it reads
    a = rng.integers(0, 998244353, 70000, dtype=np.uint64).astype(np.uint32)
    c = rng.integers(0, 754974721, 100, dtype=np.uint64).astype(np.uint32)
    d = rng.integers(0, 754974721, 100, dtype=np.uint64).astype(np.uint32)
    for p, x, y, same in [(998244353, a, a, True), (754974721, c, d, False), (998244353, a, a[:50001], False),
                          (754974721, c, c, True)]:
        dx = _dev(torch, x)
        dy = dx if same else _dev(torch, y)
        outn = len(x) + len(y) - 1
        want_t = torch.empty(outn, dtype=torch.int32, device="cuda")
        got_t = torch.full((outn,), -1, dtype=torch.int32, device="cuda")
        ctx.conv_device(p, dx, len(x), dy, len(y), None, want_t)
        ctx.synchronize()
        got_len = C.c_size_t(0)
        rc = noalloc(p, dx.data_ptr(), len(x), dy.data_ptr(), len(y), F.SIZE_MAX, got_t.data_ptr(),
                     C.byref(got_len), stream)
        torch.cuda.synchronize()
        assert rc == F.OK and got_len.value == outn
        assert torch.equal(got_t, want_t), f"p={p} {len(x)}x{len(y)} same={same}"

    # moduli the transform path cannot take: a prime whose 2-adic part is too
    # small for the product (97: 2^5 | 96, product of 81 terms), 1e9+7 (no
    # roots of unity past 2), a composite, a prime above 2^30
    e = _dev(torch, np.arange(1, 101, dtype=np.uint32))
    out = torch.zeros(256, dtype=torch.int32, device="cuda")
    for p, ln, want_rc in [(97, 41, F.ESIZE), (1000000007, 100, F.ESIZE), (998244355, 100, F.EINVAL),
                           (2147483647, 100, F.EINVAL)]:
        got_len = C.c_size_t(7)
        rc = noalloc(p, e.data_ptr(), ln, e.data_ptr(), ln, F.SIZE_MAX, out.data_ptr(), C.byref(got_len), stream)
        assert rc == want_rc and got_len.value == 0, (p, rc)
    torch.cuda.synchronize()
    assert not torch.any(out != 0), "a refused call wrote its output"

    # beyond the static array (transform of 2^21 points): refused, nothing written
    a = _dev(torch, np.ones(1 << 20, dtype=np.uint32))
    out = torch.zeros(4, dtype=torch.int32, device="cuda")
    got_len = C.c_size_t(7)
    rc = noalloc(998244353, a.data_ptr(), 1 << 20, a.data_ptr(), 1 << 20, 4, out.data_ptr(), C.byref(got_len), stream)
    assert rc == F.OK and got_len.value == 4  # truncation to n = 4 keeps it within the array
    rc = noalloc(998244353, a.data_ptr(), 1 << 20, a.data_ptr(), 1 << 20, F.SIZE_MAX, out.data_ptr(),
                 C.byref(got_len), stream)
    assert rc == F.ESIZE and got_len.value == 0
    torch.cuda.synchronize()
    ctx.close()
