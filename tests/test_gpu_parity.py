"""Parity of the CUDA path against the oracle, through the C ABI.

Bit-exact comparison (integer work): every output residue and every output
length must equal the oracle's, and the reference's error conditions must be
reported as the same errors.  Mirrors the reference's own suites
(tests/test_ntt.cpp, test_poly.cpp, test_prime_poly.cpp)."""
import numpy as np
import pytest

import fastpoly_b200 as F
from conftest import bench_checksum
from oracle.oracle import DomainError as OracleDomainError

pytestmark = pytest.mark.gpu

NATIVE = [998244353, 167772161, 469762049, 754974721]
CRT_ONLY = [1000000007, 2147483647, 1224736769, 2, 3, 17, 193, 100003]


def rnd(rng, p, n, nonzero0=False):
    a = rng.integers(0, p, n, dtype=np.uint64).astype(np.uint32)
    if nonzero0 and n:
        a[0] = a[0] or 1
    return a


def eq(got, want, what=""):
    got = np.asarray(got, dtype=np.uint32)
    want = np.asarray(want, dtype=np.uint32)
    assert got.shape == want.shape, (what, got.shape, want.shape)
    if not np.array_equal(got, want):
        bad = np.nonzero(got != want)[0]
        raise AssertionError(f"{what}: {bad.size} mismatches, first at {bad[:8].tolist()}: "
                             f"got {got[bad[:4]].tolist()} want {want[bad[:4]].tolist()}")


# ---------------------------------------------------------------- transforms

@pytest.mark.parametrize("p", NATIVE)
def test_ntt_matches_oracle(fpx, oracle, p):
    rng = np.random.default_rng(p)
    for k in list(range(1, 17)) + [18, 20]:
        n = 1 << k
        x = rnd(rng, p, n)
        y = fpx.ntt_forward(p, x)
        eq(y, oracle.ntt_forward(p, x), f"forward p={p} n={n}")
        eq(fpx.ntt_inverse(p, y), x, f"roundtrip p={p} n={n}")


def test_ntt_largest_native_sizes(fpx, oracle):
    rng = np.random.default_rng(3)
    for p, k in [(998244353, 23), (754974721, 24)]:
        n = 1 << k
        x = rnd(rng, p, n)
        y = fpx.ntt_forward(p, x)
        eq(y, oracle.ntt_forward(p, x), f"forward p={p} n=2^{k}")
        eq(fpx.ntt_inverse(p, y), x, f"roundtrip p={p} n=2^{k}")


def test_ntt_size_errors(fpx):
    p = 998244353
    for n in (1, 3, 1 << 24):
        with pytest.raises(F.NttSizeError):
            fpx.ntt_forward(p, np.zeros(n, dtype=np.uint32))


def test_ntt_montgomery_limbs(fpx, oracle):
    p, n = 998244353, 4096
    x = rnd(np.random.default_rng(1), p, n)
    limbs = np.array([oracle.to_mont(p, int(v)) for v in x], dtype=np.uint32)
    got = fpx.ntt_forward(p, limbs, repr=F.MONTGOMERY)
    want = np.array([oracle.to_mont(p, int(v)) for v in oracle.ntt_forward(p, x)], dtype=np.uint32)
    eq(got, want, "montgomery forward")


# ---------------------------------------------------------------- products

CONV_SIZES = [(1, 1), (1, 7), (5, 40), (40, 41), (41, 41), (63, 65), (100, 3000), (2048, 2049), (4096, 4097),
              (4097, 4096), (5000, 7000), (8192, 8193), (20000, 30000), (65536, 65536), (131071, 1000)]


@pytest.mark.parametrize("p", NATIVE)
def test_conv_native(fpx, oracle, p):
    rng = np.random.default_rng(11)
    for la, lb in CONV_SIZES:
        a, b = rnd(rng, p, la), rnd(rng, p, lb)
        eq(fpx.conv(p, a, b), oracle.conv(p, a, b), f"conv p={p} {la}x{lb}")
        n = (la + lb) // 3 + 1
        eq(fpx.conv(p, a, b, n), oracle.conv(p, a, b, n), f"conv trunc p={p} {la}x{lb} n={n}")
    a = rnd(rng, p, 9000)
    eq(fpx.conv(p, a, a), oracle.conv(p, a, a), "square")


@pytest.mark.parametrize("p", CRT_ONLY)
def test_conv_crt(fpx, oracle, p):
    rng = np.random.default_rng(12)
    for la, lb in [(39, 52), (41, 44), (65, 78), (259, 272), (3000, 5000), (70000, 70001)]:
        a, b = rnd(rng, p, la), rnd(rng, p, lb)
        eq(fpx.conv(p, a, b), oracle.conv(p, a, b), f"crt conv p={p} {la}x{lb}")
    ext = np.full(3000, p - 1, dtype=np.uint32)
    eq(fpx.conv(p, ext, ext), oracle.conv(p, ext, ext), f"extremes p={p}")


def test_conv_edge_cases(fpx):
    p = 998244353
    assert fpx.conv(p, [], [1]).size == 0
    assert fpx.conv(p, [1, 2], [3], 0).size == 0
    eq(fpx.conv(p, [2], [3, 4]), [6, 8])


def test_conv_large_native(fpx, oracle):
    # Two 2^22-term inputs: the 2^23-point native transform of the headline.
    p, n = 998244353, 1 << 22
    rng = np.random.default_rng(22)
    a, b = rnd(rng, p, n), rnd(rng, p, n)
    eq(fpx.conv(p, a, b), oracle.conv(p, a, b), "conv 2^22 x 2^22")


def test_conv_crt_beyond_native(fpx, oracle):
    # Full length 2^24 - 1 > 2^23: mod 998244353 this is the 3-prime CRT (convolution.hpp:108).
    p, n = 998244353, (1 << 23)
    rng = np.random.default_rng(23)
    a, b = rnd(rng, p, n), rnd(rng, p, 1 << 20)
    eq(fpx.conv(p, a, b), oracle.conv(p, a, b), "crt conv beyond native")


# ---------------------------------------------------------------- series

SERIES_N = [1, 2, 9, 31, 32, 33, 40, 41, 64, 65, 127, 128, 129, 257, 513, 4095, 4097, 8193, 20000]


@pytest.mark.parametrize("p", [998244353, 167772161, 1000000007, 2147483647, 3, 17, 97, 193, 641])
def test_series_vs_oracle(fpx, oracle, p):
    rng = np.random.default_rng(p + 5)
    for n in SERIES_N:
        a = rnd(rng, p, n + 11, nonzero0=True)
        for la in (1, 2, 8, a.size):
            eq(fpx.inv(p, a[:la], n), oracle.inv(p, a[:la], n), f"inv p={p} n={n} la={la}")
        if n <= p:
            l1 = a.copy(); l1[0] = 1
            eq(fpx.log(p, l1, n), oracle.log(p, l1, n), f"log p={p} n={n}")
        if n - 1 < p:
            e0 = a.copy(); e0[0] = 0
            eq(fpx.exp(p, e0, n), oracle.exp(p, e0, n), f"exp p={p} n={n}")
        sq = oracle.conv(p, a, a, n)
        eq(fpx.sqrt(p, sq, n), oracle.sqrt(p, sq, n), f"sqrt p={p} n={n}")
        for k in (0, 1, 2, 65, 1000003, 2**64 - 1):
            u = a[: 1 + n // 3]
            eq(fpx.pow(p, u, k, n), oracle.pow(p, u, k, n), f"pow p={p} n={n} k={k}")


@pytest.mark.parametrize("p", [998244353, 1000000007, 3])
def test_divmod_vs_oracle(fpx, oracle, p):
    rng = np.random.default_rng(p + 9)
    for la, lb in [(3, 5), (10, 1), (40, 17), (120, 50), (300, 120), (5000, 1200), (70000, 30000), (64, 64)]:
        a, b = rnd(rng, p, la), rnd(rng, p, lb)
        b[-1] = b[-1] or 1
        q, r = fpx.divmod(p, a, b)
        wq, wr = oracle.divmod(p, a, b)
        eq(q, wq, f"q p={p} {la}/{lb}")
        eq(r, wr, f"r p={p} {la}/{lb}")
        eq(fpx.div(p, a, b), wq, "div")
        eq(fpx.mod(p, a, b), wr, "mod")


def test_domain_errors(fpx):
    p = 998244353
    with pytest.raises(F.DomainError):
        fpx.inv(p, [0, 1], 8)
    with pytest.raises(F.DomainError):
        fpx.log(p, [2, 1], 3)
    with pytest.raises(F.DomainError):
        fpx.exp(p, [1, 1], 3)
    with pytest.raises(F.DomainError):
        fpx.sqrt(p, [0, 4], 5)
    with pytest.raises(F.DomainError):
        fpx.divmod(p, [1, 2], [0, 0])
    with pytest.raises(F.DomainError):
        fpx.log(3, [1, 1], 4)
    with pytest.raises(F.DomainError):
        fpx.exp(3, [0, 1], 4)
    with pytest.raises(F.DomainError):
        fpx.sqrt(2, [1, 1], 6)
    assert fpx.inv(p, [], 0).size == 0


# ---------------------------------------------------------------- goldens

def _run_case(lib, case):
    p, op = case["p"], case["op"]
    if op == "conv":
        return lib.conv(p, case["a"], case["b"], case["n"])
    if op == "pow":
        return lib.pow(p, case["a"], case["k"], case["n"])
    if op == "divmod":
        return lib.divmod(p, case["a"], case["b"])
    return getattr(lib, op)(p, case["a"], case["n"])


def test_reference_vectors(fpx, ref_vectors):
    for case in ref_vectors:
        if case["status"] == "domain_error":
            with pytest.raises(F.DomainError):
                _run_case(fpx, case)
            continue
        got = _run_case(fpx, case)
        if case["op"] == "divmod":
            eq(got[0], case["q"], f"{case['op']} p={case['p']}")
            eq(got[1], case["r"], f"{case['op']} p={case['p']}")
        else:
            eq(got, case["out"], f"{case['op']} p={case['p']}")


def test_published_checksums(fpx, oracle, published):
    checked = 0
    for row in published:
        p = row["p"]
        if row["op"].startswith("ntt") and p >= (1 << 30):
            continue  # raw GPU transforms are for p < 2^30 (products at p >= 2^30 go through the CRT)
        got = bench_checksum(oracle, p, row["op"], row["n"], fpx)
        assert f"{got:016x}" == row["checksum"], row
        checked += 1
    assert checked >= 380


def test_montgomery_repr_roundtrip(fpx, oracle):
    p = 998244353
    rng = np.random.default_rng(4)
    a, b = rnd(rng, p, 5000), rnd(rng, p, 7000)
    to_m = np.vectorize(lambda v: oracle.to_mont(p, int(v)), otypes=[np.uint32])
    got = fpx.conv(p, to_m(a), to_m(b), repr=F.MONTGOMERY)
    eq(got, to_m(oracle.conv(p, a, b)), "montgomery conv")
    a[0] = 1
    eq(fpx.inv(p, to_m(a), 3000, repr=F.MONTGOMERY), to_m(oracle.inv(p, a, 3000)), "montgomery inv")


def test_device_api(fpx, oracle):
    import torch
    p = 998244353
    rng = np.random.default_rng(5)
    a, b = rnd(rng, p, 100000), rnd(rng, p, 90000)
    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = torch.from_numpy(b.view(np.int32)).cuda()
    out = torch.empty(a.size + b.size - 1, dtype=torch.int32, device="cuda")
    n = fpx.conv_device(p, da, a.size, db, b.size, None, out)
    fpx.synchronize()
    assert n == a.size + b.size - 1
    eq(out.cpu().numpy().view(np.uint32), oracle.conv(p, a, b), "device conv")
    a[0] = 1
    da = torch.from_numpy(a.view(np.int32)).cuda()
    o2 = torch.empty(50000, dtype=torch.int32, device="cuda")
    fpx.inv_device(p, da, a.size, 50000, o2)
    fpx.synchronize()
    eq(o2.cpu().numpy().view(np.uint32), oracle.inv(p, a, 50000), "device inv")


def _coeff(a, b, t, p):
    """Exact coefficient t of a * b mod p (numpy, products below 2^60)."""
    lo, hi = max(0, t - (b.size - 1)), min(t, a.size - 1)
    if lo > hi:
        return 0
    u = np.arange(lo, hi + 1)
    prod = (a[u].astype(np.uint64) * b[t - u].astype(np.uint64)) % np.uint64(p)
    return int(prod.sum(dtype=np.uint64) % np.uint64(p))


def test_crt_blocked_product(fpx):
    """Products of more than one 2^23-term block on a prime without 2^24 roots:
    the spectra-reusing blocked path against the per-pair path of the
    reference's block scheme, bit for bit, and exact coefficients."""
    import os
    p = 1000000007
    rng = np.random.default_rng(25)
    a = rnd(rng, p, (1 << 23) + 1001)
    b = rnd(rng, p, (1 << 23) + 77)
    got = fpx.conv(p, a, b)
    sq = fpx.conv(p, a, a)
    os.environ["FPX_CRT_BLOCKED"] = "0"
    try:
        want = fpx.conv(p, a, b)
        want_sq = fpx.conv(p, a, a)
    finally:
        del os.environ["FPX_CRT_BLOCKED"]
    eq(got, want, "blocked conv")
    eq(sq, want_sq, "blocked square")
    for t in (0, 7, (1 << 23) - 1, 1 << 23, (1 << 23) + 500, (1 << 24) + 1000, got.size - 1):
        assert int(got[t]) == _coeff(a, b, t, p), t
    trunc = fpx.conv(p, a, b, (1 << 23) + 12345)
    eq(trunc, got[: (1 << 23) + 12345], "blocked truncated")
