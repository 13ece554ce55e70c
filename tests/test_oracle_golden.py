"""Pins the oracle (CPU restatement) before it is trusted as the checker:

* against every checksum the reference publishes for this path (bench CSVs);
* against the reference's own outputs on small seeded inputs over 14 moduli
  (tests/golden/reference_vectors.json, generated by make_golden.py from the
  reference compiled from its headers);
* against the reference's known-answer identities (tests/test_ntt.cpp,
  tests/test_poly.cpp, tests/test_prime_poly.cpp).
"""
import numpy as np
import pytest

from conftest import bench_case, bench_checksum  # noqa: F401
from oracle.oracle import DomainError


def test_published_checksums(oracle, published):
    checked = 0
    for row in published:
        got = bench_checksum(oracle, row["p"], row["op"], row["n"], oracle)
        assert f"{got:016x}" == row["checksum"], row
        checked += 1
    assert checked >= 400


def _run(O, case):
    p, op = case["p"], case["op"]
    if op == "conv":
        return O.conv(p, case["a"], case["b"], case["n"])
    if op == "pow":
        return O.pow(p, case["a"], case["k"], case["n"])
    if op == "divmod":
        return O.divmod(p, case["a"], case["b"])
    return getattr(O, op)(p, case["a"], case["n"])


def test_reference_vectors(oracle, ref_vectors):
    for case in ref_vectors:
        if case["status"] == "domain_error":
            with pytest.raises(DomainError):
                _run(oracle, case)
            continue
        got = _run(oracle, case)
        if case["op"] == "divmod":
            assert got[0].tolist() == case["q"], case
            assert got[1].tolist() == case["r"], case
        else:
            assert got.tolist() == case["out"], case


def test_monomial_is_dft(oracle):
    # tests/test_ntt.cpp:51-70: x^j maps to a permutation of {w^(jk)}.
    for p in (998244353, 167772161, 754974721):
        g = oracle.primitive_root(p)
        for k in range(1, 11):
            n = 1 << k
            w = pow(g, (p - 1) // n, p)
            for j in range(0, n, max(1, n // 4)):
                x = np.zeros(n, dtype=np.uint32)
                x[j] = 1
                got = sorted(oracle.ntt_forward(p, x).tolist())
                want = sorted(pow(w, j * t, p) for t in range(n))
                assert got == want


def test_constant_and_impulse(oracle):
    # tests/test_ntt.cpp:223-235
    p, n = 998244353, 64
    y = oracle.ntt_forward(p, np.full(n, 5, dtype=np.uint32))
    assert (y != 0).sum() == 1 and y[0] == 5 * n % p


def test_crt_blocks_and_prime_count(oracle):
    # tests/test_prime_poly.cpp:110-121 (Block = 64) and :235-257.
    assert oracle.crt_prime_count(3, 1 << 23) == 1
    assert oracle.crt_prime_count(100003, 64) == 2
    assert oracle.crt_prime_count(1000000007, 64) == 3
    assert oracle.crt_prime_count(641, 409) == 1
    assert oracle.crt_prime_count(641, 410) == 2
    assert oracle.crt_prime_count(167772161, 2) == 2
    assert oracle.crt_prime_count(167772161, 3) == 3
    rng = np.random.default_rng(5)
    for p in (2, 3, 193, 100003, 1000000007, 2147483647, 998244353):
        for la, lb in [(1, 14), (39, 52), (65, 78), (259, 272)]:
            a = rng.integers(0, p, la, dtype=np.uint64).astype(np.uint32)
            b = rng.integers(0, p, lb, dtype=np.uint64).astype(np.uint32)
            want = oracle.conv(p, a, b)
            for out in (1, la, la + lb - 1):
                got = oracle.crt_convolution(p, a, b, out, 64)
                assert got.tolist() == want[:out].tolist()


def test_series_identities(oracle):
    # tests/test_prime_poly.cpp:172-191: a*inv(a) = 1, exp(log a) = a, sqrt^2.
    rng = np.random.default_rng(7)
    for p in (998244353, 1000000007, 3):
        n = 2049
        a = rng.integers(0, p, n, dtype=np.uint64).astype(np.uint32)
        a[0] = 1
        unit = oracle.conv(p, a, oracle.inv(p, a, n), n)
        assert unit[0] == 1 and not unit[1:].any()
        if n <= p:
            assert oracle.exp(p, oracle.log(p, a, n), n).tolist() == a.tolist()
        sq = oracle.conv(p, a, a, n)
        root = oracle.sqrt(p, sq, n)
        assert oracle.conv(p, root, root, n).tolist() == sq.tolist()


def test_small_characteristic_contracts(oracle):
    # tests/test_prime_poly.cpp:315-345
    assert oracle.exp(3, [0, 1], 3).tolist() == [1, 1, 2]
    assert oracle.log(3, [1, 1, 2], 3).tolist() == [0, 1, 0]
    with pytest.raises(DomainError):
        oracle.log(3, [1, 1], 4)
    with pytest.raises(DomainError):
        oracle.exp(3, [0, 1], 4)
    assert oracle.exp(2, [0, 1], 2).tolist() == [1, 1]
    assert oracle.log(2, [1, 1], 2).tolist() == [0, 1]
    assert oracle.sqrt(2, [1, 0, 1, 0, 1], 6).tolist() == [1, 1, 1, 0, 0, 0]
    with pytest.raises(DomainError):
        oracle.sqrt(2, [1, 1], 6)
    assert oracle.sqrt(2, [1, 1], 1).tolist() == [1]


def test_domain_errors(oracle):
    p = 998244353
    with pytest.raises(DomainError):
        oracle.inv(p, [0, 1], 8)
    with pytest.raises(DomainError):
        oracle.inv(p, [], 3)
    with pytest.raises(DomainError):
        oracle.log(p, [2, 1], 3)
    with pytest.raises(DomainError):
        oracle.exp(p, [1, 1], 3)
    with pytest.raises(DomainError):
        oracle.sqrt(p, [0, 4], 5)
    with pytest.raises(DomainError):
        oracle.divmod(p, [1, 2], [0, 0])
    assert oracle.inv(p, [], 0).size == 0
    assert oracle.conv(p, [], [1]).size == 0


def _scale(p, x, c):
    return (np.asarray(x, np.uint64) * np.uint64(c) % np.uint64(p)).astype(np.uint32)


@pytest.mark.parametrize("p", [998244353, 1000000007, 167772161, 7340033])
def test_identities_of_phased_batch_jobs(oracle, p):
    """The formulas batches use for sqrt and pow, checked on the oracle: for p
    odd and n <= p, sqrt(u) = r0 * exp(log(u / u0) / 2) with r0 the reference's
    root of u0 (a power series has one square root with a given constant term),
    and pow(u, k) = c0^k exp((k mod p) log(u / c0)) (power.hpp:76-86)."""
    rng = np.random.default_rng(p % 1000)
    for n in (1, 2, 17, 300, 1000):
        u0 = int(rng.integers(1, p)) ** 2 % p
        u = rng.integers(0, p, n + 5, dtype=np.uint64).astype(np.uint32)
        u[0] = u0
        r0 = oracle.sqrt_mod(u0, p)
        half = (p + 1) // 2
        lg = oracle.log(p, _scale(p, u, pow(u0, p - 2, p)), n)
        via = _scale(p, oracle.exp(p, _scale(p, lg, half), n), r0)
        assert np.array_equal(via, oracle.sqrt(p, u[:n], n)), (p, n)
        k = int(rng.integers(65, 2 ** 63))
        c0 = int(u[0])
        via_pow = _scale(p, oracle.exp(p, _scale(p, oracle.log(p, _scale(p, u, pow(c0, p - 2, p)), n), k % p), n),
                         pow(c0, k, p))
        assert np.array_equal(via_pow, oracle.pow(p, u, k, n)), (p, n, k)
