"""The cluster Newton kernels for moduli without 2^13-th roots of unity.

Series inverses, exponentials and square roots modulo 1e9+7, 2^31-1 and small
primes run their first 2^13 terms on a cluster of three CTAs (k_newton_*_crt:
three-prime CRT products and Garner in shared memory) and continue with the
per-step CRT products.  Every length around the step boundaries, on both sides
of 2^13, against the oracle."""
import numpy as np
import pytest

from test_gpu_parity import eq, rnd

pytestmark = pytest.mark.gpu

MODULI = [1000000007, 2147483647, 1000000009, 97, 2]
LENGTHS = [1, 2, 3, 5, 31, 32, 33, 64, 100, 1000, 4095, 4096, 4097, 8191, 8192, 8193, 20000]


@pytest.mark.parametrize("p", MODULI)
def test_inv_crt_small_steps(fpx, oracle, p):
    rng = np.random.default_rng(p % 1000)
    for n in LENGTHS:
        for la in sorted({1, min(n, 7), n, n + 5}):
            a = rnd(rng, p, la, nonzero0=True)
            eq(fpx.inv(p, a, n), oracle.inv(p, a, n), f"inv p={p} n={n} la={la}")


def test_log_crt(fpx, oracle):
    """log goes through the same inverse."""
    p = 1000000007
    rng = np.random.default_rng(17)
    for n in (2, 33, 4096, 9000):
        a = rnd(rng, p, n)
        a[0] = 1
        eq(fpx.log(p, a, n), oracle.log(p, a, n), f"log n={n}")


EXP_LENGTHS = [2, 3, 5, 32, 33, 100, 1000, 4096, 4097, 8191, 8192, 8193, 20000]


@pytest.mark.parametrize("p", [1000000007, 2147483647, 1000000009])
def test_exp_crt_small_steps(fpx, oracle, p):
    rng = np.random.default_rng(p % 977)
    for n in EXP_LENGTHS:
        for la in sorted({2, n, n + 3}):
            a = rnd(rng, p, la)
            a[0] = 0
            eq(fpx.exp(p, a, n), oracle.exp(p, a, n), f"exp p={p} n={n} la={la}")


def test_exp_crt_small_prime(fpx, oracle):
    """n - 1 < p: lengths up to a small prime."""
    p = 97
    rng = np.random.default_rng(4)
    for n in (2, 17, 64, 96, 97):
        a = rnd(rng, p, n)
        a[0] = 0
        eq(fpx.exp(p, a, n), oracle.exp(p, a, n), f"exp p=97 n={n}")


@pytest.mark.parametrize("p", [1000000007, 2147483647, 97])
def test_sqrt_crt_small_steps(fpx, oracle, p):
    rng = np.random.default_rng(p % 991)
    for n in EXP_LENGTHS:
        a = rnd(rng, p, n)
        a[0] = 1
        sq = oracle.conv(p, a, a, n)
        eq(fpx.sqrt(p, sq, n), oracle.sqrt(p, sq, n), f"sqrt p={p} n={n}")
        # a shifted square (even valuation) and a square constant other than 1
        sh = np.concatenate([np.zeros(4, np.uint32), sq[: max(0, n - 4)]])
        eq(fpx.sqrt(p, sh, n), oracle.sqrt(p, sh, n), f"sqrt shifted p={p} n={n}")
        b = a.copy()
        b[0] = 3 % p
        sq3 = oracle.conv(p, b, b, n)
        eq(fpx.sqrt(p, sq3, n), oracle.sqrt(p, sq3, n), f"sqrt c0=9 p={p} n={n}")


def test_pow_crt(fpx, oracle):
    """pow through log and exp."""
    p = 1000000007
    rng = np.random.default_rng(23)
    for n in (10, 3000, 9000):
        a = rnd(rng, p, n, nonzero0=True)
        for k in (3, 1000003, (1 << 63) + 12345):
            eq(fpx.pow(p, a, k, n), oracle.pow(p, a, k, n), f"pow n={n} k={k}")
