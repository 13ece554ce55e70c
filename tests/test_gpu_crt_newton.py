"""The one-CTA Newton inverse for moduli without 2^13-th roots of unity.

Series inverses modulo 1e9+7, 2^31-1 and small primes run their first 2^13
terms in one CTA (k_newton_inv_crt: three-prime CRT products and Garner in
shared memory) and continue with the per-step CRT products.  Every length
around the step boundaries, on both sides of 2^13, against the oracle."""
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
