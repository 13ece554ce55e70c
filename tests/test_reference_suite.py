"""The reference's own polynomial test suites, run unchanged on the GPU library.

oracle/Makefile (target ref-tests) compiles the reference's tests/test_poly.cpp
and tests/test_prime_poly.cpp from the reference checkout without any edit:
an include redirect (tests/cpp/shim/fastpoly/*.hpp) makes their
"fastpoly/poly.hpp" / "fastpoly/fastpoly.hpp" includes resolve to the drop-in
header include/fpx/fastpoly.hpp, and the binaries link the product library
(fastpoly_b200/libfpx_b200.so).  Every check in those files -- identities over
six NTT primes, convolution boundaries, Newton series, CRT block loops with
64-term blocks, middle products, small characteristics, the Poly<M> API -- then
runs against the GPU path.  The binaries are built where the checkout is and
travel with the repository; without them these tests skip.
"""
import os
import subprocess

import pytest

from conftest import ROOT

REF = os.path.join(ROOT, "oracle", "_ref")
SUITES = ["ref_test_poly", "ref_test_prime_poly"]


@pytest.mark.gpu
@pytest.mark.parametrize("suite", SUITES)
def test_reference_suite_on_gpu(suite):
    exe = os.path.join(REF, suite)
    if not os.path.exists(exe):
        pytest.skip(f"{suite} not built (make -C oracle ref-tests where the reference checkout is)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=1200)
    fails = [ln for ln in r.stdout.splitlines() if "FAIL" in ln or "failed" in ln]
    print(r.stdout[-4000:])
    assert r.returncode == 0, "\n".join(fails[:40]) + r.stderr[-2000:]
    assert "tests passed" in r.stdout
