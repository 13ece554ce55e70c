import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product library")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    """The reference compiled from its headers (oracle/_ref), if it was built."""
    from oracle.oracle import Reference
    ref = Reference.load()
    if ref is None:
        pytest.skip("oracle/_ref not built on this host")
    return ref


@pytest.fixture(scope="session")
def published():
    with open(os.path.join(GOLDEN, "published_checksums.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ref_vectors():
    with open(os.path.join(GOLDEN, "reference_vectors.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def fpx():
    """The product library on cuda:0 (GPU tests only)."""
    import fastpoly_b200
    ctx = fastpoly_b200.Context(device=0)
    yield ctx
    ctx.close()


def rotl64(x: int, r: int) -> int:
    return ((x << r) | (x >> (64 - r))) & (2**64 - 1)


def bench_case(O, p: int, op: str, n: int):
    """The reference bench's inputs for (op, n) (bench/bench.cpp:222-373)."""
    if op in ("ntt-forward", "ntt-inverse"):
        (x,) = O.bench_rnd(p, 1 + n, n)
        return {"x": x}
    if op in ("conv", "conv-trunc"):
        a, b = O.bench_rnd(p, 2 + n, n, n)
        return {"a": a, "b": b}
    if op == "square":
        (a,) = O.bench_rnd(p, 2 + n, n)
        return {"a": a}
    if op == "divmod":
        a, b = O.bench_rnd(p, 4 + n, n, max(1, n // 2))
        return {"a": a, "b": b}
    (a,) = O.bench_rnd(p, 3 + n, n)
    a[0] = 1
    return {"a": a}


def bench_checksum(O, p: int, op: str, n: int, lib) -> int:
    """Runs `op` with `lib` (oracle or GPU library: same method names) on the
    bench inputs and returns the reference bench's checksum of the result."""
    c = bench_case(O, p, op, n)
    if op == "ntt-forward":
        return O.checksum(p, lib.ntt_forward(p, c["x"]))
    if op == "ntt-inverse":
        return O.checksum(p, lib.ntt_inverse(p, lib.ntt_forward(p, c["x"])))
    if op == "conv":
        return O.checksum(p, lib.conv(p, c["a"], c["b"]))
    if op == "conv-trunc":
        return O.checksum(p, lib.conv(p, c["a"], c["b"], n))
    if op == "square":
        return O.checksum(p, lib.conv(p, c["a"], c["a"]))
    if op == "divmod":
        q, r = lib.divmod(p, c["a"], c["b"])
        return O.checksum(p, q) ^ rotl64(O.checksum(p, r), 17)
    a = c["a"]
    if op == "inv":
        return O.checksum(p, lib.inv(p, a, n))
    if op == "log":
        return O.checksum(p, lib.log(p, a, n))
    if op == "exp":
        b = a.copy()
        b[0] = 0
        return O.checksum(p, lib.exp(p, b, n))
    if op == "sqrt":
        sq = lib.conv(p, a, a, n)
        return O.checksum(p, lib.sqrt(p, sq, n))
    if op == "pow":
        return O.checksum(p, lib.pow(p, a, 1000003, n))
    raise ValueError(op)


def as_u32(x):
    return np.asarray(x, dtype=np.uint32)
