"""Bit-exact parity with the reference at the benchmark configurations' own sizes.

The expected values are the reference's outputs (oracle/_ref, compiled from the
unmodified headers) on the same seeded inputs, committed as checksums by
tests/golden/make_config_golden.py: FNV-1a-64 over the raw Montgomery limbs xor
the length, the reference bench's own checksum (bench/bench.cpp:152-159).
Every operation here runs through the public C ABI with host buffers.

  series_2e22   inv / log / exp / sqrt / pow(1000003) mod 998244353 at n = 2^22
  conv_large    conv 2^22 x 2^22 (native), 2^23 x 2^23 mod 998244353 and mod
                1e9+7 (three-prime CRT), 2^25 x 2^25 mod 1e9+7 (block pairs,
                through the spectra-reusing path and through the per-pair path)
  inv_crt_2e22  inv mod 1e9+7 at n = 2^22, a[0] = 1 and a[0] uniform
  batch_mix     all 4608 jobs of the batch mix in one fpx_batch_run, job by job
  serve_mix     300 requests of the serving mix through the request loop

Small CRT blocks (fpx_ctx_set_crt_block) run the block-pair loops on small
inputs; they are compared with the reference's crt_convolution<M, 64>
(crt_convolution.hpp:187-205, the block size its own tests use,
tests/test_prime_poly.cpp:110-121) and with the oracle.
"""
import json
import os

import numpy as np
import pytest

import fastpoly_b200 as F
from conftest import GOLDEN, rotl64

pytestmark = pytest.mark.gpu

P, Q = 998244353, 1000000007


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(GOLDEN, "config_checksums.json")) as f:
        return json.load(f)


def cs(O, p, v) -> str:
    return f"{O.checksum(p, v):016x}"


def job_cs(O, spec, res) -> str:
    if isinstance(res, Exception):
        return "domain_error" if isinstance(res, F.DomainError) else f"error {res}"
    if spec[0] == "divmod":
        return f"{O.checksum(spec[1], res[0]) ^ rotl64(O.checksum(spec[1], res[1]), 17):016x}"
    return cs(O, spec[1], res)


def test_series_2e22(fpx, oracle, golden):
    g = golden["series_2e22"]
    n = g["n"]
    (a,) = oracle.bench_rnd(P, g["seed"], n)
    a[0] = 1
    b = a.copy()
    b[0] = 0
    want = g["checksums"]
    assert cs(oracle, P, fpx.inv(P, a, n)) == want["inv"]
    assert cs(oracle, P, fpx.log(P, a, n)) == want["log"]
    assert cs(oracle, P, fpx.exp(P, b, n)) == want["exp"]
    assert cs(oracle, P, fpx.sqrt(P, fpx.conv(P, a, a, n), n)) == want["sqrt_of_square"]
    assert cs(oracle, P, fpx.pow(P, a, 1000003, n)) == want["pow_1000003"]
    assert cs(oracle, P, fpx.sqrt(P, a, n)) == want["sqrt_direct"]


@pytest.mark.parametrize("key", ["998244353:4194304", "998244353:8388608", "1000000007:8388608",
                                 "1000000007:33554432"])
def test_conv_large(fpx, oracle, golden, key, monkeypatch):
    p, la = (int(x) for x in key.split(":"))
    a, b = oracle.bench_rnd(p, 2 + la, la, la)
    want = golden["conv_large"]["checksums"][key]
    assert cs(oracle, p, fpx.conv(p, a, b)) == want
    if la > (1 << 23):
        # the reference's own schedule: every block pair reconstructed separately
        monkeypatch.setenv("FPX_CRT_BLOCKED", "0")
        assert cs(oracle, p, fpx.conv(p, a, b)) == want


def test_inv_crt_2e22(fpx, oracle, golden):
    g = golden["inv_crt_2e22"]
    n = g["n"]
    (a,) = oracle.bench_rnd(Q, g["seed"], n)
    a[0] = 1
    assert cs(oracle, Q, fpx.inv(Q, a, n)) == g["checksums"]["a0_1"]
    a[0] = g["a0_uniform"]
    assert cs(oracle, Q, fpx.inv(Q, a, n)) == g["checksums"]["a0_uniform"]


def test_batch_mix_every_job(fpx, oracle, golden):
    import bench

    g = golden["batch_mix"]
    specs = bench.batch_mix(g["seed"])
    assert bench.mix_digest(specs) == g["inputs_sha256"], "batch_mix generator changed: regenerate the fixture"
    got = fpx.batch(specs)
    bad = [i for i, (s, r) in enumerate(zip(specs, got)) if job_cs(oracle, s, r) != g["checksums"][i]]
    assert not bad, f"{len(bad)} of {len(specs)} jobs differ from the reference, first {bad[:5]}"


def test_serve_mix_every_request(oracle, golden):
    import bench

    g = golden["serve_mix"]
    specs = bench.serve_mix(g["count"], seed=g["seed"], max_log=g["max_log"])
    assert bench.mix_digest(specs) == g["inputs_sha256"], "serve_mix generator changed: regenerate the fixture"
    srv = F.Server(0)
    try:
        tickets = [srv.submit(s) for s in specs]
        got = [srv.poll(t)[0] for t in tickets]
    finally:
        srv.stop()
    bad = [i for i, (s, r) in enumerate(zip(specs, got)) if job_cs(oracle, s, r) != g["checksums"][i]]
    assert not bad, f"{len(bad)} of {len(specs)} requests differ from the reference, first {bad[:5]}"


@pytest.mark.parametrize("blocked", ["1", "0"])
def test_small_crt_blocks_match_reference(oracle, reference, blocked, monkeypatch):
    """2^13-term blocks: products of up to 5 x 4 block pairs through the
    spectra-reusing path (blocked = 1) and the per-pair path (0)."""
    monkeypatch.setenv("FPX_CRT_BLOCKED", blocked)
    ctx = F.Context(0)
    try:
        ctx.set_crt_block(1 << 13)
        rng = np.random.default_rng(99)
        for p, la, lb, n in [(Q, 40000, 30000, None), (Q, 3 * 8192, 2 * 8192 + 5, None), (Q, 20000, 20000, 25000),
                             (2147483647, 17000, 9000, None), (Q, 16385, 100, None)]:
            a = rng.integers(0, p, la, dtype=np.uint64).astype(np.uint32)
            b = rng.integers(0, p, lb, dtype=np.uint64).astype(np.uint32)
            got = ctx.conv(p, a, b, n)
            outn = la + lb - 1 if n is None else n
            want = reference.crt_convolution64(p, a, b, outn)
            assert np.array_equal(got, want[: len(got)]) and len(got) == outn, (p, la, lb, n)
            assert np.array_equal(got, oracle.conv(p, a, b, n)), (p, la, lb, n)
        a = rng.integers(0, Q, 30000, dtype=np.uint64).astype(np.uint32)
        assert np.array_equal(ctx.conv(Q, a, a), reference.crt_convolution64(Q, a, a, 59999))  # square
        with pytest.raises(F.FpxError):
            ctx.set_crt_block(3000)
        ctx.set_crt_block(0)  # back to 2^23
        assert np.array_equal(ctx.conv(Q, a, a), reference.crt_convolution64(Q, a, a, 59999))
    finally:
        ctx.close()
