"""Generates tests/golden/config_checksums.json: the reference's own outputs on
the workloads of the five benchmark configurations, at their full sizes, as
FNV-1a-64 checksums over raw Montgomery limbs xor size (the reference bench's
checksum, bench/bench.cpp:152-159).

Run where oracle/_ref is built (it compiles the unmodified reference headers;
``make -C oracle ref``).  The fixture is committed; the GPU tests compare the
CUDA path with it and never need the reference at run time.

Workloads (inputs are regenerated by the tests from the same seeds):
  series_2e22   mod 998244353, n = 2^22, the reference bench generator
                (std::mt19937_64, seed 3+n, a[0] = 1; bench/bench.cpp:350-373):
                inv, log, exp (b[0] = 0), sqrt of conv(a, a, n), pow k = 1000003,
                and sqrt of a itself (a[0] = 1 is a square)
  conv_large    conv 2^22 x 2^22 mod 998244353 (native 2^23 points),
                2^23 x 2^23 mod 998244353 and mod 1e9+7 (three-prime CRT),
                2^25 x 2^25 mod 1e9+7 (block pairs); seed 2+n (bench.cpp:216-220)
  inv_crt_2e22  inv mod 1e9+7, n = 2^22, seed 3+n with a[0] = 1 (the bench's
                input) and with a[0] uniform in [1, p)
  batch_mix     every job of the 4608-job batch mix (bench.batch_mix(seed=4))
  serve_mix     the first 300 requests of bench.serve_mix(seed=7, max_log=18)

Usage:  python tests/golden/make_config_golden.py [--skip-2e25]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "config_checksums.json")
P = 998244353
Q = 1000000007
SERVE_COUNT, SERVE_SEED, SERVE_MAX_LOG = 300, 7, 18


def rotl64(x: int, r: int) -> int:
    return ((x << r) | (x >> (64 - r))) & (2**64 - 1)


def job_checksum(O, spec, result) -> str:
    """Checksum of one job's result: the bench's checksum, divmod as q ^ rotl(r, 17)
    (bench/bench.cpp:255-264); a domain error is the string 'domain_error'."""
    if isinstance(result, Exception):
        return "domain_error"
    p = spec[1]
    if spec[0] == "divmod":
        q, r = result
        return f"{O.checksum(p, q) ^ rotl64(O.checksum(p, r), 17):016x}"
    return f"{O.checksum(p, result):016x}"


def ref_job(R, spec):
    from oracle.oracle import DomainError
    op, p = spec[0], spec[1]
    try:
        if op == "conv":
            return R.conv(p, spec[2], spec[3])
        if op == "divmod":
            return R.divmod(p, spec[2], spec[3])
        if op == "pow":
            return R.pow(p, spec[2], spec[3], spec[4])
        return getattr(R, op)(p, spec[2], spec[3])
    except DomainError as e:
        return e


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-2e25", action="store_true", help="leave out the 2^25 x 2^25 product (18 s)")
    args = ap.parse_args()
    from oracle.oracle import Oracle, Reference
    import bench

    O = Oracle()
    R = Reference.load()
    if R is None:
        raise SystemExit("oracle/_ref is not built (make -C oracle ref)")
    out = {"checksum": "FNV-1a-64 over raw Montgomery limbs xor length (bench/bench.cpp:152-159)",
           "reference_build": os.path.basename(R.path), "backend": R.backend}

    def timed(what, fn):
        t0 = time.perf_counter()
        r = fn()
        print(f"{what}: {time.perf_counter() - t0:.2f} s", flush=True)
        return r

    n = 1 << 22
    (a,) = O.bench_rnd(P, 3 + n, n)
    a[0] = 1
    b = a.copy()
    b[0] = 0
    series = {
        "inv": timed("inv", lambda: R.inv(P, a, n)),
        "log": timed("log", lambda: R.log(P, a, n)),
        "exp": timed("exp", lambda: R.exp(P, b, n)),
        "sqrt_of_square": timed("sqrt", lambda: R.sqrt(P, R.conv(P, a, a, n), n)),
        "pow_1000003": timed("pow", lambda: R.pow(P, a, 1000003, n)),
        "sqrt_direct": timed("sqrt direct", lambda: R.sqrt(P, a, n)),
    }
    out["series_2e22"] = {"p": P, "n": n, "seed": 3 + n,
                          "checksums": {k: f"{O.checksum(P, v):016x}" for k, v in series.items()}}

    conv = {}
    for p, la in [(P, 1 << 22), (P, 1 << 23), (Q, 1 << 23)] + ([] if args.skip_2e25 else [(Q, 1 << 25)]):
        x, y = O.bench_rnd(p, 2 + la, la, la)
        r = timed(f"conv {la} mod {p}", lambda: R.conv(p, x, y))
        conv[f"{p}:{la}"] = f"{O.checksum(p, r):016x}"
    out["conv_large"] = {"seed": "2+n", "checksums": conv}

    (c,) = O.bench_rnd(Q, 3 + n, n)
    c0 = int(c[0]) or 1
    c[0] = 1
    inv1 = timed("inv crt a0=1", lambda: R.inv(Q, c, n))
    c[0] = c0
    invu = timed("inv crt a0 uniform", lambda: R.inv(Q, c, n))
    out["inv_crt_2e22"] = {"p": Q, "n": n, "seed": 3 + n, "a0_uniform": c0,
                           "checksums": {"a0_1": f"{O.checksum(Q, inv1):016x}",
                                         "a0_uniform": f"{O.checksum(Q, invu):016x}"}}

    specs = bench.batch_mix()
    t0 = time.perf_counter()
    out["batch_mix"] = {"seed": 4, "jobs": len(specs), "inputs_sha256": bench.mix_digest(specs),
                        "checksums": [job_checksum(O, s, ref_job(R, s)) for s in specs]}
    print(f"batch mix: {time.perf_counter() - t0:.1f} s", flush=True)

    specs = bench.serve_mix(SERVE_COUNT, seed=SERVE_SEED, max_log=SERVE_MAX_LOG)
    t0 = time.perf_counter()
    out["serve_mix"] = {"seed": SERVE_SEED, "count": SERVE_COUNT, "max_log": SERVE_MAX_LOG,
                        "inputs_sha256": bench.mix_digest(specs),
                        "checksums": [job_checksum(O, s, ref_job(R, s)) for s in specs]}
    print(f"serve mix: {time.perf_counter() - t0:.1f} s", flush=True)

    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
