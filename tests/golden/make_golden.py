"""Generates the golden fixtures in this directory (run in a container that has
the reference checkout; the fixtures are committed, the reference is not needed
afterwards).

published_checksums.json
    Checksums the reference publishes in its own bench CSV files
    (FNV-1a-64 over raw Montgomery limbs, xor size; bench/bench.cpp:152-159)
    for the operations on the NTT path, keyed by modulus, operation and size.
    Inputs are the reference bench generator's (std::mt19937_64, seeds
    1+n / 2+n / 3+n / 4+n; bench/bench.cpp:216-373).

reference_vectors.json
    Outputs of the reference itself (oracle/_ref, compiled from the unmodified
    headers) on small seeded inputs over many moduli, including the edge cases
    its tests cover: empty operands, truncation, short operands at the 40-term
    cut-over, valuations, non-residues, degree-dropping divisions.

Usage:  python tests/golden/make_golden.py [--reference <checkout>]
        (default: the FPX_REFERENCE environment variable)
"""
from __future__ import annotations

import argparse
import csv
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OPS = {"conv", "conv-trunc", "square", "inv", "log", "exp", "sqrt", "pow", "divmod",
       "ntt-forward", "ntt-inverse"}
# file -> modulus (None: the file has a modulus column)
FILES = {
    "performance-20261003.csv": 998244353,
    "performance-20261010-avx-lazy.csv": 998244353,
    "performance-20261011-neon.csv": 998244353,
    "performance-20261011-large.csv": 998244353,
    "performance-20261011-crt.csv": 1000000007,
    "performance-20261009-moduli.csv": None,
    "performance-20261010-avx-lazy-moduli.csv": None,
}


def published(ref_root: str):
    rows = {}
    for fname, mod in FILES.items():
        path = os.path.join(ref_root, "bench", fname)
        with open(path) as f:
            for lineno, row in enumerate(csv.DictReader(f), start=2):
                op = row.get("operation")
                if op not in OPS:
                    continue
                p = int(row["modulus"]) if mod is None else mod
                n = int(row["size"])
                key = (p, op, n)
                cs = row["checksum"].lower()
                src = f"bench/{fname}:{lineno}"
                if key in rows:
                    if rows[key]["checksum"] != cs:
                        raise SystemExit(f"conflicting published checksum for {key}: {src}")
                    continue
                rows[key] = {"p": p, "op": op, "n": n, "checksum": cs, "source": src}
    return sorted(rows.values(), key=lambda r: (r["p"], r["op"], r["n"]))


def splitmix64(seed: int, count: int):
    out, x = [], seed & (2**64 - 1)
    for _ in range(count):
        x = (x + 0x9E3779B97F4A7C15) & (2**64 - 1)
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
        out.append(z ^ (z >> 31))
    return out


def rand_poly(p: int, n: int, seed: int):
    return [int(v % p) for v in splitmix64(seed, n)]


def reference_vectors():
    from oracle.oracle import Reference, DomainError

    R = Reference.load()
    if R is None:
        raise SystemExit("oracle/_ref is not built (make -C oracle ref)")
    cases = []

    def add(op, p, args, fn):
        try:
            out = fn()
            rec = {"op": op, "p": p, **args, "status": "ok"}
            if isinstance(out, tuple):
                rec["q"], rec["r"] = [int(x) for x in out[0]], [int(x) for x in out[1]]
            else:
                rec["out"] = [int(x) for x in out]
        except DomainError:
            rec = {"op": op, "p": p, **args, "status": "domain_error"}
        cases.append(rec)

    moduli = [998244353, 167772161, 469762049, 754974721, 1000000007, 2147483647,
              1224736769, 2, 3, 17, 97, 193, 641, 100003]
    seed = 1
    for p in moduli:
        for la, lb, n in [(0, 5, None), (1, 1, None), (40, 90, None), (41, 41, None), (63, 65, 70),
                          (129, 142, None), (257, 259, 300), (7, 300, 0), (5, 9, 3)]:
            a, b = rand_poly(p, la, seed), rand_poly(p, lb, seed + 1)
            seed += 2
            add("conv", p, {"a": a, "b": b, "n": n}, lambda: R.conv(p, a, b, n))
        for n in (1, 2, 9, 31, 33, 65, 130, 257):
            a = rand_poly(p, n + 3, seed); seed += 1
            a[0] = a[0] or 1
            add("inv", p, {"a": a, "n": n}, lambda: R.inv(p, a, n))
            if n <= p:
                la = list(a); la[0] = 1
                add("log", p, {"a": la, "n": n}, lambda: R.log(p, la, n))
            if n - 1 < p:
                ea = list(a); ea[0] = 0
                add("exp", p, {"a": ea, "n": n}, lambda: R.exp(p, ea, n))
            sq = R.conv(p, a, a, n)
            add("sqrt", p, {"a": [int(x) for x in sq], "n": n}, lambda: R.sqrt(p, sq, n))
            for k in (0, 1, 2, 65, 1000003, 2**64 - 1):
                add("pow", p, {"a": a[: 1 + n // 3], "k": k, "n": n}, lambda: R.pow(p, a[: 1 + n // 3], k, n))
        # valuation / edge inputs
        add("sqrt", p, {"a": [0, 0, 4 % p, 1, 2], "n": 9}, lambda: R.sqrt(p, [0, 0, 4 % p, 1, 2], 9))
        add("sqrt", p, {"a": [0, 4 % p], "n": 5}, lambda: R.sqrt(p, [0, 4 % p], 5))
        add("pow", p, {"a": [0, 0, 1], "k": 10, "n": 5}, lambda: R.pow(p, [0, 0, 1], 10, 5))
        add("inv", p, {"a": [0, 1], "n": 8}, lambda: R.inv(p, [0, 1], 8))
        for la, lb in [(3, 5), (40, 17), (120, 50), (300, 120), (64, 1)]:
            a, b = rand_poly(p, la, seed), rand_poly(p, lb, seed + 1)
            seed += 2
            if b and b[-1] == 0:
                b[-1] = 1
            add("divmod", p, {"a": a, "b": b}, lambda: R.divmod(p, a, b))
    return cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("FPX_REFERENCE"))
    args = ap.parse_args()
    if not args.reference:
        raise SystemExit("name the reference checkout: --reference <dir> or FPX_REFERENCE")
    pub = published(args.reference)
    with open(os.path.join(HERE, "published_checksums.json"), "w") as f:
        json.dump(pub, f, indent=0)
    vecs = reference_vectors()
    with open(os.path.join(HERE, "reference_vectors.json"), "w") as f:
        json.dump(vecs, f, separators=(",", ":"))
    print(f"{len(pub)} published checksums, {len(vecs)} reference vectors")


if __name__ == "__main__":
    main()
