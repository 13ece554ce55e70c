"""The environment switches give the same values as the defaults.

FPX_PDL=0 (no programmatic dependent launch), FPX_GRAPHS=0 (no graph replay of
repeated Newton calls), FPX_AUTOTUNE=0 (default tile shapes) and
FPX_COL_FACTOR=0 (Bailey twiddles from three small tables per point instead of
column factors) and FPX_CRT_NEWTON=0 (32-term seeds and per-step CRT products
instead of the cluster CRT Newton kernels) change how the work is launched, never what
it computes: a child process with all of them off must print the same
checksums as one with the defaults.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

_CHILD = r"""
import json, hashlib
import numpy as np
import fastpoly_b200 as F
ctx = F.Context(0)
rng = np.random.default_rng(7)
out = {}
for p in (998244353, 1000000007):
    a = rng.integers(0, p, 70000, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, p, 50000, dtype=np.uint64).astype(np.uint32)
    a[0] = 1
    e = a.copy(); e[0] = 0
    res = {"conv": ctx.conv(p, a, b), "inv": ctx.inv(p, a, 90000), "log": ctx.log(p, a, 90000),
           "exp": ctx.exp(p, e, 90000)}
    for _ in range(2):  # repeats: graph capture and replay when enabled
        res["inv2"] = ctx.inv(p, a, 90000)
    big = rng.integers(0, p, 1 << 21, dtype=np.uint64).astype(np.uint32)
    res["big"] = ctx.conv(p, big, big[::-1].copy())
    for k, v in res.items():
        out[f"{p}:{k}"] = hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()
print(json.dumps(out))
"""


def _run(env):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _CHILD], env=env, cwd=root, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.splitlines()[-1])


def test_switches_same_values():
    base = dict(os.environ)
    default = _run(base)
    off = _run(dict(base, FPX_PDL="0", FPX_GRAPHS="0", FPX_AUTOTUNE="0", FPX_COL_FACTOR="0",
                    FPX_CRT_NEWTON="0"))
    assert default == off
    assert default["998244353:inv"] == default["998244353:inv2"]
