"""Column-pass tile shapes: every compiled shape gives the same values.

The tuner picks one shape per transform size by timing; whichever it picks,
the outputs must stay those of the default shape (which the parity tests pin to
the oracle).  Each candidate is forced in turn through fpx_col_shape_set and the
conv (two-operand forward pass, inverse pass), the square (one-operand forward
pass on zero-padded input) and the raw transform pair (one-operand forward pass
on full input, inverse pass with a scaled epilogue) are compared bit for bit.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import fastpoly_b200 as F

pytestmark = pytest.mark.gpu

P = 469762049  # 2^26 | p - 1: native transforms up to 2^26 points


@pytest.fixture(scope="module")
def ctx():
    return F.Context(0)


def _run_all(ctx, log_n, rng_seed):
    rng = np.random.default_rng(rng_seed)
    n = 1 << log_n
    a = rng.integers(0, P, n // 2, dtype=np.uint32)
    b = rng.integers(0, P, n // 2, dtype=np.uint32)
    x = rng.integers(0, P, n, dtype=np.uint32)
    c = ctx.conv(P, a, b)
    sq = ctx.conv(P, a, a)
    fx = ctx.ntt_forward(P, x)
    ix = ctx.ntt_inverse(P, fx)
    assert np.array_equal(ix, x)
    return c, sq, fx, ix


@pytest.mark.parametrize("log_n", [14, 16, 18, 20, 21, 22, 23, 24])
def test_every_shape_same_values(ctx, log_n):
    kinds = (F.COL_FWD1, F.COL_FWD2, F.COL_INV)
    cands = {k: ctx.col_shape_candidates(log_n, k) for k in kinds}
    assert all(len(v) >= 2 for v in cands.values())
    tuned = {k: ctx.col_shape(log_n, k) for k in kinds}
    for k in kinds:
        assert tuned[k] in cands[k]
    try:
        for k in kinds:
            ctx.set_col_shape(log_n, k, cands[k][0])
        ref = _run_all(ctx, log_n, log_n)
        for i in range(1, max(len(v) for v in cands.values())):
            for k in kinds:
                ctx.set_col_shape(log_n, k, cands[k][min(i, len(cands[k]) - 1)])
            got = _run_all(ctx, log_n, log_n)
            for name, r, g in zip(("conv", "square", "forward", "inverse"), ref, got):
                assert np.array_equal(r, g), (log_n, i, name)
    finally:
        for k in kinds:
            ctx.set_col_shape(log_n, k, tuned[k])


def test_raw_transform_round_trip(ctx):
    rng = np.random.default_rng(5)
    x = rng.integers(0, P, 1 << 23, dtype=np.uint32)
    assert np.array_equal(ctx.ntt_inverse(P, ctx.ntt_forward(P, x)), x)


def test_set_rejects_uncompiled_shape(ctx):
    with pytest.raises(F.FpxError):
        ctx.set_col_shape(23, F.COL_INV, (7, 1, 1))
    with pytest.raises(F.FpxError):
        ctx.col_shape_candidates(13, F.COL_INV)


_CHILD = r"""
import json, sys
import numpy as np
import fastpoly_b200 as F
ctx = F.Context(0)
a = np.arange(1 << 21, dtype=np.uint32)
ctx.conv(998244353, a, a[::-1].copy())
print(json.dumps([ctx.col_shape(22, k) for k in (0, 1, 2)]))
"""


def test_tuning_cache_file(tmp_path):
    path = tmp_path / "tune.txt"
    env = dict(os.environ, FPX_AUTOTUNE_CACHE=str(path))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    first = subprocess.run([sys.executable, "-c", _CHILD], env=env, cwd=root, capture_output=True, text=True,
                           timeout=600)
    assert first.returncode == 0, first.stderr
    lines = path.read_text().splitlines()
    assert len(lines) == 1 and "logN22" in lines[0]
    second = subprocess.run([sys.executable, "-c", _CHILD], env=env, cwd=root, capture_output=True, text=True,
                            timeout=600)
    assert second.returncode == 0, second.stderr
    assert json.loads(first.stdout.splitlines()[-1]) == json.loads(second.stdout.splitlines()[-1])
    assert len(path.read_text().splitlines()) == 1  # read back, not tuned again
    off = subprocess.run([sys.executable, "-c", _CHILD], env=dict(env, FPX_AUTOTUNE="0", FPX_AUTOTUNE_CACHE=""),
                         cwd=root, capture_output=True, text=True, timeout=600)
    assert off.returncode == 0, off.stderr
    defaults = json.loads(off.stdout.splitlines()[-1])
    assert all(s[0] == s[1] and s[2] == 0 for s in defaults)
