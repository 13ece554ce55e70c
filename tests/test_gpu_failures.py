"""Failure paths of the device pool, made on the host (a byte limit on the
context's pool; no device fault is involved).

* An operation whose scratch passes the limit fails with FPX_ENOMEM, returns
  every block it took, and the same context then computes correctly.
* The spectra-reusing block CRT product needs all block spectra at once; under
  a limit that refuses them it falls back to the per-pair path (the
  reference's own schedule, crt_convolution.hpp:132-205) before writing
  anything, and gives the same coefficients as the unlimited call.
"""
import numpy as np
import pytest

import fastpoly_b200 as F

pytestmark = pytest.mark.gpu

P, Q = 998244353, 1000000007


def _rnd(rng, p, n):
    return rng.integers(0, p, n, dtype=np.uint64).astype(np.uint32)


def test_pool_limit_enomem_then_usable(oracle):
    import torch

    rng = np.random.default_rng(5)
    ctx = F.Context(0, pool_limit_bytes=16 << 20)
    try:
        a, b = _rnd(rng, P, 3000), _rnd(rng, P, 5000)
        assert np.array_equal(ctx.conv(P, a, b), oracle.conv(P, a, b))
        held = ctx.pool_stats()["in_use_bytes"]
        big = _rnd(rng, P, 1 << 22)
        with pytest.raises(F.FpxError) as e:
            ctx.conv(P, big, big)  # host API: two 16 MiB uploads
        assert e.value.code == F.ENOMEM
        assert ctx.pool_stats()["in_use_bytes"] == held, "a failed call kept pool blocks"
        d = torch.from_numpy(big.view(np.int32)).cuda()
        out = torch.empty(2 * len(big) - 1, dtype=torch.int32, device="cuda")
        # device API: the 2^23-point plan (its twiddle tables stay with the
        # context) fits, the transform scratch does not
        with pytest.raises(F.FpxError) as e:
            ctx.conv_device(P, d, len(big), d, len(big), None, out)
        assert e.value.code == F.ENOMEM
        held = ctx.pool_stats()["in_use_bytes"]
        with pytest.raises(F.FpxError) as e:
            ctx.conv_device(P, d, len(big), d, len(big), None, out)
        assert e.value.code == F.ENOMEM
        assert ctx.pool_stats()["in_use_bytes"] == held, "a failed call kept pool blocks"
        # the same context, within the limit: correct
        for la, lb, p in [(3000, 5000, P), (20000, 30000, P), (5000, 7000, Q)]:
            a, b = _rnd(rng, p, la), _rnd(rng, p, lb)
            assert np.array_equal(ctx.conv(p, a, b), oracle.conv(p, a, b)), (la, lb, p)
        a[0] = 1
        assert np.array_equal(ctx.inv(Q, a, 9000), oracle.inv(Q, a, 9000))
    finally:
        ctx.close()


def test_blocked_crt_falls_back_to_pairs_under_limit(oracle):
    rng = np.random.default_rng(8)
    la = lb = 8 * 8192  # 8 x 8 blocks of 2^13 terms
    a, b = _rnd(rng, Q, la), _rnd(rng, Q, lb)
    want = oracle.conv(Q, a, b)

    # unlimited: the spectra-reusing path (16 block spectra of 2^14 points per prime)
    free = F.Context(0)
    try:
        free.set_crt_block(1 << 13)
        free.profile(True)
        assert np.array_equal(free.conv(Q, a, b), want)
        assert "spectral mac" in free.profile_report()
        free.profile(False)
        free.synchronize()
        plans = free.pool_stats()["in_use_bytes"]  # plans and tables held by the context
    finally:
        free.close()

    # a limit that fits the plans, the operands and one block pair's scratch
    # (about 0.4 MiB) but not 16 block spectra and three 2^17-word residue
    # buffers (about 2.6 MiB): the per-pair path runs instead
    io = 4 * (la + lb) + 4 * (1 << 17)
    ctx = F.Context(0, pool_limit_bytes=plans + io + (1 << 20) + (512 << 10))
    try:
        ctx.set_crt_block(1 << 13)
        ctx.profile(True)
        got = ctx.conv(Q, a, b)
        rep = ctx.profile_report()
        assert np.array_equal(got, want)
        assert "spectral mac" not in rep, "the blocked path ran under the limit"
        assert rep.get("garner", [0])[0] >= 64, rep  # one Garner pass per block pair
    finally:
        ctx.close()
