"""CUDA graphs of single Newton operations.

The second call of inv / log / exp with the same (prime, sizes, device
pointers) captures the operation into a graph; later calls replay it.  Each
call here gets new input values in the same buffers, so a replay that did not
re-read its inputs, or wrote through stale scratch, would differ from the
oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rnd(rng, p, n):
    return rng.integers(0, p, n, dtype=np.uint64).astype(np.uint32)


@pytest.mark.parametrize("p", [998244353, 167772161])
@pytest.mark.parametrize("n", [300, 9000, 70000])
def test_repeated_calls_replay(fpx, oracle, p, n):
    import torch
    rng = np.random.default_rng(n + p % 97)
    la = n + 17
    da = torch.zeros(la, dtype=torch.int32, device="cuda")
    out = torch.zeros(n, dtype=torch.int32, device="cuda")
    for op in ("inv", "log", "exp"):
        fn = getattr(fpx, op + "_device")
        ref = getattr(oracle, op)
        for call in range(4):  # direct, capture + replay, replay, replay
            a = rnd(rng, p, la)
            a[0] = {"inv": a[0] or 1, "log": 1, "exp": 0}[op]
            torch.cuda.synchronize()
            da.copy_(torch.from_numpy(a.view(np.int32)))
            torch.cuda.synchronize()
            before = fpx.launch_count()
            fn(p, da, la, n, out)
            fpx.synchronize()
            launched = fpx.launch_count() - before
            got = out.cpu().numpy().view(np.uint32)
            assert np.array_equal(got, ref(p, a, n)), (op, n, call)
            # the first call may also build tables (1/i for log / exp); the
            # capture (second call) and the replays count the same kernels
            if call == 1:
                second = launched
            elif call > 1:
                assert launched == second, (op, call, launched, second)


def test_release_pool_drops_graphs(fpx, oracle):
    import torch
    p, n = 998244353, 20000
    rng = np.random.default_rng(3)
    da = torch.zeros(n, dtype=torch.int32, device="cuda")
    out = torch.zeros(n, dtype=torch.int32, device="cuda")
    for call in range(5):
        a = rnd(rng, p, n)
        a[0] = a[0] or 1
        torch.cuda.synchronize()
        da.copy_(torch.from_numpy(a.view(np.int32)))
        torch.cuda.synchronize()
        fpx.inv_device(p, da, n, n, out)
        fpx.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32), oracle.inv(p, a, n)), call
        if call == 2:
            fpx.release_pool()


def test_host_api_repeats(fpx, oracle):
    p = 998244353
    rng = np.random.default_rng(11)
    for call in range(4):
        a = rnd(rng, p, 5000)
        a[0] = 1
        assert np.array_equal(fpx.log(p, a, 6000), oracle.log(p, a, 6000)), call
        b = a.copy()
        b[0] = 0
        assert np.array_equal(fpx.exp(p, b, 6000), oracle.exp(p, b, 6000)), call


def test_domain_error_not_captured(fpx):
    import fastpoly_b200 as F
    import torch
    p, n = 998244353, 4096
    da = torch.zeros(n, dtype=torch.int32, device="cuda")
    out = torch.zeros(n, dtype=torch.int32, device="cuda")
    for _ in range(3):
        with pytest.raises(F.FpxError):
            fpx.inv_device(p, da, n, n, out)  # constant term 0: checked before any capture
