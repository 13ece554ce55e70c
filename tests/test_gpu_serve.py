"""The request loop (fpx_serve_*): every request gets the result the single call
gives it, whatever it was batched with; admission keeps micro-batches within
the HBM budget; stopping drains the queue."""
import threading

import numpy as np
import pytest

import fastpoly_b200 as F
from test_gpu_parity import eq, rnd
from test_gpu_batch import _check

pytestmark = pytest.mark.gpu


def _mix(rng, count, max_log=16):
    ops = ["conv", "inv", "exp", "sqrt", "divmod", "pow", "log"]
    mods = [998244353, 167772161, 1000000007, 2147483647]
    out = []
    for _ in range(count):
        op = ops[rng.integers(0, len(ops))]
        p = mods[rng.integers(0, len(mods))]
        n = int(2 ** rng.uniform(4, max_log))
        a = rnd(rng, p, n, nonzero0=True)
        if op == "conv":
            out.append(("conv", p, a, rnd(rng, p, int(2 ** rng.uniform(4, max_log)))))
        elif op == "divmod":
            b = rnd(rng, p, (n + 1) // 2)
            b[-1] = b[-1] or 1
            out.append(("divmod", p, a, b))
        elif op == "pow":
            out.append(("pow", p, a[: max(1, n // 4)], int(rng.integers(0, 2**63)), n))
        elif op == "exp":
            a[0] = 0
            out.append(("exp", p, a, n))
        elif op == "log":
            a[0] = 1
            out.append(("log", p, a, n))
        elif op == "sqrt":
            a[0] = 1
            out.append(("sqrt", p, a, n))
        else:
            out.append(("inv", p, a, n))
    return out


def _alone(fpx, spec):
    op, p = spec[0], spec[1]
    try:
        if op == "conv":
            return fpx.conv(p, spec[2], spec[3])
        if op == "divmod":
            return fpx.divmod(p, spec[2], spec[3])
        if op == "pow":
            return fpx.pow(p, spec[2], spec[3], spec[4])
        return getattr(fpx, op)(p, spec[2], spec[3])
    except F.DomainError as e:
        return e


def test_served_results_equal_single_calls(fpx):
    rng = np.random.default_rng(2025)
    specs = _mix(rng, 300)
    srv = F.Server(0)
    try:
        tickets = [srv.submit(s) for s in specs]
        got = [srv.poll(t) for t in tickets]
        st = srv.stats()
    finally:
        srv.stop()
    assert st["completed"] == len(specs) and st["batches"] >= 1
    for i, s in enumerate(specs):
        res, lat = got[i]
        assert lat > 0
        _check(res, _alone(fpx, s), f"request {i} {s[0]} p={s[1]}")


def test_admission_respects_budget(fpx):
    rng = np.random.default_rng(7)
    specs = _mix(rng, 120, max_log=14)
    budget = 4 << 20
    srv = F.Server(0, hbm_budget_bytes=budget, workers=1)
    big = ("conv", 998244353, rnd(rng, 998244353, 1 << 20), rnd(rng, 998244353, 1 << 20))
    try:
        assert srv.plan_bytes(big) > budget
        tickets = [srv.submit(s) for s in specs] + [srv.submit(big)]
        got = [srv.poll(t) for t in tickets]
        st = srv.stats()
    finally:
        srv.stop()
    assert st["oversize_requests"] >= 1
    assert st["batches"] > 1
    for i, s in enumerate(specs + [big]):
        _check(got[i][0], _alone(fpx, s), f"request {i} {s[0]}")


def test_concurrent_submitters(fpx):
    rng = np.random.default_rng(11)
    specs = _mix(rng, 160, max_log=13)
    srv = F.Server(0, workers=3)
    results = [None] * len(specs)

    def client(k):
        for i in range(k, len(specs), 4):
            t = srv.submit(specs[i])
            results[i] = srv.poll(t)[0]

    try:
        th = [threading.Thread(target=client, args=(k,)) for k in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    finally:
        srv.stop()
    for i, s in enumerate(specs):
        _check(results[i], _alone(fpx, s), f"request {i} {s[0]}")


def test_poll_nonblocking_and_errors(fpx):
    srv = F.Server(0)
    try:
        p = 998244353
        t_bad = srv.submit(("inv", p, [0, 1], 8))
        t_ok = srv.submit(("conv", p, [1, 2], [3, 4]))
        r = None
        while r is None:
            r = srv.poll(t_ok, wait=False)
        eq(r[0], [3, 10, 8], "served conv")
        bad = srv.poll(t_bad)[0]
        assert isinstance(bad, F.DomainError)
    finally:
        srv.stop()


def test_stop_drains_queue():
    rng = np.random.default_rng(3)
    specs = _mix(rng, 60, max_log=12)
    srv = F.Server(0, workers=1)
    tickets = [srv.submit(s) for s in specs]
    live = dict(srv._live)
    srv.stop()
    for t in tickets:
        j = live[t][0]
        assert j.status in (F.OK, F.EDOMAIN)
