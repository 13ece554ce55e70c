"""The request loop (fpx_serve_*): every request gets the result the single call
and the oracle give it, whatever it was batched with; admission keeps all
micro-batches on the GPU within one device-wide HBM budget; short requests are
not held behind long ones; stopping drains the queue."""
import time
import threading

import numpy as np
import pytest

import fastpoly_b200 as F
from test_gpu_parity import eq, rnd
from test_gpu_batch import _check, _oracle_job

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


def test_served_results_equal_single_calls(fpx, oracle):
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
        _check(res, _oracle_job(oracle, s), f"request {i} {s[0]} p={s[1]} vs oracle")


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


def test_small_requests_not_held_behind_a_large_one(oracle):
    """A 2^22-term inverse modulo 1e9+7 (three-prime CRT Newton steps, a few ms)
    submitted first, then 40 short products: every short one completes before
    the long one, and all results are exact."""
    rng = np.random.default_rng(17)
    q = 1000000007
    big = rnd(rng, q, 1 << 22, nonzero0=True)
    smalls = [("conv", 998244353, rnd(rng, 998244353, 700), rnd(rng, 998244353, 900)) for _ in range(40)]
    srv = F.Server(0)
    try:
        t_big = time.perf_counter()
        tb = srv.submit(("inv", q, big, 1 << 22))
        subs = []
        for s in smalls:
            subs.append((time.perf_counter(), srv.submit(s)))
        done_small = []
        for t0, t in subs:
            r, lat = srv.poll(t)
            done_small.append(t0 + lat)
        rb, lat_b = srv.poll(tb)
    finally:
        srv.stop()
    done_big = t_big + lat_b
    assert max(done_small) < done_big, (max(done_small) - t_big, lat_b)
    want = oracle.inv(q, big[:4096], 4096)
    eq(rb[:4096], want, "served big inverse (first 4096 terms)")


def test_device_wide_budget(oracle):
    """Three workers share one 48 MiB budget: the planned bytes of everything on
    the GPU at once never exceed it, and every result is exact."""
    rng = np.random.default_rng(23)
    p = 998244353
    specs = [("conv", p, rnd(rng, p, 1 << 17), rnd(rng, p, 1 << 17)) for _ in range(12)]
    specs += [("conv", p, rnd(rng, p, 3000), rnd(rng, p, 2000)) for _ in range(30)]
    specs += [("inv", p, rnd(rng, p, 1 << 18, nonzero0=True), 1 << 18) for _ in range(4)]
    budget = 48 << 20
    srv = F.Server(0, hbm_budget_bytes=budget, workers=3)
    try:
        assert all(srv.plan_bytes(s) <= budget for s in specs)
        tickets = [srv.submit(s) for s in specs]
        got = [srv.poll(t)[0] for t in tickets]
        st = srv.stats()
    finally:
        srv.stop()
    assert st["oversize_requests"] == 0
    assert 0 < st["max_in_flight_bytes"] <= budget, st
    for i, s in enumerate(specs):
        _check(got[i], _oracle_job(oracle, s), f"request {i} {s[0]}")
