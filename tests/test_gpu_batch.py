"""Parity of the batched path (fpx_batch_run / fpx_batch_submit) against the
oracle and against the single-operation calls.

A batch must give every job exactly the result, length and error the
single-job function gives it, whatever else is in the batch: mixed moduli
(native primes, CRT-only moduli, p = 2), mixed sizes (direct products, one-CTA
and two-pass transforms), mixed operations, failing jobs next to good ones."""
import ctypes as C

import numpy as np
import pytest

import fastpoly_b200 as F
from test_gpu_parity import eq, rnd
from oracle.oracle import DomainError as OracleDomainError

pytestmark = pytest.mark.gpu

MODULI = [998244353, 167772161, 754974721, 1000000007, 2147483647, 7340033, 97, 2]


def _oracle_job(O, jb):
    op, p = jb[0], jb[1]
    try:
        if op == "conv":
            return O.conv(p, jb[2], jb[3], None if len(jb) < 5 else jb[4])
        if op == "pow":
            return O.pow(p, jb[2], jb[3], jb[4])
        if op == "divmod":
            return O.divmod(p, jb[2], jb[3])
        return getattr(O, op)(p, jb[2], jb[3])
    except OracleDomainError as e:
        return e


def _check(res, want, what):
    if isinstance(want, Exception):
        assert isinstance(res, F.DomainError), (what, res)
    elif isinstance(want, tuple):
        assert not isinstance(res, Exception), (what, res)
        eq(res[0], want[0], what + " q")
        eq(res[1], want[1], what + " r")
    else:
        assert not isinstance(res, Exception), (what, res)
        eq(res, want, what)


def _conv_jobs(rng):
    jobs = []
    for p in MODULI:
        for la, lb, n in [(1, 1, None), (3, 50, None), (40, 41, None), (41, 41, None), (100, 300, None),
                          (1000, 1000, 1500), (3000, 5000, None), (4097, 4096, None), (20000, 30000, None),
                          (70000, 1 << 16, 100000)]:
            jobs.append(("conv", p, rnd(rng, p, la), rnd(rng, p, lb), n))
    a = rnd(rng, 998244353, 5000)
    jobs.append(("conv", 998244353, a, a, None))   # square
    jobs.append(("conv", 998244353, a, a, 7))      # square, truncated
    jobs.append(("conv", 1000000007, a, a, None))  # CRT square
    jobs.append(("conv", 998244353, a, [], None))  # empty operand
    jobs.append(("conv", 998244353, a, a, 0))      # n = 0
    return jobs


def test_batch_conv_mixed(fpx, oracle):
    rng = np.random.default_rng(41)
    jobs = _conv_jobs(rng)
    res = fpx.batch(jobs)
    for i, jb in enumerate(jobs):
        _check(res[i], _oracle_job(oracle, jb), f"job {i} conv p={jb[1]} {len(jb[2])}x{len(jb[3])}")


SERIES_N = [1, 2, 5, 31, 32, 33, 64, 100, 1000, 4096, 5000, 8193, 20000, 65536 + 3]


@pytest.mark.parametrize("op", ["inv", "log", "exp"])
def test_batch_series_mixed(fpx, oracle, op):
    rng = np.random.default_rng({"inv": 1, "log": 2, "exp": 3}[op])
    jobs = []
    for p in [998244353, 167772161, 754974721, 1000000007, 7340033, 97]:
        for n in SERIES_N:
            if op == "log" and n > p:
                continue
            if op == "exp" and n - 1 >= p:
                continue
            for la in (1, 3, n + 7):
                a = rnd(rng, p, la, nonzero0=True)
                if op == "log":
                    a[0] = 1
                if op == "exp":
                    a[0] = 0
                jobs.append((op, p, a, n))
    res = fpx.batch(jobs)
    for i, jb in enumerate(jobs):
        _check(res[i], _oracle_job(oracle, jb), f"job {i} {op} p={jb[1]} n={jb[3]} la={len(jb[2])}")


def test_batch_everything_and_errors(fpx, oracle):
    """All operations in one batch, with failing jobs among them."""
    rng = np.random.default_rng(7)
    p = 998244353
    jobs = []
    for q in (998244353, 1000000007, 97):
        a = rnd(rng, q, 3000, nonzero0=True)
        b = rnd(rng, q, 1200)
        b[-1] = b[-1] or 1
        sq = oracle.conv(q, a, a, 2000)
        e0 = a.copy(); e0[0] = 0
        l1 = a.copy(); l1[0] = 1
        jobs += [("conv", q, a, b), ("inv", q, a, 2500), ("exp", q, e0, 90 if q == 97 else 2500),
                 ("log", q, l1, 97 if q == 97 else 2600), ("sqrt", q, sq, 2000), ("pow", q, a[:500], 1000003, 2200),
                 ("pow", q, a[:500], 3, 2200), ("divmod", q, a, b)]
    jobs += [("inv", p, [0, 1, 2], 10), ("log", p, [2, 1], 5), ("exp", p, [1, 1], 5), ("sqrt", p, [0, 4], 5),
             ("divmod", p, [1, 2], [0, 0]), ("log", 3, [1, 1], 4), ("exp", 3, [0, 1], 4), ("inv", p, [], 4)]
    res = fpx.batch(jobs)
    for i, jb in enumerate(jobs):
        _check(res[i], _oracle_job(oracle, jb), f"job {i} {jb[0]} p={jb[1]}")


def test_batch_matches_single_calls(fpx):
    """Same result alone as in the mix (the serving contract)."""
    rng = np.random.default_rng(99)
    jobs = []
    for p in (998244353, 1000000007, 167772161, 2147483647):
        for n in (300, 5000, 40000):
            a = rnd(rng, p, n, nonzero0=True)
            b = rnd(rng, p, n // 2 + 1)
            b[-1] = b[-1] or 1
            e0 = a.copy(); e0[0] = 0
            l1 = a.copy(); l1[0] = 1
            jobs += [("conv", p, a, b), ("inv", p, a, n), ("exp", p, e0, n), ("log", p, l1, n), ("divmod", p, a, b)]
    res = fpx.batch(jobs)
    for i, jb in enumerate(jobs):
        op, p = jb[0], jb[1]
        if op == "conv":
            alone = fpx.conv(p, jb[2], jb[3])
        elif op == "divmod":
            alone = fpx.divmod(p, jb[2], jb[3])
        else:
            alone = getattr(fpx, op)(p, jb[2], jb[3])
        _check(res[i], alone, f"job {i} {op} p={p}")


def test_batch_reference_vectors(fpx, ref_vectors):
    """All 1332 reference vectors as one batch."""
    jobs, want = [], []
    for case in ref_vectors:
        p, op = case["p"], case["op"]
        if op == "conv":
            jobs.append(("conv", p, case["a"], case["b"], case["n"]))
        elif op == "pow":
            jobs.append(("pow", p, case["a"], case["k"], case["n"]))
        elif op == "divmod":
            jobs.append(("divmod", p, case["a"], case["b"]))
        else:
            jobs.append((op, p, case["a"], case["n"]))
        if case["status"] == "domain_error":
            want.append(OracleDomainError(1, op))
        elif op == "divmod":
            want.append((np.asarray(case["q"], np.uint32), np.asarray(case["r"], np.uint32)))
        else:
            want.append(np.asarray(case["out"], np.uint32))
    res = fpx.batch(jobs)
    for i in range(len(jobs)):
        _check(res[i], want[i], f"vector {i} {jobs[i][0]} p={jobs[i][1]}")


def test_batch_montgomery(fpx, oracle):
    rng = np.random.default_rng(5)
    jobs, want = [], []
    for p in (998244353, 1000000007, 2):
        a, b = rnd(rng, p, 3000, nonzero0=True), rnd(rng, p, 2000)
        ma = np.array([oracle.to_mont(p, int(x)) for x in a], np.uint32)
        mb = np.array([oracle.to_mont(p, int(x)) for x in b], np.uint32)
        jobs += [("conv", p, ma, mb), ("inv", p, ma, 4000)]
        want += [oracle.conv(p, a, b), oracle.inv(p, a, 4000)]
    res = fpx.batch(jobs, repr=F.MONTGOMERY)
    for i, w in enumerate(want):
        p = jobs[i][1]
        eq(res[i], np.array([oracle.to_mont(p, int(x)) for x in w], np.uint32), f"mont job {i}")


def test_batch_device_submit(fpx, oracle):
    import torch
    rng = np.random.default_rng(8)
    p = 998244353
    specs = [(OP, n) for OP in (F.OP_CONV, F.OP_INV, F.OP_EXP) for n in (100, 3000, 50000)]
    jobs = (F.Job * len(specs))()
    keep, host = [], []
    for i, (op, n) in enumerate(specs):
        a = rnd(rng, p, n, nonzero0=True)
        if op == F.OP_EXP:
            a[0] = 0
        b = rnd(rng, p, n // 3 + 1)
        da = torch.from_numpy(a.view(np.int32)).cuda()
        db = torch.from_numpy(b.view(np.int32)).cuda()
        cap = n + b.size - 1 if op == F.OP_CONV else n
        do = torch.empty(cap, dtype=torch.int32, device="cuda")
        keep += [da, db, do]
        j = jobs[i]
        j.op, j.p, j.a, j.la, j.n, j.out = op, p, da.data_ptr(), n, n if op != F.OP_CONV else F.SIZE_MAX, do.data_ptr()
        if op == F.OP_CONV:
            j.b, j.lb = db.data_ptr(), b.size
        host.append((op, a, b, do))
    torch.cuda.synchronize()
    assert fpx.batch_submit(jobs) == F.OK
    fpx.batch_wait()
    for i, (op, a, b, do) in enumerate(host):
        got = do.cpu().numpy().view(np.uint32)[: jobs[i].out_len]
        if op == F.OP_CONV:
            want = oracle.conv(p, a, b)
        elif op == F.OP_INV:
            want = oracle.inv(p, a, a.size)
        else:
            want = oracle.exp(p, a, a.size)
        eq(got, want, f"device job {i}")


def test_batch_empty_and_invalid(fpx):
    assert fpx.batch([]) == []
    res = fpx.batch([("conv", 4, [1], [1]), ("inv", 998244353, [1, 2], 3)])
    assert isinstance(res[0], F.FpxError) and res[0].code == F.EINVAL
    eq(res[1], [1, 998244351, 4], "inv next to an invalid job")


def test_batch_launch_sharing(fpx):
    """512 inverses of mixed sizes share launches: far fewer than one set per job."""
    rng = np.random.default_rng(12)
    p = 998244353
    jobs = [("inv", p, rnd(rng, p, int(n), nonzero0=True), int(n))
            for n in np.exp2(rng.uniform(8, 14, 512)).astype(int)]
    fpx.batch(jobs[:4])
    before = fpx.launch_count()
    fpx.batch(jobs)
    used = fpx.launch_count() - before
    assert used < 200, used


def test_batch_more_cluster_jobs_than_one_launch(fpx, oracle):
    """Inverse jobs of at most 2^13 terms modulo a prime without the roots run
    as one three-CTA cluster each; more of them than one launch takes (65535
    clusters) go out in several launches."""
    p = 1000000007
    rng = np.random.default_rng(65)
    polys = [rnd(rng, p, 6, nonzero0=True) for _ in range(16)]
    want = [oracle.inv(p, a, 5) for a in polys]
    count = 65535 + 37
    got = fpx.batch([("inv", p, polys[i % 16], 5) for i in range(count)])
    for i in range(count):
        assert not isinstance(got[i], Exception), (i, got[i])
        if not np.array_equal(got[i], want[i % 16]):
            raise AssertionError(f"job {i} differs")


def test_batch_smaller_arena_takes_cached_block(oracle):
    """A batch whose scratch arena is smaller than the previous one's reuses
    memory the pool already holds (no new device allocation), with the same
    results."""
    import torch
    ctx = F.Context(0)
    try:
        p, n = 998244353, 1 << 19
        rng = np.random.default_rng(66)
        count = 64

        def jobs_of(bufs):
            jobs = (F.Job * len(bufs))()
            for j, (da, db, do) in zip(jobs, bufs):
                j.op, j.p, j.a, j.la, j.b, j.lb = F.OP_CONV, p, da.data_ptr(), da.numel(), db.data_ptr(), db.numel()
                j.n, j.out = F.SIZE_MAX, do.data_ptr()
            return jobs

        def run(jobs):
            assert ctx.batch_submit(jobs) == F.OK
            ctx.batch_wait()

        host = [(rnd(rng, p, n), rnd(rng, p, n)) for _ in range(count)]
        big = [(torch.from_numpy(a.view(np.int32)).cuda(), torch.from_numpy(b.view(np.int32)).cuda(),
                torch.empty(2 * n - 1, dtype=torch.int32, device="cuda")) for a, b in host]
        tiny = [(x[:100], y[:100], o[:199]) for x, y, o in big]
        for _ in range(6):  # descriptor ring slots sized for `count` jobs
            run(jobs_of(tiny))
        run(jobs_of(big))
        first = [o.clone() for _, _, o in big]
        for _, _, o in big:
            o.zero_()
        before = ctx.pool_stats()["system_allocations"]
        run(jobs_of(big[: count // 3]))
        assert ctx.pool_stats()["system_allocations"] == before
        for i in range(count // 3):
            assert torch.equal(big[i][2], first[i]), i
        for i in (0, count // 3 - 1):
            eq(first[i].cpu().numpy().view(np.uint32), oracle.conv(p, *host[i]), f"job {i}")
    finally:
        ctx.close()


def _derived_jobs(rng):
    """sqrt / pow / divmod jobs covering every host decision of the phased path."""
    jobs = []
    for p in (998244353, 1000000007, 167772161, 2147483647):
        a = rnd(rng, p, 3000, nonzero0=True)
        z = np.concatenate([np.zeros(6, np.uint32), a[:2000]])        # valuation 6
        tz = np.concatenate([a[:700], np.zeros(300, np.uint32)])      # trailing zeros
        sq = (rnd(rng, p, 1, nonzero0=True).astype(np.uint64) ** 2 % p).astype(np.uint32)
        root_in = np.concatenate([sq, a[1:1500]])                     # a square constant term
        jobs += [("sqrt", p, root_in, 1500), ("sqrt", p, np.concatenate([np.zeros(4, np.uint32), root_in]), 1800),
                 ("sqrt", p, root_in[:40], 70000),                    # longer than the phased limit: single path
                 ("pow", p, a[:800], (1 << 64) - 1, 2500), ("pow", p, z, 1000003, 2500), ("pow", p, tz, 999999, 2100),
                 ("pow", p, a[:300], p * 5, 900),                      # k = 0 mod p
                 ("pow", p, a[:300], 17, 900), ("pow", p, z, 10 ** 6, 30),   # binary powering; all-zero window
                 ("divmod", p, a, a[:1200]), ("divmod", p, tz, np.concatenate([a[:90], np.zeros(5, np.uint32)])),
                 ("divmod", p, a[:50], a[:400]), ("divmod", p, a, a[:1])]
    return jobs


def test_batch_sqrt_pow_divmod_phased(fpx, oracle):
    """sqrt, pow and divmod jobs run as phases of batched log / exp / inverse /
    product calls: the oracle's results, from host buffers in both limb forms."""
    rng = np.random.default_rng(71)
    jobs = _derived_jobs(rng)
    res = fpx.batch(jobs)
    for i, jb in enumerate(jobs):
        _check(res[i], _oracle_job(oracle, jb), f"job {i} {jb[0]} p={jb[1]} len={len(jb[2])}")
    # Montgomery limbs: the host decisions read converted words
    sub = [jb for jb in jobs if jb[1] in (998244353, 1000000007)]
    mj = []
    for jb in sub:
        p = jb[1]
        m = lambda x: np.array([oracle.to_mont(p, int(v)) for v in x], np.uint32)
        mj.append((jb[0], p, m(jb[2])) + ((m(jb[3]),) if jb[0] == "divmod" else jb[3:]))
    mres = fpx.batch(mj, repr=F.MONTGOMERY)
    for i, jb in enumerate(sub):
        want = _oracle_job(oracle, jb)
        p = jb[1]
        m = lambda x: np.array([oracle.to_mont(p, int(v)) for v in x], np.uint32)
        if isinstance(want, tuple):
            want = (m(want[0]), m(want[1]))
        elif not isinstance(want, Exception):
            want = m(want)
        _check(mres[i], want, f"mont job {i} {jb[0]} p={p}")


def test_batch_sqrt_pow_divmod_device_pointers(fpx, oracle):
    """The same jobs through fpx_batch_submit (the host decisions read the device)."""
    import torch
    rng = np.random.default_rng(72)
    specs = [jb for jb in _derived_jobs(rng) if jb[1] in (998244353, 2147483647)]
    jobs = (F.Job * len(specs))()
    keep = []
    for j, jb in zip(jobs, specs):
        op, p, a = jb[0], jb[1], np.asarray(jb[2], np.uint32)
        da = torch.from_numpy(a.view(np.int32).copy()).cuda()
        keep.append(da)
        j.op, j.p, j.a, j.la = F._OPS[op], p, da.data_ptr(), a.size
        if op == "divmod":
            b = np.asarray(jb[3], np.uint32)
            db = torch.from_numpy(b.view(np.int32).copy()).cuda()
            q, r = torch.zeros(a.size, dtype=torch.int32, device="cuda"), torch.zeros(b.size, dtype=torch.int32, device="cuda")
            keep += [db, q, r]
            j.b, j.lb, j.out, j.out2 = db.data_ptr(), b.size, q.data_ptr(), r.data_ptr()
        else:
            n = jb[-1]
            o = torch.zeros(n, dtype=torch.int32, device="cuda")
            keep.append(o)
            j.n, j.out = n, o.data_ptr()
            if op == "pow":
                j.k = jb[3]
    torch.cuda.synchronize()
    fpx.batch_submit(jobs)
    fpx.batch_wait()
    for i, jb in enumerate(specs):
        want = _oracle_job(oracle, jb)
        j = jobs[i]
        if isinstance(want, Exception):
            assert j.status == F.EDOMAIN, (i, jb[0])
            continue
        assert j.status == F.OK, (i, jb[0], j.status)
        if jb[0] == "divmod":
            q = keep[[k for k, t in enumerate(keep) if t.data_ptr() == j.out][0]]
            r = keep[[k for k, t in enumerate(keep) if t.data_ptr() == j.out2][0]]
            eq(q.cpu().numpy().view(np.uint32)[: j.out_len], want[0], f"device job {i} q")
            eq(r.cpu().numpy().view(np.uint32)[: j.out2_len], want[1], f"device job {i} r")
        else:
            o = keep[[k for k, t in enumerate(keep) if t.data_ptr() == j.out][0]]
            eq(o.cpu().numpy().view(np.uint32)[: j.out_len], want, f"device job {i} {jb[0]}")


def test_batch_output_buffers_not_reused_while_held(fpx, oracle):
    """Large batches return views into page-locked output buffers the context
    keeps: a later call never writes into a buffer whose results are still
    held, and hands a buffer out again once they are dropped."""
    rng = np.random.default_rng(81)
    p = 998244353

    def mix(seed):
        r = np.random.default_rng(seed)
        return [("conv", p, rnd(r, p, 1 << 17), rnd(r, p, 1 << 17)) for _ in range(8)]  # 2^21 output words

    jobs1, jobs2, jobs3 = mix(1), mix(2), mix(3)
    r1 = fpx.batch(jobs1)
    keep1 = [x.copy() for x in r1]
    r2 = fpx.batch(jobs2)
    r3 = fpx.batch(jobs3)  # both kept buffers held: a fresh one
    for i in range(8):
        eq(r1[i], keep1[i], f"first call's result {i} changed")
    for i in (0, 7):
        eq(r2[i], oracle.conv(p, jobs2[i][2], jobs2[i][3]), f"second call {i}")
        eq(r3[i], oracle.conv(p, jobs3[i][2], jobs3[i][3]), f"third call {i}")
    addr1 = r1[0].__array_interface__["data"][0]  # the first job's result starts its buffer
    del r1
    r4 = fpx.batch(jobs1)  # the first buffer is free again
    assert r4[0].__array_interface__["data"][0] == addr1
    for i in range(8):
        eq(r4[i], keep1[i], f"repeat {i}")
