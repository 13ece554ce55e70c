#!/usr/bin/env python3
"""Benchmark of the fastpoly NTT hot path on B200.

Workload (headline): conv mod 998244353 of two 2^22-term polynomials, product of
2^23 - 1 terms: the largest native transform size of that prime (N = 2^23),
seeded uniform residues.  Metric: output Mcoeff/s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fpx|reference]

`value`  device-resident throughput: inputs already in HBM, CUDA events on the
         launching stream around each step, L2 flushed (512 MiB write) between
         steps outside the events; whole-job (all ranks) coefficients / max time.
`e2e`    the same metric through the public host-buffer C ABI (fpx_conv) from
         pinned host memory: H2D of both inputs and D2H of the product per step,
         --e2e-callers host threads (default 4, one context each) calling back
         to back, as the reference baseline runs concurrent calls.
`roofline` the dominant kernel's algorithmic bytes per launch / its average
         CUDA-event duration (events the library records on its stream around
         each launch, in a pass of the same steps right after the timed ones:
         inside the timed steps they would serialise the launches), against the
         measured HBM copy bandwidth; `roofline.compute` sets the step's and each
         kernel's algorithmic butterflies against the measured butterfly rate
         (fpx_measure_butterfly_rate), the ceiling that binds this path.
`cpu_baseline` the reference library (compiled from its own headers,
         oracle/_ref) on this host's cores, bounded sample, rank 0 at N = 1.
`batch`  (N = 1) the config-4 mix in one fpx_batch_submit (polys/s, device
         buffers, CUDA events), the plain per-call path on the same buffers
         (`plain_per_call`, `batch_speedup`) and fpx_batch_run from host buffers
         (`e2e`); as --workload batch.
`serve`  (N = 1) the config-5 request loop: closed-loop saturation req/s, then
         Poisson arrivals at 50 / 80 / 100 % of it with p50 / p99 latency,
         overall and per request-size class, --requests (3000) per level; as
         --workload serve.  --headline-only leaves both out.
Multi-GPU: one process per GPU (torchrun), independent replicas ("weak").

Other workloads, one JSON line each (not the default):
  --workload batch   4096 convs + 512 inv/exp of mixed sizes and moduli in one
                     fpx_batch_submit (polys/s), beside the per-call path and
                     the reference on all host cores
  --workload serve   the request loop: burst and closed-loop saturation req/s,
                     then Poisson arrivals at 50 / 80 / 100 % of saturation
                     with p50 / p99 latency
  --workload ops     single operations of the reference's configs 1-3
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

P = 998244353
LOGN_IN = 22
N_IN = 1 << LOGN_IN
N_OUT = 2 * N_IN - 1
N_FFT = 1 << (LOGN_IN + 1)
METRIC = "Mcoeff/s 2^23 conv (% HBM roofline)"
WORKLOAD = "conv mod 998244353: two 2^22-term inputs -> 2^23-1 terms (one native 2^23-point transform size)"
L2_FLUSH_BYTES = 512 << 20

# Algorithmic bytes per launch (two HBM passes of 4 B read + 4 B write per point
# per transform; pointwise fused): column pass over both operands = 2 passes,
# fused row pass = forward a, forward b and inverse = 3 passes, inverse column = 1.
ALG_BYTES = {"colfwd": 2 * 8 * N_FFT, "rows": 3 * 8 * N_FFT, "colinv": 8 * N_FFT}
STEP_ALG_BYTES = sum(ALG_BYTES.values())
# Algorithmic multiply instructions per launch: (N/2) log2(points) butterflies per
# transform at 3 (Shoup: mul.hi + 2 mul.lo), the pointwise product at 4 (Montgomery);
# columns are 2^11-point transforms, rows 2^12-point ones (2^11 x 2^12 = N).
LOG_R, LOG_C = 11, 12
ALG_MULS = {"colfwd": 2 * (N_FFT // 2) * LOG_R * 3,
            "rows": 3 * (N_FFT // 2) * LOG_C * 3 + N_FFT * 4,
            "colinv": (N_FFT // 2) * LOG_R * 3}
STEP_ALG_MULS = sum(ALG_MULS.values())
# Algorithmic butterflies per launch ((N/2) log2(points) per transform; the
# pointwise Montgomery product counted as 1.5, its multiply-pipe cycles over a
# Shoup butterfly's): the work the measured butterfly rate bounds.
ALG_BF = {"colfwd": 2 * (N_FFT // 2) * LOG_R,
          "rows": 3 * (N_FFT // 2) * LOG_C + 1.5 * N_FFT,
          "colinv": (N_FFT // 2) * LOG_R}
STEP_ALG_BF = sum(ALG_BF.values())


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def inputs(seed: int):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, P, N_IN, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, P, N_IN, dtype=np.uint64).astype(np.uint32)
    return a, b


def direct_coeffs(a, b, p: int, ks) -> list:
    """Coefficients ks of the product a * b mod p by direct sums (numpy, each
    product reduced before the sum): an oracle-free check of the measured path."""
    a64, b64 = a.astype(np.uint64), b.astype(np.uint64)
    out = []
    for k in ks:
        lo, hi = max(0, k - (len(b) - 1)), min(k, len(a) - 1)
        t = (a64[lo:hi + 1] * b64[k - hi:k - lo + 1][::-1]) % np.uint64(p)
        out.append(int(t.sum(dtype=np.uint64) % np.uint64(p)))
    return out


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "h1_conv_ncu.json")) as f:
            d = json.load(f)
        return d["kernels"][kernel]["dram_bytes_per_launch"]
    except Exception:
        return None


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = [r.split(", ") for r in out.strip().splitlines() if r.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measure_link(mib: int = 64, reps: int = 8) -> dict:
    """Pinned host <-> device copy bandwidth of this GPU's host link (GB/s): each
    direction alone and both at once on two streams (torch copies, CUDA events)."""
    import torch
    n = mib << 18
    h_in = torch.empty(n, dtype=torch.int32).pin_memory()
    h_out = torch.empty(n, dtype=torch.int32).pin_memory()
    d_in = torch.empty(n, dtype=torch.int32, device="cuda")
    d_out = torch.zeros(n, dtype=torch.int32, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(h2d: bool, d2h: bool) -> float:
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s1)
        s2.wait_event(e0)
        for _ in range(reps):
            if h2d:
                with torch.cuda.stream(s1):
                    d_in.copy_(h_in, non_blocking=True)
            if d2h:
                with torch.cuda.stream(s2):
                    h_out.copy_(d_out, non_blocking=True)
        done = torch.cuda.Event()
        done.record(s2)
        s1.wait_event(done)
        e1.record(s1)
        torch.cuda.synchronize()
        return reps * n * 4 / (e0.elapsed_time(e1) * 1e-3) / 1e9

    timed(True, True)
    h2d, d2h, both = timed(True, False), timed(False, True), timed(True, True)
    return {"h2d_gbs": round(h2d, 1), "d2h_gbs": round(d2h, 1), "each_way_both_gbs": round(both, 1),
            "how": f"pinned {mib} MiB copies x{reps}, torch, CUDA events; both: H2D and D2H on two streams"}


def max_over_ranks(dist, values, device="cpu"):
    """Element-wise max of per-rank timings (every rank gets the result)."""
    if not dist:
        return list(values)
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def whole_job_rates(world: int, steps: int, total_ms: float, e2e_steps: int, e2e_s: float):
    """(ms per step, whole-job Mcoeff/s device-resident, whole-job Mcoeff/s end to end):
    every rank converts its own inputs each step (replicas), timed by the slowest rank."""
    ms_per_step = total_ms / steps
    value = world * N_OUT / (ms_per_step * 1e-3) / 1e6
    e2e_value = world * N_OUT * e2e_steps / e2e_s / 1e6
    return ms_per_step, value, e2e_value


def cpu_reference_sample(reps: int, threads: int | None = None):
    """The reference's conv on this host's cores: `threads` concurrent calls per rep."""
    from oracle.oracle import Reference, OP_CONV, Oracle

    a, b = inputs(1)
    ref = Reference.load()
    if threads is None:
        threads = max(1, min(os.cpu_count() or 1, 64))
    if ref is not None:
        _, _, times = ref.run(OP_CONV, P, a, b, cap=N_OUT + 1, reps=reps, threads=threads)
        t = float(np.median(times))
        return {"value": threads * N_OUT / t / 1e6, "unit": "Mcoeff/s", "cores": threads, "kind": "reference",
                "sample": f"{threads} concurrent fpx::poly::conv(2^22 x 2^22) calls, {reps} reps, median "
                          f"({ref.backend} build of the reference headers)", "seconds_per_rep": t}
    O = Oracle()
    t0 = time.perf_counter()
    O.conv(P, a, b)
    t = time.perf_counter() - t0
    return {"value": N_OUT / t / 1e6, "unit": "Mcoeff/s", "cores": 1, "kind": "port",
            "sample": "1 conv(2^22 x 2^22) by the C restatement (reference build unavailable)", "seconds_per_rep": t}


def run_reference(args):
    rank, _, world = env_rank()
    if rank != 0:
        return 0
    threads = max(1, min(os.cpu_count() or 1, 64))
    from oracle.oracle import Reference, OP_CONV
    ref = Reference.load()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference library (oracle/_ref) not built on this host"}))
        return 0
    a, b = inputs(1)
    for _ in range(args.warmup):
        ref.run(OP_CONV, P, a, b, cap=N_OUT + 1, reps=1, threads=threads)
    total = 0.0
    for _ in range(args.steps):
        _, _, t = ref.run(OP_CONV, P, a, b, cap=N_OUT + 1, reps=1, threads=threads)
        total += float(t[0])
    ms = 1e3 * total / args.steps
    value = threads * N_OUT / (total / args.steps) / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mcoeff/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "p": P, "n_in": N_IN, "n_out": N_OUT, "transform_points": N_FFT,
                       "parallelism": f"{threads} host threads", "threads": threads,
                       "step": f"{threads} concurrent conv calls"},
            "cpu_baseline": {"value": value, "unit": "Mcoeff/s", "cores": threads, "kind": "reference",
                             "sample": f"{threads} concurrent fpx::poly::conv(2^22 x 2^22) calls per step ({ref.backend})"},
            "e2e": {"value": value, "unit": "Mcoeff/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_fpx(args):
    import torch
    import fastpoly_b200 as F

    rank, local, world = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ctx = F.Context(local)
    # one stream for the library's kernels, the L2 flush and the timing events
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    torch.cuda.set_stream(stream)

    a, b = inputs(1 + rank)
    da = torch.from_numpy(a.view(np.int32)).cuda()
    db = torch.from_numpy(b.view(np.int32)).cuda()
    dout = torch.empty(N_OUT, dtype=torch.int32, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device="cuda")

    def step():
        return ctx.conv_device(P, da, N_IN, db, N_IN, None, dout)

    # correctness spot-check of the measured path: 24 coefficients (first,
    # last, the middle one with the longest sum, random others) against direct
    # sums, independent of the oracle
    step()
    torch.cuda.synchronize()
    got = dout.cpu().numpy().view(np.uint32)
    ks = [0, N_OUT - 1, N_IN - 1] + [int(k) for k in np.random.default_rng(9).integers(0, N_OUT, 21)]
    want_ks = direct_coeffs(a, b, P, ks)
    assert [int(got[k]) for k in ks] == want_ks, "conv spot-check failed"

    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = ctx.launch_count()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in ev]
    launches = ctx.launch_count() - launches0
    total_ms = float(sum(step_ms))
    # per-kernel CUDA-event times for the roofline, from a separate pass of the
    # same steps: the events the library records around each kernel serialise
    # the launches (no programmatic overlap), so they stay out of the timed steps
    ctx.profile(True)
    for _ in range(min(args.steps, 50)):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    prof = ctx.profile_report()
    ctx.profile(False)

    # e2e through the host-buffer C ABI from pinned memory: `callers` host
    # threads, each with its own context and pinned buffers, call fpx_conv
    # back to back (like the reference baseline's concurrent calls); one
    # caller's upload overlaps another's download on the full-duplex link
    import threading
    callers = max(1, args.e2e_callers)
    e2e_steps = max(3, min(args.steps, 50))
    e2e_steps += (-e2e_steps) % callers
    pinned = []
    ctxs = [ctx] + [F.Context(local) for _ in range(callers - 1)]
    for c in ctxs:
        pa = torch.from_numpy(a.view(np.int32)).pin_memory().numpy().view(np.uint32)
        pb = torch.from_numpy(b.view(np.int32)).pin_memory().numpy().view(np.uint32)
        po = torch.empty(N_OUT, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
        c.conv(P, pa, pb, out=po)
        pinned.append((c, pa, pb, po))
    go = threading.Barrier(callers + 1)

    def caller(c, pa, pb, po):
        go.wait()
        for _ in range(e2e_steps // callers):
            c.conv(P, pa, pb, out=po)

    def run_callers(bufs):
        th = [threading.Thread(target=caller, args=t) for t in bufs]
        for t in th:
            t.start()
        t0 = time.perf_counter()
        go.wait()
        for t in th:
            t.join()
        return time.perf_counter() - t0

    if dist:
        dist.barrier()
    e2e_s = run_callers(pinned)
    # the same calls from ordinary (pageable) host memory, as a drop-in user's
    # std::vector storage would be: the library stages them through its pinned
    # slots
    pageable = []
    for c in ctxs:
        pa, pb, po = a.copy(), b.copy(), np.empty(N_OUT, dtype=np.uint32)
        c.conv(P, pa, pb, out=po)
        pageable.append((c, pa, pb, po))
    e2e_pageable_s = run_callers(pageable)
    clk = clocks.stop()
    for _, _, _, po in pinned + pageable:
        assert [int(po[k]) for k in ks] == want_ks, "end-to-end result check failed"
    for c in ctxs[1:]:
        c.close()

    total_ms, e2e_s = max_over_ranks(dist, [total_ms, e2e_s], device="cuda")
    ms_per_step, value, e2e_value = whole_job_rates(world, args.steps, total_ms, e2e_steps, e2e_s)

    # roofline of the dominant kernel: the slower of bytes over HBM bandwidth and
    # multiply instructions over the measured 32-bit multiply rate
    peak, peak_kind = measured_peak_hbm()
    imad = F.measure_imad_rate(local)
    bfr = F.measure_butterfly_rate(local)
    dom = max((k for k in prof if k in ALG_BYTES), key=lambda k: prof[k][1], default=None)
    roof = None
    if dom:
        cnt, tot = prof[dom]
        avg_s = tot / cnt * 1e-3
        achieved = ALG_BYTES[dom] / avg_s / 1e9
        roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "alg_bytes_per_launch": ALG_BYTES[dom], "avg_launch_us": round(avg_s * 1e6, 2),
                "launch_timing": "CUDA events on the library's stream around each launch, profiled pass of the "
                                 "same steps right after the timed region",
                "traffic": ncu_traffic(dom),
                "step": {"alg_bytes": STEP_ALG_BYTES, "achieved": round(STEP_ALG_BYTES / (ms_per_step * 1e-3) / 1e9, 1),
                         "frac": round(STEP_ALG_BYTES / (ms_per_step * 1e-3) / 1e9 / peak, 4),
                         "alg_mul_instr": STEP_ALG_MULS,
                         "t_roof_us": round(1e6 * max(STEP_ALG_BYTES / (peak * 1e9), STEP_ALG_MULS / imad), 2),
                         "frac_of_roofline": round(max(STEP_ALG_BYTES / (peak * 1e9), STEP_ALG_MULS / imad)
                                                   / (ms_per_step * 1e-3), 4)},
                "int_mul": {"alg_mul_instr_per_launch": ALG_MULS[dom],
                            "achieved_per_s": round(ALG_MULS[dom] / avg_s, 1), "peak_per_s": round(imad, 1),
                            "frac": round(ALG_MULS[dom] / avg_s / imad, 4),
                            "peak_source": "measured in this run (fpx_measure_imad_rate)"},
                "frac_of_roofline": round(max(ALG_BYTES[dom] / (peak * 1e9), ALG_MULS[dom] / imad) / avg_s, 4),
                "kernels_us": {k: round(v[1] / v[0] * 1e3, 2) for k, v in prof.items()},
                # the binding roofline of this path: transform butterflies over the
                # measured butterfly rate (mul.hi at a quarter of the warp rate)
                "compute": {"bound": "int multiply pipe (Shoup butterflies)",
                            "peak_butterflies_per_s": round(bfr, 1),
                            "peak_source": "measured in this run (fpx_measure_butterfly_rate)",
                            "step": {"alg_butterflies": STEP_ALG_BF,
                                     "t_roof_us": round(1e6 * STEP_ALG_BF / bfr, 2),
                                     "frac": round(STEP_ALG_BF / bfr / (ms_per_step * 1e-3), 4)},
                            "kernels": {k: {"alg_butterflies": ALG_BF[k],
                                            "t_roof_us": round(1e6 * ALG_BF[k] / bfr, 2),
                                            "frac": round(ALG_BF[k] / bfr / (prof[k][1] / prof[k][0] * 1e-3), 4)}
                                        for k in ALG_BF if k in prof}}}

    line = None
    if rank == 0:
        e2e_pageable = world * N_OUT * e2e_steps / e2e_pageable_s / 1e6
        line = {"metric": METRIC, "value": round(value, 1), "unit": "Mcoeff/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "p": P, "n_in": N_IN, "n_out": N_OUT, "transform_points": N_FFT,
                           "parallelism": f"replicas x{world}", "l2": "flushed between steps (512 MiB write)"},
                "e2e": {"value": round(e2e_value, 1), "unit": "Mcoeff/s", "h2d_bytes_per_step": 2 * N_IN * 4,
                        "d2h_bytes_per_step": N_OUT * 4, "steps": e2e_steps, "callers": callers,
                        "api": f"fpx_conv (host buffers, pinned), {callers} concurrent callers, one context each",
                        "pageable": {"value": round(e2e_pageable, 1), "unit": "Mcoeff/s",
                                     "api": f"fpx_conv from pageable host memory, {callers} concurrent callers"}},
                "gpu_launches": int(launches), "roofline": roof, "clocks": clk}
        if world == 1:
            # the host link bounds e2e: 32 MiB each way per conv
            link = measure_link()
            per_dir = max(2 * N_IN, N_OUT) * 4 * (e2e_value * 1e6 / N_OUT) / 1e9
            line["e2e"]["link"] = dict(link, achieved_each_way_gbs=round(per_dir, 1),
                                       frac=round(per_dir / link["each_way_both_gbs"], 3))
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_reference_sample(reps=3)
        if world == 1 and not args.headline_only:
            # configs 4 and 5 beside the headline (own contexts, after its timing)
            cpu_s = None if args.no_cpu_baseline else 8.0
            line["batch"] = batch_summary(local, 3, 20, cpu_s)
            line["serve"] = serve_summary(local, args.requests, args.workers, args.clients, args.serve_max_log, cpu_s)
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()
    return 0


# ============================================================================
# Secondary workloads (--workload batch | serve)
# ============================================================================
BATCH_MODULI = [998244353, 1000000007]
SERVE_MODULI = [998244353, 167772161, 1000000007, 2147483647]
NAIVE = 40


def batch_mix(seed: int = 4):
    """4096 convs (operand lengths floor(2^U), U ~ Uniform[6, 16] per operand) and
    512 inv / exp (n log-uniform in [2^8, 2^14]); moduli 50/50 998244353 / 1e9+7."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(4096):
        p = BATCH_MODULI[rng.integers(0, 2)]
        la, lb = int(2 ** rng.uniform(6, 16)), int(2 ** rng.uniform(6, 16))
        specs.append(("conv", p, rng.integers(0, p, la, dtype=np.uint64).astype(np.uint32),
                      rng.integers(0, p, lb, dtype=np.uint64).astype(np.uint32)))
    for _ in range(512):
        p = BATCH_MODULI[rng.integers(0, 2)]
        n = int(2 ** rng.uniform(8, 14))
        a = rng.integers(0, p, n, dtype=np.uint64).astype(np.uint32)
        if rng.integers(0, 2) == 0:
            a[0] = a[0] or 1
            specs.append(("inv", p, a, n))
        else:
            a[0] = 0
            specs.append(("exp", p, a, n))
    return specs


def serve_mix(count: int, seed: int = 5, max_log: int = 22):
    """conv 40 %, inv 20 %, exp 15 %, sqrt 10 %, divmod 10 %, pow 5 % (k uniform u64);
    sizes log-uniform in [2^8, 2^max_log]; moduli uniform over four."""
    rng = np.random.default_rng(seed)
    ops = ["conv"] * 8 + ["inv"] * 4 + ["exp"] * 3 + ["sqrt"] * 2 + ["divmod"] * 2 + ["pow"]
    specs = []
    for _ in range(count):
        op = ops[rng.integers(0, len(ops))]
        p = SERVE_MODULI[rng.integers(0, len(SERVE_MODULI))]
        n = int(2 ** rng.uniform(8, max_log))
        a = rng.integers(0, p, n, dtype=np.uint64).astype(np.uint32)
        if op == "conv":
            m = int(2 ** rng.uniform(8, max_log))
            specs.append(("conv", p, a, rng.integers(0, p, m, dtype=np.uint64).astype(np.uint32)))
        elif op == "divmod":
            b = rng.integers(0, p, (n + 1) // 2, dtype=np.uint64).astype(np.uint32)
            b[-1] = b[-1] or 1
            specs.append(("divmod", p, a, b))
        elif op == "pow":
            specs.append(("pow", p, a, int(rng.integers(0, 2**63, dtype=np.uint64)) * 2 + int(rng.integers(0, 2)), n))
        else:
            a[0] = {"inv": a[0] or 1, "exp": 0, "sqrt": 1}[op]
            specs.append((op, p, a, n))
    return specs


def mix_digest(specs) -> str:
    """SHA-256 over every job's operation, modulus, scalars and operand words:
    identifies a generated mix (the parity fixtures record it)."""
    import hashlib
    h = hashlib.sha256()
    for s in specs:
        h.update(s[0].encode())
        h.update(int(s[1]).to_bytes(4, "little"))
        for x in s[2:]:
            if isinstance(x, np.ndarray):
                h.update(len(x).to_bytes(8, "little"))
                h.update(np.ascontiguousarray(x, dtype=np.uint32).tobytes())
            else:
                h.update(int(x).to_bytes(8, "little"))
    return h.hexdigest()


def _native(p: int, log_n: int) -> bool:
    return p % 2 == 1 and p < (1 << 30) and 1 <= log_n <= ((p - 1) & -(p - 1)).bit_length() - 1


def _tbytes(n_pts: int) -> int:
    """Algorithmic bytes of one transform: 16 N past 2^15 points (two HBM passes), else 8 N."""
    return 16 * n_pts if n_pts > (1 << 15) else 8 * n_pts


def _product_bytes(p: int, la: int, lb: int, out: int, log_n: int | None = None) -> int:
    if min(la, lb) <= NAIVE or out <= 0:
        return 4 * (la + lb + out)
    if log_n is None:
        log_n = (la + lb - 2).bit_length()
    n_pts = 1 << log_n
    if _native(p, log_n):
        return 3 * _tbytes(n_pts)
    return 3 * 3 * _tbytes(n_pts) + 16 * out


def alg_bytes(spec) -> int:
    """The job's algorithmic HBM bytes under the transform byte rule (a batched
    product with a reusable spectrum counts its transforms once)."""
    op, p = spec[0], spec[1]
    if op == "conv":
        la, lb = len(spec[2]), len(spec[3])
        return _product_bytes(p, la, lb, la + lb - 1) if la and lb else 0
    n = spec[3]
    total, m = 0, 32
    if op == "inv":
        while m < n:
            k = (2 * m - 1).bit_length()
            total += 5 * _tbytes(1 << k) if _native(p, k) else 2 * (9 * _tbytes(1 << k) + 16 * m)
            m *= 2
        return total
    # exp: extension of the running inverse plus eight transforms per doubling
    csize = 16
    while m < n:
        k = (2 * m - 1).bit_length()
        hlen = min(2 * m, n) - m
        if csize < hlen:
            kc = (2 * csize - 1).bit_length()
            total += 5 * _tbytes(1 << kc) if _native(p, kc) else 2 * (9 * _tbytes(1 << kc) + 16 * hlen)
            csize = hlen
        total += 8 * _tbytes(1 << k) if _native(p, k) else 3 * (9 * _tbytes(1 << k) + 16 * hlen)
        m *= 2
    return total


def _device_jobs(F, torch, specs):
    """Job array with device copies of every operand (one upload) and outputs."""
    words_in = sum(len(s[2]) + (len(s[3]) if s[0] in ("conv", "divmod") else 0) for s in specs)
    caps = []
    for s in specs:
        if s[0] == "conv":
            caps.append(max(len(s[2]) + len(s[3]) - 1, 1))
        elif s[0] == "divmod":
            caps.append(len(s[2]) + len(s[3]))
        else:
            caps.append(s[-1])
    host = np.concatenate([np.concatenate([s[2], s[3]]) if s[0] in ("conv", "divmod") else s[2] for s in specs])
    din = torch.from_numpy(host.view(np.int32)).cuda()
    dout = torch.empty(sum(caps), dtype=torch.int32, device="cuda")
    jobs = (F.Job * len(specs))()
    qi = qo = 0
    base_in, base_out = din.data_ptr(), dout.data_ptr()
    for i, s in enumerate(specs):
        j = jobs[i]
        j.op, j.p = F._OPS[s[0]], s[1]
        j.a, j.la = base_in + 4 * qi, len(s[2])
        qi += len(s[2])
        if s[0] in ("conv", "divmod"):
            j.b, j.lb = base_in + 4 * qi, len(s[3])
            qi += len(s[3])
        j.n = F.SIZE_MAX if s[0] == "conv" else (0 if s[0] == "divmod" else s[-1])
        if s[0] == "pow":
            j.k = s[3]
        j.out = base_out + 4 * qo
        if s[0] == "divmod":
            j.out2 = base_out + 4 * (qo + len(s[2]))
        qo += caps[i]
    assert qi == words_in
    return jobs, din, dout


def batch_summary(local: int, warmup: int, steps: int, cpu_budget_s: float | None):
    """The config-4 mix (4096 conv + 512 inv/exp) through fpx_batch_submit on
    device buffers (CUDA events, L2 flushed between steps), the plain per-call
    device path on the same buffers, fpx_batch_run end to end from host buffers,
    and optionally the reference on the host cores.  Returns one dict."""
    import torch
    import fastpoly_b200 as F

    ctx = F.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    prev = torch.cuda.current_stream()
    torch.cuda.set_stream(stream)
    specs = batch_mix()
    jobs, din, dout = _device_jobs(F, torch, specs)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device="cuda")
    step_bytes = sum(alg_bytes(s) for s in specs)

    def step():
        rc = ctx.batch_submit(jobs)
        assert rc == F.OK, rc

    for _ in range(warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    steps = max(3, min(steps, 50))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    launches0 = ctx.launch_count()
    torch.cuda.synchronize()
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    launches = (ctx.launch_count() - launches0) // steps
    ms = float(np.median([s.elapsed_time(e) for s, e in ev]))
    value = len(specs) / (ms * 1e-3)

    # the plain per-call path on the same device buffers (one call per job)
    def plain():
        for i, s in enumerate(specs):
            j = jobs[i]
            if s[0] == "conv":
                ctx.conv_device(s[1], j.a, j.la, j.b, j.lb, None, j.out)
            elif s[0] == "inv":
                ctx.inv_device(s[1], j.a, j.la, j.n, j.out)
            else:
                ctx.exp_device(s[1], j.a, j.la, j.n, j.out)
        ctx.synchronize()

    plain()
    t0 = time.perf_counter()
    plain()
    plain_s = time.perf_counter() - t0

    # end to end: host buffers through fpx_batch_run (the previous step's
    # results are still held when the next step runs, as a caller's would be)
    for _ in range(3):
        res = ctx.batch(specs)
    e2e_steps = 10
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        res = ctx.batch(specs)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    bad = sum(isinstance(r, Exception) for r in res)
    assert bad == 0, f"{bad} failed jobs"
    h2d = 4 * sum(len(s[2]) + (len(s[3]) if s[0] == "conv" else 0) for s in specs)
    d2h = 4 * sum(r.size for r in res)
    peak, peak_kind = measured_peak_hbm()
    achieved = step_bytes / (ms * 1e-3) / 1e9
    out = {"metric": "polys/s, mixed batch (4096 conv + 512 inv/exp)", "value": round(value, 1), "unit": "polys/s",
           "steps": steps, "ms_per_step": round(ms, 4),
           "config": {"workload": "4096 conv (lengths 2^U, U~U[6,16]) + 512 inv/exp (n log-uniform 2^8..2^14), "
                                  "moduli 50/50 998244353 / 1000000007, fixed seed", "jobs": len(specs),
                      "l2": "flushed between steps (512 MiB write)"},
           "plain_per_call": {"value": round(len(specs) / plain_s, 1), "unit": "polys/s",
                              "api": "fpx_conv_device / fpx_inv_device / fpx_exp_device, one call per job"},
           "batch_speedup": round(value / (len(specs) / plain_s), 2),
           "e2e": {"value": round(len(specs) / e2e_s, 1), "unit": "polys/s", "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h, "api": "fpx_batch_run (host buffers)"},
           "gpu_launches": int(launches),
           "roofline": {"bound": "hbm", "kernel": "whole batch step", "achieved": round(achieved, 1), "peak": peak,
                        "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": None,
                        "alg_bytes_per_step": step_bytes, "peak_source": peak_kind}}
    torch.cuda.set_stream(prev)
    ctx.close()
    del din, dout, flush
    if cpu_budget_s:
        out["cpu_baseline"] = cpu_mix_sample(specs, budget_s=cpu_budget_s)
    return out


def run_batch_fpx(args):
    import torch

    rank, local, world = env_rank()
    torch.cuda.set_device(local)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    b = batch_summary(local, args.warmup, args.steps, None if args.no_cpu_baseline else 20.0)
    line = dict(b, n_gpus=1, warmup=args.warmup, higher_is_better=True, scaling="weak", vs_baseline=None,
                dtype="u32", data="synthetic", clocks=clocks.stop())
    print(json.dumps(line))
    return 0


def _ref_call(ref, spec):
    from oracle.oracle import OP_CONV, OP_INV, OP_LOG, OP_EXP, OP_SQRT, OP_POW, OP_DIVMOD
    op, p = spec[0], spec[1]
    code = {"conv": OP_CONV, "inv": OP_INV, "log": OP_LOG, "exp": OP_EXP, "sqrt": OP_SQRT, "pow": OP_POW,
            "divmod": OP_DIVMOD}[op]
    if op == "conv":
        return ref.run(code, p, spec[2], spec[3], cap=len(spec[2]) + len(spec[3]))[2][0]
    if op == "divmod":
        return ref.run(code, p, spec[2], spec[3], cap=len(spec[2]) + len(spec[3]))[2][0]
    if op == "pow":
        return ref.run(code, p, spec[2], n=spec[4], k=spec[3], cap=spec[4])[2][0]
    try:
        return ref.run(code, p, spec[2], n=spec[3], cap=spec[3])[2][0]
    except Exception:
        return 0.0


def cpu_mix_sample(specs, budget_s: float = 20.0, threads: int | None = None, unit: str = "polys/s"):
    """The reference on this host's cores: one worker thread per core pulling jobs
    of the mix (the library is thread-safe across calls), until the job list or
    the time budget runs out; polys/s over the jobs finished."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.oracle import Reference
    ref = Reference.load()
    if ref is None:
        return {"value": None, "unavailable": "reference build (oracle/_ref) missing"}
    threads = threads or max(1, min(os.cpu_count() or 1, 64))
    deadline = time.perf_counter() + budget_s
    done = [0]

    def work(s):
        if time.perf_counter() > deadline:
            return
        _ref_call(ref, s)
        done[0] += 1

    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(work, specs))
    el = time.perf_counter() - t0
    return {"value": round(done[0] / el, 1), "unit": unit, "cores": threads, "kind": "reference",
            "sample": f"{done[0]} of {len(specs)} jobs of the mix on {threads} threads in {el:.1f} s ({ref.backend})"}


def run_batch_reference(args):
    rank, _, world = env_rank()
    if rank != 0:
        return 0
    specs = batch_mix()
    threads = max(1, min(os.cpu_count() or 1, 64))
    for _ in range(min(args.warmup, 1)):
        cpu_mix_sample(specs[:256], budget_s=5.0, threads=threads)
    vals = [cpu_mix_sample(specs, budget_s=20.0, threads=threads) for _ in range(max(1, min(args.steps, 3)))]
    v = float(np.median([x["value"] for x in vals]))
    line = {"impl": "reference", "metric": "polys/s, mixed batch (4096 conv + 512 inv/exp)", "value": v,
            "unit": "polys/s", "n_gpus": world, "steps": len(vals), "warmup": args.warmup,
            "ms_per_step": round(1e3 * len(specs) / v, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": "batch mix (same as --workload batch)", "threads": threads},
            "cpu_baseline": dict(vals[0], value=v),
            "e2e": {"value": v, "unit": "polys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


SIZE_CLASSES = [(8, 12), (12, 16), (16, 19), (19, 23)]  # log2 of the request size, [lo, hi)


def _size_log(spec) -> int:
    n = len(spec[2]) if spec[0] in ("conv", "divmod") else spec[-1]
    if spec[0] == "conv":
        n = max(n, len(spec[3]))
    return max(0, int(n).bit_length() - 1)


def serve_summary(local: int, count: int, workers: int, clients: int, max_log: int, cpu_budget_s: float | None):
    """The config-5 request loop: burst rate, closed-loop saturation, then Poisson
    arrivals at 50 / 80 / 100 % of saturation with p50 / p99 latency (overall and
    per request-size class), `count` requests per level.  Returns one dict."""
    import threading
    import fastpoly_b200 as F

    specs = serve_mix(count, max_log=max_log)
    cls_of = [next(k for k, (lo, hi) in enumerate(SIZE_CLASSES) if lo <= min(_size_log(sp), 22) < hi)
              for sp in specs]
    srv = F.Server(local, workers=workers)
    try:
        # warm-up: plans, pools and pinned buffers of every worker, on the same mix
        for t in [srv.submit(s) for s in specs]:
            srv.poll(t)
        # burst: everything offered at once (largest micro-batches)
        t0 = time.perf_counter()
        tickets = [srv.submit(s) for s in specs]
        fails = 0
        for t in tickets:
            r, _ = srv.poll(t)
            fails += isinstance(r, Exception)
        burst_rate = count / (time.perf_counter() - t0)

        # saturation: a closed loop of `clients` callers, each submitting its next
        # request when the previous one completes (the steady state the open-loop
        # loads below are fractions of)
        def closed_loop(n_clients):
            def client(k):
                for i in range(k, count, n_clients):
                    srv.poll(srv.submit(specs[i]))
            th = [threading.Thread(target=client, args=(k,)) for k in range(n_clients)]
            t0 = time.perf_counter()
            for t in th:
                t.start()
            for t in th:
                t.join()
            return count / (time.perf_counter() - t0)

        sat_rate = closed_loop(clients)
        loads = {}
        for frac in (0.5, 0.8, 1.0):
            rate = frac * sat_rate
            rng = np.random.default_rng(int(frac * 100))
            arrivals = np.cumsum(rng.exponential(1.0 / rate, count))
            tickets = [None] * count

            def submitter():
                start = time.perf_counter()
                for i in range(count):
                    d = start + arrivals[i] - time.perf_counter()
                    if d > 0:
                        time.sleep(d)
                    tickets[i] = srv.submit(specs[i])

            th = threading.Thread(target=submitter)
            t0 = time.perf_counter()
            th.start()
            lats = []
            for i in range(count):
                while tickets[i] is None:
                    time.sleep(0.0002)
                r, lat = srv.poll(tickets[i])
                lats.append(lat)
            th.join()
            el = time.perf_counter() - t0
            lats = np.asarray(lats)
            per_cls = {}
            for k, (lo, hi) in enumerate(SIZE_CLASSES):
                sel = lats[[c == k for c in cls_of]]
                if sel.size:
                    per_cls[f"2^{lo}..2^{hi - 1}"] = {"n": int(sel.size),
                                                      "p50_ms": round(1e3 * float(np.percentile(sel, 50)), 3),
                                                      "p99_ms": round(1e3 * float(np.percentile(sel, 99)), 3)}
            loads[f"{int(frac * 100)}%"] = {"offered_req_s": round(rate, 2), "achieved_req_s": round(count / el, 2),
                                            "p50_ms": round(1e3 * float(np.percentile(lats, 50)), 3),
                                            "p99_ms": round(1e3 * float(np.percentile(lats, 99)), 3),
                                            "by_size": per_cls}
        st = srv.stats()
    finally:
        srv.stop()
    in_bytes = 4 * sum(len(s[2]) + (len(s[3]) if s[0] in ("conv", "divmod") else 0) for s in specs)
    out_bytes = 4 * sum(len(s[2]) + len(s[3]) - 1 if s[0] == "conv" else
                        (len(s[2]) + len(s[3]) if s[0] == "divmod" else s[-1]) for s in specs)
    out = {"metric": "served requests/s at saturation (mixed ops, sizes 2^8..2^%d)" % max_log,
           "value": round(sat_rate, 2), "unit": "req/s", "ms_per_step": round(1e3 / sat_rate, 3),
           "config": {"workload": "conv 40 / inv 20 / exp 15 / sqrt 10 / divmod 10 / pow 5 %, sizes log-uniform "
                                  f"2^8..2^{max_log}, moduli 998244353 / 167772161 / 1e9+7 / 2^31-1",
                      "requests_per_level": count, "workers": workers, "failed": int(fails),
                      "saturation": f"closed loop of {clients} callers"},
           "latency": loads, "server": st, "burst_req_s": round(burst_rate, 2),
           "e2e": {"value": round(sat_rate, 2), "unit": "req/s", "h2d_bytes_per_step": in_bytes // count,
                   "d2h_bytes_per_step": out_bytes // count,
                   "api": "fpx_serve_submit / fpx_serve_poll (host buffers)"}}
    if cpu_budget_s:
        out["cpu_baseline"] = cpu_mix_sample(specs, budget_s=cpu_budget_s, unit="req/s")
    return out


def run_serve_fpx(args):
    import torch

    rank, local, world = env_rank()
    torch.cuda.set_device(local)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    sv = serve_summary(local, args.requests, args.workers, args.clients, args.serve_max_log,
                       None if args.no_cpu_baseline else 30.0)
    line = dict(sv, n_gpus=1, steps=args.requests, warmup=args.requests, higher_is_better=True, scaling="weak",
                vs_baseline=None, dtype="u32", data="synthetic", clocks=clocks.stop())
    print(json.dumps(line))
    return 0


def ops_cases():
    """Single operations of the reference's configs 1-3 (seeded uniform residues)."""
    rng = np.random.default_rng(6)

    def r(p, n, a0=None):
        a = rng.integers(0, p, n, dtype=np.uint64).astype(np.uint32)
        if a0 is not None:
            a[0] = a0
        return a

    p, q = 998244353, 1000000007
    n22 = 1 << 22
    sq = None
    return [
        ("C1 conv 2^18 x 2^18", "conv", p, (r(p, 1 << 18), r(p, 1 << 18)), None),
        ("H1 conv 2^22 x 2^22", "conv", p, (r(p, n22), r(p, n22)), None),
        ("H2 conv 2^23 x 2^23 (CRT)", "conv", p, (r(p, 1 << 23), r(p, 1 << 23)), None),
        ("C2 inv 2^22", "inv", p, (r(p, n22, 1),), n22),
        ("C2 log 2^22", "log", p, (r(p, n22, 1),), n22),
        ("C2 exp 2^22", "exp", p, (r(p, n22, 0),), n22),
        ("C2 sqrt 2^22", "sqrt", p, (r(p, n22, 1),), n22),
        ("C2 pow k=1000003 2^22", "pow", p, (r(p, n22), 1000003), n22),
        ("C3 conv 2^23 x 2^23 mod 1e9+7", "conv", q, (r(q, 1 << 23), r(q, 1 << 23)), None),
        ("C3 inv 2^22 mod 1e9+7", "inv", q, (r(q, n22, int(rng.integers(1, q))),), n22),
        ("C3 conv 2^25 x 2^25 mod 1e9+7", "conv", q, (r(q, 1 << 25), r(q, 1 << 25)), None),
    ]


def run_ops_fpx(args):
    """Device-resident time of each single operation (CUDA events, median of
    `reps`), output Mcoeff/s; the reference's single-threaded time beside it
    where one call takes under ~3 s on the host."""
    import torch
    import fastpoly_b200 as F
    from oracle.oracle import Reference, OP_CONV, OP_INV, OP_LOG, OP_EXP, OP_SQRT, OP_POW

    rank, local, world = env_rank()
    torch.cuda.set_device(local)
    ctx = F.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    torch.cuda.set_stream(stream)
    ref = None if args.no_cpu_baseline else Reference.load()
    codes = {"conv": OP_CONV, "inv": OP_INV, "log": OP_LOG, "exp": OP_EXP, "sqrt": OP_SQRT, "pow": OP_POW}
    rows = []
    for name, op, p, ins, n in ops_cases():
        a = ins[0]
        da = torch.from_numpy(a.view(np.int32)).cuda()
        if op == "conv":
            b = ins[1]
            db = torch.from_numpy(b.view(np.int32)).cuda()
            outn = a.size + b.size - 1
        else:
            outn = n
        dout = torch.empty(outn, dtype=torch.int32, device="cuda")

        def call():
            if op == "conv":
                ctx.conv_device(p, da, a.size, db, b.size, None, dout)
            elif op == "pow":
                ctx.pow_device(p, da, a.size, ins[1], n, dout)
            else:
                getattr(ctx, op + "_device")(p, da, a.size, n, dout)

        call()
        torch.cuda.synchronize()
        reps = 5
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = float(np.median(ts))
        row = {"case": name, "p": p, "out_terms": outn, "gpu_ms": round(ms, 3),
               "gpu_mcoeff_s": round(outn / (ms * 1e-3) / 1e6, 1)}
        if ref is not None and outn <= (1 << 24) and not (op == "conv" and p != 998244353 and outn > (1 << 24)):
            if op == "conv":
                _, _, t = ref.run(OP_CONV, p, a, b, cap=outn + 1)
            elif op == "pow":
                _, _, t = ref.run(OP_POW, p, a, n=n, k=ins[1], cap=n)
            else:
                _, _, t = ref.run(codes[op], p, a, n=n, cap=n)
            row["cpu_ref_1thread_ms"] = round(1e3 * float(t[0]), 1)
            row["speedup_vs_1_core"] = round(1e3 * float(t[0]) / ms, 1)
        rows.append(row)
        del da, dout
        if op == "conv":
            del db
        torch.cuda.empty_cache()
    line = {"metric": "single-operation Mcoeff/s, configs 1-3", "value": rows[1]["gpu_mcoeff_s"], "unit": "Mcoeff/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "u32", "data": "synthetic",
            "config": {"workload": "configs 1-3 single operations, device-resident, CUDA events, median of 5"},
            "ops": rows}
    if ref is not None:
        line["cpu_baseline"] = {"kind": "reference", "cores": 1, "backend": ref.backend,
                                "sample": "one call per case (cases whose output exceeds 2^24 terms skipped)"}
    print(json.dumps(line))
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="fpx", choices=["fpx", "reference"])
    ap.add_argument("--workload", default="conv", choices=["conv", "batch", "serve", "ops"],
                    help="conv: the headline 2^23 conv (default); batch: mixed batch; serve: request loop; "
                         "ops: single operations of configs 1-3")
    ap.add_argument("--requests", type=int, default=3000, help="serve: requests per load level")
    ap.add_argument("--serve-max-log", type=int, default=22, help="serve: largest size 2^k")
    ap.add_argument("--workers", type=int, default=0,
                    help="serve: worker threads (half large-lane, the rest small-lane; 0 = the library's 6)")
    ap.add_argument("--clients", type=int, default=32, help="serve: callers of the closed-loop saturation run")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="conv: leave out the batch (config 4) and serve (config 5) objects of the default line")
    ap.add_argument("--e2e-callers", type=int, default=4,
                    help="conv: concurrent host threads (one context each) of the end-to-end measurement")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.workload == "batch":
        return run_batch_reference(args) if args.impl == "reference" else run_batch_fpx(args)
    if args.workload == "ops":
        return run_ops_fpx(args)
    if args.workload == "serve":
        if args.impl == "reference":
            rank, _, world = env_rank()
            if rank == 0:
                specs = serve_mix(args.requests, max_log=args.serve_max_log)
                b = cpu_mix_sample(specs, budget_s=60.0, unit="req/s")
                print(json.dumps({"impl": "reference", "metric": "served requests/s at saturation", "value": b["value"],
                                  "unit": "req/s", "n_gpus": world, "higher_is_better": True, "cpu_baseline": b,
                                  "e2e": {"value": b["value"], "unit": "req/s", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}))
            return 0
        return run_serve_fpx(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_fpx(args)


if __name__ == "__main__":
    sys.exit(main())
