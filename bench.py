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
         pinned host memory: H2D of both inputs and D2H of the product per step.
`roofline` the dominant kernel's algorithmic bytes per launch / its average
         CUDA-event duration measured over the timed region, against the
         measured HBM copy bandwidth.
`cpu_baseline` the reference library (compiled from its own headers,
         oracle/_ref) on this host's cores, bounded sample, rank 0 at N = 1.
Multi-GPU: one process per GPU (torchrun), independent replicas ("weak").
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


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def inputs(seed: int):
    rng = np.random.default_rng(seed)
    a = rng.integers(0, P, N_IN, dtype=np.uint64).astype(np.uint32)
    b = rng.integers(0, P, N_IN, dtype=np.uint64).astype(np.uint32)
    return a, b


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
            "config": {"workload": WORKLOAD, "threads": threads, "step": f"{threads} concurrent conv calls"},
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

    # correctness spot-check of the measured path (first/last coefficients vs a
    # direct sum), cheap and independent of the oracle
    step()
    torch.cuda.synchronize()
    got = dout[:4].cpu().numpy().view(np.uint32)
    want0 = int(a[0]) * int(b[0]) % P
    assert int(got[0]) == want0, "conv spot-check failed"

    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = ctx.launch_count()
    ctx.profile(True)
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
    prof = ctx.profile_report()
    ctx.profile(False)
    launches = ctx.launch_count() - launches0
    total_ms = float(sum(step_ms))

    # e2e through the host-buffer C ABI from pinned memory
    pa = torch.from_numpy(a.view(np.int32)).pin_memory().numpy().view(np.uint32)
    pb = torch.from_numpy(b.view(np.int32)).pin_memory().numpy().view(np.uint32)
    po = torch.empty(N_OUT, dtype=torch.int32).pin_memory().numpy().view(np.uint32)
    ctx.conv(P, pa, pb, out=po)
    e2e_steps = max(3, min(args.steps, 50))
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.conv(P, pa, pb, out=po)
    e2e_s = time.perf_counter() - t0
    clk = clocks.stop()
    assert int(po[0]) == want0

    total_ms, e2e_s = max_over_ranks(dist, [total_ms, e2e_s], device="cuda")
    ms_per_step, value, e2e_value = whole_job_rates(world, args.steps, total_ms, e2e_steps, e2e_s)

    # roofline of the dominant kernel
    peak, peak_kind = measured_peak_hbm()
    dom = max((k for k in prof if k in ALG_BYTES), key=lambda k: prof[k][1], default=None)
    roof = None
    if dom:
        cnt, tot = prof[dom]
        avg_s = tot / cnt * 1e-3
        achieved = ALG_BYTES[dom] / avg_s / 1e9
        roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "alg_bytes_per_launch": ALG_BYTES[dom], "avg_launch_us": round(avg_s * 1e6, 2),
                "traffic": ncu_traffic(dom),
                "step": {"alg_bytes": STEP_ALG_BYTES, "achieved": round(STEP_ALG_BYTES / (ms_per_step * 1e-3) / 1e9, 1),
                         "frac": round(STEP_ALG_BYTES / (ms_per_step * 1e-3) / 1e9 / peak, 4)},
                "kernels_ms": {k: round(v[1] / v[0] * 1e3, 2) for k, v in prof.items()}}

    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 1), "unit": "Mcoeff/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "p": P, "n_in": N_IN, "n_out": N_OUT, "transform_points": N_FFT,
                           "parallelism": f"replicas x{world}", "l2": "flushed between steps (512 MiB write)"},
                "e2e": {"value": round(e2e_value, 1), "unit": "Mcoeff/s", "h2d_bytes_per_step": 2 * N_IN * 4,
                        "d2h_bytes_per_step": N_OUT * 4, "steps": e2e_steps,
                        "api": "fpx_conv (host buffers, pinned)"},
                "gpu_launches": int(launches), "roofline": roof, "clocks": clk}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_reference_sample(reps=3)
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="fpx", choices=["fpx", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    return run_fpx(args)


if __name__ == "__main__":
    sys.exit(main())
