#!/usr/bin/env python3
"""PALMAD throughput on B200: n = 2^21, lengths 64..512, top-1 per length.

One step = one full PALMAD run (every length 64..512 with the MERLIN
r-schedule) over the seeded synthetic series of ``datagen.palmad_series``
(random walk + sinusoid, 16 planted anomalies: noise / flatline / reversal).

Metric: matrix-equivalent pairs per second, i.e. sum over lengths m of
N_m^2 (N_m = n - m + 1 windows) divided by the time of one PALMAD run.  It
is the work an all-pairs method would do per run; the seconds per run are
reported beside it (``ms_per_step``).

Arms:
  default            libpaddi on the GPU (device-resident series for
                     ``value``; host buffers through the C ABI for ``e2e``).
  --impl reference   the reference's own CPU kernels (oracle/_ref, compiled
                     from PADDi's src/cpu_kernels/cpu_kernels.cpp) on all host
                     threads, each step a bounded sample of the same series.

Multi-GPU (torchrun): PALMAD on one series does not shard in this build, so
--gpus N runs N independent replicas (weak scaling); ``value`` sums them.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

N_SERIES = 1 << 21
MIN_L, MAX_L = 64, 512
WORKLOAD = "palmad n=2^21 L=64..512 top-1 (16 planted anomalies, seed 1)"
# the large single-GPU run: ECG-like series, CPU sample from its first 2^22 points
LARGE_N, LARGE_MIN_L, LARGE_MAX_L = 1 << 27, 128, 384
LARGE_WORKLOAD = ("palmad n=2^27 L=128..384 top-1 (ECG-like beats, 64 altered, seed 5)")
LARGE_CPU_POINTS = 1 << 22
CPU_SAMPLE_N = 1 << 14          # points per CPU sample slice
CPU_SLICES_PER_THREAD = 2
CPU_SAMPLE_LENGTHS = 8          # lengths 64..71
REF_GPU_ATTEMPTS = 8            # attempts of the reference's GPU path timed (~1 s each)
L2_FLUSH_BYTES = 512 << 20      # > 126 MB L2
# DRAM bytes (read + write) of one k_refine_umma launch from an ncu capture:
# the last refine round (windows N/2..N) of an m=300 attempt on this series
REFINE_TRAFFIC_BYTES = 13450752
REFINE_TRAFFIC_LAUNCH = "refine round over windows N/2..N at m=300, ncu dram__bytes_read+write"


def matrix_pairs(n: int, minL: int, maxL: int) -> float:
    return float(sum((n - m + 1) ** 2 for m in range(minL, maxL + 1)))


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs"), d.get("bf16_tflops"), d.get("bf16_tflops_sustained"), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        busy = [v for v in sm if mx and v > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------- dist plumbing
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_max(world, v: float) -> float:
    """Max of v over the ranks (the slowest replica sets the step time)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world: int, pairs_per_replica: float, step_ms_local: float):
    """Whole-job throughput of `world` replicas: all pairs over the max step time."""
    step_ms = reduce_max(world, step_ms_local)
    return world * pairs_per_replica / (step_ms / 1e3), step_ms


# ---------------------------------------------------------------- CPU reference
def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def has_flat_run(s, run: int) -> bool:
    """True when s holds `run` or more consecutive equal values."""
    eq = np.concatenate([[0], (np.diff(s) == 0).astype(np.int8), [0]])
    d = np.diff(eq)
    starts, ends = np.flatnonzero(d == 1), np.flatnonzero(d == -1)
    return bool(np.any(ends - starts >= run - 1))


def cpu_sample_slices(x, count: int, minl: int = MIN_L):
    """Up to `count` consecutive 2^14-point slices of the series that hold no
    flat run of MIN_L points: the reference's FP32 z-normalisation divides by
    a zero deviation on such windows and its r-schedule then never ends."""
    out = []
    for k in range(len(x) // CPU_SAMPLE_N):
        s = x[k * CPU_SAMPLE_N:(k + 1) * CPU_SAMPLE_N]
        if not has_flat_run(s, minl):
            out.append(s)
        if len(out) == count:
            break
    return out


def cpu_reference(x, steps: int, warmup: int, threads: int, minl: int = MIN_L):
    from oracle import oracle as O
    maxl = minl + CPU_SAMPLE_LENGTHS - 1
    slices = cpu_sample_slices(x, CPU_SLICES_PER_THREAD * threads, minl)
    threads = min(threads, len(slices))
    pairs = len(slices) * matrix_pairs(CPU_SAMPLE_N, minl, maxl)
    for _ in range(warmup):
        O.ref_palmad_many(slices[:1], minl, minl, threads=1)
    t = time.perf_counter()
    for _ in range(steps):
        O.ref_palmad_many(slices, minl, maxl, threads=threads)
    el = (time.perf_counter() - t) / steps
    return {"value": pairs / el, "unit": "pairs/s", "cores": threads, "kind": "reference",
            "sample": f"{len(slices)} slices of {CPU_SAMPLE_N} points of the same series "
                      f"(slices without a flat run), lengths {minl}..{maxl}, "
                      f"{threads} threads taking slices as they free up",
            "s_per_sample": el}


def full_length_point(ctx, st, x, disc, args):
    """Like for like: one attempt of the reference's CPU kernels on a whole
    series of the headline's size at length minL (one host thread: the
    reference has no parallel CPU path) at r just below the length's top-1
    distance, and the same attempt on the GPU (device time).  The series is
    the headline generator with its noise and reverse anomalies only: on the
    flat runs of the headline series the reference's FP32 statistics divide by
    a zero deviation and its attempt finds no candidate at all.  The sample
    above uses short slices, where DRAG prunes less per matrix cell, so its
    ratio favours the GPU; this one does not."""
    import torch

    from oracle import oracle as O
    from paddi_b200 import datagen
    m = args.minL
    y, _ = datagen.palmad_series(n=len(x), seed=1, kinds_cycle=("noise", "reverse"))
    top, _ = ctx.pd3(y, m, top_k=1)  # the halving schedule: this length's top-1
    r = float(np.sqrt(np.float32(top[0].dist))) * 0.999
    t = time.perf_counter()
    att, _, _ = O.ref_attempt(y, m, r)
    cpu_s = time.perf_counter() - t
    ctx.pd3(y, m, top_k=1, r=r)  # warm
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    got, _ = ctx.pd3(y, m, top_k=1, r=r)
    e1.record(st)
    e1.synchronize()
    gpu_ms = e0.elapsed_time(e1)
    return {"what": f"one attempt at m={m} on all {len(y)} points, r^2={r * r:.4f}",
            "series": "the headline generator (seed 1) with noise and reverse anomalies only "
                      "(no flat runs)",
            "reference_note": "the reference's one-pass FP32 window statistics lose the "
                              "variances of this 2^21-point random walk (values to 1.7e3): "
                              "its attempt prunes every window (cpu_found -1)",
            "cpu_s": cpu_s, "cores": 1, "gpu_ms": gpu_ms, "ratio": cpu_s * 1e3 / gpu_ms,
            "cpu_found": att["top_ind"], "gpu_found": got[0].ind if got else -1,
            "same_window": bool(got) and att["top_ind"] == got[0].ind,
            "note": "gpu_ms includes the series upload and statistics of the call"}


def reference_gpu_point(x, disc, args, plain_log):
    """The reference's own FP32 GPU kernels (src/PD3_kernels.cuh,
    src/preprocessing.cuh, built from the reference's headers into oracle/_ref)
    with its MERLIN schedule, on the same series, for the first lengths until
    REF_GPU_ATTEMPTS attempts have run; ms per attempt, and the full run
    estimated from the attempts the plain form's MERLIN schedule takes."""
    from oracle import oracle as O
    try:
        res = O.refgpu_palmad(x, args.minL, args.maxL, max_attempts=REF_GPU_ATTEMPTS)
    except (OSError, RuntimeError) as e:
        return {"unavailable": str(e)}
    if res is None:
        return {"unavailable": "oracle/_ref/libpaddi_refgpu.so not built"}
    done, att, ms = res
    ours = [(d.ind, d.dist) for d in disc[:len(done)]]
    errs = [abs(a[1] - b[1]) / b[1] for a, b in zip(done, ours) if b[1] > 0]
    per = ms / max(att, 1)
    out = {"what": "reference FP32 GPU kernels (phase 1, define, local refine, host union, "
                   "node refine) with its MERLIN schedule; first lengths only",
           "lengths": len(done), "attempts": att, "ms_per_attempt": per,
           "same_discords_on_those_lengths": [a[0] for a in done] == [b[0] for b in ours],
           "max_rel_dist_err_vs_fp64": max(errs) if errs else None}
    if plain_log is not None:
        out["est_ms_per_step"] = per * len(plain_log)
        out["est_basis"] = f"{len(plain_log)} MERLIN attempts of the plain form"
    return out


def workload(args):
    """(series, name) of the selected workload; fills args.n / minL / maxL."""
    from paddi_b200 import datagen
    if args.workload == "large":
        args.n = args.n or LARGE_N
        args.minL = args.minL or LARGE_MIN_L
        args.maxL = args.maxL or LARGE_MAX_L
        x, _ = datagen.ecg_series(n=args.n, seed=5)
        name = LARGE_WORKLOAD if (args.n, args.minL, args.maxL) == (
            LARGE_N, LARGE_MIN_L, LARGE_MAX_L) else f"palmad ECG-like n={args.n} L={args.minL}..{args.maxL}"
    else:
        args.n = args.n or N_SERIES
        args.minL = args.minL or MIN_L
        args.maxL = args.maxL or MAX_L
        x, _ = datagen.palmad_series(n=args.n, seed=1)
        name = WORKLOAD if (args.n, args.minL, args.maxL) == (N_SERIES, MIN_L, MAX_L) else \
            f"palmad n={args.n} L={args.minL}..{args.maxL}"
    return x, name


def metric_name(args):
    if args.workload == "large":
        return "PALMAD matrix-equivalent pairs/s (n=2^27, L=128..384, top-1)"
    return "PALMAD matrix-equivalent pairs/s (n=2^21, L=64..512, top-1)"


def cpu_sample_of(x, args):
    """The part of the series the CPU sample slices come from."""
    return x[:LARGE_CPU_POINTS] if args.workload == "large" else x


def run_reference(args, world, rank):
    if rank != 0:
        return
    x, name = workload(args)
    threads = min(host_threads(), 64)
    cb = cpu_reference(cpu_sample_of(x, args), args.steps, args.warmup, threads, args.minL)
    line = {"metric": metric_name(args),
            "value": cb["value"], "unit": "pairs/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cb["s_per_sample"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": name + " (bounded CPU sample)", "n": args.n,
                       "minL": args.minL, "maxL": args.maxL},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm
def _progress(rank, msg):
    if rank == 0:
        print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def run_paddi(args, world, rank, local):
    import torch

    import paddi_b200 as P

    torch.cuda.set_device(local)
    x, name = workload(args)
    n = len(x)
    dk = {"auto": P.DIST_AUTO, "fp32": P.DIST_FP32, "bf16": P.DIST_SPLIT_BF16,
          "fp16": P.DIST_SPLIT_FP16}[args.dist]
    rp = {"merlin": P.R_MERLIN, "learned": P.R_LEARNED, "bound": P.R_BOUND}[args.r_policy]
    ctx = P.Context(device=local, distance_kernel=dk, r_policy=rp)
    ctx.reserve(n, args.maxL)
    st = torch.cuda.ExternalStream(ctx.stream)
    d_x = torch.from_numpy(x).to(f"cuda:{local}")
    h_x = torch.from_numpy(x).pin_memory()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    torch.cuda.synchronize()
    pairs = matrix_pairs(n, args.minL, args.maxL)

    def flush_l2(i):
        with torch.cuda.stream(st):
            flush.fill_(float(i))

    _progress(rank, "warm-up")
    for i in range(args.warmup):
        flush_l2(i)
        ctx.palmad_device(d_x.data_ptr(), n, args.minL, args.maxL)
    torch.cuda.synchronize()
    _progress(rank, "timed steps")

    # ---- timed: device-resident series, CUDA events on the context's stream
    logs, ms = [], []
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for i in range(args.steps):
            flush_l2(i)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            disc, log = ctx.palmad_device(d_x.data_ptr(), n, args.minL, args.maxL)
            e1.record(st)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            logs.append(log)
    torch.cuda.synchronize()
    barrier(world)
    clocks = clk.summary()
    value, step_ms = replica_value(world, pairs, float(np.mean(ms)))

    _progress(rank, "end-to-end steps")
    # ---- end to end: host series through paddi_palmad (H2D inside the call)
    e2e_ms = []
    barrier(world)
    for i in range(max(1, args.steps)):
        flush_l2(i)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        d2, l2 = ctx.palmad(h_x.numpy(), args.minL, args.maxL)
        e1.record(st)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    e2e_step = reduce_max(world, float(np.mean(e2e_ms)))
    e2e_value = world * pairs / (e2e_step / 1e3)
    n_att = len(logs[-1])
    d2h = n_att * 152  # one attempt result record per attempt

    # ---- roofline of the dominant kernel group (refine or phase 1)
    last = logs[-1]
    tot = {k: sum(e[k] for e in last) for k in ("ms_stats", "ms_phase1", "ms_refine",
                                              "ms_select")}
    hbm, bf16, bf16_s, src = load_peaks()
    # dominant kernel: the dense refine.  Tensor-core attempts (split FP16/BF16)
    # and FP32 attempts are reported separately; the line's roofline is the
    # tensor-core one when it ran.
    tc = [e for e in last if e["refine_kernel"] in (2, 3)]
    f32 = [e for e in last if e["refine_kernel"] == 1]

    def rate(es):
        # the refine launches alone (the rounds' candidate re-compaction excluded)
        ms = sum(e["ms_refine_kernel"] for e in es)
        fl = sum(2.0 * e["m"] * e["refine_pairs"] for e in es)
        return (fl / (ms / 1e3) / 1e12 if ms > 0 else 0.0), ms

    def live_rate(es):
        ms = sum(e["ms_refine_kernel"] for e in es)
        fl = sum(2.0 * e["m"] * e["refine_live_pairs"] for e in es)
        return fl / (ms / 1e3) / 1e12 if ms > 0 else 0.0

    if tc:
        achieved, ms_tc = rate(tc)
        peak = bf16 / 3.0  # three 16-bit products per FP32-accurate product
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": REFINE_TRAFFIC_BYTES,
                "traffic_launch": REFINE_TRAFFIC_LAUNCH, "kernel": "k_refine_umma",
                "peak_source": f"bf16 dense {src} {bf16} TFLOP/s / 3 (split operands issue 3 MMAs)",
                "work": "2*m FLOP per (candidate, window) pair evaluated",
                "kernel_ms_per_step": ms_tc, "attempts": len(tc),
                "live_pairs_achieved": live_rate(tc),
                "live_pairs_note": "pairs whose candidate was still unpruned when its tile "
                                   "started (the rest are dead rows of a 16-candidate tile)"}
    else:
        achieved, ms32 = rate(f32)
        peak = 148 * 128 * 2 * 1.965e9 / 1e12  # FP32 FMA, nominal
        roof = {"bound": "fp32-alu", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": None, "kernel": "k_refine_fp32",
                "peak_source": "nominal FP32 FMA peak (no measured figure)",
                "work": "2*m FLOP per (candidate, window) pair evaluated",
                "kernel_ms_per_step": ms32, "attempts": len(f32)}
    roof["phase_ms"] = tot
    # phase 1 (diagonal-strip candidate selection on CUDA cores): 8 FLOP per
    # (row, diagonal) pair walked (two covariance-update FMAs, the pair test,
    # counted as in the reference's distance formula), over the phase-1 time
    # (the kernel plus a 2 MB flag reset), against the nominal FP32 peak at the
    # clock sampled during the run
    p1_pairs = sum(e["p1_pairs"] for e in last)
    p1_ms = tot["ms_phase1"]
    mhz = (clocks.get("sm_mhz") or 1965.0)
    p1_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12
    p1_ach = 8.0 * p1_pairs / (p1_ms / 1e3) / 1e12 if p1_ms > 0 else 0.0
    roof["phase1"] = {"bound": "fp32", "achieved": p1_ach, "peak": p1_peak, "unit": "TFLOP/s",
                      "frac": p1_ach / p1_peak, "kernel": "k_phase1",
                      "peak_source": f"nominal FP32 FMA peak, 148 SMs x 128 lanes x 2 at {mhz:.0f} "
                                     "MHz (no measured FP32 figure)",
                      "work": "8 FLOP per (row, diagonal) pair walked",
                      "pairs_per_step": p1_pairs, "kernel_ms_per_step": p1_ms}
    if tc and f32:
        a32, ms32 = rate(f32)
        roof["fp32_part"] = {"achieved": a32, "ms_per_step": ms32, "attempts": len(f32)}
    launches = sum(e["n_launches"] for lg in logs for e in lg)

    line = {"metric": metric_name(args),
            "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": ("f16x3->f32" if any(e["refine_kernel"] == 3 for e in last) else
                      "bf16x3->f32" if tc else "f32"), "data": "synthetic",
            "config": {"workload": name,
                       "n": args.n, "minL": args.minL, "maxL": args.maxL,
                       "distance": args.dist, "r_policy": args.r_policy,
                       "l2": "flushed between steps (512 MB write)",
                       "parallelism": f"replicas x{world}", "attempts_per_step": n_att},
            "roofline": roof, "clocks": clocks,
            "e2e": {"value": e2e_value, "unit": "pairs/s", "h2d_bytes_per_step": 4 * n,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_step},
            "gpu_launches": launches}
    # the plain form of the headline comparison: FP32 CUDA-core refine with
    # the reference's MERLIN schedule (same kernels otherwise), one timed run
    if not args.no_plain_form:
        _progress(rank, "plain FP32 form")
        with P.Context(device=local, distance_kernel=P.DIST_FP32, r_policy=P.R_MERLIN) as c2:
            c2.reserve(n, args.maxL)
            s2 = torch.cuda.ExternalStream(c2.stream)
            c2.palmad_device(d_x.data_ptr(), n, args.minL, min(args.maxL, args.minL + 8))
            flush_l2(0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s2)
            dpl, lpl = c2.palmad_device(d_x.data_ptr(), n, args.minL, args.maxL)
            e1.record(s2)
            e1.synchronize()
            ms_plain = reduce_max(world, e0.elapsed_time(e1))
        same = [(q.ind, q.dist) for q in dpl] == [(q.ind, q.dist) for q in disc]
        line["plain_form"] = {"what": "FP32 CUDA-core refine + MERLIN r-schedule",
                              "ms_per_step": ms_plain, "attempts": len(lpl),
                              "speedup_of_headline": ms_plain / step_ms,
                              "same_discords": same}
    # the form the metric names: split-BF16 tensor-core refine with the same r
    # policy (the headline's AUTO form runs split FP16), one timed run
    if not args.no_plain_form and args.dist == "auto":
        _progress(rank, "split-BF16 form")
        with P.Context(device=local, distance_kernel=P.DIST_SPLIT_BF16, r_policy=rp) as c3:
            c3.reserve(n, args.maxL)
            s3 = torch.cuda.ExternalStream(c3.stream)
            c3.palmad_device(d_x.data_ptr(), n, args.minL, min(args.maxL, args.minL + 8))
            flush_l2(0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s3)
            dbf, lbf = c3.palmad_device(d_x.data_ptr(), n, args.minL, args.maxL)
            e1.record(s3)
            e1.synchronize()
            ms_bf = reduce_max(world, e0.elapsed_time(e1))
        line["bf16_form"] = {"what": "split-BF16 tensor-core refine (three BF16 products), "
                                     f"{args.r_policy} r", "ms_per_step": ms_bf,
                             "attempts": len(lbf),
                             "same_discords": [(q.ind, q.dist) for q in dbf] ==
                                              [(q.ind, q.dist) for q in disc],
                             "speedup_over_plain": (line["plain_form"]["ms_per_step"] / ms_bf
                                                    if "plain_form" in line else None)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        _progress(rank, "CPU baseline")
        cb = cpu_reference(cpu_sample_of(x, args), 1, 0, min(host_threads(), 64), args.minL)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        line["cpu_baseline"]["like_for_like"] = False
        if args.workload == "palmad":
            line["cpu_baseline"]["full_length"] = full_length_point(ctx, st, x, disc, args)
            line["reference_gpu"] = reference_gpu_point(x, disc, args, lpl if not
                                                        args.no_plain_form else None)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["paddi", "reference"], default="paddi")
    ap.add_argument("--dist", choices=["auto", "fp32", "bf16", "fp16"], default="auto")
    ap.add_argument("--r-policy", choices=["merlin", "learned", "bound"], default="learned")
    ap.add_argument("--no-plain-form", action="store_true",
                    help="skip timing the plain FP32 + MERLIN form beside the headline")
    ap.add_argument("--workload", choices=["palmad", "large"], default="palmad",
                    help="palmad: n=2^21, L=64..512 (the headline); large: ECG-like n=2^27, "
                         "L=128..384, CPU sample from the first 2^22 points")
    ap.add_argument("--n", type=int, default=0)
    ap.add_argument("--minL", type=int, default=0)
    ap.add_argument("--maxL", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_paddi(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
