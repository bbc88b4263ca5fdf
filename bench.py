"""Benchmark of the per-step dynamics path on B200.

`python bench.py --gpus N --steps K --warmup W [--impl ours|reference] [--workload c0|c1|c2|c3|c3-f64]`

The default workload is the mixed-size batch (4096 worlds of 8..8192 bodies, mixed precision), on
which the headline metric is quoted; beside it the line carries the plain path (every world FP64,
alone, one world per launch) and, at N = 1, a served sweep (Poisson request streams of such worlds
with log-uniform step counts through the native request loop, p50/p99 latency).

A step is one Mechanism::step of the whole workload (every body advanced by dt). `value` is
body-steps/s from CUDA events on the library's stream with the state resident in HBM; `e2e` is the
same metric through the public API with page-locked host buffers: each step the dynamic state
(pose, momentum) copied in, the step, the state read back, all inside the timed region. The
explicit worlds and the two halves of the implicit ones sit in three handles on streams of their
own, each driven by a host thread, so one's copies overlap the others' steps (`e2e.one_handle`: one handle, one thread;
`e2e.records`: whole body records). Under torchrun each rank steps its own
replica of the workload (independent worlds: weak scaling, no collective in the data path); the
timing is the max over ranks.

--impl reference times the reference algorithm's CPU implementation on the host cores. The
reference (a Rust/Vulkan workspace) cannot be built here, so that arm runs the C++ f64
restatement of its functions (`cpu_baseline.kind = "port"`).
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from exgame_b200 import _lib, autotune, scenarios, sharding  # noqa: E402
from exgame_b200.abi import (BODY_DTYPE, GRAVITY_OFF, NEWTON, NEWTON_NS_PIVOT, PRECISION_F64,  # noqa: E402
                             PRECISION_MIXED, PRECISION_MIXED_FAST)

METRIC = "body-steps/s"
WORLDS = 4096      # config-3 batch size (--worlds)
SHARD = False      # --shard: one batch split over the ranks instead of one batch per rank
NS_PIVOT = False   # --ns-pivot: Newton-Schulz pivot inverses on the implicit worlds
WORLD_SIZE = 1
# DRAM bytes (read + write) of the Newton step over its algorithmic bytes, measured by ncu on one
# step of the 1024-world batch (28.33 GB against 15.62 GB); the Newton step's traffic grows with the
# islands' Newton iterations as its algorithmic bytes do, so roofline.traffic is this ratio times the
# timed step's algorithmic bytes.
NEWTON_TRAFFIC_RATIO = 28.33 / 15.62
NEWTON_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one Newton step of the first 1024 "
                         "worlds of this batch: 28.33 GB against its 15.62 GB of algorithmic bytes, ratio 1.81, "
                         "times this step's algorithmic bytes")
FP64_FMA_PER_SM_CLK = 64
FP32_FMA_PER_SM_CLK = 128


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def _with_flag(p, flag):
    q = p.copy()
    q["newton_flags"] = int(q["newton_flags"]) | flag
    return q


def workload(name, rank):
    """(list of (bodies, joints, params) worlds stepped together, config dict)"""
    if name == "c0":
        b, j, p, _ = scenarios.config0(seed=rank)
        cfg = {"workload": "1024 point masses, Plummer eps 0.05, LieEuler, dt 1e-3, f64 (config 0)",
               "bodies": 1024, "worlds": 1, "dtype": "f64"}
        return [(b, j, p)], cfg
    if name == "c1":
        b, j, p, _ = scenarios.config1(seed=1 + rank)
        cfg = {"workload": "256-body box chain, 765 joints, implicit Newton tol 1e-10, dt 1e-2, f64 (config 1)",
               "bodies": 256, "worlds": 1, "dtype": "f64"}
        return [(b, j, p)], cfg
    if name == "c2":
        (gb, gj, gp), (cb, cj, cp), _ = scenarios.config2_parts(seed=2 + rank, precision=PRECISION_MIXED,
                                                                exact_jacobian=True)
        cfg = {"workload": "65,536-body gravity (ball R 1000, LieEuler) + 16 x 256-body chains (Newton tol 1e-10), "
                           "dt 1e-3, mixed precision (config 2)", "bodies": len(gb) + len(cb), "worlds": 2,
               "dtype": "f32 forces / f64 state"}
        return [(gb, gj, gp), (cb, cj, cp)], cfg
    if name in ("c3", "c3-f64"):
        prec = PRECISION_MIXED if name == "c3" else PRECISION_F64
        nw = WORLDS
        if SHARD:  # one batch for the whole job, each rank its body-balanced share (strong scaling)
            sizes = scenarios.config3_sizes(nw, seed=3)
            mine = set(sharding.rank_share(sizes, rank, WORLD_SIZE))
            allw = scenarios.config3_worlds(nw, seed=3, precision=prec, exact_jacobian=bool(prec),
                                            only=sorted(mine))
            worlds = allw
        else:  # each rank its own seeded batch (weak scaling)
            worlds = scenarios.config3_worlds(nw, seed=3 + rank, precision=prec, exact_jacobian=bool(prec))
        if NS_PIVOT and prec:  # Newton-Schulz pivot inverses on the implicit worlds
            worlds = [(b, j, _with_flag(p, NEWTON_NS_PIVOT) if int(p["integrator"]) == NEWTON else p)
                      for b, j, p in worlds]
        n = sum(len(b) for b, _, _ in worlds)
        cfg = {"workload": f"{nw} independent worlds, body counts log-uniform in [8, 8192]: gravity worlds "
                           "(LieEuler, dt 1e-3) and random joint trees (Newton tol 1e-10, dt 1e-2), one batched launch "
                           "set per step, " + ("mixed precision, exact mid-point Newton matrix" if prec else "f64")
                           + " (config 3)",
               "bodies": n, "worlds": len(worlds), "dtype": "f32 forces / f64 state" if prec else "f64",
               "pivot_inverse": ("Newton-Schulz (warm-started, FP32 steps, FP64 correction)" if NS_PIVOT and prec
                                 else "FP64 Gauss-Jordan")}
        return worlds, cfg
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            parts = [x.strip() for x in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if parts[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def time_steps(dev, worlds, steps, flush):
    """Per-step device time (CUDA events on the library stream), L2 flushed between steps."""
    import torch
    stream = torch.cuda.ExternalStream(dev.stream())
    total = 0.0
    for _ in range(steps):
        flush()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for w in worlds:
            w.step(1)
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b) / 1e3
    return total


def dominant_kernel(dev, cfg_name, parts, steps, bench_worlds):
    """Profile a pass of `steps` steps; pick the kernel kind with the largest device time.
    Returns (kind, total_ms, launches, algorithmic flops per launch or None, bound, label)."""
    dev.profile(True)
    for _ in range(steps):
        for w in bench_worlds:
            w.step(1)
    kinds = {0: "all-pairs gravity", 1: "joint laws", 2: "explicit integrate", 3: "Newton island kernel",
             4: "body charges / world twists", 5: "Newton wave rounds"}
    per = {k: dev.profile_read(k) for k in kinds}
    dev.profile(False)
    # the two Newton schedules are one step of the implicit worlds: time them together
    newton = (per[3][0] + per[5][0], steps)
    cand = {0: per[0], 1: per[1], 2: per[2], 3: newton, 4: per[4]}
    kind = max(cand, key=lambda k: cand[k][0])
    ms, nl = cand[kind]
    flops, bound = None, "fp64"
    if kind == 0:
        pairs = 0.0
        for b, _, p in parts:
            if int(p["gravity_law"]) != GRAVITY_OFF and len(b) > 1:
                pairs += float(len(b)) ** 2
        flops = 20.0 * pairs
        bound = "fp32" if int(parts[0][2]["precision"]) != PRECISION_F64 else "fp64"
    label = kinds[kind] + (f" ({20} flop per directed pair)" if kind == 0 else "")
    if kind == 3:
        label = "Newton step of the implicit islands (island kernel + wave rounds)"
    shares = {kinds[k]: per[k][0] for k in kinds}
    return kind, ms, nl, flops, bound, label, shares


# Algorithmic bytes of one Newton iteration, FP32 Jacobian blocks: per joint 40 floats in
# (2 poses, 2 twists, dt, warp, 10 params) and 12 + 288 out; per dynamic body motor 8, twist 6 and
# wrench 6 in, 36 mass + 6 rhs + 6 scale out; per tree edge 3 x 36 factor floats.
NEWTON_BYTES_PER_JOINT = (40 + 300) * 4
NEWTON_BYTES_PER_BODY = (20 + 48) * 4
NEWTON_BYTES_PER_EDGE = 3 * 36 * 4


def newton_bytes_last_step(batch, parts):
    """Algorithmic bytes the implicit worlds moved in the last step (iterations x per-iteration bytes)."""
    total, iters = 0.0, 0
    for k, (b, j, p) in enumerate(parts):
        if int(p["integrator"]) != NEWTON:
            continue
        st = batch.world_stats(k) if hasattr(batch, "world_stats") else batch.stats()
        it = int(st["last_newton_iterations"])
        iters += it
        dyn = int((b["kinematic"] == 0).sum())
        total += it * (len(j) * NEWTON_BYTES_PER_JOINT + dyn * NEWTON_BYTES_PER_BODY
                       + max(dyn - 1, 0) * NEWTON_BYTES_PER_EDGE)
    return total, iters


WAVE_HOST_ROUNDS = 0  # --wave-host-rounds: profiler-friendly wave rounds (same arithmetic)


def make_worlds(dev, parts):
    ws = [_lib.DeviceWorld(dev, *parts[0])] if len(parts) == 1 else [_lib.DeviceBatch(dev, parts)]
    if WAVE_HOST_ROUNDS:
        for w in ws:
            w.set_option(_lib.DeviceWorld.OPT_WAVE_HOST_ROUNDS, 1)
    return ws


def plain_path(dev, parts, flush, passes=1, reference_matrix=False):
    """The plain path: every world FP64 and alone, one world per launch (a step of the workload is
    one exg_world_step per world). Returns body-steps/s over `passes` passes after one warm pass.
    The Newton matrix is the batch's own unless `reference_matrix` (the reference's -half^2 pose
    factor, which converges in more iterations to the same step)."""
    import torch
    stream = torch.cuda.ExternalStream(dev.stream())
    worlds = []
    for b, j, p in parts:
        q = p.copy()
        q["precision"] = PRECISION_F64
        if reference_matrix:
            q["newton_flags"] = 0
        worlds.append(_lib.DeviceWorld(dev, b, j, q))
    for w in worlds:
        w.step(1)
    n = sum(w.n for w in worlds)
    total = 0.0
    for _ in range(passes):
        flush()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for w in worlds:
            w.step(1)
        b.record(stream)
        b.synchronize()
        total += a.elapsed_time(b) / 1e3
    for w in worlds:
        w.close()
    return n * passes / total


def run_ours(args, rank, world_size, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    dev = _lib.Device(local_rank)
    parts, cfg = workload(args.workload, rank)
    worlds = make_worlds(dev, parts)
    # launch shapes only, timed on this workload's own steps: results do not change. Tuning
    # advances the worlds, so their initial state is put back afterwards: the warm-up and timed
    # steps are then steps 1..W+K from the initial state, the steps the reference arm times.
    tuning = None
    if args.autotune:
        initial = worlds[0].state()
        tuning = autotune.autotune(dev, workload=worlds[0], steps=2, cache=args.tuning_cache)
        worlds[0].set_state(initial)
        del initial
    n_bodies = sum(len(b) for (b, _, _) in parts)
    flush_buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2

    def flush():
        flush_buf.zero_()

    for _ in range(args.warmup):
        for w in worlds:
            w.step(1)
    dev.synchronize()
    if world_size > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = dev.kernel_launches()
    with ClockSampler(local_rank) as clk:
        time.sleep(0.3)
        t_dev = time_steps(dev, worlds, args.steps, flush)
        time.sleep(0.3)
    launches = dev.kernel_launches() - launches0
    torch.cuda.synchronize()
    t = t_dev
    dist = None
    if world_size > 1:
        import torch.distributed as dist
        t = sharding.max_over_ranks(t, dist, device="cuda")
        dist.barrier()
    total_bodies = sharding.sum_over_ranks(n_bodies, dist, device="cuda") if world_size > 1 else n_bodies
    value = total_bodies * args.steps / t

    # end to end through the public API, page-locked host buffers as a serving host keeps them:
    # the dynamic state (pose, momentum) in, one step, the state out (exg_world_set/get_state);
    # beside it the same with whole records (exg_world_set/get_bodies)
    def end_to_end(alloc, get, put):
        host = []
        for w in worlds:
            h = alloc(w.n)
            get(w, h)
            host.append(h)
        nbytes = sum(h.nbytes for h in host)
        dev.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            for w, h in zip(worlds, host):
                put(w, h)
                w.step(1)
                get(w, h)
        dev.synchronize()
        t_e = time.perf_counter() - t0
        if world_size > 1:
            t_e = sharding.max_over_ranks(t_e, dist, device="cuda")
        return {"value": total_bodies * args.steps / t_e, "unit": METRIC, "h2d_bytes_per_step": int(nbytes),
                "d2h_bytes_per_step": int(nbytes), "steps": args.steps}

    def end_to_end_overlapped():
        # the same state loop on --e2e-handles handles with streams of their own
        # (EXG_OPT_OWN_STREAM): the explicit worlds, and the implicit ones in the remaining parts;
        # each handle is driven by its own host thread, so one handle's copies run while the others
        # step
        implicit = [p for p in parts if int(p[2]["integrator"]) == NEWTON]
        k = max(1, args.e2e_handles - 1)  # the explicit worlds on one handle, the implicit ones in k parts
        groups = [[p for p in parts if int(p[2]["integrator"]) != NEWTON]] + [implicit[i::k] for i in range(k)]
        if not all(groups):
            return None
        hs = [_lib.DeviceBatch(dev, g) for g in groups]
        for h in hs:
            h.set_option(_lib.DeviceWorld.OPT_OWN_STREAM, 1)
            h.step(1)  # structure and graphs built before timing
        bufs = [_lib.host_state(h.n) for h in hs]
        for h, b in zip(hs, bufs):
            h.state(out=b)
        dev.synchronize()
        go = threading.Barrier(len(hs) + 1)

        def drive(h, b):
            go.wait()
            for _ in range(args.steps):
                h.set_state(b)
                h.step(1)
                h.state(out=b)

        threads = [threading.Thread(target=drive, args=(h, b)) for h, b in zip(hs, bufs)]
        for t in threads:
            t.start()
        go.wait()
        t0 = time.perf_counter()
        for t in threads:
            t.join()
        dev.synchronize()
        t_e = time.perf_counter() - t0
        for h in hs:
            h.close()
        if world_size > 1:
            t_e = sharding.max_over_ranks(t_e, dist, device="cuda")
        nbytes = sum(b.nbytes for b in bufs)
        return {"value": total_bodies * args.steps / t_e, "unit": METRIC, "h2d_bytes_per_step": int(nbytes),
                "d2h_bytes_per_step": int(nbytes), "steps": args.steps,
                "transfer": f"dynamic state in and out every step; {len(hs)} handles on their own streams (the "
                            f"explicit worlds, the implicit ones in {len(hs) - 1} parts), one host thread each"}

    one = end_to_end(_lib.host_state, lambda w, h: w.state(out=h), lambda w, h: w.set_state(h))
    one["transfer"] = "dynamic state (pose, momentum: 112 B per body) in and out every step, one handle"
    both = end_to_end_overlapped()
    e2e = dict(both) if both else dict(one)
    e2e["one_handle"] = one
    e2e["records"] = end_to_end(_lib.host_bodies, lambda w, h: w.bodies(out=h), lambda w, h: w.set_bodies(h))
    e2e["records"]["transfer"] = "whole body records (208 B per body) in and out every step"

    # dominant kernel, timed live with events on the library stream over a profiled pass
    kind, ms, nl, flops, bound, label, shares = dominant_kernel(dev, args.workload, parts, args.steps, worlds)
    peaks, src = load_peaks()
    sm_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    avg_s = ms / 1e3 / max(nl, 1)
    if kind == 3:  # the Newton island step: HBM-bound by its algorithmic bytes
        nbytes, iters = newton_bytes_last_step(worlds[0], parts)
        hbm = float(peaks["hbm_gbs"])
        roofline = {"bound": "hbm", "achieved": nbytes / avg_s / 1e9, "peak": hbm, "unit": "GB/s",
                    "frac": nbytes / avg_s / 1e9 / hbm, "traffic": NEWTON_TRAFFIC_RATIO * nbytes,
                    "traffic_source": NEWTON_TRAFFIC_SOURCE, "kernel": label,
                    "algorithmic_bytes_per_launch": nbytes, "newton_iterations_summed_over_islands": iters,
                    "avg_launch_us": avg_s * 1e6, "launches": nl, "device_ms_by_kernel": shares,
                    "peak_source": f"{src} HBM copy bandwidth (MEASURED_PEAKS.json hbm_gbs), of {src}"}
    else:
        per_clk = FP64_FMA_PER_SM_CLK if bound == "fp64" else FP32_FMA_PER_SM_CLK
        peak_tflops = 2.0 * per_clk * sms * sm_mhz * 1e6 / 1e12
        roofline = {"bound": bound, "achieved": (flops / avg_s / 1e12) if flops else None, "peak": peak_tflops,
                    "unit": "TFLOP/s", "frac": (flops / avg_s / 1e12 / peak_tflops) if flops else None,
                    "traffic": None, "kernel": label, "avg_launch_us": avg_s * 1e6, "launches": nl,
                    "device_ms_by_kernel": shares,
                    "peak_source": f"nominal {per_clk} {bound.upper()} FMA/clk/SM x {sms} SMs at the {src} max SM "
                                   f"clock {sm_mhz:.0f} MHz (no tensor-core or copy peak applies to this kernel)"}
    grav = gravity_roofline(dev, parts, worlds, sms, sm_mhz) if kind != 0 else None
    if grav:
        roofline["gravity"] = grav
        if int(parts[0][2]["precision"]) == PRECISION_MIXED:
            # the single-FP32 form of the same kernel on the same gravity worlds, for comparison
            gparts = []
            for b, j, p in parts:
                if int(p["gravity_law"]) != GRAVITY_OFF and len(b) > 1:
                    q = p.copy()
                    q["precision"] = PRECISION_MIXED_FAST
                    gparts.append((b, j, q))
            gw = make_worlds(dev, gparts)
            fast = gravity_roofline(dev, gparts, gw, sms, sm_mhz)
            for w in gw:
                w.close()
            fast["note"] += "; MIXED_FAST (single FP32 positions), for comparison"
            roofline["gravity_fast"] = fast
    plain = None
    if args.plain and len(parts) > 1:
        plain = {"value": plain_path(dev, parts, flush), "unit": METRIC,
                 "sample": "every world FP64 with the batch's Newton matrix, stepped alone, one exg_world_step "
                           "per world, one pass after a warm pass (device time, L2 flushed before the pass)",
                 "reference_matrix": {
                     "value": plain_path(dev, parts, flush, reference_matrix=True), "unit": METRIC,
                     "sample": "the same with the reference's Newton matrix (pose factor -half^2), which takes more "
                               "Newton iterations to the same converged step"}}
    err = error_vs_oracle(dev, parts, args.error_steps) if args.error_steps > 0 and rank == 0 else None
    return {
        "value": value, "t": t, "e2e": e2e, "roofline": roofline, "cfg": cfg, "launches": launches,
        "clocks": clk.summary(), "n_bodies": n_bodies, "plain": plain, "dev": dev, "tuning": tuning, "error": err,
    }


def gravity_roofline(dev, parts, worlds, sms, sm_mhz):
    """The all-pairs gravity kernel of the same workload, timed alone over a profiled pass."""
    pairs = sum(float(len(b)) ** 2 for b, _, p in parts if int(p["gravity_law"]) != GRAVITY_OFF and len(b) > 1)
    if pairs == 0:
        return None
    dev.profile(True)
    for w in worlds:
        w.step(1)
    ms, nl = dev.profile_read(0)
    dev.profile(False)
    mixed = int(parts[0][2]["precision"]) != PRECISION_F64
    per_clk = FP32_FMA_PER_SM_CLK if mixed else FP64_FMA_PER_SM_CLK
    peak = 2.0 * per_clk * sms * sm_mhz * 1e6 / 1e12
    achieved = 20.0 * pairs / (ms / 1e3 / max(nl, 1)) / 1e12
    return {"bound": "fp32" if mixed else "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "avg_launch_us": ms * 1e3 / max(nl, 1),
            "flops_per_launch": 20.0 * pairs, "note": "20 flop per directed pair"}


def serve_sweep(dev, rates, n_requests, pool_size, tick, rank):
    """Config 4: Poisson request streams through the native request loop (exg_server_*). Each
    request is a world drawn from a pool of config-3 worlds (log-uniform 8..8192 bodies, half
    gravity, half trees; mixed precision) with a step count log-uniform in [10, 1000]. Latency is
    measured from each request's scheduled arrival. Beside it, the plain path served FIFO: one world
    at a time in FP64 with the reference's Newton matrix, from per-world step times measured alone."""
    import torch
    rng = np.random.default_rng(44 + rank)
    pool = scenarios.config3_worlds(pool_size, seed=40 + rank, precision=PRECISION_MIXED, exact_jacobian=True)
    stream = torch.cuda.ExternalStream(dev.stream())
    # plain path: FP64 step time of every pool world alone
    plain_step_s = []
    for b, j, p in pool:
        q = p.copy()
        q["precision"] = PRECISION_F64
        q["newton_flags"] = 0
        w = _lib.DeviceWorld(dev, b, j, q)
        w.step(1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        w.step(2)
        e1.record(stream)
        e1.synchronize()
        plain_step_s.append(e0.elapsed_time(e1) / 2e3)
        w.close()
    max_b = max(len(b) for b, _, _ in pool)
    out = []
    for rate in rates:
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
        picks = rng.integers(0, len(pool), n_requests)
        steps = np.exp(rng.uniform(math.log(10), math.log(1000), n_requests)).astype(np.int64)
        srv = _lib.Server(dev, hbm_budget_bytes=150 * 10**9, max_bodies=max(4 << 20, 2 * max_b),
                          max_joints=max(12 << 20, 6 * max_b), max_worlds=2048, precision=PRECISION_MIXED,
                          steps_per_tick=tick)
        ids, lag = [], []
        t0 = time.perf_counter()
        for k in range(n_requests):
            dt = t0 + arrivals[k] - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            b, j, p = pool[picks[k]]
            ids.append(srv.submit(b, j, p, int(steps[k])))
            lag.append(time.perf_counter() - (t0 + arrivals[k]))
        lat = []
        for k, rid in enumerate(ids):
            _, info = srv.wait(rid, timeout_ms=600000)
            lat.append(float(info["latency_s"]) + lag[k])
        t_end = time.perf_counter()
        st = srv.stats()
        srv.close()
        bs = float(sum(len(pool[picks[k]][0]) * int(steps[k]) for k in range(n_requests)))
        # plain path: FIFO, one world at a time
        done, plat = 0.0, []
        for k in range(n_requests):
            start = max(arrivals[k], done)
            done = start + steps[k] * plain_step_s[picks[k]]
            plat.append(done - arrivals[k])
        out.append({
            "rate_req_s": rate, "requests": n_requests, "body_steps": bs,
            "body_steps_per_s": bs / (t_end - t0), "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "max_submit_lag_s": float(max(lag)),
            "peak_running": st["peak_running"], "ticks": st["ticks"],
            "plain_fifo": {"body_steps_per_s": bs / done, "p50_latency_s": float(np.percentile(plat, 50)),
                           "p99_latency_s": float(np.percentile(plat, 99))},
        })
    return {"pool_worlds": len(pool), "steps_per_tick": tick, "pools": 2, "sweep": out,
            "plain_fifo_model": "FIFO queue, one world at a time, service = steps x that world's FP64 step time "
                                "measured alone (device time)"}


def error_vs_oracle(dev, parts, steps):
    """The timed path's error against the f64 oracle on a sample of the workload's worlds: the same
    worlds with the same parameters in a batch of their own (a world steps bit for bit the same in
    every batch), `steps` steps on the device and in the oracle from the same initial state. Per
    world: pose error per body relative to max(1, |pose|), the worst body; momentum relative to the
    world's largest |p|; energy of the two states by the oracle's energy function."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    oracle_lib.lib().orc_set_threads(os.cpu_count() or 1)
    grav = [k for k, (b, _, p) in enumerate(parts) if int(p["integrator"]) != NEWTON and len(b) <= 1024]
    tree = [k for k, (b, _, p) in enumerate(parts) if int(p["integrator"]) == NEWTON and len(b) <= 48]
    if len(parts) <= 2:  # single-world workloads: the worlds themselves when small enough
        grav = [k for k, (b, _, p) in enumerate(parts) if len(b) <= 4096]
        tree = []
    pick = []
    for sel in (grav, tree):
        sel = sorted(sel, key=lambda k: len(parts[k][0]))
        if sel:
            pick += [sel[int(round(q * (len(sel) - 1)))] for q in (0.0, 0.5, 0.8, 1.0)]
    pick = sorted(set(pick))
    if not pick:
        return None
    sample = [parts[k] for k in pick]
    batch = _lib.DeviceBatch(dev, sample)
    batch.step(steps)
    got = [batch.world_bodies(i) for i in range(len(sample))]
    batch.close()
    t0 = time.perf_counter()
    ows = []
    for b, j, p in sample:
        q = p.copy()
        q["precision"] = PRECISION_F64
        ows.append(oracle_lib.OracleWorld(b, j, q))
    oracle_lib.worlds_step(ows, steps)
    t_orc = time.perf_counter() - t0
    worst = {"pose_rel": 0.0, "momentum_rel": 0.0, "energy_rel": 0.0}
    per = []
    for (b, j, p), g, ow in zip(sample, got, ows):
        want = ow.bodies()
        pose = float((np.abs(g["pose"] - want["pose"]).max(axis=1) /
                      np.maximum(1.0, np.abs(want["pose"]).max(axis=1))).max())
        pm = float(np.abs(want["momentum"]).max())
        mom = float(np.abs(g["momentum"] - want["momentum"]).max() / max(pm, 1e-300))
        e_w = ow.energy()
        e_g = oracle_lib.OracleWorld(g, j, ow._p).energy()
        en = abs(e_g - e_w) / max(abs(e_w), 1e-300)
        per.append({"bodies": len(b), "kind": "tree" if int(p["integrator"]) == NEWTON else "gravity",
                    "pose_rel": pose, "momentum_rel": mom, "energy_rel": en})
        for k, v in (("pose_rel", pose), ("momentum_rel", mom), ("energy_rel", en)):
            worst[k] = max(worst[k], v)
    return dict(worst, steps=steps, tolerance_pose_rel=1e-6, within=worst["pose_rel"] <= 1e-6, worlds=per,
                oracle_seconds=t_orc,
                sample="worlds of the timed workload (gravity up to 1024 bodies, trees up to 48 bodies, at the "
                       "0/50/80/100 % size quantiles of each kind), the timed path's precision and Newton matrix, "
                       "in a batch of their own, against the f64 oracle from the same initial state")


def oracle_sample(parts):
    """The CPU legs' bounded sample of a large batch: every 16th world in size order, so the sample
    has the batch's size distribution. Returns (worlds, description)."""
    if len(parts) <= 64:
        return parts, "the whole workload"
    order = sorted(range(len(parts)), key=lambda k: (len(parts[k][0]), k))
    pick = sorted(order[8::16])
    sample = [parts[k] for k in pick]
    nb = sum(len(b) for b, _, _ in sample)
    tot = sum(len(b) for b, _, _ in parts)
    return sample, (f"{len(sample)} of {len(parts)} worlds (every 16th in size order), {nb} of {tot} bodies "
                    f"({100.0 * nb / tot:.2f} %)")


def cpu_baseline(args, threads):
    """The oracle (C++ f64 restatement) on a bounded sample of the same workload, worlds spread over
    the host threads (OpenMP, largest first)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    L = oracle_lib.lib()
    L.orc_set_threads(int(threads))
    parts, cfg = workload(args.workload, 0)
    parts, desc = oracle_sample(parts)
    parts = sorted(parts, key=lambda x: -len(x[0]))
    worlds = [oracle_lib.OracleWorld(b, j, p) for (b, j, p) in parts]
    n = sum(w.n for w in worlds)
    budget = args.cpu_seconds
    steps, t0 = 0, time.perf_counter()
    while True:
        oracle_lib.worlds_step(worlds, 1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= budget or steps >= 100000:
            break
    return {"value": n * steps / el, "unit": METRIC, "cores": int(threads), "kind": "port",
            "sample": f"{steps} steps of {desc}, on {threads} host threads (worlds in parallel), {el:.1f} s"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c0", "c1", "c2", "c3", "c3-f64"])
    ap.add_argument("--worlds", type=int, default=4096, help="worlds of the config-3 batch")
    ap.add_argument("--autotune", type=int, default=1, help="tune launch shapes on this GPU first")
    ap.add_argument("--tuning-cache", default=None,
                    help="JSON file of tuned launch shapes per GPU and batch-shape bucket: reused on a hit, written on a miss")
    ap.add_argument("--wave-host-rounds", type=int, default=0,
                    help="drive the wave's rounds from the host (for profilers that skip conditional graph nodes)")
    ap.add_argument("--shard", action="store_true",
                    help="split one batch over the ranks by body count (strong scaling) instead of one batch per rank")
    ap.add_argument("--serve-rates", default="100,1000,10000",
                    help="request rates (req/s) of the served sweep at N=1; empty to skip")
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-pool", type=int, default=256)
    ap.add_argument("--serve-tick", type=int, default=16)
    ap.add_argument("--plain", type=int, default=1, help="also time the plain one-world-per-launch FP64 path")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--e2e-handles", type=int, default=4,
                    help="handles of the overlapped end-to-end loop (one for the explicit worlds, the rest split the "
                         "implicit ones)")
    ap.add_argument("--ns-pivot", type=int, default=0,
                    help="1: the implicit worlds invert their pivot blocks by Newton-Schulz (EXG_NEWTON_NS_PIVOT)")
    ap.add_argument("--error-steps", type=int, default=1000,
                    help="steps of the sampled worlds compared with the f64 oracle after the run (0: skip)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    threads = os.cpu_count() or 1
    global WORLDS, SHARD, WORLD_SIZE, WAVE_HOST_ROUNDS, NS_PIVOT
    WORLDS, SHARD, WORLD_SIZE, WAVE_HOST_ROUNDS = args.worlds, args.shard, world_size, args.wave_host_rounds
    NS_PIVOT = bool(args.ns_pivot)

    if args.impl == "reference":
        if rank != 0:
            return
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib
        oracle_lib.lib().orc_set_threads(threads)
        parts, cfg = workload(args.workload, 0)
        parts, desc = oracle_sample(parts)
        parts = sorted(parts, key=lambda x: -len(x[0]))  # largest first over the threads
        sample = f"{args.steps} timed steps after {args.warmup} warm-up steps of {desc}, worlds in parallel"
        worlds = [oracle_lib.OracleWorld(b, j, p) for (b, j, p) in parts]
        n = sum(w.n for w in worlds)
        oracle_lib.worlds_step(worlds, args.warmup)
        t0 = time.perf_counter()
        oracle_lib.worlds_step(worlds, args.steps)
        el = time.perf_counter() - t0
        v = n * args.steps / el
        line = {"metric": METRIC, "value": v, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": cfg["dtype"],
                "data": "synthetic (seeded; the reference publishes no dataset)", "config": cfg,
                "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
                                 "sample": sample + f", {n} bodies"},
                "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world_size > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    r = run_ours(args, rank, world_size, local_rank)
    cpu = cpu_baseline(args, threads) if rank == 0 and world_size == 1 else None
    serving = None
    if rank == 0 and world_size == 1 and args.serve_rates:
        rates = [float(x) for x in args.serve_rates.split(",") if x]
        serving = serve_sweep(r["dev"], rates, args.serve_requests, args.serve_pool, args.serve_tick, rank)
        for s in serving["sweep"]:  # served throughput against the batch rate of the same kind of worlds
            s["fraction_of_batch_value"] = s["body_steps_per_s"] / r["value"]
    if rank == 0:
        line = {
            "metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["t"] / args.steps * 1e3, "higher_is_better": True,
            "scaling": "strong" if args.shard else "weak", "vs_baseline": None, "dtype": r["cfg"]["dtype"],
            "data": "synthetic (seeded; the reference publishes no dataset)",
            "config": dict(r["cfg"], autotune=r["tuning"], parallelism=(f"worlds sharded over {world_size} ranks by body count" if args.shard
                                                  else f"replicas x{world_size} (independent worlds)"),
                           l2="flushed between timed steps (256 MB write)"),
            "e2e": r["e2e"], "gpu_launches": r["launches"], "roofline": r["roofline"], "cpu_baseline": cpu,
            "clocks": r["clocks"], "plain_path": r["plain"], "serving": serving, "error_vs_oracle": r["error"],
        }
        print(json.dumps(line))
    if world_size > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
