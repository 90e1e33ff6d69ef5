#!/usr/bin/env python
"""SCFT inner-loop benchmark: iterations/s on the 128^3, Ns = 200 diblock workload.

Workload (one step = one SCFT iteration): AB diblock melt, 128^3 grid, box
8.0 Rg, f_A = 0.35, chiN = 25, Ns = 200 (70 + 130 contour steps per sweep, two
sweeps), Anderson mixing of depth 10, mixed precision (FP32 propagators and
FFTs; FP64 Q, F, quadrature and Anderson normal equations).  Synthetic seeded
fields (U(-0.05, 0.05) plus a hexagonal-cylinder seed).

Our arm prints one JSON line with the device-timed whole-job rate (`value`),
the end-to-end rate through the public API with host buffers (`e2e`), the
roofline of the propagator step (CUDA events around the sweeps inside the
timed iterations), the CPU baseline (the FP64 oracle on the host cores) and
the SM clocks sampled during the timed region.  At N = 1 it adds the
mixed-vs-FP64 precision check (1000 iterations of both), the FP64 path's rate
on the same workload (`fp64_path`, `mixed_over_fp64`) and the batched blend
workload (64 instances of uneven size as one batch against a loop of
single-instance launches, `batched`).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

For N > 1 each rank runs an independent replica (the single-instance path
does not shard; weak scaling), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

METRIC = "SCFT iter/s at 128³ Ns=200: mixed vs FP64 at |ΔF/F|<1e-6; % HBM roofline"
UNIT = "iter/s"
WORKLOAD = ("diblock128: AB diblock melt 128^3, box 8.0 Rg, f_A=0.35, chiN=25, Ns=200, "
            "Anderson depth 10, mixed precision")
TRIBLOCK = ("triblock256: ABC linear triblock 256^3, box 16 Rg, fractions (0.3, 0.4, 0.3), "
            "chiN AB 30, BC 30, AC 45, Ns=400, Anderson depth 20, mixed precision")
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=128, help="grid extent (128 is the benchmark)")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--precision-iters", type=int, default=1000,
                    help="iterations of the mixed-vs-FP64 comparison (0 = skip)")
    ap.add_argument("--prep", type=int, default=-1,
                    help="setup iterations before warm-up (default: fill the Anderson history)")
    ap.add_argument("--fp64-steps", type=int, default=10,
                    help="timed iterations of the FP64 path for the mixed/FP64 ratio (0 = skip)")
    ap.add_argument("--batch-instances", type=int, default=64,
                    help="instances of the batched blend workload (0 = skip)")
    ap.add_argument("--batch-steps", type=int, default=10)
    ap.add_argument("--scale256", type=int, default=5,
                    help="timed iterations of the 256^3 ABC scale case (0 = skip)")
    ap.add_argument("--batch128", type=int, default=2,
                    help="instances of the 128^3 mixed workload run as one batch (0 = skip)")
    ap.add_argument("--no-cufft", dest="cufft", action="store_false",
                    help="skip the cuFFT (torch.fft) comparison of the propagator step")
    ap.add_argument("--variant", type=int, default=-1,
                    help="pin the propagator kernel variant (0..31) instead of autotuning, e.g. "
                         "so that a profiler run uses the variant the plain run chose")
    ap.add_argument("--workload", choices=["diblock128", "triblock256"], default="diblock128",
                    help="triblock256: the 256^3 ABC scale case (about 75 GB on the device; "
                         "reports the variable-cell stress step instead of the 128^3 extras)")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(n: int, precision: str):
    """DRAM bytes per propagator step from the committed ncu summary, or None."""
    f = ROOT / "profiles" / f"propagator_step_{n}cubed_{precision}.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_step:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.tmp = None

    def start(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.tmp.flush()
        rows = [r.split(",") for r in Path(self.tmp.name).read_text().splitlines() if r.strip()]
        os.unlink(self.tmp.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def oracle_config(n: int):
    from polyswift_plusplus_b200 import workloads as W
    cfg, w = W.diblock128(precision="fp64", n=n)
    return cfg, w


def cpu_baseline_full_iteration(n: int) -> dict:
    """One full FP64 oracle iteration of the same workload on all host threads."""
    import oracle as O
    threads = O.set_threads(cpu_threads())
    cfg, w = oracle_config(n)
    o = O.Oracle(cfg)
    o.restore(w)
    t0 = time.perf_counter()
    o.update(1)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": 1.0 / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"one full FP64 iteration of the {n}^3 workload ({dt:.2f} s wall) by the C "
                      "restatement of the reference dataflow (c2c FFT pairs, OpenMP)"}


FP64_FINISH = 20  # final iterations of a mixed run done in FP64 (precision escalation)


def precision_check(n: int, iters: int, device: int) -> dict:
    """Mixed, escalated and FP64 device paths from the same fields, `iters` iterations each.

    "mixed": every iteration with FP32 sweeps; its F sits on the FP32 noise floor
    of Q (about 1e-6).  "escalated": FP32 sweeps for iters - 20 iterations, then
    the same handle switched to FP64 sweeps (fields and Anderson history carry
    over) for the last 20.  The FP64 and escalated runs are timed end to end on
    the device (the switch's allocation and re-tuning included).
    """
    import numpy as np
    import torch

    from polyswift_plusplus_b200 import workloads as W
    from polyswift_plusplus_b200.scft import ScftSolver
    res = {}
    v64 = -1
    for mode in ("fp64", "mixed", "escalated"):
        cfg, w = W.diblock128(precision="fp64" if mode == "fp64" else "mixed", n=n)
        cfg.device = device
        s = ScftSolver(cfg)
        s.restore(w)
        st = torch.cuda.ExternalStream(s.stream_ptr, device=torch.device("cuda", device))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        if mode == "escalated":
            s.update(iters - FP64_FINISH)
            s.set_precision("fp64")
            if v64 >= 0:
                s.set_variant(v64)  # the FP64 run's tuned variant: no re-tuning at the switch
            s.update(FP64_FINISH)
        else:
            s.update(iters)
        e1.record(st)
        e1.synchronize()
        if mode == "fp64":
            v64 = s.variant()[0]
        res[mode] = (s.scalars(), [s.phi(i) for i in range(len(cfg.fields))], e0.elapsed_time(e1) / 1000.0)
        s.close()
    a, pa, ta = res["fp64"]

    def cmp(mode):
        b, pb, tb = res[mode]
        spec = max(float(np.abs(np.abs(np.fft.fftn(x.reshape(n, n, n))) -
                                np.abs(np.fft.fftn(y.reshape(n, n, n)))).max()) / x.size
                   for x, y in zip(pa, pb))
        return {"dF_over_F": abs(b["free_energy"] - a["free_energy"]) / abs(a["free_energy"]),
                "dF_over_F_total": abs(b["free_energy_nodis"] - a["free_energy_nodis"])
                / abs(a["free_energy_nodis"]),
                "max_dphi": float(max(np.abs(x - y).max() for x, y in zip(pa, pb))),
                "max_d_abs_fft_phi": spec, "F": b["free_energy"], "dh_norm": b["dh_norm"],
                "time_s": tb, "iter_per_s": iters / tb}
    return {"iterations": iters, "F_fp64": a["free_energy"], "dh_norm_fp64": a["dh_norm"],
            "fp64_time_s": ta, "fp64_iter_per_s": iters / ta, "fp64_variant": v64,
            "mixed": cmp("mixed"),
            "escalated": dict(cmp("escalated"), fp64_finish_iterations=FP64_FINISH,
                              speedup_vs_fp64=ta / res["escalated"][2]),
            "note": "max_dphi includes a rigid translation of the pattern (a zero mode of the "
                    "saddle point); max_d_abs_fft_phi is translation invariant"}


def l2_copy_bandwidth(device: int, mbytes: int = 32, copies: int = 64, reps: int = 5) -> float:
    """Copy bandwidth of an L2-resident buffer (read + write bytes per second,
    GB/s): a tensor of `mbytes` MB copied into another `copies` times inside one
    CUDA graph (no launch gaps), replayed `reps` times; both buffers together
    stay well inside the 126 MB L2.  The ceiling for passes whose data stays in
    L2."""
    import torch
    dev = torch.device("cuda", device)
    n = mbytes * (1 << 20) // 4
    a = torch.ones(n, device=dev)
    b = torch.empty(n, device=dev)
    side = torch.cuda.Stream(device=dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        for _ in range(3):
            b.copy_(a)
    torch.cuda.current_stream(dev).wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(copies):
            b.copy_(a)
    graph.replay()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        graph.replay()
    e1.record()
    e1.synchronize()
    secs = e0.elapsed_time(e1) / 1000.0
    del graph
    return 2.0 * n * 4 * copies * reps / secs / 1e9


def cufft_comparison(n: int, device: int, reps: int = 3, steps: int = 200) -> dict:
    """The propagator step built from library FFTs, for comparison only: torch.fft
    (cuFFT) r2c and c2r of n^3 FP32 data, unnormalised, with the two real-space
    multiplies by the Boltzmann factors and the multiply by exp(-ds k^2) as
    elementwise kernels, both sweeps at once (a batch of two), q(s+ds) written
    into the stored propagator like the hand-written path.  `steps` steps are
    captured in one CUDA graph and replayed; the figure is device time per step."""
    import torch
    dev = torch.device("cuda", device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(1)
    q0 = torch.rand((2, n, n, n), device=dev, generator=gen) + 0.5
    wf = torch.rand((2, n, n, n), device=dev, generator=gen) * 0.01 + 0.99
    kk = torch.rand((n, n, n // 2 + 1), device=dev, generator=gen) / float(n ** 3)
    slices = torch.empty((steps, 2, n, n, n), device=dev)

    def body():
        cur = q0
        for k in range(steps):
            spec = torch.fft.rfftn(cur * wf, dim=(1, 2, 3), norm="backward")
            spec.mul_(kk)
            torch.mul(torch.fft.irfftn(spec, s=(n, n, n), dim=(1, 2, 3), norm="forward"), wf,
                      out=slices[k])
            cur = slices[k]

    side = torch.cuda.Stream(device=dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        body()  # plans and allocator warm-up
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize(dev)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        body()
    graph.replay()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        graph.replay()
    e1.record()
    e1.synchronize()
    us = e0.elapsed_time(e1) * 1000.0 / (reps * steps)
    del graph, slices
    torch.cuda.empty_cache()
    return {"step_us": us, "steps": steps, "reps": reps,
            "what": f"torch.fft rfftn/irfftn (cuFFT) of two {n}^3 FP32 sweeps per step + three "
                    "elementwise multiplies, CUDA graph of 200 steps, slices stored"}


def fp64_rate(n: int, steps: int, device: int) -> dict:
    """Device-timed iter/s of the plain FP64 path on the same workload and state
    preparation (the comparison the mixed path is quoted against)."""
    import torch

    from polyswift_plusplus_b200 import workloads as W
    from polyswift_plusplus_b200.scft import ScftSolver
    cfg, w = W.diblock128(precision="fp64", n=n)
    cfg.device = device
    s = ScftSolver(cfg)
    s.restore(w)
    s.update(cfg.updater.anderson_start + cfg.updater.anderson_depth + 3)
    st = torch.cuda.ExternalStream(s.stream_ptr, device=torch.device("cuda", device))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    s.update(steps)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    v, _ = s.variant()
    s.close()
    return {"value": steps / (ms / 1000.0), "unit": UNIT, "steps": steps, "kernel_variant": v}


def batched_rate(count: int, steps: int, device: int) -> dict:
    """The batched blend workload: `count` diblock / A-homopolymer instances of
    uneven grid (32..96)^3, chiN and f_A, FP32 sweeps, Anderson depth 10, Ns = 100,
    as one batch (merged sweeps, one graph per iteration) and as a loop of
    single-instance launches; aggregate instance-iterations/s of each."""
    import torch

    from polyswift_plusplus_b200 import workloads as W
    from polyswift_plusplus_b200.scft import ScftBatch, ScftSolver
    items = W.blend_instances(count=count)
    for c, _ in items:
        c.device = device
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b = ScftBatch([c for c, _ in items])
    for i, (_, w) in enumerate(items):
        b.instance(i).restore(w)
    b.update(3)                      # eager iteration, per-class autotune, graph capture
    st = torch.cuda.ExternalStream(b.stream_ptr, device=torch.device("cuda", device))
    torch.cuda.synchronize()
    e0.record(st)
    b.update(steps)
    e1.record(st)
    e1.synchronize()
    ms_batch = e0.elapsed_time(e1)
    _, variants = b.classes()
    launches = b.launches_per_iteration
    b.close()
    ms_loop = 0.0
    for c, w in items:
        s = ScftSolver(c)
        s.restore(w)
        s.update(3)
        st = torch.cuda.ExternalStream(s.stream_ptr, device=torch.device("cuda", device))
        torch.cuda.synchronize()
        e0.record(st)
        s.update(steps)
        e1.record(st)
        e1.synchronize()
        ms_loop += e0.elapsed_time(e1)
        s.close()
    sizes = sorted({c.n[0] for c, _ in items})
    return {"workload": f"blend{count}: {count} AB-diblock/A-homopolymer instances, grids "
                        f"{sizes}^3, chiN~U[12,30], f_A~U[0.2,0.5], phi_h~U[0,0.2], Ns=100, "
                        "FP32 sweeps, Anderson depth 10",
            "value": count * steps / (ms_batch / 1000.0), "unit": "instance-iter/s",
            "single_loop_value": count * steps / (ms_loop / 1000.0),
            "speedup_vs_single_loop": ms_loop / ms_batch, "steps": steps,
            "class_variants": variants, "launches_per_iteration": launches}


def batched128_rate(count: int, steps: int, device: int) -> dict:
    """`count` seeded instances of the 128^3 Ns=200 mixed workload as one batch
    (the mixed-precision batched path: every instance's sweeps in the same
    launches, one graph per iteration); aggregate instance-iterations/s after
    each instance's Anderson history has filled."""
    import torch

    from polyswift_plusplus_b200 import workloads as W
    from polyswift_plusplus_b200.scft import ScftBatch
    cfgs, fields = [], []
    for i in range(count):
        cfg, _ = W.diblock128(precision="mixed")
        cfg.seed = 38383 + i
        cfg.device = device
        hx = W.hex_seed(cfg)
        r = W.random_fields(cfg, 0.05)
        cfgs.append(cfg)
        fields.append([r[0] + hx, r[1] - hx])
    b = ScftBatch(cfgs)
    for i, w in enumerate(fields):
        b.instance(i).restore(w)
    u = cfgs[0].updater
    b.update(u.anderson_start + u.anderson_depth + 3)
    st = torch.cuda.ExternalStream(b.stream_ptr, device=torch.device("cuda", device))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    b.update(steps)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    _, variants = b.classes()
    launches = b.launches_per_iteration
    fe = [sc["free_energy"] for sc in b.scalars()]
    b.close()
    return {"workload": f"{count} seeded instances of diblock128 (seeds 38383..{38383 + count - 1}), "
                        "FP32 sweeps, FP64 Q/F/quadrature/Anderson, as one batch",
            "value": count * steps / (ms / 1000.0), "unit": "instance-iter/s", "steps": steps,
            "class_variants": variants, "launches_per_iteration": launches,
            "free_energy": fe}


def scale256_rate(steps: int, device: int) -> dict:
    """The 256^3 ABC triblock scale case (box 16 Rg, fractions 0.3/0.4/0.3,
    chiN 30/30/45, Ns = 400, mixed precision; about 75 GB on the device):
    device-timed iterations/s and time per propagator step after 3 warm-up
    iterations, autotuned kernel variant.  The iterations are in the workload's
    steepest-descent phase (Anderson starts at iteration 200); the propagator
    sweeps, which dominate, are the same either way."""
    import torch

    from polyswift_plusplus_b200 import workloads as W
    from polyswift_plusplus_b200.scft import ScftSolver
    cfg, w = W.triblock256(precision="mixed")
    cfg.device = device
    s = ScftSolver(cfg)
    s.restore(w)
    s.update(3)
    s.enable_sweep_timing(steps)
    st = torch.cuda.ExternalStream(s.stream_ptr, device=torch.device("cuda", device))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    s.update(steps)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    sweep_ms, sweep_bytes, sweep_steps = s.sweep_timing()
    v, _ = s.variant()
    s.close()
    step_us = 1000.0 * statistics.mean(sweep_ms) / max(sweep_steps, 1) if sweep_ms else None
    return {"workload": TRIBLOCK, "value": steps / (ms / 1000.0), "unit": UNIT, "steps": steps,
            "step_us": step_us, "kernel_variant": v,
            "algorithmic_bytes_per_step": 3 * cfg.n_total * 4}


def run_reference(args, world, rank):
    """The reference's CPU path: its C restatement (the reference itself cannot be
    built), one full FP64 iteration of the same workload per timed step."""
    if world > 1 and rank != 0:
        return
    import oracle as O
    threads = O.set_threads(cpu_threads())
    cfg, w = oracle_config(args.n)
    o = O.Oracle(cfg)
    o.restore(w)
    for _ in range(args.warmup):
        o.propagate_sample(4)          # warm-up: thread pool, FFT plans, page faults
    o.update(1)                        # one untimed full iteration
    samples = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.update(1)
        samples.append(time.perf_counter() - t0)
    o.close()
    t_iter = statistics.mean(samples)
    value = 1.0 / t_iter
    sample = (f"each timed step = one full FP64 iteration of the {args.n}^3 workload (400 "
              "propagator steps of c2c FFT pairs, quadrature, field update), "
              f"{t_iter:.2f} s wall on {threads} threads; warm-up: {args.warmup} short propagator "
              "samples and one full iteration")
    out = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t_iter,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": {"workload": WORKLOAD.replace("mixed precision", "FP64"),
                                           "grid": args.n, "ns": 200},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_ours(args, world, rank, local):
    import torch
    import torch.distributed as dist

    from polyswift_plusplus_b200 import workloads as W
    from polyswift_plusplus_b200.scft import ScftSolver

    torch.cuda.set_device(local)
    tri = args.workload == "triblock256"
    if tri:
        cfg, w = W.triblock256(precision=args.precision)
        wl, grid, ns, upd = TRIBLOCK, 256, 400, "anderson20"
    else:
        cfg, w = W.diblock128(precision=args.precision, n=args.n)
        wl, grid, ns, upd = WORKLOAD, args.n, 200, "anderson10"
    cfg.device = local
    solver = ScftSolver(cfg)
    if args.variant >= 0:
        solver.set_variant(args.variant)
    solver.restore(w)
    stream = torch.cuda.ExternalStream(solver.stream_ptr, device=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])

    def max_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # State preparation: run past the steepest-descent phase until the Anderson
    # history is full, so every timed iteration does the full depth-10 mix.
    prep = cfg.updater.anderson_start + cfg.updater.anderson_depth if args.prep < 0 else args.prep
    solver.update(prep)
    # warm-up
    solver.update(args.warmup)
    solver.enable_sweep_timing(args.steps)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.update(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = max_ranks(e0.elapsed_time(e1))
    value = world * args.steps / (ms / 1000.0)
    sweep_ms, sweep_bytes, sweep_steps = solver.sweep_timing()
    launches = solver.launches_per_iteration * args.steps
    variant, variant_ms = solver.variant()

    # End to end through the public API, every step: the fields w_i and p go up
    # from pinned host memory, one iteration runs, and the scalars and the
    # fields the reference's updater hands back to its PhysFields (w_i, phi_i,
    # p: the whole-iteration plugin's update(t)) come down to pinned host memory.
    # The headline uploads with ps_gpu_set_fields_async (p's copy overlaps the
    # iteration's sweeps; its field update waits for it) and reads the fields
    # back with ps_gpu_get_fields_async (the copy of step t overlaps step t + 1;
    # all copies end inside the timed region); beside it the same with blocking
    # copies, and blocking uploads with the scalars only.
    n_e2e = max(1, min(args.e2e_steps, args.steps))
    N = cfg.n_total
    nf = len(cfg.fields)
    host_w = [torch.from_numpy(x.copy()).pin_memory() for x in w]
    host_p = torch.zeros(N, dtype=torch.float64).pin_memory()
    out_w = [torch.empty(N, dtype=torch.float64).pin_memory() for _ in range(nf)]
    out_phi = [torch.empty(N, dtype=torch.float64).pin_memory() for _ in range(nf)]
    out_p = torch.empty(N, dtype=torch.float64).pin_memory()

    def e2e_run(mode: str):
        barrier()
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        sc = None
        for _ in range(n_e2e):
            if mode == "async":  # w ahead of the iteration, p beside its sweeps
                for i, hw in enumerate(host_w):
                    solver.set_field_async(0, i, hw)
                solver.set_field_async(2, 0, host_p)
            else:
                for i, hw in enumerate(host_w):
                    solver.set_field(0, i, hw)
                solver.set_field(2, 0, host_p)
            solver.update(1)
            sc = solver.scalars()
            if mode == "sync":
                for i in range(nf):
                    solver.get_field(0, i, out=out_w[i])
                    solver.get_field(1, i, out=out_phi[i])
                solver.get_field(2, 0, out=out_p)
            elif mode == "async":
                for i in range(nf):
                    solver.get_field_async(0, i, out_w[i])
                    solver.get_field_async(1, i, out_phi[i])
                solver.get_field_async(2, 0, out_p)
        if mode == "async":
            solver.fields_wait()  # every copy has landed before the end event
        f1.record(stream)
        f1.synchronize()
        barrier()
        return world * n_e2e / (max_ranks(f0.elapsed_time(f1)) / 1000.0), sc

    # the read-back's device snapshots are allocated on first use: not in the timed region
    for i in range(nf):
        solver.get_field_async(0, i, out_w[i])
        solver.get_field_async(1, i, out_phi[i])
    solver.get_field_async(2, 0, out_p)
    solver.fields_wait()
    e2e_value, last = e2e_run("async")
    e2e_sync_value, _ = e2e_run("sync")
    e2e_scalars_value, _ = e2e_run("scalars")
    h2d = (nf + 1) * N * 8
    d2h = 120 + (2 * nf + 1) * N * 8  # sizeof(ps_scalars) + w_i, phi_i, p

    peak, peak_kind = peaks()
    mean_sweep = statistics.mean(sweep_ms) if sweep_ms else float("nan")
    achieved = sweep_bytes / (mean_sweep / 1000.0) / 1e9 if sweep_ms else None
    per_step_ms = mean_sweep / max(sweep_steps, 1)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": profile_traffic(grid, args.precision),
                "kernel": "propagator step (plane_kernel + pencil_kernel per step of every sweep)",
                "peak_source": f"{peak_kind} hbm_gbs (burst copy)",
                "algorithmic_bytes_per_step": 3 * N * (4 if args.precision == "mixed" else 8),
                "step_us": per_step_ms * 1000.0, "samples": len(sweep_ms)}
    # The step's spectrum passes stay in L2: per propagator step (one sweep,
    # like step_us) the plane pass reads the half spectrum and the Boltzmann
    # factors and writes the slice and the spectrum, and the pencil pass reads
    # and writes the spectrum.
    sq = 4 if args.precision == "mixed" else 8
    spec_b = grid * grid * (grid // 2 + 1) * 2 * sq
    l2_bytes = 2 * spec_b + 2 * N * sq + 2 * spec_b
    if rank == 0 and not tri:  # the two-pass design of the 128^2 fused planes
        try:
            l2_peak = l2_copy_bandwidth(local)
            l2_ach = l2_bytes / (per_step_ms / 1000.0) / 1e9
            roofline["l2"] = {"bound": "l2", "achieved": l2_ach, "peak": l2_peak, "unit": "GB/s",
                              "frac": l2_ach / l2_peak, "bytes_per_step": l2_bytes,
                              "floor_step_us": l2_bytes / (l2_peak * 1e9) * 1e6,
                              "what": "L2 traffic per propagator step (two half-spectrum round trips, "
                                      "Boltzmann factors, slice write) against the measured copy "
                                      "bandwidth of a 32 MB L2-resident buffer (torch copies in a "
                                      "CUDA graph)"}
        except Exception as e:
            roofline["l2"] = {"error": f"{type(e).__name__}: {e}"}
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None,
           "dtype": "f32 propagators + f64 reductions" if args.precision == "mixed" else "f64",
           "data": "synthetic",
           "config": {"workload": wl if args.precision == "mixed" else
                      wl.replace("mixed precision", "FP64"),
                      "grid": grid, "ns": ns, "precision": args.precision, "updater": upd,
                      "parallelism": f"replicas x{world}",
                      "kernel_variant": variant,
                      "variant_sweep_ms": [round(x, 3) for x in variant_ms],
                      "state": f"{prep} iterations before warm-up: timed iterations use the full "
                               "Anderson history",
                      "l2": "inputs larger than L2: "
                            f"{sweep_steps * N * (4 if args.precision == 'mixed' else 8) / 1e9:.1f} GB "
                            "of propagator slices per iteration"},
           "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h, "steps": n_e2e,
                   "what": "per step: w_i and p up from pinned host memory, one iteration, the "
                           "scalars and w_i, phi_i, p back to pinned host memory (asynchronous "
                           "copies: p's upload overlaps the iteration's sweeps, the read-back "
                           "overlaps the next step)",
                   "blocking_copies": {"value": e2e_sync_value, "d2h_bytes_per_step": d2h},
                   "scalars_only": {"value": e2e_scalars_value, "d2h_bytes_per_step": 120}},
           "gpu_launches": launches, "roofline": roofline, "clocks": clk,
           "free_energy": last["free_energy"] if last else None}
    wcell = [solver.w(i) for i in range(len(cfg.fields))] if tri and rank == 0 else None
    solver.close()
    if tri:
        # one variable-cell step's stress: FP64 adjoint with sqrt(Ns) checkpoints
        if rank == 0 and world == 1:
            from polyswift_plusplus_b200.cell import stress
            t0 = time.perf_counter()
            Fc, g = stress(cfg, wcell, 0, local)
            out["cell_step"] = {"seconds": time.perf_counter() - t0, "F": Fc, "dF_dL_box": list(g),
                                "what": "dF/dL_box of the current fields by the FP64 adjoint "
                                        "(forward + backward sweeps, sqrt(Ns) checkpoints)"}
        if rank == 0:
            print(json.dumps(out), flush=True)
        return
    if rank == 0 and world == 1 and args.precision == "mixed" and args.precision_iters > 0:
        out["precision"] = precision_check(args.n, args.precision_iters, local)
        mix, esc = out["precision"]["mixed"], out["precision"]["escalated"]
        # The rate of the whole 1000-iteration job that meets the metric's
        # accuracy condition |dF/F| < 1e-6 against the FP64 path: the FP32-sweep
        # job when it does, else the job that finishes its last iterations with
        # FP64 sweeps (switch included).
        job, name = (mix, "mixed") if mix["dF_over_F"] < 1e-6 else (esc, "escalated")
        out["value_at_tolerance"] = {
            "value": job["iter_per_s"], "unit": UNIT, "dF_over_F": job["dF_over_F"],
            "job": name, "iterations": args.precision_iters,
            "fp64_finish_iterations": esc["fp64_finish_iterations"] if name == "escalated" else 0,
            "what": "device-timed rate of the whole job from the seeded start"}
    if rank == 0 and world == 1 and args.precision == "mixed" and args.cufft:
        try:
            cmpf = cufft_comparison(args.n, local)
            out["roofline"]["cufft_step_us"] = cmpf["step_us"]
            out["cufft_comparison"] = dict(cmpf, speedup_of_hand_written=cmpf["step_us"] /
                                           out["roofline"]["step_us"])
        except Exception as e:  # a comparison only: never lose the bench line to it
            out["cufft_comparison"] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0 and world == 1 and args.precision == "mixed" and args.fp64_steps > 0:
        out["fp64_path"] = fp64_rate(args.n, args.fp64_steps, local)
        out["mixed_over_fp64"] = value / out["fp64_path"]["value"]
    if rank == 0 and world == 1 and args.batch_instances > 0:
        out["batched"] = batched_rate(args.batch_instances, args.batch_steps, local)
    if rank == 0 and world == 1 and args.precision == "mixed" and args.scale256 > 0:
        try:
            out["scale256"] = scale256_rate(args.scale256, local)
        except Exception as e:  # e.g. a device with less memory than the case needs
            out["scale256"] = {"error": f"{type(e).__name__}: {e}"}
    if rank == 0 and world == 1 and args.precision == "mixed" and args.batch128 > 0:
        out["batched128"] = batched128_rate(args.batch128, args.batch_steps, local)
        if "fp64_path" in out:
            out["batched128"]["over_fp64_path"] = (out["batched128"]["value"] /
                                                   out["fp64_path"]["value"])
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_full_iteration(args.n)
    if rank == 0:
        print(json.dumps(out), flush=True)


def main():
    args = parse_args()
    world, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
