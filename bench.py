#!/usr/bin/env python3
"""Benchmark of the B200 MPM step: particle-updates/s on the 3-D dam break
(256x128x128 cells, ~8.08 M particles, weakly compressible Tait fluid,
quadratic B-splines, slip walls), mixed FP32 precision.

One "step" is one full explicit MPM time step of the reference's time loop
(sort, P2G, nodal update + BCs, G2P + F + stress + advection) over all
particles.  value = particles x steps / device time of the timed steps (CUDA
events on the library's stream, max over ranks).  e2e = the same metric for a
whole job through the C ABI with host buffers: upload of the host particle
arrays, the steps, and download of the particle arrays, over steps.

--impl reference times the oracle port of the reference's CPU path
(oracle/exg_oracle.cpp, OpenMP, all host threads) on a bounded sample of the
same workload; the reference itself cannot be built (its AMReX dependency is
absent).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

METRIC = "particle-updates/s at 1 B200 (mixed FP32 step vs plain FP64 step at stated error; % HBM roofline)"
UNIT = "particle-updates/s"

# Algorithmic bytes per particle per launch (compulsory traffic of the
# canonical particle state; positions FP64, other fields FP32 in mixed,
# FP64 in fp64):
#   P2G  reads x(3 f64) v(3) m V sigma(6)                           = 24 + 11w
#   G2P  reads x(3 f64) v(3) E(9) eps(6) m V0 mat phase              = 24 + 20w + 5
#        writes x(3 f64) v(3) E(9) eps(6) sigma(6) V                 = 24 + 25w
ALGO_BYTES = {
    "p2g": lambda w: 24 + 11 * w,
    "g2p": lambda w: 24 + 20 * w + 5 + 24 + 25 * w,
}


def read_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic(kernel: str):
    """Per-particle DRAM bytes of `kernel` from the committed ncu summary."""
    f = ROOT / "profiles" / "dam_break_traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.out = ROOT / "gpurun_out" / f"clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.out.parent.mkdir(exist_ok=True)
            self.f = open(self.out, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not self.out.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons)}


def workload(args, precision):
    from exagoop_b200 import native as nt, scenes
    f = args.scale
    if args.config == "dam_break":
        n = (int(256 * f), int(128 * f), int(128 * f))
        s, p = scenes.dam_break(n=n, size=(1.0, 0.5, 0.5), block=(0.4, 0.5, 0.3), seed=1234, precision=precision)
        name = f"dam_break_{n[0]}x{n[1]}x{n[2]}_quadratic_tait"
    elif args.config == "spheres":
        s, p = scenes.sphere_collision(n=int(256 * f), precision=precision)
        name = f"sphere_collision_{int(256 * f)}^3_cubic_elastic"
    else:
        s, p = scenes.axial_bar(precision=precision)
        name = "axial_bar_64x4x4_linear_elastic"
    if args.tile:
        s.tile = args.tile
    return s, p, name


def job_reduce(ms, units, world, device="cuda"):
    """Whole-job figures over the ranks: the slowest rank's device time
    (max) and the units all ranks processed (sum).  Every rank calls it
    once, in the same order (NCCL on the GPUs, gloo in the CPU tests)."""
    if world == 1:
        return float(ms), int(units)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    torch.distributed.all_reduce(u)
    return float(t.item()), int(u.item())


def time_steps(ctx, K, W):
    import torch
    stream = torch.cuda.ExternalStream(ctx.stream())
    for _ in range(W):
        ctx.step(1)
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.step(K)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)  # ms


def run_ours(args, rank, world):
    import torch
    from exagoop_b200 import native as nt

    torch.cuda.set_device(rank % torch.cuda.device_count())
    dev = torch.cuda.current_device()
    prec = nt.PREC_MIXED if args.precision == "mixed" else nt.PREC_FP64
    s, p, name = workload(args, prec)
    ctx = nt.Context(s, device=dev)
    ctx.upload(p)
    ctx.Initialise_Internal_Forces()
    # device-timed steps (inputs resident; particle state 8 M x ~300 B >> L2)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        ms = time_steps(ctx, args.steps, args.warmup)
    ms, n_total = job_reduce(ms, p.n, world)
    value = n_total * args.steps / (ms * 1e-3)
    # per-stage device times (eager, CUDA events between the stages)
    ctx.stage_timing(True)
    ctx.step(max(3, min(10, args.steps)))
    st = ctx.last_step_timing()
    ctx.stage_timing(False)
    w = 4 if prec == nt.PREC_MIXED else 8
    stages = {"sort": st[0], "p2g": st[1], "nodal": st[2], "g2p": st[3]}
    dom = max(("p2g", "g2p"), key=lambda k: stages[k])
    peak, peak_kind = read_peaks()
    achieved = ALGO_BYTES[dom](w) * p.n / (stages[dom] * 1e-3) / 1e9
    traffic_pp = read_traffic(dom)
    # end to end through the C ABI with host buffers in page-locked memory:
    # upload, steps, download into a pinned result set
    hp = p.pinned_copy()
    q = nt.Particles(p.n, pinned=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.upload(hp)
    ctx.step(args.steps)
    ctx.download_into(q)
    e2e_s = time.perf_counter() - t0
    h2d = p.pos.nbytes + p.rdata.nbytes + p.idata.nbytes
    e2e = {"value": n_total * args.steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(h2d / args.steps)}
    del q
    # plain FP64 step for the mixed/FP64 ratio (same workload)
    fp64_value = None
    if args.precision == "mixed" and not args.no_fp64:
        del ctx
        s64, p64, _ = workload(args, nt.PREC_FP64)
        c64 = nt.Context(s64, device=dev)
        c64.upload(p64)
        c64.Initialise_Internal_Forces()
        ms64 = time_steps(c64, max(3, args.steps // 2), args.warmup)
        fp64_value = p64.n * max(3, args.steps // 2) / (ms64 * 1e-3)
        del c64
    # kernels per fused step: dt_finalize, keys, tile_scan, touched, scatter,
    # tile_sort, scales, p2g_cell, nodes, g2p_fused, copy_lost,
    # time_advance (USL); MUSL adds reset_accum, state_reduce, scales,
    # p2g_cell, nodes and a second g2p_fused
    launches = args.steps * (12 if s.stress_update_scheme == 0 else 18)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if prec == nt.PREC_MIXED else "f64",
        "data": "synthetic (seeded lattice, jittered)",
        "config": {"workload": name, "particles": int(p.n), "grid": list(s.ncells), "order": int(s.order[0]),
                   "precision": args.precision, "tile": ctx_tile(s), "l2": "inputs larger than L2",
                   "parallelism": f"replicas{world}" if world > 1 else "single"},
        "clocks": clk.summary(),
        "e2e": e2e,
        "gpu_launches": launches,
        "stages_ms": {k: round(v, 4) for k, v in stages.items()},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_particle": ALGO_BYTES[dom](w),
                     "traffic": (traffic_pp * p.n) if traffic_pp else None},
        "fp64_value": fp64_value,
        "mixed_over_fp64": (value / world / fp64_value) if fp64_value else None,
    }
    return line, p


def run_batch(args, rank, world):
    """The batched uneven scenes: 64 independent dam breaks (grid sides from
    {32,48,64,96,128}, fill fractions in [0.1,0.4], seeded) advanced by
    exg_batch_step, one launch per hot kernel over all scenes."""
    import torch
    from exagoop_b200 import native as nt, scenes

    torch.cuda.set_device(rank % torch.cuda.device_count())
    dev = torch.cuda.current_device()
    prec = nt.PREC_MIXED if args.precision == "mixed" else nt.PREC_FP64
    seed = 2024 + rank
    specs = scenes.batched_specs(n_scenes=args.scenes, seed=seed, precision=prec)
    b = nt.Batch(specs, device=dev)
    total = 0
    for sc, (s, p) in zip(b.scenes, scenes.batched_dam_breaks(n_scenes=args.scenes, seed=seed, precision=prec)):
        sc.upload(p)
        sc.Initialise_Internal_Forces()
        total += p.n
        del p
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        ms = time_steps(b, args.steps, args.warmup)
    ms, total_all = job_reduce(ms, total, world)
    value = total_all * args.steps / (ms * 1e-3)
    sides = [int(s.ncells[0]) for s in specs]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if prec == nt.PREC_MIXED else "f64",
        "data": "synthetic (seeded lattices, jittered)",
        "config": {"workload": f"batched_dam_breaks_{len(specs)}_scenes", "particles": total_all,
                   "particles_per_gpu": total, "grid_sides": sides, "order": 2, "precision": args.precision,
                   "tile": 8, "l2": "inputs larger than L2",
                   "parallelism": f"replicas{world}" if world > 1 else "single"},
        "clocks": clk.summary(),
        "e2e": None,
        # per scene: dt_finalize, keys, tile_scan, touched, scatter,
        # tile_sort, scales, copy_lost, time_advance; per batch: plan and the
        # batched P2G, nodal and G2P kernels
        "gpu_launches": args.steps * (len(specs) * 9 + 4),
        "roofline": None,
        "cpu_baseline": None,
    }
    b.close()
    return line


def ctx_tile(s):
    return int(s.tile) if s.tile else 8


def cpu_sample(args, threads, nsteps, warmup=0, budget_s=None):
    """Oracle (CPU port of the reference path) on the same workload: all
    particles, `warmup` untimed steps then up to `nsteps` timed steps, each
    timed separately; with a budget, timing stops once the timed steps have
    used it (at least one step is timed)."""
    import orc
    from exagoop_b200 import native as nt
    s, p, name = workload(args, nt.PREC_FP64)
    o = orc.Oracle(s, threads=threads)
    o.upload(p)
    o.init_internal_forces()
    for _ in range(warmup):
        o.step(1)
    done, spent = 0, 0.0
    while done < nsteps:
        t0 = time.perf_counter()
        o.step(1)
        spent += time.perf_counter() - t0
        done += 1
        if budget_s is not None and spent >= budget_s:
            break
    desc = f"{name}: all {p.n} particles, {done} timed steps after {warmup} warm-up, FP64"
    return p.n * done / spent, desc, name, done


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="dam_break", choices=["dam_break", "spheres", "axial_bar", "batch"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--scale", type=float, default=1.0, help="grid scale factor (1 = the benchmark size)")
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--scenes", type=int, default=64, help="scenes of --config batch")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        # the CPU path on the host cores: rank 0 alone, the others exit
        if rank != 0:
            return
        v, desc, name, done = cpu_sample(args, threads, args.steps, warmup=args.warmup, budget_s=120.0)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": done, "steps_requested": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lattice, jittered)",
            "config": {"workload": name, "precision": "fp64 (CPU oracle port)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return

    if world > 1:
        import torch
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.config == "batch":
        line = run_batch(args, rank, world)
        if rank == 0:
            print(json.dumps(line))
        if world > 1:
            import torch
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    line, p = run_ours(args, rank, world)
    if rank == 0:
        if not args.no_cpu:
            v, desc, _, _ = cpu_sample(args, threads, args.cpu_steps)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}
        print(json.dumps(line))
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
