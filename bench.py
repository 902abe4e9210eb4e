#!/usr/bin/env python3
"""Benchmark of the B200 MPM step in particle-updates/s.

Headline workload: the elastic sphere collision on a 256^3 grid (two
linear-elastic spheres of radius 0.2, 8,996,032 particles, cubic
B-splines), mixed FP32 precision, against the plain FP64 step on the same
particles (mixed_over_fp64) and with the relative L2 error of the mixed path
against the FP64 path after 1000 steps measured in the same run.  The 3-D
dam break (256x128x128 cells, 7,990,272 particles, weakly compressible Tait
fluid, quadratic B-splines, slip walls) is measured in the same run as a
second workload ("secondary").

One "step" is one full explicit MPM time step of the reference's time loop
(sort, P2G, nodal update + BCs, G2P + F + stress + advection) over all
particles.  value = particles x steps / device time of the timed steps (CUDA
events on the library's stream, max over ranks).  e2e = the same metric for a
whole job through the C ABI with host buffers: upload of the host particle
arrays, the steps, and download of the particle arrays, over steps.

--impl reference times the oracle port of the reference's CPU path
(oracle/exg_oracle.cpp built -march=native on the host, OpenMP, all host
threads) on a bounded sample of the same workload; the reference itself
cannot be built (its AMReX dependency is absent).
"""
from __future__ import annotations

import argparse
import json
import os
import platform
import subprocess
import sys
import tempfile
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


def read_traffic(workload: str, kernel: str):
    """Per-particle DRAM bytes of `kernel` on `workload` from the committed
    ncu summary (profiles/traffic.txt: lines '<workload> <kernel> <bytes>')."""
    f = ROOT / "profiles" / "traffic.txt"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 3 and parts[0] == workload and parts[1] == kernel:
            try:
                return float(parts[2])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs
    (samples go to a temporary file, removed afterwards)."""

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        fd, name = tempfile.mkstemp(prefix="exg_clocks_", suffix=".csv")
        os.close(fd)
        self.out = Path(name)

    def __enter__(self):
        try:
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
        try:
            self.out.unlink()
        except OSError:
            pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons)}


def workload(config, scale=1.0, tile=0):
    """(specs, particles, name) of a benchmark workload in FP64 specs (the
    caller sets the precision)."""
    from exagoop_b200 import scenes
    f = scale
    if config == "dam_break":
        n = (int(256 * f), int(128 * f), int(128 * f))
        s, p = scenes.dam_break(n=n, size=(1.0, 0.5, 0.5), block=(0.4, 0.5, 0.3), seed=1234)
        name = f"dam_break_{n[0]}x{n[1]}x{n[2]}_quadratic_tait"
    elif config == "spheres":
        s, p = scenes.sphere_collision(n=int(256 * f))
        name = f"sphere_collision_{int(256 * f)}^3_cubic_elastic"
    else:
        s, p = scenes.axial_bar()
        name = "axial_bar_64x4x4_linear_elastic"
    if tile:
        s.tile = tile
    return s, p, name


def with_precision(specs, precision):
    s = specs.copy()
    s.precision = precision
    return s


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


def stage_times(ctx, nsteps):
    """Per-stage device times (eager steps, CUDA events between the stages
    on the library's stream)."""
    ctx.stage_timing(True)
    ctx.step(nsteps)
    st = ctx.last_step_timing()
    ctx.stage_timing(False)
    return {"sort": st[0], "p2g": st[1], "nodal": st[2], "g2p": st[3]}


def roofline(stages, w, n, wl_name, peak, peak_kind):
    """HBM roofline of the P2G and G2P kernels: algorithmic bytes per launch
    over the launch's measured duration, against the measured copy peak."""
    out = {}
    for k in ("p2g", "g2p"):
        ach = ALGO_BYTES[k](w) * n / (stages[k] * 1e-3) / 1e9
        tr = read_traffic(wl_name, k)
        out[k] = {"achieved": ach, "frac": ach / peak, "algorithmic_bytes_per_particle": ALGO_BYTES[k](w),
                  "traffic": tr * n if tr else None}
    dom = max(("p2g", "g2p"), key=lambda k: stages[k])
    r = {"bound": "hbm", "kernel": dom, "achieved": out[dom]["achieved"], "peak": peak, "unit": "GB/s",
         "frac": out[dom]["frac"], "peak_source": peak_kind,
         "algorithmic_bytes_per_particle": out[dom]["algorithmic_bytes_per_particle"],
         "traffic": out[dom]["traffic"], "kernels": out}
    return r


def accuracy(s, p, dev, nsteps):
    """Relative L2 error of every output field of the mixed path against the
    plain FP64 GPU path (itself pinned to the FP64 oracle by the parity
    tests) after nsteps fused steps."""
    from exagoop_b200 import native as nt
    res = {}
    for prec in (nt.PREC_MIXED, nt.PREC_FP64):
        c = nt.Context(with_precision(s, prec), device=dev)
        c.upload(p)
        c.Initialise_Internal_Forces()
        c.step(nsteps)
        res[prec] = c.download()
        c.close()
    g, r = res[nt.PREC_MIXED], res[nt.PREC_FP64]
    out = {}
    for name, f, k in [("vel", nt.R_VEL, 3), ("stress", nt.R_STRESS, 6), ("strain", nt.R_STRAIN, 6),
                       ("defgrad", nt.R_DEFGRAD, 9), ("jacobian", nt.R_JACOBIAN, 1)]:
        a, b = g.rdata[f:f + k], r.rdata[f:f + k]
        out[name] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    out["position"] = float(np.linalg.norm(g.pos - r.pos) / np.linalg.norm(r.pos))
    return out


def measure(args, config, rank, world, dev, with_e2e, with_accuracy):
    """Mixed step (timed, staged, end to end) and the plain FP64 step of one
    workload on this rank's GPU."""
    import torch
    from exagoop_b200 import native as nt

    s, p, name = workload(config, args.scale, args.tile)
    prec = nt.PREC_MIXED if args.precision == "mixed" else nt.PREC_FP64
    ctx = nt.Context(with_precision(s, prec), device=dev)
    ctx.upload(p)
    ctx.Initialise_Internal_Forces()
    if args.p2g_variant >= 0 or args.g2p_variant >= 0:
        ctx.set_variants(args.p2g_variant, args.g2p_variant)  # pinned: no tuning run
    # device-timed steps (inputs resident; particle state 8-9 M x ~300 B >> L2)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        ms = time_steps(ctx, args.steps, args.warmup)
    ms, n_total = job_reduce(ms, p.n, world)
    value = n_total * args.steps / (ms * 1e-3)
    stages = stage_times(ctx, max(3, min(10, args.steps)))
    variants = ctx.variants()
    w = 4 if prec == nt.PREC_MIXED else 8
    peak, peak_kind = read_peaks()
    out = {"name": name, "particles": int(p.n), "grid": list(s.ncells), "order": int(s.order[0]),
           "tile": ctx.tile(), "value": value, "ms": ms, "clocks": clk.summary(),
           "stages_ms": {k: round(v, 4) for k, v in stages.items()},
           "roofline": roofline(stages, w, p.n, name, peak, peak_kind),
           "musl": int(s.stress_update_scheme != 0), "n_total": n_total,
           "variants": {"p2g": variants["p2g"], "g2p": variants["g2p"],
                        "p2g_ms": [round(x, 4) for x in variants["p2g_ms"]],
                        "g2p_ms": [round(x, 4) for x in variants["g2p_ms"]]}}
    if with_e2e:
        # end to end through the C ABI with host buffers in page-locked
        # memory: upload, steps, download into a pinned result set
        hp = p.pinned_copy()
        q = nt.Particles(p.n, pinned=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.upload(hp)
        ctx.step(args.steps)
        ctx.download_into(q)
        e2e_s = time.perf_counter() - t0
        nbytes = p.pos.nbytes + p.rdata.nbytes + p.idata.nbytes
        out["e2e"] = {"value": n_total * args.steps / e2e_s, "unit": UNIT,
                      "h2d_bytes_per_step": int(nbytes / args.steps), "d2h_bytes_per_step": int(nbytes / args.steps)}
        del q, hp
    ctx.close()
    del ctx
    if args.precision == "mixed" and not args.no_fp64:
        c64 = nt.Context(with_precision(s, nt.PREC_FP64), device=dev)
        c64.upload(p)
        c64.Initialise_Internal_Forces()
        k64 = max(3, args.steps // 2)
        ms64 = time_steps(c64, k64, args.warmup)
        out["fp64_value"] = p.n * k64 / (ms64 * 1e-3)
        out["fp64_stages_ms"] = {k: round(v, 4) for k, v in stage_times(c64, 3).items()}
        out["mixed_over_fp64"] = value / world / out["fp64_value"]
        c64.close()
        del c64
    if with_accuracy and args.precision == "mixed" and args.accuracy_steps > 0:
        out["accuracy"] = {"steps": args.accuracy_steps, "against": "plain FP64 GPU step (oracle-pinned)",
                           "rel_l2": accuracy(s, p, dev, args.accuracy_steps)}
    return out, (s, p, name)


def run_ours(args, rank, world):
    import torch

    torch.cuda.set_device(rank % torch.cuda.device_count())
    dev = torch.cuda.current_device()
    head, _ = measure(args, args.config, rank, world, dev, with_e2e=True, with_accuracy=(rank == 0))
    # kernels per fused step: dt_finalize, keys, tile_scan, touched, scatter,
    # tile_sort, scales, p2g_fact, nodes, g2p_fused, copy_lost,
    # time_advance (USL); MUSL adds reset_accum, state_reduce, scales,
    # p2g_fact, nodes and a second g2p_fused
    launches = args.steps * (12 if not head["musl"] else 18)
    prec_dtype = "f32+f64" if args.precision == "mixed" else "f64"
    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": prec_dtype,
        "data": "synthetic (seeded lattice)",
        "config": {"workload": head["name"], "particles": head["particles"], "grid": head["grid"],
                   "order": head["order"], "precision": args.precision, "tile": head["tile"],
                   "l2": "inputs larger than L2", "parallelism": f"replicas{world}" if world > 1 else "single",
                   "autotuned_variants": head["variants"]},
        "clocks": head["clocks"],
        "e2e": head["e2e"],
        "gpu_launches": launches,
        "stages_ms": head["stages_ms"],
        "roofline": head["roofline"],
        "fp64_value": head.get("fp64_value"),
        "fp64_stages_ms": head.get("fp64_stages_ms"),
        "mixed_over_fp64": head.get("mixed_over_fp64"),
    }
    if "accuracy" in head:
        line["accuracy"] = head["accuracy"]
    if args.config == "spheres" and not args.no_secondary:
        sec, _ = measure(args, "dam_break", rank, world, dev, with_e2e=False, with_accuracy=False)
        line["secondary"] = {
            "workload": sec["name"], "particles": sec["particles"], "grid": sec["grid"], "order": sec["order"],
            "value": sec["value"], "ms_per_step": sec["ms"] / args.steps, "stages_ms": sec["stages_ms"],
            "roofline": sec["roofline"], "fp64_value": sec.get("fp64_value"),
            "fp64_stages_ms": sec.get("fp64_stages_ms"), "mixed_over_fp64": sec.get("mixed_over_fp64"),
            "clocks": sec["clocks"], "autotuned_variants": sec["variants"]}
    return line


BATCH_SEED = 2024


def batch_share(n_scenes, rank, world):
    """This rank's scenes of the one seeded batch: the scenes are dealt to
    the ranks by particle count (scenes.partition_scenes), every rank
    computing the same partition without communication."""
    from exagoop_b200 import scenes
    counts = scenes.batched_scene_particle_counts(n_scenes=n_scenes, seed=BATCH_SEED)
    parts = scenes.partition_scenes(counts, world)
    return parts[rank], counts


def run_batch(args, rank, world):
    """The batched uneven scenes: 64 independent dam breaks (grid sides from
    {32,48,64,96,128}, fill fractions in [0.1,0.4], seeded) advanced by
    exg_batch_step, one launch per hot kernel over all scenes.  With N ranks
    the same 64 scenes are partitioned over the GPUs by particle count
    (strong scaling: the total work is fixed); no collective is on the data
    path."""
    import torch
    from exagoop_b200 import native as nt, scenes

    torch.cuda.set_device(rank % torch.cuda.device_count())
    dev = torch.cuda.current_device()
    prec = nt.PREC_MIXED if args.precision == "mixed" else nt.PREC_FP64
    mine, counts = batch_share(args.scenes, rank, world)
    seed = BATCH_SEED
    specs = scenes.batched_specs(n_scenes=args.scenes, seed=seed, precision=prec, only=set(mine))
    b = nt.Batch(specs, device=dev)
    total = 0
    for sc, (s, p) in zip(b.scenes, scenes.batched_dam_breaks(n_scenes=args.scenes, seed=seed, precision=prec,
                                                              only=set(mine))):
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
    # per-stage device times (eager steps, CUDA events between the stages)
    b.stage_timing(True)
    b.step(max(3, min(10, args.steps)))
    st = b.last_step_timing()
    b.stage_timing(False)
    stages = {"sort": st[0], "p2g": st[1], "nodal": st[2], "g2p": st[3]}
    peak, peak_kind = read_peaks()
    w = 4 if prec == nt.PREC_MIXED else 8
    name = f"batched_dam_breaks_{args.scenes}_scenes"
    rl = roofline(stages, w, total, name, peak, peak_kind)
    # end to end through the C ABI with host buffers: every scene of this
    # rank uploaded from its own page-locked host arrays (pinned before the
    # timed region, as the single-scene leg's), the steps, every scene
    # downloaded back into them
    e2e = None
    if not args.no_e2e:
        host = [p.pinned_copy() for _, p in scenes.batched_dam_breaks(n_scenes=args.scenes, seed=seed,
                                                                      precision=prec, only=set(mine))]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for sc, p in zip(b.scenes, host):
            sc.upload(p)
        b.step(args.steps)
        for sc, p in zip(b.scenes, host):
            sc.download_into(p)
        e2e_s = time.perf_counter() - t0
        nbytes = sum(p.pos.nbytes + p.rdata.nbytes + p.idata.nbytes for p in host)
        e2e_s = job_reduce(e2e_s * 1e3, 0, world)[0] * 1e-3
        e2e = {"value": total_all * args.steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(nbytes / args.steps), "d2h_bytes_per_step": int(nbytes / args.steps)}
        del host
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32+f64" if prec == nt.PREC_MIXED else "f64",
        "data": "synthetic (seeded lattices, jittered)",
        "config": {"workload": f"batched_dam_breaks_{args.scenes}_scenes", "particles": total_all,
                   "particles_rank0": total, "scenes_rank0": len(mine), "grid_sides_rank0": sides, "order": 2,
                   "precision": args.precision, "tile": 8, "l2": "inputs larger than L2",
                   "parallelism": f"scenes partitioned over {world} GPUs by particle count" if world > 1
                   else "single"},
        "clocks": clk.summary(),
        "e2e": e2e,
        # per step, whatever the number of scenes: step start, keys, tile
        # scan, scatter, plan, tile sort, touched, scales, plan, then the
        # batched P2G, nodal and G2P kernels, lost particles, time advance
        "gpu_launches": args.steps * 14,
        "stages_ms": {k: round(v, 4) for k, v in stages.items()},
        "roofline": rl,
        "cpu_baseline": None,
    }
    b.close()
    return line


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown CPU"


def cpu_sample(config, scale, tile, threads, nsteps, warmup=1, budget_s=None):
    """Oracle (CPU port of the reference path, built for this host's ISA) on
    the same workload: all particles, `warmup` untimed steps then up to
    `nsteps` timed steps, each timed separately; with a budget, timing stops
    once the timed steps have used it (at least one step is timed).  Loads
    only the oracle library, never libexg.so."""
    import orc
    isa = orc.use_native()
    s, p, name = workload(config, scale, tile)
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
    desc = (f"{name}: all {p.n} particles, {done} timed steps after {warmup} warm-up, FP64, "
            f"oracle {isa}, {threads} threads on {cpu_model()}")
    return p.n * done / spent, desc, name, done


def cpu_sample_batch(n_scenes, threads, nsteps=2):
    """Oracle on a bounded sample of the batch: the first four scenes of the
    seeded set, one warm-up step and nsteps timed steps each, FP64."""
    import orc
    from exagoop_b200 import scenes
    isa = orc.use_native()
    pts, spent = 0, 0.0
    picked = list(range(min(4, n_scenes)))
    for s, p in scenes.batched_dam_breaks(n_scenes=n_scenes, seed=BATCH_SEED, only=set(picked)):
        s = s.copy()
        from exagoop_b200 import native as nt
        s.precision = nt.PREC_FP64
        o = orc.Oracle(s, threads=threads)
        o.upload(p)
        o.init_internal_forces()
        o.step(1)
        t0 = time.perf_counter()
        o.step(nsteps)
        spent += time.perf_counter() - t0
        pts += p.n * nsteps
    desc = (f"batched dam breaks: scenes {picked} of the {n_scenes}-scene set, 1 warm-up + {nsteps} timed steps "
            f"each, FP64, oracle {isa}, {threads} threads on {cpu_model()}")
    return pts / spent, desc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="spheres", choices=["spheres", "dam_break", "axial_bar", "batch"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--scale", type=float, default=1.0, help="grid scale factor (1 = the benchmark size)")
    ap.add_argument("--cpu-steps", type=int, default=3, help="timed oracle steps of the cpu_baseline leg")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="steps of the mixed-vs-FP64 error measurement (0 skips it)")
    ap.add_argument("--scenes", type=int, default=64, help="scenes of --config batch")
    ap.add_argument("--p2g-variant", type=int, default=-1, help="pin the P2G launch variant (-1: autotune)")
    ap.add_argument("--g2p-variant", type=int, default=-1, help="pin the G2P launch variant (-1: autotune)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (batch)")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        # the CPU path on the host cores: rank 0 alone, the others exit
        if rank != 0:
            return
        # one warm-up step (a full FP64 step of 8-9 M particles takes
        # seconds on the host), then timed steps within a 90 s budget
        v, desc, name, done = cpu_sample(args.config if args.config != "batch" else "dam_break", args.scale,
                                         args.tile, threads, args.steps, warmup=1, budget_s=90.0)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": done, "steps_requested": args.steps, "warmup": 1, "warmup_requested": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded lattice)",
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
            if not args.no_cpu:
                v, desc = cpu_sample_batch(args.scenes, threads)
                line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}
            print(json.dumps(line))
        if world > 1:
            import torch
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    line = run_ours(args, rank, world)
    if rank == 0:
        if not args.no_cpu:
            v, desc, _, _ = cpu_sample(args.config, args.scale, args.tile, threads, args.cpu_steps, warmup=1)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc}
        print(json.dumps(line))
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
