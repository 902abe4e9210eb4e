"""Generates tests/golden/self_divergence.json: how far the FP64 oracle drifts
from itself over 1000 steps on each long-run accuracy workload when its
rounding changes, per output field (relative L2).  tests/test_gpu_accuracy.py
bounds the FP64 GPU path's 1000-step error by 10x this (and never below
1e-10): the GPU's nodal sums are exact fixed-point sums and the oracle's are
sequential FP64 sums, so the two paths differ by rounding every step, and
this measures what each workload makes of such differences.

Probes, each against the oracle run on all host threads:
  ulp1, ulp2  every initial position, velocity component and diagonal entry
              of F one ulp up or down (two seeds);
  order       the oracle on one thread (its P2G sums nodes in particle
              order; on many threads OpenMP atomics interleave the threads'
              contributions, as the reference's GPU atomics do);
  noise       after every step, every position, velocity and stress
              component one ulp up or down (a two-ulp spread, as two
              correct implementations round each step's results apart);
              a fluid particle's pressure moves by K 2^-52 instead (the
              Tait pressure K((1/J)^gamma - 1) is a difference of numbers
              near 1, so two correct evaluations of the power differ by
              an ulp of 1, which is K 2^-52 in p), equally on the three
              diagonal stress components.
The workloads and sizes are those of tests/test_gpu_accuracy.py.  CPU only;
run from the repository root (it takes a few minutes):

    python tests/golden/make_self_divergence.py
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))

from exagoop_b200 import native as nt  # noqa: E402
import orc  # noqa: E402
import test_gpu_accuracy as acc  # noqa: E402


def run(s, p, phi, threads):
    o = orc.Oracle(s, threads=threads)
    o.upload(p)
    if phi is not None:
        o.set_levelset(0, phi)
    o.init_internal_forces()
    assert o.step(1000) == 0
    return o.download()


def run_noisy(s, p, phi, threads, seed):
    o = orc.Oracle(s, threads=threads)
    o.upload(p)
    if phi is not None:
        o.set_levelset(0, phi)
    o.init_internal_forces()
    rng = np.random.default_rng(seed)

    def ulp(a):
        return np.where(rng.random(a.shape) < 0.5, np.nextafter(a, -np.inf), np.nextafter(a, np.inf))

    for _ in range(1000):
        assert o.step(1) == 0
        q = o.download()
        q.pos[:] = ulp(q.pos)
        q.rdata[nt.R_VEL:nt.R_VEL + 3] = ulp(q.rdata[nt.R_VEL:nt.R_VEL + 3])
        q.rdata[nt.R_STRESS:nt.R_STRESS + 6] = ulp(q.rdata[nt.R_STRESS:nt.R_STRESS + 6])
        fluid = q.idata[nt.I_MODEL] == 1
        if fluid.any():
            dp = np.where(rng.random(q.n) < 0.5, -1.0, 1.0) * q.rdata[nt.R_BULK] * 2.0 ** -52
            for c in (0, 3, 5):
                q.rdata[nt.R_STRESS + c] = np.where(fluid, q.rdata[nt.R_STRESS + c] - dp, q.rdata[nt.R_STRESS + c])
        o.upload(q)
    return o.download()


def perturbed(p, seed):
    q = p.copy()
    rng = np.random.default_rng(seed)

    def ulp(a):
        return np.where(rng.random(a.shape) < 0.5, np.nextafter(a, -np.inf), np.nextafter(a, np.inf))

    q.pos[:] = ulp(q.pos)
    q.rdata[nt.R_VEL:nt.R_VEL + 3] = ulp(q.rdata[nt.R_VEL:nt.R_VEL + 3])
    for a in (0, 4, 8):
        q.rdata[nt.R_DEFGRAD + a] = ulp(q.rdata[nt.R_DEFGRAD + a])
    return q


def main():
    threads = os.cpu_count() or 1
    out = {}
    for name in ["spheres", "dam_break", "twisted_column", "heated_block"]:
        s, p, phi = acc.workload(name)
        th = bool(s.use_temp)
        base = run(s, p, phi, threads)
        probes = {
            "ulp1": acc.l2_errors(run(s, perturbed(p, 1), phi, threads), base, th),
            "ulp2": acc.l2_errors(run(s, perturbed(p, 2), phi, threads), base, th),
            "order": acc.l2_errors(run(s, p, phi, 1), base, th),
            "noise": acc.l2_errors(run_noisy(s, p, phi, threads, 3), base, th),
        }
        fields = probes["ulp1"].keys()
        out[name] = {"max": {f: max(pr[f] for pr in probes.values()) for f in fields}, "probes": probes,
                     "particles": int(p.n), "threads": threads}
        print(name, json.dumps({f: float(f"{v:.2e}") for f, v in out[name]["max"].items()}), flush=True)
    (HERE / "self_divergence.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
