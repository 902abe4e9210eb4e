#!/usr/bin/env python3
"""Generate the golden fixtures of the reference's per-step math.

Inputs are seeded; outputs come from the reference's OWN source code
(Source/interpolants.H, Source/mpm_kernels.H, Source/constitutive_models.H,
Source/mpm_eb.H) compiled by oracle/Makefile's `refpin` target into
oracle/_ref/libexg_refpin.so.  Run from the repository root, with the
reference tree present:

    make -C oracle refpin && python tests/golden/make_golden.py

The fixtures let the oracle be checked against the reference's arithmetic
where the reference tree is absent (on the GPU box, in CI).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent
REFPIN = ROOT / "oracle" / "_ref" / "libexg_refpin.so"

pd = C.POINTER(C.c_double)
pi = C.POINTER(C.c_int)


def P(a):
    return a.ctypes.data_as(pd if a.dtype == np.float64 else pi)


def load():
    L = C.CDLL(str(REFPIN))
    for n in ("ref_cubic1d", "ref_cubic1d_der", "ref_quad1d", "ref_quad1d_der"):
        getattr(L, n).restype = C.c_double
        getattr(L, n).argtypes = [C.c_int, C.c_double]
    L.ref_basisval_and_grad.restype = C.c_double
    L.ref_basisval_and_grad.argtypes = [pi, pi, pd, pd, pd, pi, pi, pi, pi, pd]
    L.ref_interp_two.restype = None
    L.ref_interp_two.argtypes = [C.c_int, pd, pi, pi, pi, pd, pd, pd, pi, pi, pi, pi, pi, pd]
    L.ref_applybc.restype = C.c_int
    L.ref_applybc.argtypes = [pd, pd, C.c_double, pd, C.c_int]
    L.ref_linear_elastic.argtypes = [pd, pd, C.c_double, C.c_double]
    L.ref_newtonian.argtypes = [pd, pd, C.c_double, C.c_double]
    L.ref_neo_hookean.argtypes = [pd, pd, C.c_double, C.c_double]
    L.ref_linear_elastic_delta.argtypes = [pd, pd, C.c_double, C.c_double]
    L.ref_defgrad_update.argtypes = [pd, pd, C.c_double]
    L.ref_levelset.restype = C.c_double
    L.ref_levelset.argtypes = [pd, pi, pi, pd, pd, pd, pd]
    return L


def stencil_bounds(iv, nc, order, periodic):
    # compute_bounds (mpm_particle_grid_ops.cpp:255-299), for case generation
    if order == 1:
        return 0, 2
    if periodic:
        return -1, 3
    if iv == 0:
        return 0, 3
    if iv == nc - 1:
        return -1, 2
    return -1, 3


def main():
    L = load()
    rng = np.random.default_rng(20261203)

    # 1-D splines: value and derivative of every shape type over the support
    z = np.concatenate([np.linspace(-1.999, 1.999, 1601), rng.uniform(-1.99, 1.99, 400)])
    spl = np.zeros((4, 5, z.size))
    fns = [L.ref_cubic1d, L.ref_cubic1d_der, L.ref_quad1d, L.ref_quad1d_der]
    for k, f in enumerate(fns):
        for t in range(1, 5):
            spl[k, t] = [f(t, float(v)) for v in z]
    np.savez_compressed(OUT / "splines.npz", z=z, values=spl)

    # basisval_and_grad over random cells, stencil offsets, orders, periodicity
    cases = []
    for _ in range(2000):
        nc = rng.integers(5, 12, 3).astype(np.int32)
        order = rng.integers(1, 4, 3).astype(np.int32)
        if rng.random() < 0.5:
            order[:] = order[0]
        periodic = (rng.random(3) < 0.15).astype(np.int32)
        plo = rng.uniform(-1, 1, 3)
        dx = rng.uniform(0.05, 0.3, 3)
        cell = np.array([rng.integers(0, nc[d]) for d in range(3)], dtype=np.int32)
        # positions near cell faces too
        frac = rng.uniform(0, 1, 3)
        frac[rng.random(3) < 0.1] = 0.0
        x = plo + (cell + frac) * dx
        st = np.array([rng.integers(*stencil_bounds(cell[d], nc[d], order[d], periodic[d])) for d in range(3)],
                      dtype=np.int32)
        lo = np.zeros(3, dtype=np.int32)
        hi = (nc - 1).astype(np.int32)
        grad = np.zeros(3)
        N = L.ref_basisval_and_grad(P(st), P(cell), P(x), P(plo), P(dx), P(order), P(periodic), P(lo), P(hi),
                                    P(grad))
        cases.append(np.concatenate([nc, order, periodic, cell, st, plo, dx, x, [N], grad]).astype(np.float64))
    np.savez_compressed(OUT / "basis.npz", cases=np.array(cases))

    # *_interp_two over a random node array (node box [-1, nc+1])
    rows = []
    nodes_all = []
    for case in range(48):
        nc = rng.integers(5, 8, 3).astype(np.int32)
        order = np.full(3, rng.integers(1, 4), dtype=np.int32)
        if case % 5 == 0:
            order = rng.integers(1, 4, 3).astype(np.int32)
        periodic = np.zeros(3, dtype=np.int32)
        plo = rng.uniform(-1, 1, 3)
        dx = rng.uniform(0.05, 0.3, 3)
        alo = np.full(3, -1, dtype=np.int32)
        ahi = (nc + 1).astype(np.int32)
        shape = tuple((ahi - alo + 1)[::-1])
        nodes = rng.normal(0, 1, (2,) + shape)
        cell = np.array([rng.integers(0, nc[d]) for d in range(3)], dtype=np.int32)
        x = plo + (cell + rng.uniform(0, 1, 3)) * dx
        mn = np.zeros(3, dtype=np.int32)
        mx = np.zeros(3, dtype=np.int32)
        for d in range(3):
            mn[d], mx[d] = stencil_bounds(cell[d], nc[d], order[d], 0)
        lo = np.zeros(3, dtype=np.int32)
        hi = (nc - 1).astype(np.int32)
        for scheme in (1, 2, 3):
            vals = np.zeros(2)
            buf = np.ascontiguousarray(nodes)
            L.ref_interp_two(scheme, P(x), P(cell), P(mn), P(mx), P(plo), P(dx), P(buf), P(alo), P(ahi),
                             P(periodic), P(lo), P(hi), P(vals))
            rows.append(np.concatenate([[case, scheme], nc, order, cell, mn, mx, plo, dx, x, vals]))
        nodes_all.append(nodes.ravel())
    offs = np.cumsum([0] + [a.size for a in nodes_all])
    np.savez_compressed(OUT / "interp.npz", rows=np.array(rows), nodes=np.concatenate(nodes_all), offsets=offs)

    # applybc (mpm_kernels.H:27-113)
    rows = []
    for _ in range(1500):
        vin = rng.normal(0, 1, 3)
        n = rng.normal(0, 1, 3)
        n /= np.linalg.norm(n)
        if rng.random() < 0.3:
            n = np.eye(3)[rng.integers(0, 3)] * rng.choice([-1, 1])
        mu = rng.uniform(0, 1)
        bc = int(rng.integers(0, 4))
        out = rng.normal(0, 1, 3)  # relvel_out keeps its input where applybc does not write
        o2 = out.copy()
        mod = L.ref_applybc(P(vin), P(o2), mu, P(n), bc)
        rows.append(np.concatenate([vin, n, [mu, bc], out, o2, [mod]]))
    np.savez_compressed(OUT / "applybc.npz", rows=np.array(rows))

    # constitutive models (constitutive_models.H:21-159) and the F update
    rows = []
    for _ in range(600):
        eps = rng.normal(0, 1e-3, 6)
        E, nu = rng.uniform(1e2, 1e9), rng.uniform(0, 0.49)
        s1 = np.zeros(6)
        L.ref_linear_elastic(P(eps), P(s1), E, nu)
        mu, p = rng.uniform(0, 1e-2), rng.normal(0, 1e4)
        s2 = np.zeros(6)
        L.ref_newtonian(P(eps), P(s2), mu, p)
        F = np.eye(3).ravel() + rng.normal(0, 1e-2, 9)
        g = rng.normal(0, 10, 9)
        if rng.random() < 0.05:
            g *= 1e6  # |grad v|^2 >= 1e10: F left unchanged
        dt = rng.uniform(1e-6, 1e-3)
        F2 = F.copy()
        L.ref_defgrad_update(P(F2), P(g), dt)
        rows.append(np.concatenate([eps, [E, nu], s1, [mu, p], s2, F, g, [dt], F2]))
    np.savez_compressed(OUT / "constitutive.npz", rows=np.array(rows))

    # neo-Hookean stress (constitutive_models.H:161-250) from F, and the
    # incremental linear-elastic operator (:69-104)
    rng2 = np.random.default_rng(20261204)
    rows = []
    for i in range(400):
        scale = 1e-2 if i < 300 else 0.3  # small and large deformations
        F = np.eye(3).ravel() + rng2.normal(0, scale, 9)
        E, nu = rng2.uniform(1e2, 1e9), rng2.uniform(0, 0.49)
        s = np.zeros(6)
        L.ref_neo_hookean(P(F), P(s), E, nu)
        deps = rng2.normal(0, 1e-4, 6)
        ds = np.zeros(6)
        L.ref_linear_elastic_delta(P(deps), P(ds), E, nu)
        rows.append(np.concatenate([F, [E, nu], s, deps, ds]))
    np.savez_compressed(OUT / "neo_hookean.npz", rows=np.array(rows))

    # level-set sampling (mpm_eb.H:176-288) on a node array with one ghost layer
    nc = np.array([10, 8, 9], dtype=np.int32)
    plo = np.array([0.0, -0.5, 0.25])
    dx = np.array([0.1, 0.125, 0.08])
    alo = np.full(3, -1, dtype=np.int32)
    ahi = (nc + 1).astype(np.int32)
    shape = tuple((ahi - alo + 1)[::-1])
    phi = rng.normal(0, 1, shape)
    rows = []
    for _ in range(1000):
        x = plo + rng.uniform(-0.5, 1.0, 3) * nc * dx if rng.random() < 0.1 else plo + rng.uniform(0, 1, 3) * nc * dx
        g = np.zeros(3)
        v = L.ref_levelset(P(np.ascontiguousarray(phi)), P(alo), P(ahi), P(plo), P(dx), P(x), P(g))
        rows.append(np.concatenate([x, [v], g]))
    np.savez_compressed(OUT / "levelset.npz", nc=nc, plo=plo, dx=dx, phi=phi, rows=np.array(rows))
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
