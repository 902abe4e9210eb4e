"""GPU parity on the benchmark workloads at their full sizes, and on the paths
with code of their own that the small scenes leave out.

* Axial bar (64x4x4 cells, 8,192 particles, linear B-splines): FP64 against
  the oracle for the whole 1000 steps.
* Dam break (256x128x128 cells, 7,990,272 particles, quadratic Tait fluid),
  elastic spheres (256^3 cells, 8,996,032 particles, cubic) and the twisted
  column (64x64x384 cells, 1,572,864 particles, level-set obstacles, rigid
  particles, heat): FP64 against the oracle for a few full steps at full
  size (the oracle takes seconds per step there), and the mixed path's
  error after the same steps.
* Spheres at full size for 1000 steps: the mixed path against the plain FP64
  GPU path (which the short full-size runs pin to the oracle), relative L2
  of velocity and stress within 1e-4.
* UDF wall velocities (compute_udf_wall_vel_at_nodes / apply_udf_nodal_bcs,
  Source/nodal_data_ops.cpp:929-1175), every diagnostic of
  Do_All_Diagnostics (Source/mpm_diagnostics.cpp:23-216), and the status
  codes of a non-finite particle (EXG_ERR_NAN) and of particles outside the
  domain (EXG_ERR_DOMAIN from Redistribute).

FP64 tolerance: 1e-10 relative to the field's max norm, as every parity
test, with the conditioning terms of tests/parity.py (the Tait pressure's
sensitivity to J; nodal velocities at light nodes)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from exagoop_b200 import native as nt, scenes
import orc
import parity

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
THREADS = os.cpu_count() or 1
FIELDS = [("vel", nt.R_VEL, 3), ("vel_prime", nt.R_VEL_PRIME, 3), ("strainrate", nt.R_STRAINRATE, 6),
          ("strain", nt.R_STRAIN, 6), ("stress", nt.R_STRESS, 6), ("defgrad", nt.R_DEFGRAD, 9),
          ("volume", nt.R_VOLUME, 1), ("density", nt.R_DENSITY, 1), ("jacobian", nt.R_JACOBIAN, 1),
          ("pressure", nt.R_PRESSURE, 1)]


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def max_rel_errors(g, r, fields=FIELDS):
    fields = [x for x in fields if np.abs(r.rdata[x[1]:x[1] + x[2]]).max() > 0]
    out = parity.field_errors(g, r, fields)
    out["position"] = float(np.abs(g.pos - r.pos).max() / max(1.0, np.abs(r.pos).max()))
    return out


def l2_errors(g, r):
    out = {}
    for name, f, k in FIELDS:
        b = r.rdata[f:f + k]
        nb = np.linalg.norm(b)
        if nb > 0:
            out[name] = float(np.linalg.norm(g.rdata[f:f + k] - b) / nb)
    return out


def gpu_run(specs, parts, nsteps, precision, phi=None):
    s = specs.copy()
    s.precision = precision
    ctx = nt.Context(s)
    if phi is not None:
        ctx.set_levelset(0, phi)
    ctx.upload(parts)
    ctx.Initialise_Internal_Forces()
    ctx.step(nsteps)
    out = ctx.download(), ctx.diagnostics(), ctx.time()
    ctx.close()
    return out


def oracle_run(specs, parts, nsteps, phi=None, threads=THREADS):
    o = orc.Oracle(specs, threads=threads)
    o.upload(parts)
    if phi is not None:
        o.set_levelset(0, phi)
    o.init_internal_forces()
    assert o.step(nsteps) == 0
    return o.download(), o.diagnostics(), o.time()


def diag_from_particles(q):
    """Do_All_Diagnostics evaluated in numpy on a particle set: TKE and TSE
    (Source/mpm_diagnostics.cpp:23-72, the shear terms doubled), total mass,
    momentum, mass-weighted velocity components and speed (:91-178) and the
    bounding box (:192-216), over all particles."""
    m, V = q.rdata[nt.R_MASS], q.rdata[nt.R_VOLUME]
    v = q.rdata[nt.R_VEL:nt.R_VEL + 3]
    sg, ep = q.rdata[nt.R_STRESS:nt.R_STRESS + 6], q.rdata[nt.R_STRAIN:nt.R_STRAIN + 6]
    se = sg[0] * ep[0] + sg[3] * ep[3] + sg[5] * ep[5] + 2.0 * (sg[1] * ep[1] + sg[4] * ep[4] + sg[2] * ep[2])
    M = m.sum()
    return {"tke": float((0.5 * m * (v * v).sum(0)).sum()), "tse": float((0.5 * V * se).sum()), "mass": float(M),
            "momentum": [float((m * v[d]).sum()) for d in range(3)],
            "mwa_vel": [float((m * v[d]).sum() / M) for d in range(3)],
            "mwa_velmag": float((m * np.sqrt((v * v).sum(0))).sum() / M),
            "minpos": [float(q.pos[d].min()) for d in range(3)], "maxpos": [float(q.pos[d].max()) for d in range(3)]}


def diag_close(a, b, tol):
    """Every diagnostic of a within tol of b (momentum components, which can
    cancel to ~0, against total mass x mass-weighted speed; velocity
    components against the mass-weighted speed)."""
    for k in ("tke", "tse", "mass", "mwa_velmag"):
        assert a[k] == pytest.approx(b[k], rel=tol, abs=1e-300), k
    vscale = b["mwa_velmag"] or 1.0
    for d in range(3):
        assert abs(a["momentum"][d] - b["momentum"][d]) <= tol * b["mass"] * vscale, ("momentum", d)
        assert abs(a["mwa_vel"][d] - b["mwa_vel"][d]) <= tol * vscale, ("mwa_vel", d)
        assert a["minpos"][d] == b["minpos"][d] and a["maxpos"][d] == b["maxpos"][d], ("bounding box", d)


def check_diag(gd, od, g=None, r=None):
    """Diagnostics parity in two parts: each side's reductions equal the
    reference's formulas evaluated on that side's own particles (the GPU
    reduces in a fixed two-pass tree, within 1e-12; the oracle sequentially,
    within n eps),
    and the two sides' particles agree field by field (the parity checks).
    Directly against each other the aggregates agree within 1e-9 (sums of
    fields that agree to 1e-10 of their max norm, some cancelling), the
    total mass within 1e-12."""
    if g is not None:
        diag_close(gd, diag_from_particles(g), 1e-12)
    if r is not None:
        # the oracle sums sequentially, as a single-threaded reduction does:
        # its rounding grows with the particle count (n eps)
        diag_close(od, diag_from_particles(r), max(1e-12, 2.2e-16 * r.n))
    assert gd["mass"] == pytest.approx(od["mass"], rel=1e-12)
    assert gd["np"] == od["np"]
    for k in ("tke", "tse", "mwa_velmag"):
        assert gd[k] == pytest.approx(od[k], rel=1e-9, abs=1e-300), k
    for d in range(3):
        assert gd["minpos"][d] == pytest.approx(od["minpos"][d], rel=1e-12, abs=1e-15), ("minpos", d)
        assert gd["maxpos"][d] == pytest.approx(od["maxpos"][d], rel=1e-12, abs=1e-15), ("maxpos", d)


def full_size_case(name):
    if name == "dam_break":
        s, p = scenes.dam_break()
        return s, p, None, 3
    if name == "spheres":
        s, p = scenes.sphere_collision(n=256)
        return s, p, None, 3
    s, p, phi = scenes.twisted_column(precision=nt.PREC_FP64)
    return s, p, phi, 5


def test_axial_bar_1000_steps_fp64():
    # the benchmark's CPU-runnable case exactly: 64x4x4 cells, 8192
    # particles, linear B-splines, fixed dt, 1000 steps
    s, p = scenes.axial_bar()
    assert p.n == 8192
    g, gd, gt = gpu_run(s, p, 1000, nt.PREC_FP64)
    r, od, ot = oracle_run(s, p, 1000)
    errs = max_rel_errors(g, r)
    print(json.dumps({"workload": "axial_bar_64x4x4", "steps": 1000, "fp64_max_rel": errs}))
    assert max(errs.values()) < TOL64, errs
    assert gt[2] == ot[2] == 1000 and gt[0] == pytest.approx(ot[0], rel=1e-14)
    check_diag(gd, od, g, r)


@pytest.mark.parametrize("name", ["dam_break", "spheres", "twisted_column"])
def test_full_size_against_oracle(name):
    s, p, phi, nsteps = full_size_case(name)
    r, od, _ = oracle_run(s, p, nsteps, phi)
    g, gd, _ = gpu_run(s, p, nsteps, nt.PREC_FP64, phi)
    fields = FIELDS + ([("temperature", nt.R_TEMPERATURE, 1)] if s.use_temp else [])
    errs = max_rel_errors(g, r, fields)
    gm, _, _ = gpu_run(s, p, nsteps, nt.PREC_MIXED, phi)
    mixed = l2_errors(gm, r)
    print(json.dumps({"workload": name, "particles": int(p.n), "steps": nsteps, "fp64_max_rel": errs,
                      "mixed_rel_l2": mixed}))
    assert max(errs.values()) < TOL64, errs
    if s.use_temp:
        # q = -k sum_I T_I grad N_I cancels ~300 K temperatures down to their
        # 1e-2 K spread: the tolerance carries that conditioning factor
        T = r.rdata[nt.R_TEMPERATURE]
        cond = np.abs(T).max() / (T.max() - T.min())
        q0, q1 = g.rdata[nt.R_HEATFLUX:nt.R_HEATFLUX + 3], r.rdata[nt.R_HEATFLUX:nt.R_HEATFLUX + 3]
        assert rel(q0, q1) < TOL64 * cond, rel(q0, q1)
    check_diag(gd, od, g, r)
    assert mixed["vel"] < 1e-4 and mixed["stress"] < 1e-4, mixed


def test_spheres_mixed_1000_steps_against_fp64():
    # the accuracy target at the 9M-particle workload: relative L2 of the
    # mixed path after 1000 steps against the plain FP64 GPU path, which
    # test_full_size_against_oracle pins to the oracle at this size
    s, p = scenes.sphere_collision(n=256)
    g64, _, t64 = gpu_run(s, p, 1000, nt.PREC_FP64)
    gm, _, tm = gpu_run(s, p, 1000, nt.PREC_MIXED)
    errs = l2_errors(gm, g64)
    errs["position"] = float(np.linalg.norm(gm.pos - g64.pos) / np.linalg.norm(g64.pos))
    print(json.dumps({"workload": "sphere_collision_256^3", "particles": int(p.n), "steps": 1000,
                      "mixed_vs_fp64_rel_l2": errs, "time": [t64[0], tm[0]]}))
    assert errs["vel"] < 1e-4 and errs["stress"] < 1e-4, errs


UDF_V = C.CFUNCTYPE(None, C.c_double, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double))
OMEGA = 0.5


@UDF_V
def _udf_twist(x, y, z, t, vel):
    # the twisted column's top-face UDF (Tests/3D_Twisted_Column/UDF/
    # wall_vel_twist.c) about the axis x = 0.6, y = 0.3, ramped in time
    vel[0] = -OMEGA * (y - 0.3) * (1.0 + t)
    vel[1] = OMEGA * (x - 0.6) * (1.0 + t)
    vel[2] = 0.0


@UDF_V
def _udf_shear(x, y, z, t, vel):
    vel[0] = 0.02 * z
    vel[1] = -0.5 + 0.1 * x
    vel[2] = 0.03 * np.sin(3.0 * y)


def udf_scene(seed):
    rng = np.random.default_rng(seed)
    s = scenes.base_specs((0.1, -0.2, 0.0), (1.1, 0.8, 0.8), (20, 20, 16), 2)
    s.gravity[2] = -3.0
    # z-hi noslip with the twist UDF (v = W), x-lo slip with a UDF (only the
    # normal component is set)
    s.bchi[2] = nt.BC_NOSLIP
    s.udf_wallvel_hi[2] = C.cast(_udf_twist, C.c_void_p).value
    s.bclo[0] = nt.BC_SLIP
    s.udf_wallvel_lo[0] = C.cast(_udf_shear, C.c_void_p).value
    n = 6000
    dx = [(s.phi[d] - s.plo[d]) / s.ncells[d] for d in range(3)]
    pos = np.stack([rng.uniform(s.plo[d] + 0.01, s.phi[d] - 0.01, n) for d in range(3)])
    p = scenes.make_particles(pos, dx, (2, 2, 2), 900.0, 0, E=2e3, nu=0.25)
    p.rdata[nt.R_VEL:nt.R_VEL + 3] = rng.normal(0, 0.3, (3, n))
    return s, p


def test_udf_wall_velocity_step_functions():
    s, p = udf_scene(5)
    ctx = nt.Context(s)
    ctx.upload(p)
    o = orc.Oracle(s)
    o.upload(p)
    dt, t = 1e-4, 0.35
    ctx.P2G_Momentum(1, 1, 1)
    ctx.backup_current_velocity()
    ctx.Nodal_Time_Update_Momentum(dt)
    ctx.Apply_Nodal_BCs(dt, t)
    o.p2g_momentum(1, 1, 1)
    o.backup_current_velocity()
    o.nodal_time_update_momentum(dt)
    o.apply_nodal_bcs(dt, t)
    nn = [s.ncells[d] + 1 for d in range(3)]
    m = o.nodes(nt.N_MASS)
    assert rel(ctx.nodes(nt.N_MASS), m) < TOL64
    for comp in [nt.N_VEL, nt.N_VEL + 1, nt.N_VEL + 2, nt.N_DVEL, nt.N_DVEL + 1, nt.N_DVEL + 2]:
        e_v, e_p = parity.node_velocity_check(m, ctx.nodes(comp), o.nodes(comp))
        assert e_v < TOL64 and e_p < TOL64, (comp, e_v, e_p)
    # the top face carries the UDF velocity exactly (noslip: v = W)
    vx = ctx.nodes(nt.N_VEL).reshape(nn[2], nn[1], nn[0])
    k, j, i = nn[2] - 1, 7, 11
    x, y = s.plo[0] + i * (s.phi[0] - s.plo[0]) / s.ncells[0], s.plo[1] + j * (s.phi[1] - s.plo[1]) / s.ncells[1]
    assert vx[k, j, i] == pytest.approx(-OMEGA * (y - 0.3) * (1.0 + t), rel=1e-14)


def test_udf_wall_velocity_fused_steps():
    s, p = udf_scene(6)
    g, gd, _ = gpu_run(s, p, 12, nt.PREC_FP64)
    r, od, _ = oracle_run(s, p, 12)
    errs = max_rel_errors(g, r)
    assert max(errs.values()) < TOL64, errs
    check_diag(gd, od, g, r)


def test_diagnostics_every_field():
    # TKE, TSE, total mass and momentum, mass-weighted velocity components
    # and magnitude, and the bounding box after fused steps, with rigid
    # particles (they count in every sum, as in the reference's reductions)
    s, p = scenes.sphere_collision(n=32)
    p.idata[nt.I_PHASE, ::29] = 1
    g, gd, _ = gpu_run(s, p, 25, nt.PREC_FP64)
    r, od, _ = oracle_run(s, p, 25)
    check_diag(gd, od, g, r)
    # and against a direct numpy evaluation of the reference formulas
    m = r.rdata[nt.R_MASS]
    v = r.rdata[nt.R_VEL:nt.R_VEL + 3]
    assert gd["mass"] == pytest.approx(m.sum(), rel=1e-13)
    for d in range(3):
        assert gd["mwa_vel"][d] == pytest.approx((m * v[d]).sum() / m.sum(), rel=1e-9, abs=1e-15)
        assert gd["minpos"][d] == r.pos[d].min() and gd["maxpos"][d] == r.pos[d].max()
    assert gd["mwa_velmag"] == pytest.approx((m * np.sqrt((v * v).sum(0))).sum() / m.sum(), rel=1e-12)
    assert gd["tke"] == pytest.approx(0.5 * (m * (v * v).sum(0)).sum(), rel=1e-12)


def test_nonfinite_particle_reports_nan_status():
    s, p = scenes.sphere_collision(n=32)
    p.rdata[nt.R_VEL + 2, 101] = np.nan
    ctx = nt.Context(s)
    ctx.upload(p)
    with pytest.raises(nt.ExgError) as e:
        ctx.step(1)
    assert e.value.code == -4  # EXG_ERR_NAN
    # the status word is cleared once reported
    assert ctx.L.exg_check_status(ctx.h) == 0
    ctx.close()


def test_particles_outside_the_domain_are_dropped_with_a_status():
    s, p = scenes.sphere_collision(n=32)
    out = [7, 500, 9001]
    p.pos[0, out[0]] = s.phi[0] + 0.05
    p.pos[1, out[1]] = s.plo[1] - 1e-3
    p.pos[2, out[2]] = 2.0
    ctx = nt.Context(s)
    ctx.upload(p)
    with pytest.raises(nt.ExgError) as e:
        ctx.Redistribute()
    assert e.value.code == -5  # EXG_ERR_DOMAIN
    assert "3 particles" in str(e.value)
    ctx.close()
    # the fused steps carry on without them, as the oracle (and AMReX's
    # Redistribute) drop them
    keep = np.setdiff1d(np.arange(p.n), out)
    g, _, _ = gpu_run(s, p, 5, nt.PREC_FP64)
    q = nt.Particles(len(keep))
    q.pos[:] = p.pos[:, keep]
    q.rdata[:] = p.rdata[:, keep]
    q.idata[:] = p.idata[:, keep]
    r, _, _ = oracle_run(s, q, 5)
    sub = nt.Particles(len(keep))
    sub.pos[:] = g.pos[:, keep]
    sub.rdata[:] = g.rdata[:, keep]
    sub.idata[:] = g.idata[:, keep]
    errs = max_rel_errors(sub, r)
    assert max(errs.values()) < TOL64, errs
    # the dropped particles stay in storage, inert, where they were
    for i in out:
        assert np.array_equal(g.pos[:, i], p.pos[:, i])
