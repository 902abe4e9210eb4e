"""GPU parity: every step function of the C ABI against the FP64 oracle on
the same seeded inputs.  FP64 tolerance: 1e-10 relative to the field's max
norm (deterministic fixed-point P2G sums in a different order from the
oracle's sequential sums), with the Tait-pressure conditioning term of
tests/parity.py; integer binning bit-exact."""
import numpy as np
import pytest

from exagoop_b200 import native as nt, scenes
import orc
import parity

pytestmark = pytest.mark.gpu

TOL64 = 1e-10


def rel(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale


def pair(specs, parts, phi=None):
    ctx = nt.Context(specs)
    ctx.upload(parts)
    o = orc.Oracle(specs)
    o.upload(parts)
    if phi is not None:
        ctx.set_levelset(0, phi)
        o.set_levelset(0, phi)
    return ctx, o


def check_particles(g, r, tol=TOL64, fields=None):
    fields = fields or [("vel", nt.R_VEL, 3), ("vel_prime", nt.R_VEL_PRIME, 3), ("strainrate", nt.R_STRAINRATE, 6),
                        ("strain", nt.R_STRAIN, 6), ("stress", nt.R_STRESS, 6), ("defgrad", nt.R_DEFGRAD, 9),
                        ("volume", nt.R_VOLUME, 1), ("density", nt.R_DENSITY, 1), ("jacobian", nt.R_JACOBIAN, 1),
                        ("pressure", nt.R_PRESSURE, 1)]
    for name, e in parity.field_errors(g, r, fields).items():
        assert e < tol, f"{name}: max rel err {e:.3e}"
    e = np.abs(g.pos - r.pos).max()
    assert e < tol * max(1.0, np.abs(r.pos).max()), f"position: max abs err {e:.3e}"


def small_dam(order=2, seed=3, n=(32, 16, 16)):
    return scenes.dam_break(n=n, size=(1.0, 0.5, 0.5), block=(0.4, 0.5, 0.3), seed=seed, order=order)


def random_scene(seed, n=(20, 12, 16), npart=4000, order=2, outside=0):
    rng = np.random.default_rng(seed)
    s = scenes.base_specs((0.1, -0.2, 0.0), (1.1, 0.4, 0.8), n, order)
    s.gravity[2] = -3.0
    dx = [(s.phi[d] - s.plo[d]) / n[d] for d in range(3)]
    pos = np.stack([rng.uniform(s.plo[d], s.phi[d], npart) for d in range(3)])
    if outside:
        pos[0, :outside] = s.phi[0] + 0.01
    p = scenes.make_particles(pos, dx, (2, 2, 2), 900.0, 0, E=2e3, nu=0.25)
    p.rdata[nt.R_VEL:nt.R_VEL + 3] = rng.normal(0, 0.3, (3, npart))
    p.rdata[nt.R_STRESS:nt.R_STRESS + 6] = rng.normal(0, 50.0, (6, npart))
    return s, p


def test_sort_bitexact():
    s, p = random_scene(11, outside=37)
    ctx, o = pair(s, p)
    keys, perm = ctx.sort_keys()
    okeys, operm = o.sort_keys(ctx.tile())
    assert np.array_equal(keys, okeys)
    assert np.array_equal(perm, operm)


def test_sort_bitexact_clustered():
    # many particles per cell and whole empty tiles
    s, p = random_scene(12, npart=20000)
    p.pos[:, ::3] = p.pos[:, :1]  # a third of the particles in one cell
    ctx, o = pair(s, p)
    keys, perm = ctx.sort_keys()
    okeys, operm = o.sort_keys(ctx.tile())
    assert np.array_equal(keys, okeys) and np.array_equal(perm, operm)


@pytest.mark.parametrize("pile", [33, 40, 300, 3000])
def test_sort_bitexact_crowded_cells(pile):
    # cells above the linear-rank limit (32) are sorted by the whole block:
    # several crowded cells in one tile, sizes just above the limit, not a
    # power of two, and one tile past the shared-memory capacity (5120)
    s, p = random_scene(12, npart=24000)
    rng = np.random.default_rng(pile)
    lo = np.array([s.plo[d] for d in range(3)])
    dx = np.array([(s.phi[d] - s.plo[d]) / s.ncells[d] for d in range(3)])
    for k in range(6):
        c = lo + (np.array([3, 4 + (k % 2), 3 + k // 2]) + 0.5) * dx
        idx = rng.choice(p.n, size=pile, replace=False)
        p.pos[:, idx] = c[:, None] + (rng.random((3, pile)) - 0.5) * 0.9 * dx[:, None]
    ctx, o = pair(s, p)
    keys, perm = ctx.sort_keys()
    okeys, operm = o.sort_keys(ctx.tile())
    assert np.array_equal(keys, okeys) and np.array_equal(perm, operm)


@pytest.mark.parametrize("order", [1, 2, 3])
def test_p2g_momentum(order):
    s, p = random_scene(20 + order, order=order)
    s.external_loads = 1
    for d in range(3):
        s.force_slab_lo[d] = s.plo[d] + 0.2 * (s.phi[d] - s.plo[d])
        s.force_slab_hi[d] = s.plo[d] + 0.6 * (s.phi[d] - s.plo[d])
        s.extforce[d] = 0.5 * (d + 1)
    ctx, o = pair(s, p)
    ctx.P2G_Momentum(1, 1, 1)
    o.p2g_momentum(1, 1, 1)
    m = o.nodes(nt.N_MASS)
    assert rel(ctx.nodes(nt.N_MASS), m) < TOL64
    for c in range(3):
        e = rel(ctx.nodes(nt.N_FRC + c), o.nodes(nt.N_FRC + c))
        assert e < TOL64, f"node force {c}: {e:.3e}"
        e_v, e_p = parity.node_velocity_check(m, ctx.nodes(nt.N_VEL + c), o.nodes(nt.N_VEL + c))
        assert e_v < TOL64 and e_p < TOL64, f"node velocity {c}: {e_v:.3e} {e_p:.3e}"


@pytest.mark.parametrize("order,tol", [(2, 1e-12), (3, 1e-9)])
def test_p2g_light_node_velocities_fp64(order, tol):
    # nodes that only the edges of particles' supports reach carry tiny
    # masses; their velocities p / m must keep relative precision (the FP64
    # fixed point is 96 bits wide; with 64 bits the error at nodes of 1e-10
    # of the largest mass was about 5e-7 of the velocity scale), because the
    # G2P's velocity gradient weights them by dN, which vanishes more slowly
    # than N.  Cubic: near the end of its support the weight
    # -r^3/6 + r^2 - 2r + 4/3 cancels terms of order 1 down to (2 - r)^3 / 6,
    # so two evaluation orders differ by an ulp of 1 there, which at such
    # nodes is ~1e-11 of the velocity scale; hence the looser cubic bound.
    s, p = small_dam(order=order, seed=60 + order)
    rng = np.random.default_rng(order)
    p.rdata[nt.R_VEL:nt.R_VEL + 3] = rng.normal(0, 0.3, (3, p.n))
    # a spray of single particles in the empty part of the box: nodes at
    # the ends of their supports get masses many decades below the block's
    spray = rng.choice(p.n, 400, replace=False)
    for d, (lo, hi) in enumerate([(0.55, 0.95), (0.05, 0.45), (0.05, 0.45)]):
        p.pos[d, spray] = rng.uniform(lo, hi, 400)
    ctx, o = pair(s, p)
    ctx.P2G_Momentum(1, 1, 1)
    o.p2g_momentum(1, 1, 1)
    m = o.nodes(nt.N_MASS)
    light = (m > 1e-10 * m.max()) & (m < 1e-4 * m.max())
    assert light.sum() >= 5  # nodes beyond the block's faces
    for c in range(3):
        vo, vg = o.nodes(nt.N_VEL + c), ctx.nodes(nt.N_VEL + c)
        e = np.abs(vg - vo)[light].max() / np.abs(vo).max()
        assert e < tol, f"velocity {c} at light nodes: {e:.3e}"


def test_p2g_mixed_orders():
    # ncells < 5 on one axis: quadratic falls back to linear there
    s, p = random_scene(31, n=(20, 4, 12), order=2)
    assert list(s.order) == [2, 1, 2]
    ctx, o = pair(s, p)
    ctx.P2G_Momentum(1, 1, 1)
    o.p2g_momentum(1, 1, 1)
    for comp in range(7):
        assert rel(ctx.nodes(comp), o.nodes(comp)) < TOL64


@pytest.mark.parametrize("bc", [nt.BC_NOSLIP, nt.BC_SLIP, nt.BC_PARTIALSLIP])
def test_nodal_ops_and_bcs(bc):
    s, p = random_scene(40 + bc, order=2)
    for d in range(3):
        s.bclo[d] = bc
        s.bchi[d] = nt.BC_SLIP if d == 1 else bc
        s.wall_mu_lo[d] = 0.3
        s.wall_vel_lo[3 * d + (d + 1) % 3] = 0.05
    ctx, o = pair(s, p)
    dt = 1e-4
    ctx.P2G_Momentum(1, 1, 1)
    ctx.backup_current_velocity()
    ctx.Nodal_Time_Update_Momentum(dt)
    ctx.Apply_Nodal_BCs(dt, 0.0)
    o.p2g_momentum(1, 1, 1)
    o.backup_current_velocity()
    o.nodal_time_update_momentum(dt)
    o.apply_nodal_bcs(dt, 0.0)
    m = o.nodes(nt.N_MASS)
    for comp in [nt.N_MASS, nt.N_MASS_OLD]:
        assert rel(ctx.nodes(comp), o.nodes(comp)) < TOL64, comp
    for comp in [nt.N_VEL, nt.N_VEL + 1, nt.N_VEL + 2, nt.N_DVEL, nt.N_DVEL + 1, nt.N_DVEL + 2]:
        e_v, e_p = parity.node_velocity_check(m, ctx.nodes(comp), o.nodes(comp))
        assert e_v < TOL64 and e_p < TOL64, (comp, e_v, e_p)


@pytest.mark.parametrize("order", [1, 2, 3])
def test_g2p_move_volume_stress(order):
    s, p = random_scene(50 + order, order=order)
    p.idata[nt.I_PHASE, ::17] = 1  # rigid particles: advected only
    ctx, o = pair(s, p)
    dt = 2e-4
    for x in (ctx,):
        x.P2G_Momentum(1, 1, 1)
        x.backup_current_velocity()
        x.Nodal_Time_Update_Momentum(dt)
        x.Apply_Nodal_BCs(dt, 0.0)
        x.G2P_Momentum(1, 1, dt)
        x.Update_MP_Positions(dt)
        x.Update_MP_Volume()
        x.Calculate_MP_Stress_Strain(0.0, dt)
    o.p2g_momentum(1, 1, 1)
    o.backup_current_velocity()
    o.nodal_time_update_momentum(dt)
    o.apply_nodal_bcs(dt, 0.0)
    o.g2p_momentum(1, 1, dt)
    o.update_mp_positions(dt)
    o.update_mp_volume()
    o.calculate_mp_stress_strain(0.0, dt)
    check_particles(ctx.download(), o.download())


def test_init_internal_forces():
    s, p = small_dam()
    ctx, o = pair(s, p)
    ctx.Initialise_Internal_Forces()
    o.init_internal_forces()
    check_particles(ctx.download(), o.download())


def test_time_step_cfl():
    s, p = small_dam()
    ctx, o = pair(s, p)
    dt = ctx.Calculate_time_step()
    assert dt == pytest.approx(o.calculate_time_step(), rel=1e-14)


def run_both(specs, parts, nsteps, phi=None):
    ctx, o = pair(specs, parts, phi)
    ctx.Initialise_Internal_Forces()
    o.init_internal_forces()
    ctx.step(nsteps)
    assert o.step(nsteps) == 0
    return ctx, o


def test_fused_axial_bar():
    s, p = scenes.axial_bar(nx=32)
    ctx, o = run_both(s, p, 50)
    check_particles(ctx.download(), o.download())
    t, dt, n = ctx.time()
    to, dto, no = o.time()
    assert n == no == 50 and t == pytest.approx(to, rel=1e-14)


def test_fused_dam_break_quadratic():
    s, p = small_dam()
    ctx, o = run_both(s, p, 20)
    check_particles(ctx.download(), o.download())
    gd, od = ctx.diagnostics(), o.diagnostics()
    for k in ("tke", "tse", "mass"):
        assert gd[k] == pytest.approx(od[k], rel=1e-10, abs=1e-300), k


def test_fused_spheres_cubic():
    s, p = scenes.sphere_collision(n=32)
    ctx, o = run_both(s, p, 20)
    check_particles(ctx.download(), o.download())


def test_fused_musl():
    s, p = small_dam(seed=5)
    s.stress_update_scheme = 1
    ctx, o = run_both(s, p, 10)
    check_particles(ctx.download(), o.download())


def test_fused_levelset_obstacles():
    s, p, phi = scenes.twisted_column(n=(16, 16, 48), precision=nt.PREC_FP64, n_obstacles=6, heat=False)
    ctx, o = run_both(s, p, 20, phi)
    check_particles(ctx.download(), o.download())


def test_fused_twisted_column_heat():
    # the twisted column with its temperature field (rigid particles,
    # obstacles, noslip base, thermal deposit and G2P every step)
    s, p, phi = scenes.twisted_column(n=(16, 16, 48), precision=nt.PREC_FP64, n_obstacles=6, heat=True)
    ctx, o = run_both(s, p, 20, phi)
    g, r = ctx.download(), o.download()
    check_particles(g, r, fields=[("vel", nt.R_VEL, 3), ("stress", nt.R_STRESS, 6)])
    T = r.rdata[nt.R_TEMPERATURE]
    e = np.abs(g.rdata[nt.R_TEMPERATURE] - T).max()
    assert e < TOL64 * np.abs(T).max(), f"temperature: max abs err {e:.3e}"
    # q = -k sum_I T_I grad N_I cancels temperatures of ~300 K down to
    # their 1e-2 K spread: the tolerance carries that conditioning factor
    cond = np.abs(T).max() / (T.max() - T.min())
    q0, q1 = g.rdata[nt.R_HEATFLUX:nt.R_HEATFLUX + 3], r.rdata[nt.R_HEATFLUX:nt.R_HEATFLUX + 3]
    assert rel(q0, q1) < TOL64 * cond, f"heatflux: {rel(q0, q1):.3e} (conditioning {cond:.1f})"


def test_fused_deterministic():
    s, p = small_dam(seed=9)
    a, _ = pair(s, p)
    b, _ = pair(s, p)
    for x in (a, b):
        x.Initialise_Internal_Forces()
        x.step(15)
    pa, pb = a.download(), b.download()
    assert np.array_equal(pa.rdata, pb.rdata) and np.array_equal(pa.pos, pb.pos)


def mixed_vs_oracle(specs, parts, nsteps):
    s64 = specs.copy()
    sm = specs.copy()
    sm.precision = nt.PREC_MIXED
    ctx = nt.Context(sm)
    ctx.upload(parts)
    ctx.Initialise_Internal_Forces()
    o = orc.Oracle(s64)
    o.upload(parts)
    o.init_internal_forces()
    ctx.step(nsteps)
    o.step(nsteps)
    g, r = ctx.download(), o.download()
    out = {}
    for name, f, k in [("vel", nt.R_VEL, 3), ("stress", nt.R_STRESS, 6), ("strain", nt.R_STRAIN, 6),
                       ("jacobian", nt.R_JACOBIAN, 1)]:
        a, b = g.rdata[f:f + k], r.rdata[f:f + k]
        out[name] = np.linalg.norm(a - b) / np.linalg.norm(b)
    return out


def test_mixed_precision_error_elastic():
    # the north-star target: <= 1e-4 relative L2 in velocity and stress
    # against the FP64 oracle (elastic spheres, cubic B-splines)
    s, p = scenes.sphere_collision(n=32)
    e = mixed_vs_oracle(s, p, 300)
    assert e["vel"] < 1e-4 and e["stress"] < 1e-4, e
    assert e["jacobian"] < 1e-6, e


def test_mixed_precision_error_fluid():
    # the 1e-4 target on the dam break (Tait fluid, quadratic B-splines, slip
    # walls).  Its stress is the Tait pressure K((1/J)^7 - 1), which 100 steps
    # into the collapse is still small against K, so it carries the relative
    # error of J multiplied by gamma K / |p| (about 1e4): J is bounded at 1e-8
    # (2.5e-11 measured; stress 1.9e-7, velocity 1.8e-7)
    s, p = small_dam(seed=13)
    e = mixed_vs_oracle(s, p, 100)
    assert e["vel"] < 1e-4 and e["stress"] < 1e-4, e
    assert e["jacobian"] < 1e-8, e


def test_reupload_same_size_reuses_storage():
    # a second upload of the same particle count keeps storage and step
    # graphs; the steps that follow match a fresh context bit for bit
    s, p = small_dam(seed=21)
    a = nt.Context(s)
    a.upload(p)
    a.Initialise_Internal_Forces()
    a.step(7)
    a.upload(p)
    a.Initialise_Internal_Forces()
    a.step(5)
    b = nt.Context(s)
    b.upload(p)
    b.Initialise_Internal_Forces()
    b.step(5)
    pa, pb = a.download(), b.download()
    assert np.array_equal(pa.rdata, pb.rdata) and np.array_equal(pa.pos, pb.pos)


def test_reupload_that_changes_the_g2p_variant_rebuilds_graphs():
    # a fluid-only set runs the lean fused G2P; re-uploading the same count
    # as neo-Hookean solids must rebuild the step graphs with the full one
    s, p = small_dam(seed=23)
    s.precision = nt.PREC_FP64
    ctx = nt.Context(s)
    ctx.upload(p)
    ctx.Initialise_Internal_Forces()
    ctx.step(4)
    q = p.copy()
    q.idata[nt.I_MODEL] = 2
    q.rdata[nt.R_E] = 2e5
    q.rdata[nt.R_NU] = 0.3
    ctx.upload(q)
    ctx.set_time(0.0, 0)
    ctx.Initialise_Internal_Forces()
    ctx.step(6)
    got = ctx.download()
    o = orc.Oracle(s)
    o.upload(q)
    o.init_internal_forces()
    assert o.step(6) == 0
    r = o.download()
    for name, f, k in [("vel", nt.R_VEL, 3), ("stress", nt.R_STRESS, 6), ("defgrad", nt.R_DEFGRAD, 9)]:
        e = np.abs(got.rdata[f:f + k] - r.rdata[f:f + k]).max() / np.abs(r.rdata[f:f + k]).max()
        assert e < 1e-10, (name, e)


def test_large_upload_material_table_round_trip():
    # above 2^20 particles the host loops of upload and download run in
    # chunks on several threads: materials that alternate in runs across
    # the chunk boundaries come back per particle as they went in
    s, _ = small_dam(seed=24)
    n = 1_500_000
    rng = np.random.default_rng(24)
    p = nt.Particles(n)
    for d in range(3):
        p.pos[d] = s.plo[d] + (s.phi[d] - s.plo[d]) * rng.uniform(0.05, 0.95, n)
    p.rdata[nt.R_MASS] = 1e-3
    p.rdata[nt.R_VOLUME] = 1e-6
    p.rdata[nt.R_VOL_INIT] = 1e-6
    p.rdata[nt.R_DENSITY] = 1000.0
    p.rdata[nt.R_JACOBIAN] = 1.0
    for q in (0, 4, 8):
        p.rdata[nt.R_DEFGRAD + q] = 1.0
    run = (np.arange(n) // 7919) % 5
    table = [(1e5, 0.3, 0.0, 0.0, 0.0, 0), (2e6, 0.0, 2e6, 7.0, 1e-3, 1), (3e5, 0.25, 0.0, 0.0, 0.0, 2),
             (4e5, 0.2, 0.0, 0.0, 0.0, 0), (0.0, 0.0, 1e6, 1.5, 2e-3, 1)]
    for f, k in [(nt.R_E, 0), (nt.R_NU, 1), (nt.R_BULK, 2), (nt.R_GAMMA, 3), (nt.R_VISC, 4)]:
        p.rdata[f] = np.array([t[k] for t in table])[run]
    p.idata[nt.I_MODEL] = np.array([t[5] for t in table])[run]
    p.idata[nt.I_RIGID_ID] = np.arange(n) % 11
    ctx = nt.Context(s)
    ctx.upload(p)
    got = ctx.download()
    for f in (nt.R_E, nt.R_NU, nt.R_BULK, nt.R_GAMMA, nt.R_VISC, nt.R_RADIUS, nt.R_YACC):
        assert np.array_equal(got.rdata[f], p.rdata[f]), f
    assert np.array_equal(got.idata, p.idata)
    assert np.array_equal(got.pos, p.pos)
    ctx.close()


def test_pinned_particle_sets_round_trip():
    s, p = small_dam(seed=22)
    hp = p.pinned_copy()
    ctx = nt.Context(s)
    ctx.upload(hp)
    q = nt.Particles(p.n, pinned=True)
    ctx.download_into(q)
    assert np.array_equal(q.pos, p.pos)
    for f in (nt.R_VEL, nt.R_MASS, nt.R_DENSITY):
        assert np.allclose(q.rdata[f], p.rdata[f], rtol=0, atol=0)


def test_fused_neo_hookean_spheres():
    # constitutive model 2 (constitutive_models.H:161-250) at 4x the speed
    # of the elastic spheres, so the collision strains are not small
    s, p = scenes.sphere_collision(n=32, model=2, speed=0.4)
    ctx, o = run_both(s, p, 30)
    check_particles(ctx.download(), o.download())


def test_neo_hookean_step_functions():
    s, p = random_scene(61, order=2)
    p.idata[nt.I_MODEL] = 2
    p.rdata[nt.R_E], p.rdata[nt.R_NU] = 2e3, 0.25
    rng = np.random.default_rng(3)
    p.rdata[nt.R_DEFGRAD:nt.R_DEFGRAD + 9] += rng.normal(0, 0.05, (9, p.n))
    ctx, o = pair(s, p)
    dt = 2e-4
    ctx.P2G_Momentum(1, 1, 1)
    ctx.backup_current_velocity()
    ctx.Nodal_Time_Update_Momentum(dt)
    ctx.Apply_Nodal_BCs(dt, 0.0)
    ctx.G2P_Momentum(1, 1, dt)
    ctx.Update_MP_Volume()
    ctx.Calculate_MP_Stress_Strain(0.0, dt)
    o.p2g_momentum(1, 1, 1)
    o.backup_current_velocity()
    o.nodal_time_update_momentum(dt)
    o.apply_nodal_bcs(dt, 0.0)
    o.g2p_momentum(1, 1, dt)
    o.update_mp_volume()
    o.calculate_mp_stress_strain(0.0, dt)
    check_particles(ctx.download(), o.download())


def test_fused_incremental_strain():
    # calculate_strain_based_on_delta = 1: sigma += C : (dt D), the
    # initial internal forces still from the total formulation
    s, p = scenes.sphere_collision(n=32)
    s.calculate_strain_based_on_delta = 1
    s.applied_strainrate = 0.01
    s.applied_strainrate_time = 0.05
    ctx, o = run_both(s, p, 25)
    check_particles(ctx.download(), o.download())


def test_incremental_strain_rejects_fluid():
    s, p = small_dam()
    s.calculate_strain_based_on_delta = 1
    ctx = nt.Context(s)
    with pytest.raises(nt.ExgError):
        ctx.upload(p)
