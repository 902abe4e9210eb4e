"""Physics-level pins of the oracle: the reference's own acceptance checks
(Tests/1D_Axial_Bar_Vibration/PostProcess/validate.py: RMS of v_x against
the analytic first mode) on the 3-D bar, energy conservation for pure FLIP,
and the step bookkeeping.  CPU only."""
import numpy as np

from exagoop_b200 import native as nt, scenes
import orc


def free_end_bar(nx=40, length=1.25):
    dx = length / nx
    s = scenes.base_specs((0, 0, 0), (length, 4 * dx, 4 * dx), (nx, 4, 4), 1)
    s.alpha_pic_flip = 1.0
    s.fixed_timestep = 1
    s.timestep = 0.1 * dx / 10.0
    s.bclo[0] = nt.BC_NOSLIP
    pos = scenes.lattice((0, 0, 0), (1.0, 4 * dx, 4 * dx), (dx, dx, dx), (2, 2, 2))
    p = scenes.make_particles(pos, (dx, dx, dx), (2, 2, 2), 1.0, 0, E=100.0, nu=0.0)
    p.rdata[nt.R_VEL] = 0.1 * np.sin(np.pi * p.pos[0] / 2)
    return s, p


def test_axial_bar_first_mode():
    # bar of length 1 fixed at x = 0 and free at x = 1 (buffer cells beyond),
    # v = V0 sin(pi x / 2L) cos(omega t), omega = pi / (2L) sqrt(E / rho)
    s, p = free_end_bar()
    o = orc.Oracle(s)
    o.upload(p)
    o.init_internal_forces()
    n = int(round(0.2 / s.timestep))
    assert o.step(n) == 0
    q = o.download()
    t, _, steps = o.time()
    assert steps == n
    exact = 0.1 * np.sin(np.pi * q.pos[0] / 2) * np.cos(np.pi / 2 * 10.0 * t)
    rms = np.sqrt(np.mean((q.rdata[nt.R_VEL] - exact) ** 2))
    assert rms < 1e-2  # validate.py's criterion is RMS < 1e-1 for V0 = 0.1


def test_flip_energy_conservation():
    s, p = free_end_bar()
    o = orc.Oracle(s)
    o.upload(p)
    o.init_internal_forces()
    e0 = o.diagnostics()
    o.step(300)
    e1 = o.diagnostics()
    E0 = e0["tke"] + e0["tse"]
    E1 = e1["tke"] + e1["tse"]
    assert abs(E1 - E0) / E0 < 0.03
    assert e1["mass"] == e0["mass"]


def test_dt_cfl_and_clamp():
    s, p = scenes.dam_break(n=(16, 8, 8), size=(1.0, 0.5, 0.5), block=(0.4, 0.5, 0.3), seed=1)
    o = orc.Oracle(s)
    o.upload(p)
    dt = o.calculate_time_step()
    c = np.sqrt(2e6 / 1000.0)
    assert abs(dt - 0.1 * (1.0 / 16) / c) / dt < 1e-12
    s.dt_max_limit = 1e-5
    o2 = orc.Oracle(s)
    o2.upload(p)
    assert o2.calculate_time_step() == 1e-5


def periodic_heated_block(n=8, seed=3):
    # a fully periodic block of the heated_block material (no walls, no
    # heat sources): the thermal update only moves heat between particles
    s, p, _ = scenes.heated_block(n=(n, n, n), size=(0.4, 0.4, 0.4), fill=1.0, seed=seed)
    for d in range(3):
        s.periodic[d] = 1
        s.bclo[d] = s.bchi[d] = nt.BC_PERIODIC
        s.bclo_temp[d] = s.bchi_temp[d] = nt.BCT_PERIODIC
        s.gravity[d] = 0.0
    p.rdata[nt.R_HEATSRC] = 0.0
    return s, p


def test_thermal_energy_conserved_without_walls_or_sources():
    # sum_p m cp T changes by dt sum_I source_I = dt sum_p V q . sum_I grad N_I
    # = 0 (the shape functions sum to one) when no BC touches a node
    s, p = periodic_heated_block()
    o = orc.Oracle(s)
    o.upload(p)
    o.init_internal_forces()

    def heat(q):
        return float(np.sum(q.rdata[nt.R_MASS] * q.rdata[nt.R_SPHEAT] * q.rdata[nt.R_TEMPERATURE]))

    h0 = heat(o.download())
    assert o.step(40) == 0
    q = o.download()
    assert abs(heat(q) - h0) / h0 < 1e-12
    # conduction smooths the seeded +-20 K field
    assert q.rdata[nt.R_TEMPERATURE].std() < p.rdata[nt.R_TEMPERATURE].std()


def test_isothermal_walls_pull_temperatures():
    # walls held at 350 K on every face heat a 300 K block
    s, p, _ = scenes.heated_block(n=(8, 8, 8), size=(0.4, 0.4, 0.4), fill=1.0, seed=4)
    for d in range(3):
        s.bclo_temp[d] = s.bchi_temp[d] = nt.BCT_ISOTHERMAL
        s.T_wall_lo[d] = s.T_wall_hi[d] = 350.0
        s.gravity[d] = 0.0
    p.rdata[nt.R_TEMPERATURE] = 300.0
    p.rdata[nt.R_HEATSRC] = 0.0
    p.rdata[nt.R_HEATFLUX:nt.R_HEATFLUX + 3] = 0.0
    o = orc.Oracle(s)
    o.upload(p)
    o.init_internal_forces()
    t0 = o.download().rdata[nt.R_TEMPERATURE].mean()
    o.step(30)
    q = o.download()
    t1 = q.rdata[nt.R_TEMPERATURE]
    # heat flows in, and the particles next to the walls are the warm ones
    # (the explicit nodal jump to the wall value can overshoot it on the
    # particles: the scheme does not clamp)
    assert t1.mean() > t0
    r = np.abs(q.pos - 0.2).max(axis=0)
    assert t1[r > 0.15].mean() > t1[r < 0.1].mean() + 10.0
