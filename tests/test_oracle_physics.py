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
