"""Seeded synthetic scenes with the shapes, sizes and parameters of the
benchmark workloads (no dataset is used; every particle set is generated here).

Particles sit on the regular per-cell lattice of the reference's generator
(offsets (k + 0.5) / n of a cell per axis, as Tests/*/PreProcess/
Generate_MPs_Inputfile_Generic.py places them) and get the derived fields
InitParticles sets (Source/mpm_init.cpp:1120-1160): V = 4/3 pi r^3 with the
reference's truncated constants, m = rho V, J = 1, F = I.
"""
from __future__ import annotations

import numpy as np

from . import native as nt

FOURBYTHREE = 1.3333333333  # Source/constants.H:9
PI = 3.141592654            # Source/constants.H:10


def lattice(lo, hi, dx, ppc):
    """Lattice points of a box [lo, hi) with ppc points per cell edge."""
    axes = []
    for d in range(3):
        h = dx[d] / ppc[d]
        n = int(np.floor((hi[d] - lo[d]) / h + 1e-9))
        start = lo[d] + 0.5 * h
        pts = start + h * np.arange(n)
        axes.append(pts[pts < hi[d]])
    g = np.meshgrid(*axes, indexing="ij")
    return np.stack([a.ravel(order="F") for a in g])  # x fastest


def make_particles(pos: np.ndarray, dx, ppc, density, model: int, E=0.0, nu=0.0, K=0.0, gamma=0.0, visc=0.0):
    n = pos.shape[1]
    p = nt.Particles(n)
    p.pos[:] = pos
    vol = (dx[0] / ppc[0]) * (dx[1] / ppc[1]) * (dx[2] / ppc[2])
    radius = (vol / (FOURBYTHREE * PI)) ** (1.0 / 3.0)
    v = FOURBYTHREE * PI * radius ** 3
    p.rdata[nt.R_RADIUS] = radius
    p.rdata[nt.R_DENSITY] = density
    p.rdata[nt.R_VOLUME] = v
    p.rdata[nt.R_VOL_INIT] = v
    p.rdata[nt.R_MASS] = density * v
    p.rdata[nt.R_JACOBIAN] = 1.0
    for d in range(3):
        p.rdata[nt.R_DEFGRAD + 4 * d] = 1.0
    p.idata[nt.I_MODEL] = model
    p.idata[nt.I_RIGID_ID] = -1
    if model in (0, 2):  # linear elastic, neo-Hookean
        p.rdata[nt.R_E] = E
        p.rdata[nt.R_NU] = nu
    else:
        p.rdata[nt.R_BULK] = K
        p.rdata[nt.R_GAMMA] = gamma
        p.rdata[nt.R_VISC] = visc
    return p


def base_specs(plo, phi, ncells, order, precision=nt.PREC_FP64):
    s = nt.specs_defaults()
    for d in range(3):
        s.plo[d], s.phi[d], s.ncells[d] = plo[d], phi[d], ncells[d]
        s.gravity[d] = 0.0
    s.order_scheme = order
    for d in range(3):
        s.order[d] = order if (order == 1 or ncells[d] >= 5) else 1
    s.mass_tolerance = 1e-18
    s.precision = precision
    s.max_steps = 1000000
    s.final_time = 1e30
    s.applied_strainrate_time = s.final_time
    return s


def axial_bar(nx=64, steps=1000, precision=nt.PREC_FP64):
    """3-D linear-elastic axial bar: 64x4x4 cells, dx = 1/64, the bar fills
    x in [0,1], 2x2x2 lattice (8192 particles), E = 100, nu = 0, rho = 1,
    v_x = 0.1 sin(pi x / 2), x = 0 face fixed (noslip), x = 1 face slip (the
    reference has no free-end BC), linear shape functions, FLIP 0.99,
    dt = 0.1 dx / sqrt(E / rho)."""
    dx = 1.0 / nx
    ny = 4
    s = base_specs((0, 0, 0), (1.0, ny * dx, ny * dx), (nx, ny, ny), 1, precision)
    s.alpha_pic_flip = 0.99
    s.fixed_timestep = 1
    s.timestep = 0.1 * dx / np.sqrt(100.0 / 1.0)
    s.bclo[0] = nt.BC_NOSLIP
    s.bchi[0] = nt.BC_SLIP
    pos = lattice((0, 0, 0), (1.0, ny * dx, ny * dx), (dx, dx, dx), (2, 2, 2))
    p = make_particles(pos, (dx, dx, dx), (2, 2, 2), 1.0, 0, E=100.0, nu=0.0)
    p.rdata[nt.R_VEL] = 0.1 * np.sin(np.pi * p.pos[0] / 2.0)
    return s, p


def dam_break_specs(n, size, precision=nt.PREC_FP64, order=2):
    """Specs of dam_break: gravity -9.81 in z, CFL 0.1, FLIP 0.99, slip walls."""
    s = base_specs((0, 0, 0), size, n, order, precision)
    s.gravity[2] = -9.81
    s.cfl = 0.1
    s.alpha_pic_flip = 0.99
    return s


def dam_break(n=(256, 128, 128), size=(1.0, 0.5, 0.5), block=(0.4, 0.5, 0.3), seed=1234,
              precision=nt.PREC_FP64, order=2):
    """3-D dam break of a weakly compressible fluid: Tait EOS K = 2e6 Pa,
    gamma = 7, rho0 = 1000, mu = 1e-3; gravity -9.81 in z; the water block in
    the low corner at 2x2x2 particles per cell, jittered uniformly within
    +-0.25 dx from a seed; quadratic B-splines, slip walls, CFL dt."""
    dx = tuple(size[d] / n[d] for d in range(3))
    s = dam_break_specs(n, size, precision, order)
    pos = lattice((0, 0, 0), block, dx, (2, 2, 2))
    rng = np.random.default_rng(seed)
    pos = pos + rng.uniform(-0.25, 0.25, size=pos.shape) * np.array(dx)[:, None]
    for d in range(3):
        pos[d] = np.clip(pos[d], 1e-9 * size[d], size[d] * (1 - 1e-9))
    p = make_particles(pos, dx, (2, 2, 2), 1000.0, 1, K=2e6, gamma=7.0, visc=1e-3)
    return s, p


def sphere_collision(n=256, radius=0.2, precision=nt.PREC_FP64, order=3, speed=0.1, model=0):
    """Two linear-elastic spheres (E = 1e3, nu = 0.3, rho = 1000) of radius
    0.2 centred at (0.3,0.5,0.5) and (0.7,0.5,0.5) moving at +-0.1 m/s in x,
    in a unit cube on an n^3 grid, 2x2x2 lattice; cubic B-splines."""
    dx = 1.0 / n
    s = base_specs((0, 0, 0), (1, 1, 1), (n, n, n), order, precision)
    s.alpha_pic_flip = 0.99
    # the unit cube's lattice restricted to the spheres' bounding box: the
    # same points, in the same (x fastest) order, as filtering the whole cube
    h = dx / 2
    axes = []
    for lo_c, hi_c in ((0.3 - radius, 0.7 + radius), (0.5 - radius, 0.5 + radius), (0.5 - radius, 0.5 + radius)):
        pts = 0.5 * h + h * np.arange(2 * n)
        axes.append(pts[(pts > lo_c - h) & (pts < hi_c + h)])
    g = np.meshgrid(*axes, indexing="ij")
    pos = np.stack([a.ravel(order="F") for a in g])
    c1 = np.array([0.3, 0.5, 0.5])[:, None]
    c2 = np.array([0.7, 0.5, 0.5])[:, None]
    in1 = ((pos - c1) ** 2).sum(0) < radius ** 2
    in2 = ((pos - c2) ** 2).sum(0) < radius ** 2
    sel = in1 | in2
    pos = np.ascontiguousarray(pos[:, sel])
    p = make_particles(pos, (dx, dx, dx), (2, 2, 2), 1000.0, model, E=1e3, nu=0.3)
    p.rdata[nt.R_VEL] = np.where(in1[sel], speed, -speed)
    return s, p


def sphere_union_levelset(specs, centers, radii) -> np.ndarray:
    """One nodal level set, phi = min_i (|x - c_i| - r_i), phi < 0 inside:
    the union of analytic spheres as one body (the MultiUDF union of
    Source/mpm_eb_udf_build.cpp:42-68)."""
    nn = [specs.ncells[d] + 1 for d in range(3)]
    dx = [(specs.phi[d] - specs.plo[d]) / specs.ncells[d] for d in range(3)]
    ax = [specs.plo[d] + dx[d] * np.arange(nn[d]) for d in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    phi = np.full(x.shape, np.inf)
    for c, r in zip(centers, radii):
        phi = np.minimum(phi, np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - r)
    return np.ascontiguousarray(phi.ravel())


def twisted_column(n=(64, 64, 384), size=(0.2, 0.2, 1.2), col=(0.1, 0.1, 0.6), seed=4321,
                   precision=nt.PREC_MIXED, n_obstacles=20, rigid_frac=0.05, order=2, heat=True):
    """Twisted elastic column with obstacles and heat: column col (E = 1e5,
    nu = 0.3, rho = 1000) standing on a noslip base, initial angular velocity
    10 rad/s about its axis, seeded analytic sphere obstacles (r in
    [0.02, 0.05]) as one union level-set body, a seeded fraction of particles
    flagged rigid, quadratic B-splines; with heat, mpm.use_temp = 1 and
    temperatures 300 K plus a seeded Gaussian perturbation of 1e-2 K,
    conductivity 1 W/m/K, cp 1000 J/kg/K, adiabatic walls.  Returns (specs,
    particles, phi)."""
    dx = tuple(size[d] / n[d] for d in range(3))
    s = base_specs((0, 0, 0), size, n, order, precision)
    s.bclo[2] = nt.BC_NOSLIP
    s.alpha_pic_flip = 0.99
    cx, cy = size[0] / 2, size[1] / 2
    lo = (cx - col[0] / 2, cy - col[1] / 2, 0.0)
    hi = (cx + col[0] / 2, cy + col[1] / 2, col[2])
    pos = lattice(lo, hi, dx, (2, 2, 2))
    p = make_particles(pos, dx, (2, 2, 2), 1000.0, 0, E=1e5, nu=0.3)
    omega = 10.0
    p.rdata[nt.R_VEL + 0] = -omega * (p.pos[1] - cy)
    p.rdata[nt.R_VEL + 1] = omega * (p.pos[0] - cx)
    rng = np.random.default_rng(seed)
    p.idata[nt.I_PHASE] = (rng.random(p.n) < rigid_frac).astype(np.int32)
    if heat:
        s.use_temp = 1
        p.rdata[nt.R_TEMPERATURE] = 300.0 + 1e-2 * rng.standard_normal(p.n)
        p.rdata[nt.R_SPHEAT] = 1000.0
        p.rdata[nt.R_THERMCOND] = 1.0
    centers, radii = [], []
    while len(centers) < n_obstacles:
        r = rng.uniform(0.02, 0.05)
        c = rng.uniform([r, r, r], [size[0] - r, size[1] - r, size[2] - r])
        # keep obstacles clear of the column's initial volume
        if (abs(c[0] - cx) < col[0] / 2 + r and abs(c[1] - cy) < col[1] / 2 + r and c[2] < col[2] + r):
            continue
        centers.append(c)
        radii.append(r)
    s.num_bodies = 1
    s.bodies[0].mom_bc = nt.BC_NOSLIP
    phi = sphere_union_levelset(s, centers, radii)
    return s, p, phi


def heated_block(n=(24, 16, 20), size=(1.2, 0.8, 1.0), fill=0.7, order=2, seed=7, precision=nt.PREC_FP64,
                 body_bc=0):
    """Thermo-mechanical block (mpm.use_temp = 1): a linear-elastic block
    (E = 1e4, nu = 0.25, rho = 2000) filling x, y and the lower `fill` of z,
    2x2x2 particles per cell jittered by +-0.2 dx; seeded temperatures
    300 +- 20 K, cp = 900, k = 50, heat sources 1e5 W/m^3 +- 50 %, heat
    fluxes and velocities of seeded noise; gravity -9.81 in z, slip walls.
    Thermal walls: x-lo isothermal 350 K, x-hi convective (h = 20,
    T_inf = 290 K), y-lo user flux 500 W/m^2, y-hi adiabatic, z-lo
    isothermal 280 K, z-hi convective.  body_bc > 0 adds a sphere body
    (r = 0.25 at the block centre) with that thermal BC (1 isothermal
    320 K, 3 heat flux 2e3 W/m^2, 4 convective h = 50, T_inf = 310 K).
    Returns (specs, particles, phi or None)."""
    dx = tuple(size[d] / n[d] for d in range(3))
    s = base_specs((0, 0, 0), size, n, order, precision)
    s.gravity[2] = -9.81
    s.alpha_pic_flip = 0.95
    s.cfl = 0.2
    s.use_temp = 1
    s.bclo_temp[0], s.T_wall_lo[0] = nt.BCT_ISOTHERMAL, 350.0
    s.bchi_temp[0], s.h_hi[0], s.Tinf_hi[0] = nt.BCT_CONVECTION, 20.0, 290.0
    s.bclo_temp[1], s.flux_lo[1] = nt.BCT_USERFLUX, 500.0
    s.bchi_temp[1] = nt.BCT_ADIABATIC
    s.bclo_temp[2], s.T_wall_lo[2] = nt.BCT_ISOTHERMAL, 280.0
    s.bchi_temp[2], s.h_hi[2], s.Tinf_hi[2] = nt.BCT_CONVECTION, 5.0, 300.0
    hi = (size[0], size[1], fill * size[2])
    pos = lattice((0, 0, 0), hi, dx, (2, 2, 2))
    rng = np.random.default_rng(seed)
    pos = pos + rng.uniform(-0.2, 0.2, size=pos.shape) * np.array(dx)[:, None]
    for d in range(3):
        pos[d] = np.clip(pos[d], 1e-9 * size[d], size[d] * (1 - 1e-9))
    p = make_particles(pos, dx, (2, 2, 2), 2000.0, 0, E=1e4, nu=0.25)
    p.rdata[nt.R_VEL:nt.R_VEL + 3] = rng.normal(0, 0.02, (3, p.n))
    p.rdata[nt.R_TEMPERATURE] = 300.0 + rng.uniform(-20.0, 20.0, p.n)
    p.rdata[nt.R_SPHEAT] = 900.0
    p.rdata[nt.R_THERMCOND] = 50.0
    p.rdata[nt.R_HEATSRC] = 1e5 * (1.0 + rng.uniform(-0.5, 0.5, p.n))
    p.rdata[nt.R_HEATFLUX:nt.R_HEATFLUX + 3] = rng.normal(0, 100.0, (3, p.n))
    phi = None
    if body_bc:
        s.num_bodies = 1
        b = s.bodies[0]
        b.mom_bc = nt.BC_SLIP
        b.temp_bc = body_bc
        b.T_wall, b.heat_flux, b.h_conv, b.T_inf = 320.0, 2e3, 50.0, 310.0
        c = (size[0] / 2, size[1] / 2, fill * size[2] / 2)
        phi = sphere_union_levelset(s, [c], [0.25])
    return s, p, phi


def batched_dam_breaks(n_scenes=64, sides=(32, 48, 64, 96, 128), fill=(0.1, 0.4), seed=2024, precision=nt.PREC_MIXED,
                       only=None):
    """Generator of the batched uneven scenes: n_scenes independent dam
    breaks (the dam_break fluid and walls) in unit cubes with a cubic grid
    side drawn from `sides` and a water fill fraction f drawn uniformly from
    `fill`; the block spans x in [0, 2f], all of y and z in [0, 0.5] (volume
    fraction f) at 2x2x2 particles per cell, jittered.  Yields (specs,
    particles) one scene at a time, so the host holds one scene's arrays.
    `only` restricts it to the listed scene indices (each scene keeps its own
    seed, so a subset is the same scenes as in the whole set)."""
    draws = batched_scene_sizes(n_scenes, sides, fill, seed)
    for i, (n, f) in enumerate(draws):
        if only is not None and i not in only:
            continue
        yield dam_break(n=(n, n, n), size=(1.0, 1.0, 1.0), block=(2.0 * f, 1.0, 0.5), seed=seed + 1 + i,
                        precision=precision)


def batched_specs(n_scenes=64, sides=(32, 48, 64, 96, 128), fill=(0.1, 0.4), seed=2024, precision=nt.PREC_MIXED,
                  only=None):
    """Specs of the scenes batched_dam_breaks yields, without particles."""
    return [dam_break_specs((n, n, n), (1.0, 1.0, 1.0), precision)
            for i, (n, _) in enumerate(batched_scene_sizes(n_scenes, sides, fill, seed))
            if only is None or i in only]


def lattice_count(lo, hi, dx, ppc) -> int:
    """Number of points lattice(lo, hi, dx, ppc) generates, without them."""
    n = 1
    for d in range(3):
        h = dx[d] / ppc[d]
        k = int(np.floor((hi[d] - lo[d]) / h + 1e-9))
        pts = lo[d] + 0.5 * h + h * np.arange(k)
        n *= int((pts < hi[d]).sum())
    return n


def batched_scene_particle_counts(n_scenes=64, sides=(32, 48, 64, 96, 128), fill=(0.1, 0.4), seed=2024):
    """Particles of every scene batched_dam_breaks generates (jitter and
    clipping keep the lattice count), computed without generating them."""
    return [lattice_count((0, 0, 0), (2.0 * f, 1.0, 0.5), (1.0 / n,) * 3, (2, 2, 2))
            for n, f in batched_scene_sizes(n_scenes, sides, fill, seed)]


def partition_scenes(counts, nparts):
    """Scenes dealt to nparts ranks by particle count, largest first, each
    to the rank with the fewest particles so far (ties to the lower rank and
    the lower scene index): the scene-level counterpart of the reference's
    DistributionMapping of its boxes over MPI ranks (Source/mpm_init.cpp:
    154-158).  Returns each rank's ascending list of scene indices; every
    rank computes the same lists, with no communication."""
    order = sorted(range(len(counts)), key=lambda i: (-counts[i], i))
    load = [0] * nparts
    parts = [[] for _ in range(nparts)]
    for i in order:
        r = min(range(nparts), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += counts[i]
    return [sorted(p) for p in parts]


def batched_scene_sizes(n_scenes=64, sides=(32, 48, 64, 96, 128), fill=(0.1, 0.4), seed=2024):
    """(side, fill) of every scene batched_dam_breaks generates."""
    rng = np.random.default_rng(seed)
    return [(int(rng.choice(sides)), float(rng.uniform(*fill))) for _ in range(n_scenes)]
