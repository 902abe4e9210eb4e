"""Reference cases through the compatibility layer: inputs files and ASCII
material-point files written by the reference's own pre-processor
(tests/golden/make_reference_cases.py runs its write_inputs_file and
write_particles_ascii_streaming on two small 3-D configurations) are read by
exg_inputs_parse / exg_specs_from_inputs and exg_particles_read_ascii.  On
the GPU the cases run through the replacement driver, whose matpnt dumps are
read with the column map of the reference's post-processing (x y z, then
realData index + 3), and through the C ABI against the FP64 oracle."""
import json
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from exagoop_b200 import native as nt

GOLD = Path(__file__).resolve().parent / "golden"
ROOT = Path(__file__).resolve().parents[1]
CASES = ["dam_break_3d", "elastic_block_3d"]
FOURBYTHREE, PI = 1.3333333333, 3.141592654  # Source/constants.H:9-10
BC = {"slip": nt.BC_SLIP, "noslip": nt.BC_NOSLIP, "partialslip": nt.BC_PARTIALSLIP}


def case(name):
    cfg = json.loads((GOLD / f"refcase_{name}.json").read_text())
    return cfg, nt.Inputs(str(GOLD / f"refcase_{name}.inp"))


@pytest.mark.parametrize("name", CASES)
def test_generated_inputs_file_parses(name):
    cfg, inp = case(name)
    s = inp.specs()
    g = cfg["grid"]
    ax = "xyz"
    for d in range(3):
        assert s.plo[d] == g[f"{ax[d]}min"] and s.phi[d] == g[f"{ax[d]}max"] and s.ncells[d] == g[f"n{ax[d]}"]
        assert s.order[d] == cfg["order_scheme"]
        assert s.gravity[d] == cfg["gravity"][d]
    # every 3-D domain the pre-processor writes is periodic in z
    assert list(s.periodic) == [0, 0, 1]
    for d, lo, hi in ((0, "xlo", "xhi"), (1, "ylo", "yhi")):
        assert s.bclo[d] == BC[cfg["boundary_conditions"][lo]["mom"]]
        assert s.bchi[d] == BC[cfg["boundary_conditions"][hi]["mom"]]
    assert s.stress_update_scheme == (1 if cfg["stress_update_scheme"] == "MUSL" else 0)
    assert s.alpha_pic_flip == cfg["alpha_pic_flip"] and s.cfl == cfg["CFL"]
    assert s.mass_tolerance == 1e-18
    sim = cfg["simulation"]
    assert s.max_steps == sim["max_steps"] and s.final_time == sim["final_time"]
    assert s.fixed_timestep == sim["fixed_timestep"]
    if sim["fixed_timestep"]:
        assert s.timestep == sim["timestep"]
    assert s.print_diagnostics == cfg["diagnostics"].get("print_diagnostics", 0)
    assert inp.get("mpm.particle_file") == f"refcase_{name}.dat"  # quotes removed, as ParmParse does


@pytest.mark.parametrize("name", CASES)
def test_generated_particle_file_reads(name):
    cfg, _ = case(name)
    p = nt.Particles.read_ascii(str(GOLD / f"refcase_{name}.dat"))
    assert p.n == cfg["particles"]
    body = cfg["body"]
    sh = body["shape"]
    for d, ax in enumerate("xyz"):
        assert p.pos[d].min() > sh[f"{ax}min"] and p.pos[d].max() < sh[f"{ax}max"]
    # lattice offsets (k + 0.5) / ppc of a cell, printed with 7 digits
    g = cfg["grid"]
    dx = (g["xmax"] - g["xmin"]) / g["nx"]
    off = (p.pos[0] - g["xmin"]) / (dx / cfg["ppc"][0]) - 0.5
    assert np.abs(off - np.round(off)).max() < 1e-4
    v = body["initial_velocity"]
    assert np.allclose(p.rdata[nt.R_VEL:nt.R_VEL + 3].T, [v["vx"], v["vy"], v["vz"]], rtol=1e-6)
    assert np.all(p.rdata[nt.R_DENSITY] == cfg["density"])
    r = p.rdata[nt.R_RADIUS]
    vol = FOURBYTHREE * PI * r ** 3
    assert np.array_equal(p.rdata[nt.R_VOLUME], vol) and np.array_equal(p.rdata[nt.R_MASS], cfg["density"] * vol)
    cm = body["constitutive_model"]
    if cm["type"] == "fluid":
        assert np.all(p.idata[nt.I_MODEL] == 1)
        assert np.all(p.rdata[nt.R_BULK] == cm["Bulk_modulus"]) and np.all(p.rdata[nt.R_GAMMA] == cm["Gamma_pressure"])
        assert np.all(p.rdata[nt.R_VISC] == cm["Dynamic_viscosity"])
    else:
        assert np.all(p.idata[nt.I_MODEL] == 0)
        assert np.all(p.rdata[nt.R_E] == cm["E"]) and np.all(p.rdata[nt.R_NU] == cm["nu"])
    assert np.all(p.rdata[nt.R_DEFGRAD] == 1.0) and np.all(p.rdata[nt.R_JACOBIAN] == 1.0)


def steps_of(s):
    """Steps the driver's time loop (main.cpp:83-187) takes for these specs."""
    return int(s.max_steps)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_reference_case_against_oracle(name):
    import orc
    cfg, inp = case(name)
    s = inp.specs()
    p = nt.Particles.read_ascii(str(GOLD / f"refcase_{name}.dat"))
    n = 20
    ctx = nt.Context(s)
    ctx.upload(p)
    ctx.Initialise_Internal_Forces()
    ctx.step(n)
    g = ctx.download()
    ctx.close()
    o = orc.Oracle(s, threads=os.cpu_count() or 1)
    o.upload(p)
    o.init_internal_forces()
    assert o.step(n) == 0
    r = o.download()
    # stresses are compared against the stress of a 1e-5 strain of the
    # stiffest modulus: the elastic block translates rigidly, so its stress
    # is rounding noise (~1e-16 of the modulus) that two correct codes need
    # not share; 1e-10 of that floor is 1e-15 of the modulus
    stiff = max(r.rdata[nt.R_E].max(), r.rdata[nt.R_BULK].max())
    for f, k, floor in [(nt.R_VEL, 3, 0.0), (nt.R_STRESS, 6, 1e-5 * stiff), (nt.R_DEFGRAD, 9, 0.0),
                        (nt.R_DENSITY, 1, 0.0)]:
        b = r.rdata[f:f + k]
        assert np.abs(g.rdata[f:f + k] - b).max() <= 1e-10 * max(np.abs(b).max(), floor, 1e-300), f
    assert np.abs(g.pos - r.pos).max() < 1e-12


@pytest.mark.gpu
def test_driver_dumps_in_the_reference_column_layout(tmp_path):
    # the elastic case through exagoop_b200/exg_driver: its last matpnt dump,
    # read the way the reference's post-processing reads it, equals a
    # context stepped as far through the C ABI
    name = "elastic_block_3d"
    cfg, inp = case(name)
    for ext in ("inp", "dat"):
        shutil.copy(GOLD / f"refcase_{name}.{ext}", tmp_path / f"refcase_{name}.{ext}")
    drv = ROOT / "exagoop_b200" / "exg_driver"
    out = subprocess.run([str(drv), f"refcase_{name}.inp", "exg.precision=fp64"], cwd=tmp_path,
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    s = inp.specs()
    nsteps = steps_of(s)
    t_end = nsteps * s.timestep
    dump = tmp_path / "Solution" / "ascii_files" / f"refcase_{name}" / f"matpnt_t{t_end:.6f}"
    assert dump.exists(), sorted(str(x) for x in tmp_path.rglob("matpnt*"))
    head = dump.read_text().splitlines()[:5]
    assert head == [str(cfg["particles"]), "46", "3", "0", "0"]
    data = np.loadtxt(dump, skiprows=5)
    assert data.shape == (cfg["particles"], 3 + 46 + 3)
    p = nt.Particles.read_ascii(str(GOLD / f"refcase_{name}.dat"))
    ctx = nt.Context(s)
    ctx.upload(p)
    ctx.Initialise_Internal_Forces()
    ctx.step(nsteps)
    g = ctx.download()
    ctx.close()
    dim = 3
    assert np.allclose(data[:, 0:3].T, g.pos, rtol=1e-11, atol=1e-12)
    # realData index + AMREX_SPACEDIM, as the reference's readers index it
    for f, k in [(nt.R_RADIUS, 1), (nt.R_VEL, 3), (nt.R_VEL_PRIME, 3), (nt.R_STRAINRATE, 6), (nt.R_STRAIN, 6),
                 (nt.R_STRESS, 6), (nt.R_DEFGRAD, 9), (nt.R_VOLUME, 1), (nt.R_MASS, 1), (nt.R_DENSITY, 1),
                 (nt.R_JACOBIAN, 1), (nt.R_PRESSURE, 1), (nt.R_VOL_INIT, 1), (nt.R_E, 1), (nt.R_NU, 1)]:
        col = data[:, f + dim:f + dim + k].T
        ref = g.rdata[f:f + k]
        assert np.allclose(col, ref, rtol=1e-11, atol=1e-11 * max(np.abs(ref).max(), 1e-300)), f
    assert np.array_equal(data[:, 3 + 46:].T.astype(np.int32), g.idata)
