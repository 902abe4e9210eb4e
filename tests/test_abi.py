"""The C-ABI library loads without a GPU and exports every symbol that
include/exg.h declares; host-only entry points work on the CPU."""
import re
from pathlib import Path

import numpy as np
import pytest

from exagoop_b200 import native as nt

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "exg.h").read_text()
    return sorted(set(re.findall(r"\b(exg_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol():
    L = nt.lib()
    names = declared_symbols()
    assert len(names) >= 40
    for n in names:
        assert hasattr(L, n), n
    assert sorted(nt.EXPORTED) == names


def test_struct_sizes_match_header():
    # ctypes mirrors must match the C layout; exg_specs_default writes the
    # whole struct, so a short mirror would be overrun (checked by a guard)
    import ctypes as C

    class Guarded(C.Structure):
        _fields_ = [("s", nt.Specs), ("guard", C.c_uint64 * 8)]

    g = Guarded()
    for i in range(8):
        g.guard[i] = 0xDEADBEEFCAFEF00D
    nt.lib().exg_specs_default(C.byref(g.s))
    assert all(g.guard[i] == 0xDEADBEEFCAFEF00D for i in range(8))
    assert g.s.mass_tolerance == 1e-8 and g.s.alpha_pic_flip == 0.95 and g.s.cfl == 0.1


def test_python_specs_defaults_match_the_library():
    # the CPU-only benchmark legs build specs without loading libexg.so; the
    # Python mirror must equal exg_specs_default byte for byte
    import ctypes as C

    a, b = nt.default_specs(), nt.specs_defaults()
    assert C.string_at(C.addressof(a), C.sizeof(a)) == C.string_at(C.addressof(b), C.sizeof(b))


INPUTS = """
# inputs in the reference's key set
mpm.prob_lo = 0.0 0.0 0.0
mpm.prob_hi = 1.0 0.5 0.5      # domain
mpm.ncells = 64 32 4
mpm.is_it_periodic = 0 0 0
mpm.max_grid_size = 32
mpm.max_steps = 100
mpm.final_time = 2.0
mpm.order_scheme = 3
mpm.stress_update_scheme = "MUSL"
mpm.alpha_pic_flip = 0.9
mpm.fixed_timestep = 1
mpm.timestep = 1e-4
mpm.gravity = 0.0 0.0 -9.81
mpm.bc_xlo_mom = noslip
mpm.bc_zhi_mom = partialslip
mpm.bc_zhi_mom.wall_mu = 0.25
mpm.bc_ylo_mom.wall_vel = 0.1 0.0 0.0
eb2.body_names = ball
ball.geom_type = sphere
ball.sphere_radius = 0.1
ball.sphere_center = 0.5 0.25 0.25
ball.levelset_mom = partialslip
ball.lset_wall_mu = 0.4
exg.precision = mixed
"""


def test_inputs_to_specs():
    inp = nt.Inputs(text=INPUTS, overrides=["mpm.max_steps=7", "mpm.CFL=0.2"])
    s = inp.specs()
    assert list(s.ncells) == [64, 32, 4]
    assert s.max_steps == 7 and s.cfl == 0.2
    assert s.stress_update_scheme == 1 and s.alpha_pic_flip == 0.9
    assert s.fixed_timestep == 1 and s.timestep == 1e-4
    assert list(s.order) == [3, 3, 1]  # ncells < 5 falls back to linear (mpm_init.cpp:231)
    assert s.bclo[0] == nt.BC_NOSLIP and s.bchi[2] == nt.BC_PARTIALSLIP and s.bclo[1] == nt.BC_SLIP
    assert s.wall_mu_hi[2] == 0.25 and s.wall_mu_lo[0] == 0.1
    assert s.wall_vel_lo[3] == 0.1
    assert s.applied_strainrate_time == 2.0 and s.write_output_time == 0.2
    assert s.num_bodies == 1 and s.bodies[0].mom_bc == nt.BC_PARTIALSLIP and s.bodies[0].wall_mu == 0.4
    assert s.precision == nt.PREC_MIXED
    phi = inp.levelset(s, 0)
    nn = [s.ncells[d] + 1 for d in range(3)]
    i, j, k = 32, 16, 2
    assert phi[(k * nn[1] + j) * nn[0] + i] < 0  # inside the ball
    assert phi[0] > 0


def test_inputs_errors():
    bad = INPUTS.replace('"MUSL"', "XUSL")
    try:
        nt.Inputs(text=bad).specs()
    except nt.ExgError as e:
        assert e.code == -1 and "USL/MUSL" in str(e)
    else:
        raise AssertionError("bad stress_update_scheme accepted")


def test_ascii_particle_file(tmp_path):
    f = tmp_path / "mpm_particles.dat"
    f.write_text("dim: 3\nnumber_of_material_points: 2\n# phase x y z radius density vx vy vz model ...\n"
                 "0 0.1 0.2 0.3 0.01 1000 1 2 3 0 1e5 0.3\n"
                 "1 0.4 0.5 0.6 0.02 500 0 0 0 1 2e6 7 0.001\n")
    p = nt.Particles.read_ascii(str(f))
    assert p.n == 2
    assert p.idata[nt.I_PHASE].tolist() == [0, 1] and p.idata[nt.I_MODEL].tolist() == [0, 1]
    v = 1.3333333333 * 3.141592654 * 0.01 ** 3
    assert p.rdata[nt.R_VOLUME, 0] == v and p.rdata[nt.R_MASS, 0] == 1000 * v
    assert p.rdata[nt.R_BULK, 1] == 2e6 and p.rdata[nt.R_GAMMA, 1] == 7
    assert np.allclose(p.pos[:, 1], [0.4, 0.5, 0.6])
    assert p.rdata[nt.R_DEFGRAD, 0] == 1.0 and p.rdata[nt.R_DEFGRAD + 1, 0] == 0.0


def test_grid_beyond_the_32_bit_bin_keys_is_refused():
    # spec validation runs before any CUDA call, so no GPU is needed: 1624^3
    # cells pad to 204^3 tiles of 512 cells, 4.35e9 keys, beyond 2^32 - 1
    s = nt.specs_defaults()
    for d in range(3):
        s.ncells[d] = 1624
    with pytest.raises(nt.ExgError) as e:
        nt.Context(s)
    assert e.value.code == -1  # EXG_ERR_CONFIG
