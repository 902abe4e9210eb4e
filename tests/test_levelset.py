"""Level-set bodies built from the inputs (mpm_ebtools::init_eb,
Source/mpm_eb.cpp:402-547): the analytic shapes parsed from the eb2.* /
<body>.* keys, the host builder against the closed-form signed distances,
and (GPU) the device builder bit-for-bit against the host builder, unions of
spheres against the NumPy union, a stepped scene whose level set came from
the device builder against the same scene given the host level set, and the
command-line driver on an inputs file with a body."""
import numpy as np
import pytest

from exagoop_b200 import native as nt, scenes

INPUTS = """
mpm.prob_lo = 0.0 0.0 0.0
mpm.prob_hi = 1.0 0.5 0.5
mpm.ncells = 40 20 24
mpm.order_scheme = 2
mpm.is_it_periodic = 0 0 0
mpm.max_grid_size = 32
mpm.max_steps = 10
mpm.final_time = 1.0
eb2.body_names = ball floor post crate hollow
ball.geom_type = sphere
ball.sphere_radius = 0.1
ball.sphere_center = 0.5 0.25 0.25
floor.geom_type = plane
floor.plane_point = 0.0 0.0 0.05
floor.plane_normal = 0.0 0.3 1.0
post.geom_type = cylinder
post.cylinder_radius = 0.07
post.cylinder_center = 0.2 0.25 0.2
post.cylinder_height = 0.3
post.cylinder_direction = 2
crate.geom_type = box
crate.box_lo = 0.7 0.1 0.05
crate.box_hi = 0.9 0.3 0.2
hollow.geom_type = sphere
hollow.sphere_radius = 0.2
hollow.sphere_center = 0.5 0.25 0.25
hollow.sphere_has_fluid_inside = 1
"""


def node_coords(s):
    nn = [s.ncells[d] + 1 for d in range(3)]
    dx = [(s.phi[d] - s.plo[d]) / s.ncells[d] for d in range(3)]
    ax = [s.plo[d] + dx[d] * np.arange(nn[d]) for d in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    return x.ravel(), y.ravel(), z.ravel()


def closed_form(s):
    x, y, z = node_coords(s)
    ball = np.sqrt((x - 0.5) ** 2 + (y - 0.25) ** 2 + (z - 0.25) ** 2) - 0.1
    n = np.array([0.0, 0.3, 1.0])
    floor = (x * n[0] + y * n[1] + (z - 0.05) * n[2]) / np.linalg.norm(n)
    q0 = np.sqrt((x - 0.2) ** 2 + (y - 0.25) ** 2) - 0.07
    q1 = np.abs(z - 0.2) - 0.15
    post = np.hypot(np.maximum(q0, 0), np.maximum(q1, 0)) + np.minimum(np.maximum(q0, q1), 0)
    lo, hi = np.array([0.7, 0.1, 0.05]), np.array([0.9, 0.3, 0.2])
    q = np.stack([np.abs(x - 0.8), np.abs(y - 0.2), np.abs(z - 0.125)]) - ((hi - lo) / 2)[:, None]
    crate = np.sqrt((np.maximum(q, 0) ** 2).sum(0)) + np.minimum(q.max(0), 0)
    hollow = -(np.sqrt((x - 0.5) ** 2 + (y - 0.25) ** 2 + (z - 0.25) ** 2) - 0.2)
    return [ball, floor, post, crate, hollow]


def test_shapes_from_inputs():
    inp = nt.Inputs(text=INPUTS)
    s = inp.specs()
    assert s.num_bodies == 5
    sh = [inp.levelset_shape(b) for b in range(5)]
    assert sh[0].kind == nt.LS_SPHERE and sh[0].radius == 0.1 and list(sh[0].center) == [0.5, 0.25, 0.25]
    assert sh[1].kind == nt.LS_PLANE and list(sh[1].normal) == [0.0, 0.3, 1.0]
    assert sh[2].kind == nt.LS_CYLINDER and sh[2].dir == 2 and sh[2].height == 0.3
    assert sh[3].kind == nt.LS_BOX and list(sh[3].hi) == [0.9, 0.3, 0.2]
    assert sh[4].inside == 1 and sh[0].inside == 0


def test_host_builder_matches_closed_form():
    inp = nt.Inputs(text=INPUTS)
    s = inp.specs()
    for b, ref in enumerate(closed_form(s)):
        phi = inp.levelset(s, b)
        assert np.abs(phi - ref).max() < 1e-15, b


def test_udf_body_has_no_analytic_shape():
    inp = nt.Inputs(text=INPUTS.replace("ball.geom_type = sphere", "ball.geom_type = udf_cpp\n"
                                        "ball.udf_so_file = ./missing.so"))
    with pytest.raises(nt.ExgError) as e:
        inp.levelset_shape(0)
    assert e.value.code == -9  # EXG_ERR_UNSUPPORTED


@pytest.mark.gpu
def test_device_builder_is_bitwise_host_builder():
    inp = nt.Inputs(text=INPUTS)
    s = inp.specs()
    ctx = nt.Context(s)
    ctx.init_levelsets(inp)
    for b in range(5):
        assert np.array_equal(ctx.get_levelset(b), inp.levelset(s, b)), b
    # one body rebuilt from an explicit shape list
    ctx.build_levelset(2, [inp.levelset_shape(3)])
    assert np.array_equal(ctx.get_levelset(2), inp.levelset(s, 3))
    ctx.close()


@pytest.mark.gpu
def test_device_union_of_spheres_matches_numpy():
    s, _ = scenes.dam_break(n=(48, 24, 24), size=(1.0, 0.5, 0.5), precision=nt.PREC_FP64)
    rng = np.random.default_rng(5)
    centers = rng.uniform([0.1, 0.1, 0.1], [0.9, 0.4, 0.4], size=(20, 3))
    radii = rng.uniform(0.02, 0.08, size=20)
    ctx = nt.Context(s)
    ctx.build_levelset(0, [nt.LsShape.sphere(c, r) for c, r in zip(centers, radii)])
    assert np.array_equal(ctx.get_levelset(0), scenes.sphere_union_levelset(s, centers, radii))
    with pytest.raises(nt.ExgError):
        ctx.get_levelset(1)  # never built
    with pytest.raises(nt.ExgError):
        ctx.build_levelset(0, [nt.LsShape(kind=9)])
    ctx.close()


@pytest.mark.gpu
def test_stepping_with_device_level_set_matches_host_level_set():
    s, p, _ = scenes.twisted_column(n=(16, 16, 48), precision=nt.PREC_FP64, n_obstacles=6, heat=False)
    rng = np.random.default_rng(11)
    centers = rng.uniform([0.02, 0.02, 0.1], [0.18, 0.18, 1.1], size=(6, 3))
    radii = rng.uniform(0.02, 0.05, size=6)
    out = []
    for use_device in (False, True):
        ctx = nt.Context(s)
        if use_device:
            ctx.build_levelset(0, [nt.LsShape.sphere(c, r) for c, r in zip(centers, radii)])
        else:
            ctx.set_levelset(0, scenes.sphere_union_levelset(s, centers, radii))
        ctx.upload(p)
        ctx.Initialise_Internal_Forces()
        ctx.step(20)
        out.append(ctx.download())
        ctx.close()
    assert np.array_equal(out[0].rdata, out[1].rdata)
    assert np.array_equal(out[0].pos, out[1].pos)


DRIVER_INPUTS = """
mpm.prob_lo = 0.0 0.0 0.0
mpm.prob_hi = 1.0 1.0 1.0
mpm.ncells = 16 16 16
mpm.is_it_periodic = 0 0 0
mpm.max_grid_size = 16
mpm.max_steps = 60
mpm.final_time = 10.0
mpm.order_scheme = 2
mpm.fixed_timestep = 1
mpm.timestep = 1e-3
mpm.gravity = 0.0 0.0 -9.81
mpm.bc_zlo_mom = noslip
mpm.particle_file = particles.dat
mpm.write_ascii = 1
mpm.write_output_time = 100.0
mpm.print_diagnostics = 1
mpm.do_calculate_tke_tse = 1
mpm.write_diag_output_time = 0.0
mpm.screen_output_time = 100.0
eb2.body_names = rock
rock.geom_type = sphere
rock.sphere_radius = 0.15
rock.sphere_center = 0.5 0.5 0.35
rock.levelset_mom = slipwall
exg.precision = fp64
"""


def write_block(path):
    h = 1.0 / 32
    c = (np.arange(12) + 0.5) * h
    g = np.stack(np.meshgrid(0.3 + c, 0.3 + c, 0.52 + c[:8], indexing="ij"), -1).reshape(-1, 3)
    rad = (3 * h ** 3 / (4 * np.pi)) ** (1 / 3)
    lines = [f"0 {x:.17g} {y:.17g} {z:.17g} {rad:.17g} 1000 0 0 -2 0 2e5 0.3" for x, y, z in g]
    path.write_text(f"dim: 3\nnumber_of_material_points: {len(g)}\n# phase x y z radius density vx vy vz "
                    f"model E nu\n" + "\n".join(lines) + "\n")
    return len(g)


@pytest.mark.gpu
def test_driver_runs_inputs_with_a_level_set_body(tmp_path):
    """The command-line driver on an inputs file with an analytic body (built
    on the GPU) against the same run through the Python API."""
    import subprocess
    from pathlib import Path
    n = write_block(tmp_path / "particles.dat")
    (tmp_path / "inputs").write_text(DRIVER_INPUTS)
    drv = Path(nt.__file__).resolve().parent / "exg_driver"
    r = subprocess.run([str(drv), "inputs"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    dumps = sorted((tmp_path / "Solution" / "ascii_files").iterdir())
    assert len(dumps) == 2
    rows = dumps[-1].read_text().split("\n")
    assert int(rows[0]) == n
    got = np.array([[float(v) for v in ln.split()] for ln in rows[5:] if ln.strip()])
    energies = (tmp_path / "Diagnostics" / "Total_Energies.dat").read_text().split("\n")
    assert len([e for e in energies[1:] if e.strip()]) == 60

    inp = nt.Inputs(text=DRIVER_INPUTS)
    ctx = nt.Context(inp.specs())
    ctx.init_levelsets(inp)
    ctx.upload(nt.Particles.read_ascii(str(tmp_path / "particles.dat")))
    ctx.Initialise_Internal_Forces()
    ctx.step(60)
    ref = ctx.download()
    ctx.close()
    assert np.allclose(got[:, :3], ref.pos.T, rtol=1e-10, atol=1e-12)
    v = got[:, 3 + nt.R_VEL:3 + nt.R_VEL + 3]
    assert np.allclose(v, ref.rdata[nt.R_VEL:nt.R_VEL + 3].T, rtol=1e-10, atol=1e-12)
    assert np.abs(v[:, :2]).max() > 1e-2  # the block hit the rock and spread sideways
