"""GPU parity of the thermal step functions (USE_TEMP build of the reference)
against the FP64 oracle on the same seeded inputs: P2G_Temperature, the
nodal backup / time update / store-delta, Apply_Nodal_BCs_Temperature
(domain walls of every kind, UDF walls, level-set bodies), G2P_Temperature,
the thermal prologue of Initialise_Internal_Forces and the fused USL / MUSL
steps.  FP64 tolerance: 1e-10 relative to the field's max norm."""
import ctypes as C

import numpy as np
import pytest

from exagoop_b200 import native as nt, scenes
import orc

pytestmark = pytest.mark.gpu

TOL64 = 1e-10
THERMAL_NODES = [("mass_spheat", nt.N_MASS_SPHEAT), ("mass_spheat_temp", nt.N_MASS_SPHEAT_TEMP),
                 ("temperature", nt.N_TEMPERATURE), ("source", nt.N_SOURCE_TEMP),
                 ("delta_temperature", nt.N_DELTA_TEMPERATURE), ("mass_cond", nt.N_MASS_COND)]
THERMAL_PARTS = [("temperature", nt.R_TEMPERATURE, 1), ("heatflux", nt.R_HEATFLUX, 3)]


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


def check_nodes(ctx, o, comps=THERMAL_NODES, tol=TOL64):
    for name, comp in comps:
        e = rel(ctx.nodes(comp), o.nodes(comp))
        assert e < tol, f"node {name}: max rel err {e:.3e}"


def check_parts(g, r, fields, tol=TOL64):
    for name, f, k in fields:
        e = rel(g.rdata[f:f + k], r.rdata[f:f + k])
        assert e < tol, f"{name}: max rel err {e:.3e}"


@pytest.mark.parametrize("order", [1, 2, 3])
@pytest.mark.parametrize("flags", [(1, 1, 1), (1, 1, 0), (1, 0, 1)])
def test_p2g_temperature(order, flags):
    s, p, _ = scenes.heated_block(order=order, seed=10 + order)
    ctx, o = pair(s, p)
    ctx.P2G_Momentum(1, 1, 1)
    o.p2g_momentum(1, 1, 1)
    ctx.P2G_Temperature(*flags)
    o.p2g_temperature(*flags)
    check_nodes(ctx, o, [c for c in THERMAL_NODES if c[1] != nt.N_DELTA_TEMPERATURE])


def nodal_sequence(x, dt, time, dirichlet_only, oracle):
    if oracle:
        x.p2g_momentum(1, 1, 1)
        x.p2g_temperature(1, 1, 1)
        x.backup_current_temperature()
        x.nodal_time_update_temperature(dt)
        x.apply_nodal_bcs_temperature(dt, time, dirichlet_only)
        x.store_delta_temperature()
    else:
        x.P2G_Momentum(1, 1, 1)
        x.P2G_Temperature(1, 1, 1)
        x.backup_current_temperature()
        x.Nodal_Time_Update_Temperature(dt)
        x.Apply_Nodal_BCs_Temperature(dt, time, dirichlet_only)
        x.store_delta_temperature()


@pytest.mark.parametrize("body_bc", [0, 1, 3, 4])
def test_nodal_temperature_bcs(body_bc):
    s, p, phi = scenes.heated_block(seed=20 + body_bc, body_bc=body_bc)
    ctx, o = pair(s, p, phi)
    nodal_sequence(ctx, 0.01, 0.0, 0, False)
    nodal_sequence(o, 0.01, 0.0, 0, True)
    check_nodes(ctx, o)


def test_nodal_temperature_bcs_dirichlet_only():
    # MUSL's first thermal BC pass applies only isothermal bodies
    s, p, phi = scenes.heated_block(seed=31, body_bc=4)
    ctx, o = pair(s, p, phi)
    nodal_sequence(ctx, 0.01, 0.0, 1, False)
    nodal_sequence(o, 0.01, 0.0, 1, True)
    check_nodes(ctx, o)


@pytest.mark.parametrize("walls", ["corners", "periodic_x"])
def test_wall_chains(walls):
    # every face of the box with a BC that reads its neighbour: corner and
    # edge nodes take the sweep-order values of chains of two and three links
    # (a periodic axis needs at least three 8-cell tiles)
    s, p, _ = scenes.heated_block(n=(24, 16, 16), size=(1.2, 0.8, 0.8), fill=1.0, seed=41)
    for d in range(3):
        s.bclo_temp[d], s.flux_lo[d] = nt.BCT_USERFLUX, 300.0 * (d + 1)
        s.bchi_temp[d], s.h_hi[d], s.Tinf_hi[d] = nt.BCT_CONVECTION, 10.0 * (d + 1), 280.0 + 5 * d
    s.bchi_temp[1] = nt.BCT_ADIABATIC
    if walls == "periodic_x":
        s.periodic[0] = 1
        s.bclo[0] = s.bchi[0] = nt.BC_PERIODIC
        s.bclo_temp[0] = s.bchi_temp[0] = nt.BCT_PERIODIC
    ctx, o = pair(s, p)
    nodal_sequence(ctx, 0.01, 0.0, 0, False)
    nodal_sequence(o, 0.01, 0.0, 0, True)
    check_nodes(ctx, o)


UDF_T = C.CFUNCTYPE(None, C.c_double, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double))


@UDF_T
def _udf_conv(x, y, z, t, out):
    out[0] = 15.0 + 10.0 * x + 5.0 * z + t
    out[1] = 290.0 + 20.0 * z


@UDF_T
def _udf_iso(x, y, z, t, out):
    out[0] = 330.0 + 10.0 * y - 5.0 * z
    out[1] = 0.0


def test_udf_temperature_walls():
    s, p, _ = scenes.heated_block(seed=51)
    s.bclo_temp[1] = nt.BCT_CONVECTION
    s.udf_temp_lo[1] = C.cast(_udf_conv, C.c_void_p).value
    s.bchi_temp[0] = nt.BCT_ISOTHERMAL
    s.udf_temp_hi[0] = C.cast(_udf_iso, C.c_void_p).value
    ctx, o = pair(s, p)
    nodal_sequence(ctx, 0.01, 0.25, 0, False)
    nodal_sequence(o, 0.01, 0.25, 0, True)
    check_nodes(ctx, o)


@pytest.mark.parametrize("order", [1, 2, 3])
def test_g2p_temperature(order):
    s, p, phi = scenes.heated_block(order=order, seed=60 + order, body_bc=3)
    ctx, o = pair(s, p, phi)
    nodal_sequence(ctx, 0.01, 0.0, 0, False)
    nodal_sequence(o, 0.01, 0.0, 0, True)
    ctx.G2P_Temperature(1, 1)
    o.g2p_temperature(1, 1)
    check_parts(ctx.download(), o.download(), THERMAL_PARTS)


def test_g2p_temperature_mixed_orders():
    # 4 cells in y: quadratic falls back to linear on that axis
    s, p, _ = scenes.heated_block(n=(20, 4, 12), order=2, seed=71)
    assert list(s.order) == [2, 1, 2]
    ctx, o = pair(s, p)
    nodal_sequence(ctx, 0.01, 0.0, 0, False)
    nodal_sequence(o, 0.01, 0.0, 0, True)
    ctx.G2P_Temperature(1, 1)
    o.g2p_temperature(1, 1)
    check_parts(ctx.download(), o.download(), THERMAL_PARTS)


def test_init_internal_forces_thermal():
    s, p, phi = scenes.heated_block(seed=81, body_bc=1)
    ctx, o = pair(s, p, phi)
    ctx.Initialise_Internal_Forces()
    o.init_internal_forces()
    check_parts(ctx.download(), o.download(), THERMAL_PARTS + [("stress", nt.R_STRESS, 6)])


FUSED_FIELDS = THERMAL_PARTS + [("vel", nt.R_VEL, 3), ("stress", nt.R_STRESS, 6), ("jacobian", nt.R_JACOBIAN, 1)]


@pytest.mark.parametrize("scheme,body_bc", [(0, 0), (0, 4), (1, 0), (1, 1), (1, 3)])
def test_fused_thermal_step(scheme, body_bc):
    s, p, phi = scenes.heated_block(seed=90 + 10 * scheme + body_bc, body_bc=body_bc)
    s.stress_update_scheme = scheme
    ctx, o = pair(s, p, phi)
    ctx.Initialise_Internal_Forces()
    o.init_internal_forces()
    ctx.step(10)
    assert o.step(10) == 0
    check_parts(ctx.download(), o.download(), FUSED_FIELDS)
    # nodal T = (m cp T) / (m cp): the fixed-point deposit has absolute, not
    # relative, precision, so nodes at the rim of the support (mass below
    # 1e-6 of its maximum, which particles weight by ~N as well) are left out;
    # the momentum mass marks them (MUSL's second deposit zeroes m cp).
    # delta T = T - T_old inherits the absolute error of T, so its bound is
    # relative to max |T|
    m = o.nodes(nt.N_MASS)
    sel = m >= 1e-6 * m.max()
    T = o.nodes(nt.N_TEMPERATURE)[sel]
    Tscale = np.abs(T).max()
    for name, comp in [("temperature", nt.N_TEMPERATURE), ("delta_temperature", nt.N_DELTA_TEMPERATURE)]:
        e = np.abs(ctx.nodes(comp)[sel] - o.nodes(comp)[sel]).max() / Tscale
        assert e < TOL64, f"node {name}: max err {e:.3e} of max |T|"


def test_fused_thermal_udf():
    s, p, _ = scenes.heated_block(seed=97)
    s.bclo_temp[1] = nt.BCT_CONVECTION
    s.udf_temp_lo[1] = C.cast(_udf_conv, C.c_void_p).value
    ctx, o = pair(s, p)
    ctx.Initialise_Internal_Forces()
    o.init_internal_forces()
    ctx.step(6)
    assert o.step(6) == 0
    check_parts(ctx.download(), o.download(), FUSED_FIELDS)


def test_mixed_precision_thermal():
    # FP32 state with FP64 temperatures and positions against the FP64
    # oracle after 40 steps: temperatures to 1e-6 relative
    s, p, _ = scenes.heated_block(seed=99)
    sm = s.copy()
    sm.precision = nt.PREC_MIXED
    ctx = nt.Context(sm)
    ctx.upload(p)
    ctx.Initialise_Internal_Forces()
    o = orc.Oracle(s)
    o.upload(p)
    o.init_internal_forces()
    ctx.step(40)
    o.step(40)
    g, r = ctx.download(), o.download()
    eT = np.linalg.norm(g.rdata[nt.R_TEMPERATURE] - r.rdata[nt.R_TEMPERATURE]) / np.linalg.norm(r.rdata[nt.R_TEMPERATURE])
    assert eT < 1e-6, eT


def test_fused_thermal_periodic_conserves_heat():
    # fully periodic, no sources: the GPU step matches the oracle and keeps
    # sum m cp T to round-off (no BC touches a node)
    s, p, _ = scenes.heated_block(n=(24, 24, 24), size=(0.6, 0.6, 0.6), fill=1.0, seed=7)
    for d in range(3):
        s.periodic[d] = 1
        s.bclo[d] = s.bchi[d] = nt.BC_PERIODIC
        s.bclo_temp[d] = s.bchi_temp[d] = nt.BCT_PERIODIC
        s.gravity[d] = 0.0
    p.rdata[nt.R_HEATSRC] = 0.0
    ctx, o = pair(s, p)
    ctx.Initialise_Internal_Forces()
    o.init_internal_forces()

    def heat(q):
        return float(np.sum(q.rdata[nt.R_MASS] * q.rdata[nt.R_SPHEAT] * q.rdata[nt.R_TEMPERATURE]))

    h0 = heat(ctx.download())
    ctx.step(10)
    assert o.step(10) == 0
    g, r = ctx.download(), o.download()
    check_parts(g, r, FUSED_FIELDS)
    assert abs(heat(g) - h0) / h0 < 1e-12
