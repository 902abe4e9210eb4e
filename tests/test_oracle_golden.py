"""The oracle's restated math against golden vectors produced by the
reference's own header-only sources (tests/golden/make_golden.py, via the
reference pin), and against the live reference pin where the reference tree
is present.  CPU only."""
from pathlib import Path

import ctypes as C
import numpy as np
import pytest

from exagoop_b200 import native as nt, scenes
import orc

G = Path(__file__).resolve().parent / "golden"
pd = C.POINTER(C.c_double)
pi = C.POINTER(C.c_int)


def P(a):
    return a.ctypes.data_as(pd if a.dtype == np.float64 else pi)


def test_splines_bit_exact():
    f = np.load(G / "splines.npz")
    z, vals = f["z"], f["values"]
    L = orc.lib()
    for kind in range(4):
        for t in range(1, 5):
            got = np.array([L.orc_fn_spline(kind, t, float(v)) for v in z])
            assert np.array_equal(got, vals[kind, t]), (kind, t)


def oracle_for(nc, order, periodic, plo, dx):
    s = nt.default_specs()
    for d in range(3):
        s.ncells[d] = int(nc[d])
        s.order[d] = int(order[d])
        s.periodic[d] = int(periodic[d])
        s.plo[d] = float(plo[d])
        s.phi[d] = float(plo[d] + dx[d] * nc[d])
    return orc.Oracle(s)


def test_basis_and_grad():
    cases = np.load(G / "basis.npz")["cases"]
    worst = 0.0
    skipped = 0
    for row in cases:
        nc, order, per, cell, st = (row[0:3], row[3:6], row[6:9], row[9:12], row[12:15])
        plo, dx, x, N, grad = row[15:18], row[18:21], row[21:24], row[24], row[25:28]
        # a cubic coordinate that rounds outside [-2, 2) makes the reference
        # index its coefficient table out of bounds (interpolants.H:222);
        # those rows hold undefined values and are not compared
        z = (x - (plo + (cell + st) * dx)) / dx
        iv = np.floor(z) + 2
        if np.any((order == 3) & ((iv < 0) | (iv > 3))):
            skipped += 1
            continue
        o = oracle_for(nc.astype(int), order.astype(int), per.astype(int), plo, dx)
        g = np.zeros(3)
        got = o.L.orc_fn_basis_and_grad(o.h, P(st.astype(np.int32)), P(cell.astype(np.int32)), P(x.copy()), P(g))
        scale = max(1.0, abs(N))
        worst = max(worst, abs(got - N) / scale)
        gs = max(1.0, np.abs(grad).max())
        worst = max(worst, np.abs(g - grad).max() / gs)
    # dx is rebuilt as (hi - lo) / ncells, as AMReX does; a coordinate on a
    # knot can then fall in the neighbouring polynomial piece, and the
    # reference's truncated constants (onebysix = 0.16666666666667,
    # fourbythree = 1.3333333333) leave the pieces ~1e-11 apart at the knots
    assert worst < 1e-10
    assert skipped < len(cases) // 50


def test_interp_two():
    f = np.load(G / "interp.npz")
    rows, nodes, offs = f["rows"], f["nodes"], f["offsets"]
    worst = 0.0
    for row in rows:
        case, scheme = int(row[0]), int(row[1])
        nc, order, cell, mn, mx = (row[2:5].astype(int), row[5:8].astype(int), row[8:11].astype(np.int32),
                                   row[11:14].astype(np.int32), row[14:17].astype(np.int32))
        plo, dx, x, vals = row[17:20], row[20:23], row[23:26], row[26:28]
        o = oracle_for(nc, order, (0, 0, 0), plo, dx)
        arr = nodes[offs[case]:offs[case + 1]].reshape((2, nc[2] + 3, nc[1] + 3, nc[0] + 3))
        for c in range(2):
            inner = np.ascontiguousarray(arr[c, 1:-1, 1:-1, 1:-1]).ravel()
            o.L.orc_set_nodes(o.h, c, P(inner))
        got = np.zeros(2)
        o.L.orc_fn_interp_two(o.h, scheme, P(x.copy()), P(cell), P(mn), P(mx), 0, 1, P(got))
        worst = max(worst, np.abs(got - vals).max() / max(1.0, np.abs(vals).max()))
    assert worst < 1e-12


def test_applybc_bit_exact():
    rows = np.load(G / "applybc.npz")["rows"]
    L = orc.lib()
    for r in rows:
        vin, n, mu, bc, out0, out1, mod = r[0:3], r[3:6], r[6], int(r[7]), r[8:11], r[11:14], int(r[14])
        o = out0.copy()
        m = L.orc_fn_applybc(P(vin.copy()), P(o), mu, P(n.copy()), bc)
        assert m == mod
        assert np.array_equal(o, out1)


def test_constitutive_and_defgrad_bit_exact():
    rows = np.load(G / "constitutive.npz")["rows"]
    L = orc.lib()
    for r in rows:
        eps, E, nu, s1, mu, p, s2 = r[0:6], r[6], r[7], r[8:14], r[14], r[15], r[16:22]
        F, g, dt, F2 = r[22:31], r[31:40], r[40], r[41:50]
        a = np.zeros(6)
        L.orc_fn_linear_elastic(P(eps.copy()), P(a), E, nu)
        assert np.array_equal(a, s1)
        b = np.zeros(6)
        L.orc_fn_newtonian(P(eps.copy()), P(b), mu, p)
        assert np.array_equal(b, s2)
        f = F.copy()
        L.orc_fn_defgrad(P(f), P(g.copy()), dt)
        assert np.array_equal(f, F2)


def test_neo_hookean_and_delta_bit_exact():
    # neo_hookean (constitutive_models.H:161-250) and linear_elastic_delta
    # (:69-104) against the reference's own header, small and large strains
    rows = np.load(G / "neo_hookean.npz")["rows"]
    L = orc.lib()
    for r in rows:
        F, E, nu, s_ref, deps, ds_ref = r[0:9], r[9], r[10], r[11:17], r[17:23], r[23:29]
        a = np.zeros(6)
        L.orc_fn_neo_hookean(P(F.copy()), P(a), E, nu)
        assert np.array_equal(a, s_ref)
        b = np.zeros(6)
        L.orc_fn_linear_elastic(P(deps.copy()), P(b), E, nu)  # the delta operator is Hooke's
        assert np.array_equal(b, ds_ref)


def test_levelset_sampling():
    f = np.load(G / "levelset.npz")
    nc, plo, dx, phi, rows = f["nc"], f["plo"], f["dx"], f["phi"], f["rows"]
    o = oracle_for(nc, (1, 1, 1), (0, 0, 0), plo, dx)
    inner = np.ascontiguousarray(phi[1:-1, 1:-1, 1:-1]).ravel()
    o.set_levelset(0, inner)
    n_checked = 0
    for r in rows:
        x, v, g = r[0:3], r[3], r[4:7]
        idx = np.floor((x - plo + 1e-20) / dx).astype(int)
        if np.any(idx < 0) or np.any(idx + 1 > nc):
            continue  # corners in the ghost layer: the oracle uses 1.0 there
        gg = np.zeros(3)
        got = o.L.orc_fn_levelset(o.h, 0, P(x.copy()), P(gg))
        assert abs(got - v) <= 1e-12 * max(1, abs(v))
        assert np.abs(gg - g).max() <= 1e-12 * max(1, np.abs(g).max())
        n_checked += 1
    assert n_checked > 500


@pytest.mark.skipif(not orc.REFPIN.exists(), reason="reference tree not present")
def test_live_reference_pin_splines():
    L = C.CDLL(str(orc.REFPIN))
    for n in ("ref_cubic1d", "ref_quad1d_der"):
        getattr(L, n).restype = C.c_double
        getattr(L, n).argtypes = [C.c_int, C.c_double]
    O = orc.lib()
    for z in np.linspace(-1.99, 1.99, 97):
        for t in range(1, 5):
            assert O.orc_fn_spline(0, t, z) == L.ref_cubic1d(t, z)
            assert O.orc_fn_spline(3, t, z) == L.ref_quad1d_der(t, z)


def test_partition_of_unity():
    # sum_I N_I = 1 and sum_I grad N_I = 0 inside the domain, every order and
    # near each boundary (known-answer property of the B-spline basis)
    L = orc.lib()
    rng = np.random.default_rng(5)
    for order in (1, 2, 3):
        o = oracle_for((9, 9, 9), (order,) * 3, (0, 0, 0), (0, 0, 0), (0.1, 0.1, 0.1))
        for _ in range(300):
            cell = rng.integers(0, 9, 3).astype(np.int32)
            x = (cell + rng.uniform(0, 1, 3)) * 0.1
            s, gs = 0.0, np.zeros(3)
            rng_b = [(0, 2) if order == 1 else ((0, 3) if c == 0 else ((-1, 2) if c == 8 else (-1, 3))) for c in cell]
            for n in range(*rng_b[2]):
                for m in range(*rng_b[1]):
                    for l in range(*rng_b[0]):
                        g = np.zeros(3)
                        s += L.orc_fn_basis_and_grad(o.h, P(np.array([l, m, n], dtype=np.int32)), P(cell), P(x), P(g))
                        gs += g
            # the reference's boundary-modified quadratic spline is not a
            # partition of unity on the first/last interval (type-2/4 pieces)
            interior = np.all((cell >= 2) & (cell <= 6))
            if order == 1 or interior:
                assert abs(s - 1.0) < 1e-9, (order, cell, s)
                assert np.abs(gs).max() < 1e-7, (order, cell, gs)
