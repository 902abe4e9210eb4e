"""exg_p2g_momentum_noalloc: the P2G entry point for callers that cannot call
cudaMalloc (inside another component's global-mode graph capture, under a
host-owned device pool or fixed memory budget, in allocation-free real-time
loops).  Its scratch is a static device array, so the test gives it only
caller-owned input and output buffers and checks two calls in a row against
exg_p2g_momentum of a context on the same particles, within the FP64 parity
tolerance of the other GPU tests.  The cases cover every path with code of
its own in the no-alloc kernels: uniform orders 1-3, mixed per-axis orders,
a periodic axis (the wrap of node ncells onto node 0), the external-force
slab, nodes below mass_tolerance (velocity zeroed), a non-finite input (NaN
outputs) and a large grid followed by a smaller one (only the words a call
uses are cleared).  Collected last so that a stop at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from exagoop_b200 import native as nt, scenes

pytestmark = pytest.mark.gpu

TOL64 = 1e-10


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def scene(seed, order, n=(20, 12, 16), npart=5000, periodic_axis=None, slab=False, mass_quantile=None):
    rng = np.random.default_rng(seed)
    s = scenes.base_specs((0.1, -0.2, 0.0), (1.1, 0.4, 0.8), n, order)
    s.gravity[2] = -3.0
    if periodic_axis is not None:
        s.periodic[periodic_axis] = 1
        s.bclo[periodic_axis] = s.bchi[periodic_axis] = nt.BC_PERIODIC
    if slab:
        s.external_loads = 1
        for d in range(3):
            s.force_slab_lo[d] = s.plo[d] + 0.25 * (s.phi[d] - s.plo[d])
            s.force_slab_hi[d] = s.plo[d] + 0.7 * (s.phi[d] - s.plo[d])
            s.extforce[d] = 0.3 * (d + 1)
    dx = [(s.phi[d] - s.plo[d]) / n[d] for d in range(3)]
    pos = np.stack([rng.uniform(s.plo[d], s.phi[d], npart) for d in range(3)])
    p = scenes.make_particles(pos, dx, (2, 2, 2), 900.0, 0, E=2e3, nu=0.25)
    p.rdata[nt.R_VEL:nt.R_VEL + 3] = rng.normal(0, 0.3, (3, npart))
    p.rdata[nt.R_STRESS:nt.R_STRESS + 6] = rng.normal(0, 50.0, (6, npart))
    p.idata[nt.I_PHASE, ::13] = 1
    return s, p


class Buffers:
    """Device copies of a particle set and caller-owned nodal outputs."""

    def __init__(self, s, p):
        import torch
        dev = torch.device("cuda:0")
        self.pos = torch.from_numpy(p.pos).to(dev).contiguous()
        self.rdata = torch.from_numpy(p.rdata).to(dev).contiguous()
        self.idata = torch.from_numpy(p.idata).to(dev).contiguous()
        self.nn = (s.ncells[0] + 1) * (s.ncells[1] + 1) * (s.ncells[2] + 1)
        self.mass = torch.zeros(self.nn, dtype=torch.float64, device=dev)
        self.vel = torch.zeros(3 * self.nn, dtype=torch.float64, device=dev)
        self.frc = torch.zeros(3 * self.nn, dtype=torch.float64, device=dev)
        self.soa = nt.ParticleSoA(p.n, C.cast(self.pos.data_ptr(), C.POINTER(C.c_double)),
                                  C.cast(self.rdata.data_ptr(), C.POINTER(C.c_double)),
                                  C.cast(self.idata.data_ptr(), C.POINTER(C.c_int32)))
        self.stream = torch.cuda.current_stream(dev).cuda_stream

    def call(self, s):
        import torch
        # garbage in the outputs: every node must be written
        self.mass.fill_(123.0)
        self.vel.fill_(-7.0)
        self.frc.fill_(3.0)
        dp = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_double))  # noqa: E731
        rc = nt.lib().exg_p2g_momentum_noalloc(C.byref(s), C.byref(self.soa), dp(self.mass), dp(self.vel),
                                               dp(self.frc), C.c_void_p(self.stream))
        torch.cuda.synchronize()
        nn = self.nn
        return rc, [self.mass.cpu().numpy()] + [self.vel[d * nn:(d + 1) * nn].cpu().numpy() for d in range(3)] + \
            [self.frc[d * nn:(d + 1) * nn].cpu().numpy() for d in range(3)]


def context_p2g(s, p):
    ctx = nt.Context(s)
    ctx.upload(p)
    ctx.P2G_Momentum(1, 1, 1)
    ref = [ctx.nodes(nt.N_MASS)] + [ctx.nodes(nt.N_VEL + d) for d in range(3)] + \
          [ctx.nodes(nt.N_FRC + d) for d in range(3)]
    ctx.close()
    return ref


CASES = {
    "linear": dict(order=1),
    "quadratic": dict(order=2),
    "cubic": dict(order=3),
    # order 3 with ncells[0] = 4 < 5: Initialise_Domain's fallback makes
    # x linear, so the orders per axis are (1, 3, 3)
    "mixed_orders_1_3_3": dict(order=3, n=(4, 12, 16)),
    "periodic_y": dict(order=2, n=(20, 24, 16), periodic_axis=1),
    "force_slab": dict(order=3, slab=True),
    # mass_tolerance near the 20 % quantile of the positive nodal masses: the
    # lighter nodes get zero velocity (deposit_onto_grid_momentum's cut)
    "below_mass_tolerance": dict(order=2, mass_quantile=0.2),
}


@pytest.mark.parametrize("case", list(CASES))
def test_noalloc_matches_context_p2g(case):
    kw = CASES[case]
    s, p = scene(70 + len(case), **{k: v for k, v in kw.items() if k != "mass_quantile"})
    if case == "mixed_orders_1_3_3":
        assert list(s.order) == [1, 3, 3]
    ref = context_p2g(s, p)
    if kw.get("mass_quantile"):
        # halfway between two neighbouring nodal masses near the quantile,
        # where the gap is widest: no node sits within rounding of the cut
        ms = np.sort(ref[0][ref[0] > 0])
        i0 = int(kw["mass_quantile"] * len(ms))
        win = np.arange(max(i0 - 50, 0), min(i0 + 50, len(ms) - 1))
        i = win[np.argmax((ms[win + 1] - ms[win]) / ms[win])]
        s.mass_tolerance = float(0.5 * (ms[i] + ms[i + 1]))
        ref = context_p2g(s, p)
    if case == "below_mass_tolerance":
        m = ref[0]
        low = (m > 0) & (m < s.mass_tolerance)
        assert low.any() and (m >= s.mass_tolerance).any()
        assert all(np.all(ref[1 + d][low] == 0.0) for d in range(3))
    buf = Buffers(s, p)
    for call in range(2):
        rc, got = buf.call(s)
        assert rc == 0
        for k, (g, r) in enumerate(zip(got, ref)):
            assert rel(g, r) < TOL64, (case, call, k, rel(g, r))


def test_noalloc_large_grid_then_small_grid():
    # the second call clears only the words of its own (smaller) grid; what
    # the first call left beyond them must not reach its results
    big_s, big_p = scene(81, 3, n=(60, 60, 60), npart=40000)
    assert (61 ** 3) <= nt.EXG_NOALLOC_MAX_NODES
    rc, _ = Buffers(big_s, big_p).call(big_s)
    assert rc == 0
    s, p = scene(82, 2, n=(9, 17, 13), npart=3000)
    ref = context_p2g(s, p)
    rc, got = Buffers(s, p).call(s)
    assert rc == 0
    for k, (g, r) in enumerate(zip(got, ref)):
        assert rel(g, r) < TOL64, (k, rel(g, r))


def test_noalloc_nonfinite_input_gives_nan():
    s, p = scene(90, 2)
    p.rdata[nt.R_VEL + 1, 17] = np.nan  # a phase-0 particle (17 % 13 != 0)
    buf = Buffers(s, p)
    rc, got = buf.call(s)
    assert rc == 0  # the call does not wait for the GPU
    assert all(np.isnan(g).all() for g in got)
    # the next call with finite inputs is clean again
    p.rdata[nt.R_VEL + 1, 17] = 0.1
    ref = context_p2g(s, p)
    rc, got = Buffers(s, p).call(s)
    assert rc == 0
    for k, (g, r) in enumerate(zip(got, ref)):
        assert rel(g, r) < TOL64, (k, rel(g, r))


def test_noalloc_rejects_null_particle_arrays():
    s, p = scene(91, 2)
    buf = Buffers(s, p)
    soa = nt.ParticleSoA(p.n, None, buf.soa.rdata, buf.soa.idata)
    dp = C.cast(buf.mass.data_ptr(), C.POINTER(C.c_double))
    rc = nt.lib().exg_p2g_momentum_noalloc(C.byref(s), C.byref(soa), dp, dp, dp, None)
    assert rc == -8  # EXG_ERR_ARG, nothing launched


def test_noalloc_rejects_oversized_grid():
    import torch

    s, p = scene(5, 2)
    for d in range(3):
        s.ncells[d] = 80  # 81^3 nodes > EXG_NOALLOC_MAX_NODES
    assert 81 ** 3 > nt.EXG_NOALLOC_MAX_NODES
    dev = torch.device("cuda:0")
    pos = torch.from_numpy(p.pos).to(dev).contiguous()
    rdata = torch.from_numpy(p.rdata).to(dev).contiguous()
    idata = torch.from_numpy(p.idata).to(dev).contiguous()
    soa = nt.ParticleSoA(p.n, C.cast(pos.data_ptr(), C.POINTER(C.c_double)),
                         C.cast(rdata.data_ptr(), C.POINTER(C.c_double)),
                         C.cast(idata.data_ptr(), C.POINTER(C.c_int32)))
    out = torch.zeros(8, dtype=torch.float64, device=dev)
    ptr = C.cast(out.data_ptr(), C.POINTER(C.c_double))
    rc = nt.lib().exg_p2g_momentum_noalloc(C.byref(s), C.byref(soa), ptr, ptr, ptr, None)
    assert rc == -6  # EXG_ERR_OVERFLOW, nothing launched
