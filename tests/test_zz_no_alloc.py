"""exg_p2g_momentum_noalloc: the P2G entry point for callers that cannot call
cudaMalloc (inside another component's global-mode graph capture, under a
host-owned device pool or fixed memory budget, in allocation-free real-time
loops).  Its scratch is a static device array, so the test gives it only
caller-owned input and output buffers and checks two calls in a row against
exg_p2g_momentum of a context on the same particles, within the FP64 parity
tolerance of the other GPU tests.  Collected last so that a stop at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

from exagoop_b200 import native as nt, scenes

pytestmark = pytest.mark.gpu

TOL64 = 1e-10


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def scene(seed, order, n=(20, 12, 16), npart=5000):
    rng = np.random.default_rng(seed)
    s = scenes.base_specs((0.1, -0.2, 0.0), (1.1, 0.4, 0.8), n, order)
    s.gravity[2] = -3.0
    dx = [(s.phi[d] - s.plo[d]) / n[d] for d in range(3)]
    pos = np.stack([rng.uniform(s.plo[d], s.phi[d], npart) for d in range(3)])
    p = scenes.make_particles(pos, dx, (2, 2, 2), 900.0, 0, E=2e3, nu=0.25)
    p.rdata[nt.R_VEL:nt.R_VEL + 3] = rng.normal(0, 0.3, (3, npart))
    p.rdata[nt.R_STRESS:nt.R_STRESS + 6] = rng.normal(0, 50.0, (6, npart))
    p.idata[nt.I_PHASE, ::13] = 1
    return s, p


@pytest.mark.parametrize("order", [1, 2, 3])
def test_noalloc_matches_context_p2g(order):
    import torch

    s, p = scene(70 + order, order)
    ctx = nt.Context(s)
    ctx.upload(p)
    ctx.P2G_Momentum(1, 1, 1)
    ref = [ctx.nodes(nt.N_MASS)] + [ctx.nodes(nt.N_VEL + d) for d in range(3)] + \
          [ctx.nodes(nt.N_FRC + d) for d in range(3)]
    ctx.close()

    dev = torch.device("cuda:0")
    pos = torch.from_numpy(p.pos).to(dev).contiguous()
    rdata = torch.from_numpy(p.rdata).to(dev).contiguous()
    idata = torch.from_numpy(p.idata).to(dev).contiguous()
    nn = (s.ncells[0] + 1) * (s.ncells[1] + 1) * (s.ncells[2] + 1)
    mass = torch.zeros(nn, dtype=torch.float64, device=dev)
    vel = torch.zeros(3 * nn, dtype=torch.float64, device=dev)
    frc = torch.zeros(3 * nn, dtype=torch.float64, device=dev)
    soa = nt.ParticleSoA(p.n, C.cast(pos.data_ptr(), C.POINTER(C.c_double)),
                         C.cast(rdata.data_ptr(), C.POINTER(C.c_double)),
                         C.cast(idata.data_ptr(), C.POINTER(C.c_int32)))
    stream = torch.cuda.current_stream(dev).cuda_stream
    L = nt.lib()
    for call in range(2):
        # garbage in the outputs: every node must be written
        mass.fill_(123.0)
        vel.fill_(-7.0)
        frc.fill_(3.0)
        rc = L.exg_p2g_momentum_noalloc(C.byref(s), C.byref(soa),
                                        C.cast(mass.data_ptr(), C.POINTER(C.c_double)),
                                        C.cast(vel.data_ptr(), C.POINTER(C.c_double)),
                                        C.cast(frc.data_ptr(), C.POINTER(C.c_double)), C.c_void_p(stream))
        assert rc == 0
        torch.cuda.synchronize()
        got = [mass.cpu().numpy()] + [vel[d * nn:(d + 1) * nn].cpu().numpy() for d in range(3)] + \
              [frc[d * nn:(d + 1) * nn].cpu().numpy() for d in range(3)]
        for k, (g, r) in enumerate(zip(got, ref)):
            assert rel(g, r) < TOL64, (call, k, rel(g, r))


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
