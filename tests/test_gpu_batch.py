"""Batches of independent scenes (exg_batch): every scene of a batch ends
bit-for-bit where the same scene ends when stepped alone through its own
context (the batched kernels run the same tile code over the concatenated
tile lists), and within 1e-10 of the FP64 oracle; incompatible scene sets
are rejected."""
import numpy as np
import pytest

from exagoop_b200 import native as nt, scenes
import orc

pytestmark = pytest.mark.gpu

TOL64 = 1e-10


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def uneven_scenes(precision):
    out = []
    for n, block, seed in [((32, 16, 16), (0.4, 0.5, 0.3), 1), ((24, 24, 24), (0.3, 0.5, 0.2), 2),
                           ((40, 16, 24), (0.2, 0.5, 0.45), 3)]:
        s, p = scenes.dam_break(n=n, size=(1.0, 0.5, 0.5) if n[1] == 16 else (0.5, 0.5, 0.5), block=block,
                                seed=seed, precision=precision)
        out.append((s, p, None))
    s, p, phi = scenes.twisted_column(n=(16, 16, 48), precision=precision, n_obstacles=6, heat=False)
    out.append((s, p, phi))
    return out


def run_batch(items, nsteps):
    b = nt.Batch([s for s, _, _ in items])
    for sc, (s, p, phi) in zip(b.scenes, items):
        if phi is not None:
            sc.set_levelset(0, phi)
        sc.upload(p)
        sc.Initialise_Internal_Forces()
    b.step(nsteps)
    return b, [sc.download() for sc in b.scenes]


def run_single(s, p, phi, nsteps):
    ctx = nt.Context(s)
    if phi is not None:
        ctx.set_levelset(0, phi)
    ctx.upload(p)
    ctx.Initialise_Internal_Forces()
    ctx.step(nsteps)
    return ctx, ctx.download()


@pytest.mark.parametrize("precision", [nt.PREC_FP64, nt.PREC_MIXED])
def test_batch_matches_single_contexts(precision):
    items = uneven_scenes(precision)
    b, got = run_batch(items, 12)
    for i, (s, p, phi) in enumerate(items):
        ctx, ref = run_single(s, p, phi, 12)
        assert np.array_equal(got[i].rdata, ref.rdata), f"scene {i}"
        assert np.array_equal(got[i].pos, ref.pos), f"scene {i}"
        assert b.scenes[i].time() == ctx.time()
    b.close()


def test_batch_matches_oracle():
    items = uneven_scenes(nt.PREC_FP64)
    b, got = run_batch(items, 10)
    for i, (s, p, phi) in enumerate(items):
        o = orc.Oracle(s)
        o.upload(p)
        if phi is not None:
            o.set_levelset(0, phi)
        o.init_internal_forces()
        assert o.step(10) == 0
        r = o.download()
        for name, f, k in [("vel", nt.R_VEL, 3), ("stress", nt.R_STRESS, 6), ("defgrad", nt.R_DEFGRAD, 9),
                           ("jacobian", nt.R_JACOBIAN, 1)]:
            e = rel(got[i].rdata[f:f + k], r.rdata[f:f + k])
            assert e < TOL64, f"scene {i} {name}: {e:.3e}"
        assert np.abs(got[i].pos - r.pos).max() < TOL64
    b.close()


def test_batch_rejects_incompatible_scenes():
    s1, _ = scenes.dam_break(n=(32, 16, 16), precision=nt.PREC_FP64)
    s2, _ = scenes.sphere_collision(n=32)  # cubic
    with pytest.raises(nt.ExgError):
        nt.Batch([s1, s2])
    s3 = s1.copy()
    s3.stress_update_scheme = 1
    with pytest.raises(nt.ExgError):
        nt.Batch([s1, s3])
    s4, _, _ = scenes.heated_block()
    with pytest.raises(nt.ExgError):
        nt.Batch([s4])
