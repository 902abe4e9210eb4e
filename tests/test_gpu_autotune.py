"""The launch-variant autotuner (exg_autotune, exg_set_variants,
exg_get_variants), and the fused G2P's two ways of staging node blocks.  Every P2G variant (rows per pass x threads per block)
and every fused-G2P variant (threads per block x blocks per SM) must give
bit-identical particles after fused steps: the P2G sums each node over a
cell's particles in storage order with the same expression whatever the
launch shape, then adds cells exactly in fixed point; the G2P updates each
particle independently.  The tuner's choice must be the one the steps use."""
import numpy as np
import pytest

from exagoop_b200 import native as nt, scenes

pytestmark = pytest.mark.gpu

NV = 3


def small(name, precision):
    if name == "spheres_cubic":
        s, p = scenes.sphere_collision(n=32)
        # off the lattice, so that weights reach the ends of their supports
        # (where the truncated spline constants make them a little negative),
        # and some rigid particles, which no variant deposits
        dx = 1.0 / 32
        p.pos += np.random.default_rng(5).uniform(-0.45, 0.45, p.pos.shape) * dx
        p.idata[nt.I_PHASE, ::23] = 1
    else:
        s, p = scenes.dam_break(n=(32, 16, 16), size=(1.0, 0.5, 0.5), block=(0.4, 0.5, 0.3), seed=31)
    s.precision = precision
    s.autotune = 0
    return s, p


def run(s, p, steps, p2g=None, g2p=None, tune=False):
    ctx = nt.Context(s)
    ctx.upload(p)
    ctx.Initialise_Internal_Forces()
    if tune:
        ctx.autotune()
    if p2g is not None or g2p is not None:
        ctx.set_variants(-1 if p2g is None else p2g, -1 if g2p is None else g2p)
    ctx.step(steps)
    out = ctx.download(), ctx.variants()
    ctx.close()
    return out


def same(a, b):
    return np.array_equal(a.rdata, b.rdata) and np.array_equal(a.pos, b.pos) and np.array_equal(a.idata, b.idata)


@pytest.mark.parametrize("precision", [nt.PREC_MIXED, nt.PREC_FP64])
@pytest.mark.parametrize("name", ["spheres_cubic", "dam_break_quadratic"])
def test_every_variant_is_bit_identical(name, precision):
    s, p = small(name, precision)
    ref, v = run(s, p, 12, 0, 0)
    assert v["p2g"] == 0 and v["g2p"] == 0
    for k in range(1, NV):
        got, v = run(s, p, 12, k, 0)
        assert v["p2g"] == k and same(got, ref), ("p2g variant", k)
        got, v = run(s, p, 12, 0, k)
        assert v["g2p"] == k and same(got, ref), ("g2p variant", k)
    got, _ = run(s, p, 12, NV - 1, NV - 1)
    assert same(got, ref)


@pytest.mark.parametrize("name", ["spheres_cubic", "dam_break_quadratic"])
def test_autotune_measures_and_uses_its_choice(name):
    s, p = small(name, nt.PREC_MIXED)
    got, v = run(s, p, 10, tune=True)
    assert 0 <= v["p2g"] < NV and 0 <= v["g2p"] < NV
    assert all(t > 0 for t in v["p2g_ms"]) and all(t > 0 for t in v["g2p_ms"])
    assert v["p2g_ms"][v["p2g"]] == min(v["p2g_ms"]) and v["g2p_ms"][v["g2p"]] == min(v["g2p_ms"])
    # the tuning run leaves the state as it found it: the steps that follow
    # equal an untuned run bit for bit
    ref, _ = run(s, p, 10, 0, 0)
    assert same(got, ref)


def test_first_step_tunes_when_enabled():
    s, p = small("spheres_cubic", nt.PREC_MIXED)
    s.autotune = 1
    ctx = nt.Context(s)
    ctx.upload(p)
    ctx.Initialise_Internal_Forces()
    ctx.step(3)
    v = ctx.variants()
    assert 0 <= v["p2g"] < NV and 0 <= v["g2p"] < NV
    got = ctx.download()
    ctx.close()
    ref, _ = run(s, p, 3, 0, 0)
    assert same(got, ref)


def test_set_variants_rejects_out_of_range():
    s, p = small("spheres_cubic", nt.PREC_MIXED)
    ctx = nt.Context(s)
    with pytest.raises(nt.ExgError):
        ctx.set_variants(NV, 0)
    with pytest.raises(nt.ExgError):
        ctx.set_variants(0, -2)
    ctx.close()


@pytest.mark.parametrize("name", ["spheres_cubic", "dam_break_quadratic"])
@pytest.mark.parametrize("precision", [nt.PREC_MIXED, nt.PREC_FP64])
def test_tma_and_plain_node_staging_agree(name, precision, monkeypatch):
    # the fused G2P stages each tile's node block by one TMA box from the
    # nodal records, or (EXG_NO_TMA, and on periodic grids) by plain loads:
    # the same values in the same layout, so the steps agree bit for bit
    s, p = small(name, precision)
    ref, _ = run(s, p, 8, 0, 0)
    monkeypatch.setenv("EXG_NO_TMA", "1")
    got, _ = run(s, p, 8, 0, 0)
    assert same(got, ref)
