"""Autotuner and tuning knobs: every candidate the tuner may pick renders the
same image (the knobs change launch shapes, queue sizes and the BVH build,
never the sample streams), and the search returns a configuration no slower
than the starting one."""
import numpy as np
import pytest

import agentray
import agentray.scenes as S
import oracle as O
from agentray import _abi as A
from agentray import autotune

pytestmark = pytest.mark.gpu


def _render(scene, cam, integ, w, h):
    out = np.empty(w * h * 3, np.float32)
    integ.render(scene, cam, w, h, out=out)
    return out.reshape(h, w, 3)


def test_set_tuning_validates(ctx):
    before = ctx.tuning()
    with pytest.raises(agentray.AgentRayError):
        ctx.set_tuning(shade_block=96)
    with pytest.raises(agentray.AgentRayError):
        ctx.set_tuning(traversal_blocks_per_sm=9)
    with pytest.raises(ValueError):
        ctx.set_tuning(no_such_knob=1)
    assert ctx.tuning() == before


@pytest.mark.parametrize("kind", ["pt", "bdpt"])
def test_tuning_knobs_keep_the_image(ctx, kind):
    sd, cam = S.served_scene(0)
    scene = agentray.Scene(ctx, sd)
    if kind == "pt":
        integ = agentray.PathTracer(agentray.PathTracerConfig(spp=4, seed=9, film_precision=A.FILM_F64))
    else:
        integ = agentray.BidirectionalPathTracer(agentray.BdptConfig(spp=4, seed=9, film_precision=A.FILM_F64))
    w = h = 64
    base = _render(scene, cam, integ, w, h)
    default = ctx.tuning()
    try:
        ctx.set_tuning(path_capacity=1 << 14, traversal_blocks_per_sm=3, shade_block=64, bdpt_batch_mib=64)
        other = _render(scene, cam, integ, w, h)
    finally:
        ctx.set_tuning(**default)
    np.testing.assert_allclose(other, base, rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("width,leaf", [(4, 1), (6, 2), (2, 3)])
def test_bvh_width_and_leaf_keep_closest_hits(ctx, width, leaf):
    sd, _ = S.served_scene(2)
    scene = agentray.Scene(ctx, sd)
    scene.rebuild(max_leaf_size=leaf, bvh_width=width)
    ot, dt = S.soup_rays(50_000, seed=11)
    ot[:, :3] = ot[:, :3] * np.array([10.0, 5.0, 10.0], np.float32)
    hits, inst = scene.trace_closest(ot, dt)
    ref = O.OracleScene(sd).trace_closest(ot, dt)
    g_prim = hits[:, 3].view(np.uint32)
    same = (g_prim == ref["prim"]) & (inst == ref["inst"])
    tie = np.abs(hits[:, 0] - ref["t"]) <= 1e-6 * np.maximum(1.0, np.abs(ref["t"]))
    assert (same | tie).mean() > 0.9999


def test_autotune_and_cache(ctx, tmp_path):
    sd, cam = S.served_scene(1)
    scene = agentray.Scene(ctx, sd)
    default = ctx.tuning()
    path = str(tmp_path / "tune.json")
    try:
        r = autotune.tune(ctx, scene, cam, integrator="pt", width=128, height=128, spp=2, repeats=2,
                          cache_path=path)
        assert not r["cached"]
        assert r["candidates"] >= 8
        assert r["best_ms"] <= r["default_ms"]
        assert ctx.tuning() == r["tuning"]
        print(f"\nautotune served scene 1 PT 128x128x2: {r}")
        again = autotune.tune(ctx, scene, cam, integrator="pt", width=128, height=128, spp=2, cache_path=path)
        assert again["cached"] and again["tuning"] == r["tuning"]
    finally:
        ctx.set_tuning(**default)
        scene.rebuild()
