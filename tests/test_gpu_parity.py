"""GPU parity: libagentray (CUDA, sm_100a) against the CPU oracle on the same
seeded inputs.  Bars:
  * BVH: closest-hit (inst_id, prim_id) equal to the oracle's restatement of
    the reference traversal; a mismatch is tolerated only for ties
    (|t_gpu - t_ref| <= 1e-6 * max(1, t)) or hits within 1e-6 of a triangle edge
    in barycentric terms.  Any-hit booleans likewise.
  * Images: same counter-based sample stream -> per-pixel agreement (rel. 1e-3)
    on >= 99.5% of pixels and means within 1e-4 (PT, BDPT, GDPT, textures,
    glass, the imported OBJ scene and the full-size config-3/4 room); an
    independent-seed run must pass a per-pixel Welch test (|t| > 4.5 on at
    most 0.5-1% of pixels).
  * Red-black SOR: bit-exact to the oracle.
  * Film output: 8-bit bytes equal up to 1 LSB on < 0.1% (CUDA vs libm powf);
    EXR files byte-identical.
"""
import numpy as np
import pytest

import agentray
import agentray.scenes as S
import oracle as O
from agentray import _abi as A
from agentray.scene_data import integrator_cfg

pytestmark = pytest.mark.gpu

INVALID = 0xFFFFFFFF


def _edge_case(u, v, eps=1e-6):
    return (u <= eps) | (v <= eps) | (u + v >= 1 - eps)


def _compare_hits(gpu_hits, gpu_inst, ref, eps_t=1e-6):
    g_prim = gpu_hits[:, 3].view(np.uint32)
    g_t = gpu_hits[:, 0]
    same = (g_prim == ref["prim"]) & (gpu_inst == ref["inst"])
    both = (g_prim != INVALID) & (ref["prim"] != INVALID)
    tie = both & (np.abs(g_t - ref["t"]) <= eps_t * np.maximum(1.0, np.abs(ref["t"])))
    # a hit within 1e-6 of a triangle edge may be found or missed by either
    # side; a miss on one side is excused only by the other side's edge hit
    edge = (((ref["prim"] != INVALID) & _edge_case(ref["u"], ref["v"])) |
            ((g_prim != INVALID) & _edge_case(gpu_hits[:, 1], gpu_hits[:, 2])))
    bad = ~(same | tie | edge)
    return same, bad


def test_closest_hit_soup(ctx):
    sc = S.triangle_soup(200_000, seed=2)
    g = agentray.Scene(ctx, sc)
    osc = O.OracleScene(sc)
    ot, dt = S.soup_rays(200_000, seed=3)
    hits, inst = g.trace_closest(ot, dt)
    ref = osc.trace_closest(ot, dt)
    same, bad = _compare_hits(hits, inst, ref)
    assert bad.sum() == 0, f"{bad.sum()} mismatches"
    assert same.mean() > 0.999
    # exact t/u/v where the same triangle is hit
    m = same & (ref["prim"] != INVALID)
    np.testing.assert_array_equal(hits[m, 0], ref["t"][m])
    np.testing.assert_array_equal(hits[m, 1], ref["u"][m])
    np.testing.assert_array_equal(hits[m, 2], ref["v"][m])


def test_bvh_benchmark_scale_hits_match_oracle(ctx):
    # The BVH micro-benchmark at its own size: 1M triangles (seed 2) and the
    # first 1M of its 16M rays (seed 3), closest hit and any hit (t_max 0.25),
    # against the oracle's restated reference traversal.  Deep trees and full
    # traversal stacks are exercised exactly where the benchmark runs.
    sc = S.triangle_soup(1_000_000, seed=2)
    g = agentray.Scene(ctx, sc)
    osc = O.OracleScene(sc)
    ot, dt = S.soup_rays(16_000_000, seed=3)
    ot, dt = ot[:1_000_000].copy(), dt[:1_000_000].copy()
    hits, inst = g.trace_closest(ot, dt)
    ref = osc.trace_closest(ot, dt)
    same, bad = _compare_hits(hits, inst, ref)
    assert bad.sum() == 0, f"{bad.sum()} unexcused closest-hit mismatches"
    assert same.mean() > 0.999
    m = same & (ref["prim"] != INVALID)
    np.testing.assert_array_equal(hits[m, 0], ref["t"][m])
    dt[:, 3] = 0.25
    occ = g.trace_any(ot, dt)
    oref = osc.trace_any(ot, dt)
    mism = occ != oref
    if mism.any():
        r = osc.trace_closest(ot[mism], dt[mism])
        gh, _ = g.trace_closest(ot[mism], dt[mism])
        near = lambda t, u, v: _edge_case(u, v) | (np.abs(t - 0.25) < 1e-6)
        ok = np.where(oref[mism] != 0, near(r["t"], r["u"], r["v"]), near(gh[:, 0], gh[:, 1], gh[:, 2]))
        assert np.all(ok), f"{(~ok).sum()} unexcused of {mism.sum()} any-hit mismatches"
    assert (occ == oref).mean() > 0.9999
    osc.close()


def test_any_hit_soup(ctx):
    sc = S.triangle_soup(100_000, seed=7)
    g = agentray.Scene(ctx, sc)
    osc = O.OracleScene(sc)
    ot, dt = S.soup_rays(100_000, seed=8, tmax=0.25)
    occ = g.trace_any(ot, dt)
    ref = osc.trace_any(ot, dt)
    mism = occ != ref
    if mism.any():
        # excused only by a boundary case on the side that reports occlusion:
        # its hit lies within 1e-6 of a triangle edge or of t_max
        r = osc.trace_closest(ot[mism], dt[mism])
        gh, _ = g.trace_closest(ot[mism], dt[mism])
        near = lambda t, u, v: _edge_case(u, v) | (np.abs(t - 0.25) < 1e-6)
        ok = np.where(ref[mism] != 0, near(r["t"], r["u"], r["v"]), near(gh[:, 0], gh[:, 1], gh[:, 2]))
        assert np.all(ok), f"{(~ok).sum()} unexcused of {mism.sum()} mismatches"
    assert (occ == ref).mean() > 0.9999


@pytest.mark.parametrize("opts", [None, dict(max_leaf_size=4, sah_node_cost=8.0)])
def test_closest_hit_instanced_room(ctx, opts):
    # opts: the default build, and the largest leaves the API allows (4
    # triangles, node cost 8 so that the SAH keeps full leaves).
    sc, cam = S.room(seed=4, sphere_levels=(3, 3, 2, 2), n_boxes=120)
    g = agentray.Scene(ctx, sc)
    if opts:
        g.rebuild(**opts)
    osc = O.OracleScene(sc)
    rng = np.random.default_rng(9)
    n = 100_000
    ot = np.zeros((n, 4), np.float32)
    dt = np.zeros((n, 4), np.float32)
    ot[:, :3] = rng.uniform((0.1, 0.1, 0.1), (9.9, 4.9, 9.9), (n, 3))
    ot[:, 3] = 1e-4
    d = rng.normal(size=(n, 3))
    dt[:, :3] = d / np.linalg.norm(d, axis=1, keepdims=True)
    dt[:, 3] = np.inf
    hits, inst = g.trace_closest(ot, dt)
    ref = osc.trace_closest(ot, dt)
    same, bad = _compare_hits(hits, inst, ref)
    assert bad.sum() == 0, f"{bad.sum()} mismatches"
    assert same.mean() > 0.999
    assert g.stats()["num_instances"] == len(sc.objects)


def test_empty_and_degenerate_rays(ctx):
    sc = S.triangle_soup(1000, seed=1)
    g = agentray.Scene(ctx, sc)
    osc = O.OracleScene(sc)
    hits, inst = g.trace_closest(np.zeros((0, 4), np.float32), np.zeros((0, 4), np.float32))
    assert hits.shape == (0, 4)
    # axis-aligned directions (zero components) and a t-range that excludes all hits
    ot, dt = S.soup_rays(5000, seed=4)
    dt[:2500, :3] = np.eye(3, dtype=np.float32)[np.arange(2500) % 3] * np.where(np.arange(2500) % 2, 1, -1)[:, None]
    dt[4000:, 3] = 1e-5
    dt[3900:4000, :3] = 0.0  # zero directions: Ray::new gives NaN, which hits nothing
    assert (np.signbit(dt[:2500, :3]) & (dt[:2500, :3] == 0)).any()  # -0.0 components included
    hits, inst = g.trace_closest(ot, dt)
    ref = osc.trace_closest(ot, dt)
    same, bad = _compare_hits(hits, inst, ref)
    assert bad.sum() == 0, f"{bad.sum()} mismatches"
    assert same[:2500].mean() > 0.999
    assert np.all(hits[3900:, 3].view(np.uint32) == INVALID)
    assert np.all(ref["prim"][3900:4000] == INVALID)
    occ = g.trace_any(ot, dt)
    assert not occ[3900:4000].any()
    assert (occ == osc.trace_any(ot, dt)).mean() > 0.999


def _render_gpu(ctx, sc, cam, cfg, w, h):
    g = agentray.Scene(ctx, sc)
    out = np.empty(w * h * 3, np.float32)
    import ctypes as C
    agentray.check(agentray.lib().ar_render(ctx.handle, g.handle, C.byref(cam.desc()), C.byref(cfg), w, h,
                                            out.ctypes.data, 0))
    return out.reshape(h, w, 3).astype(np.float64)


@pytest.mark.parametrize("point_light", [False, True])
def test_pt_same_stream_matches_oracle(ctx, point_light):
    sc, cam = S.cornell_box(1, point_light=point_light)
    cfg = integrator_cfg(A.INTEGRATOR_PT, spp=16, max_depth=8, rr_depth=3, seed=5)
    w = h = 64
    gpu = _render_gpu(ctx, sc, cam, cfg, w, h)
    ref = O.OracleScene(sc).render(cam, cfg, w, h, sampler=O.SAMPLER_COUNTER)
    close = np.abs(gpu - ref) <= 1e-3 * np.maximum(1.0, np.abs(ref))
    assert close.all(axis=2).mean() >= 0.995, close.all(axis=2).mean()
    assert abs(gpu.mean() - ref.mean()) / ref.mean() < 1e-4


def welch_fail_fraction(a_reps, b_reps, thresh=4.5):
    """Per-pixel Welch t-test on replicate means (independent seeds).  Pixels
    with zero spread on both sides must agree to 1e-5 relative."""
    ma, mb = a_reps.mean(0), b_reps.mean(0)
    va, vb = a_reps.var(0, ddof=1), b_reps.var(0, ddof=1)
    k = a_reps.shape[0]
    se = np.sqrt(va / k + vb / k)
    zero = se == 0
    t = np.where(zero, 0.0, (ma - mb) / np.where(zero, 1.0, se))
    exact_bad = zero & (np.abs(ma - mb) > 1e-5 * np.maximum(1.0, np.abs(mb)))
    return float(((np.abs(t) > thresh) | exact_bad).mean())


def test_pt_statistically_equal_to_independent_oracle(ctx):
    # GPU and oracle on disjoint seeds: 8 replicates of 16 spp each.
    sc, cam = S.cornell_box(1)
    w = h = 48
    osc = O.OracleScene(sc)
    g = np.stack([_render_gpu(ctx, sc, cam, integrator_cfg(A.INTEGRATOR_PT, spp=16, seed=100 + k), w, h)
                  for k in range(8)])
    r = np.stack([osc.render(cam, integrator_cfg(A.INTEGRATOR_PT, spp=16, seed=200 + k), w, h,
                             sampler=O.SAMPLER_COUNTER) for k in range(8)])
    assert welch_fail_fraction(g, r) < 0.005
    # the reference's own sampler (xoshiro256++ per-pixel stream) agrees in distribution too
    x = np.stack([osc.render(cam, integrator_cfg(A.INTEGRATOR_PT, spp=16, seed=300 + k), w, h,
                             sampler=O.SAMPLER_XOSHIRO) for k in range(8)])
    assert welch_fail_fraction(g, x) < 0.005


def test_pt_film_f64_matches_f32(ctx):
    sc, cam = S.cornell_box(1)
    a = _render_gpu(ctx, sc, cam, integrator_cfg(A.INTEGRATOR_PT, spp=8, seed=3, film_precision=A.FILM_F32), 32, 32)
    b = _render_gpu(ctx, sc, cam, integrator_cfg(A.INTEGRATOR_PT, spp=8, seed=3, film_precision=A.FILM_F64), 32, 32)
    np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6)


def test_sor_bit_exact(ctx):
    rng = np.random.default_rng(1)
    h, w = 37, 53
    primal = rng.uniform(0.0, 2.0, (h, w, 3)).astype(np.float32)
    gx = (rng.normal(size=(h, w, 3)) * 0.2).astype(np.float32)
    gy = (rng.normal(size=(h, w, 3)) * 0.2).astype(np.float32)
    gx[:, -1] = 0
    gy[-1, :] = 0
    ref = O.poisson_sor_f32(primal, gx, gy, 0.2, 200, 1.6)
    out, _ = agentray.poisson_reconstruct(ctx, primal, gx, gy, 0.2, A.POISSON_SOR, 200, 1.6)
    np.testing.assert_array_equal(out, ref)


def test_cg_fp64_refined_reaches_tolerance(ctx):
    rng = np.random.default_rng(2)
    h, w = 96, 128
    primal = rng.uniform(0.0, 2.0, (h, w, 3)).astype(np.float32)
    gx = (rng.normal(size=(h, w, 3)) * 0.2).astype(np.float32)
    gy = (rng.normal(size=(h, w, 3)) * 0.2).astype(np.float32)
    gx[:, -1] = 0
    gy[-1, :] = 0
    exact, _ = O.poisson_exact_f64(primal, gx, gy, 0.2)
    out, res = agentray.poisson_reconstruct(ctx, primal, gx, gy, 0.2, A.POISSON_CG, 2000, 1.6, 1e-6)
    assert 0 <= res <= 1e-6
    np.testing.assert_allclose(out, np.maximum(exact, 0), atol=5e-5 * np.abs(exact).max())


def test_gdpt_same_stream_matches_oracle(ctx):
    sc, cam = S.cornell_box(1)
    cfg = integrator_cfg(A.INTEGRATOR_GDPT, spp=8, max_depth=6, seed=2)
    w, h = 48, 40
    gpu = _render_gpu(ctx, sc, cam, cfg, w, h)
    ref = O.OracleScene(sc).render(cam, cfg, w, h, sampler=O.SAMPLER_COUNTER)
    assert abs(gpu.mean() - ref.mean()) / ref.mean() < 1e-4
    close = np.abs(gpu - ref) <= 1e-3 * np.maximum(1.0, np.abs(ref))
    assert close.all(axis=2).mean() >= 0.995


@pytest.mark.parametrize("point_light", [True, False])
def test_bdpt_same_stream_matches_oracle(ctx, point_light):
    sc, cam = S.cornell_box(1, point_light=point_light)
    cfg = integrator_cfg(A.INTEGRATOR_BDPT, spp=8, max_depth=6, rr_depth=3, seed=4)
    w = h = 48
    gpu = _render_gpu(ctx, sc, cam, cfg, w, h)
    ref = O.OracleScene(sc).render(cam, cfg, w, h, sampler=O.SAMPLER_COUNTER)
    assert abs(gpu.mean() - ref.mean()) / ref.mean() < 1e-4
    close = np.abs(gpu - ref) <= 1e-3 * np.maximum(1.0, np.abs(ref))
    assert close.all(axis=2).mean() >= 0.995, close.all(axis=2).mean()


def test_bdpt_statistically_equal_to_independent_oracle(ctx):
    sc, cam = S.cornell_box(1)
    w = h = 32
    osc = O.OracleScene(sc)
    g = np.stack([_render_gpu(ctx, sc, cam, integrator_cfg(A.INTEGRATOR_BDPT, spp=16, max_depth=6, seed=400 + k),
                              w, h) for k in range(8)])
    r = np.stack([osc.render(cam, integrator_cfg(A.INTEGRATOR_BDPT, spp=16, max_depth=6, seed=500 + k), w, h,
                             sampler=O.SAMPLER_COUNTER) for k in range(8)])
    assert welch_fail_fraction(g, r) < 0.01


def test_pt_furnace_analytic(ctx):
    """Point light at the centre of a closed Lambertian sphere (albedo 0.5):
    one bounce gives albedo/pi * I/r^2, D bounces the geometric series."""
    import math
    sc, cam = S.furnace(albedo=0.5)
    one = _render_gpu(ctx, sc, cam, integrator_cfg(A.INTEGRATOR_PT, spp=2, max_depth=1, seed=1), 16, 16)
    assert np.allclose(one, 0.5 / math.pi, rtol=0.02)
    many = _render_gpu(ctx, sc, cam, integrator_cfg(A.INTEGRATOR_PT, spp=256, max_depth=4, rr_depth=10, seed=2),
                       16, 16)
    expect = 0.5 / math.pi * sum(0.5 ** k for k in range(4))
    assert abs(many.mean() - expect) / expect < 0.02


@pytest.mark.parametrize("tm,wp", [(A.TONEMAP_CLAMP, 1.0), (A.TONEMAP_REINHARD, 1.0),
                                   (A.TONEMAP_REINHARD_EXTENDED, 4.0)])
def test_film_to_rgb8_matches_oracle(ctx, tm, wp):
    # Bytes: equal except where CUDA's powf and the host's differ by an ulp on a
    # rounding boundary (at most 1 LSB, on < 0.1% of the values).
    sc, cam = S.cornell_box(1)
    film = agentray.PathTracer(agentray.PathTracerConfig(spp=4, seed=3)).render(agentray.Scene(ctx, sc), cam, 64, 48)
    hdr = film.rgb.copy()
    for scale in (1.0, 3.0):
        g = agentray.film_to_rgb8(ctx, hdr, tm, 2.2, scale, wp)
        r = O.film_to_rgb8(hdr, tm, wp, 2.2, scale)
        d = np.abs(g.astype(int) - r.astype(int))
        assert d.max() <= 1 and (d > 0).mean() < 1e-3, (d.max(), (d > 0).mean())
    import torch
    dev = agentray.film_to_rgb8(ctx, torch.from_numpy(hdr).cuda(), tm, 2.2, 1.0, wp)
    np.testing.assert_array_equal(dev.cpu().numpy(), agentray.film_to_rgb8(ctx, hdr, tm, 2.2, 1.0, wp))


# Same stream through glass: the sampling angles' sines and cosines come from
# one routine (ar_trig.h) on both sides, and every other operation on the path
# is an IEEE-rounded add, multiply, divide or square root, so refracted paths
# follow the same surfaces and the images agree like the opaque ones.  (The
# one remaining source of difference is a tie: two surfaces at the same t, as
# when a glass box stands on the floor; the scene lifts the box 2 mm.)
@pytest.mark.parametrize("kind,spp", [(A.INTEGRATOR_PT, 16), (A.INTEGRATOR_BDPT, 8)])
def test_dielectric_same_stream_matches_oracle(ctx, kind, spp):
    # DielectricBsdf (rough GGX glass): refraction, total internal reflection
    # and the reference's face-forwarded frame (wo.z > 0, so eta is always the
    # "entering" one), in PT and BDPT.
    sc, cam = S.cornell_box(1, glass=True)
    cfg = integrator_cfg(kind, spp=spp, max_depth=8, rr_depth=3, seed=6)
    w = h = 48
    gpu = _render_gpu(ctx, sc, cam, cfg, w, h)
    ref = O.OracleScene(sc).render(cam, cfg, w, h, sampler=O.SAMPLER_COUNTER)
    assert np.isfinite(gpu).all()
    assert abs(gpu.mean() - ref.mean()) / ref.mean() < 1e-4
    close = np.abs(gpu - ref) <= 1e-3 * np.maximum(1.0, np.abs(ref))
    assert close.all(axis=2).mean() >= 0.995, close.all(axis=2).mean()


# The config-3/4 room at its full size (195,452 triangles: icospheres and 500
# instanced boxes, Lambertian and GGX conductors 50/50, two quad lights) at a
# reduced resolution and spp: PT (depth 8), BDPT (path length 10) and GDPT.
@pytest.mark.parametrize("kind,depth", [(A.INTEGRATOR_PT, 8), (A.INTEGRATOR_BDPT, 10), (A.INTEGRATOR_GDPT, 8)])
def test_room_same_stream_matches_oracle(ctx, kind, depth):
    sc, cam = S.room(4)
    cfg = integrator_cfg(kind, spp=8, max_depth=depth, rr_depth=3, seed=21)
    w = h = 96
    gpu = _render_gpu(ctx, sc, cam, cfg, w, h)
    ref = O.OracleScene(sc).render(cam, cfg, w, h, sampler=O.SAMPLER_COUNTER)
    assert np.isfinite(gpu).all()
    assert abs(gpu.mean() - ref.mean()) / ref.mean() < 1e-4
    close = np.abs(gpu - ref) <= 1e-3 * np.maximum(1.0, np.abs(ref))
    assert close.all(axis=2).mean() >= 0.995, close.all(axis=2).mean()


@pytest.mark.parametrize("kind", [A.INTEGRATOR_PT, A.INTEGRATOR_BDPT])
def test_dielectric_statistically_equal_to_independent_oracle(ctx, kind):
    sc, cam = S.cornell_box(1, glass=True)
    w = h = 32
    osc = O.OracleScene(sc)
    g = np.stack([_render_gpu(ctx, sc, cam, integrator_cfg(kind, spp=16, max_depth=8, seed=700 + k), w, h)
                  for k in range(8)])
    r = np.stack([osc.render(cam, integrator_cfg(kind, spp=16, max_depth=8, seed=800 + k), w, h,
                             sampler=O.SAMPLER_COUNTER) for k in range(8)])
    assert welch_fail_fraction(g, r) < 0.01


@pytest.mark.parametrize("kind", [A.INTEGRATOR_PT, A.INTEGRATOR_BDPT])
def test_sample_range_shards_sum_to_full_render(ctx, kind):
    # Multi-GPU sharding on one GPU: disjoint sample ranges rendered apart
    # (ar_render_samples) sum to the one-call render (FP64 films).
    from agentray import distributed as D
    sc, cam = S.cornell_box(1)
    g = agentray.Scene(ctx, sc)
    cls, cfg_cls = ((agentray.PathTracer, agentray.PathTracerConfig) if kind == A.INTEGRATOR_PT else
                    (agentray.BidirectionalPathTracer, agentray.BdptConfig))
    integ = cls(cfg_cls(spp=10, max_depth=6, seed=12, film_precision=A.FILM_F64))
    w, h = 40, 32
    full = integ.render(g, cam, w, h).rgb.astype(np.float64)
    parts = [D.render_shard(integ, g, cam, w, h, *D.shard_range(10, r, 3), np.zeros(w * h * 3, np.float32))
             for r in range(3)]
    total = np.sum([p.astype(np.float64) for p in parts], axis=0).reshape(h, w, 3)
    np.testing.assert_allclose(total, full, rtol=1e-5, atol=1e-6)
    with pytest.raises(agentray.AgentRayError):
        D.render_shard(integ, g, cam, w, h, 5, 11, np.zeros(w * h * 3, np.float32))


@pytest.mark.parametrize("kind,spp", [(A.INTEGRATOR_PT, 16), (A.INTEGRATOR_BDPT, 8)])
def test_textured_same_stream_matches_oracle(ctx, kind, spp):
    # ImageTexture albedo (sRGB decode, bilinear, repeat wrap with uv outside
    # [0, 1) and negative) on the floor and back wall, in PT and in BDPT
    # (where light-subpath vertices carry their uv to the connections).
    sc, cam = S.cornell_box(1, textured=True)
    cfg = integrator_cfg(kind, spp=spp, max_depth=8, rr_depth=3, seed=7)
    w = h = 48
    gpu = _render_gpu(ctx, sc, cam, cfg, w, h)
    ref = O.OracleScene(sc).render(cam, cfg, w, h, sampler=O.SAMPLER_COUNTER)
    close = np.abs(gpu - ref) <= 1e-3 * np.maximum(1.0, np.abs(ref))
    assert close.all(axis=2).mean() >= 0.995, close.all(axis=2).mean()
    assert abs(gpu.mean() - ref.mean()) / ref.mean() < 1e-4
    plain = _render_gpu(ctx, S.cornell_box(1)[0], cam, cfg, w, h)
    assert np.abs(plain - gpu).mean() > 1e-3  # the textures do change the image


@pytest.mark.parametrize("kind,spp", [(A.INTEGRATOR_PT, 16), (A.INTEGRATOR_BDPT, 8)])
def test_imported_obj_scene_renders_like_oracle(ctx, tmp_path, kind, spp):
    # An OBJ/MTL scene through the importer: a textured floor (map_Kd PNG,
    # tiled uv), a conductor and a glass box, lit by a quad light.
    from agentray import importer as I
    agentray.write_png(str(tmp_path / "floor.png"), S.checker_texture(16, 4, seed=3))
    (tmp_path / "s.mtl").write_text("newmtl floor\nKd 0.5 0.5 0.5\nmap_Kd floor.png\n"
                                    "newmtl metal\nKs 0.8 0.7 0.5\nNs 400\n"
                                    "newmtl glass\nd 0.1\nNi 1.5\nNs 1000\n")
    obj = ["mtllib s.mtl", "v -2 0 -2", "v 2 0 -2", "v 2 0 2", "v -2 0 2",
           "vt 0 0", "vt 8 0", "vt 8 8", "vt 0 8", "o floor", "usemtl floor", "f 1/1 4/4 3/3 2/2"]
    nv = 4
    # the glass box floats 2 mm above the floor: standing on it, its bottom face
    # would share the floor's plane and a ray leaving the box downward would
    # hit both at the same t (a tie two traversal orders may break differently)
    for name, (cx, cz), y0 in (("metal", (-0.4, 0.0), 0.0), ("glass", (0.4, 0.1), 0.002)):
        c = np.array([[x, y, z] for x in (cx - 0.2, cx + 0.2) for y in (y0, 0.5) for z in (cz - 0.2, cz + 0.2)])
        obj += [f"o {name}", f"usemtl {name}"] + ["v %r %r %r" % tuple(float(x) for x in p) for p in c]
        for f in ((0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)):
            obj.append("f " + " ".join(str(nv + 1 + i) for i in f))
        nv += 8
    (tmp_path / "s.obj").write_text("\n".join(obj) + "\n")
    sc = agentray.scene_data.SceneData(A.LIGHT_DIST_POWER)
    I.load_obj_scene(sc, str(tmp_path / "s.obj"))
    S.add_quad_light(sc, (-0.3, 1.5, -0.3), (0.6, 0.0, 0.0), (0.0, 0.0, 0.6), (10.0, 10.0, 10.0))
    cam = agentray.scene_data.Camera((0.0, 1.0, 2.2), (0.0, 0.2, 0.0), (0.0, 1.0, 0.0), 45.0, 1.0)
    cfg = integrator_cfg(kind, spp=spp, max_depth=8, rr_depth=3, seed=9)
    gpu = _render_gpu(ctx, sc, cam, cfg, 40, 40)
    ref = O.OracleScene(sc).render(cam, cfg, 40, 40, sampler=O.SAMPLER_COUNTER)
    assert np.isfinite(gpu).all()
    assert abs(gpu.mean() - ref.mean()) / ref.mean() < 1e-4
    close = np.abs(gpu - ref) <= 1e-3 * np.maximum(1.0, np.abs(ref))
    assert close.all(axis=2).mean() >= 0.995, close.all(axis=2).mean()


@pytest.mark.parametrize("h,w", [(37, 29), (1, 1), (256, 200)])
def test_film_save_exr_matches_oracle_bytes(ctx, tmp_path, h, w):
    # ar_film_save_exr (device f16 conversion, channel split, ZIP reorder +
    # predictor; host deflate) writes the same file, byte for byte, as the
    # oracle's restatement of Film::save_exr, from host and device inputs.
    import torch
    rng = np.random.default_rng(h + w)
    hdr = rng.lognormal(-1.0, 2.0, (h, w, 3)).astype(np.float32)
    flat = hdr.reshape(-1)
    special = np.array([np.nan, 7e4, 3e-6, -2.5, 0.0, np.inf, 0, 0], np.float32)
    special.view(np.uint32)[6:8] = [0xFFC12345, 0x7F812345]  # NaN payloads, a signalling NaN
    k = min(flat.size, special.size)
    flat.view(np.uint32)[:k] = special.view(np.uint32)[:k]
    O.film_save_exr(hdr, str(tmp_path / "o.exr"), scale=0.75)
    agentray.film_save_exr(ctx, hdr, str(tmp_path / "g.exr"), scale=0.75)
    agentray.film_save_exr(ctx, torch.from_numpy(hdr).cuda(), str(tmp_path / "d.exr"), scale=0.75)
    want = (tmp_path / "o.exr").read_bytes()
    assert (tmp_path / "g.exr").read_bytes() == want
    assert (tmp_path / "d.exr").read_bytes() == want


def test_gdpt_textured_same_stream_matches_oracle(ctx):
    # GDPT's base/offset path roles shade textured surfaces through the same
    # kernels: primal and gradient films against the oracle's.
    sc, cam = S.cornell_box(1, textured=True)
    cfg = integrator_cfg(A.INTEGRATOR_GDPT, spp=8, max_depth=6, seed=11)
    w, h = 48, 40
    gpu = _render_gpu(ctx, sc, cam, cfg, w, h)
    ref = O.OracleScene(sc).render(cam, cfg, w, h, sampler=O.SAMPLER_COUNTER)
    assert np.isfinite(gpu).all()
    assert abs(gpu.mean() - ref.mean()) / ref.mean() < 1e-4
    close = np.abs(gpu - ref) <= 1e-3 * np.maximum(1.0, np.abs(ref))
    assert close.all(axis=2).mean() >= 0.995, close.all(axis=2).mean()


def test_trace_device_tensors_match_host_arrays(ctx):
    # Scene.trace_closest / trace_any take torch CUDA tensors (results stay on
    # the device) as well as host arrays; both give the same answers.
    import torch
    soup = S.triangle_soup(5000, seed=8)
    g = agentray.Scene(ctx, soup)
    ot, dt = S.soup_rays(4000, seed=9)
    h_hits, h_inst = g.trace_closest(ot, dt)
    d_hits, d_inst = g.trace_closest(torch.from_numpy(ot).cuda(), torch.from_numpy(dt).cuda())
    np.testing.assert_array_equal(d_hits.cpu().numpy().view(np.uint32), h_hits.view(np.uint32))
    np.testing.assert_array_equal(d_inst.cpu().numpy().view(np.uint32), h_inst.view(np.uint32))
    h_occ = g.trace_any(ot, dt)
    d_occ = g.trace_any(torch.from_numpy(ot).cuda().double(), torch.from_numpy(dt).cuda().double())
    np.testing.assert_array_equal(d_occ.cpu().numpy(), h_occ)


def test_host_array_batches_pipeline_in_chunks(ctx):
    # Host-array ray batches larger than one 4M-ray chunk go through the
    # library's copy/trace pipeline (two staging slots, copy streams): every
    # combination of host and device inputs and outputs gives the same hits,
    # for closest and any hit, on an odd-sized batch of three chunks.
    import ctypes as C
    import torch
    sc = S.triangle_soup(200_000, seed=4)
    g = agentray.Scene(ctx, sc)
    n = 9_000_001
    ot, dt = S.soup_rays(n, seed=5, tmax=0.3)
    ot_d, dt_d = torch.from_numpy(ot).cuda(), torch.from_numpy(dt).cuda()
    ref_h, ref_i = g.trace_closest(ot_d, dt_d)
    ref_h, ref_i = ref_h.cpu().numpy(), ref_i.cpu().numpy().view(np.uint32)
    pin_h = torch.empty((n, 4), dtype=torch.float32, pin_memory=True).numpy()
    pin_i = torch.empty(n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    hh, hi = g.trace_closest(ot, dt, out=(pin_h, pin_i))           # host in, host out (pinned)
    np.testing.assert_array_equal(hh.view(np.uint32), ref_h.view(np.uint32))
    np.testing.assert_array_equal(hi, ref_i)
    hh2, hi2 = g.trace_closest(ot, dt)                               # host in, host out (pageable)
    np.testing.assert_array_equal(hh2.view(np.uint32), ref_h.view(np.uint32))
    # host in, device out and device in, host out, through the C ABI
    lib = agentray.lib()
    bh = A.RayBatch(ot.ctypes.data, dt.ctypes.data, n, 0, 0)
    dh = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    di = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    agentray.check(lib.ar_trace_closest(ctx.handle, g.handle, C.byref(bh), dh.data_ptr(), di.data_ptr(), 1))
    agentray.check(lib.ar_context_synchronize(ctx.handle))
    np.testing.assert_array_equal(dh.cpu().numpy().view(np.uint32), ref_h.view(np.uint32))
    bd = A.RayBatch(ot_d.data_ptr(), dt_d.data_ptr(), n, 1, 0)
    oh = np.empty((n, 4), np.float32)
    oi = np.empty(n, np.uint32)
    agentray.check(lib.ar_trace_closest(ctx.handle, g.handle, C.byref(bd), oh.ctypes.data, oi.ctypes.data, 0))
    np.testing.assert_array_equal(oh.view(np.uint32), ref_h.view(np.uint32))
    np.testing.assert_array_equal(oi, ref_i)
    occ_ref = g.trace_any(ot_d, dt_d).cpu().numpy()
    np.testing.assert_array_equal(g.trace_any(ot, dt), occ_ref)
    assert 0.05 < occ_ref.mean() < 0.95
