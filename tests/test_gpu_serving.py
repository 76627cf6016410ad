"""GPU serving tests: continuous batching must not change any job's result.

Each job keys its sample stream by (seed, pixel, sample), so a job rendered
alone (ar_render) and the same job rendered by the server while other jobs of
other scenes/resolutions/integrators share its kernels must agree; with f64
films the only difference is the order of floating-point atomics
(tolerance: 1e-5 relative)."""
import numpy as np
import pytest

import agentray
import agentray.scenes as S
from agentray import _abi as A

pytestmark = pytest.mark.gpu


def _pt(spp, depth=8, seed=0, f64=True):
    return agentray.PathTracer(agentray.PathTracerConfig(spp=spp, max_depth=depth, rr_depth=3, seed=seed,
                                                         film_precision=A.FILM_F64 if f64 else A.FILM_F32))


def _bdpt(spp, depth=6, seed=0, f64=True):
    return agentray.BidirectionalPathTracer(agentray.BdptConfig(spp=spp, max_depth=depth, rr_depth=3, seed=seed,
                                                                film_precision=A.FILM_F64 if f64 else A.FILM_F32))


def _gdpt(spp, seed=0):
    return agentray.GradientDomainPathTracer(agentray.GdptConfig(spp=spp, max_depth=6, seed=seed,
                                                                 film_precision=A.FILM_F64))


def test_alone_equals_mixed(ctx):
    cb, cb_cam = S.cornell_box(1)
    s0, s0_cam = S.served_scene(0)
    scenes = {"cornell": agentray.Scene(ctx, cb), "served0": agentray.Scene(ctx, s0)}
    cams = {"cornell": cb_cam, "served0": s0_cam}
    jobs = [("cornell", _pt(16, seed=1), 64, 64), ("served0", _pt(4, seed=2), 96, 80),
            ("cornell", _bdpt(8, seed=3), 48, 48), ("served0", _bdpt(4, seed=4), 64, 64),
            ("cornell", _gdpt(8, seed=5), 64, 48)]
    alone = [integ.render(scenes[s], cams[s], w, h).rgb.copy() for s, integ, w, h in jobs]
    srv = agentray.Server(ctx, path_capacity=1 << 18, bdpt_batch_samples=1 << 14)
    ids = []
    # interleave the checked jobs with filler jobs of other sizes
    for k, (s, integ, w, h) in enumerate(jobs):
        ids.append(srv.submit(scenes[s], cams[s], integ, w, h))
        srv.submit(scenes["served0"], s0_cam, _pt(4, seed=100 + k, f64=False), 128, 128)
        srv.submit(scenes["cornell"], cb_cam, _bdpt(2, seed=200 + k, f64=False), 32, 32)
    for jid in ids:
        assert srv.wait(jid)["status"] == "done"
    for jid, ref in zip(ids, alone):
        out = srv.result(jid)
        np.testing.assert_allclose(out, ref, rtol=1e-5, atol=1e-6)
    st = srv.stats()
    srv.close()
    assert st["jobs_done"] >= len(jobs)
    assert st["pt_ticks"] > 0 and st["bdpt_batches"] > 0
    # the copy and launch counters: every image came back to host memory, and
    # each tick launches 5 kernels, each BDPT batch at least 10
    assert st["d2h_bytes"] >= sum(w * h * 12 for _, _, w, h in jobs)
    assert st["h2d_bytes"] > 0
    assert st["kernel_launches"] >= 5 * st["pt_ticks"] + 10 * st["bdpt_batches"]


def test_rejection_and_cancellation(ctx):
    cb, cam = S.cornell_box(1)
    scene = agentray.Scene(ctx, cb)
    # budget fits one 64x64 f32 job at a time, not a 1024x1024 one
    srv = agentray.Server(ctx, film_budget_bytes=4 << 20, path_capacity=1 << 16)
    big = srv.submit(scene, cam, _pt(1, f64=False), 1024, 1024)
    queued = [srv.submit(scene, cam, _pt(64, f64=False), 64, 64) for _ in range(6)]
    victim = queued[-1]
    try:
        srv.cancel(victim)
        cancelled = True
    except agentray.AgentRayError:
        cancelled = False  # the worker admitted it first
    assert srv.wait(big)["status"] == "rejected"
    for jid in queued[:-1]:
        info = srv.wait(jid)
        assert info["status"] == "done"
        assert info["admit_ms"] >= info["submit_ms"] and info["done_ms"] >= info["admit_ms"]
    if cancelled:
        assert srv.poll(victim)["status"] == "cancelled"
    st = srv.stats()
    srv.close()
    assert st["jobs_rejected"] == 1
    assert st["film_bytes_peak"] <= 4 << 20
    assert st["film_bytes_in_use"] == 0


def test_server_results_match_plain_path_f32(ctx):
    # Default f32 films: same images up to atomic ordering.
    s1, cam = S.served_scene(1)
    scene = agentray.Scene(ctx, s1)
    integ = _pt(8, seed=9, f64=False)
    ref = integ.render(scene, cam, 128, 128).rgb.copy()
    srv = agentray.Server(ctx)
    jid = srv.submit(scene, cam, integ, 128, 128)
    assert srv.wait(jid)["status"] == "done"
    out = srv.result(jid)
    srv.close()
    np.testing.assert_allclose(out, ref, rtol=1e-4, atol=1e-5)


def test_device_outputs_match_host_outputs(ctx):
    # Server.submit(out=<CUDA tensor>) keeps the image on the GPU; it is the
    # same image as the host-buffer path (f64 films: atomic order only).
    import torch
    cb, cam = S.cornell_box(1)
    scene = agentray.Scene(ctx, cb)
    srv = agentray.Server(ctx, path_capacity=1 << 18, bdpt_batch_samples=1 << 14)
    jobs = [(_pt(8, seed=31), 64, 48), (_bdpt(4, seed=32), 48, 40)]
    host = [srv.submit(scene, cam, integ, w, h) for integ, w, h in jobs]
    outs = [torch.full((w * h * 3,), float("nan"), dtype=torch.float32, device="cuda") for _, w, h in jobs]
    dev = [srv.submit(scene, cam, integ, w, h, out=o) for (integ, w, h), o in zip(jobs, outs)]
    for jid in host + dev:
        assert srv.wait(jid)["status"] == "done"
    for (integ, w, h), hj, dj in zip(jobs, host, dev):
        d = srv.result(dj).cpu().numpy().reshape(h, w, 3)
        assert np.isfinite(d).all()
        np.testing.assert_allclose(d, srv.result(hj), rtol=1e-5, atol=1e-6)
    srv.close()


def test_graph_replay_across_streams_and_depths(ctx):
    # The PT tick and each BDPT batch depth are CUDA graphs captured on the
    # context's stream: a render after the stream changes (graphs captured
    # again) and renders alternating batch depths give the images of a fresh
    # context (FP64 films: equal up to the order of the atomic adds).
    import torch
    sc, cam = S.cornell_box(1)
    ref_ctx = agentray.Context(0)
    jobs = [(_bdpt(4, seed=31), 48, 40), (_pt(4, seed=32), 40, 48)]
    deep = agentray.BidirectionalPathTracer(agentray.BdptConfig(spp=4, max_depth=3, rr_depth=2, seed=33,
                                                                film_precision=A.FILM_F64))
    want = [integ.render(agentray.Scene(ref_ctx, sc), cam, w, h).rgb.copy() for integ, w, h in jobs]
    want_deep = deep.render(agentray.Scene(ref_ctx, sc), cam, 32, 32).rgb.copy()
    ref_ctx.close()
    scene = agentray.Scene(ctx, sc)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    try:
        for st in (s1, s2, None):
            ctx.set_stream(st.cuda_stream if st is not None else None)
            for (integ, w, h), ref in zip(jobs, want):
                np.testing.assert_allclose(integ.render(scene, cam, w, h).rgb, ref, rtol=1e-6, atol=1e-7)
            np.testing.assert_allclose(deep.render(scene, cam, 32, 32).rgb, want_deep, rtol=1e-6, atol=1e-7)
    finally:
        ctx.set_stream(None)


@pytest.mark.parametrize("kind", ["pt", "bdpt"])
def test_split_order_shortest_first(ctx, kind):
    """Past the equal share, capacity goes to the waiting jobs shortest first
    (ties in arrival order): a medium job that does not fit in its share,
    queued behind three large jobs, finishes before the second and third of
    them, and the large ones finish one after another in arrival order."""
    cb, cam = S.cornell_box(1)
    scene = agentray.Scene(ctx, cb)
    if kind == "pt":
        # 2^16 path slots: each large job is 16 pool-fulls, the medium one 2
        srv = agentray.Server(ctx, path_capacity=1 << 16)
        large = [(_pt(16, seed=10 + k, f64=False), 256, 256) for k in range(3)]
        medium = (_pt(8, seed=20, f64=False), 128, 128)
    else:
        # 2^14-sample batches: each large job is 8 batches, the medium one 2
        srv = agentray.Server(ctx, path_capacity=1 << 16, bdpt_batch_samples=1 << 14)
        large = [(_bdpt(8, seed=10 + k, f64=False), 128, 128) for k in range(3)]
        medium = (_bdpt(8, seed=20, f64=False), 64, 64)
    ids = [srv.submit(scene, cam, integ, w, h) for integ, w, h in large]
    mid = srv.submit(scene, cam, *medium)
    done = [srv.wait(j)["done_ms"] for j in ids]
    m_done = srv.wait(mid)["done_ms"]
    srv.close()
    assert done[0] < done[1] < done[2]
    assert m_done < done[1]
