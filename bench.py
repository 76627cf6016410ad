"""Benchmark driver: one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workloads (seeded synthetic scenes with the stated shapes; no dataset exists):
  pt_cornell  (default) unidirectional PT, procedural Cornell box: 5 walls + 2
              rotated boxes = 34 triangles, 0.25 x 0.25 quad light of radiance
              15, albedos U[0.2,0.8], 256x256, 16 spp, max depth 8, RR from
              depth 3, f32 film.  One step = one full render (1,048,576 path
              samples).  Metric: Mpath-samples/s.
  bvh         BVH micro-benchmark: 1M triangles, 16M closest-hit rays
              (secondary line; metric Mrays/s).

Timing: W warm-up steps, then K steps, each bracketed by CUDA events on the
stream the library launches on (the context is bound to torch's current
stream); L2 is flushed (256 MiB write) before every timed step, outside its
events.  Multi-GPU: one process per GPU; each rank renders its own job
(seed = rank; weak scaling, no data-path collective); the time is the max over
ranks.  `e2e` times the public C-ABI path with host buffers: scene upload from
host arrays (Scene::new: BVH build + copies) + render + device->host readback.
`--impl reference` times the reference algorithm on the host cores (the C++
restatement of agent-ray's CPU integrator, the reference's own sampler).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "agent-ray_b200"), os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402

METRIC = "Mpath-samples/s at equal relMSE, batched vs plain GPU; served p50/p99 latency"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return PEAKS_FALLBACK, "fallback"


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_{device}_{os.getpid()}.csv")

    def __enter__(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def profile_traffic(name):
    """Per-launch DRAM bytes of `name` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"{name}.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


def reference_traversal_counts(scene_data, cam, w, h, n=65536, seed=7):
    """Mean AABB tests and triangle tests per ray of the reference binary SAH
    traversal (oracle counters) on this workload's primary rays and on rays
    with origins/directions uniform inside the scene bounds (bounce proxy)."""
    import oracle as O
    osc = O.OracleScene(scene_data)
    rng = np.random.default_rng(seed)
    # primary rays through random pixels
    from agentray.scene_data import Camera  # noqa: F401
    lf = np.array(cam.lookfrom, np.float64)
    la = np.array(cam.lookat, np.float64)
    up = np.array(cam.vup, np.float64)
    th = np.radians(cam.vfov_deg)
    vh = 2 * np.tan(th / 2)
    vw = cam.aspect * vh
    wv = (lf - la) / np.linalg.norm(lf - la)
    u = np.cross(up, wv)
    u /= np.linalg.norm(u)
    v = np.cross(wv, u)
    ll = lf - vw * u / 2 - vh * v / 2 - wv
    su, sv = rng.uniform(size=(n, 1)), rng.uniform(size=(n, 1))
    d = ll + su * vw * u + sv * vh * v - lf
    ot = np.zeros((2 * n, 4), np.float32)
    dt = np.zeros((2 * n, 4), np.float32)
    ot[:n, :3] = lf
    ot[:n, 3] = 1e-3
    dt[:n, :3] = d
    dt[:, 3] = np.inf
    allp = np.concatenate([m.positions for m in scene_data.meshes])
    lo, hi = allp.min(0), allp.max(0)
    ot[n:, :3] = rng.uniform(lo, hi, (n, 3))
    ot[n:, 3] = 1e-4
    dd = rng.normal(size=(n, 3))
    dt[n:, :3] = dd / np.linalg.norm(dd, axis=1, keepdims=True)
    r = osc.trace_closest(ot, dt, stats=True)
    return r["stats"]["nodes"] / (2 * n), r["stats"]["tris"] / (2 * n)


def run_reference(args, rank, world):
    """--impl reference: the reference CPU algorithm (oracle restatement,
    xoshiro256++ per-pixel streams like IndependentSampler) on all host cores."""
    if rank != 0:
        return
    import oracle as O
    import agentray.scenes as S
    from agentray import _abi as A
    from agentray.scene_data import integrator_cfg
    cores = os.cpu_count() or 1
    sc, cam = S.cornell_box(1)
    osc = O.OracleScene(sc)
    cfg = integrator_cfg(A.INTEGRATOR_PT, spp=16, max_depth=8, rr_depth=3)
    w = h = 256
    for _ in range(args.warmup):
        osc.render(cam, cfg, w, h, sampler=O.SAMPLER_XOSHIRO, threads=cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        osc.render(cam, cfg, w, h, sampler=O.SAMPLER_XOSHIRO, threads=cores)
        times.append(time.perf_counter() - t0)
    samples = w * h * cfg.spp
    value = samples * args.steps / sum(times) / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mpath-samples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene)",
            "config": {"workload": "pt_cornell: PT Cornell box 34 tris + quad light, 256x256, 16 spp, depth 8, RR 3",
                       "width": w, "height": h, "spp": 16},
            "cpu_baseline": {"value": value, "unit": "Mpath-samples/s", "cores": cores, "kind": "port",
                             "sample": "full workload per step (256x256x16 spp)"},
            "e2e": {"value": value, "unit": "Mpath-samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_pt(sc, cam, cfg):
    import oracle as O
    cores = os.cpu_count() or 1
    osc = O.OracleScene(sc)
    w = h = 256
    osc.render(cam, cfg, 32, 32, sampler=O.SAMPLER_XOSHIRO, threads=cores)
    t0 = time.perf_counter()
    reps = 0
    while True:
        osc.render(cam, cfg, w, h, sampler=O.SAMPLER_XOSHIRO, threads=cores)
        reps += 1
        if time.perf_counter() - t0 > 2.0 or reps >= 10:
            break
    dt = time.perf_counter() - t0
    return {"value": reps * w * h * cfg.spp / dt / 1e6, "unit": "Mpath-samples/s", "cores": cores, "kind": "port",
            "sample": f"{reps} full 256x256x16spp render(s) of the same scene, reference sampler, "
                      f"{dt:.2f} s wall on {cores} threads"}


def run_ours(args, rank, local, world):
    import torch
    import agentray
    import agentray.scenes as S
    from agentray import _abi as A
    from agentray.scene_data import integrator_cfg

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    peaks, peak_kind = load_peaks()
    ctx = agentray.Context(local)
    # A dedicated stream: the library launches on it, and every timing event is
    # recorded on it (torch's legacy default stream has handle 0, which the C ABI
    # reads as "use the context's own stream").
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if dist is not None:
            dist.barrier()

    if args.workload == "bvh":
        return run_bvh(args, rank, world, ctx, torch, flush, barrier, dist, peaks, peak_kind)

    sc, cam = S.cornell_box(1)
    W = H = 256
    spp = 16
    cfg = integrator_cfg(A.INTEGRATOR_PT, spp=spp, max_depth=8, rr_depth=3, seed=rank)
    scene = agentray.Scene(ctx, sc)
    out = torch.empty(W * H * 3, dtype=torch.float32, device="cuda")
    pt = agentray.PathTracer(agentray.PathTracerConfig(spp=spp, max_depth=8, rr_depth=3, seed=rank))
    for _ in range(max(3, args.warmup)):
        pt.render(scene, cam, W, H, out=out)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    step_ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            pt.render(scene, cam, W, H, out=out)
            e1.record(stream)
            step_ms.append((e0, e1))
        torch.cuda.synchronize()
    st = ctx.render_stats()
    # per render: `ticks` graph replays of (plan, generate, extend, shade, shadow)
    launches = args.steps * st["extend_launches"] * 5
    barrier()
    # Instrumented pass (same workload, same number of renders): the stages are
    # launched individually with CUDA events on the library stream.
    ctx.profile(True)
    ctx.profile_reset()
    for _ in range(args.steps):
        flush.zero_()
        pt.render(scene, cam, W, H, out=out)
    torch.cuda.synchronize()
    ctx.profile(False)
    prof = ctx.profile_read()
    total_ms = sum(a.elapsed_time(b) for a, b in step_ms)
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    stats = ctx.render_stats()
    samples = W * H * spp
    value = world * samples * args.steps / (total_ms / 1e3) / 1e6

    # end to end through the public API with host buffers
    e2e_ms = []
    host_out = np.empty(W * H * 3, np.float32)
    h2d = 0
    for i in range(2 + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s2 = agentray.Scene(ctx, sc)
        pt.render(s2, cam, W, H, out=host_out)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) * 1e3
        h2d = s2.stats()["device_bytes"]
        s2.close()
        if i >= 2:
            e2e_ms.append(dt)
    e2e_value = samples / (statistics.mean(e2e_ms) / 1e3) / 1e6

    line = None
    if rank == 0:
        nodes, tris = reference_traversal_counts(sc, cam, W, H)
        b_ray = 32 + 16 + 32 * nodes + 36 * tris
        ln, ms = prof.get("pt_extend", (0, 0.0))
        rays_per_launch = stats["extend_rays"] / max(1, stats["extend_launches"])
        avg_s = (ms / max(1, ln)) / 1e3
        achieved = rays_per_launch * b_ray / avg_s / 1e9 if avg_s > 0 else 0.0
        traffic = profile_traffic("pt_extend_cornell")
        line = {
            "metric": METRIC, "value": value, "unit": "Mpath-samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": "pt_cornell: PT Cornell box 34 tris + quad light, 256x256, 16 spp, depth 8, RR 3",
                       "width": W, "height": H, "spp": spp, "max_depth": 8, "rr_depth": 3,
                       "l2": "flushed (256 MiB write) before each timed step", "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "Mpath-samples/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": W * H * 3 * 4,
                    "includes": "Scene::new (host BVH build + upload) + render + readback"},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": "pt_extend", "achieved": achieved, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                         "peak_kind": peak_kind,
                         "bytes_model": f"rays/launch {rays_per_launch:.0f} x (48 + 32*{nodes:.2f} nodes + "
                                        f"36*{tris:.2f} tris) B; reference-traversal counts"},
            "kernels_ms": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()},
            "render_stats": stats,
        }
    clocks = clk.summary()
    if rank == 0:
        line["clocks"] = clocks
        line["cpu_baseline"] = cpu_baseline_pt(sc, cam, integrator_cfg(A.INTEGRATOR_PT, spp=16, max_depth=8,
                                                                       rr_depth=3))
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_bvh(args, rank, world, ctx, torch, flush, barrier, dist, peaks, peak_kind):
    import agentray
    import agentray.scenes as S
    n_tris, n_rays = 1_000_000, 16_000_000
    sc = S.triangle_soup(n_tris, seed=2)
    scene = agentray.Scene(ctx, sc)
    ot, dt = S.soup_rays(n_rays, seed=3)
    ot_d = torch.from_numpy(ot).cuda()
    dt_d = torch.from_numpy(dt).cuda()
    stream = torch.cuda.current_stream()
    assert stream.cuda_stream != 0
    for _ in range(max(3, args.warmup)):
        scene.trace_closest(ot_d, dt_d)
    torch.cuda.synchronize()
    ctx.profile(True)
    ctx.profile_reset()
    barrier()
    ev = []
    with ClockSampler(torch.cuda.current_device()) as clk:
        for _ in range(args.steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            scene.trace_closest(ot_d, dt_d)
            b.record(stream)
            ev.append((a, b))
        torch.cuda.synchronize()
    ctx.profile(False)
    prof = ctx.profile_read()
    total_ms = sum(a.elapsed_time(b) for a, b in ev)
    value = world * n_rays * args.steps / (total_ms / 1e3) / 1e6
    if rank == 0:
        import oracle as O
        osc = O.OracleScene(sc)
        r = osc.trace_closest(ot[:200_000], dt[:200_000], stats=True)
        nodes = r["stats"]["nodes"] / 200_000
        tris = r["stats"]["tris"] / 200_000
        b_ray = 32 + 16 + 32 * nodes + 36 * tris
        ln, ms = prof.get("trace_closest", (1, total_ms))
        achieved = n_rays * b_ray / ((ms / ln) / 1e3) / 1e9
        t0 = time.perf_counter()
        osc.trace_closest(ot[:2_000_000], dt[:2_000_000])
        cpu = 2_000_000 / (time.perf_counter() - t0) / 1e6
        line = {"metric": "Mrays/s (closest hit)", "value": value, "unit": "Mrays/s", "n_gpus": world,
                "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": {"workload": "bvh: 1M tris, 16M rays closest hit", "l2": "flushed"},
                "gpu_launches": args.steps,
                "roofline": {"bound": "hbm", "kernel": "trace_closest", "achieved": achieved, "peak": peaks["hbm_gbs"],
                             "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                             "traffic": profile_traffic("trace_closest_soup"), "peak_kind": peak_kind,
                             "bytes_model": f"48 + 32*{nodes:.1f} + 36*{tris:.1f} B/ray"},
                "clocks": clk.summary(),
                "cpu_baseline": {"value": cpu, "unit": "Mrays/s", "cores": os.cpu_count(), "kind": "port",
                                 "sample": "2M of the 16M rays, reference binary SAH traversal"}}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pt_cornell", choices=["pt_cornell", "bvh"])
    args = ap.parse_args()
    rank, local, world = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    run_ours(args, rank, local, world)


if __name__ == "__main__":
    main()
