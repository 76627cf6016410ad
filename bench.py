"""Benchmark driver: one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload served|pt_cornell|pt_cornell_glass|pt_cornell_textured|pt_served4|
                                bdpt_served4|bdpt_room|gdpt_room|bvh]
                    [--timed-jobs T] [--config-steps C] [--no-configs]

Workloads (seeded synthetic inputs with the stated shapes; no dataset exists):
  served      (default) the served batched-rendering stream (config 5): a
              seeded stream of 2000 jobs over 8 procedural scenes of
              10k-1M triangles, resolution from {128,256,512,1024}^2, spp
              from {4,16,64}, PT or BDPT 70/30 (depth 8, RR from 3,
              power-heuristic MIS).  Metric: Mpath-samples/s.  The timed
              set is fixed: jobs [0, T) of the stream (T = 400), whatever K
              is; a step is 1/K of it, and the K steps are submitted back to
              back as one backlog (continuous batching).  `value` keeps the
              images on the GPU, `e2e` renders the same jobs into pinned host
              buffers, `served` replays the same jobs as Poisson arrivals at
              80% of the capacity `value` measured (p50/p99 overall and per
              class), and `plain` renders them one at a time through
              ar_render (the reference's Integrator::render unit), with the
              batched-vs-plain speed-up per job class.  The line carries a
              `configs` object with configs 1-4 measured in the same process
              (pt_cornell, bvh, bdpt_room, gdpt_room; C timed steps each).
  pt_cornell  PT Cornell box (34 tris + quad light, 256x256, 16 spp, depth 8);
              one step = one full render.
  pt_cornell_glass  config 1 with rough-glass (DielectricBsdf) objects.
  pt_cornell_textured  config 1 with checker ImageTextures on the floor and
              back wall (bilinear, repeat-wrapped uv).
  pt_served4  PT on served scene 4 (139k tris, 335 instances), 512x512, 16 spp.
  bdpt_served4 BDPT on served scene 4, 512x512, 16 spp, depth 8.
  bdpt_room   BDPT on the 200k-tri room, 512x512, 64 spp, depth 10, FP64 film.
  gdpt_room   GDPT on the room, 1024x1024, 32 spp, CG Poisson to 1e-6.
  bvh         BVH micro-benchmark: 1M triangles, 16M closest-hit rays (Mrays/s),
              any hit with t_max 0.25 beside it.

Timing: CUDA events on the stream the library launches on (single renders,
bvh) or, for the server (which runs on its own internal streams), events
recorded on an idle stream around the timed set (submission -> last result),
i.e. device timestamps of its wall span.  L2 is flushed (256 MiB write)
before every timed step outside its events.  Multi-GPU: one process per GPU,
each rank serves its own seeded stream (weak scaling, no data-path
collective); time is the max over ranks.  `--impl reference` times the
reference algorithm (the C++ restatement of agent-ray's CPU integrators with
the reference's xoshiro sampler) on all host cores on a bounded sample of the
same timed set.
"""
import argparse
import json
import os
import statistics
import subprocess
import tempfile
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "agent-ray_b200"), os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402

METRIC = "Mpath-samples/s at equal relMSE, batched vs plain GPU; served p50/p99 latency"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0}
SERVED_DESC = ("served: Poisson stream of 2000 jobs over 8 procedural scenes (10k-1M tris), res {128..1024}^2, "
               "spp {4,16,64}, PT/BDPT 70/30, depth 8")


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return PEAKS_FALLBACK, "fallback"


def max_over_ranks(dist, value, device):
    """The job's time: the largest per-rank device time (every rank calls this
    at the same point; `dist` is None on one process)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_stream(n_jobs, rank):
    """Each rank serves its own seeded job stream (weak scaling)."""
    import agentray.scenes as S
    return S.served_stream(n_jobs, seed=5 + 1000 * rank)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        # raw samples go to $AR_CLOCK_LOG_DIR (default: the system temp dir);
        # the JSON line carries their summary
        log_dir = os.environ.get("AR_CLOCK_LOG_DIR") or tempfile.gettempdir()
        self.path = os.path.join(log_dir, f"clocks_{device}_{os.getpid()}.csv")

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

    def fill(self, fn, t_start, min_s=0.5):
        """For timed regions shorter than a few sampling periods (100 ms, after
        nvidia-smi's own start-up): keeps the GPU on the same work, untimed,
        until min_s after the region started, so that the readings are taken
        under this load.  Returns True when it ran anything."""
        if not self.proc or time.perf_counter() - t_start >= min_s:
            return False
        while time.perf_counter() - t_start < min_s:
            fn()
        return True

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_median": statistics.median(power) if power else None}


def profile_value(name, key):
    """A `key: value` line of the committed ncu summary profiles/<name>.txt."""
    p = os.path.join(ROOT, "profiles", f"{name}.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(key + ":"):
            return float(line.split(":")[1].split()[0])
    return None


def profile_traffic(name, rays_per_launch=None):
    """DRAM bytes (read + write) per launch of the kernel `name` profiles:
    the summary's per-ray figure times this launch's rays when both are
    known, else its per-launch figure."""
    per_ray = profile_value(name, "dram_bytes_per_ray")
    if per_ray is not None and rays_per_launch:
        return per_ray * rays_per_launch
    return profile_value(name, "dram_bytes_per_launch")


def camera_rays(cam, n, rng):
    lf = np.array(cam.lookfrom, np.float64)
    la = np.array(cam.lookat, np.float64)
    up = np.array(cam.vup, np.float64)
    vh = 2 * np.tan(np.radians(cam.vfov_deg) / 2)
    vw = cam.aspect * vh
    wv = (lf - la) / np.linalg.norm(lf - la)
    u = np.cross(up, wv)
    u /= np.linalg.norm(u)
    v = np.cross(wv, u)
    ll = lf - vw * u / 2 - vh * v / 2 - wv
    su, sv = rng.uniform(size=(n, 1)), rng.uniform(size=(n, 1))
    return np.broadcast_to(lf, (n, 3)), ll + su * vw * u + sv * vh * v - lf


def reference_traversal_counts(scene_data, cam, n=32768, seed=7):
    """Mean AABB tests and triangle tests per ray of the reference binary SAH
    traversal (oracle counters) on primary rays and on rays uniform inside the
    scene bounds (a proxy for bounce rays)."""
    import oracle as O
    osc = O.OracleScene(scene_data)
    rng = np.random.default_rng(seed)
    o, d = camera_rays(cam, n, rng)
    ot = np.zeros((2 * n, 4), np.float32)
    dt = np.zeros((2 * n, 4), np.float32)
    ot[:n, :3] = o
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
    osc.close()
    return r["stats"]["nodes"] / (2 * n), r["stats"]["tris"] / (2 * n)


def make_integrator(agentray, job, seed):
    if job["integrator"] == "bdpt":
        return agentray.BidirectionalPathTracer(agentray.BdptConfig(spp=job["spp"], max_depth=8, rr_depth=3,
                                                                    seed=seed))
    return agentray.PathTracer(agentray.PathTracerConfig(spp=job["spp"], max_depth=8, rr_depth=3, seed=seed))


def job_cfg(job, seed):
    from agentray import _abi as A
    from agentray.scene_data import integrator_cfg
    kind = A.INTEGRATOR_BDPT if job["integrator"] == "bdpt" else A.INTEGRATOR_PT
    return integrator_cfg(kind, spp=job["spp"], max_depth=8, rr_depth=3, seed=seed)


# ----------------------------------------------------------------- served ----
def wait_or_dump(srv, job_id, timeout_ms=300_000.0):
    """Waits for a job; on timeout prints the server's queue state and raises."""
    try:
        return srv.wait(job_id, timeout_ms)
    except Exception:
        print("job", job_id, srv.poll(job_id), "\nserver state:\n" + srv.debug_dump(), "\nstats:", srv.stats(),
              file=sys.stderr, flush=True)
        raise


def job_class(job):
    return f"{job['integrator']}_{job['res']}x{job['spp']}"


def samples_of(jobs):
    return sum(j["res"] ** 2 * j["spp"] for j in jobs)


# Jobs whose samples cannot fill the 2^22 path slots (PT) or one 2^21-sample
# BDPT batch by themselves: the classes where batching several jobs can help.
SMALL_CLASSES = [(128, 4), (128, 16), (128, 64), (256, 4), (256, 16), (512, 4)]


def run_served(args, rank, local, world, torch, ctx, barrier, dist, peaks, peak_kind, stream):
    """The served stream (config 5) on a fixed job set: jobs [0, timed_jobs) of
    the seeded 2000-job stream, the same set whatever --steps is.

    value   the set submitted as a backlog (K steps = K consecutive slices of
            the set, submitted back to back) with images kept on the GPU;
    e2e     the same jobs with images returned to pinned host buffers;
    served  the same jobs (new seeds) arriving as a Poisson process at 80% of
            the capacity `value` measured on this job mix: p50/p99 latency
            overall and per resolution x integrator class;
    plain   the same jobs one at a time through ar_render (the reference's
            Integrator::render unit), and per job class the small-job speed-up
            of batching (each class's jobs as one backlog vs one at a time)."""
    import agentray
    import agentray.scenes as S

    full = rank_stream(args.jobs, rank)
    T = min(args.timed_jobs, len(full))
    timed = full[:T]
    K = max(1, args.steps)
    W = max(3, args.warmup)
    chunks = [list(c) for c in np.array_split(np.arange(T), K)]
    warm_jobs = full[T:T + W * args.window_jobs]
    built = [S.served_scene(k) for k in range(8)]
    scenes = [agentray.Scene(ctx, sd) for sd, _ in built]
    cams = [cam for _, cam in built]
    srv = agentray.Server(ctx, film_budget_bytes=24 << 30, path_capacity=args.path_capacity,
                          bdpt_batch_samples=args.bdpt_batch, bdpt_max_depth=8)
    side = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    dev_out = [torch.empty(j["res"] ** 2 * 3, dtype=torch.float32, device="cuda") for j in timed]
    host_out = [torch.empty(j["res"] ** 2 * 3, dtype=torch.float32, pin_memory=True).numpy() for j in timed]

    def submit(job, seed, out):
        return srv.submit(scenes[job["scene"]], cams[job["scene"]], make_integrator(agentray, job, seed),
                          job["res"], job["res"], out=out)

    def run_backlog(idx, outs, base_seed, arrivals=None):
        """Submits timed[i] for i in idx (all at once, or at `arrivals` seconds
        after the start), waits for all; returns (device-span ms, wall s,
        infos, server-stats delta)."""
        flush.zero_()
        torch.cuda.synchronize()
        st0 = srv.stats()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(side)
        t0 = time.perf_counter()
        ids = []
        for n, i in enumerate(idx):
            if arrivals is not None:
                delay = arrivals[n] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
            ids.append(submit(timed[i], base_seed + i, outs[i] if outs is not None else None))
        infos = [wait_or_dump(srv, x) for x in ids]
        e1.record(side)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        st1 = srv.stats()
        for x in ids:
            srv.forget(x)
        assert all(i["status"] == "done" for i in infos), [i["status"] for i in infos]
        return e0.elapsed_time(e1), wall, infos, {k: st1[k] - st0[k] for k in st1}

    # warm-up: the first step submits the timed set at 1 spp as one backlog, so
    # the server's film pool holds buffers for every job of the set before the
    # timed passes; the others run window_jobs jobs from beyond the timed set.
    # Then the plain path once per integrator.
    ids = [srv.submit(scenes[j["scene"]], cams[j["scene"]], make_integrator(agentray, dict(j, spp=1), 800 + i),
                      j["res"], j["res"], out=dev_out[i]) for i, j in enumerate(timed)]
    for x in ids:
        wait_or_dump(srv, x)
        srv.forget(x)
    for w in range(1, W):
        ids = [srv.submit(scenes[j["scene"]], cams[j["scene"]], make_integrator(agentray, j, 900 + w * 100 + i),
                          j["res"], j["res"]) for i, j in enumerate(warm_jobs[w * args.window_jobs:
                                                                          (w + 1) * args.window_jobs])]
        for x in ids:
            wait_or_dump(srv, x)
            srv.forget(x)
    for j in (dict(timed[0], res=128, spp=4, integrator="pt"), dict(timed[0], res=128, spp=4, integrator="bdpt")):
        make_integrator(agentray, j, 1).render(scenes[j["scene"]], cams[j["scene"]], 128, 128,
                                               out=dev_out[0][:128 * 128 * 3])
    torch.cuda.synchronize()

    # value: the whole set as a backlog, images on the device
    barrier()
    all_idx = [i for c in chunks for i in c]
    with ClockSampler(local) as clk:
        value_ms, _, _, vstats = run_backlog(all_idx, dev_out, 10_000)
    total_samples = samples_of(timed)
    value = world * total_samples / (max_over_ranks(dist, value_ms, "cuda") / 1e3) / 1e6
    capacity_sps = total_samples / (value_ms / 1e3)

    # e2e: the same jobs and seeds, images into pinned host buffers
    e2e_ms, e2e_wall, _, estats = run_backlog(all_idx, host_out, 10_000)
    e2e_value = world * total_samples / (max_over_ranks(dist, e2e_ms, "cuda") / 1e3) / 1e6

    # served: Poisson arrivals of the same jobs at 80% of this mix's capacity
    rate = 0.8 * capacity_sps / (total_samples / T)
    arrivals = np.cumsum(np.random.default_rng(77 + rank).exponential(1.0 / rate, T))
    _, served_wall, infos, _ = run_backlog(list(range(T)), host_out, 50_000, arrivals=arrivals)
    lat = np.array([i["done_ms"] - i["submit_ms"] for i in infos])
    by_class = {}
    for job, l in zip(timed, lat):
        by_class.setdefault(f"{job['integrator']}_{job['res']}", []).append(l)
    served = {"jobs": T, "arrival_rate_jobs_per_s": rate, "load": 0.8,
              "load_basis": "80% of `value`'s measured capacity on this same job set",
              "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
              "mean_ms": float(lat.mean()), "max_ms": float(lat.max()),
              "span_s": served_wall,
              "throughput_mpath_samples_per_s": total_samples / served_wall / 1e6,
              "by_class": {k: {"jobs": len(v), "p50_ms": float(np.percentile(v, 50)),
                               "p99_ms": float(np.percentile(v, 99))} for k, v in sorted(by_class.items())}}
    relmse = served_relmse(agentray, srv, scenes, cams, full)

    # per-class batching of the small jobs: each class's jobs as one backlog
    batched_class = {}
    for integ in ("pt", "bdpt"):
        for res, spp in SMALL_CLASSES:
            idx = [i for i, j in enumerate(timed) if (j["integrator"], j["res"], j["spp"]) == (integ, res, spp)]
            if not idx:
                continue
            ms, _, _, _ = run_backlog(idx, dev_out, 10_000)
            batched_class[f"{integ}_{res}x{spp}"] = (len(idx), samples_of([timed[i] for i in idx]), ms)
    srv_stats = srv.stats()
    srv.close()

    # plain: one job at a time through ar_render, the same jobs and seeds
    flush.zero_()
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(T + 1)]
    evs[0].record(stream)
    for i, job in enumerate(timed):
        make_integrator(agentray, job, 10_000 + i).render(scenes[job["scene"]], cams[job["scene"]], job["res"],
                                                          job["res"], out=dev_out[i])
        evs[i + 1].record(stream)
    torch.cuda.synchronize()
    plain_ms = evs[0].elapsed_time(evs[T])
    job_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(T)]
    plain_value = total_samples / (plain_ms / 1e3) / 1e6
    per_class = {}
    for i, job in enumerate(timed):
        c = per_class.setdefault(job_class(job), {"jobs": 0, "samples": 0, "plain_ms": 0.0})
        c["jobs"] += 1
        c["samples"] += job["res"] ** 2 * job["spp"]
        c["plain_ms"] += job_ms[i]
    small_plain_ms = 0.0
    for name, c in per_class.items():
        c["plain_mpath_samples_per_s"] = c["samples"] / (c["plain_ms"] / 1e3) / 1e6
        c["plain_time_share"] = c["plain_ms"] / plain_ms
        if name in batched_class:
            n, smp, ms = batched_class[name]
            c["batched_mpath_samples_per_s"] = smp / (ms / 1e3) / 1e6
            c["speedup_batched_vs_plain"] = c["batched_mpath_samples_per_s"] / c["plain_mpath_samples_per_s"]
            small_plain_ms += c["plain_ms"]
    small_share = small_plain_ms / plain_ms
    plain = {"value": plain_value, "unit": "Mpath-samples/s", "jobs": T,
             "speedup_batched_vs_plain": value / world / plain_value,
             "small_job_plain_time_share": small_share,
             "bound_if_small_jobs_were_free": 1.0 / max(1e-9, 1.0 - small_share),
             "small_classes": "jobs of < 2^22 samples: " + ", ".join(f"{r}^2x{s}" for r, s in SMALL_CLASSES),
             "equal_relmse": "same per-job sample keys: images equal up to atomic-add order "
                             "(tests/test_gpu_serving.py); relmse below",
             "per_class": dict(sorted(per_class.items()))}

    if rank != 0:
        return None
    mix_full = {}
    for j in full:
        mix_full[j["integrator"]] = mix_full.get(j["integrator"], 0) + j["res"] ** 2 * j["spp"]
    mix_t = {}
    for j in timed:
        mix_t[j["integrator"]] = mix_t.get(j["integrator"], 0) + j["res"] ** 2 * j["spp"]
    line = {
        "metric": METRIC, "value": value, "unit": "Mpath-samples/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": value_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded procedural scenes and job stream)",
        "config": {"workload": SERVED_DESC,
                   "timed_set": f"jobs [0, {T}) of the seeded {len(full)}-job stream (fixed, independent of --steps)",
                   "timed_samples": total_samples,
                   "bdpt_sample_share": {"timed_set": mix_t.get("bdpt", 0) / total_samples,
                                         "full_stream": mix_full.get("bdpt", 0) / samples_of(full)},
                   "step": f"1/{K} of the timed set, submitted back to back (one backlog)",
                   "warmup": f"{W} steps: the timed set at 1 spp as one backlog, then {W - 1} x {args.window_jobs} "
                             f"jobs from beyond the timed set",
                   "l2": "flushed (256 MiB write) before the timed set",
                   "parallelism": f"replicas x{world}",
                   "server": {"path_capacity": args.path_capacity, "bdpt_batch_samples": args.bdpt_batch}},
        "e2e": {"value": e2e_value, "unit": "Mpath-samples/s", "h2d_bytes_per_step": estats["h2d_bytes"] / K,
                "d2h_bytes_per_step": estats["d2h_bytes"] / K,
                "note": "the same jobs and seeds as `value`: per step the job descriptors (job-table entries, "
                        "BDPT batch descriptors) go host->device, completion snapshots and every image "
                        "device->host into pinned buffers; scenes resident"},
        "plain": plain,
        "served": served,
        "relmse": relmse,
        "server_stats": srv_stats,
        "gpu_launches": int(vstats["kernel_launches"]),
        "clocks": clk.summary(),
    }
    line["roofline"] = served_roofline(args, ctx, agentray, S, scenes, cams, built, peaks, peak_kind, torch,
                                       line["clocks"])
    line["cpu_baseline"] = cpu_baseline_served(timed, built, n_samples_target=args.cpu_samples)
    return line


def served_relmse(agentray, srv, scenes, cams, stream):
    """relMSE (mean of (x - ref)^2 / (ref^2 + 1e-2)) of a PT and a BDPT job,
    rendered by the server inside a mix of stream jobs and by the plain path,
    against an FP64-film 2048-spp render of the same scene (tests pin the GPU's
    relMSE to the FP64 CPU oracle's).  Scene 0, 128x128, 16 spp, depth 8."""
    from agentray import _abi as A
    k, r, spp = 0, 128, 16

    def rel(x, ref):
        return float(np.mean((x.astype(np.float64) - ref) ** 2 / (ref ** 2 + 1e-2)))

    out = {}
    mix = [j for j in stream[:64] if j["res"] <= 512][:6]
    for name, cls, cfg_cls in (("pt", agentray.PathTracer, agentray.PathTracerConfig),
                               ("bdpt", agentray.BidirectionalPathTracer, agentray.BdptConfig)):
        ref_img = np.empty(r * r * 3, np.float32)
        cls(cfg_cls(spp=2048, max_depth=8, rr_depth=3, seed=99, film_precision=A.FILM_F64)).render(
            scenes[k], cams[k], r, r, out=ref_img)
        ref = ref_img.astype(np.float64)
        job = cls(cfg_cls(spp=spp, max_depth=8, rr_depth=3, seed=123))
        ids = [srv.submit(scenes[j["scene"]], cams[j["scene"]], make_integrator(agentray, j, 777 + i), j["res"],
                          j["res"]) for i, j in enumerate(mix[:3])]
        jid = srv.submit(scenes[k], cams[k], job, r, r)
        ids += [srv.submit(scenes[j["scene"]], cams[j["scene"]], make_integrator(agentray, j, 888 + i), j["res"],
                           j["res"]) for i, j in enumerate(mix[3:])]
        for i in ids + [jid]:
            wait_or_dump(srv, i)
        served_img = srv.result(jid).reshape(-1).copy()
        for i in ids + [jid]:
            srv.forget(i)
        plain_img = np.empty(r * r * 3, np.float32)
        job.render(scenes[k], cams[k], r, r, out=plain_img)
        out[name] = {"served_in_mix": rel(served_img, ref), "plain": rel(plain_img, ref)}
    out["case"] = (f"served scene {k}, {r}x{r}, {spp} spp, depth 8; served inside a mix of {len(mix)} stream jobs; "
                   f"reference: FP64-film 2048 spp")
    return out


def issue_ceiling(name, rays_per_s, clocks):
    """Second ceiling for a traversal kernel: warp instructions issued per
    second (rays/s x warp instructions per ray, from the kernel's ncu summary)
    against the SMs' issue rate (148 SMs x 4 schedulers x 1 warp instruction
    per cycle at the sampled SM clock)."""
    inst = profile_value(name, "warp_inst_per_ray")
    mhz = (clocks or {}).get("sm_mhz") or 1965.0
    peak = 148 * 4 * mhz * 1e6 / 1e9
    if inst is None:
        return {"source": f"profiles/{name}.txt has no warp_inst_per_ray line", "peak_ginst_s": peak}
    achieved = rays_per_s * inst / 1e9
    return {"bound": "issue", "warp_inst_per_ray": inst, "achieved_ginst_s": achieved, "peak_ginst_s": peak,
            "frac": achieved / peak, "sm_mhz": mhz, "source": f"profiles/{name}.txt (ncu smsp__inst_executed)"}


def served_roofline(args, ctx, agentray, S, scenes, cams, built, peaks, peak_kind, torch, clocks):
    """Per-launch timing of the dominant kernel (pt_extend) on the middle
    scene (k=4, 139k tris) at 512x512 x 16 spp, with the reference-traversal
    bytes model and the issue-rate ceiling."""
    k = 4
    pt = agentray.PathTracer(agentray.PathTracerConfig(spp=16, max_depth=8, rr_depth=3, seed=3))
    out = torch.empty(512 * 512 * 3, dtype=torch.float32, device="cuda")
    pt.render(scenes[k], cams[k], 512, 512, out=out)
    ctx.profile(True)
    ctx.profile_reset()
    for _ in range(2):
        pt.render(scenes[k], cams[k], 512, 512, out=out)
    torch.cuda.synchronize()
    ctx.profile(False)
    prof = ctx.profile_read()
    stats = ctx.render_stats()
    nodes, tris = reference_traversal_counts(built[k][0], cams[k])
    b_ray = 32 + 16 + 32 * nodes + 36 * tris
    ln, ms = prof.get("pt_extend", (1, 0.0))
    rays_per_launch = stats["extend_rays"] / max(1, stats["extend_launches"])
    avg_s = (ms / max(1, ln)) / 1e3
    achieved = rays_per_launch * b_ray / avg_s / 1e9 if avg_s > 0 else 0.0
    return {"bound": "hbm", "kernel": "pt_extend", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"], "traffic": profile_traffic("pt_extend_served4", rays_per_launch),
            "peak_kind": peak_kind,
            "case": "served scene 4 (138,944 tris), 512x512, 16 spp, PT depth 8",
            "bytes_model": f"rays/launch {rays_per_launch:.0f} x (48 + 32*{nodes:.2f} nodes + 36*{tris:.2f} tris) B; "
                           f"reference-traversal counts",
            "issue": issue_ceiling("pt_extend_served4", rays_per_launch / avg_s if avg_s > 0 else 0.0, clocks),
            "kernels_ms": {k2: {"launches": v[0], "ms": v[1]} for k2, v in prof.items()}}


def cpu_jobs_sample(stream, n_samples_target):
    """A bounded, representative sample of the stream for the CPU: the first
    jobs of the stream, each rendered at 1 spp over its full resolution, until
    about `n_samples_target` samples are covered."""
    out, total = [], 0
    for job in stream:
        if total >= n_samples_target:
            break
        out.append(job)
        total += job["res"] ** 2
    return out


def cpu_render_rate(stream, built, n_samples_target, threads):
    import oracle as O
    jobs = cpu_jobs_sample(stream, n_samples_target)
    cache = {}
    samples, secs = 0, 0.0
    for i, job in enumerate(jobs):
        k = job["scene"]
        if k not in cache:
            cache[k] = O.OracleScene(built[k][0])
        cfg = job_cfg(dict(job, spp=1), seed=i)
        t0 = time.perf_counter()
        cache[k].render(built[k][1], cfg, job["res"], job["res"], sampler=O.SAMPLER_XOSHIRO, threads=threads)
        secs += time.perf_counter() - t0
        samples += job["res"] ** 2
    return samples / secs / 1e6, len(jobs), samples, secs


def cpu_baseline_served(stream, built, n_samples_target):
    cores = os.cpu_count() or 1
    rate, n, samples, secs = cpu_render_rate(stream, built, n_samples_target, cores)
    return {"value": rate, "unit": "Mpath-samples/s", "cores": cores, "kind": "port",
            "sample": f"first {n} jobs of the timed set at 1 spp (full resolution, same scene/integrator mix): "
                      f"{samples} path samples in {secs:.1f} s on {cores} threads"}


# ------------------------------------------------------------- pt_cornell ----
def run_pt_cornell(args, rank, local, world, torch, ctx, barrier, dist, peaks, peak_kind, stream):
    import agentray
    import agentray.scenes as S
    from agentray import _abi as A
    from agentray.scene_data import integrator_cfg

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    if args.workload == "pt_served4":
        sc, cam = S.served_scene(4)
        W = H = 512
        desc = "pt_served4: PT on served scene 4 (138,944 tris, 335 instances, 2 quad lights), 512x512, 16 spp, depth 8"
        prof_name = "pt_extend_served4"
    elif args.workload == "pt_cornell_textured":
        sc, cam = S.cornell_box(1, textured=True)
        W = H = 256
        desc = ("pt_cornell_textured: PT Cornell box with 16x16 and 7x7 checker ImageTextures (sRGB, bilinear, "
                "repeat) on floor and back wall, 256x256, 16 spp, depth 8, RR 3")
        prof_name = "pt_extend_cornell_textured"
    elif args.workload == "pt_cornell_glass":
        sc, cam = S.cornell_box(1, glass=True)
        W = H = 256
        desc = ("pt_cornell_glass: PT Cornell box with a rough-glass box (eta 1.5, alpha 0.2) and glass sphere "
                "(eta 1.33, alpha 0.05), 256x256, 16 spp, depth 8, RR 3")
        prof_name = "pt_extend_cornell_glass"
    else:
        sc, cam = S.cornell_box(1)
        W = H = 256
        desc = "pt_cornell: PT Cornell box 34 tris + quad light, 256x256, 16 spp, depth 8, RR 3"
        prof_name = "pt_extend_cornell"
    spp = 16
    if args.res or args.spp:  # a reduced case for profiling
        W = H = args.res or W
        spp = args.spp or spp
        desc += f" [resized: {W}x{H}, {spp} spp]"
    scene = agentray.Scene(ctx, sc)
    out = torch.empty(W * H * 3, dtype=torch.float32, device="cuda")
    pt = agentray.PathTracer(agentray.PathTracerConfig(spp=spp, max_depth=8, rr_depth=3, seed=rank))
    for _ in range(max(3, args.warmup)):
        pt.render(scene, cam, W, H, out=out)
    torch.cuda.synchronize()
    barrier()
    step_ms = []
    with ClockSampler(local) as clk:
        t_start = time.perf_counter()
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
        padded = clk.fill(lambda: (pt.render(scene, cam, W, H, out=out), torch.cuda.synchronize()), t_start)
    launches = args.steps * st["extend_launches"] * 5
    barrier()
    ctx.profile(True)
    ctx.profile_reset()
    for _ in range(args.steps):
        flush.zero_()
        pt.render(scene, cam, W, H, out=out)
    torch.cuda.synchronize()
    ctx.profile(False)
    prof = ctx.profile_read()
    total_ms = max_over_ranks(dist, sum(a.elapsed_time(b) for a, b in step_ms), "cuda")
    stats = ctx.render_stats()
    samples = W * H * spp
    value = world * samples * args.steps / (total_ms / 1e3) / 1e6
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
    if rank == 0:
        nodes, tris = reference_traversal_counts(sc, cam)
        b_ray = 32 + 16 + 32 * nodes + 36 * tris
        ln, ms = prof.get("pt_extend", (0, 0.0))
        rays_per_launch = stats["extend_rays"] / max(1, stats["extend_launches"])
        avg_s = (ms / max(1, ln)) / 1e3
        achieved = rays_per_launch * b_ray / avg_s / 1e9 if avg_s > 0 else 0.0
        import oracle as O
        osc = O.OracleScene(sc)
        cfg = integrator_cfg(A.INTEGRATOR_PT, spp=16, max_depth=8, rr_depth=3)
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        osc.render(cam, cfg, W, H, sampler=O.SAMPLER_XOSHIRO, threads=cores)
        cpu_s = time.perf_counter() - t0
        clocks = clk.summary()
        if padded:
            clocks["window"] = ("the timed steps, then untimed renders of the same workload up to 0.5 s after "
                                "they began (the timed steps are shorter than the 100 ms sampling period)")
        line = {
            "metric": METRIC, "value": value, "unit": "Mpath-samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": desc,
                       "l2": "flushed (256 MiB write) before each timed step", "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "Mpath-samples/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": W * H * 3 * 4,
                    "includes": "Scene::new (host BVH build + upload) + render + readback"},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": "pt_extend", "achieved": achieved, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                         "traffic": profile_traffic(prof_name, rays_per_launch), "peak_kind": peak_kind,
                         "bytes_model": f"rays/launch {rays_per_launch:.0f} x (48 + 32*{nodes:.2f} nodes + "
                                        f"36*{tris:.2f} tris) B; reference-traversal counts",
                         "issue": issue_ceiling(prof_name, rays_per_launch / avg_s if avg_s > 0 else 0.0,
                                                clocks)},
            "kernels_ms": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()},
            "render_stats": stats, "clocks": clocks,
            "cpu_baseline": {"value": samples / cpu_s / 1e6, "unit": "Mpath-samples/s", "cores": cores,
                             "kind": "port", "sample": f"one full {W}x{H}x{spp}spp render, reference sampler"}}
        return line
    return None


# ------------------------------------------------------------------ rooms ----
def run_room(args, rank, local, world, torch, ctx, barrier, dist, peaks, peak_kind, stream):
    """The 200k-triangle room: BDPT 512x512 x 64 spp, path length 10, FP64
    film (bdpt_room), or GDPT 1024x1024 x 32 spp with the CG + FP64-refined
    Poisson solve to relative residual 1e-6 (gdpt_room).  One step = one
    full render."""
    import agentray
    import agentray.scenes as S
    from agentray import _abi as A
    from agentray.scene_data import integrator_cfg

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    sc, cam = S.served_scene(4) if args.workload == "bdpt_served4" else S.room(4)
    scene = agentray.Scene(ctx, sc)
    ntri = scene.stats()["num_triangles"]
    if args.workload == "bdpt_served4":
        W = H = args.res or 512
        spp = args.spp or 16
        integ = agentray.BidirectionalPathTracer(agentray.BdptConfig(spp=spp, max_depth=8, rr_depth=3, seed=4 + rank))
        cfg = integrator_cfg(A.INTEGRATOR_BDPT, spp=1, max_depth=8, rr_depth=3)
        desc = (f"bdpt_served4: BDPT+MIS on served scene 4 ({ntri} tris, 335 instances, 2 quad lights), {W}x{H}, "
                f"{spp} spp, max depth 8")
        top = "bdpt_shadow"
        dtype = "f32"
    elif args.workload == "bdpt_room":
        W = H = args.res or 512
        spp = args.spp or 64
        integ = agentray.BidirectionalPathTracer(agentray.BdptConfig(spp=spp, max_depth=10, rr_depth=3, seed=4 + rank,
                                                                     film_precision=A.FILM_F64))
        cfg = integrator_cfg(A.INTEGRATOR_BDPT, spp=1, max_depth=10, rr_depth=3)
        desc = (f"bdpt_room: BDPT+MIS (power, beta 2) on the room ({ntri} tris: icospheres + 500 instanced boxes, "
                f"Lambert/GGX 50/50, 2 quad lights), {W}x{H}, {spp} spp, max depth 10, FP64 film")
        top = "bdpt_shadow"
        dtype = "f32 transport, f64 film"
    else:
        W = H = args.res or 1024
        spp = args.spp or 32
        integ = agentray.GradientDomainPathTracer(agentray.GdptConfig(
            spp=spp, max_depth=8, rr_depth=3, alpha=0.2, poisson_solver=A.POISSON_CG, poisson_tolerance=1e-6,
            seed=4 + rank))
        cfg = integrator_cfg(A.INTEGRATOR_GDPT, spp=1, max_depth=8, rr_depth=3, alpha=0.2,
                             poisson_solver=A.POISSON_SOR, poisson_iterations=200)
        desc = (f"gdpt_room: GDPT (random replay, x/y shifts) on the room ({ntri} tris), {W}x{H}, {spp} spp, "
                f"alpha 0.2, Poisson by FP32 CG with FP64 residual refinement to rel. residual 1e-6")
        top = "pt_extend"
        dtype = "f32 transport, f64 Poisson residuals"
    out = torch.empty(W * H * 3, dtype=torch.float32, device="cuda")
    for _ in range(max(3, args.warmup)):
        integ.render(scene, cam, W, H, out=out)
    torch.cuda.synchronize()
    barrier()
    evs = []
    with ClockSampler(local) as clk:
        t_start = time.perf_counter()
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            integ.render(scene, cam, W, H, out=out)
            e1.record(stream)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        stats = ctx.render_stats()
        padded = clk.fill(lambda: (integ.render(scene, cam, W, H, out=out), torch.cuda.synchronize()), t_start)
    total_ms = max_over_ranks(dist, sum(a.elapsed_time(b) for a, b in evs), "cuda")
    samples = W * H * spp
    value = world * samples * args.steps / (total_ms / 1e3) / 1e6
    ctx.profile(True)
    ctx.profile_reset()
    flush.zero_()
    integ.render(scene, cam, W, H, out=out)
    torch.cuda.synchronize()
    ctx.profile(False)
    prof = ctx.profile_read()
    pstats = ctx.render_stats()
    host_out = np.empty(W * H * 3, np.float32)
    e2e = []
    for _ in range(max(1, min(3, args.steps))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        integ.render(scene, cam, W, H, out=host_out)
        e2e.append(time.perf_counter() - t0)
    e2e_value = samples / statistics.mean(e2e) / 1e6
    if rank == 0:
        nodes, tris = reference_traversal_counts(sc, cam)
        b_ray = 32 + 16 + 32 * nodes + 36 * tris
        ln, ms = prof.get(top, (1, 0.0))
        rays = pstats["shadow_rays"] if top == "bdpt_shadow" else pstats["extend_rays"]
        achieved = rays * b_ray / (ms / 1e3) / 1e9 if ms > 0 else 0.0
        clocks = clk.summary()
        if padded:
            clocks["window"] = ("the timed steps, then untimed renders of the same workload up to 0.5 s after "
                                "they began (the timed steps are shorter than the 100 ms sampling period)")
        prof_name = {"bdpt_served4": "bdpt_served4", "bdpt_room": "bdpt_shadow_room",
                     "gdpt_room": "pt_extend_room"}[args.workload]
        import oracle as O
        osc = O.OracleScene(sc)
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        osc.render(cam, cfg, W, H, sampler=O.SAMPLER_XOSHIRO, threads=cores)
        cpu_s = time.perf_counter() - t0
        osc.close()
        line = {
            "metric": METRIC, "value": value, "unit": "Mpath-samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded procedural scene)",
            "config": {"workload": desc, "l2": "flushed (256 MiB write) before each timed step",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "Mpath-samples/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": W * H * 3 * 4, "note": "scene resident; image returned to a host buffer"},
            "gpu_launches": int(sum(v[0] for v in prof.values()) * args.steps),
            "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                         "traffic": profile_traffic(prof_name, rays / max(1, ln)),
                         "peak_kind": peak_kind,
                         "bytes_model": f"{rays} rays x (48 + 32*{nodes:.2f} nodes + 36*{tris:.2f} tris) B over "
                                        f"{ln} launches; reference-traversal counts of primary/interior rays",
                         "issue": issue_ceiling(prof_name, rays / (ms / 1e3) if ms > 0 else 0.0, clocks)},
            "kernels_ms": {k: {"launches": v[0], "ms": v[1]} for k, v in prof.items()},
            "render_stats": stats, "clocks": clocks,
            "cpu_baseline": {"value": W * H / cpu_s / 1e6, "unit": "Mpath-samples/s", "cores": cores, "kind": "port",
                             "sample": f"one {W}x{H} render at 1 spp, reference sampler"}}
        return line
    return None


# -------------------------------------------------------------------- bvh ----
def run_bvh(args, rank, local, world, torch, ctx, barrier, dist, peaks, peak_kind, stream):
    """Config 2: 1M-triangle soup, 16M rays.  One step = one closest-hit
    launch over the 16M rays (rays resident in HBM); any-hit (t_max 0.25) is
    timed the same way beside it; e2e passes host arrays (rays in, hits out)."""
    import agentray
    import agentray.scenes as S
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    n_tris, n_rays = 1_000_000, args.rays or 16_000_000
    sc = S.triangle_soup(n_tris, seed=2)
    t0 = time.perf_counter()
    scene = agentray.Scene(ctx, sc)
    build_s = time.perf_counter() - t0
    ot, dt = S.soup_rays(n_rays, seed=3)
    ot_d = torch.from_numpy(ot).cuda()
    dt_d = torch.from_numpy(dt).cuda()
    dt_any = dt_d.clone()
    dt_any[:, 3] = 0.25
    for _ in range(max(3, args.warmup)):
        scene.trace_closest(ot_d, dt_d)
        scene.trace_any(ot_d, dt_any)
    torch.cuda.synchronize()
    barrier()

    def timed(fn):
        ev = []
        for _ in range(args.steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            ev.append((a, b))
        torch.cuda.synchronize()
        return max_over_ranks(dist, sum(a.elapsed_time(b) for a, b in ev), "cuda")

    with ClockSampler(local) as clk:
        total_ms = timed(lambda: scene.trace_closest(ot_d, dt_d))
    any_ms = timed(lambda: scene.trace_any(ot_d, dt_any))
    value = world * n_rays * args.steps / (total_ms / 1e3) / 1e6
    any_value = world * n_rays * args.steps / (any_ms / 1e3) / 1e6
    # e2e: host arrays in pinned memory, rays copied in and hits copied out each step
    ot_h = torch.from_numpy(ot).pin_memory().numpy()
    dt_h = torch.from_numpy(dt).pin_memory().numpy()
    hits_h = torch.empty((n_rays, 4), dtype=torch.float32, pin_memory=True).numpy()
    inst_h = torch.empty(n_rays, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    e2e = []
    for _ in range(max(1, min(3, args.steps))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        scene.trace_closest(ot_h, dt_h, out=(hits_h, inst_h))
        e2e.append(time.perf_counter() - t0)
    e2e_value = n_rays / statistics.mean(e2e) / 1e6
    if rank == 0:
        import oracle as O
        osc = O.OracleScene(sc)
        r = osc.trace_closest(ot[:200_000], dt[:200_000], stats=True)
        nodes = r["stats"]["nodes"] / 200_000
        tris = r["stats"]["tris"] / 200_000
        b_ray = 32 + 16 + 32 * nodes + 36 * tris
        rays_per_s = n_rays / (total_ms / args.steps / 1e3)
        achieved = rays_per_s * b_ray / 1e9
        t0 = time.perf_counter()
        osc.trace_closest(ot[:2_000_000], dt[:2_000_000])
        cpu = 2_000_000 / (time.perf_counter() - t0) / 1e6
        osc.close()
        clocks = clk.summary()
        line = {"metric": "Mrays/s (closest hit)", "value": value, "unit": "Mrays/s", "n_gpus": world,
                "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": f"bvh: 1M-triangle soup (seed 2), {n_rays / 1e6:g}M rays (seed 3), closest "
                                       f"hit; any hit with t_max 0.25 beside it",
                           "l2": f"flushed; rays {n_rays * 32 / 1e6:.0f} MB"},
                "any_hit": {"value": any_value, "unit": "Mrays/s", "ms_per_step": any_ms / args.steps},
                "host_bvh_build_s": build_s,
                "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": n_rays * 32,
                        "d2h_bytes_per_step": n_rays * 20,
                        "note": "rays from pinned host arrays, hits (t, u, v, prim; instance id) back into pinned "
                                "host arrays; the library copies 4M-ray chunks on two copy streams while the "
                                "previous chunk is traced"},
                "gpu_launches": args.steps,
                "roofline": {"bound": "hbm", "kernel": "trace_closest", "achieved": achieved,
                             "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                             "traffic": profile_traffic("trace_closest_soup", n_rays), "peak_kind": peak_kind,
                             "bytes_model": f"48 + 32*{nodes:.1f} + 36*{tris:.1f} B/ray (reference binary SAH "
                                            f"traversal counts)",
                             "issue": issue_ceiling("trace_closest_soup", rays_per_s, clocks)},
                "clocks": clocks,
                "cpu_baseline": {"value": cpu, "unit": "Mrays/s", "cores": os.cpu_count(), "kind": "port",
                                 "sample": "2M of the 16M rays, reference binary SAH traversal"}}
        return line
    return None


# -------------------------------------------------------------- reference ----
def run_reference(args, rank, world):
    """--impl reference: the reference CPU algorithms (oracle restatement with
    the reference's xoshiro256++ per-pixel streams) on all host cores; each
    step renders a bounded slice of the served stream (jobs at 1 spp over their
    full resolution, ~args.cpu_samples samples per step)."""
    if rank != 0:
        return
    import agentray.scenes as S
    cores = os.cpu_count() or 1
    stream = S.served_stream(args.jobs, seed=5)[:args.timed_jobs]
    built = [S.served_scene(k) for k in range(8)]
    for w in range(args.warmup):
        cpu_render_rate(stream[w * 3:], built, 16384, cores)
    rates, tot_samples, tot_secs = [], 0, 0.0
    for k in range(args.steps):
        start = (k * 7) % max(1, len(stream) - 16)
        rate, n, samples, secs = cpu_render_rate(stream[start:], built, args.cpu_samples // max(1, args.steps),
                                                 cores)
        tot_samples += samples
        tot_secs += secs
    value = tot_samples / tot_secs / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mpath-samples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scenes and job stream)",
            "config": {"workload": SERVED_DESC,
                       "timed_set": f"jobs [0, {args.timed_jobs}) of the seeded {args.jobs}-job stream"},
            "cpu_baseline": {"value": value, "unit": "Mpath-samples/s", "cores": cores, "kind": "port",
                             "sample": f"{args.steps} slices of the timed set, jobs at 1 spp over full resolution, "
                                       f"{tot_samples} samples in {tot_secs:.1f} s"},
            "e2e": {"value": value, "unit": "Mpath-samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="served",
                    choices=["served", "pt_cornell", "pt_cornell_glass", "pt_cornell_textured", "pt_served4",
                             "bdpt_served4", "bdpt_room",
                             "gdpt_room", "bvh"])
    ap.add_argument("--jobs", type=int, default=2000)
    ap.add_argument("--timed-jobs", dest="timed_jobs", type=int, default=400,
                    help="served: the fixed timed set is jobs [0, timed_jobs) of the stream")
    ap.add_argument("--window-jobs", dest="window_jobs", type=int, default=8,
                    help="served: jobs per warm-up step")
    ap.add_argument("--config-steps", dest="config_steps", type=int, default=5,
                    help="served: timed steps of each configs.* sub-line (configs 1-4)")
    ap.add_argument("--no-configs", dest="no_configs", action="store_true",
                    help="served: skip the configs 1-4 sub-lines")
    ap.add_argument("--path-capacity", dest="path_capacity", type=int, default=1 << 22)
    ap.add_argument("--bdpt-batch", dest="bdpt_batch", type=int, default=1 << 21)
    ap.add_argument("--bdpt-batch-mib", dest="bdpt_batch_mib", type=int, default=0,
                    help="HBM per plain-path BDPT batch (0: the library default)")
    ap.add_argument("--cpu-samples", dest="cpu_samples", type=int, default=4_000_000)
    ap.add_argument("--res", type=int, default=0, help="single-render workloads: override the resolution "
                                                         "(reduced cases for profiling)")
    ap.add_argument("--spp", type=int, default=0, help="single-render workloads: override spp")
    ap.add_argument("--rays", type=int, default=0, help="bvh: override the ray count")
    args = ap.parse_args()
    rank, local, world = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    import agentray
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    peaks, peak_kind = load_peaks()
    ctx = agentray.Context(local)
    # A dedicated stream: the library launches on it, and every timing event is
    # recorded on it (torch's legacy default stream has handle 0, which the C ABI
    # reads as "use the context's own stream").
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    if args.bdpt_batch_mib:
        ctx.set_tuning(bdpt_batch_mib=args.bdpt_batch_mib)

    def barrier():
        if dist is not None:
            dist.barrier()

    def run_one(a):
        if a.workload in ("pt_cornell", "pt_cornell_glass", "pt_cornell_textured", "pt_served4"):
            return run_pt_cornell(a, rank, local, world, torch, ctx, barrier, dist, peaks, peak_kind, stream)
        if a.workload in ("bdpt_served4", "bdpt_room", "gdpt_room"):
            return run_room(a, rank, local, world, torch, ctx, barrier, dist, peaks, peak_kind, stream)
        return run_bvh(a, rank, local, world, torch, ctx, barrier, dist, peaks, peak_kind, stream)

    if args.workload == "served":
        line = run_served(args, rank, local, world, torch, ctx, barrier, dist, peaks, peak_kind, stream)
        if not args.no_configs:
            # configs 1-4, each measured in this process after the served run
            subs = {}
            for name in ("pt_cornell", "bvh", "bdpt_room", "gdpt_room"):
                a = argparse.Namespace(**vars(args))
                a.workload, a.steps, a.warmup = name, args.config_steps, 3
                subs[name] = run_one(a)
            if line is not None:
                line["configs"] = subs
    else:
        line = run_one(args)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
