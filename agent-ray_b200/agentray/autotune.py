"""Autotuner front end: runs ar_autotune for a workload and caches the result.

ar_autotune (C ABI) does the search on the device: coordinate descent over
the wide-BVH build (children per node, triangles per leaf), the persistent
traversal grid, the shading block size and the queue capacities, each
candidate timed with CUDA events.  This module keys results by GPU model,
scene size and workload in a JSON file, so a later process applies the
stored parameters without searching again.
"""
import ctypes as C
import json
import os

from . import _abi as A
from ._lib import check, lib

_KINDS = {"pt": A.INTEGRATOR_PT, "bdpt": A.INTEGRATOR_BDPT, "gdpt": A.INTEGRATOR_GDPT}


def _device_name(device):
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(device)
    except ImportError:
        pass
    return "unknown"


def cache_key(device_name, scene_stats, integrator, width, height, spp):
    return (f"{device_name}|tris={scene_stats['num_triangles']}|inst={scene_stats['num_instances']}|"
            f"{integrator}|{width}x{height}|spp={spp}")


def apply(ctx, scene, entry):
    """Applies a stored result: context tuning, then the scene's accel build."""
    ctx.set_tuning(**entry["tuning"])
    a = entry["accel"]
    scene.rebuild(max_leaf_size=a["max_leaf_size"] or 3, sah_bins=a["sah_bins"] or 32,
                  bvh_width=a["bvh_width"] or 8, sah_node_cost=a.get("sah_node_cost") or 0.5)


def load_cache(path):
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def store_cache(path, cache):
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tune(ctx, scene, camera, integrator="pt", width=256, height=256, spp=4, max_depth=8, repeats=3,
         tune_accel=True, cache_path=None):
    """Returns the tuning entry for this workload, searching only when
    `cache_path` holds none for it.  The result is applied to ctx and scene."""
    key = cache_key(_device_name(ctx.device), scene.stats(), integrator, width, height, spp)
    cache = load_cache(cache_path)
    if key in cache:
        apply(ctx, scene, cache[key])
        return dict(cache[key], cached=True)
    o = A.TuneOpts(_KINDS[integrator], width, height, spp, max_depth, repeats, 1 if tune_accel else 0, 0)
    r = A.TuneResult()
    cam = camera.desc()
    check(lib().ar_autotune(ctx.handle, scene.handle, C.byref(cam), C.byref(o), C.byref(r)))
    entry = {"tuning": {k: getattr(r.tuning, k) for k, _ in A.Tuning._fields_},
             "accel": {k: getattr(r.accel, k) for k, _ in A.AccelOpts._fields_},
             "default_ms": r.default_ms, "best_ms": r.best_ms, "candidates": r.candidates}
    if cache_path:
        cache[key] = entry
        store_cache(cache_path, cache)
    return dict(entry, cached=False)
