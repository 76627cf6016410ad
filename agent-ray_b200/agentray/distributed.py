"""Multi-GPU rendering of one job by sample sharding.

Every rank renders a disjoint range of each pixel's samples with
ar_render_samples (same seed, so the sample streams are those of the
one-process render), weighted by 1/spp; one all-reduce (SUM) of the images
over the process group (NCCL for CUDA tensors, gloo for host tensors) gives
every rank the full image.  This is the one exchange step the path has: the
per-sample work needs no communication.  PT and BDPT (GDPT solves its Poisson
system after all samples).
"""
import ctypes as C

import numpy as np

from ._lib import check, lib


def shard_range(spp, rank, world):
    """Samples [begin, end) of rank `rank` out of `world`: contiguous,
    disjoint, covering [0, spp), sizes differing by at most one."""
    return spp * rank // world, spp * (rank + 1) // world


def render_shard(integrator, scene, camera, width, height, begin, end, out):
    """Renders samples [begin, end) of every pixel into `out` (a float32 CUDA
    tensor or numpy array of width*height*3)."""
    cfg = integrator.cfg()
    cam = camera.desc()
    on_device = not isinstance(out, np.ndarray)
    if on_device:
        with scene.ctx.on_torch_stream(out):
            check(lib().ar_render_samples(scene.ctx.handle, scene.handle, C.byref(cam), C.byref(cfg), width, height,
                                          begin, end, out.data_ptr(), 1))
        return out
    check(lib().ar_render_samples(scene.ctx.handle, scene.handle, C.byref(cam), C.byref(cfg), width, height, begin,
                                  end, out.ctypes.data, 0))
    return out


def render(integrator, scene, camera, width, height, group=None, device="cuda", render_fn=None):
    """The full (height, width, 3) image on every rank of `group`
    (torch.distributed, already initialised).  `render_fn(begin, end, out)`
    replaces the GPU render of a range (host-only tests)."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    begin, end = shard_range(integrator.config.spp, rank, world)
    out = torch.zeros(width * height * 3, dtype=torch.float32, device=device)
    if end > begin:
        if render_fn is not None:
            render_fn(begin, end, out)
        elif out.is_cuda:
            render_shard(integrator, scene, camera, width, height, begin, end, out)
            torch.cuda.current_stream().synchronize()
        else:
            render_shard(integrator, scene, camera, width, height, begin, end, out.numpy())
    dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out.view(height, width, 3)
