"""agentray — Python host mirror of agent-ray's rendering API over libagentray.

The reference crate's surface (src/integrators/mod.rs:18-26, src/scene.rs,
src/cameras.rs, src/film.rs) maps as follows:

  Scene::new(objects, lights, light_dist)      -> Scene(context, scene_data)
  PinholeCamera::from_lookat(...)              -> Camera(lookfrom, lookat, vup, vfov, aspect)
  PathTracer::new(PathTracerConfig{..})        -> PathTracer(PathTracerConfig(..))
  BidirectionalPathTracer / BdptConfig         -> BidirectionalPathTracer(BdptConfig(..))
  GradientDomainPathTracer / GdptConfig        -> GradientDomainPathTracer(GdptConfig(..))
  Integrator::render(&scene, &camera, w, h)    -> integrator.render(scene, camera, w, h) -> Film
  Film::to_hdr_vec()                           -> Film.to_hdr_vec()  ((H*W, 3) float32)
  Scene::intersect / occluded (ray batches)    -> Scene.trace_closest / Scene.trace_any
  Film::to_rgb_image / save_exr                -> Film.to_rgb_image / save_png / save_exr
  load_obj_scene(path, transform)              -> importer.load_obj_scene(scene_data, path, transform)

Rendering, tracing and film output run in the CUDA library; on the host there
is only I/O (OBJ/MTL/PNG reading, PNG writing) and descriptor assembly.
"""
import contextlib
import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _abi as A
from ._lib import AgentRayError, check, lib
from .scene_data import Camera, Light, Material, Mesh, Object, SceneData, integrator_cfg

__all__ = ["Context", "Scene", "Camera", "Film", "PathTracer", "PathTracerConfig", "BidirectionalPathTracer",
           "BdptConfig", "GradientDomainPathTracer", "GdptConfig", "SceneData", "Mesh", "Object", "Material",
           "Light", "AgentRayError", "integrator_cfg", "lib", "Server", "poisson_reconstruct", "film_to_rgb8",
           "film_save_exr", "write_png"]


class Context:
    """One CUDA device + stream (ar_context)."""

    def __init__(self, device=0):
        self.device = device
        self.handle = C.c_void_p()
        self._stream = None  # None: the context's own stream
        check(lib().ar_context_create(device, C.byref(self.handle)))

    def set_stream(self, stream_ptr):
        """Launch on this cudaStream_t (an int); None or 0 restores the
        context's own stream."""
        check(lib().ar_context_set_stream(self.handle, C.c_void_p(stream_ptr or None)))
        self._stream = stream_ptr or None

    @contextlib.contextmanager
    def on_torch_stream(self, tensor):
        """Runs the enclosed library calls on torch's current stream of
        `tensor`'s device, so that they are ordered after the torch work that
        produced their device inputs and before the torch work that reads
        their device outputs."""
        import torch
        ts = torch.cuda.current_stream(tensor.device)
        if ts.cuda_stream == 0:
            # torch's legacy default stream cannot be handed to the library (a
            # null stream selects the context's own): order by synchronising.
            ts.synchronize()
            try:
                yield
            finally:
                self.synchronize()
            return
        prev = self._stream
        self.set_stream(ts.cuda_stream)
        try:
            yield
        finally:
            self.set_stream(prev)

    def synchronize(self):
        check(lib().ar_context_synchronize(self.handle))

    def render_stats(self):
        s = A.RenderStats()
        check(lib().ar_get_render_stats(self.handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in A.RenderStats._fields_}

    def profile(self, enable=True):
        check(lib().ar_profile_enable(self.handle, 1 if enable else 0))

    def profile_reset(self):
        check(lib().ar_profile_reset(self.handle))

    def profile_read(self):
        """{kernel name: (launches, summed device ms)} since the last reset."""
        cap = 64
        names = C.create_string_buffer(8192)
        ms = (C.c_double * cap)()
        ln = (C.c_uint64 * cap)()
        n = C.c_uint32(cap)
        check(lib().ar_profile_read(self.handle, names, 8192, ms, ln, C.byref(n)))
        keys = names.value.decode().split("\n")[: n.value]
        return {k: (int(ln[i]), float(ms[i])) for i, k in enumerate(keys)}

    def tuning(self):
        """Launch shapes and queue capacities of this context (ar_tuning)."""
        t = A.Tuning()
        check(lib().ar_context_get_tuning(self.handle, C.byref(t)))
        return {k: getattr(t, k) for k, _ in A.Tuning._fields_}

    def set_tuning(self, **kw):
        """Updates some of path_capacity, traversal_blocks_per_sm, shade_block,
        bdpt_batch_mib (the rest keep their values)."""
        cur = self.tuning()
        unknown = set(kw) - set(cur)
        if unknown:
            raise ValueError(f"unknown tuning keys {sorted(unknown)}")
        cur.update(kw)
        t = A.Tuning(**cur)
        check(lib().ar_context_set_tuning(self.handle, C.byref(t)))

    def close(self):
        if self.handle:
            lib().ar_context_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """Device-resident scene with its acceleration structures (Scene::new)."""

    def __init__(self, ctx: Context, data: SceneData):
        self.ctx = ctx
        self.data = data
        self.handle = C.c_void_p()
        desc, keep = data.desc()
        check(lib().ar_scene_create(ctx.handle, C.byref(desc), C.byref(self.handle)))
        del keep

    def stats(self):
        s = A.SceneStats()
        check(lib().ar_scene_get_stats(self.handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in A.SceneStats._fields_ if not k.startswith("_")}

    def rebuild(self, max_leaf_size=3, sah_bins=32, build_threads=0, bvh_width=8, sah_node_cost=0.5):
        o = A.AccelOpts(max_leaf_size, sah_bins, build_threads, bvh_width, sah_node_cost, 0)
        check(lib().ar_scene_build_accel(self.ctx.handle, self.handle, C.byref(o)))

    @staticmethod
    def _batch(org_tmin, dir_tmax, on_device):
        b = A.RayBatch()
        if on_device:
            b.org_tmin, b.dir_tmax, b.count = org_tmin.data_ptr(), dir_tmax.data_ptr(), org_tmin.shape[0]
        else:
            b.org_tmin, b.dir_tmax, b.count = org_tmin.ctypes.data, dir_tmax.ctypes.data, org_tmin.shape[0]
        b.on_device = 1 if on_device else 0
        return b

    def trace_closest(self, org_tmin, dir_tmax, out=None):
        """Closest hit for (n,4) float32 ray arrays (numpy on the host, or torch
        CUDA tensors).  Returns (hits (n,4): t,u,v,prim_id-bits; inst_ids (n,)).
        Host arrays may come with `out` = (hits, inst_ids) numpy arrays to fill
        (pinned ones let the copies overlap the traversal)."""
        dev = not isinstance(org_tmin, np.ndarray)
        if dev:
            import torch
            org_tmin, dir_tmax = self._device_rays(org_tmin, dir_tmax)
            hits = torch.empty((org_tmin.shape[0], 4), dtype=torch.float32, device=org_tmin.device)
            inst = torch.empty((org_tmin.shape[0],), dtype=torch.int32, device=org_tmin.device)
            b = self._batch(org_tmin, dir_tmax, True)
            with self.ctx.on_torch_stream(org_tmin):
                check(lib().ar_trace_closest(self.ctx.handle, self.handle, C.byref(b), hits.data_ptr(),
                                             inst.data_ptr(), 1))
            return hits, inst
        org_tmin = np.ascontiguousarray(org_tmin, np.float32)
        dir_tmax = np.ascontiguousarray(dir_tmax, np.float32)
        n = org_tmin.shape[0]
        if out is not None:
            hits, inst = out
            assert hits.shape == (n, 4) and hits.dtype == np.float32 and hits.flags.c_contiguous
            assert inst.shape == (n,) and inst.dtype == np.uint32 and inst.flags.c_contiguous
        else:
            hits = np.empty((n, 4), np.float32)
            inst = np.empty(n, np.uint32)
        b = self._batch(org_tmin, dir_tmax, False)
        check(lib().ar_trace_closest(self.ctx.handle, self.handle, C.byref(b), hits.ctypes.data, inst.ctypes.data,
                                     0))
        return hits, inst

    @staticmethod
    def _device_rays(org_tmin, dir_tmax):
        """Contiguous float32 (n, 4) CUDA tensors on one device."""
        import torch
        if not (isinstance(dir_tmax, torch.Tensor) and org_tmin.is_cuda and dir_tmax.device == org_tmin.device):
            raise ValueError("org_tmin and dir_tmax must be CUDA tensors on the same device")
        if org_tmin.dim() != 2 or org_tmin.shape[1] != 4 or dir_tmax.shape != org_tmin.shape:
            raise ValueError("rays must be (n, 4) arrays")
        return org_tmin.to(torch.float32).contiguous(), dir_tmax.to(torch.float32).contiguous()

    def trace_any(self, org_tmin, dir_tmax, out=None):
        """Occlusion (Scene::occluded) for (n,4) float32 ray arrays (numpy on the
        host, or torch CUDA tensors).  Returns (n,) uint8: 1 = occluded."""
        if not isinstance(org_tmin, np.ndarray):
            import torch
            org_tmin, dir_tmax = self._device_rays(org_tmin, dir_tmax)
            occ = torch.empty((org_tmin.shape[0],), dtype=torch.uint8, device=org_tmin.device)
            b = self._batch(org_tmin, dir_tmax, True)
            with self.ctx.on_torch_stream(org_tmin):
                check(lib().ar_trace_any(self.ctx.handle, self.handle, C.byref(b), occ.data_ptr(), 1))
            return occ
        org_tmin = np.ascontiguousarray(org_tmin, np.float32)
        dir_tmax = np.ascontiguousarray(dir_tmax, np.float32)
        occ = np.empty(org_tmin.shape[0], np.uint8) if out is None else out
        assert occ.shape == (org_tmin.shape[0],) and occ.dtype == np.uint8 and occ.flags.c_contiguous
        b = self._batch(org_tmin, dir_tmax, False)
        check(lib().ar_trace_any(self.ctx.handle, self.handle, C.byref(b), occ.ctypes.data, 0))
        return occ

    def close(self):
        if self.handle:
            lib().ar_scene_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Film:
    """Linear HDR film (src/film.rs), already divided by spp."""

    def __init__(self, rgb: np.ndarray, width: int, height: int, ctx=None):
        self.rgb = rgb.reshape(height, width, 3)
        self.width = width
        self.height = height
        self.ctx = ctx

    def to_hdr_vec(self):
        return self.rgb.reshape(-1, 3)

    def get_pixel(self, x, y):
        return self.rgb[y, x]

    def to_rgb_image(self, tone_mapper=A.TONEMAP_CLAMP, gamma=2.2, scale=1.0, white_point=1.0):
        """Film::to_rgb_image (src/film.rs:276-302) on the GPU: (H, W, 3) uint8."""
        return film_to_rgb8(self.ctx, self.rgb, tone_mapper, gamma, scale, white_point)

    def save_png(self, path, tone_mapper=A.TONEMAP_CLAMP, gamma=2.2, scale=1.0, white_point=1.0):
        write_png(path, self.to_rgb_image(tone_mapper, gamma, scale, white_point))

    def save_exr(self, path, scale=1.0):
        """Film::save_exr (src/film.rs:304-346): linear HALF RGB, ZIP-compressed OpenEXR."""
        film_save_exr(self.ctx, self.rgb, path, scale)


def film_to_rgb8(ctx, hdr, tone_mapper=A.TONEMAP_CLAMP, gamma=2.2, scale=1.0, white_point=1.0):
    """Tone-maps an (H, W, 3) float32 image (host array or CUDA tensor) to
    8-bit RGB with ar_film_to_rgb8; returns a host array, or a CUDA uint8
    tensor for a CUDA input."""
    if ctx is None:
        raise ValueError("a Context is needed to tone-map on the GPU")
    if not isinstance(hdr, np.ndarray):
        import torch
        hdr = hdr.to(torch.float32).contiguous()
        h, w = hdr.shape[0], hdr.shape[1]
        out = torch.empty((h, w, 3), dtype=torch.uint8, device=hdr.device)
        with ctx.on_torch_stream(hdr):
            check(lib().ar_film_to_rgb8(ctx.handle, hdr.data_ptr(), w, h, tone_mapper, white_point, gamma, scale,
                                        out.data_ptr(), 1))
        return out
    x = np.ascontiguousarray(hdr, np.float32)
    h, w = x.shape[0], x.shape[1]
    out = np.empty((h, w, 3), np.uint8)
    check(lib().ar_film_to_rgb8(ctx.handle, x.ctypes.data, w, h, tone_mapper, white_point, gamma, scale,
                                out.ctypes.data, 0))
    return out


def film_save_exr(ctx, hdr, path, scale=1.0):
    """Writes an (H, W, 3) float32 image (host array or CUDA tensor) * scale as
    a ZIP-compressed HALF OpenEXR file with ar_film_save_exr."""
    if ctx is None:
        raise ValueError("a Context is needed to pack the EXR on the GPU")
    p = os.fsencode(path)
    if not isinstance(hdr, np.ndarray):
        import torch
        x = hdr.to(torch.float32).contiguous()
        with ctx.on_torch_stream(x):
            check(lib().ar_film_save_exr(ctx.handle, x.data_ptr(), x.shape[1], x.shape[0], scale, 1, p))
        return
    x = np.ascontiguousarray(hdr, np.float32)
    check(lib().ar_film_save_exr(ctx.handle, x.ctypes.data, x.shape[1], x.shape[0], scale, 0, p))


def write_png(path, rgb8):
    """Writes an (H, W, 3) uint8 image as an 8-bit RGB PNG (zlib, no filter)."""
    import struct
    import zlib
    h, w, _ = rgb8.shape
    raw = b"".join(b"\x00" + np.ascontiguousarray(rgb8[y]).tobytes() for y in range(h))

    def chunk(tag, data):
        c = struct.pack(">I", len(data)) + tag + data
        return c + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)
    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))


@dataclass
class PathTracerConfig:
    """src/integrators/path_tracer.rs:18-31"""
    spp: int = 64
    max_depth: int = 8
    rr_depth: int = 3
    seed: int = 0
    film_precision: int = A.FILM_F32


@dataclass
class BdptConfig:
    """src/integrators/bidirectional_path_tracer.rs:102-133"""
    spp: int = 64
    max_depth: int = 8
    rr_depth: int = 3
    mis_mode: int = A.MIS_POWER
    mis_beta: float = 2.0
    seed: int = 0
    film_precision: int = A.FILM_F32


@dataclass
class GdptConfig:
    """src/integrators/gradient_domain_pt.rs:47-76 (+ solver choice)."""
    spp: int = 64
    max_depth: int = 8
    rr_depth: int = 3
    alpha: float = 0.2
    poisson_iterations: int = 200
    sor_omega: float = 1.6
    poisson_solver: int = A.POISSON_SOR
    poisson_tolerance: float = 1e-6
    seed: int = 0
    film_precision: int = A.FILM_F32
    # extension: A.GDPT_CONSISTENT_DIVERGENCE solves with -div G (converges to
    # the primal-domain image); 0 reproduces the reference's +div G
    gdpt_flags: int = 0


class _Integrator:
    kind = A.INTEGRATOR_PT

    def __init__(self, config):
        self.config = config

    def cfg(self):
        c = self.config
        return integrator_cfg(self.kind, spp=c.spp, max_depth=c.max_depth, rr_depth=c.rr_depth,
                              mis_mode=getattr(c, "mis_mode", A.MIS_POWER), mis_beta=getattr(c, "mis_beta", 2.0),
                              alpha=getattr(c, "alpha", 0.2), poisson_iterations=getattr(c, "poisson_iterations", 200),
                              sor_omega=getattr(c, "sor_omega", 1.6),
                              poisson_solver=getattr(c, "poisson_solver", A.POISSON_SOR),
                              poisson_tolerance=getattr(c, "poisson_tolerance", 1e-6), seed=c.seed,
                              film_precision=c.film_precision, gdpt_flags=getattr(c, "gdpt_flags", 0))

    def render(self, scene: Scene, camera: Camera, width: int, height: int, out=None) -> Film:
        """Integrator::render.  `out` may be a CUDA float32 tensor of W*H*3 to
        keep the image on the device."""
        cfg = self.cfg()
        cam = camera.desc()
        if out is not None and not isinstance(out, np.ndarray):
            with scene.ctx.on_torch_stream(out):
                check(lib().ar_render(scene.ctx.handle, scene.handle, C.byref(cam), C.byref(cfg), width, height,
                                      out.data_ptr(), 1))
            return out
        buf = np.empty(width * height * 3, np.float32) if out is None else out
        check(lib().ar_render(scene.ctx.handle, scene.handle, C.byref(cam), C.byref(cfg), width, height,
                              buf.ctypes.data, 0))
        return Film(buf, width, height, scene.ctx)


class PathTracer(_Integrator):
    kind = A.INTEGRATOR_PT


class BidirectionalPathTracer(_Integrator):
    kind = A.INTEGRATOR_BDPT


class GradientDomainPathTracer(_Integrator):
    kind = A.INTEGRATOR_GDPT


class Server:
    """Render server (ar_server): continuously batches submitted jobs into
    shared wavefront kernels on one GPU.  submit() returns a job id at once;
    the image lands in the job's host buffer before its status becomes DONE."""

    STATUS = {A.JOB_PENDING: "pending", A.JOB_RUNNING: "running", A.JOB_DONE: "done", A.JOB_REJECTED: "rejected",
              A.JOB_CANCELLED: "cancelled", A.JOB_FAILED: "failed"}

    def __init__(self, ctx: Context, film_budget_bytes=0, path_capacity=0, bdpt_batch_samples=0, bdpt_max_depth=0,
                 max_active_jobs=0):
        self.ctx = ctx
        self.handle = C.c_void_p()
        o = A.ServerOpts(film_budget_bytes, path_capacity, bdpt_batch_samples, bdpt_max_depth, max_active_jobs)
        check(lib().ar_server_create(ctx.handle, C.byref(o), C.byref(self.handle)))
        self.outputs = {}
        self._keep = {}

    def submit(self, scene: Scene, camera: Camera, integrator, width, height, out=None):
        """Queues a job.  `out` may be a host numpy buffer (default: a new one)
        or a CUDA float32 tensor of W*H*3 elements to keep the image on the GPU."""
        on_device = out is not None and not isinstance(out, np.ndarray)
        if out is None:
            out = np.empty(width * height * 3, np.float32)
        if on_device:
            # the server writes `out` from its own streams: let the torch work
            # queued on this memory finish first
            import torch
            torch.cuda.current_stream(out.device).synchronize()
        ptr = out.data_ptr() if on_device else out.ctypes.data
        cam = camera.desc()
        cfg = integrator.cfg()
        jid = C.c_uint64()
        check(lib().ar_job_submit(self.handle, scene.handle, C.byref(cam), C.byref(cfg), width, height, ptr,
                                  1 if on_device else 0, C.byref(jid)))
        self.outputs[jid.value] = out if on_device else out.reshape(height, width, 3)
        self._keep[jid.value] = scene
        return jid.value

    def forget(self, job_id):
        """Drops the Python-side references of a finished job."""
        self.outputs.pop(job_id, None)
        self._keep.pop(job_id, None)

    @staticmethod
    def _info(i):
        return {"status": Server.STATUS[i.status], "error": i.error, "submit_ms": i.submit_ms,
                "admit_ms": i.admit_ms, "done_ms": i.done_ms, "path_samples": i.path_samples}

    def poll(self, job_id):
        i = A.JobInfo()
        check(lib().ar_job_poll(self.handle, job_id, C.byref(i)))
        return self._info(i)

    def wait(self, job_id, timeout_ms=600_000.0):
        i = A.JobInfo()
        check(lib().ar_job_wait(self.handle, job_id, timeout_ms, C.byref(i)))
        return self._info(i)

    def cancel(self, job_id):
        check(lib().ar_job_cancel(self.handle, job_id))

    def result(self, job_id):
        return self.outputs[job_id]

    def stats(self):
        s = A.ServerStats()
        check(lib().ar_server_get_stats(self.handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in A.ServerStats._fields_}

    def now_ms(self):
        return lib().ar_server_now_ms(self.handle)

    def debug_dump(self):
        buf = C.create_string_buffer(1 << 16)
        check(lib().ar_server_debug_dump(self.handle, buf, 1 << 16))
        return buf.value.decode()

    def close(self):
        if self.handle:
            check(lib().ar_server_destroy(self.handle))
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def poisson_reconstruct(ctx: Context, primal, grad_x, grad_y, alpha=0.2, solver=A.POISSON_SOR, iterations=200,
                        omega=1.6, tolerance=1e-6, gdpt_flags=0):
    """screened_poisson_reconstruct on the GPU for (H, W, 3) float32 films.
    Returns (image, fp64 relative residual or -1 for SOR)."""
    h, w, _ = primal.shape
    p = np.ascontiguousarray(primal, np.float32)
    x = np.ascontiguousarray(grad_x, np.float32)
    y = np.ascontiguousarray(grad_y, np.float32)
    out = np.empty_like(p)
    cfg = integrator_cfg(A.INTEGRATOR_GDPT, alpha=alpha, poisson_iterations=iterations, sor_omega=omega,
                         poisson_solver=solver, poisson_tolerance=tolerance, gdpt_flags=gdpt_flags)
    res = C.c_double(0.0)
    check(lib().ar_poisson_reconstruct(ctx.handle, C.byref(cfg), w, h, p.ctypes.data, x.ctypes.data, y.ctypes.data,
                                       out.ctypes.data, 0, C.byref(res)))
    return out, res.value
