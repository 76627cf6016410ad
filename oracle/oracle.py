"""ctypes binding of the CPU restatement oracle (oracle/_build/liboracle_agentray.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py, to check and to time against; never
by the product path.

PARITY UNPINNED: agent-ray is Rust, has no tests or golden vectors, and cannot
be built here; the oracle is a line-by-line C++ restatement (see ar_*.hpp).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle_agentray.so")

SAMPLER_XOSHIRO = 0
SAMPLER_COUNTER = 1

_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lb = C.CDLL(LIB_PATH)
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        lb.oracle_scene_create.argtypes = [vp, C.c_int, C.POINTER(vp)]
        lb.oracle_scene_destroy.argtypes = [vp]
        lb.oracle_scene_destroy.restype = None
        lb.oracle_trace.argtypes = [vp, vp, vp, u64, C.c_int, vp, vp, vp, vp, vp, vp, vp, u32]
        lb.oracle_render.argtypes = [vp, vp, vp, u32, u32, u32, u32, vp, vp, vp, vp]
        lb.oracle_poisson_sor_f32.argtypes = [u32, u32, vp, vp, vp, C.c_float, u32, C.c_float, vp]
        lb.oracle_poisson_exact_f64.argtypes = [u32, u32, vp, vp, vp, C.c_double, C.c_double, u32, vp, vp]
        lb.oracle_counter_u01.argtypes = [u64, u32, u32, u32, u32, vp]
        lb.oracle_xoshiro_f32.argtypes = [u32, u32, u32, vp]
        lb.oracle_sincos_f32.argtypes = [vp, u64, vp, vp]
        lb.oracle_blas_stats.argtypes = [vp, u32, vp]
        lb.oracle_film_to_rgb8.argtypes = [vp, u32, u32, u32, C.c_float, C.c_float, C.c_float, vp]
        lb.oracle_texture_sample.argtypes = [vp, u32, u32, vp, u32, vp]
        _lib = lb
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


class OracleScene:
    def __init__(self, scene_data, precision=32):
        self.precision = precision
        desc, keep = scene_data.desc()
        self.h = C.c_void_p()
        lib().oracle_scene_create(C.addressof(desc), precision, C.byref(self.h))
        del keep

    def close(self):
        if self.h:
            lib().oracle_scene_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def trace_closest(self, org_tmin, dir_tmax, threads=0, stats=False):
        n = org_tmin.shape[0]
        ot = np.ascontiguousarray(org_tmin, np.float32)
        dt = np.ascontiguousarray(dir_tmax, np.float32)
        t = np.empty(n, np.float32)
        u = np.empty(n, np.float32)
        v = np.empty(n, np.float32)
        prim = np.empty(n, np.uint32)
        inst = np.empty(n, np.uint32)
        st = np.zeros(3, np.uint64) if stats else None
        lib().oracle_trace(self.h, _p(ot), _p(dt), n, 0, _p(t), _p(u), _p(v), _p(prim), _p(inst), None, _p(st),
                           threads)
        out = dict(t=t, u=u, v=v, prim=prim, inst=inst)
        if stats:
            out["stats"] = dict(nodes=int(st[0]), tris=int(st[1]), instances=int(st[2]))
        return out

    def trace_any(self, org_tmin, dir_tmax, threads=0):
        n = org_tmin.shape[0]
        ot = np.ascontiguousarray(org_tmin, np.float32)
        dt = np.ascontiguousarray(dir_tmax, np.float32)
        occ = np.empty(n, np.uint8)
        lib().oracle_trace(self.h, _p(ot), _p(dt), n, 1, None, None, None, None, None, _p(occ), None, threads)
        return occ

    def render(self, camera, cfg, width, height, sampler=SAMPLER_COUNTER, threads=0, moments=False, gdpt_films=False):
        """Returns the (H, W, 3) float64 image; with moments=True also the per-pixel
        mean squared sample radiance (PT) or, for GDPT, with gdpt_films=True the
        (primal, dx, dy) films."""
        cam = camera.desc()
        n = width * height * 3
        out = np.empty(n, np.float64)
        a0 = np.empty(n, np.float64) if (moments or gdpt_films) else None
        a1 = np.empty(n, np.float64) if gdpt_films else None
        a2 = np.empty(n, np.float64) if gdpt_films else None
        rc = lib().oracle_render(self.h, C.addressof(cam), C.addressof(cfg), width, height, sampler, threads,
                                 _p(out), _p(a0), _p(a1), _p(a2))
        if rc != 0:
            raise RuntimeError("oracle_render failed")
        img = out.reshape(height, width, 3)
        if gdpt_films:
            return img, a0.reshape(height, width, 3), a1.reshape(height, width, 3), a2.reshape(height, width, 3)
        if moments:
            return img, a0.reshape(height, width, 3)
        return img

    def blas_stats(self, mesh=0):
        o = np.zeros(3, np.uint64)
        lib().oracle_blas_stats(self.h, mesh, _p(o))
        return dict(nodes=int(o[0]), leaves=int(o[1]), depth=int(o[2]))


def poisson_sor_f32(primal, gx, gy, alpha, iters, omega):
    h, w, _ = primal.shape
    p = np.ascontiguousarray(primal, np.float32)
    x = np.ascontiguousarray(gx, np.float32)
    y = np.ascontiguousarray(gy, np.float32)
    out = np.empty_like(p)
    lib().oracle_poisson_sor_f32(w, h, _p(p), _p(x), _p(y), alpha, iters, omega, _p(out))
    return out


def poisson_exact_f64(primal, gx, gy, alpha, tol=1e-12, max_iters=10000):
    h, w, _ = primal.shape
    p = np.ascontiguousarray(primal, np.float64)
    x = np.ascontiguousarray(gx, np.float64)
    y = np.ascontiguousarray(gy, np.float64)
    out = np.empty_like(p)
    rr = np.zeros(1, np.float64)
    lib().oracle_poisson_exact_f64(w, h, _p(p), _p(x), _p(y), alpha, tol, max_iters, _p(out), _p(rr))
    return out, float(rr[0])


def counter_u01(seed, pixel, sample, dim0, n):
    out = np.empty(n, np.float32)
    lib().oracle_counter_u01(seed, pixel, sample, dim0, n, _p(out))
    return out


def xoshiro_f32(px, py, n):
    out = np.empty(n, np.float32)
    lib().oracle_xoshiro_f32(px, py, n, _p(out))
    return out


def sincos_f32(x):
    """(sin, cos) of float32 angles as the FP32 oracle (and the kernels) compute them."""
    x = np.ascontiguousarray(x, np.float32)
    s = np.empty_like(x)
    c = np.empty_like(x)
    lib().oracle_sincos_f32(_p(x), x.size, _p(s), _p(c))
    return s, c


def film_to_rgb8(hdr, tone_mapper=0, white_point=1.0, gamma=2.2, scale=1.0):
    """Film::to_rgb_image on an (H, W, 3) float32 image -> (H, W, 3) uint8."""
    h, w, _ = hdr.shape
    x = np.ascontiguousarray(hdr, np.float32)
    out = np.empty((h, w, 3), np.uint8)
    lib().oracle_film_to_rgb8(_p(x), w, h, tone_mapper, white_point, gamma, scale, _p(out))
    return out



def texture_sample(rgb8, uv):
    """ImageTexture::sample of an (H, W, 3) uint8 sRGB image at (N, 2) uv -> (N, 3) float32."""
    img = np.ascontiguousarray(rgb8, np.uint8)
    q = np.ascontiguousarray(uv, np.float32).reshape(-1, 2)
    out = np.empty((q.shape[0], 3), np.float32)
    rc = lib().oracle_texture_sample(_p(img), img.shape[1], img.shape[0], _p(q), q.shape[0], _p(out))
    assert rc == 0
    return out


def f32_to_f16_bits(x):
    """half::f16::from_f32 on float32 values -> uint16 bits: IEEE round to
    nearest even; a NaN keeps its sign and top 10 mantissa bits with the quiet bit set."""
    x = np.asarray(x, np.float32)
    with np.errstate(over="ignore", invalid="ignore"):
        bits = x.astype(np.float16).view(np.uint16).copy()
    nan = np.isnan(x)
    if nan.any():
        b = x.view(np.uint32)[nan]
        bits[nan] = (((b >> 16) & 0x8000) | 0x7E00 | ((b & 0x7FFFFF) >> 13)).astype(np.uint16)
    return bits


def film_save_exr(hdr, path, scale=1.0):
    """Film::save_exr (src/film.rs:304-346) restated: (H, W, 3) float32 * scale
    as HALF B/G/R channels of a single-part scanline OpenEXR file, ZIP
    compression (16 scanlines per chunk; byte reorder, +128 delta predictor,
    zlib at the default level; a chunk deflate does not shrink is stored raw),
    attributes in name order, the layer named "beauty"."""
    import struct
    import zlib
    h, w, _ = hdr.shape
    with np.errstate(invalid="ignore"):
        v = f32_to_f16_bits(np.asarray(hdr, np.float32) * np.float32(scale))  # (H, W, 3)
    planar = np.ascontiguousarray(v[:, :, ::-1].transpose(0, 2, 1))  # (H, [B, G, R], W)

    def attr(name, typ, data):
        return name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(data)) + data
    ch = b"".join(c + b"\0" + struct.pack("<iIii", 1, 0, 1, 1) for c in (b"B", b"G", b"R")) + b"\0"
    box = struct.pack("<4i", 0, 0, w - 1, h - 1)
    head = (struct.pack("<II", 20000630, 2) + attr("channels", "chlist", ch) +
            attr("compression", "compression", b"\x03") + attr("dataWindow", "box2i", box) +
            attr("displayWindow", "box2i", box) + attr("lineOrder", "lineOrder", b"\x00") +
            attr("name", "string", b"beauty") + attr("pixelAspectRatio", "float", struct.pack("<f", 1.0)) +
            attr("screenWindowCenter", "v2f", struct.pack("<2f", 0.0, 0.0)) +
            attr("screenWindowWidth", "float", struct.pack("<f", 1.0)) + b"\0")
    chunks = []
    for y0 in range(0, h, 16):
        raw = planar[y0:y0 + 16].astype("<u2").tobytes()
        r = np.frombuffer(raw, np.uint8)
        t = np.concatenate([r[0::2], r[1::2]]).astype(np.int32)
        t[1:] = (t[1:] - t[:-1] + 384) & 0xFF
        z = zlib.compress(t.astype(np.uint8).tobytes(), 6)
        chunks.append((y0, z if len(z) < len(raw) else raw))
    offs, at = [], len(head) + 8 * len(chunks)
    for y0, d in chunks:
        offs.append(at)
        at += 8 + len(d)
    out = head + struct.pack("<%dQ" % len(offs), *offs) + b"".join(
        struct.pack("<ii", y0, len(d)) + d for y0, d in chunks)
    with open(path, "wb") as f:
        f.write(out)
