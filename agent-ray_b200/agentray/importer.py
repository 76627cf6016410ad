"""OBJ/MTL import (load_obj_scene, src/importer.rs:75-241) and PNG texture
decoding for ImageTexture::load (src/texture.rs:77-94).

The reference reads OBJ through `tobj` with GPU_LOAD_OPTIONS (triangulated,
one index per (position, texcoord, normal) triple, a model per object/group
and material) and converts each MTL material to a BSDF:
  d < 0.5                 -> DielectricBsdf(eta = max(Ni, 1), alpha)
  luminance(Ks) > 0.04    -> ConductorBsdf(f0 = Ks, alpha)
  map_Kd that loads       -> Lambertian with the ImageTexture
  otherwise               -> Lambertian(Kd, default 0.5)
with alpha = sqrt(2 / (Ns + 2)) clamped to [1e-3, 1].  Without an MTL every
model gets one grey Lambertian.  Textures decode here from PNG (8-bit gray,
gray+alpha, RGB or RGBA, non-interlaced); other formats fall back to Kd, as
the reference falls back when `image::open` fails.
"""
import os
import struct
import zlib

import numpy as np

from . import _abi as A
from .scene_data import Material, Mesh, Object


# ------------------------------------------------------------------- PNG --
def read_png(path):
    """Decodes an 8-bit non-interlaced PNG to an (H, W, 3) uint8 RGB array."""
    data = open(path, "rb").read()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG file")
    pos, idat, hdr = 8, [], None
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif tag == b"IDAT":
            idat.append(body)
        elif tag == b"IEND":
            break
        pos += 12 + n
    if hdr is None:
        raise ValueError("PNG without IHDR")
    w, h, depth, ctype, _, _, interlace = hdr
    channels = {0: 1, 2: 3, 4: 2, 6: 4}.get(ctype)
    if depth != 8 or channels is None or interlace != 0:
        raise ValueError(f"unsupported PNG (depth {depth}, colour type {ctype}, interlace {interlace})")
    raw = zlib.decompress(b"".join(idat))
    stride = w * channels
    out = np.zeros((h, stride), np.uint8)
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        f = raw[y * (stride + 1)]
        line = np.frombuffer(raw, np.uint8, stride, y * (stride + 1) + 1).astype(np.int32)
        if f in (0, 1, 2):  # none / sub / up reconstruct without a scalar loop
            if f == 1:
                cur = np.cumsum(line.reshape(w, channels), axis=0).reshape(stride) & 0xFF
            else:
                cur = (line + (prev if f == 2 else 0)) & 0xFF
            out[y] = cur
            prev = cur
            continue
        # average / Paeth depend on the reconstructed left neighbour: a scalar
        # loop over Python ints (several times faster than numpy scalars)
        ln, up, cur = line.tolist(), prev.tolist(), [0] * stride
        for x in range(stride):
            a = cur[x - channels] if x >= channels else 0
            b = up[x]
            if f == 3:
                p = (a + b) >> 1
            elif f == 4:
                c = up[x - channels] if x >= channels else 0
                pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            else:
                raise ValueError(f"bad PNG filter {f}")
            cur[x] = (ln[x] + p) & 0xFF
        cur = np.array(cur, np.int32)
        out[y] = cur
        prev = cur
    px = out.reshape(h, w, channels)
    if channels == 1:
        return np.repeat(px, 3, axis=2)
    if channels == 2:
        return np.repeat(px[:, :, :1], 3, axis=2)
    return np.ascontiguousarray(px[:, :, :3])


# ------------------------------------------------------------------- MTL --
def ns_to_roughness(ns):
    """importer.rs:86-88: alpha = sqrt(2 / (Ns + 2)), clamped to [1e-3, 1]."""
    a = np.sqrt(np.float32(2.0) / (np.float32(ns) + np.float32(2.0)), dtype=np.float32)
    return float(min(max(a, np.float32(1e-3)), np.float32(1.0)))


def _luminance(c):
    return 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]


def parse_mtl(path):
    """The MTL statements the reference's conversion reads, as tobj parses them
    (Kd, Ks, Ns, Ni, d, map_Kd; `Tr` is not read, so only `d` makes a
    material transparent)."""
    mats, cur = {}, None
    for raw in open(path, encoding="utf-8", errors="replace"):
        t = raw.strip().split()
        if not t or t[0].startswith("#"):
            continue
        key, args = t[0], t[1:]
        if key == "newmtl":
            cur = {"name": " ".join(args)}
            mats[cur["name"]] = cur
        elif cur is None:
            continue
        elif key in ("Kd", "Ks"):
            cur[key] = [float(x) for x in args[:3]]
        elif key in ("Ns", "Ni", "d"):
            cur[key] = float(args[0])
        elif key == "map_Kd":  # the rest of the line, as tobj reads it
            cur["map_Kd"] = raw.strip()[len("map_Kd"):].strip()
    return mats


def convert_material(m, base_dir, scene):
    """importer.rs:99-151: one MTL material -> a Material of `scene`."""
    ks = m.get("Ks", [0.0, 0.0, 0.0])
    ns = max(m.get("Ns", 0.0), 0.0)
    d = m.get("d", 1.0)
    ni = max(m.get("Ni", 1.5), 1.0)
    rough = ns_to_roughness(ns)
    if d < 0.5:
        return Material(A.MATERIAL_DIELECTRIC, roughness=rough, eta=ni)
    if _luminance(ks) > 0.04:
        return Material(A.MATERIAL_CONDUCTOR, f0=tuple(ks), roughness=rough)
    if "map_Kd" in m:
        try:
            tex = scene.add_texture(read_png(os.path.join(base_dir, m["map_Kd"].replace("\\", "/"))))
            return Material(A.MATERIAL_LAMBERTIAN, albedo_texture=tex)
        except (OSError, ValueError):
            pass  # the reference also falls back to the constant colour
    return Material(A.MATERIAL_LAMBERTIAN, albedo=tuple(m.get("Kd", [0.5, 0.5, 0.5])))


# ------------------------------------------------------------------- OBJ --
def _models(path):
    """Faces grouped into models (per o/g and per material), tobj-style."""
    v, vt, vn = [], [], []
    models, mtllib = [], None
    cur = {"name": "", "mat": None, "faces": []}

    def new_model(name=None, mat=None):
        nonlocal cur
        if cur["faces"]:
            models.append(cur)
        cur = {"name": cur["name"] if name is None else name, "mat": mat, "faces": []}

    def idx(s, n):
        i = int(s)
        return i - 1 if i > 0 else n + i
    for raw in open(path, encoding="utf-8", errors="replace"):
        t = raw.strip().split()
        if not t or t[0].startswith("#"):
            continue
        key, args = t[0], t[1:]
        if key == "v":
            v.append([float(x) for x in args[:3]])
        elif key == "vt":
            vt.append([float(x) for x in args[:2]])
        elif key == "vn":
            vn.append([float(x) for x in args[:3]])
        elif key == "f":
            corners = []
            for a in args:
                if "/" not in a:  # position only
                    corners.append((idx(a, len(v)), -1, -1))
                    continue
                p = a.split("/")
                corners.append((idx(p[0], len(v)), idx(p[1], len(vt)) if len(p) > 1 and p[1] else -1,
                                idx(p[2], len(vn)) if len(p) > 2 and p[2] else -1))
            for k in range(1, len(corners) - 1):  # fan triangulation
                cur["faces"].append((corners[0], corners[k], corners[k + 1]))
        elif key in ("o", "g"):
            new_model(name=" ".join(args), mat=cur["mat"])
        elif key == "usemtl":
            new_model(mat=" ".join(args))
        elif key == "mtllib":
            mtllib = " ".join(args)
    new_model()
    return np.array(v, np.float32), np.array(vt, np.float32), np.array(vn, np.float32), models, mtllib


def load_obj_scene(scene, path, transform=None):
    """Adds the OBJ file's models to `scene` as objects placed by `transform`
    (4x4 row-major, default identity); returns the new object indices."""
    base = os.path.dirname(os.path.abspath(path))
    v, vt, vn, models, mtllib = _models(path)
    names, mat_ids = [], []
    if mtllib and os.path.exists(os.path.join(base, mtllib)):
        mtl = parse_mtl(os.path.join(base, mtllib))
        for name, m in mtl.items():
            names.append(name)
            mat_ids.append(scene.add_material(convert_material(m, base, scene)))
    if not mat_ids:
        names, mat_ids = [None], [scene.add_material(Material(A.MATERIAL_LAMBERTIAN, albedo=(0.5, 0.5, 0.5)))]
    xf = np.eye(4, dtype=np.float32) if transform is None else np.asarray(transform, np.float32)
    inv = np.linalg.inv(xf.astype(np.float64)).astype(np.float32)
    objects = []
    for mdl in models:
        c = np.asarray(mdl["faces"], np.int64).reshape(-1, 3)  # corners: (v, vt, vn), -1 = absent
        has_uv = len(vt) > 0 and bool((c[:, 1] >= 0).all())
        has_n = len(vn) > 0 and bool((c[:, 2] >= 0).all())
        key = c.copy()
        if not has_uv:
            key[:, 1] = -1
        if not has_n:
            key[:, 2] = -1
        # single index per distinct (v, vt, vn), numbered in order of first use
        uniq, first, inverse = np.unique(key, axis=0, return_index=True, return_inverse=True)
        order = np.argsort(first, kind="stable")
        rank = np.empty(len(order), np.int64)
        rank[order] = np.arange(len(order))
        tris = rank[inverse.reshape(-1)].reshape(-1, 3)
        corner = uniq[order]
        pos = v[corner[:, 0]]
        uv = vt[corner[:, 1]] if has_uv else None
        nrm = vn[corner[:, 2]] if has_n else None
        slot = names.index(mdl["mat"]) if mdl["mat"] in names else 0
        mesh = Mesh(np.ascontiguousarray(pos, np.float32), tris.astype(np.uint32),
                    normals=None if nrm is None else np.ascontiguousarray(nrm, np.float32),
                    material_slots=np.array([slot], np.uint32),
                    tex_coords=None if uv is None else np.ascontiguousarray(uv, np.float32))
        objects.append(scene.add_object(Object(scene.add_mesh(mesh), list(mat_ids), xf, inv)))
    return objects
