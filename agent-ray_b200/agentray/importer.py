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
model gets one grey Lambertian.  Textures decode here from PNG (every colour
type, bit depth and interlace mode); other formats fall back to Kd, as the
reference falls back when `image::open` fails.
"""
import os
import struct
import zlib

import numpy as np

from . import _abi as A
from .scene_data import Material, Mesh, Object


# ------------------------------------------------------------------- PNG --
_ADAM7 = ((0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2))


def _unfilter(raw, pos, rows, stride, bpp):
    """Reverses the PNG row filters of `rows` rows of `stride` bytes starting
    at raw[pos]; bpp = bytes per complete pixel (at least 1).  Returns the
    (rows, stride) uint8 array and the position after the last row."""
    out = np.zeros((rows, stride), np.uint8)
    prev = np.zeros(stride, np.int32)
    for y in range(rows):
        f = raw[pos]
        line = np.frombuffer(raw, np.uint8, stride, pos + 1).astype(np.int32)
        pos += stride + 1
        if f in (0, 1, 2):  # none / sub / up reconstruct without a scalar loop
            if f == 1:
                if stride % bpp == 0:
                    cur = np.cumsum(line.reshape(-1, bpp), axis=0).reshape(stride) & 0xFF
                else:
                    cur = line.copy()
                    for x in range(bpp, stride):
                        cur[x] = (cur[x] + cur[x - bpp]) & 0xFF
            else:
                cur = (line + (prev if f == 2 else 0)) & 0xFF
            out[y] = cur
            prev = cur
            continue
        # average / Paeth depend on the reconstructed left neighbour: a scalar
        # loop over Python ints (several times faster than numpy scalars)
        ln, up, cur = line.tolist(), prev.tolist(), [0] * stride
        for x in range(stride):
            a = cur[x - bpp] if x >= bpp else 0
            b = up[x]
            if f == 3:
                p = (a + b) >> 1
            elif f == 4:
                c = up[x - bpp] if x >= bpp else 0
                pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            else:
                raise ValueError(f"bad PNG filter {f}")
            cur[x] = (ln[x] + p) & 0xFF
        cur = np.array(cur, np.int32)
        out[y] = cur
        prev = cur
    return out, pos


def _samples(rows, w, channels, depth):
    """Unpacked samples (h, w, channels) of unfiltered rows (uint16 for depth 16)."""
    h = rows.shape[0]
    if depth == 8:
        return rows[:, :w * channels].reshape(h, w, channels)
    if depth == 16:
        return (rows[:, :2 * w * channels].astype(np.uint16).reshape(h, w * channels, 2) *
                np.array([256, 1], np.uint16)).sum(axis=2, dtype=np.uint16).reshape(h, w, channels)
    bits = np.unpackbits(rows, axis=1)[:, :w * channels * depth].reshape(h, w * channels, depth)
    weights = (1 << np.arange(depth - 1, -1, -1)).astype(np.uint8)
    return (bits * weights).sum(axis=2, dtype=np.uint8).reshape(h, w, channels)


def read_png(path):
    """Decodes a PNG (grey, grey+alpha, RGB, RGBA or palette; 1-16 bits per
    sample; plain or Adam7-interlaced) to an (H, W, 3) uint8 RGB array, as
    ImageTexture::load's `image::open(..).into_rgb8()` does: alpha dropped,
    grey replicated, sub-8-bit grey scaled to 0..255, 16-bit samples rounded
    to the nearest 8-bit value (v / 257)."""
    data = open(path, "rb").read()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG file")
    pos, idat, hdr, plte = 8, [], None, None
    while pos + 8 <= len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif tag == b"PLTE":
            plte = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif tag == b"IDAT":
            idat.append(body)
        elif tag == b"IEND":
            break
        pos += 12 + n
    if hdr is None:
        raise ValueError("PNG without IHDR")
    w, h, depth, ctype, _, _, interlace = hdr
    channels = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}.get(ctype)
    allowed = {0: (1, 2, 4, 8, 16), 2: (8, 16), 3: (1, 2, 4, 8), 4: (8, 16), 6: (8, 16)}
    if channels is None or depth not in allowed[ctype] or interlace not in (0, 1) or w == 0 or h == 0:
        raise ValueError(f"unsupported PNG (depth {depth}, colour type {ctype}, interlace {interlace})")
    if ctype == 3 and plte is None:
        raise ValueError("palette PNG without PLTE")
    raw = zlib.decompress(b"".join(idat))
    bpp = max(1, channels * depth // 8)
    if interlace == 0:
        rows, _ = _unfilter(raw, 0, h, (w * channels * depth + 7) // 8, bpp)
        px = _samples(rows, w, channels, depth)
    else:  # Adam7: seven sub-images, each filtered on its own
        px = np.zeros((h, w, channels), np.uint16 if depth == 16 else np.uint8)
        pos = 0
        for x0, y0, dx, dy in _ADAM7:
            pw, ph = (w - x0 + dx - 1) // dx, (h - y0 + dy - 1) // dy
            if pw <= 0 or ph <= 0:
                continue
            rows, pos = _unfilter(raw, pos, ph, (pw * channels * depth + 7) // 8, bpp)
            px[y0::dy, x0::dx] = _samples(rows, pw, channels, depth)
    if ctype == 3:
        idx = px[:, :, 0].astype(np.int64)
        if idx.max() >= plte.shape[0]:
            raise ValueError("palette index out of range")
        return np.ascontiguousarray(plte[idx])
    if depth == 16:
        px = ((px.astype(np.uint32) * 255 + 32767) // 65535).astype(np.uint8)
    elif depth < 8:
        px = (px.astype(np.uint16) * 255 // ((1 << depth) - 1)).astype(np.uint8)
    if channels <= 2:
        return np.ascontiguousarray(np.repeat(px[:, :, :1], 3, axis=2))
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


def _mesh_of(mdl, v, vt, vn, slot):
    """One model as a Mesh with a single material slot (tobj GPU_LOAD_OPTIONS:
    triangulated, one index per distinct (position, texcoord, normal))."""
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
    return Mesh(np.ascontiguousarray(pos, np.float32), tris.astype(np.uint32),
                normals=None if nrm is None else np.ascontiguousarray(nrm, np.float32),
                material_slots=np.array([slot], np.uint32),
                tex_coords=None if uv is None else np.ascontiguousarray(uv, np.float32))


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
        slot = names.index(mdl["mat"]) if mdl["mat"] in names else 0
        mesh = _mesh_of(mdl, v, vt, vn, slot)
        objects.append(scene.add_object(Object(scene.add_mesh(mesh), list(mat_ids), xf, inv)))
    return objects


def load_obj_meshes(path):
    """TriangleMesh::load_obj (src/primitives/mesh.rs:19-73): the OBJ file's
    models as meshes; each mesh's one material slot is its model's index in
    the MTL file's material list (0 without one)."""
    base = os.path.dirname(os.path.abspath(path))
    v, vt, vn, models, mtllib = _models(path)
    names = []
    if mtllib and os.path.exists(os.path.join(base, mtllib)):
        names = list(parse_mtl(os.path.join(base, mtllib)).keys())
    return [_mesh_of(m, v, vt, vn, names.index(m["mat"]) if m["mat"] in names else 0) for m in models]
