"""ImageTexture (src/texture.rs:65-151) and the OBJ/MTL importer
(src/importer.rs:75-241): the oracle's texture sampling against a numpy
restatement, the PNG decoder against every filter type, and the importer's
triangulation, single-index remap, model split and material rules."""
import os
import struct
import zlib

import numpy as np
import pytest

import oracle as O
import agentray.scenes as S
from agentray import _abi as A
from agentray import importer as I
from agentray.scene_data import SceneData


def _np_srgb_to_linear(x):
    x = x.astype(np.float32)
    lo = x / np.float32(12.92)
    hi = np.power((x + np.float32(0.055)) / np.float32(1.055), np.float32(2.4), dtype=np.float32)
    return np.where(x <= np.float32(0.04045), lo, hi).astype(np.float32)


def _np_texture_sample(img, uv):
    """texture.rs:100-136 restated in numpy (float64 math, f32 inputs)."""
    h, w, _ = img.shape
    lin = _np_srgb_to_linear(img.astype(np.float32) / np.float32(255.0)).astype(np.float64)
    f = uv - np.trunc(uv)
    r = np.fmod(f, 1.0)
    r = np.where(r < 0, r + 1.0, r)
    u = r[:, 0] * w - 0.5
    v = r[:, 1] * h - 0.5
    x0, y0 = np.floor(u).astype(np.int64), np.floor(v).astype(np.int64)
    tx, ty = (u - np.floor(u))[:, None], (v - np.floor(v))[:, None]

    def fetch(x, y):
        return lin[np.mod(y, h), np.mod(x, w)]
    return (fetch(x0, y0) * (1 - tx) * (1 - ty) + fetch(x0 + 1, y0) * tx * (1 - ty) +
            fetch(x0, y0 + 1) * (1 - tx) * ty + fetch(x0 + 1, y0 + 1) * tx * ty)


def test_oracle_texture_sample_matches_numpy_restatement():
    rng = np.random.default_rng(11)
    img = rng.integers(0, 256, (5, 7, 3), dtype=np.uint8)
    uv = np.concatenate([rng.uniform(-3.0, 3.0, (2000, 2)),
                         np.array([[0, 0], [1, 1], [-1, -1], [0.5, 0.5], [-1e-9, 2.0], [0.999999, -0.25]])])
    uv = uv.astype(np.float32)
    got = O.texture_sample(img, uv)
    ref = _np_texture_sample(img, uv.astype(np.float64))
    assert np.abs(got - ref).max() < 2e-5


def test_oracle_texture_texel_centres_are_exact_linear_values():
    img = S.checker_texture(8, 4, seed=2)
    y, x = np.mgrid[0:8, 0:8]
    uv = np.stack([(x.ravel() + 0.5) / 8, (y.ravel() + 0.5) / 8], 1).astype(np.float32)
    got = O.texture_sample(img, uv).reshape(8, 8, 3)
    np.testing.assert_allclose(got, _np_srgb_to_linear(img / np.float32(255.0)), rtol=0, atol=1e-6)


def _png_bytes(img, filters):
    """An 8-bit RGB PNG whose row y uses filter type filters[y % len]."""
    h, w, c = img.shape
    bpp, rows = c, []
    prev = np.zeros(w * c, np.int32)
    for y in range(h):
        line = img[y].reshape(-1).astype(np.int32)
        f = filters[y % len(filters)]
        enc = np.zeros_like(line)
        for x in range(w * c):
            a = line[x - bpp] if x >= bpp else 0
            b = prev[x]
            cc = prev[x - bpp] if x >= bpp else 0
            if f == 0:
                p = 0
            elif f == 1:
                p = a
            elif f == 2:
                p = b
            elif f == 3:
                p = (a + b) // 2
            else:
                pa, pb, pc = abs(b - cc), abs(a - cc), abs(a + b - 2 * cc)
                p = a if pa <= pb and pa <= pc else (b if pb <= pc else cc)
            enc[x] = (line[x] - p) & 0xFF
        rows.append(bytes([f]) + enc.astype(np.uint8).tobytes())
        prev = line

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)
    ctype = {1: 0, 2: 4, 3: 2, 4: 6}[c]
    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, ctype, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(b"".join(rows))) + chunk(b"IEND", b""))


@pytest.mark.parametrize("channels", [1, 2, 3, 4])
def test_png_decoder_all_filters(tmp_path, channels):
    rng = np.random.default_rng(channels)
    img = rng.integers(0, 256, (10, 9, channels), dtype=np.uint8)
    p = tmp_path / "t.png"
    p.write_bytes(_png_bytes(img, [0, 1, 2, 3, 4]))
    got = I.read_png(str(p))
    want = (np.repeat(img[:, :, :1], 3, axis=2) if channels <= 2 else img[:, :, :3])
    np.testing.assert_array_equal(got, want)


def test_png_writer_round_trip(tmp_path):
    import agentray
    img = S.checker_texture(12, 3, seed=4)
    agentray.write_png(str(tmp_path / "c.png"), img)
    np.testing.assert_array_equal(I.read_png(str(tmp_path / "c.png")), img)


def test_ns_to_roughness():
    # the crate's design notes: Ns=0 -> alpha=1 (rough), Ns=1000 -> alpha~0.044
    assert I.ns_to_roughness(1000.0) == pytest.approx(0.044, abs=1e-3)
    assert I.ns_to_roughness(0.0) == 1.0
    assert I.ns_to_roughness(1e9) == pytest.approx(1e-3)  # clamped at the low end
    assert I.ns_to_roughness(98.0) == pytest.approx(np.sqrt(2.0 / 100.0), rel=1e-6)


MTL = """# materials
newmtl glass
Kd 0.9 0.9 0.9
d 0.2
Ni 1.45
Ns 200
newmtl metal
Ks 0.9 0.6 0.3
Ns 50
newmtl tex
Kd 0.1 0.2 0.3
map_Kd sub\\checker.png
newmtl broken
Kd 0.3 0.4 0.5
map_Kd missing.png
newmtl plain
Kd 0.25 0.5 0.75
Ks 0.01 0.01 0.01
newmtl lowni
d 0.1
Ni 0.5
newmtl tr_only
Tr 0.9
Kd 0.2 0.2 0.2
"""

OBJ = """mtllib scene.mtl
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v 0.5 1.5 0
vt 0 0
vt 1 0
vt 1 1
vt 0 1
vn 0 0 1
o quad
usemtl tex
f 1/1/1 2/2/1 3/3/1 4/4/1
usemtl metal
f -5/1/1 -3/3/1 -1/4/1
o penta
usemtl plain
f 1 2 3 5 4
g other
usemtl nosuch
f 1 2 3
"""


def test_material_rules(tmp_path):
    (tmp_path / "sub").mkdir()
    import agentray
    agentray.write_png(str(tmp_path / "sub" / "checker.png"), S.checker_texture(4, 2))
    (tmp_path / "scene.mtl").write_text(MTL)
    sc = SceneData()
    mats = {}
    for name, m in I.parse_mtl(str(tmp_path / "scene.mtl")).items():
        mats[name] = sc.materials[sc.add_material(I.convert_material(m, str(tmp_path), sc))]
    assert mats["glass"].kind == A.MATERIAL_DIELECTRIC and mats["glass"].eta == pytest.approx(1.45)
    assert mats["glass"].roughness == pytest.approx(np.sqrt(2.0 / 202.0), rel=1e-6)
    assert mats["metal"].kind == A.MATERIAL_CONDUCTOR and mats["metal"].f0 == pytest.approx((0.9, 0.6, 0.3))
    assert mats["tex"].kind == A.MATERIAL_LAMBERTIAN and mats["tex"].albedo_texture == 0
    np.testing.assert_array_equal(sc.textures[0], S.checker_texture(4, 2))
    assert mats["broken"].albedo_texture == -1 and mats["broken"].albedo == pytest.approx((0.3, 0.4, 0.5))
    assert mats["plain"].kind == A.MATERIAL_LAMBERTIAN and mats["plain"].albedo == pytest.approx((0.25, 0.5, 0.75))
    assert mats["lowni"].kind == A.MATERIAL_DIELECTRIC and mats["lowni"].eta == 1.0  # Ni clamped to >= 1
    assert mats["tr_only"].kind == A.MATERIAL_LAMBERTIAN  # tobj does not read Tr


def test_load_obj_scene_structure(tmp_path):
    import agentray
    (tmp_path / "sub").mkdir()
    agentray.write_png(str(tmp_path / "sub" / "checker.png"), S.checker_texture(4, 2))
    (tmp_path / "scene.mtl").write_text(MTL)
    (tmp_path / "scene.obj").write_text(OBJ)
    sc = SceneData()
    xf = np.eye(4, dtype=np.float32)
    xf[:3, 3] = [1.0, 2.0, 3.0]
    objs = I.load_obj_scene(sc, str(tmp_path / "scene.obj"), xf)
    assert len(objs) == 4 and len(sc.materials) == 7 and len(sc.textures) == 1
    meshes = [sc.meshes[sc.objects[o].mesh] for o in objs]
    # model 0: the quad fan-triangulated, uv and normals kept, 4 unique (v, vt, vn)
    m0 = meshes[0]
    assert m0.indices.tolist() == [[0, 1, 2], [0, 2, 3]]
    assert m0.tex_coords.shape == (4, 2) and m0.normals.shape == (4, 3)
    assert int(m0.material_slots[0]) == 2  # "tex" is the third MTL material
    # model 1: negative indices resolve against the vertices read so far
    m1 = meshes[1]
    np.testing.assert_array_equal(m1.positions, np.array([[0, 0, 0], [1, 1, 0], [0.5, 1.5, 0]], np.float32))
    assert int(m1.material_slots[0]) == 1
    # model 2: pentagon -> 3 fan triangles, no uv / normals
    m2 = meshes[2]
    assert m2.num_triangles == 3 and m2.tex_coords is None and m2.normals is None
    assert int(m2.material_slots[0]) == 4
    # model 3: unknown material -> slot 0
    assert int(meshes[3].material_slots[0]) == 0
    for o in objs:
        np.testing.assert_allclose(sc.objects[o].transform, xf)
        np.testing.assert_allclose(sc.objects[o].inv_transform @ xf, np.eye(4), atol=1e-6)
        assert sc.objects[o].materials == list(range(7))


def test_load_obj_without_mtl_is_grey(tmp_path):
    (tmp_path / "a.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    sc = SceneData()
    objs = I.load_obj_scene(sc, str(tmp_path / "a.obj"))
    assert len(objs) == 1 and len(sc.materials) == 1
    assert sc.materials[0].kind == A.MATERIAL_LAMBERTIAN and sc.materials[0].albedo == (0.5, 0.5, 0.5)


def test_imported_cornell_renders_like_builtin(tmp_path):
    # The Cornell box written out as OBJ/MTL (one object per wall/box, its
    # material by usemtl) and imported renders to the same image in the
    # oracle as the built-in scene it came from.
    sc, cam = S.cornell_box(1)
    mtl, obj, nv = [], ["mtllib box.mtl"], 0
    emitters = []
    for k, o in enumerate(sc.objects):
        m = sc.materials[o.materials[0]]
        if m.emitter_light >= 0:  # the quad light's emitting surface stays as it is
            emitters.append(o)
            continue
        mtl += [f"newmtl m{k}", "Kd %r %r %r" % tuple(float(x) for x in m.albedo)]
        me = sc.meshes[o.mesh]
        p = np.c_[me.positions, np.ones(len(me.positions), np.float32)] @ o.transform.T
        obj.append(f"o obj{k}")
        obj.append(f"usemtl m{k}")
        obj += ["v %r %r %r" % tuple(float(np.float32(c)) for c in q[:3]) for q in p]
        obj += ["f %d %d %d" % tuple(int(i) + 1 + nv for i in t) for t in me.indices]
        nv += len(me.positions)
    (tmp_path / "box.mtl").write_text("\n".join(mtl) + "\n")
    (tmp_path / "box.obj").write_text("\n".join(obj) + "\n")
    imp = SceneData(sc.light_distribution)
    I.load_obj_scene(imp, str(tmp_path / "box.obj"))
    for l in sc.lights:
        imp.add_light(l)
    for o in emitters:
        from agentray.scene_data import Object
        imp.add_object(Object(imp.add_mesh(sc.meshes[o.mesh]), [imp.add_material(sc.materials[o.materials[0]])],
                              o.transform, o.inv_transform))
    from agentray.scene_data import integrator_cfg
    cfg = integrator_cfg(A.INTEGRATOR_PT, spp=4, max_depth=5, seed=3)
    a = O.OracleScene(sc).render(cam, cfg, 24, 24)
    b = O.OracleScene(imp).render(cam, cfg, 24, 24)
    # the built-in boxes are instanced with transforms, the imported ones baked
    # into world space: intersections agree to rounding, not bit for bit
    assert abs(a.mean() - b.mean()) / a.mean() < 2e-2
    close = np.abs(a - b) <= 1e-3 * np.maximum(1.0, np.abs(a))
    assert close.all(axis=2).mean() > 0.9


# The reference checkout's assets/fireplace_room folder, named by the
# AGENTRAY_FIREPLACE_DIR environment variable; the test skips when it is unset.
FIREPLACE = os.environ.get("AGENTRAY_FIREPLACE_DIR", "")


@pytest.mark.skipif(not (FIREPLACE and os.path.isdir(FIREPLACE)),
                    reason="AGENTRAY_FIREPLACE_DIR does not name the reference's fireplace_room asset folder")
def test_fireplace_mtl_and_textures():
    # The reference's own asset (its OBJ is not shipped): every MTL material
    # converts, and each map_Kd PNG decodes to the same pixels as OpenCV's
    # decoder gives.
    cv2 = pytest.importorskip("cv2")
    sc = SceneData()
    mtl = I.parse_mtl(os.path.join(FIREPLACE, "fireplace_room.mtl"))
    assert len(mtl) == 22
    kinds = {}
    for name, m in mtl.items():
        kinds[name] = sc.materials[sc.add_material(I.convert_material(m, FIREPLACE, sc))].kind
    assert kinds["grey_and_white_room:BrushedStainlessSteel"] == A.MATERIAL_CONDUCTOR
    assert kinds["grey_and_white_room:Floor"] == A.MATERIAL_LAMBERTIAN
    textured = [m for m in mtl.values() if "map_Kd" in m]
    assert len(sc.textures) == len(textured) > 0
    for m, img in zip(textured, sc.textures):
        ref = cv2.imread(os.path.join(FIREPLACE, m["map_Kd"].replace("\\", "/")), cv2.IMREAD_COLOR)[:, :, ::-1]
        np.testing.assert_array_equal(img, ref)


def test_obj_normals_without_uv_and_ignored_statements(tmp_path):
    # `f v//vn` keeps normals without uv; points, lines, smoothing groups and
    # degenerate faces (< 3 corners) make no triangles (GPU_LOAD_OPTIONS
    # ignores points and lines).
    (tmp_path / "n.obj").write_text(
        "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nvn 0 0 1\nvn 0 0 -1\n"
        "s 1\np 1\nl 1 2\nf 1//1 2//1 3//1\nf 2//2 4//2 3//2\nf 1 2\n")
    sc = SceneData()
    objs = I.load_obj_scene(sc, str(tmp_path / "n.obj"))
    assert len(objs) == 1
    m = sc.meshes[sc.objects[objs[0]].mesh]
    assert m.num_triangles == 2 and m.tex_coords is None
    # vertex 2 and 3 appear with two different normals -> split (single index)
    assert m.positions.shape[0] == 6 and m.normals.shape == (6, 3)
    np.testing.assert_array_equal(m.normals[m.indices[1]], np.array([[0, 0, -1]] * 3, np.float32))


_ADAM7 = ((0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2))


def _pack_rows(samples, depth):
    """(h, w, c) integer samples -> list of packed scanline bytes (big-endian)."""
    h = samples.shape[0]
    flat = samples.reshape(h, -1).astype(np.uint32)
    if depth == 16:
        return [np.stack([r >> 8, r & 0xFF], 1).astype(np.uint8).tobytes() for r in flat]
    if depth == 8:
        return [r.astype(np.uint8).tobytes() for r in flat]
    out = []
    for r in flat:
        bits = ((r[:, None] >> np.arange(depth - 1, -1, -1)) & 1).astype(np.uint8).reshape(-1)
        out.append(np.packbits(bits).tobytes())
    return out


def _png_generic(samples, ctype, depth, palette=None, interlace=False):
    h, w = samples.shape[:2]
    if interlace:
        body = b""
        for x0, y0, dx, dy in _ADAM7:
            sub = samples[y0::dy, x0::dx]
            if sub.shape[0] and sub.shape[1]:
                body += b"".join(b"\0" + r for r in _pack_rows(sub, depth))
    else:
        body = b"".join(b"\0" + r for r in _pack_rows(samples, depth))

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)
    out = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, int(interlace)))
    if palette is not None:
        out += chunk(b"PLTE", palette.astype(np.uint8).tobytes())
    return out + chunk(b"IDAT", zlib.compress(body)) + chunk(b"IEND", b"")


@pytest.mark.parametrize("interlace", [False, True])
@pytest.mark.parametrize("ctype,depth", [(0, 1), (0, 2), (0, 4), (0, 16), (2, 16), (4, 16), (6, 16),
                                         (3, 1), (3, 2), (3, 4), (3, 8), (2, 8)])
def test_png_decoder_depths_palettes_interlace(tmp_path, ctype, depth, interlace):
    # image::open(..).into_rgb8(): palette -> its RGB entry, sub-8-bit grey
    # scaled to 0..255, 16-bit rounded to the nearest 8-bit value, alpha dropped
    rng = np.random.default_rng(ctype * 100 + depth)
    h, w = 13, 11  # odd sizes: partial Adam7 passes and partial bytes
    channels = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    top = (1 << depth) - 1
    palette = None
    if ctype == 3:
        palette = rng.integers(0, 256, (top + 1, 3))
    samples = rng.integers(0, top + 1, (h, w, channels))
    p = tmp_path / "t.png"
    p.write_bytes(_png_generic(samples, ctype, depth, palette, interlace))
    got = I.read_png(str(p))
    if ctype == 3:
        want = palette[samples[:, :, 0]]
    else:
        if depth == 16:
            s8 = (samples * 255 + 32767) // 65535
        else:
            s8 = samples * 255 // top
        want = np.repeat(s8[:, :, :1], 3, axis=2) if channels <= 2 else s8[:, :, :3]
    np.testing.assert_array_equal(got, want.astype(np.uint8))
    if depth <= 8:  # OpenCV's decoder (libpng) agrees where its 8-bit conversion is the same
        cv2 = pytest.importorskip("cv2")
        ref = cv2.imread(str(p), cv2.IMREAD_COLOR)[:, :, ::-1]
        np.testing.assert_array_equal(got, ref)


def test_load_obj_meshes(tmp_path):
    # TriangleMesh::load_obj: meshes only, slot = the model's MTL material index
    (tmp_path / "scene.mtl").write_text(MTL)
    (tmp_path / "scene.obj").write_text(OBJ)
    meshes = I.load_obj_meshes(str(tmp_path / "scene.obj"))
    assert [int(m.material_slots[0]) for m in meshes] == [2, 1, 4, 0]
    assert [m.num_triangles for m in meshes] == [2, 1, 3, 1]
    sc = SceneData()
    objs = I.load_obj_scene(sc, str(tmp_path / "scene.obj"))
    for m, o in zip(meshes, objs):
        ms = sc.meshes[sc.objects[o].mesh]
        np.testing.assert_array_equal(m.positions, ms.positions)
        np.testing.assert_array_equal(m.indices, ms.indices)


def test_mtl_defaults(tmp_path):
    # an MTL material with no statements: Kd 0.5 grey, Ks 0, Ns 0, d 1, Ni 1.5
    # -> a grey Lambertian (the crate's defaults)
    (tmp_path / "e.mtl").write_text("newmtl empty\n")
    sc = SceneData()
    m = I.convert_material(I.parse_mtl(str(tmp_path / "e.mtl"))["empty"], str(tmp_path), sc)
    assert m.kind == A.MATERIAL_LAMBERTIAN and m.albedo == (0.5, 0.5, 0.5) and m.albedo_texture == -1
