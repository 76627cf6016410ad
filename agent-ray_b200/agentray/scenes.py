"""Seeded procedural scenes for the benchmark and parity workloads.

Every generator is deterministic in its seed; the reference ships no scene
assets for these workloads (its fireplace OBJ is missing), so synthetic scenes
with the stated shapes, sizes and value distributions stand in:

  cornell_box      5 axis-aligned walls + 2 rotated boxes = 34 triangles, one
                   0.25 x 0.25 quad light of radiance 15, albedos U[0.2, 0.8]
  triangle_soup    N triangles, centroids U[0,1]^3, edge lengths log-uniform
                   in [1e-3, 5e-2] (the BVH micro-benchmark) + its ray batch
  room             ~200k triangles: room box, icospheres and 500 randomly
                   transformed instanced boxes, Lambertian/GGX 50/50, 2 quad lights
"""
import math

import numpy as np

from . import _abi as A
from .scene_data import Camera, Light, Material, Mesh, Object, SceneData


# ---------------------------------------------------------------- geometry --
def quad_mesh(corner, e1, e2):
    c = np.asarray(corner, np.float64)
    e1 = np.asarray(e1, np.float64)
    e2 = np.asarray(e2, np.float64)
    pos = np.stack([c, c + e1, c + e1 + e2, c + e2]).astype(np.float32)
    idx = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    return Mesh(pos, idx)


def unit_cube_mesh():
    p = np.array([[x, y, z] for z in (-0.5, 0.5) for y in (-0.5, 0.5) for x in (-0.5, 0.5)], np.float32)
    f = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    idx = []
    for a, b, c, d in f:
        idx += [(a, b, c), (a, c, d)]
    return Mesh(p, np.array(idx, np.uint32))


def icosphere(level):
    t = (1.0 + 5 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mid])
        nf = f.shape[0]
        m01 = base + inv[0:nf]
        m12 = base + inv[nf:2 * nf]
        m20 = base + inv[2 * nf:3 * nf]
        f = np.concatenate([np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
                            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    pos = v.astype(np.float32)
    return Mesh(pos, f.astype(np.uint32), normals=pos.copy())


def trs(translate=(0, 0, 0), rot=None, scale=(1, 1, 1)):
    """4x4 (row-major math) = T * R * S, and its float64 inverse, both as float32."""
    m = np.eye(4)
    r = np.eye(3) if rot is None else np.asarray(rot, np.float64)
    m[:3, :3] = r @ np.diag(np.asarray(scale, np.float64))
    m[:3, 3] = translate
    return m.astype(np.float32), np.linalg.inv(m).astype(np.float32)


def rot_y(deg):
    a = math.radians(deg)
    return np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])


def random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def add_quad_light(sc, corner, e1, e2, radiance, visible=True):
    """Quad area light (extension) and, when visible, its emitting geometry."""
    li = sc.add_light(Light(A.LIGHT_QUAD, tuple(corner), tuple(radiance), tuple(e1), tuple(e2)))
    if visible:
        mi = sc.add_material(Material(A.MATERIAL_LAMBERTIAN, albedo=(0.0, 0.0, 0.0), emitter_light=li))
        me = sc.add_mesh(quad_mesh(corner, e1, e2))
        sc.add_object(Object(me, [mi]))
    return li


# ------------------------------------------------------------------ scenes --
def checker_texture(n=16, cells=4, seed=0):
    """A seeded n x n 8-bit sRGB image: a checkerboard of random colours."""
    rng = np.random.default_rng(seed)
    cols = rng.integers(0, 256, (cells * cells, 3), dtype=np.uint8)
    y, x = np.mgrid[0:n, 0:n]
    cell = (y * cells // n) * cells + (x * cells // n)
    return cols[cell]


def cornell_box(seed=1, light_radiance=15.0, point_light=False, glass=False, textured=False):
    """Config-1 Cornell box: 5 walls (10 tris) + 2 rotated boxes (24 tris) and a
    0.25 x 0.25 quad light of radiance 15 just below the ceiling.  textured=True
    gives the floor and back wall checker ImageTextures.  glass=True
    makes the tall box a rough dielectric (eta 1.5, alpha 0.2), lifted 2 mm
    off the floor, and adds a dielectric icosphere (eta 1.33, alpha 0.05)."""
    rng = np.random.default_rng(seed)
    sc = SceneData(A.LIGHT_DIST_POWER)
    walls = [((0, 0, 0), (0, 0, 1), (1, 0, 0)),   # floor
             ((0, 1, 0), (1, 0, 0), (0, 0, 1)),   # ceiling
             ((0, 0, 0), (1, 0, 0), (0, 1, 0)),   # back
             ((0, 0, 0), (0, 1, 0), (0, 0, 1)),   # left
             ((1, 0, 0), (0, 0, 1), (0, 1, 0))]   # right
    for k, (c, e1, e2) in enumerate(walls):
        mesh = quad_mesh(c, e1, e2)
        mat = sc.add_material(Material(A.MATERIAL_LAMBERTIAN, albedo=tuple(rng.uniform(0.2, 0.8, 3))))
        if textured and k in (0, 2):
            # floor and back wall: checker ImageTextures, uv repeating past [0, 1)
            # and (back wall) negative, to exercise the repeat wrap
            mesh.tex_coords = (np.array([[0, 0], [3, 0], [3, 3], [0, 3]], np.float32) if k == 0 else
                               np.array([[-1.25, -0.5], [0.75, -0.5], [0.75, 1.5], [-1.25, 1.5]], np.float32))
            tex = sc.add_texture(checker_texture(16 if k == 0 else 7, 4, seed=10 + k))
            mat = sc.add_material(Material(A.MATERIAL_LAMBERTIAN, albedo_texture=tex))
        m = sc.add_mesh(mesh)
        sc.add_object(Object(m, [mat]))
    cube = sc.add_mesh(unit_cube_mesh())
    for k, ((tx, ty, tz), deg, (sx, sy, sz)) in enumerate([((0.33, 0.3, 0.35), 15.0, (0.3, 0.6, 0.3)),
                                                          ((0.67, 0.15, 0.62), -18.0, (0.3, 0.3, 0.3))]):
        mat = sc.add_material(Material(A.MATERIAL_LAMBERTIAN, albedo=tuple(rng.uniform(0.2, 0.8, 3))))
        if glass and k == 0:
            mat = sc.add_material(Material(A.MATERIAL_DIELECTRIC, roughness=0.2, eta=1.5))
            # lifted 2 mm off the floor: a glass box standing on it would put
            # its bottom face in the floor's plane, and a ray leaving the box
            # downward would hit both at the same t (a tie that any two
            # traversal orders may break differently)
            ty += 0.002
        xf, inv = trs((tx, ty, tz), rot_y(deg), (sx, sy, sz))
        sc.add_object(Object(cube, [mat], xf, inv))
    if glass:
        sph = sc.add_mesh(icosphere(3))
        mat = sc.add_material(Material(A.MATERIAL_DIELECTRIC, roughness=0.05, eta=1.33))
        xf, inv = trs((0.7, 0.45, 0.6), None, (0.14, 0.14, 0.14))
        sc.add_object(Object(sph, [mat], xf, inv))
    if point_light:
        sc.add_light(Light(A.LIGHT_POINT, (0.5, 0.9, 0.5), (light_radiance * 0.0625,) * 3))
    else:
        add_quad_light(sc, (0.375, 0.995, 0.375), (0.25, 0.0, 0.0), (0.0, 0.0, 0.25), (light_radiance,) * 3)
    cam = Camera((0.5, 0.5, 2.2), (0.5, 0.5, 0.0), (0.0, 1.0, 0.0), 40.0, 1.0)
    return sc, cam


def triangle_soup(n_tris, seed=2):
    """BVH micro-benchmark geometry: centroids U[0,1]^3, 3 vertices at random
    unit directions scaled by an edge length log-uniform in [1e-3, 5e-2]."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.0, 1.0, (n_tris, 1, 3))
    d = rng.normal(size=(n_tris, 3, 3))
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    length = np.exp(rng.uniform(math.log(1e-3), math.log(5e-2), (n_tris, 1, 1)))
    pos = (c + d * length).reshape(-1, 3).astype(np.float32)
    idx = np.arange(3 * n_tris, dtype=np.uint32).reshape(-1, 3)
    sc = SceneData(A.LIGHT_DIST_NONE)
    m = sc.add_mesh(Mesh(pos, idx))
    mat = sc.add_material(Material())
    sc.add_object(Object(m, [mat]))
    return sc


def soup_rays(n_rays, seed=3, tmax=float("inf"), tmin=1e-4):
    """Rays for the micro-benchmark: origins U[0,1]^3, directions uniform on S^2.
    Returns (org_tmin, dir_tmax) float32 arrays of shape (n, 4)."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(0.0, 1.0, (n_rays, 3)).astype(np.float32)
    d = rng.normal(size=(n_rays, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    ot = np.empty((n_rays, 4), np.float32)
    dt = np.empty((n_rays, 4), np.float32)
    ot[:, :3] = o
    ot[:, 3] = tmin
    dt[:, :3] = d.astype(np.float32)
    dt[:, 3] = tmax
    return ot, dt


def random_material(rng):
    if rng.uniform() < 0.5:
        return Material(A.MATERIAL_LAMBERTIAN, albedo=tuple(rng.uniform(0.2, 0.8, 3)))
    return Material(A.MATERIAL_CONDUCTOR, f0=tuple(rng.uniform(0.5, 0.95, 3)), roughness=float(rng.uniform(0.1, 0.5)))


def room(seed=4, sphere_levels=(6, 6, 5, 4), n_boxes=500, point_lights=False):
    """Config-3/4 room: a 10 x 5 x 10 box, icospheres (default 2 x level 6,
    level 5, level 4) and `n_boxes` instanced unit boxes with random
    rotation/scale/position; Lambertian and GGX conductors 50/50; 2 quad lights.
    Defaults give 195,452 triangles (within 5% of 200k)."""
    rng = np.random.default_rng(seed)
    sc = SceneData(A.LIGHT_DIST_POWER)
    W, H, D = 10.0, 5.0, 10.0
    walls = [((0, 0, 0), (0, 0, D), (W, 0, 0)), ((0, H, 0), (W, 0, 0), (0, 0, D)), ((0, 0, 0), (W, 0, 0), (0, H, 0)),
             ((0, 0, D), (0, H, 0), (W, 0, 0)), ((0, 0, 0), (0, H, 0), (0, 0, D)), ((W, 0, 0), (0, 0, D), (0, H, 0))]
    pos, idx = [], []
    for k, (c, e1, e2) in enumerate(walls):
        q = quad_mesh(c, e1, e2)
        pos.append(q.positions)
        idx.append(q.indices + 4 * k)
    slots = np.repeat(np.arange(6, dtype=np.uint32), 2)
    m = sc.add_mesh(Mesh(np.concatenate(pos), np.concatenate(idx), material_slots=slots))
    wall_mats = [sc.add_material(Material(A.MATERIAL_LAMBERTIAN, albedo=tuple(rng.uniform(0.2, 0.8, 3))))
                 for _ in range(6)]
    sc.add_object(Object(m, wall_mats))
    spheres = [((2.5, 1.2, 3.0), 1.2), ((7.5, 1.2, 3.5), 1.2), ((5.0, 0.9, 6.5), 0.9), ((2.0, 0.6, 7.5), 0.6)]
    for lvl, (ctr, r) in zip(sphere_levels, spheres):
        me = sc.add_mesh(icosphere(lvl))
        mat = sc.add_material(random_material(rng))
        xf, inv = trs(ctr, None, (r, r, r))
        sc.add_object(Object(me, [mat], xf, inv))
    cube = sc.add_mesh(unit_cube_mesh())
    for _ in range(n_boxes):
        mat = sc.add_material(random_material(rng))
        s = rng.uniform(0.1, 0.5, 3)
        t = (rng.uniform(0.3, W - 0.3), rng.uniform(0.2, H - 0.6), rng.uniform(0.3, D - 0.3))
        xf, inv = trs(t, random_rotation(rng), s)
        sc.add_object(Object(cube, [mat], xf, inv))
    if point_lights:
        sc.add_light(Light(A.LIGHT_POINT, (3.0, 4.5, 5.0), (20.0, 20.0, 20.0)))
        sc.add_light(Light(A.LIGHT_POINT, (7.0, 4.5, 5.0), (15.0, 18.0, 20.0)))
    else:
        add_quad_light(sc, (2.5, 4.99, 4.5), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), (12.0, 12.0, 12.0))
        add_quad_light(sc, (6.5, 4.99, 4.5), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), (10.0, 11.0, 12.0))
    cam = Camera((5.0, 2.5, 9.6), (5.0, 1.8, 0.0), (0.0, 1.0, 0.0), 60.0, 1.0)
    return sc, cam


SERVED_TRIANGLES = [10_000, 19_307, 37_276, 71_969, 138_950, 268_270, 517_947, 1_000_000]


def served_scene(k, seed=5):
    """Scene k of the 8 served-stream scenes: triangle counts log-spaced from
    10k to 1M (SERVED_TRIANGLES), built from a room box, icospheres and
    instanced boxes, Lambertian/GGX 50/50, two quad lights.  Returns
    (scene_data, camera)."""
    target = SERVED_TRIANGLES[k]
    rng = np.random.default_rng(seed * 100 + k)
    sc = SceneData(A.LIGHT_DIST_POWER)
    W, H, D = 10.0, 5.0, 10.0
    walls = [((0, 0, 0), (0, 0, D), (W, 0, 0)), ((0, H, 0), (W, 0, 0), (0, 0, D)), ((0, 0, 0), (W, 0, 0), (0, H, 0)),
             ((0, 0, D), (0, H, 0), (W, 0, 0)), ((0, 0, 0), (0, H, 0), (0, 0, D)), ((W, 0, 0), (0, 0, D), (0, H, 0))]
    pos, idx = [], []
    for i, (c, e1, e2) in enumerate(walls):
        q = quad_mesh(c, e1, e2)
        pos.append(q.positions)
        idx.append(q.indices + 4 * i)
    m = sc.add_mesh(Mesh(np.concatenate(pos), np.concatenate(idx)))
    sc.add_object(Object(m, [sc.add_material(Material(A.MATERIAL_LAMBERTIAN, albedo=tuple(rng.uniform(0.2, 0.8, 3))))]))
    remaining = target - 12 - 4
    n_boxes = min(300, max(20, remaining // 200))
    remaining -= 12 * n_boxes
    sphere_meshes = {}
    eye = np.array([5.0, 2.5, 9.6])

    def clear_of_eye(p, radius):
        return np.linalg.norm(np.asarray(p) - eye) > radius + 0.6
    while remaining >= 20 * 4 ** 2:
        lvl = max(l for l in range(2, 9) if 20 * 4 ** l <= remaining)
        if lvl not in sphere_meshes:
            sphere_meshes[lvl] = sc.add_mesh(icosphere(lvl))
        r = float(rng.uniform(0.4, 1.2))
        ctr = (rng.uniform(1.0, W - 1.0), r, rng.uniform(1.0, D - 1.0))
        while not clear_of_eye(ctr, r):
            ctr = (rng.uniform(1.0, W - 1.0), r, rng.uniform(1.0, D - 1.0))
        xf, inv = trs(ctr, None, (r, r, r))
        sc.add_object(Object(sphere_meshes[lvl], [sc.add_material(random_material(rng))], xf, inv))
        remaining -= 20 * 4 ** lvl
    n_boxes += remaining // 12
    cube = sc.add_mesh(unit_cube_mesh())
    for _ in range(n_boxes):
        s = rng.uniform(0.1, 0.5, 3)
        t = (rng.uniform(0.3, W - 0.3), rng.uniform(0.2, H - 0.6), rng.uniform(0.3, D - 0.3))
        while not clear_of_eye(t, 0.45):
            t = (rng.uniform(0.3, W - 0.3), rng.uniform(0.2, H - 0.6), rng.uniform(0.3, D - 0.3))
        xf, inv = trs(t, random_rotation(rng), s)
        sc.add_object(Object(cube, [sc.add_material(random_material(rng))], xf, inv))
    add_quad_light(sc, (2.5, 4.99, 4.5), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), (12.0, 12.0, 12.0))
    add_quad_light(sc, (6.5, 4.99, 4.5), (1.0, 0.0, 0.0), (0.0, 0.0, 1.0), (10.0, 11.0, 12.0))
    cam = Camera((5.0, 2.5, 9.6), (5.0, 1.8, 0.0), (0.0, 1.0, 0.0), 60.0, 1.0)
    return sc, cam


def served_stream(n_jobs=2000, seed=5, rate_hz=1.0):
    """The served workload: Poisson arrivals (rate_hz jobs/s), scene uniform
    over the 8 served scenes, resolution from {128,256,512,1024}^2, spp from
    {4,16,64}, PT or BDPT 70/30.  Returns a list of dicts."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n_jobs))
    res = rng.choice([128, 256, 512, 1024], n_jobs)
    spp = rng.choice([4, 16, 64], n_jobs)
    scene = rng.integers(0, 8, n_jobs)
    bdpt = rng.uniform(size=n_jobs) < 0.3
    return [{"arrival_s": float(t[i]), "scene": int(scene[i]), "res": int(res[i]), "spp": int(spp[i]),
             "integrator": "bdpt" if bdpt[i] else "pt"} for i in range(n_jobs)]


def furnace(albedo=0.5, seed=0):
    """Closed Lambertian sphere of uniform albedo around a point light at its
    centre (an analytic check: every surface point sees irradiance I / r^2)."""
    sc = SceneData(A.LIGHT_DIST_POWER)
    me = sc.add_mesh(icosphere(4))
    mat = sc.add_material(Material(A.MATERIAL_LAMBERTIAN, albedo=(albedo,) * 3))
    sc.add_object(Object(me, [mat]))
    sc.add_light(Light(A.LIGHT_POINT, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0)))
    cam = Camera((0.0, 0.0, 0.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), 30.0, 1.0)
    return sc, cam
