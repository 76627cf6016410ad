"""Host-side scene description (the reference's Scene / SceneObject / TriangleMesh,
src/scene.rs:17-139, src/primitives/mesh.rs:7-16) as numpy arrays, convertible to
the C-ABI ``ar_scene_desc``.  The same bytes feed the GPU library and the CPU
oracle, so both see identical geometry, transforms and materials."""
import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _abi as A


@dataclass
class Mesh:
    positions: np.ndarray                 # (V, 3) float32
    indices: np.ndarray                   # (T, 3) uint32
    normals: Optional[np.ndarray] = None  # (V, 3) float32
    material_slots: Optional[np.ndarray] = None  # (1,) or (T,) uint32
    tex_coords: Optional[np.ndarray] = None  # (V, 2) float32

    @property
    def num_triangles(self):
        return int(self.indices.shape[0])


@dataclass
class Material:
    kind: int = A.MATERIAL_LAMBERTIAN
    albedo: tuple = (0.8, 0.8, 0.8)
    f0: tuple = (0.9, 0.9, 0.9)
    roughness: float = 0.3
    emitter_light: int = -1
    eta: float = 1.5  # dielectric interior index of refraction
    albedo_texture: int = -1  # Lambertian: index into SceneData.textures


@dataclass
class Light:
    kind: int = A.LIGHT_POINT
    position: tuple = (0.0, 0.0, 0.0)   # point position / quad corner
    intensity: tuple = (1.0, 1.0, 1.0)  # point intensity / quad radiance
    edge1: tuple = (0.0, 0.0, 0.0)
    edge2: tuple = (0.0, 0.0, 0.0)


@dataclass
class Object:
    mesh: int
    materials: List[int]
    transform: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=np.float32))  # row-major math matrix
    inv_transform: Optional[np.ndarray] = None


@dataclass
class Camera:
    """PinholeCamera::from_lookat arguments (src/cameras.rs:91-123)."""
    lookfrom: tuple
    lookat: tuple
    vup: tuple = (0.0, 1.0, 0.0)
    vfov_deg: float = 40.0
    aspect: float = 1.0

    def desc(self):
        d = A.CameraDesc()
        d.lookfrom[:] = [float(x) for x in self.lookfrom]
        d.lookat[:] = [float(x) for x in self.lookat]
        d.vup[:] = [float(x) for x in self.vup]
        d.vfov_deg = float(self.vfov_deg)
        d.aspect = float(self.aspect)
        return d


def _colmajor(m: np.ndarray):
    """Math (row-major) 4x4 -> glam column-major float[16]."""
    return np.ascontiguousarray(np.asarray(m, dtype=np.float32).T).reshape(16)


class SceneData:
    """A renderable scene: meshes, objects (instances), materials, lights."""

    def __init__(self, light_distribution=A.LIGHT_DIST_POWER):
        self.meshes: List[Mesh] = []
        self.objects: List[Object] = []
        self.materials: List[Material] = []
        self.lights: List[Light] = []
        self.textures: List[np.ndarray] = []  # (H, W, 3) uint8 sRGB images (ImageTexture)
        self.light_distribution = light_distribution

    def add_mesh(self, mesh: Mesh) -> int:
        self.meshes.append(mesh)
        return len(self.meshes) - 1

    def add_material(self, mat: Material) -> int:
        self.materials.append(mat)
        return len(self.materials) - 1

    def add_object(self, obj: Object) -> int:
        self.objects.append(obj)
        return len(self.objects) - 1

    def add_texture(self, rgb8: np.ndarray) -> int:
        """Adds an 8-bit sRGB image (H, W, 3), row 0 at the top (ImageTexture::load)."""
        img = np.ascontiguousarray(rgb8, dtype=np.uint8)
        if img.ndim != 3 or img.shape[2] != 3 or img.shape[0] == 0 or img.shape[1] == 0:
            raise ValueError("texture must be a non-empty (H, W, 3) uint8 image")
        self.textures.append(img)
        return len(self.textures) - 1

    def add_light(self, light: Light) -> int:
        self.lights.append(light)
        return len(self.lights) - 1

    @property
    def num_triangles(self):
        return sum(self.meshes[o.mesh].num_triangles for o in self.objects)

    def desc(self):
        """Builds an ar_scene_desc.  Returns (desc, keepalive): the arrays in
        `keepalive` must outlive every use of `desc`."""
        keep = []
        meshes = (A.MeshDesc * max(1, len(self.meshes)))()
        for i, m in enumerate(self.meshes):
            pos = np.ascontiguousarray(m.positions, dtype=np.float32)
            idx = np.ascontiguousarray(m.indices, dtype=np.uint32)
            slots = np.ascontiguousarray(
                m.material_slots if m.material_slots is not None else np.zeros(1, np.uint32), dtype=np.uint32)
            keep += [pos, idx, slots]
            meshes[i].positions = pos.ctypes.data
            meshes[i].indices = idx.ctypes.data
            meshes[i].material_slots = slots.ctypes.data
            meshes[i].num_material_slots = slots.size
            meshes[i].num_vertices = pos.shape[0]
            meshes[i].num_triangles = idx.shape[0]
            if m.normals is not None:
                nrm = np.ascontiguousarray(m.normals, dtype=np.float32)
                keep.append(nrm)
                meshes[i].normals = nrm.ctypes.data
            if m.tex_coords is not None:
                uv = np.ascontiguousarray(m.tex_coords, dtype=np.float32)
                keep.append(uv)
                meshes[i].tex_coords = uv.ctypes.data
        objs = (A.ObjectDesc * max(1, len(self.objects)))()
        for i, o in enumerate(self.objects):
            objs[i].transform[:] = _colmajor(o.transform).tolist()
            if o.inv_transform is not None:
                objs[i].inv_transform[:] = _colmajor(o.inv_transform).tolist()
                objs[i].has_inverse = 1
            mats = np.ascontiguousarray(o.materials, dtype=np.uint32)
            keep.append(mats)
            objs[i].materials = mats.ctypes.data
            objs[i].num_materials = mats.size
            objs[i].mesh = o.mesh
        mats_d = (A.MaterialDesc * max(1, len(self.materials)))()
        for i, m in enumerate(self.materials):
            mats_d[i].kind = m.kind
            mats_d[i].emitter_light = m.emitter_light
            mats_d[i].albedo[:] = [float(x) for x in m.albedo]
            mats_d[i].f0[:] = [float(x) for x in m.f0]
            mats_d[i].roughness = float(m.roughness)
            mats_d[i].eta = float(m.eta)
            mats_d[i].albedo_texture = int(m.albedo_texture)
        lights_d = (A.LightDesc * max(1, len(self.lights)))()
        for i, l in enumerate(self.lights):
            lights_d[i].kind = l.kind
            lights_d[i].position[:] = [float(x) for x in l.position]
            lights_d[i].intensity[:] = [float(x) for x in l.intensity]
            lights_d[i].edge1[:] = [float(x) for x in l.edge1]
            lights_d[i].edge2[:] = [float(x) for x in l.edge2]
        texs_d = (A.TextureDesc * max(1, len(self.textures)))()
        for i, t in enumerate(self.textures):
            texs_d[i].rgb8 = t.ctypes.data
            texs_d[i].height, texs_d[i].width = int(t.shape[0]), int(t.shape[1])
        keep += [meshes, objs, mats_d, lights_d, texs_d]
        d = A.SceneDesc()
        d.meshes = C.addressof(meshes)
        d.objects = C.addressof(objs)
        d.materials = C.addressof(mats_d)
        d.lights = C.addressof(lights_d)
        d.textures = C.addressof(texs_d)
        d.num_textures = len(self.textures)
        d.num_meshes = len(self.meshes)
        d.num_objects = len(self.objects)
        d.num_materials = len(self.materials)
        d.num_lights = len(self.lights)
        d.light_distribution = self.light_distribution
        return d, keep


def integrator_cfg(integrator=A.INTEGRATOR_PT, spp=16, max_depth=8, rr_depth=3, mis_mode=A.MIS_POWER,
                   mis_beta=2.0, alpha=0.2, poisson_iterations=200, sor_omega=1.6, poisson_solver=A.POISSON_SOR,
                   poisson_tolerance=1e-6, seed=0, film_precision=A.FILM_F32, gdpt_flags=0):
    c = A.IntegratorCfg()
    c.integrator = integrator
    c.spp = spp
    c.max_depth = max_depth
    c.rr_depth = rr_depth
    c.mis_mode = mis_mode
    c.mis_beta = mis_beta
    c.alpha = alpha
    c.poisson_iterations = poisson_iterations
    c.sor_omega = sor_omega
    c.poisson_solver = poisson_solver
    c.poisson_tolerance = poisson_tolerance
    c.seed = seed
    c.film_precision = film_precision
    c.gdpt_flags = gdpt_flags
    return c
