"""ctypes mirror of include/agentray.h (struct layouts and constants).

Shared by the product binding (agentray._lib) and by the test oracle binding,
so both consume byte-identical scene descriptions.
"""
import ctypes as C

AR_OK = 0
AR_ERR_INVALID_ARGUMENT = -1
AR_ERR_CUDA = -2
AR_ERR_OUT_OF_MEMORY = -3
AR_ERR_UNSUPPORTED = -4
AR_ERR_TIMEOUT = -5
AR_ERR_NOT_FOUND = -6
AR_ERR_REJECTED = -7
AR_ERR_INTERNAL = -8

MATERIAL_LAMBERTIAN = 0
MATERIAL_CONDUCTOR = 1
MATERIAL_DIELECTRIC = 2
LIGHT_POINT = 0
LIGHT_QUAD = 1
LIGHT_DIST_NONE = 0
LIGHT_DIST_UNIFORM = 1
LIGHT_DIST_POWER = 2
INTEGRATOR_PT = 0
INTEGRATOR_BDPT = 1
INTEGRATOR_GDPT = 2
MIS_POWER = 0
MIS_UNIFORM = 1
POISSON_SOR = 0
POISSON_CG = 1
FILM_F32 = 0
FILM_F64 = 1
GDPT_CONSISTENT_DIVERGENCE = 1
TONEMAP_CLAMP = 0
TONEMAP_REINHARD = 1
TONEMAP_REINHARD_EXTENDED = 2

u32 = C.c_uint32
f32 = C.c_float


class MeshDesc(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("normals", C.c_void_p), ("indices", C.c_void_p),
                ("material_slots", C.c_void_p), ("tex_coords", C.c_void_p), ("num_vertices", u32),
                ("num_triangles", u32), ("num_material_slots", u32), ("_pad", u32)]


class ObjectDesc(C.Structure):
    _fields_ = [("transform", f32 * 16), ("inv_transform", f32 * 16), ("materials", C.c_void_p),
                ("mesh", u32), ("num_materials", u32), ("has_inverse", u32), ("_pad", u32)]


class MaterialDesc(C.Structure):
    _fields_ = [("kind", u32), ("emitter_light", C.c_int32), ("albedo", f32 * 3), ("f0", f32 * 3),
                ("roughness", f32), ("eta", f32), ("albedo_texture", C.c_int32), ("_pad", u32)]


class TextureDesc(C.Structure):
    _fields_ = [("rgb8", C.c_void_p), ("width", u32), ("height", u32)]


class LightDesc(C.Structure):
    _fields_ = [("kind", u32), ("_pad", u32), ("position", f32 * 3), ("intensity", f32 * 3),
                ("edge1", f32 * 3), ("edge2", f32 * 3)]


class SceneDesc(C.Structure):
    _fields_ = [("meshes", C.c_void_p), ("objects", C.c_void_p), ("materials", C.c_void_p),
                ("lights", C.c_void_p), ("textures", C.c_void_p), ("num_meshes", u32), ("num_objects", u32),
                ("num_materials", u32), ("num_lights", u32), ("light_distribution", u32), ("num_textures", u32)]


class CameraDesc(C.Structure):
    _fields_ = [("lookfrom", f32 * 3), ("lookat", f32 * 3), ("vup", f32 * 3), ("vfov_deg", f32),
                ("aspect", f32)]


class IntegratorCfg(C.Structure):
    _fields_ = [("integrator", u32), ("spp", u32), ("max_depth", u32), ("rr_depth", u32), ("mis_mode", u32),
                ("mis_beta", f32), ("alpha", f32), ("poisson_iterations", u32), ("sor_omega", f32),
                ("poisson_solver", u32), ("poisson_tolerance", C.c_double), ("seed", C.c_uint64),
                ("film_precision", u32), ("gdpt_flags", u32)]


class RayBatch(C.Structure):
    _fields_ = [("org_tmin", C.c_void_p), ("dir_tmax", C.c_void_p), ("count", C.c_uint64), ("on_device", u32),
                ("_pad", u32)]


class Hit(C.Structure):
    _fields_ = [("t", f32), ("u", f32), ("v", f32), ("prim_id", u32)]


class AccelOpts(C.Structure):
    _fields_ = [("max_leaf_size", u32), ("sah_bins", u32), ("build_threads", u32), ("bvh_width", u32),
                ("sah_node_cost", f32), ("_pad", u32)]


class Tuning(C.Structure):
    _fields_ = [("path_capacity", u32), ("traversal_blocks_per_sm", u32), ("shade_block", u32),
                ("bdpt_batch_mib", u32)]


class TuneOpts(C.Structure):
    _fields_ = [("integrator", u32), ("width", u32), ("height", u32), ("spp", u32), ("max_depth", u32),
                ("repeats", u32), ("tune_accel", u32), ("_pad", u32)]


class TuneResult(C.Structure):
    _fields_ = [("tuning", Tuning), ("accel", AccelOpts), ("default_ms", C.c_double), ("best_ms", C.c_double),
                ("candidates", u32), ("_pad", u32)]


class SceneStats(C.Structure):
    _fields_ = [("num_triangles", C.c_uint64), ("num_instances", C.c_uint64), ("num_blas_nodes", C.c_uint64),
                ("num_tlas_nodes", C.c_uint64), ("device_bytes", C.c_uint64), ("max_stack_depth", u32),
                ("_pad", u32), ("build_seconds", C.c_double)]


assert C.sizeof(IntegratorCfg) == 64
assert C.sizeof(ObjectDesc) == 152
assert C.sizeof(MaterialDesc) == 48
assert C.sizeof(MeshDesc) == 56
assert C.sizeof(TextureDesc) == 16
assert C.sizeof(SceneDesc) == 64
assert C.sizeof(LightDesc) == 56


JOB_PENDING, JOB_RUNNING, JOB_DONE, JOB_REJECTED, JOB_CANCELLED, JOB_FAILED = range(6)


class ServerOpts(C.Structure):
    _fields_ = [("film_budget_bytes", C.c_uint64), ("path_capacity", u32), ("bdpt_batch_samples", u32),
                ("bdpt_max_depth", u32), ("max_active_jobs", u32)]


class JobInfo(C.Structure):
    _fields_ = [("status", u32), ("error", C.c_int32), ("submit_ms", C.c_double), ("admit_ms", C.c_double),
                ("done_ms", C.c_double), ("path_samples", C.c_uint64)]


class ServerStats(C.Structure):
    _fields_ = [("jobs_submitted", C.c_uint64), ("jobs_done", C.c_uint64), ("jobs_rejected", C.c_uint64),
                ("jobs_cancelled", C.c_uint64), ("jobs_failed", C.c_uint64), ("path_samples_done", C.c_uint64),
                ("pt_ticks", C.c_uint64), ("bdpt_batches", C.c_uint64), ("film_bytes_in_use", C.c_uint64),
                ("film_bytes_peak", C.c_uint64), ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
                ("kernel_launches", C.c_uint64)]


class RenderStats(C.Structure):
    _fields_ = [("path_samples", C.c_uint64), ("paths", C.c_uint64), ("extend_rays", C.c_uint64),
                ("shadow_rays", C.c_uint64), ("extend_launches", C.c_uint64), ("shadow_launches", C.c_uint64)]
