/*
 * agentray.h — C ABI of the B200 light-transport library (libagentray.so).
 *
 * This is the drop-in boundary for agent-ray's light-transport hot path.  The
 * reference crate exposes it as Rust traits; each entry point below names the
 * reference interface it replaces (paths are inside the agent-ray crate):
 *
 *   Integrator::render(&Scene, &dyn Camera, w, h) -> Arc<Film>
 *       src/integrators/mod.rs:18-26                    -> ar_render
 *   Scene::new(objects, lights, light_dist)
 *       src/scene.rs:125-139 (+ SceneObject::new :29-35) -> ar_scene_create
 *   BLASAccel::build / TLAS::build
 *       src/accel/bvh.rs:326-344, :395-411               -> ar_scene_build_accel
 *   Scene::intersect(&Ray) -> Option<(f32, ShadingPoint)> / TLAS::intersect
 *       src/scene.rs:142-162, src/accel/bvh.rs:413-447   -> ar_trace_closest
 *   Scene::occluded(&Ray) -> bool
 *       src/scene.rs:166-168                             -> ar_trace_any
 *   Film::to_hdr_vec() -> Vec<Vec3A>
 *       src/film.rs:272-274                              -> the out_rgb buffer of ar_render
 *
 * Conventions
 *   - Every function returns an int status: AR_OK (0) or a negative AR_ERR_*.
 *     ar_last_error() returns a message for the calling thread's last error.
 *     No C++ exception crosses this ABI.
 *   - Scene descriptors hold host pointers; ar_scene_create copies everything
 *     it needs, so the caller keeps ownership and may free them afterwards.
 *   - Matrices are 4x4 column-major (glam::Mat4 memory layout).
 *   - Rays follow the reference Ray::new (src/geometry.rs:12-20): the library
 *     normalises the direction exactly as glam's Vec3A::normalize does.
 *   - A context owns one CUDA stream.  A context is externally synchronised:
 *     one host thread at a time.  Different contexts are independent.
 *   - Buffers flagged `on_device` are CUDA device pointers on the context's
 *     device; otherwise they are host pointers (pinned or pageable).
 */
#ifndef AGENTRAY_H
#define AGENTRAY_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AR_ABI_VERSION 1

enum ar_status {
    AR_OK = 0,
    AR_ERR_INVALID_ARGUMENT = -1,
    AR_ERR_CUDA = -2,
    AR_ERR_OUT_OF_MEMORY = -3,
    AR_ERR_UNSUPPORTED = -4,
    AR_ERR_TIMEOUT = -5,
    AR_ERR_NOT_FOUND = -6,
    AR_ERR_REJECTED = -7,
    AR_ERR_INTERNAL = -8
};

typedef struct ar_context ar_context;
typedef struct ar_scene ar_scene;

/* ---- scene description (src/primitives/mesh.rs:7-16, src/scene.rs:17-48) ---- */

typedef struct ar_mesh_desc {
    const float* positions;          /* num_vertices * 3 */
    const float* normals;            /* num_vertices * 3, or NULL (geometric normal is used) */
    const uint32_t* indices;         /* num_triangles * 3 */
    const uint32_t* material_slots;  /* 1 entry (shared slot) or num_triangles entries */
    const float* tex_coords;         /* num_vertices * 2, or NULL: tex_uv is then the barycentric (u, v)
                                        (SceneObject::tex_uv, src/scene.rs:54-66) */
    uint32_t num_vertices;
    uint32_t num_triangles;
    uint32_t num_material_slots;
    uint32_t _pad;
} ar_mesh_desc;

/* One SceneObject: a mesh placed by a local->world transform, with its
 * slot -> material table (src/scene.rs:17-48). */
typedef struct ar_object_desc {
    float transform[16];             /* column-major local->world */
    float inv_transform[16];         /* column-major world->local, used when has_inverse != 0 */
    const uint32_t* materials;       /* slot -> index into ar_scene_desc.materials */
    uint32_t mesh;
    uint32_t num_materials;
    uint32_t has_inverse;
    uint32_t _pad;
} ar_object_desc;

enum ar_material_kind {
    AR_MATERIAL_LAMBERTIAN = 0,      /* src/surfaces/lambertian.rs */
    AR_MATERIAL_CONDUCTOR = 1,       /* src/surfaces/microfacet.rs:86-152 (GGX) */
    AR_MATERIAL_DIELECTRIC = 2       /* src/surfaces/microfacet.rs:155-307 (rough GGX glass) */
};

typedef struct ar_material_desc {
    uint32_t kind;
    int32_t emitter_light;           /* >= 0: this surface is the emitting face of quad light
                                        `emitter_light` (area-light extension); -1 otherwise */
    float albedo[3];                 /* Lambertian albedo (constant texture) */
    float f0[3];                     /* conductor reflectance at normal incidence */
    float roughness;                 /* conductor / dielectric GGX alpha, clamped to [1e-3, 1] */
    float eta;                       /* dielectric interior index of refraction (> 0) */
    int32_t albedo_texture;          /* Lambertian: index into ar_scene_desc.textures (ImageTexture), or -1 */
    uint32_t _pad;
} ar_material_desc;

/* ImageTexture (src/texture.rs:65-151): 8-bit sRGB texels, decoded to linear
 * at scene creation, sampled bilinearly with repeat wrap. */
typedef struct ar_texture_desc {
    const uint8_t* rgb8;             /* width * height * 3 bytes, row-major from the top row */
    uint32_t width, height;
} ar_texture_desc;

enum ar_light_kind {
    AR_LIGHT_POINT = 0,              /* src/lights/point.rs */
    AR_LIGHT_QUAD = 1                /* one-sided quad area light {corner, edge1, edge2, radiance}: an
                                        extension the configs need (the crate has point lights only) */
};

typedef struct ar_light_desc {
    uint32_t kind;
    uint32_t _pad;
    float position[3];               /* point: position;  quad: corner */
    float intensity[3];              /* point: intensity (W/sr); quad: radiance */
    float edge1[3];                  /* quad only: corner + s*edge1 + t*edge2, normal = edge1 x edge2 */
    float edge2[3];
} ar_light_desc;

enum ar_light_distribution {
    AR_LIGHT_DIST_NONE = 0,
    AR_LIGHT_DIST_UNIFORM = 1,       /* src/lights.rs:136-159 */
    AR_LIGHT_DIST_POWER = 2          /* src/lights.rs:171-235 */
};

typedef struct ar_scene_desc {
    const ar_mesh_desc* meshes;
    const ar_object_desc* objects;
    const ar_material_desc* materials;
    const ar_light_desc* lights;
    const ar_texture_desc* textures;
    uint32_t num_meshes;
    uint32_t num_objects;
    uint32_t num_materials;
    uint32_t num_lights;
    uint32_t light_distribution;
    uint32_t num_textures;
} ar_scene_desc;

/* PinholeCamera::from_lookat (src/cameras.rs:91-123). */
typedef struct ar_camera_desc {
    float lookfrom[3];
    float lookat[3];
    float vup[3];
    float vfov_deg;
    float aspect;
} ar_camera_desc;

/* ---- integrator configuration (config structs of src/integrators/) ---- */

enum ar_integrator_kind {
    AR_INTEGRATOR_PT = 0,            /* PathTracerConfig, src/integrators/path_tracer.rs:18-31 */
    AR_INTEGRATOR_BDPT = 1,          /* BdptConfig, src/integrators/bidirectional_path_tracer.rs:102-133 */
    AR_INTEGRATOR_GDPT = 2           /* GdptConfig, src/integrators/gradient_domain_pt.rs:47-76 */
};
enum ar_mis_mode { AR_MIS_POWER = 0, AR_MIS_UNIFORM = 1 };
enum ar_poisson_solver {
    AR_POISSON_SOR = 0,              /* the reference red-black SOR, gradient_domain_pt.rs:449-630 */
    AR_POISSON_CG = 1                /* FP32 conjugate gradient with FP64 residual refinement */
};
enum ar_film_precision { AR_FILM_F32 = 0, AR_FILM_F64 = 1 };

/* GDPT options beyond the reference (extension; off by default).
 * AR_GDPT_CONSISTENT_DIVERGENCE: the reference builds the Poisson right-hand
 * side as alpha*primal + div G (gradient_domain_pt.rs:503-541) while its
 * stencil is (alpha + N) I - sum I(n); with G = I(x+1) - I(x) the consistent
 * right-hand side is alpha*primal - div G.  With the flag set the solve uses
 * that sign and converges to the primal-domain image; without it the output
 * equals the reference's. */
enum ar_gdpt_flags { AR_GDPT_CONSISTENT_DIVERGENCE = 1 };

typedef struct ar_integrator_cfg {
    uint32_t integrator;             /* ar_integrator_kind */
    uint32_t spp;
    uint32_t max_depth;
    uint32_t rr_depth;
    uint32_t mis_mode;               /* BDPT */
    float mis_beta;                  /* BDPT */
    float alpha;                     /* GDPT screening weight */
    uint32_t poisson_iterations;     /* GDPT SOR iterations / CG iteration cap */
    float sor_omega;                 /* GDPT SOR relaxation */
    uint32_t poisson_solver;         /* ar_poisson_solver */
    double poisson_tolerance;        /* CG: relative residual target (FP64) */
    uint64_t seed;                   /* sampler key; 0 reproduces the default stream */
    uint32_t film_precision;         /* ar_film_precision */
    uint32_t gdpt_flags;             /* ar_gdpt_flags; 0 reproduces the reference */
} ar_integrator_cfg;

/* ---- ray batches (src/geometry.rs:3-20, src/accel/bvh.rs:10-20) ---- */

typedef struct ar_ray_batch {
    const float* org_tmin;           /* count * 4: origin.xyz, t_min */
    const float* dir_tmax;           /* count * 4: direction.xyz (normalised by the library), t_max */
    uint64_t count;
    uint32_t on_device;
    uint32_t _pad;
} ar_ray_batch;

/* RayHit (src/accel/bvh.rs:10-20): t, barycentric (u, v) and prim_id; miss =
 * t = +inf, prim_id = inst_id = 0xFFFFFFFF (RayHit::INVALID_ID). */
typedef struct ar_hit {
    float t;
    float u;
    float v;
    uint32_t prim_id;
} ar_hit;

typedef struct ar_accel_opts {
    uint32_t max_leaf_size;          /* 1..4 triangles per BLAS leaf (default 3); TLAS leaves hold one instance */
    uint32_t sah_bins;               /* binned SAH bins (default 32) */
    uint32_t build_threads;          /* host threads for the build (0 = all cores) */
    uint32_t bvh_width;              /* children per node, 2..8 (0 = 8); the node format is 8-wide */
    float sah_node_cost;             /* binary-SAH cost of a node relative to one triangle test (0 = 0.5) */
    uint32_t _pad;
} ar_accel_opts;

typedef struct ar_scene_stats {
    uint64_t num_triangles;
    uint64_t num_instances;
    uint64_t num_blas_nodes;         /* 8-wide nodes across all meshes */
    uint64_t num_tlas_nodes;
    uint64_t device_bytes;           /* total device memory held by the scene */
    uint32_t max_stack_depth;        /* worst-case traversal stack entries */
    uint32_t _pad;
    double build_seconds;
} ar_scene_stats;

/* ---- entry points ---- */

const char* ar_last_error(void);
int ar_abi_version(void);

int ar_context_create(int device, ar_context** out);
int ar_context_destroy(ar_context* ctx);
/* Use the caller's CUDA stream (cudaStream_t passed as void*) instead of the
 * context's own; NULL restores the context stream. */
int ar_context_set_stream(ar_context* ctx, void* cuda_stream);
int ar_context_synchronize(ar_context* ctx);

/* Launch and queue parameters of a context (the autotuner's search space).
 * No reference counterpart: the reference's CPU integrators have no such knobs. */
typedef struct ar_tuning {
    uint32_t path_capacity;          /* PT/GDPT engine path slots (queue capacity; 0: 2^22) */
    uint32_t traversal_blocks_per_sm;/* persistent traversal grid, 128-thread blocks per SM, 1..8 (0: 8) */
    uint32_t shade_block;            /* threads per block of the shading stage: 64, 128 or 256 (0: 256) */
    uint32_t bdpt_batch_mib;         /* HBM for one BDPT batch of ar_render, MiB (0: 12288);
                                        a render of more than one batch keeps two
                                        (two lanes) */
} ar_tuning;

int ar_context_get_tuning(const ar_context* ctx, ar_tuning* out);
/* Applies `t` to later renders (synchronises the context's stream first). */
int ar_context_set_tuning(ar_context* ctx, const ar_tuning* t);

typedef struct ar_tune_opts {
    uint32_t integrator;             /* AR_INTEGRATOR_PT / _BDPT / _GDPT: the workload timed */
    uint32_t width, height;          /* size of the timed render (0: 256 x 256) */
    uint32_t spp;                    /* spp of the timed render (0: 4) */
    uint32_t max_depth;              /* 0: 8 */
    uint32_t repeats;                /* timed renders per candidate, the median counts (0: 3) */
    uint32_t tune_accel;             /* 1: also search BVH width and leaf size (rebuilds the scene's accel) */
    uint32_t _pad;
} ar_tune_opts;

typedef struct ar_tune_result {
    ar_tuning tuning;                /* best launch/queue parameters (applied to ctx) */
    ar_accel_opts accel;             /* best build options (the scene is left built with them) */
    double default_ms;               /* median render time with the starting parameters */
    double best_ms;                  /* median render time with the result */
    uint32_t candidates;             /* configurations timed */
    uint32_t _pad;
} ar_tune_result;

/* Project autotuner: coordinate descent over BVH width, leaf size, traversal
 * grid, shading block size and queue capacities, each candidate timed with
 * CUDA events on the context's stream.  Leaves the best tuning applied to `ctx`
 * and `scene` built with the best accel options.  No reference counterpart. */
int ar_autotune(ar_context* ctx, ar_scene* scene, const ar_camera_desc* camera, const ar_tune_opts* opts,
                ar_tune_result* out);

int ar_scene_create(ar_context* ctx, const ar_scene_desc* desc, ar_scene** out);
int ar_scene_destroy(ar_scene* scene);
/* (Re)build the acceleration structures with explicit options.  ar_scene_create
 * already builds with defaults. */
int ar_scene_build_accel(ar_context* ctx, ar_scene* scene, const ar_accel_opts* opts);
int ar_scene_get_stats(const ar_scene* scene, ar_scene_stats* out);

/* Closest hit for every ray (Scene::intersect / TLAS::intersect).  `hits` and
 * `inst_ids` have `rays->count` entries and live where `out_on_device` says. */
int ar_trace_closest(ar_context* ctx, const ar_scene* scene, const ar_ray_batch* rays,
                     ar_hit* hits, uint32_t* inst_ids, uint32_t out_on_device);
/* Occlusion for every ray (Scene::occluded): occluded[i] = 1 if any triangle is
 * hit with t in [t_min, t_max]. */
int ar_trace_any(ar_context* ctx, const ar_scene* scene, const ar_ray_batch* rays,
                 uint8_t* occluded, uint32_t out_on_device);

/* Integrator::render: W*H*3 linear HDR floats, row-major from the top-left,
 * already divided by spp (Film::to_hdr_vec). */
int ar_render(ar_context* ctx, const ar_scene* scene, const ar_camera_desc* camera,
              const ar_integrator_cfg* cfg, uint32_t width, uint32_t height,
              float* out_rgb, uint32_t out_on_device);

/* Renders only samples [sample_begin, sample_end) of every pixel, each weighted
 * by 1/spp, so the images of disjoint ranges sum to the ar_render image (with
 * the same seed): multi-GPU sample sharding, each rank rendering its range
 * before a film sum (e.g. an NCCL all-reduce).  PT and BDPT only (GDPT solves
 * its Poisson system after all samples).  No reference counterpart: the
 * reference renders all samples in one process. */
int ar_render_samples(ar_context* ctx, const ar_scene* scene, const ar_camera_desc* camera,
                      const ar_integrator_cfg* cfg, uint32_t width, uint32_t height, uint32_t sample_begin,
                      uint32_t sample_end, float* out_rgb, uint32_t out_on_device);

/* ---- film output (src/film.rs:136-302) ---- */

enum ar_tone_mapper {
    AR_TONEMAP_CLAMP = 0,            /* ToneMapper::Clamp */
    AR_TONEMAP_REINHARD = 1,         /* ToneMapper::Reinhard (luminance-preserving) */
    AR_TONEMAP_REINHARD_EXTENDED = 2 /* ToneMapper::ReinhardExtended { white_point } */
};

/* Film::to_rgb_image: scale, tone-map, encode with 1/gamma and quantise to
 * 8-bit RGB (W*H*3 bytes, row-major from the top-left).  `hdr_rgb` and
 * `out_rgb8` are host pointers, or device pointers with on_device = 1. */
int ar_film_to_rgb8(ar_context* ctx, const float* hdr_rgb, uint32_t width, uint32_t height, uint32_t tone_mapper,
                    float white_point, float gamma, float scale, uint8_t* out_rgb8, uint32_t on_device);

/* Film::save_exr (src/film.rs:304-346): writes linear RGB * scale, without
 * tone mapping, to `path` as an OpenEXR scanline file with HALF channels
 * B, G, R (f16 round-to-nearest-even) and ZIP compression (16 scanlines per
 * chunk).  The f16 conversion, channel split and ZIP byte reorder + predictor
 * run on the device; deflate runs on host threads.  `hdr_rgb` is a host
 * pointer, or a device pointer with on_device = 1. */
int ar_film_save_exr(ar_context* ctx, const float* hdr_rgb, uint32_t width, uint32_t height, float scale,
                     uint32_t on_device, const char* path);

/* screened_poisson_reconstruct (src/integrators/gradient_domain_pt.rs:449-630):
 * reconstructs an image from interleaved-RGB primal and forward-difference
 * gradient films (W*H*3 f32 each) with cfg->alpha and cfg->poisson_solver
 * (SOR: cfg->poisson_iterations sweeps with cfg->sor_omega; CG: to
 * cfg->poisson_tolerance).  `rel_residual` (optional, host) receives the final
 * FP64 relative residual of the CG solver (-1 for SOR). */
int ar_poisson_reconstruct(ar_context* ctx, const ar_integrator_cfg* cfg, uint32_t width, uint32_t height,
                           const float* primal, const float* grad_x, const float* grad_y, float* out,
                           uint32_t on_device, double* rel_residual);

/* Scratch-free red-black SOR (no counterpart in the reference).  For callers
 * that cannot allocate device memory while they run: a frame loop or a plugin
 * whose host owns the device memory pool, or code between CUDA-graph captures
 * where cudaMalloc would synchronise.  Same result as ar_poisson_reconstruct
 * with AR_POISSON_SOR (cfg->poisson_solver must be AR_POISSON_SOR, else
 * AR_ERR_UNSUPPORTED), but: all pointers are device pointers on the current
 * device (anything else fails with AR_ERR_INVALID_ARGUMENT before any launch);
 * work is queued on `cuda_stream` (NULL: the legacy default stream)
 * without synchronising; no context is needed and nothing is allocated.  The
 * solver's scratch is a static device array of 6 MiB that every GPU loading the
 * library keeps until exit, which limits images to AR_STATIC_SOR_MAX_PIXELS
 * pixels (larger ones fail with AR_ERR_INVALID_ARGUMENT).  The first call on a
 * device looks the array up (do it before any stream capture); calls that
 * overlap on the GPU share the array and race, so serialise them. */
#define AR_STATIC_SOR_MAX_PIXELS (512u * 512u)
int ar_poisson_sor_static(const ar_integrator_cfg* cfg, uint32_t width, uint32_t height, const float* primal,
                          const float* grad_x, const float* grad_y, float* out, void* cuda_stream);

/* ---- serving (no counterpart in the reference: it renders one job per call) ----
 * A server owns a worker thread that continuously batches every admitted job
 * into shared wavefront kernels: PT and GDPT paths stream through one path pool
 * refilled every tick; BDPT jobs share sample batches.  Jobs are admitted in
 * arrival order while their films fit the HBM budget; a job whose films alone
 * exceed the budget is REJECTED.  Each tick (and each BDPT batch), a running
 * job whose remaining samples fit in an equal share of the free capacity takes
 * them all; the rest goes to the other jobs smallest first, a job's size
 * discounted by 1 + (seconds waited) / 2, ties in arrival order.  Results are
 * written to the caller's host buffer (W*H*3 f32, like ar_render) before the
 * job reports DONE. */
typedef struct ar_server ar_server;

enum ar_job_status {
    AR_JOB_PENDING = 0,
    AR_JOB_RUNNING = 1,
    AR_JOB_DONE = 2,
    AR_JOB_REJECTED = 3,
    AR_JOB_CANCELLED = 4,
    AR_JOB_FAILED = 5
};

typedef struct ar_server_opts {
    uint64_t film_budget_bytes;      /* HBM for job films (0: 8 GiB) */
    uint32_t path_capacity;          /* path slots of the streaming engine (0: 2^22) */
    uint32_t bdpt_batch_samples;     /* samples per BDPT batch (0: 2^20); the server keeps
                                        two batches' buffers (two lanes) */
    uint32_t bdpt_max_depth;         /* largest BDPT max_depth accepted (0: 10) */
    uint32_t max_active_jobs;        /* 0: 1024 */
} ar_server_opts;

typedef struct ar_job_info {
    uint32_t status;                 /* ar_job_status */
    int32_t error;                   /* ar_status of a FAILED job */
    double submit_ms, admit_ms, done_ms;  /* server clock */
    uint64_t path_samples;
} ar_job_info;

typedef struct ar_server_stats {
    uint64_t jobs_submitted, jobs_done, jobs_rejected, jobs_cancelled, jobs_failed;
    uint64_t path_samples_done;
    uint64_t pt_ticks, bdpt_batches;
    uint64_t film_bytes_in_use, film_bytes_peak;
    /* host<->device bytes the server copied (job tables, batch descriptors,
     * completion snapshots, results into host buffers) and the kernels it
     * launched, since creation */
    uint64_t h2d_bytes, d2h_bytes, kernel_launches;
} ar_server_stats;

int ar_server_create(ar_context* ctx, const ar_server_opts* opts, ar_server** out);
/* Waits for admitted jobs to finish, then stops the worker. */
int ar_server_destroy(ar_server* server);
/* Non-blocking: queues the job and returns its id.  `scene` must stay alive
 * until the job finishes; `out_rgb` (W*H*3 floats; a device pointer on the
 * server's device when out_on_device != 0, else host memory) receives the image. */
int ar_job_submit(ar_server* server, const ar_scene* scene, const ar_camera_desc* camera,
                  const ar_integrator_cfg* cfg, uint32_t width, uint32_t height, float* out_rgb,
                  uint32_t out_on_device, uint64_t* job_id);
int ar_job_poll(ar_server* server, uint64_t job_id, ar_job_info* info);
/* Blocks until the job leaves PENDING/RUNNING or timeout_ms passes
 * (AR_ERR_TIMEOUT). */
int ar_job_wait(ar_server* server, uint64_t job_id, double timeout_ms, ar_job_info* info);
/* Cancels a job that has not been admitted yet (AR_ERR_NOT_FOUND otherwise). */
int ar_job_cancel(ar_server* server, uint64_t job_id);
int ar_server_get_stats(ar_server* server, ar_server_stats* out);
double ar_server_now_ms(ar_server* server);
/* Text summary of the worker's queues (pending / active / finishing jobs and
 * their progress), for diagnostics. */
int ar_server_debug_dump(ar_server* server, char* buf, uint32_t capacity);

/* ---- instrumentation (no counterpart in the reference) ---- */

/* Work counters of the last ar_render on this context. */
typedef struct ar_render_stats {
    uint64_t path_samples;           /* camera samples (GDPT: base samples) */
    uint64_t paths;                  /* traced paths (GDPT: base + offsets) */
    uint64_t extend_rays;            /* closest-hit queries */
    uint64_t shadow_rays;            /* any-hit queries */
    uint64_t extend_launches;
    uint64_t shadow_launches;
} ar_render_stats;
int ar_get_render_stats(const ar_context* ctx, ar_render_stats* out);

/* When enabled, every kernel launch of the context is bracketed by CUDA events
 * on the context stream; ar_profile_read returns, per kernel name, the launch
 * count and summed device milliseconds since the last reset. */
int ar_profile_enable(ar_context* ctx, int enable);
int ar_profile_reset(ar_context* ctx);
/* names: '\n'-separated kernel names written into `names` (capacity bytes);
 * ms/launches: arrays of `*count` entries (capacity given in *count on entry). */
int ar_profile_read(ar_context* ctx, char* names, uint32_t capacity, double* ms, uint64_t* launches,
                    uint32_t* count);

#ifdef __cplusplus
}
#endif

#endif /* AGENTRAY_H */
