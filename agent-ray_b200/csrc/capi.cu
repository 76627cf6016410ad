// extern "C" entry points of libagentray (declared in include/agentray.h).
#include <cstring>
#include <memory>
#include <string>

#include "ar_internal.hpp"
#include "ar_render.hpp"

namespace ar {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

void create_scene(ar_context* ctx, const ar_scene_desc* d, ar_scene** out);
void build_scene_accel(ar_scene* s, const ar_accel_opts* o);
void launch_trace(ar_context* ctx, const ar_scene* sc, const float4* ot, const float4* dt, uint64_t n, bool any,
                  float4* hits, uint32_t* inst, uint8_t* occ);

// Checks the device error flag after a synchronisation.
void check_device_flag(ar_context* ctx) {
    int flag = 0;
    AR_CUDA(cudaMemcpyAsync(&flag, ctx->err_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    AR_CUDA(cudaStreamSynchronize(ctx->stream));
    if (flag) {
        AR_CUDA(cudaMemsetAsync(ctx->err_flag.ptr, 0, sizeof(int), ctx->stream));
        AR_CUDA(cudaStreamSynchronize(ctx->stream));
        throw ArError{flag == 2 ? AR_ERR_TIMEOUT : AR_ERR_INTERNAL,
                      flag == 1   ? "traversal stack overflow"
                      : flag == 3 ? "traversal step budget exceeded"
                      : flag == 4 ? "BDPT connection queue overflow"
                                  : "device work budget exceeded"};
    }
}

ar_context* context_create_internal(int device) {
    int count = 0;
    AR_CUDA(cudaGetDeviceCount(&count));
    AR_REQUIRE(device >= 0 && device < count, AR_ERR_INVALID_ARGUMENT, "no such CUDA device");
    AR_CUDA(cudaSetDevice(device));
    auto ctx = std::make_unique<ar_context>();
    ctx->device = device;
    AR_CUDA(cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
    ctx->stream = ctx->own_stream;
    AR_CUDA(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
    ctx->err_flag.alloc(64);
    AR_CUDA(cudaMemset(ctx->err_flag.ptr, 0, 64));
    ctx->fetch.alloc(256);
    ctx->stats_d.alloc(8 * sizeof(uint64_t));
    AR_CUDA(cudaMemset(ctx->stats_d.ptr, 0, 8 * sizeof(uint64_t)));
    AR_CUDA(cudaMallocHost(&ctx->stats_h, 8 * sizeof(uint64_t)));
    std::memset(ctx->stats_h, 0, 8 * sizeof(uint64_t));
    return ctx.release();
}

void context_destroy_internal(ar_context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->engine) engine_destroy(ctx->engine);
    ctx->engine = nullptr;
    bdpt_destroy(ctx->bdpt);
    ctx->bdpt = nullptr;
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    if (ctx->stats_h) cudaFreeHost(ctx->stats_h);
    delete ctx;
}

}  // namespace ar

using namespace ar;

extern "C" {

const char* ar_last_error(void) { return g_last_error.c_str(); }

int ar_abi_version(void) { return AR_ABI_VERSION; }

int ar_context_create(int device, ar_context** out) {
    return guarded([&] {
        AR_REQUIRE(out, AR_ERR_INVALID_ARGUMENT, "out is null");
        *out = context_create_internal(device);
    });
}

int ar_context_destroy(ar_context* ctx) {
    return guarded([&] { context_destroy_internal(ctx); });
}

int ar_context_set_stream(ar_context* ctx, void* stream) {
    return guarded([&] {
        AR_REQUIRE(ctx, AR_ERR_INVALID_ARGUMENT, "ctx is null");
        ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    });
}

int ar_context_synchronize(ar_context* ctx) {
    return guarded([&] {
        AR_REQUIRE(ctx, AR_ERR_INVALID_ARGUMENT, "ctx is null");
        AR_CUDA(cudaStreamSynchronize(ctx->stream));
        check_device_flag(ctx);
    });
}

int ar_scene_create(ar_context* ctx, const ar_scene_desc* desc, ar_scene** out) {
    return guarded([&] { create_scene(ctx, desc, out); });
}

int ar_scene_destroy(ar_scene* scene) {
    return guarded([&] {
        if (!scene) return;
        cudaSetDevice(scene->device);
        delete scene;
    });
}

int ar_scene_build_accel(ar_context* ctx, ar_scene* scene, const ar_accel_opts* opts) {
    return guarded([&] {
        AR_REQUIRE(ctx && scene, AR_ERR_INVALID_ARGUMENT, "null argument");
        AR_CUDA(cudaSetDevice(ctx->device));
        AR_CUDA(cudaStreamSynchronize(ctx->stream));
        build_scene_accel(scene, opts);
    });
}

int ar_scene_get_stats(const ar_scene* scene, ar_scene_stats* out) {
    return guarded([&] {
        AR_REQUIRE(scene && out, AR_ERR_INVALID_ARGUMENT, "null argument");
        *out = scene->stats;
    });
}

static void trace_common(ar_context* ctx, const ar_scene* scene, const ar_ray_batch* rays, bool any, ar_hit* hits,
                         uint32_t* inst, uint8_t* occ, uint32_t out_on_device) {
    AR_REQUIRE(ctx && scene && rays, AR_ERR_INVALID_ARGUMENT, "null argument");
    AR_REQUIRE(rays->count == 0 || (rays->org_tmin && rays->dir_tmax), AR_ERR_INVALID_ARGUMENT, "null ray arrays");
    AR_REQUIRE(any ? (occ != nullptr || rays->count == 0) : ((hits && inst) || rays->count == 0),
               AR_ERR_INVALID_ARGUMENT, "null output arrays");
    AR_CUDA(cudaSetDevice(ctx->device));
    const uint64_t n = rays->count;
    if (n == 0) return;
    const size_t ray_bytes = n * sizeof(float4);
    const size_t out_bytes = any ? n : n * (sizeof(float4) + sizeof(uint32_t));
    size_t need = (rays->on_device ? 0 : 2 * ray_bytes) + (out_on_device ? 0 : out_bytes + 256);
    ctx->io.ensure(need + 512);
    char* base = ctx->io.buf.as<char>();
    const float4 *ot, *dt;
    size_t off = 0;
    if (rays->on_device) {
        ot = reinterpret_cast<const float4*>(rays->org_tmin);
        dt = reinterpret_cast<const float4*>(rays->dir_tmax);
    } else {
        float4* o = reinterpret_cast<float4*>(base);
        float4* d = reinterpret_cast<float4*>(base + ray_bytes);
        AR_CUDA(cudaMemcpyAsync(o, rays->org_tmin, ray_bytes, cudaMemcpyHostToDevice, ctx->stream));
        AR_CUDA(cudaMemcpyAsync(d, rays->dir_tmax, ray_bytes, cudaMemcpyHostToDevice, ctx->stream));
        ot = o;
        dt = d;
        off = 2 * ray_bytes;
    }
    float4* dh = nullptr;
    uint32_t* di = nullptr;
    uint8_t* dor = nullptr;
    if (out_on_device) {
        dh = reinterpret_cast<float4*>(hits);
        di = inst;
        dor = occ;
    } else if (any) {
        dor = reinterpret_cast<uint8_t*>(base + off);
    } else {
        dh = reinterpret_cast<float4*>(base + off);
        di = reinterpret_cast<uint32_t*>(base + off + n * sizeof(float4));
    }
    launch_trace(ctx, scene, ot, dt, n, any, dh, di, dor);
    if (!out_on_device) {
        if (any) {
            AR_CUDA(cudaMemcpyAsync(occ, dor, n, cudaMemcpyDeviceToHost, ctx->stream));
        } else {
            AR_CUDA(cudaMemcpyAsync(hits, dh, n * sizeof(float4), cudaMemcpyDeviceToHost, ctx->stream));
            AR_CUDA(cudaMemcpyAsync(inst, di, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
        }
        check_device_flag(ctx);  // synchronises
    }
}

int ar_trace_closest(ar_context* ctx, const ar_scene* scene, const ar_ray_batch* rays, ar_hit* hits,
                     uint32_t* inst_ids, uint32_t out_on_device) {
    return guarded([&] { trace_common(ctx, scene, rays, false, hits, inst_ids, nullptr, out_on_device); });
}

int ar_trace_any(ar_context* ctx, const ar_scene* scene, const ar_ray_batch* rays, uint8_t* occluded,
                 uint32_t out_on_device) {
    return guarded([&] { trace_common(ctx, scene, rays, true, nullptr, nullptr, occluded, out_on_device); });
}

int ar_render(ar_context* ctx, const ar_scene* scene, const ar_camera_desc* camera, const ar_integrator_cfg* cfg,
              uint32_t width, uint32_t height, float* out_rgb, uint32_t out_on_device) {
    return guarded([&] {
        AR_REQUIRE(ctx && scene && camera && cfg && out_rgb, AR_ERR_INVALID_ARGUMENT, "null argument");
        AR_REQUIRE(width > 0 && height > 0, AR_ERR_INVALID_ARGUMENT, "empty image");
        AR_REQUIRE(cfg->spp > 0, AR_ERR_INVALID_ARGUMENT, "spp must be positive");
        AR_CUDA(cudaSetDevice(ctx->device));
        render(ctx, scene, *camera, *cfg, width, height, out_rgb, out_on_device != 0);
    });
}

int ar_render_samples(ar_context* ctx, const ar_scene* scene, const ar_camera_desc* camera,
                      const ar_integrator_cfg* cfg, uint32_t width, uint32_t height, uint32_t sample_begin,
                      uint32_t sample_end, float* out_rgb, uint32_t out_on_device) {
    return guarded([&] {
        AR_REQUIRE(ctx && scene && camera && cfg && out_rgb, AR_ERR_INVALID_ARGUMENT, "null argument");
        AR_REQUIRE(width > 0 && height > 0, AR_ERR_INVALID_ARGUMENT, "empty image");
        AR_REQUIRE(cfg->spp > 0, AR_ERR_INVALID_ARGUMENT, "spp must be positive");
        AR_REQUIRE(sample_begin < sample_end && sample_end <= cfg->spp, AR_ERR_INVALID_ARGUMENT,
                   "sample range must be a non-empty part of [0, spp)");
        AR_REQUIRE(cfg->integrator != AR_INTEGRATOR_GDPT, AR_ERR_INVALID_ARGUMENT,
                   "GDPT reconstructs from all samples: shard PT or BDPT");
        AR_CUDA(cudaSetDevice(ctx->device));
        struct Reset {
            ar_context* c;
            ~Reset() { c->range_begin = c->range_end = 0; }
        } reset{ctx};
        ctx->range_begin = sample_begin;
        ctx->range_end = sample_end;
        render(ctx, scene, *camera, *cfg, width, height, out_rgb, out_on_device != 0);
    });
}

int ar_poisson_reconstruct(ar_context* ctx, const ar_integrator_cfg* cfg, uint32_t width, uint32_t height,
                           const float* primal, const float* grad_x, const float* grad_y, float* out,
                           uint32_t on_device, double* rel_residual) {
    return guarded([&] {
        AR_REQUIRE(ctx && cfg && primal && grad_x && grad_y && out, AR_ERR_INVALID_ARGUMENT, "null argument");
        AR_REQUIRE(width > 0 && height > 0, AR_ERR_INVALID_ARGUMENT, "empty image");
        // the solver kernels index interleaved RGB planes with 32-bit offsets
        AR_REQUIRE(uint64_t(width) * height * 3 <= UINT32_MAX, AR_ERR_INVALID_ARGUMENT,
                   "image too large for the Poisson solver (W*H*3 must fit in 32 bits)");
        AR_CUDA(cudaSetDevice(ctx->device));
        const size_t count = size_t(width) * height * 3;
        if (on_device) {
            require_device_ptr(primal, ctx->device, "primal");
            require_device_ptr(grad_x, ctx->device, "grad_x");
            require_device_ptr(grad_y, ctx->device, "grad_y");
            require_device_ptr(out, ctx->device, "out");
            poisson_reconstruct(ctx, *cfg, width, height, primal, grad_x, grad_y, out, rel_residual);
            return;
        }
        DevBuf tmp;
        tmp.alloc(4 * count * sizeof(float));
        float* d = tmp.as<float>();
        AR_CUDA(cudaMemcpyAsync(d, primal, count * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        AR_CUDA(cudaMemcpyAsync(d + count, grad_x, count * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        AR_CUDA(cudaMemcpyAsync(d + 2 * count, grad_y, count * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        poisson_reconstruct(ctx, *cfg, width, height, d, d + count, d + 2 * count, d + 3 * count, rel_residual);
        AR_CUDA(cudaMemcpyAsync(out, d + 3 * count, count * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        AR_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

}  // extern "C"
