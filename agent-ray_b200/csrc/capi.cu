// extern "C" entry points of libagentray (declared in include/agentray.h).
#include <algorithm>
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
    if (ctx->lane_stream) cudaStreamSynchronize(ctx->lane_stream);
    bdpt_destroy(ctx->bdpt2);
    ctx->bdpt2 = nullptr;
    for (cudaEvent_t e : ctx->lane_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->lane_stream) cudaStreamDestroy(ctx->lane_stream);
    if (ctx->copy_in) cudaStreamSynchronize(ctx->copy_in);
    if (ctx->copy_out) cudaStreamSynchronize(ctx->copy_out);
    for (cudaEvent_t e : ctx->trace_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->copy_in) cudaStreamDestroy(ctx->copy_in);
    if (ctx->copy_out) cudaStreamDestroy(ctx->copy_out);
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

// Rays per chunk of a host-array batch: 4M rays stage 128 MB of rays and
// 80 MB of hits per slot.
constexpr uint64_t kTraceChunk = 1ull << 22;

// ar_trace_closest / ar_trace_any.  Device arrays are traced in one launch on
// the context stream.  A batch with host arrays goes in chunks through two
// staging slots: a chunk's rays go up on copy_in while the previous chunk is
// traced on the context stream, and its hits come back on copy_out while the
// next one is traced, so the PCIe copies (both directions at once) hide
// behind the traversal.  Returns once host outputs are complete.
static void trace_common(ar_context* ctx, const ar_scene* scene, const ar_ray_batch* rays, bool any, ar_hit* hits,
                         uint32_t* inst, uint8_t* occ, uint32_t out_on_device) {
    AR_REQUIRE(ctx && scene && rays, AR_ERR_INVALID_ARGUMENT, "null argument");
    AR_REQUIRE(rays->count == 0 || (rays->org_tmin && rays->dir_tmax), AR_ERR_INVALID_ARGUMENT, "null ray arrays");
    AR_REQUIRE(any ? (occ != nullptr || rays->count == 0) : ((hits && inst) || rays->count == 0),
               AR_ERR_INVALID_ARGUMENT, "null output arrays");
    AR_CUDA(cudaSetDevice(ctx->device));
    const uint64_t n = rays->count;
    if (n == 0) return;
    const float4* host_o = reinterpret_cast<const float4*>(rays->org_tmin);
    const float4* host_d = reinterpret_cast<const float4*>(rays->dir_tmax);
    float4* hit_out = reinterpret_cast<float4*>(hits);
    if (rays->on_device && out_on_device) {
        launch_trace(ctx, scene, host_o, host_d, n, any, hit_out, inst, occ);
        return;
    }
    if (!ctx->copy_in) {
        AR_CUDA(cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking));
        AR_CUDA(cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking));
        for (cudaEvent_t& ev : ctx->trace_ev) AR_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    const uint64_t chunk = std::min(n, kTraceChunk);
    const int slots = n > chunk ? 2 : 1;
    const size_t in_bytes = rays->on_device ? 0 : 2 * chunk * sizeof(float4);
    const size_t out_bytes = out_on_device ? 0 : (any ? chunk : chunk * (sizeof(float4) + sizeof(uint32_t)));
    const size_t slot_bytes = ((in_bytes + out_bytes + 255) / 256) * 256 + 256;
    ctx->io.ensure(slots * slot_bytes);
    cudaEvent_t* in_done = ctx->trace_ev;        // [2]: a slot's rays are on the device
    cudaEvent_t* traced = ctx->trace_ev + 2;     // [2]: a slot's chunk is traced
    cudaEvent_t* slot_free = ctx->trace_ev + 4;  // [2]: a slot's hits are back on the host
    cudaEvent_t start = ctx->trace_ev[6];
    // staging may still be read by work queued earlier on the context stream
    AR_CUDA(cudaEventRecord(start, ctx->stream));
    AR_CUDA(cudaStreamWaitEvent(ctx->copy_in, start, 0));
    uint64_t k = 0;
    for (uint64_t off = 0; off < n; off += chunk, ++k) {
        const uint64_t m = std::min(chunk, n - off);
        const int s = int(k % 2);
        char* base = ctx->io.buf.as<char>() + s * slot_bytes;
        if (k >= 2) AR_CUDA(cudaStreamWaitEvent(ctx->copy_in, out_on_device ? traced[s] : slot_free[s], 0));
        const float4 *ot, *dt;
        if (rays->on_device) {
            ot = host_o + off;
            dt = host_d + off;
        } else {
            float4* o = reinterpret_cast<float4*>(base);
            float4* d = o + chunk;
            AR_CUDA(cudaMemcpyAsync(o, host_o + off, m * sizeof(float4), cudaMemcpyHostToDevice, ctx->copy_in));
            AR_CUDA(cudaMemcpyAsync(d, host_d + off, m * sizeof(float4), cudaMemcpyHostToDevice, ctx->copy_in));
            AR_CUDA(cudaEventRecord(in_done[s], ctx->copy_in));
            AR_CUDA(cudaStreamWaitEvent(ctx->stream, in_done[s], 0));
            ot = o;
            dt = d;
        }
        if (rays->on_device && k >= 2 && !out_on_device)
            AR_CUDA(cudaStreamWaitEvent(ctx->stream, slot_free[s], 0));
        float4* dh = nullptr;
        uint32_t* di = nullptr;
        uint8_t* dor = nullptr;
        char* outb = base + in_bytes;
        if (out_on_device) {
            dh = any ? nullptr : hit_out + off;
            di = any ? nullptr : inst + off;
            dor = any ? occ + off : nullptr;
        } else if (any) {
            dor = reinterpret_cast<uint8_t*>(outb);
        } else {
            dh = reinterpret_cast<float4*>(outb);
            di = reinterpret_cast<uint32_t*>(outb + chunk * sizeof(float4));
        }
        launch_trace(ctx, scene, ot, dt, m, any, dh, di, dor);
        AR_CUDA(cudaEventRecord(traced[s], ctx->stream));
        if (!out_on_device) {
            AR_CUDA(cudaStreamWaitEvent(ctx->copy_out, traced[s], 0));
            if (any) {
                AR_CUDA(cudaMemcpyAsync(occ + off, dor, m, cudaMemcpyDeviceToHost, ctx->copy_out));
            } else {
                AR_CUDA(cudaMemcpyAsync(hit_out + off, dh, m * sizeof(float4), cudaMemcpyDeviceToHost,
                                        ctx->copy_out));
                AR_CUDA(cudaMemcpyAsync(inst + off, di, m * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                        ctx->copy_out));
            }
            AR_CUDA(cudaEventRecord(slot_free[s], ctx->copy_out));
        }
    }
    if (!out_on_device) {
        AR_CUDA(cudaStreamSynchronize(ctx->copy_out));
        check_device_flag(ctx);  // synchronises the context stream
    } else {
        // the context stream carries on; later uploads into the staging wait for it
        AR_CUDA(cudaStreamSynchronize(ctx->copy_in));
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
