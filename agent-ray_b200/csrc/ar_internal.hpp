// Host-side internals of libagentray: context, scene handle, error plumbing.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/agentray.h"
#include "ar_types.h"
#include "bvh_build.hpp"

namespace ar {

// Thread-local last-error message (ar_last_error).
void set_error(const std::string& msg);

struct ArError {
    int code;
    std::string msg;
};

#define AR_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw ::ar::ArError{AR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

#define AR_REQUIRE(cond, code, msg)                  \
    do {                                             \
        if (!(cond)) throw ::ar::ArError{code, msg}; \
    } while (0)

// Runs `f` and converts exceptions into an ar_status.
template <class F>
int guarded(F&& f) {
    try {
        f();
        return AR_OK;
    } catch (const ArError& e) {
        set_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return AR_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_error(e.what());
        return AR_ERR_INTERNAL;
    }
}

// Fails with AR_ERR_INVALID_ARGUMENT unless `p` is device (or managed) memory
// that `device` can address: a host pointer or another GPU's buffer handed to
// a kernel would fault the GPU instead of returning an error.  Allocates
// nothing; safe during stream capture.
inline void require_device_ptr(const void* p, int device, const char* what) {
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw ArError{AR_ERR_INVALID_ARGUMENT, std::string(what) + ": not a CUDA pointer"};
    }
    const bool dev = a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
    if (!dev || (a.type == cudaMemoryTypeDevice && a.device != device))
        throw ArError{AR_ERR_INVALID_ARGUMENT,
                      std::string(what) + ": not device memory of device " + std::to_string(device)};
}

// Device buffer owned by a scene or context.
struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    void alloc(size_t n);
    void free();
    template <class T>
    T* as() const { return static_cast<T*>(ptr); }
    ~DevBuf() { free(); }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

// Grow-only device scratch arena (wavefront queues, films).
struct Workspace {
    DevBuf buf;
    size_t need = 0;
    void ensure(size_t bytes);
};

}  // namespace ar

namespace ar {

struct PathEngine;
void engine_destroy(PathEngine* e);
struct BdptBatcher;
void bdpt_destroy(BdptBatcher* b);

// Optional per-kernel CUDA-event timing on the context stream.
struct Profiler {
    bool on = false;
    struct Pending {
        const char* name;
        cudaEvent_t start, stop;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    struct Total {
        std::string name;
        double ms = 0;
        uint64_t launches = 0;
    };
    std::vector<Total> totals;
    cudaEvent_t take();
    void begin(cudaStream_t s, const char* name);
    void end(cudaStream_t s);
    void drain();  // synchronises on pending events and folds them into totals
    ~Profiler();
};

// RAII bracket around one kernel launch.
struct KernelScope {
    Profiler& p;
    cudaStream_t s;
    KernelScope(Profiler& prof, cudaStream_t st, const char* name) : p(prof), s(st) {
        if (p.on) p.begin(s, name);
    }
    ~KernelScope() {
        if (p.on) p.end(s);
    }
};

}  // namespace ar

struct ar_context {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    ar::DevBuf err_flag;      // int: device-side error flag (stack overflow, budget)
    ar::DevBuf stats_d;       // uint64[8]: render work counters
    ar::DevBuf fetch;         // uint32: ray-fetch cursor of the batched trace launches
    ar::Workspace work;       // wavefront state
    ar::Workspace io;         // staging for host <-> device transfers
    ar::Workspace films;      // accumulation films of the current render
    ar::Workspace solver;     // Poisson solver buffers
    ar::Profiler prof;
    uint64_t* stats_h = nullptr;  // pinned copy of stats_d, valid after a sync
    ar_render_stats last_stats{};
    bool stats_pending = false;
    ar::PathEngine* engine = nullptr;  // streaming wavefront engine for ar_render
    uint32_t engine_capacity = 1u << 22;
    // launch shapes (ar_tuning)
    uint32_t trav_blocks_per_sm = 8;       // persistent traversal grid, blocks per SM
    uint32_t shade_block = 256;            // threads per block of the shading stage
    size_t bdpt_budget = size_t(12) << 30;  // HBM for one plain-path BDPT batch
    // samples [range_begin, range_end) of each pixel for the next render
    // (ar_render_samples); range_end == 0 renders all spp samples
    uint32_t range_begin = 0, range_end = 0;
    ar::BdptBatcher* bdpt = nullptr;   // BDPT batch buffers for ar_render
    // second BDPT lane of ar_render: its batch buffers and stream, and the
    // events that fork it from and join it to the context stream
    ar::BdptBatcher* bdpt2 = nullptr;
    cudaStream_t lane_stream = nullptr;
    cudaEvent_t lane_ev[2] = {};
    // Host-array ray batches (ar_trace_*): copy streams and events that let the
    // copies of one chunk overlap the traversal of the previous one.
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    cudaEvent_t trace_ev[7] = {};
};

struct ar_scene {
    int device = 0;
    // host copies needed for (re)builds
    struct MeshHost {
        std::vector<float> pos;
        std::vector<uint32_t> idx;
        bool has_normals = false;
        uint32_t ntri = 0;
    };
    std::vector<MeshHost> meshes;
    std::vector<ar_object_desc> objects;
    std::vector<std::vector<uint32_t>> object_mats;
    std::vector<float> light_power_weights;
    // device data
    ar::DevBuf nodes, tris, instances, objects_d, meshes_d, indices, normals, slots, mat_table, materials, lights,
        light_cdf, light_pmf, texcoords, texels, textures;
    ar::DevScene view{};
    ar_scene_stats stats{};
    ar_accel_opts accel{};  // options of the last build
    std::vector<ar::LightRecord> lights_h;
    std::vector<ar::MaterialRecord> materials_h;
    uint32_t light_dist = 0;
    std::vector<float> cdf_h, pmf_h;
};
