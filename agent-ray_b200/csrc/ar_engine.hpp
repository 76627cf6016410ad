// Streaming wavefront engine for path-traced jobs (PT and GDPT paths).
//
// A fixed capacity of path slots is refilled every tick from a device-side job
// table, so paths of many render jobs (different scenes, cameras,
// resolutions, spp) share the same kernels and the wavefront never drains
// between bounces.  One tick:
//
//   plan      (1 block)   free slots -> samples taken from active jobs, FIFO
//   generate              new camera paths appended after the continuing ones
//   extend                closest hit
//   shade                 emission, NEE shadow ray, BSDF sample, roulette;
//                         continuing paths are compacted into the other buffer
//   shadow                any hit; visible NEE contributions; finished paths
//                         deposit into their job's film
//
// The tick is captured once per buffer parity as a CUDA graph and replayed.
#pragma once
#include <utility>
#include <vector>

#include "ar_render.hpp"

namespace ar {

constexpr uint32_t kMaxActiveJobs = 1024;
// Kernels in one tick: plan, generate, extend, shade, shadow.
constexpr uint32_t kEngineTickKernels = 5;

// Device job-table entry.
struct alignas(16) JobDev {
    DevScene sc;
    CameraDev cam;
    uint32_t width, height, spp, max_depth, rr_depth, gdpt, film64, roles;
    uint64_t seed;
    float inv_spp;
    float pad0;
    void* film[3];
    unsigned long long total_samples;  // W*H*spp
    unsigned long long next_sample;    // generation cursor (advanced by the plan kernel)
    unsigned long long total_paths;    // samples * roles
    unsigned long long done_paths;     // finished (deposited) paths
};

struct PathEngine;

// Creates an engine with `capacity` path slots on the context's device.
PathEngine* engine_create(ar_context* ctx, uint32_t capacity);
void engine_destroy(PathEngine* e);
// Registers a job in slot `slot` of the device job table (host -> device copy
// on the engine stream) and makes it active.  The films must be zeroed.
void engine_add_job(PathEngine* e, uint32_t slot, const JobDev& job);
// Removes a finished job from the active list.
void engine_remove_job(PathEngine* e, uint32_t slot);
// Batched form of the two calls above: one staged upload for many changes.
// The tick plan serves jobs past their equal share in the order of the active
// list: `order`, when given, is that list (a permutation of the active slots
// after the changes); otherwise the slots are sorted by total paths, ties in
// arrival order.  Returns the bytes copied host -> device.
size_t engine_update(PathEngine* e, const std::vector<std::pair<uint32_t, JobDev>>& adds,
                     const std::vector<uint32_t>& removes, const std::vector<uint32_t>* order = nullptr);
// Enqueues one tick (graph replay) on the context stream.
void engine_tick(PathEngine* e);
// Enqueues an async copy of every job's done_paths into pinned host memory;
// returns the host array (valid after the stream reaches this point).
const unsigned long long* engine_snapshot_done(PathEngine* e);
// The pinned array engine_snapshot_done fills (read it after the copy completes).
const unsigned long long* engine_snapshot_host(const PathEngine* e);
// Number of ticks issued so far, path statistics.
uint64_t engine_ticks(const PathEngine* e);
uint32_t engine_capacity(const PathEngine* e);
bool engine_has_active(const PathEngine* e);
// Enqueue a copy of the counters (paths generated, extend rays, shadow rays).
void engine_stats(PathEngine* e, unsigned long long* out3_pinned);

}  // namespace ar
