// Batched bidirectional path tracer (see bdpt.cu).
#pragma once
#include <vector>

#include "ar_render.hpp"

namespace ar {

constexpr uint32_t kMaxBdptJobs = 1024;

// Per-job parameters of a BDPT batch (BdptConfig + scene + camera + film).
struct alignas(16) BdJob {
    DevScene sc;
    CameraDev cam;
    uint32_t width, height, spp, max_depth, rr_depth, mis_mode;
    float mis_beta;
    uint32_t film64;
    uint64_t seed;
    float inv_spp;
    float pad;
    void* film;
};

// Batch samples [offset, offset + nsamples) are samples
// [sample_begin, sample_begin + nsamples) of job `job` (index into the
// batch's job list).  Segments are sorted by offset and contiguous.
struct BdSegment {
    uint32_t job, offset, nsamples, pad;
    unsigned long long sample_begin;
};

struct BdptBatcher;

BdptBatcher* bdpt_create(ar_context* ctx, uint32_t max_depth_cap, uint32_t batch);
void bdpt_destroy(BdptBatcher* b);
uint32_t bdpt_batch_capacity(const BdptBatcher* b);
uint32_t bdpt_max_depth_cap(const BdptBatcher* b);
size_t bdpt_batch_bytes(uint32_t max_depth, uint32_t batch);
// Enqueues one batch on `stream` (nullptr: the context stream); returns the
// number of kernels it launched.
uint32_t bdpt_run_batch(BdptBatcher* b, const std::vector<BdJob>& jobs, const std::vector<BdSegment>& segs,
                        cudaStream_t stream = nullptr);
BdJob make_bdpt_job(const ar_scene* sc, const CameraDev& cam, const ar_integrator_cfg& cfg, uint32_t w, uint32_t h,
                    void* film);

}  // namespace ar
