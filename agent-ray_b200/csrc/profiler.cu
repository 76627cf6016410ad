// Per-kernel CUDA-event timing (ar_profile_*) and render work counters.
#include <cstring>

#include "ar_internal.hpp"

namespace ar {

cudaEvent_t Profiler::take() {
    if (pool.empty()) {
        cudaEvent_t e;
        AR_CUDA(cudaEventCreate(&e));
        return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
}

void Profiler::begin(cudaStream_t s, const char* name) {
    Pending p{name, take(), take()};
    AR_CUDA(cudaEventRecord(p.start, s));
    pending.push_back(p);
}

void Profiler::end(cudaStream_t s) {
    if (!pending.empty()) AR_CUDA(cudaEventRecord(pending.back().stop, s));
}

void Profiler::drain() {
    for (auto& p : pending) {
        AR_CUDA(cudaEventSynchronize(p.stop));
        float ms = 0.f;
        AR_CUDA(cudaEventElapsedTime(&ms, p.start, p.stop));
        Total* t = nullptr;
        for (auto& x : totals)
            if (x.name == p.name) t = &x;
        if (!t) {
            totals.push_back(Total{p.name, 0.0, 0});
            t = &totals.back();
        }
        t->ms += ms;
        t->launches++;
        pool.push_back(p.start);
        pool.push_back(p.stop);
    }
    pending.clear();
}

Profiler::~Profiler() {
    for (auto& p : pending) {
        cudaEventDestroy(p.start);
        cudaEventDestroy(p.stop);
    }
    for (auto e : pool) cudaEventDestroy(e);
}

}  // namespace ar

using namespace ar;

extern "C" {

int ar_profile_enable(ar_context* ctx, int enable) {
    return guarded([&] {
        AR_REQUIRE(ctx, AR_ERR_INVALID_ARGUMENT, "ctx is null");
        ctx->prof.on = enable != 0;
    });
}

int ar_profile_reset(ar_context* ctx) {
    return guarded([&] {
        AR_REQUIRE(ctx, AR_ERR_INVALID_ARGUMENT, "ctx is null");
        ctx->prof.drain();
        ctx->prof.totals.clear();
    });
}

int ar_profile_read(ar_context* ctx, char* names, uint32_t capacity, double* ms, uint64_t* launches,
                    uint32_t* count) {
    return guarded([&] {
        AR_REQUIRE(ctx && names && ms && launches && count, AR_ERR_INVALID_ARGUMENT, "null argument");
        ctx->prof.drain();
        std::string all;
        uint32_t n = 0;
        for (auto& t : ctx->prof.totals) {
            if (n >= *count) break;
            all += t.name;
            all += '\n';
            ms[n] = t.ms;
            launches[n] = t.launches;
            n++;
        }
        AR_REQUIRE(all.size() + 1 <= capacity, AR_ERR_INVALID_ARGUMENT, "names buffer too small");
        std::memcpy(names, all.c_str(), all.size() + 1);
        *count = n;
    });
}

int ar_get_render_stats(const ar_context* ctx, ar_render_stats* out) {
    return guarded([&] {
        AR_REQUIRE(ctx && out, AR_ERR_INVALID_ARGUMENT, "null argument");
        ar_context* c = const_cast<ar_context*>(ctx);
        if (c->stats_pending) {
            AR_CUDA(cudaStreamSynchronize(c->stream));
            c->last_stats.paths = c->stats_h[0];
            c->last_stats.extend_rays = c->stats_h[1];
            c->last_stats.shadow_rays = c->stats_h[2];
            c->stats_pending = false;
        }
        *out = c->last_stats;
    });
}

}  // extern "C"
