// Project autotuner (ar_autotune) and the context tuning accessors.
//
// The search space is what the wavefront kernels leave open at run time: the
// persistent traversal grid (blocks per SM; the block shape is fixed at 128
// threads by the traversal launch bounds), the shading stage's block size,
// the queue capacities (PT/GDPT path slots, BDPT batch memory) and the
// wide-BVH build (SAH node cost, children per node, triangles per leaf).  Coordinate
// descent: each knob in turn is swept with the others at their current best,
// every candidate timed as the median of `repeats` renders of the workload
// with CUDA events on the context's stream, after one untimed render.
#include <algorithm>
#include <vector>

#include "ar_internal.hpp"
#include "ar_render.hpp"

namespace ar {

void build_scene_accel(ar_scene* s, const ar_accel_opts* o);
void check_device_flag(ar_context* ctx);

namespace {

ar_tuning get_tuning(const ar_context* ctx) {
    ar_tuning t{};
    t.path_capacity = ctx->engine_capacity;
    t.traversal_blocks_per_sm = ctx->trav_blocks_per_sm;
    t.shade_block = ctx->shade_block;
    t.bdpt_batch_mib = uint32_t(ctx->bdpt_budget >> 20);
    return t;
}

void set_tuning(ar_context* ctx, const ar_tuning& t) {
    const uint32_t cap = t.path_capacity ? t.path_capacity : (1u << 22);
    const uint32_t tb = t.traversal_blocks_per_sm ? t.traversal_blocks_per_sm : 8u;
    const uint32_t sb = t.shade_block ? t.shade_block : 256u;
    const uint32_t mib = t.bdpt_batch_mib ? t.bdpt_batch_mib : 12288u;
    AR_REQUIRE(cap >= 4096 && cap <= (1u << 26), AR_ERR_INVALID_ARGUMENT, "path_capacity must be in [4096, 2^26]");
    AR_REQUIRE(tb >= 1 && tb <= 8, AR_ERR_INVALID_ARGUMENT, "traversal_blocks_per_sm must be 1..8");
    AR_REQUIRE(sb == 64 || sb == 128 || sb == 256, AR_ERR_INVALID_ARGUMENT, "shade_block must be 64, 128 or 256");
    AR_REQUIRE(mib >= 64 && mib <= (1u << 20), AR_ERR_INVALID_ARGUMENT, "bdpt_batch_mib must be in [64, 2^20]");
    AR_CUDA(cudaStreamSynchronize(ctx->stream));
    if (cap != ctx->engine_capacity || tb != ctx->trav_blocks_per_sm || sb != ctx->shade_block) {
        engine_destroy(ctx->engine);  // its captured tick graphs hold the old launch shapes
        ctx->engine = nullptr;
    }
    if ((size_t(mib) << 20) != ctx->bdpt_budget) {
        bdpt_destroy(ctx->bdpt);
        ctx->bdpt = nullptr;
        if (ctx->lane_stream) AR_CUDA(cudaStreamSynchronize(ctx->lane_stream));
        bdpt_destroy(ctx->bdpt2);
        ctx->bdpt2 = nullptr;
    }
    ctx->engine_capacity = cap;
    ctx->trav_blocks_per_sm = tb;
    ctx->shade_block = sb;
    ctx->bdpt_budget = size_t(mib) << 20;
}

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    Timer() {
        AR_CUDA(cudaEventCreate(&a));
        AR_CUDA(cudaEventCreate(&b));
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

// Median device time of `reps` renders after one untimed render.
double time_render(ar_context* ctx, const ar_scene* sc, const ar_camera_desc& cam, const ar_integrator_cfg& cfg,
                   uint32_t w, uint32_t h, float* out, uint32_t reps, Timer& tm) {
    render(ctx, sc, cam, cfg, w, h, out, true);
    AR_CUDA(cudaStreamSynchronize(ctx->stream));
    check_device_flag(ctx);
    std::vector<double> t;
    for (uint32_t r = 0; r < reps; ++r) {
        AR_CUDA(cudaEventRecord(tm.a, ctx->stream));
        render(ctx, sc, cam, cfg, w, h, out, true);
        AR_CUDA(cudaEventRecord(tm.b, ctx->stream));
        AR_CUDA(cudaEventSynchronize(tm.b));
        float ms = 0.f;
        AR_CUDA(cudaEventElapsedTime(&ms, tm.a, tm.b));
        t.push_back(ms);
    }
    check_device_flag(ctx);
    std::sort(t.begin(), t.end());
    return t[t.size() / 2];
}

bool same_accel(const ar_accel_opts& a, const ar_accel_opts& b) {
    const auto width = [](uint32_t w) { return w ? w : 8u; };
    const auto leaf = [](uint32_t l) { return l ? l : 3u; };
    const auto cost = [](float c) { return c > 0.f ? c : 0.5f; };
    return width(a.bvh_width) == width(b.bvh_width) && leaf(a.max_leaf_size) == leaf(b.max_leaf_size) &&
           a.sah_bins == b.sah_bins && cost(a.sah_node_cost) == cost(b.sah_node_cost);
}

void autotune(ar_context* ctx, ar_scene* sc, const ar_camera_desc& cam, const ar_tune_opts& o, ar_tune_result& r) {
    AR_REQUIRE(o.integrator == AR_INTEGRATOR_PT || o.integrator == AR_INTEGRATOR_BDPT ||
                   o.integrator == AR_INTEGRATOR_GDPT,
               AR_ERR_INVALID_ARGUMENT, "unknown integrator");
    const uint32_t w = o.width ? o.width : 256, h = o.height ? o.height : 256;
    const uint32_t reps = o.repeats ? o.repeats : 3;
    ar_integrator_cfg cfg{};
    cfg.integrator = o.integrator;
    cfg.spp = o.spp ? o.spp : 4;
    cfg.max_depth = o.max_depth ? o.max_depth : 8;
    cfg.rr_depth = 3;
    cfg.mis_mode = AR_MIS_POWER;
    cfg.mis_beta = 2.0f;
    cfg.alpha = 0.2f;
    cfg.poisson_iterations = 200;
    cfg.sor_omega = 1.6f;
    cfg.poisson_solver = AR_POISSON_SOR;
    cfg.poisson_tolerance = 1e-6;
    cfg.seed = 1;
    DevBuf out;
    out.alloc(size_t(w) * h * 3 * sizeof(float));
    Timer tm;
    ar_tuning best = get_tuning(ctx);
    ar_accel_opts best_accel = sc->accel;
    const auto run = [&]() { return time_render(ctx, sc, cam, cfg, w, h, out.as<float>(), reps, tm); };
    double best_ms = run();
    r.default_ms = best_ms;
    r.candidates = 1;
    const double kGain = 0.99;  // a candidate must win by 1% to move

    if (o.tune_accel) {
        const auto try_accel = [&](const ar_accel_opts& a) {
            if (same_accel(a, best_accel)) return;
            build_scene_accel(sc, &a);
            const double ms = run();
            r.candidates++;
            if (ms < best_ms * kGain) {
                best_ms = ms;
                best_accel = a;
            }
        };
        for (const float cost : {0.5f, 1.0f, 2.0f}) {
            ar_accel_opts a = best_accel;
            a.sah_node_cost = cost;
            try_accel(a);
        }
        for (const uint32_t width : {8u, 6u, 4u}) {
            for (const uint32_t leaf : {4u, 3u, 2u, 1u}) {
                ar_accel_opts a = best_accel;
                a.bvh_width = width;
                a.max_leaf_size = leaf;
                try_accel(a);
            }
        }
        if (!same_accel(sc->accel, best_accel)) build_scene_accel(sc, &best_accel);
    }
    const auto sweep = [&](uint32_t ar_tuning::*field, std::initializer_list<uint32_t> values) {
        for (const uint32_t v : values) {
            if (best.*field == v) continue;
            ar_tuning t = best;
            t.*field = v;
            set_tuning(ctx, t);
            const double ms = run();
            r.candidates++;
            if (ms < best_ms * kGain) {
                best_ms = ms;
                best = t;
            }
        }
        set_tuning(ctx, best);
    };
    sweep(&ar_tuning::traversal_blocks_per_sm, {8u, 6u, 4u});
    sweep(&ar_tuning::shade_block, {256u, 128u, 64u});
    if (o.integrator == AR_INTEGRATOR_BDPT)
        sweep(&ar_tuning::bdpt_batch_mib, {3072u, 6144u, 12288u, 24576u});
    else
        sweep(&ar_tuning::path_capacity, {1u << 20, 1u << 21, 1u << 22, 1u << 23});
    r.tuning = best;
    r.accel = best_accel;
    r.best_ms = best_ms;
}

}  // namespace
}  // namespace ar

using namespace ar;

extern "C" {

int ar_context_get_tuning(const ar_context* ctx, ar_tuning* out) {
    return guarded([&] {
        AR_REQUIRE(ctx && out, AR_ERR_INVALID_ARGUMENT, "null argument");
        *out = get_tuning(ctx);
    });
}

int ar_context_set_tuning(ar_context* ctx, const ar_tuning* t) {
    return guarded([&] {
        AR_REQUIRE(ctx && t, AR_ERR_INVALID_ARGUMENT, "null argument");
        AR_CUDA(cudaSetDevice(ctx->device));
        set_tuning(ctx, *t);
    });
}

int ar_autotune(ar_context* ctx, ar_scene* scene, const ar_camera_desc* camera, const ar_tune_opts* opts,
                ar_tune_result* out) {
    return guarded([&] {
        AR_REQUIRE(ctx && scene && camera && opts && out, AR_ERR_INVALID_ARGUMENT, "null argument");
        AR_CUDA(cudaSetDevice(ctx->device));
        AR_CUDA(cudaStreamSynchronize(ctx->stream));
        ar_tune_result r{};
        autotune(ctx, scene, *camera, *opts, r);
        *out = r;
    });
}

}  // extern "C"
