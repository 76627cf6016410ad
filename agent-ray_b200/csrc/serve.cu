// Render server: continuous batching of render jobs into shared wavefront
// kernels (ar_server_* / ar_job_* in include/agentray.h).
//
// One worker thread owns two internal contexts (streams) on the device:
//   * the PT stream runs the streaming path engine (PT and GDPT jobs); every
//     admitted job's samples flow into the same path pool, free slots split
//     in equal shares among the jobs with samples left, the rest oldest first;
//   * the BDPT stream runs sample batches that mix every active BDPT job,
//     split the same way.
// Admission is FIFO under an HBM budget for job films; completion is detected
// from pinned snapshots of the per-job done counters (PT) or batch events
// (BDPT), then the film is converted (GDPT: Poisson-reconstructed) and copied
// to the caller's host or device buffer before the job reports DONE.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ar_bdpt.hpp"
#include "ar_engine.hpp"

namespace ar {

ar_context* context_create_internal(int device);
void context_destroy_internal(ar_context* ctx);

namespace {

// Device buffers for job films and staging: size classes of 1 MiB steps,
// recycled per class, carved from 256 MiB (or larger) arena chunks, so that a
// burst of admissions costs one cudaMalloc per chunk rather than two per job
// (cudaMalloc can stall the device's queued work), and none once the pool has
// served the peak load.
class DevicePool {
  public:
    void* get(size_t bytes) {
        bytes = round(bytes);
        auto& v = free_[bytes];
        if (!v.empty()) {
            void* p = v.back();
            v.pop_back();
            return p;
        }
        if (chunks_.empty() || used_ + bytes > chunk_bytes_) {
            const size_t n = std::max(kChunk, bytes);
            void* c = nullptr;
            const cudaError_t e = cudaMalloc(&c, n);
            if (e != cudaSuccess)
                throw ArError{AR_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
            chunks_.push_back(c);
            chunk_bytes_ = n;
            used_ = 0;
        }
        void* p = static_cast<char*>(chunks_.back()) + used_;
        used_ += bytes;
        return p;
    }
    void put(void* p, size_t bytes) {
        if (p) free_[round(bytes)].push_back(p);
    }
    ~DevicePool() {
        for (void* c : chunks_) cudaFree(c);
    }
    static size_t round(size_t b) { return (b + (1u << 20) - 1) & ~size_t((1u << 20) - 1); }

  private:
    static constexpr size_t kChunk = size_t(256) << 20;
    std::map<size_t, std::vector<void*>> free_;
    std::vector<void*> chunks_;
    size_t chunk_bytes_ = 0, used_ = 0;
};

enum class Kind { PathTraced, Bidirectional };

struct SJob {
    uint64_t id = 0;
    const ar_scene* scene = nullptr;
    ar_camera_desc cam{};
    ar_integrator_cfg cfg{};
    uint32_t w = 0, h = 0;
    float* out = nullptr;
    bool out_on_device = false;
    Kind kind = Kind::PathTraced;
    // shared with API threads (guarded by the server mutex)
    uint32_t status = AR_JOB_PENDING;
    int32_t error = 0;
    double t_submit = 0, t_admit = 0, t_done = 0;
    uint64_t samples = 0;
    // worker-owned
    void* films = nullptr;
    size_t films_bytes = 0;
    void* scratch = nullptr;  // f32 output (and f32 copies of GDPT films)
    size_t scratch_bytes = 0;
    uint32_t slot = kInvalid;
    uint64_t total_paths = 0;
    uint64_t bd_next = 0;
    uint32_t bd_outstanding = 0;  // issued BDPT batches of this job not yet complete
    uint64_t min_snap = 0;  // first done-counter snapshot issued after admission
    uint64_t last_done = 0; // done paths seen in the last snapshot (diagnostics)
    bool bd_issued = false;
    cudaEvent_t fin = nullptr;
    cudaStream_t fin_stream = nullptr;
};

}  // namespace

struct ServerImpl {
    int device = 0;
    ar_server_opts opts{};
    // BDPT batches run on two lanes (context + batch buffers), each with one
    // batch in flight: the stage tails of one batch (the last rays of a depth,
    // the connection and shadow stages) overlap the other's work.  Lane 0's
    // stream also carries the BDPT films' clears and the results.
    static constexpr int kBdLanes = 2;
    ar_context* ctx_pt = nullptr;
    ar_context* ctx_bd[kBdLanes] = {};
    PathEngine* engine = nullptr;
    BdptBatcher* bdpt[kBdLanes] = {};
    DevicePool pool;
    std::chrono::steady_clock::time_point t0;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    uint64_t next_id = 1;
    std::unordered_map<uint64_t, std::unique_ptr<SJob>> jobs;
    std::deque<SJob*> incoming;

    // worker state
    std::deque<SJob*> pending;
    std::vector<SJob*> active_pt, active_bd, finishing;
    std::vector<uint32_t> free_slots;
    uint64_t film_in_use = 0;
    ar_server_stats stats{};
    // Order of the jobs past their equal share (PT ticks and BDPT batches):
    // size / (1 + waited / kAgingMs), smallest first, ties in arrival order.
    // Shortest job first while waits are short; a large job's key shrinks as
    // it waits, so smaller arrivals cannot hold it back indefinitely.  The PT
    // order is re-sent at every engine update and at most every kReorderMs.
    static constexpr double kAgingMs = 2000.0, kReorderMs = 50.0;
    double last_reorder_ms = 0;
    std::vector<uint32_t> pt_order_sent;
    double age_key(const SJob* j, uint64_t size, double now) const {
        return double(size) / (1.0 + std::max(0.0, now - j->t_admit) / kAgingMs);
    }
    std::vector<uint32_t> pt_order() {
        const double now = now_ms();
        std::vector<SJob*> v = active_pt;
        std::stable_sort(v.begin(), v.end(), [&](const SJob* a, const SJob* b) {
            return age_key(a, a->total_paths, now) < age_key(b, b->total_paths, now);
        });
        std::vector<uint32_t> slots;
        for (SJob* j : v) slots.push_back(j->slot);
        last_reorder_ms = now;
        pt_order_sent = slots;
        return slots;
    }
    // PT tick throttle and done snapshots
    static constexpr int kInflight = 4;
    cudaEvent_t tick_ev[kInflight] = {};
    uint64_t tick_count = 0;
    cudaEvent_t snap_ev = nullptr;
    bool snap_pending = false;
    uint64_t snap_issued = 0;   // id of the last snapshot issued (1-based)
    // BDPT batches in flight, one per lane
    struct BdLane {
        cudaEvent_t done = nullptr;
        bool busy = false;
        std::vector<SJob*> members;
    } bd_lane[kBdLanes];
    cudaEvent_t bd_admitted = nullptr;  // lane 0: the BDPT films cleared so far
    uint64_t bd_issued_batches = 0, bd_done_batches = 0;
    std::thread worker;

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }

    void fail(SJob* j, int code) {
        std::lock_guard<std::mutex> lk(mu);
        j->status = AR_JOB_FAILED;
        j->error = code;
        j->t_done = now_ms();
        stats.jobs_failed++;
        cv_done.notify_all();
    }

    size_t footprint(const SJob* j) const {
        const size_t px = size_t(j->w) * j->h * 3;
        const bool f64 = j->cfg.film_precision == AR_FILM_F64;
        const int nf = j->cfg.integrator == AR_INTEGRATOR_GDPT ? 3 : 1;
        return DevicePool::round(px * (f64 ? 8 : 4) * nf) + DevicePool::round(px * 4 * (nf == 3 ? 4 : 1));
    }

    void admit() {
        std::vector<std::pair<uint32_t, JobDev>> adds;
        while (!pending.empty()) {
            SJob* j = pending.front();
            {
                std::lock_guard<std::mutex> lk(mu);
                if (j->status != AR_JOB_PENDING) {  // cancelled while queued
                    pending.pop_front();
                    continue;
                }
            }
            const size_t fp = footprint(j);
            if (fp > opts.film_budget_bytes) {
                pending.pop_front();
                std::lock_guard<std::mutex> lk(mu);
                j->status = AR_JOB_REJECTED;
                j->t_done = now_ms();
                stats.jobs_rejected++;
                cv_done.notify_all();
                continue;
            }
            if (film_in_use + fp > opts.film_budget_bytes) break;
            if (j->kind == Kind::PathTraced && free_slots.empty()) break;
            if (j->kind == Kind::Bidirectional && active_bd.size() >= kMaxBdptJobs) break;
            pending.pop_front();
            const bool f64 = j->cfg.film_precision == AR_FILM_F64;
            const int nf = j->cfg.integrator == AR_INTEGRATOR_GDPT ? 3 : 1;
            const size_t px = size_t(j->w) * j->h * 3;
            j->films_bytes = px * (f64 ? 8 : 4) * nf;
            j->scratch_bytes = px * 4 * (nf == 3 ? 4 : 1);
            j->films = pool.get(j->films_bytes);
            j->scratch = pool.get(j->scratch_bytes);
            film_in_use += fp;
            stats.film_bytes_in_use = film_in_use;
            stats.film_bytes_peak = std::max(stats.film_bytes_peak, film_in_use);
            const CameraDev cam = make_camera(j->cam);
            if (j->kind == Kind::PathTraced) {
                AR_CUDA(cudaMemsetAsync(j->films, 0, j->films_bytes, ctx_pt->stream));
                j->min_snap = snap_issued + 1;  // an older snapshot predates this job's table entry
                j->slot = free_slots.back();
                free_slots.pop_back();
                JobDev J{};
                J.sc = j->scene->view;
                J.cam = cam;
                J.width = j->w;
                J.height = j->h;
                J.spp = j->cfg.spp;
                J.max_depth = j->cfg.max_depth;
                J.rr_depth = j->cfg.rr_depth;
                J.gdpt = nf == 3 ? 1u : 0u;
                J.film64 = f64 ? 1u : 0u;
                J.roles = uint32_t(nf);
                J.seed = j->cfg.seed;
                J.inv_spp = 1.0f / float(j->cfg.spp);
                for (int f = 0; f < nf; ++f) J.film[f] = static_cast<char*>(j->films) + f * (px * (f64 ? 8 : 4));
                J.total_samples = j->samples;
                J.total_paths = j->samples * uint64_t(nf);
                j->total_paths = J.total_paths;
                adds.push_back({j->slot, J});
                active_pt.push_back(j);
            } else {
                AR_CUDA(cudaMemsetAsync(j->films, 0, j->films_bytes, ctx_bd[0]->stream));
                AR_CUDA(cudaEventRecord(bd_admitted, ctx_bd[0]->stream));
                active_bd.push_back(j);
            }
            std::lock_guard<std::mutex> lk(mu);
            j->status = AR_JOB_RUNNING;
            j->t_admit = now_ms();
        }
        if (!adds.empty()) {
            const std::vector<uint32_t> order = pt_order();
            stats.h2d_bytes += engine_update(engine, adds, {}, &order);
        }
    }

    // Converts / reconstructs the film and copies it to the caller's buffer.
    void finish(SJob* j, ar_context* c) {
        const size_t count = size_t(j->w) * j->h * 3;
        const bool f64 = j->cfg.film_precision == AR_FILM_F64;
        float* outd = static_cast<float*>(j->scratch);
        if (j->cfg.integrator == AR_INTEGRATOR_GDPT) {
            float* f32 = outd + count;
            const size_t fb = count * (f64 ? 8 : 4);
            for (int f = 0; f < 3; ++f)
                film_to_f32(c, static_cast<char*>(j->films) + f * fb, f64, count, f32 + f * count);
            stats.kernel_launches +=
                3 + poisson_reconstruct(c, j->cfg, j->w, j->h, f32, f32 + count, f32 + 2 * count, outd, nullptr);
        } else {
            film_to_f32(c, j->films, f64, count, outd);
            stats.kernel_launches += 1;
        }
        AR_CUDA(cudaMemcpyAsync(j->out, outd, count * sizeof(float),
                                j->out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
        if (!j->out_on_device) stats.d2h_bytes += count * sizeof(float);
        AR_CUDA(cudaEventCreateWithFlags(&j->fin, cudaEventDisableTiming));
        AR_CUDA(cudaEventRecord(j->fin, c->stream));
        j->fin_stream = c->stream;
        finishing.push_back(j);
    }

    void step_pt() {
        if (active_pt.empty()) return;
        // at most kInflight ticks queued ahead of the GPU
        cudaEvent_t& ev = tick_ev[tick_count % kInflight];
        if (tick_count >= kInflight) AR_CUDA(cudaEventSynchronize(ev));
        engine_tick(engine);
        AR_CUDA(cudaEventRecord(ev, ctx_pt->stream));
        tick_count++;
        stats.pt_ticks++;
        stats.kernel_launches += kEngineTickKernels;
        if (snap_pending && cudaEventQuery(snap_ev) == cudaSuccess) {
            snap_pending = false;
            const unsigned long long* done = engine_snapshot_host(engine);
            std::vector<uint32_t> removes;
            std::vector<SJob*> still;
            for (SJob* j : active_pt) {
                j->last_done = done[j->slot];
                if (snap_issued >= j->min_snap && done[j->slot] >= j->total_paths) {
                    removes.push_back(j->slot);
                    finish(j, ctx_pt);
                } else {
                    still.push_back(j);
                }
            }
            active_pt.swap(still);
            if (!removes.empty()) {
                const std::vector<uint32_t> order = pt_order();
                stats.h2d_bytes += engine_update(engine, {}, removes, &order);
            }
        }
        if (active_pt.size() > 1 && now_ms() - last_reorder_ms >= kReorderMs) {
            const std::vector<uint32_t> before = pt_order_sent;
            const std::vector<uint32_t> order = pt_order();
            if (order != before) stats.h2d_bytes += engine_update(engine, {}, {}, &order);
        }
        if (!snap_pending) {
            engine_snapshot_done(engine);
            stats.d2h_bytes += kMaxActiveJobs * sizeof(unsigned long long);
            AR_CUDA(cudaEventRecord(snap_ev, ctx_pt->stream));
            snap_pending = true;
            snap_issued++;
        }
    }

    void step_bd() {
        // reap finished batches
        for (BdLane& L : bd_lane) {
            if (!L.busy || cudaEventQuery(L.done) != cudaSuccess) continue;
            for (SJob* j : L.members) j->bd_outstanding--;
            L.members.clear();
            L.busy = false;
            bd_done_batches++;
        }
        if (!active_bd.empty()) {
            std::vector<SJob*> still;
            for (SJob* j : active_bd) {
                if (j->bd_issued && j->bd_outstanding == 0) finish(j, ctx_bd[0]);
                else still.push_back(j);
            }
            active_bd.swap(still);
        }
        for (int lane = 0; lane < kBdLanes; ++lane) {
            BdLane& L = bd_lane[lane];
            if (L.busy) continue;
            std::vector<BdJob> jobs;
            std::vector<BdSegment> segs;
            // A waiting job whose remaining samples fit in an equal share of the
            // batch takes them all; the rest of the batch goes to the other jobs
            // in the aged shortest-first order (as the PT tick plan does), so one
            // job at a time fills the batch and it mostly traces one scene.
            const uint32_t cap = bdpt_batch_capacity(bdpt[lane]);
            std::vector<SJob*> order;
            for (SJob* j : active_bd)
                if (!j->bd_issued) order.push_back(j);
            const double now = now_ms();
            std::stable_sort(order.begin(), order.end(), [&](const SJob* a, const SJob* b) {
                return age_key(a, a->samples, now) < age_key(b, b->samples, now);
            });
            const uint64_t share = order.empty() ? 0 : cap / order.size();
            uint64_t left = cap;
            for (SJob* j : order)
                if (j->samples - j->bd_next <= share) left -= j->samples - j->bd_next;
            uint32_t used = 0;
            for (SJob* j : order) {
                const uint64_t rem = j->samples - j->bd_next;
                uint64_t take = rem;
                if (rem > share) {
                    take = std::min<uint64_t>(rem, left);
                    left -= take;
                }
                if (take == 0) continue;
                const CameraDev cam = make_camera(j->cam);
                segs.push_back(BdSegment{uint32_t(jobs.size()), used, uint32_t(take), 0, j->bd_next});
                jobs.push_back(make_bdpt_job(j->scene, cam, j->cfg, j->w, j->h, j->films));
                L.members.push_back(j);
                j->bd_next += take;
                used += uint32_t(take);
            }
            if (segs.empty()) return;
            ar_context* c = ctx_bd[lane];
            if (lane != 0) AR_CUDA(cudaStreamWaitEvent(c->stream, bd_admitted, 0));  // films cleared first
            stats.kernel_launches += bdpt_run_batch(bdpt[lane], jobs, segs);
            stats.h2d_bytes += jobs.size() * sizeof(BdJob) + segs.size() * sizeof(BdSegment);
            AR_CUDA(cudaEventRecord(L.done, c->stream));
            L.busy = true;
            bd_issued_batches++;
            stats.bdpt_batches++;
            for (SJob* j : L.members) {
                j->bd_outstanding++;
                if (j->bd_next >= j->samples) j->bd_issued = true;
            }
        }
    }

    void reap() {
        std::vector<SJob*> still;
        for (SJob* j : finishing) {
            if (cudaEventQuery(j->fin) != cudaSuccess) {
                still.push_back(j);
                continue;
            }
            cudaEventDestroy(j->fin);
            j->fin = nullptr;
            pool.put(j->films, j->films_bytes);
            pool.put(j->scratch, j->scratch_bytes);
            j->films = j->scratch = nullptr;
            film_in_use -= footprint(j);
            stats.film_bytes_in_use = film_in_use;
            if (j->slot != kInvalid) free_slots.push_back(j->slot);
            j->slot = kInvalid;
            std::lock_guard<std::mutex> lk(mu);
            j->status = AR_JOB_DONE;
            j->t_done = now_ms();
            stats.jobs_done++;
            stats.path_samples_done += j->samples;
            cv_done.notify_all();
        }
        finishing.swap(still);
    }

    bool busy() const { return !pending.empty() || !active_pt.empty() || !active_bd.empty() || !finishing.empty(); }

    // Diagnostics: the worker formats its state when asked (its queues are
    // not shared with API threads).
    bool debug_requested = false;
    std::string debug_text;
    void maybe_dump() {
        {
            std::lock_guard<std::mutex> lk(mu);
            if (!debug_requested) return;
        }
        std::string s = "ticks=" + std::to_string(tick_count) + " snap_issued=" + std::to_string(snap_issued) +
                        " snap_pending=" + std::to_string(snap_pending) + " bd_issued=" +
                        std::to_string(bd_issued_batches) + " bd_done=" + std::to_string(bd_done_batches) +
                        " film_in_use=" + std::to_string(film_in_use) + " pending=" + std::to_string(pending.size()) +
                        "\n";
        for (SJob* j : pending) s += "  pending job " + std::to_string(j->id) + "\n";
        for (SJob* j : active_pt)
            s += "  pt job " + std::to_string(j->id) + " slot=" + std::to_string(j->slot) + " done=" +
                 std::to_string(j->last_done) + "/" + std::to_string(j->total_paths) +
                 " min_snap=" + std::to_string(j->min_snap) + "\n";
        for (SJob* j : active_bd)
            s += "  bdpt job " + std::to_string(j->id) + " next=" + std::to_string(j->bd_next) + "/" +
                 std::to_string(j->samples) + " issued=" + std::to_string(j->bd_issued) +
                 " batches_in_flight=" + std::to_string(j->bd_outstanding) + "\n";
        for (SJob* j : finishing) s += "  finishing job " + std::to_string(j->id) + "\n";
        std::lock_guard<std::mutex> lk(mu);
        debug_text = s;
        debug_requested = false;
        cv_done.notify_all();
    }

    // Frees the device state (after the worker has stopped, or when creation
    // fails part way); safe on partly created state.
    void release() {
        cudaSetDevice(device);
        if (ctx_pt) cudaStreamSynchronize(ctx_pt->stream);
        for (ar_context* c : ctx_bd)
            if (c) cudaStreamSynchronize(c->stream);
        for (auto& e : tick_ev)
            if (e) cudaEventDestroy(e);
        for (auto& L : bd_lane)
            if (L.done) cudaEventDestroy(L.done);
        if (bd_admitted) cudaEventDestroy(bd_admitted);
        if (snap_ev) cudaEventDestroy(snap_ev);
        if (engine) engine_destroy(engine);
        for (BdptBatcher*& b : bdpt) {
            bdpt_destroy(b);
            b = nullptr;
        }
        if (ctx_pt) context_destroy_internal(ctx_pt);
        for (ar_context*& c : ctx_bd) {
            if (c) context_destroy_internal(c);
            c = nullptr;
        }
        engine = nullptr;
        ctx_pt = nullptr;
    }

    void run() {
        AR_CUDA(cudaSetDevice(device));
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                if (!busy() && incoming.empty()) {
                    if (stop) break;
                    cv_work.wait_for(lk, std::chrono::milliseconds(2));
                }
                while (!incoming.empty()) {
                    SJob* j = incoming.front();
                    incoming.pop_front();
                    if (j->status == AR_JOB_PENDING) pending.push_back(j);
                }
            }
            try {
                admit();
                step_pt();
                step_bd();
                reap();
                maybe_dump();
            } catch (const ArError& e) {
                set_error(e.msg);
                // Drop the failed PT jobs from the engine's active list too, so
                // that later admissions start from a list that matches
                // active_pt.  Their slots stay out of the free list: paths of a
                // failed job may still be in flight, keyed by its slot.
                std::vector<uint32_t> slots;
                for (SJob* j : active_pt)
                    if (j->slot != kInvalid) slots.push_back(j->slot);
                try {
                    if (!slots.empty()) engine_update(engine, {}, slots);
                } catch (const ArError&) {
                    // the engine could not be updated (a sticky CUDA error)
                }
                pt_order_sent.clear();
                for (SJob* j : active_pt) fail(j, e.code);
                for (SJob* j : active_bd) fail(j, e.code);
                for (SJob* j : finishing) fail(j, e.code);
                active_pt.clear();
                active_bd.clear();
                finishing.clear();
            }
            if (!busy()) {
                // idle: release throttle state so the next burst starts clean
                std::unique_lock<std::mutex> lk(mu);
                if (incoming.empty() && stop) break;
            }
        }
    }
};

}  // namespace ar

struct ar_server {
    std::unique_ptr<ar::ServerImpl> impl;
};

using namespace ar;

extern "C" {

int ar_server_create(ar_context* ctx, const ar_server_opts* o, ar_server** out) {
    return guarded([&] {
        AR_REQUIRE(ctx && out, AR_ERR_INVALID_ARGUMENT, "null argument");
        auto s = std::make_unique<ar_server>();
        s->impl = std::make_unique<ServerImpl>();
        ServerImpl& S = *s->impl;
        S.device = ctx->device;
        if (o) S.opts = *o;
        if (!S.opts.film_budget_bytes) S.opts.film_budget_bytes = 8ull << 30;
        if (!S.opts.path_capacity) S.opts.path_capacity = 1u << 22;
        if (!S.opts.bdpt_batch_samples) S.opts.bdpt_batch_samples = 1u << 20;
        if (!S.opts.bdpt_max_depth) S.opts.bdpt_max_depth = 10;
        if (!S.opts.max_active_jobs || S.opts.max_active_jobs > kMaxActiveJobs) S.opts.max_active_jobs = kMaxActiveJobs;
        S.t0 = std::chrono::steady_clock::now();
        try {
            S.ctx_pt = context_create_internal(ctx->device);
            {
                // PT ticks are short and latency-bound: their stream gets the
                // device's highest priority, so a tick's blocks go ahead of the
                // BDPT lanes' whenever SMs free up
                int least = 0, greatest = 0;
                AR_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
                cudaStream_t hp = nullptr;
                AR_CUDA(cudaStreamCreateWithPriority(&hp, cudaStreamNonBlocking, greatest));
                AR_CUDA(cudaStreamDestroy(S.ctx_pt->own_stream));
                S.ctx_pt->own_stream = S.ctx_pt->stream = hp;
            }
            for (auto& c : S.ctx_bd) c = context_create_internal(ctx->device);
            for (ar_context* c : {S.ctx_pt, S.ctx_bd[0], S.ctx_bd[1]}) {  // launch shapes follow the caller's context
                c->trav_blocks_per_sm = ctx->trav_blocks_per_sm;
                c->shade_block = ctx->shade_block;
            }
            S.engine = engine_create(S.ctx_pt, S.opts.path_capacity);
            for (int l = 0; l < ServerImpl::kBdLanes; ++l)
                S.bdpt[l] = bdpt_create(S.ctx_bd[l], S.opts.bdpt_max_depth, S.opts.bdpt_batch_samples);
            for (uint32_t i = S.opts.max_active_jobs; i-- > 0;) S.free_slots.push_back(i);
            for (auto& e : S.tick_ev) AR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            for (auto& L : S.bd_lane) AR_CUDA(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming));
            AR_CUDA(cudaEventCreateWithFlags(&S.bd_admitted, cudaEventDisableTiming));
            AR_CUDA(cudaEventCreateWithFlags(&S.snap_ev, cudaEventDisableTiming));
            AR_CUDA(cudaStreamSynchronize(S.ctx_pt->stream));
            for (ar_context* c : S.ctx_bd) AR_CUDA(cudaStreamSynchronize(c->stream));
        } catch (...) {
            S.release();
            throw;
        }
        S.worker = std::thread([&S] { S.run(); });
        *out = s.release();
    });
}

int ar_server_destroy(ar_server* s) {
    return guarded([&] {
        if (!s) return;
        ServerImpl& S = *s->impl;
        {
            std::lock_guard<std::mutex> lk(S.mu);
            S.stop = true;
        }
        S.cv_work.notify_all();
        if (S.worker.joinable()) S.worker.join();
        S.release();
        delete s;
    });
}

int ar_job_submit(ar_server* s, const ar_scene* scene, const ar_camera_desc* camera, const ar_integrator_cfg* cfg,
                  uint32_t width, uint32_t height, float* out_rgb, uint32_t out_on_device, uint64_t* job_id) {
    return guarded([&] {
        AR_REQUIRE(s && scene && camera && cfg && out_rgb && job_id, AR_ERR_INVALID_ARGUMENT, "null argument");
        AR_REQUIRE(width > 0 && height > 0 && cfg->spp > 0, AR_ERR_INVALID_ARGUMENT, "empty job");
        AR_REQUIRE(cfg->integrator <= AR_INTEGRATOR_GDPT, AR_ERR_INVALID_ARGUMENT, "unknown integrator");
        ServerImpl& S = *s->impl;
        AR_REQUIRE(scene->device == S.device, AR_ERR_INVALID_ARGUMENT, "scene lives on another device");
        if (cfg->integrator == AR_INTEGRATOR_BDPT)
            AR_REQUIRE(cfg->max_depth <= S.opts.bdpt_max_depth, AR_ERR_INVALID_ARGUMENT,
                       "BDPT max_depth above the server's bdpt_max_depth");
        else
            AR_REQUIRE(cfg->max_depth <= 255, AR_ERR_INVALID_ARGUMENT, "max_depth must be <= 255");
        auto j = std::make_unique<SJob>();
        j->scene = scene;
        j->cam = *camera;
        j->cfg = *cfg;
        j->w = width;
        j->h = height;
        j->out = out_rgb;
        j->out_on_device = out_on_device != 0;
        j->kind = cfg->integrator == AR_INTEGRATOR_BDPT ? Kind::Bidirectional : Kind::PathTraced;
        j->samples = uint64_t(width) * height * cfg->spp;
        {
            std::lock_guard<std::mutex> lk(S.mu);
            j->id = S.next_id++;
            j->t_submit = S.now_ms();
            *job_id = j->id;
            S.incoming.push_back(j.get());
            S.stats.jobs_submitted++;
            S.jobs[j->id] = std::move(j);
        }
        S.cv_work.notify_one();
    });
}

static void fill_info(const SJob& j, ar_job_info* info) {
    info->status = j.status;
    info->error = j.error;
    info->submit_ms = j.t_submit;
    info->admit_ms = j.t_admit;
    info->done_ms = j.t_done;
    info->path_samples = j.samples;
}

int ar_job_poll(ar_server* s, uint64_t id, ar_job_info* info) {
    return guarded([&] {
        AR_REQUIRE(s && info, AR_ERR_INVALID_ARGUMENT, "null argument");
        ServerImpl& S = *s->impl;
        std::lock_guard<std::mutex> lk(S.mu);
        auto it = S.jobs.find(id);
        AR_REQUIRE(it != S.jobs.end(), AR_ERR_NOT_FOUND, "unknown job id");
        fill_info(*it->second, info);
    });
}

int ar_job_wait(ar_server* s, uint64_t id, double timeout_ms, ar_job_info* info) {
    return guarded([&] {
        AR_REQUIRE(s, AR_ERR_INVALID_ARGUMENT, "null argument");
        ServerImpl& S = *s->impl;
        std::unique_lock<std::mutex> lk(S.mu);
        auto it = S.jobs.find(id);
        AR_REQUIRE(it != S.jobs.end(), AR_ERR_NOT_FOUND, "unknown job id");
        SJob* j = it->second.get();
        const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double, std::milli>(timeout_ms);
        while (j->status == AR_JOB_PENDING || j->status == AR_JOB_RUNNING) {
            if (S.cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
                (j->status == AR_JOB_PENDING || j->status == AR_JOB_RUNNING)) {
                if (info) fill_info(*j, info);
                throw ArError{AR_ERR_TIMEOUT, "job still running"};
            }
        }
        if (info) fill_info(*j, info);
    });
}

int ar_job_cancel(ar_server* s, uint64_t id) {
    return guarded([&] {
        AR_REQUIRE(s, AR_ERR_INVALID_ARGUMENT, "null argument");
        ServerImpl& S = *s->impl;
        std::lock_guard<std::mutex> lk(S.mu);
        auto it = S.jobs.find(id);
        AR_REQUIRE(it != S.jobs.end(), AR_ERR_NOT_FOUND, "unknown job id");
        SJob* j = it->second.get();
        // Only jobs not yet admitted can be withdrawn; the worker skips them.
        AR_REQUIRE(j->status == AR_JOB_PENDING, AR_ERR_NOT_FOUND, "job already admitted or finished");
        auto q = std::find(S.incoming.begin(), S.incoming.end(), j);
        if (q != S.incoming.end()) S.incoming.erase(q);
        j->status = AR_JOB_CANCELLED;
        j->t_done = S.now_ms();
        S.stats.jobs_cancelled++;
        S.cv_done.notify_all();
    });
}

int ar_server_get_stats(ar_server* s, ar_server_stats* out) {
    return guarded([&] {
        AR_REQUIRE(s && out, AR_ERR_INVALID_ARGUMENT, "null argument");
        std::lock_guard<std::mutex> lk(s->impl->mu);
        *out = s->impl->stats;
    });
}

double ar_server_now_ms(ar_server* s) { return s ? s->impl->now_ms() : 0.0; }

int ar_server_debug_dump(ar_server* s, char* buf, uint32_t capacity) {
    return guarded([&] {
        AR_REQUIRE(s && buf && capacity > 0, AR_ERR_INVALID_ARGUMENT, "null argument");
        ServerImpl& S = *s->impl;
        std::unique_lock<std::mutex> lk(S.mu);
        S.debug_requested = true;
        S.cv_work.notify_all();
        const auto deadline = std::chrono::steady_clock::now() + std::chrono::seconds(5);
        while (S.debug_requested)
            if (S.cv_done.wait_until(lk, deadline) == std::cv_status::timeout) break;
        std::string t = S.debug_requested ? std::string("worker did not answer within 5 s\n") : S.debug_text;
        S.debug_requested = false;
        const size_t n = std::min<size_t>(t.size(), capacity - 1);
        std::memcpy(buf, t.data(), n);
        buf[n] = 0;
    });
}

}  // extern "C"
