// Streaming wavefront path tracer: PathTracer::li / render
// (src/integrators/path_tracer.rs:59-190) and the base/offset paths of the
// gradient-domain tracer (trace_with_gradients, gradient_domain_pt.rs:266-342),
// restructured as the tick pipeline described in ar_engine.hpp.
//
// Path state is SoA and moves with the compacted queue (double buffered), so
// every stage reads contiguous 16-byte records; finished paths deposit L/spp
// into their job's film exactly once and bump the job's done counter.
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include <cooperative_groups.h>

#include "ar_engine.hpp"
#include "ar_shading.cuh"

namespace cg = cooperative_groups;

namespace ar {

namespace {

constexpr uint32_t kRoleBase = 0, kRoleRight = 1, kRoleDown = 2;
constexpr uint32_t kDead = 0x80000000u;  // meta flag: slot holds no live path

struct PathBuf {
    float4* ray_o;  // origin, tmin
    float4* ray_d;  // direction, tmax
    float4* thr;    // throughput, previous bsdf pdf
    float4* rad;    // radiance
    uint4* key;     // job, pixel, sample, meta (depth | dim << 8 | role << 24 | dead)
};

struct Segment {
    uint32_t job, path_offset, nsamples, roles;
    unsigned long long sample_begin;
};

struct EngineDev {
    JobDev* jobs;
    const uint32_t* active;
    const uint32_t* n_active;
    PathBuf buf[2];
    float4* hit;
    uint32_t* hit_inst;
    float4* sh_o;
    float4* sh_d;
    float4* sh_c;   // contribution rgb, flags (bit0: final)
    float4* sh_L;   // radiance before this bounce's NEE (final paths)
    uint4* sh_key;  // job, pixel, role, out index
    uint32_t* cnt;  // [0],[1]: queue length per buffer; [2]: shadow count; [3]: new paths; [4]: segments
    Segment* plan;
    uint32_t capacity;
    unsigned long long* stats;  // [0] paths generated, [1] closest-hit rays, [2] shadow rays
    int* err;
};

__device__ __forceinline__ void film_add(const JobDev& J, int which, uint32_t pix, f3 v) {
    if (J.film64) {
        double* f = static_cast<double*>(J.film[which]) + 3 * size_t(pix);
        atomicAdd(f, double(v.x));
        atomicAdd(f + 1, double(v.y));
        atomicAdd(f + 2, double(v.z));
    } else {
        float* f = static_cast<float*>(J.film[which]) + 3 * size_t(pix);
        atomicAdd(f, v.x);
        atomicAdd(f + 1, v.y);
        atomicAdd(f + 2, v.z);
    }
}

// Counts one finished path of `job`: lanes of the warp that finish paths of the
// same job share one atomic.
__device__ __forceinline__ void count_done(const EngineDev& E, uint32_t job) {
    cg::coalesced_group g = cg::coalesced_threads();
    cg::coalesced_group same = cg::labeled_partition(g, job);
    if (same.thread_rank() == 0) atomicAdd(&E.jobs[job].done_paths, (unsigned long long)same.size());
}

// A finished path adds L/spp to its job's film(s) and counts as done.
__device__ __forceinline__ void deposit(const EngineDev& E, uint32_t job, uint32_t pixel, uint32_t role, f3 L) {
    JobDev& J = E.jobs[job];
    const f3 v = L * J.inv_spp;
    if (!J.gdpt) {
        film_add(J, 0, pixel, v);
    } else {
        const uint32_t px = pixel % J.width, py = pixel / J.width;
        if (role == kRoleBase) {
            film_add(J, 0, pixel, v);
            if (px + 1 < J.width) film_add(J, 1, pixel, -v);
            if (py + 1 < J.height) film_add(J, 2, pixel, -v);
        } else {
            film_add(J, role == kRoleRight ? 1 : 2, pixel, v);
        }
    }
    count_done(E, job);
}

// Free slots -> samples of the active jobs.  A job whose remaining paths fit
// in an equal share of the free slots takes them all (so a small job finishes
// in the tick it arrives instead of waiting behind a large one); what those
// leave goes to the other jobs in the order of the active list, which the host
// sets (by default fewest total paths first, ties in arrival order; the
// server ages that order by waiting time): capacity goes to one job at a time,
// so a tick's paths mostly trace one scene, as one job alone would, and a
// medium job does not wait behind a huge one.  Every
// free slot is used as before, only the split changes.  Images do not depend
// on the split: every sample is keyed by (job seed, pixel, sample).
__global__ void k_plan(EngineDev E, int q) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t n_cont = E.cnt[q];
    uint32_t used = 0, nseg = 0;
    const uint32_t na = *E.n_active;
    const uint32_t free_paths = E.capacity - n_cont;
    uint32_t waiting = 0;
    for (uint32_t a = 0; a < na; ++a) {
        const JobDev& J = E.jobs[E.active[a]];
        if (J.total_samples > J.next_sample) waiting++;
    }
    const unsigned long long share = waiting ? free_paths / waiting : 0;
    uint32_t left = free_paths;
    for (uint32_t a = 0; a < na; ++a) {  // jobs that fit in their share
        const JobDev& J = E.jobs[E.active[a]];
        const unsigned long long rem = J.total_samples - J.next_sample;
        if (rem * J.roles <= share) left -= uint32_t(rem) * J.roles;
    }
    for (uint32_t a = 0; a < na; ++a) {  // those, and the rest in list order
        const uint32_t j = E.active[a];
        JobDev& J = E.jobs[j];
        const unsigned long long rem = J.total_samples - J.next_sample;
        if (rem == 0) continue;
        unsigned long long take = rem;
        if (rem * J.roles > share) {
            take = min(rem, (unsigned long long)(left / J.roles));
            left -= uint32_t(take) * J.roles;
        }
        if (take == 0) continue;
        E.plan[nseg] = Segment{j, n_cont + used, uint32_t(take), J.roles, J.next_sample};
        J.next_sample += take;
        used += uint32_t(take) * J.roles;
        nseg++;
    }
    E.cnt[3] = used;
    E.cnt[4] = nseg;
    E.cnt[q] = n_cont + used;
    E.cnt[q ^ 1] = 0;
    E.cnt[2] = 0;
    E.cnt[8] = 0;  // ray-fetch cursors of the extend and shadow stages
    E.cnt[9] = 0;
    E.stats[0] += used;
}

__global__ void __launch_bounds__(256) k_generate(EngineDev E, int q) {
    const uint32_t n_new = E.cnt[3], nseg = E.cnt[4];
    const uint32_t base_off = E.cnt[q] - n_new;
    const PathBuf B = E.buf[q];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += gridDim.x * blockDim.x) {
        const uint32_t k = base_off + i;
        uint32_t lo = 0, hi = nseg;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (E.plan[mid].path_offset <= k) lo = mid; else hi = mid;
        }
        const Segment sg = E.plan[lo];
        const JobDev& J = E.jobs[sg.job];
        const uint32_t rel = k - sg.path_offset;
        const uint32_t si = rel / sg.roles, role = rel - si * sg.roles;
        const unsigned long long g = sg.sample_begin + si;
        const uint32_t npix = J.width * J.height;
        const uint32_t pixel = uint32_t(g % npix), sample = uint32_t(g / npix);
        const uint32_t px = pixel % J.width, py = pixel / J.width;
        const bool skip = (role == kRoleRight && px + 1 >= J.width) || (role == kRoleDown && py + 1 >= J.height);
        if (skip) {
            // Offset path outside the image: zero gradient, no trace (gdpt.rs:298-327).
            B.key[k] = make_uint4(sg.job, pixel, sample, kDead | (role << 24));
            count_done(E, sg.job);
            continue;
        }
        const uint64_t key = counter_key(J.seed, pixel, sample);
        const float jx = counter_u01(key, 0), jy = counter_u01(key, 1);
        const uint32_t ox = px + (role == kRoleRight ? 1u : 0u), oy = py + (role == kRoleDown ? 1u : 0u);
        const Ray r = camera_ray(J.cam, (float(ox) + jx) / float(J.width), 1.0f - (float(oy) + jy) / float(J.height));
        B.ray_o[k] = make_float4(r.o.x, r.o.y, r.o.z, r.tmin);
        B.ray_d[k] = make_float4(r.d.x, r.d.y, r.d.z, r.tmax);
        B.thr[k] = make_float4(1.f, 1.f, 1.f, 0.f);
        B.rad[k] = make_float4(0.f, 0.f, 0.f, 0.f);
        B.key[k] = make_uint4(sg.job, pixel, sample, (2u << 8) | (role << 24));
    }
}

__global__ void AR_TRAVERSAL_BOUNDS k_extend(const __grid_constant__ EngineDev E, int q) {
    const uint32_t n = E.cnt[q];
    const PathBuf B = E.buf[q];
    if (blockIdx.x == 0 && threadIdx.x == 0) E.stats[1] += n;
    run_traversal<false>(
        &E.cnt[8], n, E.err,
        [&](uint32_t j, const DevScene*& s, Ray& r) {
            const uint4 kk = B.key[j];
            s = &E.jobs[kk.x].sc;
            if (kk.w & kDead) {
                r = Ray{mk(0.f, 0.f, 0.f), mk(0.f, 0.f, 1.f), 1.f, 0.f};  // empty t-range: a miss
            } else {
                const float4 a = B.ray_o[j], b = B.ray_d[j];
                r = Ray{mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w};
            }
        },
        [&](uint32_t j, const HitRec& h) {
            E.hit[j] = make_float4(h.t, h.u, h.v, __uint_as_float(h.slot));
            E.hit_inst[j] = h.inst;
        });
}

// At least 4 blocks of 256 per SM (<= 64 registers): shading is bound by the
// latency of its scattered scene loads, and the doubled occupancy outweighs the
// spills (stage time -19% on a 139k-triangle scene at 512x512x16).
__global__ void __launch_bounds__(256, 4) k_shade(EngineDev E, int q) {
    const uint32_t n = E.cnt[q];
    const PathBuf B = E.buf[q], O = E.buf[q ^ 1];
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t j = base + threadIdx.x;
        bool cont = false, shadow = false, live = false;
        uint4 kk = make_uint4(0, 0, 0, 0);
        f3 new_o, new_d, sh_o, sh_d, sh_c, L, thr;
        float sh_tmax = 0.f, prev_pdf = 0.f;
        if (j < n) {
            kk = ld_once(B.key + j);  // the path's records are read once per tick: evict-first
            live = !(kk.w & kDead);
        }
        if (live) {
            const JobDev& J = E.jobs[kk.x];
            const float4 h = ld_once(E.hit + j);
            const float4 t4 = ld_once(B.thr + j), r4 = ld_once(B.rad + j);
            thr = mk(t4.x, t4.y, t4.z);
            prev_pdf = t4.w;
            L = mk(r4.x, r4.y, r4.z);
            const uint32_t depth = kk.w & 0xffu;
            uint32_t dim = (kk.w >> 8) & 0xffffu;
            const uint32_t slot = __float_as_uint(h.w);
            if (slot != kInvalid) {
                const DevScene& sc = J.sc;
                const uint64_t key = counter_key(J.seed, kk.y, kk.z);
                const float4 ro4 = ld_once(B.ray_o + j), rd4 = ld_once(B.ray_d + j);
                const f3 ro = mk(ro4.x, ro4.y, ro4.z), rd = mk(rd4.x, rd4.y, rd4.z);
                const Shade s = make_shade(sc, ro, rd, h.x, h.y, h.z, slot, ld_once(E.hit_inst + j));
                const MatView m = load_mat_at(sc, s.mat, s.tu, s.tv);
                const f3 wo = -rd;
                const f3 wo_l = to_local(s.onb, wo);
                const bool lights_on = light_enabled(sc);
                // Emission on hit (area-light extension).
                if (m.emitter >= 0) {
                    const LightView lt = load_light(sc, uint32_t(m.emitter));
                    const float cos_l = dot(lt.n, wo);
                    if (cos_l > 0.f) {
                        if (depth == 0 || !lights_on) {
                            L = L + thr * lt.inten;
                        } else {
                            const float pdf_light =
                                light_pmf_of(sc, uint32_t(m.emitter)) * (h.x * h.x) / (cos_l * lt.area);
                            L = L + (thr * lt.inten) * power_heuristic(prev_pdf, pdf_light);
                        }
                    }
                }
                // Next-event estimation (path_tracer.rs:79-117).
                if (lights_on) {
                    const float u_sel = counter_u01(key, dim++);
                    const float ulx = counter_u01(key, dim++);
                    const float uly = counter_u01(key, dim++);
                    uint32_t li;
                    float sel;
                    light_select(sc, u_sel, li, sel);
                    const LightView light = load_light(sc, li);
                    f3 wi, lrad;
                    float dist, lpdf;
                    if (light_sample(light, s.p, ulx, uly, wi, dist, lrad, lpdf)) {
                        const f3 wi_l = to_local(s.onb, wi);
                        const float cos_wi = fabsf(wi_l.z);
                        if (cos_wi > 0.f) {
                            const f3 f = bsdf_eval(m, wi_l, wo_l);
                            f3 c;
                            if (light.kind == AR_LIGHT_POINT) {
                                c = ((thr * f) * cos_wi) * lrad / sel;
                            } else {
                                const float pdf_light = lpdf * sel;
                                const float w = power_heuristic(pdf_light, bsdf_pdf(m, wi_l, wo_l));
                                c = ((((thr * f) * cos_wi) * lrad) * w) / pdf_light;
                            }
                            if (!is_zero(c)) {
                                sh_o = s.p + (s.n * 1e-4f) * signum(dot(wi, s.n));
                                sh_d = normalize(wi);
                                sh_tmax = dist * (1.0f - 1e-4f);
                                sh_c = c;
                                shadow = true;
                            }
                        }
                    }
                }
                // BSDF sampling, Russian roulette, spawn (:119-153).
                const float usel = counter_u01(key, dim++);
                const float udx = counter_u01(key, dim++);
                const float udy = counter_u01(key, dim++);
                f3 wi, f;
                float pdf;
                if (bsdf_sample(m, wo_l, usel, udx, udy, wi, pdf, f) && pdf != 0.f && !is_zero(f)) {
                    thr = thr * ((f * fabsf(wi.z)) / pdf);
                    prev_pdf = pdf;
                    bool alive = true;
                    if (depth + 1 >= J.rr_depth) {
                        const float survival = fminf(max3(thr), 0.95f);
                        if (counter_u01(key, dim++) > survival) alive = false;
                        else thr = thr / survival;
                    }
                    if (alive && depth + 1 < J.max_depth) {
                        const f3 wi_w = to_world(s.onb, wi);
                        new_o = s.p + (s.n * 1e-4f) * signum(dot(wi_w, s.n));
                        new_d = normalize(wi_w);
                        cont = true;
                    }
                }
                kk.w = (kk.w & 0xff000000u) | (dim << 8) | (depth + 1);
            }
        }
        const uint32_t rs = warp_alloc(&E.cnt[q ^ 1], cont);
        const uint32_t ss = warp_alloc(&E.cnt[2], shadow);
        if (!live) continue;
        if (cont) {
            O.ray_o[rs] = make_float4(new_o.x, new_o.y, new_o.z, 1e-4f);
            O.ray_d[rs] = make_float4(new_d.x, new_d.y, new_d.z, FLT_MAX);
            O.thr[rs] = make_float4(thr.x, thr.y, thr.z, prev_pdf);
            O.rad[rs] = make_float4(L.x, L.y, L.z, 0.f);
            O.key[rs] = kk;
        }
        const uint32_t role = (kk.w >> 24) & 3u;
        if (shadow) {
            st_once(E.sh_o + ss, make_float4(sh_o.x, sh_o.y, sh_o.z, 0.f));
            st_once(E.sh_d + ss, make_float4(sh_d.x, sh_d.y, sh_d.z, sh_tmax));
            st_once(E.sh_c + ss, make_float4(sh_c.x, sh_c.y, sh_c.z, __uint_as_float(cont ? 0u : 1u)));
            st_once(E.sh_L + ss, make_float4(L.x, L.y, L.z, 0.f));
            st_once(E.sh_key + ss, make_uint4(kk.x, kk.y, role, rs));
        } else if (!cont) {
            deposit(E, kk.x, kk.y, role, L);
        }
    }
}

__global__ void AR_TRAVERSAL_BOUNDS k_shadow(const __grid_constant__ EngineDev E, int q) {
    const uint32_t n = E.cnt[2];
    const PathBuf O = E.buf[q ^ 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) E.stats[2] += n;
    run_traversal<true>(
        &E.cnt[9], n, E.err,
        [&](uint32_t m, const DevScene*& s, Ray& r) {
            const float4 a = ld_once(E.sh_o + m), b = ld_once(E.sh_d + m);
            s = &E.jobs[E.sh_key[m].x].sc;
            r = Ray{mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w};
        },
        [&](uint32_t m, const HitRec& h) {
            const uint4 sk = ld_once(E.sh_key + m);
            const float4 c = ld_once(E.sh_c + m);
            const bool visible = h.slot == kInvalid;
            if (__float_as_uint(c.w) & 1u) {
                const float4 l = ld_once(E.sh_L + m);
                f3 L = mk(l.x, l.y, l.z);
                if (visible) L = L + mk(c.x, c.y, c.z);
                deposit(E, sk.x, sk.y, sk.z, L);
            } else if (visible) {
                float4 r = O.rad[sk.w];
                r.x += c.x;
                r.y += c.y;
                r.z += c.z;
                O.rad[sk.w] = r;
            }
        });
}

template <class T>
T* carve(char*& cur, size_t n) {
    cur = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(cur) + 255) & ~uintptr_t(255));
    T* p = reinterpret_cast<T*>(cur);
    cur += n * sizeof(T);
    return p;
}

}  // namespace

struct PathEngine {
    ar_context* ctx = nullptr;
    uint32_t cap = 0;
    DevBuf mem, jobs_d, active_d;
    EngineDev E{};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaStream_t captured_stream = nullptr;
    int parity = 0;
    uint64_t ticks = 0;
    std::vector<uint32_t> active;   // job slots in the order the tick plan serves them past their share
    std::vector<unsigned long long> total_paths = std::vector<unsigned long long>(kMaxActiveJobs, 0);
    unsigned long long* done_h = nullptr;
    // plain renders: completion events of the two ticks in flight, and the
    // engine's counters (paths, extend rays, shadow rays) as pinned copies,
    // read after the render's final synchronisation
    cudaEvent_t tick_ev[2] = {nullptr, nullptr};
    unsigned long long* stats_pin = nullptr;
    unsigned long long stats_seen[3] = {0, 0, 0};
    // Pinned staging for job-table updates, two halves used alternately; each
    // half is reused only after the event of its last copy has completed.
    struct Staging {
        JobDev* jobs = nullptr;
        uint32_t* active = nullptr;
        cudaEvent_t ev = nullptr;
    } stage[2];
    int stage_next = 0;

    // The five stages of one tick, with the context's launch shapes (each
    // stage bracketed by a profiler scope when profiling is on).
    void launch_tick(int q, cudaStream_t s) {
        const int wide = ctx->num_sms * 8;
        const int tgrid = ctx->num_sms * int(ctx->trav_blocks_per_sm);
        const int sb = int(ctx->shade_block);
        { KernelScope k(ctx->prof, s, "pt_plan"); k_plan<<<1, 32, 0, s>>>(E, q); }
        { KernelScope k(ctx->prof, s, "pt_generate"); k_generate<<<wide, 256, 0, s>>>(E, q); }
        { KernelScope k(ctx->prof, s, "pt_extend"); k_extend<<<tgrid, 128, 0, s>>>(E, q); }
        { KernelScope k(ctx->prof, s, "pt_shade"); k_shade<<<wide * (256 / sb), sb, 0, s>>>(E, q); }
        { KernelScope k(ctx->prof, s, "pt_shadow"); k_shadow<<<tgrid, 128, 0, s>>>(E, q); }
    }

    void build_graphs() {
        for (int q = 0; q < 2; ++q) {
            if (graph[q]) cudaGraphExecDestroy(graph[q]);
            graph[q] = nullptr;
        }
        cudaStream_t s = ctx->stream;
        for (int q = 0; q < 2; ++q) {
            cudaGraph_t g;
            AR_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            launch_tick(q, s);
            AR_CUDA(cudaStreamEndCapture(s, &g));
            AR_CUDA(cudaGraphInstantiate(&graph[q], g, 0));
            cudaGraphDestroy(g);
        }
        captured_stream = s;
    }

    ~PathEngine() {
        for (int q = 0; q < 2; ++q)
            if (graph[q]) cudaGraphExecDestroy(graph[q]);
        if (done_h) cudaFreeHost(done_h);
        if (stats_pin) cudaFreeHost(stats_pin);
        for (cudaEvent_t ev : tick_ev)
            if (ev) cudaEventDestroy(ev);
        for (auto& s : stage) {
            if (s.jobs) cudaFreeHost(s.jobs);
            if (s.active) cudaFreeHost(s.active);
            if (s.ev) cudaEventDestroy(s.ev);
        }
    }
};

PathEngine* engine_create(ar_context* ctx, uint32_t capacity) {
    auto e = std::make_unique<PathEngine>();
    e->ctx = ctx;
    e->cap = capacity;
    const size_t c = capacity;
    size_t bytes = 2 * c * (4 * sizeof(float4) + sizeof(uint4)) + c * (sizeof(float4) + sizeof(uint32_t)) +
                   c * (4 * sizeof(float4) + sizeof(uint4)) + 64 * sizeof(uint32_t) +
                   kMaxActiveJobs * sizeof(Segment) + 8 * sizeof(unsigned long long) + 32 * 256;
    e->mem.alloc(bytes);
    char* cur = e->mem.as<char>();
    for (int b = 0; b < 2; ++b) {
        e->E.buf[b].ray_o = carve<float4>(cur, c);
        e->E.buf[b].ray_d = carve<float4>(cur, c);
        e->E.buf[b].thr = carve<float4>(cur, c);
        e->E.buf[b].rad = carve<float4>(cur, c);
        e->E.buf[b].key = carve<uint4>(cur, c);
    }
    e->E.hit = carve<float4>(cur, c);
    e->E.hit_inst = carve<uint32_t>(cur, c);
    e->E.sh_o = carve<float4>(cur, c);
    e->E.sh_d = carve<float4>(cur, c);
    e->E.sh_c = carve<float4>(cur, c);
    e->E.sh_L = carve<float4>(cur, c);
    e->E.sh_key = carve<uint4>(cur, c);
    e->E.cnt = carve<uint32_t>(cur, 64);
    e->E.plan = carve<Segment>(cur, kMaxActiveJobs);
    e->E.stats = carve<unsigned long long>(cur, 8);
    e->E.capacity = capacity;
    e->E.err = ctx->err_flag.as<int>();
    e->jobs_d.alloc(kMaxActiveJobs * sizeof(JobDev));
    e->active_d.alloc((kMaxActiveJobs + 1) * sizeof(uint32_t));
    e->E.jobs = e->jobs_d.as<JobDev>();
    e->E.active = e->active_d.as<uint32_t>();
    e->E.n_active = e->active_d.as<uint32_t>() + kMaxActiveJobs;
    AR_CUDA(cudaMemsetAsync(e->E.cnt, 0, 64 * sizeof(uint32_t), ctx->stream));
    AR_CUDA(cudaMemsetAsync(e->E.stats, 0, 8 * sizeof(unsigned long long), ctx->stream));
    AR_CUDA(cudaMemsetAsync(e->active_d.ptr, 0, (kMaxActiveJobs + 1) * sizeof(uint32_t), ctx->stream));
    AR_CUDA(cudaMallocHost(&e->done_h, kMaxActiveJobs * sizeof(unsigned long long)));
    AR_CUDA(cudaMallocHost(&e->stats_pin, 3 * sizeof(unsigned long long)));
    for (cudaEvent_t& ev : e->tick_ev) AR_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    for (auto& s : e->stage) {
        AR_CUDA(cudaMallocHost(&s.jobs, kMaxActiveJobs * sizeof(JobDev)));
        AR_CUDA(cudaMallocHost(&s.active, (kMaxActiveJobs + 1) * sizeof(uint32_t)));
        AR_CUDA(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
        AR_CUDA(cudaEventRecord(s.ev, ctx->stream));
    }
    e->build_graphs();
    return e.release();
}

void engine_destroy(PathEngine* e) { delete e; }

size_t engine_update(PathEngine* e, const std::vector<std::pair<uint32_t, JobDev>>& adds,
                     const std::vector<uint32_t>& removes, const std::vector<uint32_t>* order) {
    if (adds.empty() && removes.empty() && !order) return 0;
    // the active list after the changes, checked before anything is copied
    std::vector<uint32_t> next = e->active;
    for (uint32_t slot : removes) {
        auto it = std::find(next.begin(), next.end(), slot);
        if (it != next.end()) next.erase(it);
    }
    AR_REQUIRE(next.size() + adds.size() <= kMaxActiveJobs, AR_ERR_REJECTED, "too many active jobs");
    for (const auto& a : adds) {
        AR_REQUIRE(a.first < kMaxActiveJobs, AR_ERR_INVALID_ARGUMENT, "job slot out of range");
        next.push_back(a.first);
    }
    if (order) {
        std::vector<uint32_t> x = next, y = *order;
        std::sort(x.begin(), x.end());
        std::sort(y.begin(), y.end());
        AR_REQUIRE(x == y, AR_ERR_INTERNAL, "engine order is not a permutation of the active jobs");
    }
    auto& st = e->stage[e->stage_next];
    e->stage_next ^= 1;
    AR_CUDA(cudaEventSynchronize(st.ev));  // its previous copies have been consumed
    for (size_t i = 0; i < adds.size(); ++i) {
        const uint32_t slot = adds[i].first;
        st.jobs[i] = adds[i].second;
        AR_CUDA(cudaMemcpyAsync(e->E.jobs + slot, &st.jobs[i], sizeof(JobDev), cudaMemcpyHostToDevice,
                                e->ctx->stream));
        e->total_paths[slot] = adds[i].second.total_paths;
    }
    // the tick plan serves jobs past their equal share in this order
    if (order) {
        next = *order;
    } else {
        std::stable_sort(next.begin(), next.end(),
                         [&](uint32_t x, uint32_t y) { return e->total_paths[x] < e->total_paths[y]; });
    }
    e->active.swap(next);
    for (size_t i = 0; i < e->active.size(); ++i) st.active[i] = e->active[i];
    st.active[kMaxActiveJobs] = uint32_t(e->active.size());
    if (!e->active.empty())
        AR_CUDA(cudaMemcpyAsync(e->active_d.ptr, st.active, e->active.size() * sizeof(uint32_t),
                                cudaMemcpyHostToDevice, e->ctx->stream));
    AR_CUDA(cudaMemcpyAsync(e->active_d.as<uint32_t>() + kMaxActiveJobs, st.active + kMaxActiveJobs,
                            sizeof(uint32_t), cudaMemcpyHostToDevice, e->ctx->stream));
    AR_CUDA(cudaEventRecord(st.ev, e->ctx->stream));
    return adds.size() * sizeof(JobDev) + (e->active.size() + 1) * sizeof(uint32_t);
}

void engine_add_job(PathEngine* e, uint32_t slot, const JobDev& job) { engine_update(e, {{slot, job}}, {}); }

void engine_remove_job(PathEngine* e, uint32_t slot) { engine_update(e, {}, {slot}); }

void engine_tick(PathEngine* e) {
    ar_context* ctx = e->ctx;
    const int q = e->parity;
    if (ctx->prof.on) {
        // Profiling: launch the stages individually, each bracketed by events.
        e->launch_tick(q, ctx->stream);
        AR_CUDA(cudaGetLastError());
    } else {
        if (e->captured_stream != ctx->stream) e->build_graphs();
        AR_CUDA(cudaGraphLaunch(e->graph[q], ctx->stream));
    }
    e->parity ^= 1;
    e->ticks++;
}

const unsigned long long* engine_snapshot_done(PathEngine* e) {
    // done_paths lives at a fixed offset inside each JobDev: gather with one
    // strided 2D copy.
    const size_t off = offsetof(JobDev, done_paths);
    AR_CUDA(cudaMemcpy2DAsync(e->done_h, sizeof(unsigned long long), reinterpret_cast<char*>(e->E.jobs) + off,
                              sizeof(JobDev), sizeof(unsigned long long), kMaxActiveJobs, cudaMemcpyDeviceToHost,
                              e->ctx->stream));
    return e->done_h;
}

const unsigned long long* engine_snapshot_host(const PathEngine* e) { return e->done_h; }

uint64_t engine_ticks(const PathEngine* e) { return e->ticks; }
uint32_t engine_capacity(const PathEngine* e) { return e->cap; }
bool engine_has_active(const PathEngine* e) { return !e->active.empty(); }

void engine_stats(PathEngine* e, unsigned long long* out3_pinned) {
    AR_CUDA(cudaMemcpyAsync(out3_pinned, e->E.stats, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            e->ctx->stream));
}

// Single-job render through the engine (Integrator::render for PT / GDPT
// paths): the "plain" one-job-at-a-time path.
void render_pt_films(ar_context* ctx, const ar_scene* sc, const CameraDev& cam, const ar_integrator_cfg& cfg,
                     uint32_t w, uint32_t h, bool gdpt, void* films) {
    AR_REQUIRE(cfg.max_depth <= 255, AR_ERR_INVALID_ARGUMENT, "max_depth must be <= 255");
    if (!ctx->engine) ctx->engine = engine_create(ctx, ctx->engine_capacity);
    PathEngine* e = ctx->engine;
    const uint32_t roles = gdpt ? 3u : 1u;
    const bool f64 = cfg.film_precision == AR_FILM_F64;
    const size_t film_bytes = size_t(w) * h * 3 * (f64 ? sizeof(double) : sizeof(float));
    AR_CUDA(cudaMemsetAsync(films, 0, film_bytes * roles, ctx->stream));
    JobDev J{};
    J.sc = sc->view;
    J.cam = cam;
    J.width = w;
    J.height = h;
    J.spp = cfg.spp;
    J.max_depth = cfg.max_depth;
    J.rr_depth = cfg.rr_depth;
    J.gdpt = gdpt ? 1u : 0u;
    J.film64 = f64 ? 1u : 0u;
    J.roles = roles;
    J.seed = cfg.seed;
    J.inv_spp = 1.0f / float(cfg.spp);
    for (uint32_t f = 0; f < roles; ++f) J.film[f] = static_cast<char*>(films) + f * film_bytes;
    const uint64_t npix = uint64_t(w) * h;
    const uint32_t s0 = ctx->range_end ? ctx->range_begin : 0u, s1 = ctx->range_end ? ctx->range_end : cfg.spp;
    J.total_samples = npix * s1;  // sample g of the job is pixel g % npix, sample g / npix
    J.total_paths = npix * (s1 - s0) * roles;
    J.next_sample = npix * s0;
    J.done_paths = 0;
    const uint32_t slot = 0;
    engine_add_job(e, slot, J);
    // Tick until every path has deposited; completion is checked one tick behind
    // so the GPU always has the next tick queued.
    cudaEvent_t* ev = e->tick_ev;
    unsigned long long* done_pinned = e->done_h;  // two entries, one per in-flight tick
    uint64_t issued = 0;
    const uint64_t tick_cap = 1ull << 26;
    bool done = false;
    while (!done) {
        engine_tick(e);
        const int cur = int(issued & 1);
        AR_CUDA(cudaMemcpyAsync(done_pinned + cur, &e->E.jobs[slot].done_paths, sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, ctx->stream));
        AR_CUDA(cudaEventRecord(ev[cur], ctx->stream));
        issued++;
        if (issued >= 2) {
            const int prev = int((issued - 2) & 1);  // the tick before the one just queued
            AR_CUDA(cudaEventSynchronize(ev[prev]));
            if (done_pinned[prev] >= J.total_paths) done = true;
        }
        AR_REQUIRE(issued < tick_cap, AR_ERR_TIMEOUT, "render did not converge");
    }
    AR_CUDA(cudaMemcpyAsync(e->stats_pin, e->E.stats, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            ctx->stream));
    AR_CUDA(cudaStreamSynchronize(ctx->stream));
    engine_remove_job(e, slot);
    // the counters are cumulative over the engine's life; only this path ticks it
    const unsigned long long* after = e->stats_pin;
    ctx->last_stats.path_samples = npix * (s1 - s0);
    ctx->last_stats.paths = after[0] - e->stats_seen[0];
    ctx->last_stats.extend_rays = after[1] - e->stats_seen[1];
    ctx->last_stats.shadow_rays = after[2] - e->stats_seen[2];
    for (int k = 0; k < 3; ++k) e->stats_seen[k] = after[k];
    ctx->last_stats.extend_launches = issued;
    ctx->last_stats.shadow_launches = issued;
    ctx->stats_pending = false;
}

}  // namespace ar
