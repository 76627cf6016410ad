// Wavefront path tracer: PathTracer::li / render (src/integrators/path_tracer.rs:59-190)
// and the base/offset paths of the gradient-domain tracer (trace_with_gradients,
// src/integrators/gradient_domain_pt.rs:266-342), restructured into stages:
//
//   generate -> [ extend (closest hit) -> shade (emission, NEE, BSDF sample,
//                 Russian roulette, compaction) -> shadow (any hit) ] x max_depth
//
// Paths live in SoA slots; the ray and hit queues are compacted with warp
// ballots so every stage reads contiguous 16-byte records.  Each path deposits
// its radiance into the film exactly once, when it terminates.
#include <algorithm>
#include <cmath>

#include "ar_shading.cuh"

namespace ar {

namespace {

constexpr uint32_t kRoleBase = 0, kRoleRight = 1, kRoleDown = 2;

struct PtState {
    // path slots
    uint2* key;       // pixel, sample
    float4* thr;      // throughput rgb, previous bsdf pdf
    float4* rad;      // radiance rgb
    uint32_t* meta;   // depth | dim << 8 | role << 24
    // ray queues (double buffered) and hits
    float4* ray_o[2];
    float4* ray_d[2];
    uint32_t* qpath[2];
    float4* hit;
    uint32_t* hit_inst;
    // shadow queue
    float4* sh_o;
    float4* sh_d;
    float4* sh_c;
    uint32_t* sh_path;  // path | kFinal
    uint32_t* counts;   // [0..max_depth]: rays entering bounce d; [64 + d]: shadow rays of bounce d
};
constexpr uint32_t kFinal = 0x80000000u;

struct PtParams {
    DevScene sc;
    CameraDev cam;
    PtState st;
    uint32_t width, height, spp, max_depth, rr_depth;
    uint32_t gdpt, film64;
    uint64_t seed;
    uint64_t sample_begin;  // first (sample-major) path sample of this chunk
    uint32_t chunk_samples;
    float inv_spp;
    void* film[3];  // PT: film[0]; GDPT: primal, dx, dy
};

__device__ __forceinline__ void film_add(const PtParams& P, int which, uint32_t pix, f3 v) {
    if (P.film64) {
        double* f = static_cast<double*>(P.film[which]) + 3 * size_t(pix);
        atomicAdd(f, double(v.x));
        atomicAdd(f + 1, double(v.y));
        atomicAdd(f + 2, double(v.z));
    } else {
        float* f = static_cast<float*>(P.film[which]) + 3 * size_t(pix);
        atomicAdd(f, v.x);
        atomicAdd(f + 1, v.y);
        atomicAdd(f + 2, v.z);
    }
}

// A finished path adds L/spp to its film(s).
__device__ __forceinline__ void deposit(const PtParams& P, uint32_t p, f3 L) {
    const uint2 k = P.st.key[p];
    const uint32_t role = P.st.meta[p] >> 24;
    const f3 v = L * P.inv_spp;
    if (!P.gdpt) {
        film_add(P, 0, k.x, v);
        return;
    }
    const uint32_t px = k.x % P.width, py = k.x / P.width;
    if (role == kRoleBase) {
        film_add(P, 0, k.x, v);
        if (px + 1 < P.width) film_add(P, 1, k.x, -v);
        if (py + 1 < P.height) film_add(P, 2, k.x, -v);
    } else {
        film_add(P, role == kRoleRight ? 1 : 2, k.x, v);
    }
}

__global__ void __launch_bounds__(256) k_generate(PtParams P) {
    const uint32_t npix = P.width * P.height;
    const uint32_t roles = P.gdpt ? 3u : 1u;
    const uint32_t total = P.chunk_samples * roles;
    for (uint32_t base = blockIdx.x * blockDim.x; base < total; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        bool live = i < total;
        uint32_t p = i, pixel = 0, sample = 0, role = 0, px = 0, py = 0;
        if (live) {
            const uint32_t si = i / roles;
            role = i - si * roles;
            const uint64_t g = P.sample_begin + si;
            pixel = uint32_t(g % npix);
            sample = uint32_t(g / npix);
            px = pixel % P.width;
            py = pixel / P.width;
            if (role == kRoleRight && px + 1 >= P.width) live = false;
            if (role == kRoleDown && py + 1 >= P.height) live = false;
        }
        const uint32_t slot = warp_alloc(&P.st.counts[0], live);
        if (!live) continue;
        const uint64_t key = counter_key(P.seed, pixel, sample);
        const float jx = counter_u01(key, 0), jy = counter_u01(key, 1);
        const uint32_t ox = px + (role == kRoleRight ? 1u : 0u), oy = py + (role == kRoleDown ? 1u : 0u);
        const float u = (float(ox) + jx) / float(P.width);
        const float v = 1.0f - (float(oy) + jy) / float(P.height);
        const Ray r = camera_ray(P.cam, u, v);
        P.st.key[p] = make_uint2(pixel, sample);
        P.st.thr[p] = make_float4(1.f, 1.f, 1.f, 0.f);
        P.st.rad[p] = make_float4(0.f, 0.f, 0.f, 0.f);
        P.st.meta[p] = (2u << 8) | (role << 24);
        P.st.ray_o[0][slot] = make_float4(r.o.x, r.o.y, r.o.z, r.tmin);
        P.st.ray_d[0][slot] = make_float4(r.d.x, r.d.y, r.d.z, r.tmax);
        P.st.qpath[0][slot] = p;
    }
}

__global__ void __launch_bounds__(128) k_extend(PtParams P, uint32_t depth, int* err) {
    const uint32_t n = P.st.counts[depth];
    const int q = depth & 1;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const float4 a = P.st.ray_o[q][j], b = P.st.ray_d[q][j];
        const Ray r{mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w};
        HitRec h;
        traverse<false>(P.sc, r, h, err);
        P.st.hit[j] = make_float4(h.t, h.u, h.v, __uint_as_float(h.slot));
        P.st.hit_inst[j] = h.inst;
    }
}

__global__ void __launch_bounds__(256) k_shade(PtParams P, uint32_t depth) {
    const uint32_t n = P.st.counts[depth];
    const int q = depth & 1;
    uint32_t* out_count = &P.st.counts[depth + 1];
    uint32_t* sh_count = &P.st.counts[64 + depth];
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t j = base + threadIdx.x;
        const bool active = j < n;
        bool cont = false, shadow = false;
        uint32_t p = 0;
        f3 new_o, new_d, sh_o, sh_d, sh_c;
        float sh_tmax = 0.f;
        f3 L, thr;
        float prev_pdf = 0.f;
        uint32_t meta = 0;
        if (active) {
            p = P.st.qpath[q][j];
            const float4 h = P.st.hit[j];
            const float4 t4 = P.st.thr[p], r4 = P.st.rad[p];
            thr = mk(t4.x, t4.y, t4.z);
            prev_pdf = t4.w;
            L = mk(r4.x, r4.y, r4.z);
            meta = P.st.meta[p];
            const uint32_t slot = __float_as_uint(h.w);
            if (slot != kInvalid) {
                const uint2 k = P.st.key[p];
                const uint64_t key = counter_key(P.seed, k.x, k.y);
                uint32_t dim = (meta >> 8) & 0xffffu;
                const float4 ro4 = P.st.ray_o[q][j], rd4 = P.st.ray_d[q][j];
                const f3 ro = mk(ro4.x, ro4.y, ro4.z), rd = mk(rd4.x, rd4.y, rd4.z);
                const Shade s = make_shade(P.sc, ro, rd, h.x, h.y, h.z, slot, P.st.hit_inst[j]);
                const MatView m = load_mat(P.sc, s.mat);
                const f3 wo = -rd;
                const f3 wo_l = to_local(s.onb, wo);
                const bool lights_on = light_enabled(P.sc);
                // Emission on hit (area-light extension).
                if (m.emitter >= 0) {
                    const LightView lt = load_light(P.sc, uint32_t(m.emitter));
                    const float cos_l = dot(lt.n, wo);
                    if (cos_l > 0.f) {
                        if (depth == 0 || !lights_on) {
                            L = L + thr * lt.inten;
                        } else {
                            const float pdf_light =
                                light_pmf_of(P.sc, uint32_t(m.emitter)) * (h.x * h.x) / (cos_l * lt.area);
                            const float w = power_heuristic(prev_pdf, pdf_light);
                            L = L + (thr * lt.inten) * w;
                        }
                    }
                }
                // Next-event estimation: one light, one shadow ray.
                if (lights_on) {
                    const float u_sel = counter_u01(key, dim++);
                    const float ulx = counter_u01(key, dim++);
                    const float uly = counter_u01(key, dim++);
                    uint32_t li;
                    float sel;
                    light_select(P.sc, u_sel, li, sel);
                    const LightView light = load_light(P.sc, li);
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
                                const f3 off = (s.n * 1e-4f) * signum(dot(wi, s.n));
                                sh_o = s.p + off;
                                sh_d = normalize(wi);
                                sh_tmax = dist * (1.0f - 1e-4f);
                                sh_c = c;
                                shadow = true;
                            }
                        }
                    }
                }
                // BSDF sampling, Russian roulette, spawn.
                const float u_bsel = counter_u01(key, dim++);
                (void)u_bsel;
                const float udx = counter_u01(key, dim++);
                const float udy = counter_u01(key, dim++);
                f3 wi, f;
                float pdf;
                if (bsdf_sample(m, wo_l, udx, udy, wi, pdf, f) && pdf != 0.f && !is_zero(f)) {
                    const float cos_wi = fabsf(wi.z);
                    thr = thr * ((f * cos_wi) / pdf);
                    prev_pdf = pdf;
                    bool alive = true;
                    if (depth + 1 >= P.rr_depth) {
                        const float survival = fminf(max3(thr), 0.95f);
                        if (counter_u01(key, dim++) > survival) alive = false;
                        else thr = thr / survival;
                    }
                    if (alive && depth + 1 < P.max_depth) {
                        const f3 wi_w = to_world(s.onb, wi);
                        const f3 off = (s.n * 1e-4f) * signum(dot(wi_w, s.n));
                        new_o = s.p + off;
                        new_d = normalize(wi_w);
                        cont = true;
                    }
                }
                meta = (meta & 0xff000000u) | (dim << 8) | (depth + 1);
            }
        }
        const uint32_t rs = warp_alloc(out_count, cont);
        const uint32_t ss = warp_alloc(sh_count, shadow);
        if (!active) continue;
        if (cont) {
            P.st.ray_o[q ^ 1][rs] = make_float4(new_o.x, new_o.y, new_o.z, 1e-4f);
            P.st.ray_d[q ^ 1][rs] = make_float4(new_d.x, new_d.y, new_d.z, FLT_MAX);
            P.st.qpath[q ^ 1][rs] = p;
            P.st.thr[p] = make_float4(thr.x, thr.y, thr.z, prev_pdf);
            P.st.meta[p] = meta;
        }
        if (shadow) {
            P.st.sh_o[ss] = make_float4(sh_o.x, sh_o.y, sh_o.z, 0.f);
            P.st.sh_d[ss] = make_float4(sh_d.x, sh_d.y, sh_d.z, sh_tmax);
            P.st.sh_c[ss] = make_float4(sh_c.x, sh_c.y, sh_c.z, 0.f);
            P.st.sh_path[ss] = p | (cont ? 0u : kFinal);
        }
        if (cont || shadow) {
            P.st.rad[p] = make_float4(L.x, L.y, L.z, 0.f);
        } else {
            deposit(P, p, L);
        }
    }
}

__global__ void __launch_bounds__(128) k_shadow(PtParams P, uint32_t depth, int* err) {
    const uint32_t n = P.st.counts[64 + depth];
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
        const float4 a = P.st.sh_o[m], b = P.st.sh_d[m];
        const Ray r{mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w};
        HitRec h;
        traverse<true>(P.sc, r, h, err);
        const uint32_t e = P.st.sh_path[m];
        const uint32_t p = e & ~kFinal;
        const float4 r4 = P.st.rad[p];
        f3 L = mk(r4.x, r4.y, r4.z);
        if (h.slot == kInvalid) {
            const float4 c = P.st.sh_c[m];
            L = L + mk(c.x, c.y, c.z);
        }
        if (e & kFinal) deposit(P, p, L);
        else P.st.rad[p] = make_float4(L.x, L.y, L.z, 0.f);
    }
}

// Folds one chunk's queue counters into the context's 64-bit work counters:
// [0] paths, [1] closest-hit rays, [2] shadow rays.
__global__ void k_count(const uint32_t* counts, uint32_t max_depth, unsigned long long* stats) {
    __shared__ unsigned long long ext, sh;
    if (threadIdx.x == 0) { ext = 0; sh = 0; }
    __syncthreads();
    if (threadIdx.x < max_depth) {
        atomicAdd(&ext, (unsigned long long)counts[threadIdx.x]);
        atomicAdd(&sh, (unsigned long long)counts[64 + threadIdx.x]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        stats[0] += counts[0];
        stats[1] += ext;
        stats[2] += sh;
    }
}

template <class T>
T* carve(char*& cur, size_t n) {
    cur = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(cur) + 255) & ~uintptr_t(255));
    T* p = reinterpret_cast<T*>(cur);
    cur += n * sizeof(T);
    return p;
}

}  // namespace

void render_pt_films(ar_context* ctx, const ar_scene* sc, const CameraDev& cam, const ar_integrator_cfg& cfg,
                     uint32_t w, uint32_t h, bool gdpt, void* films) {
    AR_REQUIRE(cfg.max_depth <= 63, AR_ERR_INVALID_ARGUMENT, "max_depth must be <= 63");
    const uint64_t total = uint64_t(w) * h * cfg.spp;
    const uint32_t roles = gdpt ? 3u : 1u;
    // Path capacity: up to 2M path slots per chunk.
    const uint32_t cap_paths = 1u << 21;
    const uint32_t chunk = uint32_t(std::min<uint64_t>(total, cap_paths / roles));
    const uint32_t cap = chunk * roles;
    size_t bytes = 0;
    bytes += cap * (sizeof(uint2) + 2 * sizeof(float4) + sizeof(uint32_t));
    bytes += 2 * cap * (2 * sizeof(float4) + sizeof(uint32_t));
    bytes += cap * (sizeof(float4) + sizeof(uint32_t));
    bytes += cap * (3 * sizeof(float4) + sizeof(uint32_t));
    bytes += 128 * sizeof(uint32_t) + 32 * 256;
    ctx->work.ensure(bytes);
    char* cur = ctx->work.buf.as<char>();
    PtParams P{};
    P.sc = sc->view;
    P.cam = cam;
    P.st.key = carve<uint2>(cur, cap);
    P.st.thr = carve<float4>(cur, cap);
    P.st.rad = carve<float4>(cur, cap);
    P.st.meta = carve<uint32_t>(cur, cap);
    for (int b = 0; b < 2; ++b) {
        P.st.ray_o[b] = carve<float4>(cur, cap);
        P.st.ray_d[b] = carve<float4>(cur, cap);
        P.st.qpath[b] = carve<uint32_t>(cur, cap);
    }
    P.st.hit = carve<float4>(cur, cap);
    P.st.hit_inst = carve<uint32_t>(cur, cap);
    P.st.sh_o = carve<float4>(cur, cap);
    P.st.sh_d = carve<float4>(cur, cap);
    P.st.sh_c = carve<float4>(cur, cap);
    P.st.sh_path = carve<uint32_t>(cur, cap);
    P.st.counts = carve<uint32_t>(cur, 128);
    P.width = w;
    P.height = h;
    P.spp = cfg.spp;
    P.max_depth = cfg.max_depth;
    P.rr_depth = cfg.rr_depth;
    P.gdpt = gdpt ? 1u : 0u;
    P.film64 = cfg.film_precision == AR_FILM_F64 ? 1u : 0u;
    P.seed = cfg.seed;
    P.inv_spp = 1.0f / float(cfg.spp);
    const size_t film_bytes = size_t(w) * h * 3 * (P.film64 ? sizeof(double) : sizeof(float));
    for (int f = 0; f < int(roles); ++f) {
        P.film[f] = static_cast<char*>(films) + f * film_bytes;
    }
    AR_CUDA(cudaMemsetAsync(films, 0, film_bytes * roles, ctx->stream));
    AR_CUDA(cudaMemsetAsync(ctx->stats_d.ptr, 0, 8 * sizeof(uint64_t), ctx->stream));
    const int grid_wide = ctx->num_sms * 8;
    int* err = ctx->err_flag.as<int>();
    uint64_t chunks = 0;
    for (uint64_t begin = 0; begin < total; begin += chunk, ++chunks) {
        P.sample_begin = begin;
        P.chunk_samples = uint32_t(std::min<uint64_t>(chunk, total - begin));
        AR_CUDA(cudaMemsetAsync(P.st.counts, 0, 128 * sizeof(uint32_t), ctx->stream));
        const int gen_grid = int(std::min<uint64_t>((uint64_t(P.chunk_samples) * roles + 255) / 256, grid_wide));
        {
            KernelScope ks(ctx->prof, ctx->stream, "pt_generate");
            k_generate<<<std::max(1, gen_grid), 256, 0, ctx->stream>>>(P);
        }
        for (uint32_t d = 0; d < cfg.max_depth; ++d) {
            {
                KernelScope ks(ctx->prof, ctx->stream, "pt_extend");
                k_extend<<<ctx->num_sms * 16, 128, 0, ctx->stream>>>(P, d, err);
            }
            {
                KernelScope ks(ctx->prof, ctx->stream, "pt_shade");
                k_shade<<<grid_wide, 256, 0, ctx->stream>>>(P, d);
            }
            {
                KernelScope ks(ctx->prof, ctx->stream, "pt_shadow");
                k_shadow<<<ctx->num_sms * 16, 128, 0, ctx->stream>>>(P, d, err);
            }
        }
        k_count<<<1, 64, 0, ctx->stream>>>(P.st.counts, cfg.max_depth, ctx->stats_d.as<unsigned long long>());
        AR_CUDA(cudaGetLastError());
    }
    // Counters land in pinned memory; ar_get_render_stats reads them after a sync.
    AR_CUDA(cudaMemcpyAsync(ctx->stats_h, ctx->stats_d.ptr, 8 * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                            ctx->stream));
    ctx->stats_pending = true;
    ctx->last_stats.path_samples = total;
    ctx->last_stats.extend_launches = chunks * cfg.max_depth;
    ctx->last_stats.shadow_launches = chunks * cfg.max_depth;
}

}  // namespace ar
