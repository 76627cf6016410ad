// ORACLE — test infrastructure only.  C entry points over the CPU restatement
// of agent-ray (ar_*.hpp) for the pytest suite, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py.  PARITY UNPINNED (see ar_math.hpp).
#include <cmath>
#include <chrono>
#include <cstdio>
#include <memory>
#include "ar_integrators.hpp"

using namespace oracle;

namespace {
struct OracleScene {
    int precision;  // 32 or 64
    std::unique_ptr<Scene<float>> f;
    std::unique_ptr<Scene<double>> d;
};

template <class T>
void trace_impl(const Scene<T>& sc, const float* ot, const float* dt, uint64_t n, int any, float* t_out, float* u_out,
                float* v_out, uint32_t* prim, uint32_t* inst, uint8_t* occ, uint64_t* stats, uint32_t threads) {
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    std::atomic<uint64_t> next{0};
    std::vector<TraversalStats> st(threads);
    std::vector<std::thread> pool;
    const uint64_t chunk = 1024;
    for (uint32_t th = 0; th < threads; ++th)
        pool.emplace_back([&, th] {
            for (;;) {
                uint64_t b = next.fetch_add(chunk);
                if (b >= n) break;
                uint64_t e = std::min(n, b + chunk);
                for (uint64_t i = b; i < e; ++i) {
                    Ray<T> r = Ray<T>::make(V3<T>(T(ot[4 * i]), T(ot[4 * i + 1]), T(ot[4 * i + 2])),
                                            V3<T>(T(dt[4 * i]), T(dt[4 * i + 1]), T(dt[4 * i + 2])), T(ot[4 * i + 3]),
                                            T(dt[4 * i + 3]));
                    Hit<T> h = sc.tlas_intersect(r, stats ? &st[th] : nullptr);
                    if (any) {
                        occ[i] = h.valid ? 1 : 0;
                        continue;
                    }
                    if (h.valid) {
                        t_out[i] = float(h.t);
                        u_out[i] = float(h.u);
                        v_out[i] = float(h.v);
                        prim[i] = h.prim;
                        inst[i] = h.inst;
                    } else {
                        t_out[i] = INFINITY;
                        u_out[i] = 0.f;
                        v_out[i] = 0.f;
                        prim[i] = 0xFFFFFFFFu;
                        inst[i] = 0xFFFFFFFFu;
                    }
                }
            }
        });
    for (auto& p : pool) p.join();
    if (stats) {
        stats[0] = stats[1] = stats[2] = 0;
        for (auto& s : st) {
            stats[0] += s.nodes;
            stats[1] += s.tris;
            stats[2] += s.instances;
        }
    }
}

template <class T>
int render_impl(const Scene<T>& sc, const ar_camera_desc* cd, const ar_integrator_cfg* cfg, uint32_t w, uint32_t h,
                uint32_t sampler, uint32_t threads, double* out, double* moments, double* gx_out, double* gy_out) {
    Camera<T> cam = Camera<T>::from_lookat(*cd);
    RenderOpts o;
    o.sampler = sampler;
    o.threads = threads;
    o.seed = cfg->seed;
    size_t n = size_t(w) * h * 3;
    std::vector<T> buf(n), mom(moments ? n : 0);
    if (cfg->integrator == AR_INTEGRATOR_PT) {
        render_pt(sc, cam, *cfg, w, h, o, buf.data(), moments ? mom.data() : nullptr);
    } else if (cfg->integrator == AR_INTEGRATOR_BDPT) {
        render_bdpt(sc, cam, *cfg, w, h, o, buf.data());
    } else if (cfg->integrator == AR_INTEGRATOR_GDPT) {
        std::vector<T> pr(n), gx(n), gy(n);
        render_gdpt_films(sc, cam, *cfg, w, h, o, pr.data(), gx.data(), gy.data());
        if (gx_out)
            for (size_t i = 0; i < n; ++i) { gx_out[i] = double(gx[i]); gy_out[i] = double(gy[i]); }
        if (moments)
            for (size_t i = 0; i < n; ++i) mom[i] = pr[i];  // primal film
        poisson_sor(w, h, pr.data(), gx.data(), gy.data(), T(cfg->alpha), cfg->poisson_iterations, T(cfg->sor_omega),
                    buf.data(), (cfg->gdpt_flags & AR_GDPT_CONSISTENT_DIVERGENCE) != 0);
    } else {
        return -1;
    }
    for (size_t i = 0; i < n; ++i) out[i] = double(buf[i]);
    if (moments)
        for (size_t i = 0; i < n; ++i) moments[i] = double(mom[i]);
    return 0;
}
}  // namespace

extern "C" {

int oracle_scene_create(const ar_scene_desc* desc, int precision, void** out) {
    auto* s = new OracleScene();
    s->precision = precision;
    if (precision == 64) {
        s->d.reset(new Scene<double>());
        s->d->load(*desc);
    } else {
        s->f.reset(new Scene<float>());
        s->f->load(*desc);
    }
    *out = s;
    return 0;
}

void oracle_scene_destroy(void* s) { delete static_cast<OracleScene*>(s); }

// Closest hit (any == 0) or occlusion (any != 0) for n rays given as float4
// (origin, t_min) and (direction, t_max).  stats (optional, 3 entries): node
// visits, triangle tests and instance entries of the reference traversal.
int oracle_trace(void* sp, const float* org_tmin, const float* dir_tmax, uint64_t n, int any, float* t, float* u,
                 float* v, uint32_t* prim, uint32_t* inst, uint8_t* occluded, uint64_t* stats, uint32_t threads) {
    auto* s = static_cast<OracleScene*>(sp);
    if (s->precision == 64)
        trace_impl(*s->d, org_tmin, dir_tmax, n, any, t, u, v, prim, inst, occluded, stats, threads);
    else
        trace_impl(*s->f, org_tmin, dir_tmax, n, any, t, u, v, prim, inst, occluded, stats, threads);
    return 0;
}

// Integrator::render.  out: W*H*3.  For PT, `aux0` (optional) receives the
// per-pixel mean of squared sample radiance; for GDPT `aux0` receives the
// primal film and aux1/aux2 the dx/dy gradient films.
int oracle_render(void* sp, const ar_camera_desc* cam, const ar_integrator_cfg* cfg, uint32_t w, uint32_t h,
                  uint32_t sampler, uint32_t threads, double* out, double* aux0, double* aux1, double* aux2) {
    auto* s = static_cast<OracleScene*>(sp);
    if (s->precision == 64) return render_impl(*s->d, cam, cfg, w, h, sampler, threads, out, aux0, aux1, aux2);
    return render_impl(*s->f, cam, cfg, w, h, sampler, threads, out, aux0, aux1, aux2);
}

// screened_poisson_reconstruct in f32 (the reference precision).
int oracle_poisson_sor_f32(uint32_t w, uint32_t h, const float* primal, const float* gx, const float* gy, float alpha,
                           uint32_t iters, float omega, float* out) {
    poisson_sor<float>(w, h, primal, gx, gy, alpha, iters, omega, out);
    return 0;
}

// Unclamped FP64 solution of the screened-Poisson system (converged CG).
int oracle_poisson_exact_f64(uint32_t w, uint32_t h, const double* primal, const double* gx, const double* gy,
                             double alpha, double tol, uint32_t max_iters, double* out, double* rel_res) {
    poisson_cg_exact(w, h, primal, gx, gy, alpha, tol, max_iters, out, rel_res);
    return 0;
}

// Counter-sampler values u(dim) for dims [dim0, dim0 + n).
int oracle_counter_u01(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t dim0, uint32_t n, float* out) {
    uint64_t key = counter_key(seed, pixel, sample);
    for (uint32_t i = 0; i < n; ++i) out[i] = counter_u01(key, dim0 + i);
    return 0;
}

// Film::to_rgb_image (src/film.rs:276-302) with tonemap_pixel (:153-181):
// scale, tone-map, clamp, powf(1/gamma), (x * 255 + 0.5).min(255) as u8.
// Every operation is a separate f32 rounding in the reference's order.
int oracle_film_to_rgb8(const float* hdr, uint32_t w, uint32_t h, uint32_t tm, float white_point, float gamma,
                        float scale, uint8_t* out) {
    const float inv_gamma = 1.0f / gamma;
    const size_t n = size_t(w) * h;
    for (size_t i = 0; i < n; ++i) {
        float c[3] = {hdr[3 * i] * scale, hdr[3 * i + 1] * scale, hdr[3 * i + 2] * scale};
        float s = 1.0f;
        const float lum = (0.2126f * c[0] + 0.7152f * c[1]) + 0.0722f * c[2];
        if (tm == 1) {
            s = lum > 1e-6f ? (lum / (1.0f + lum)) / lum : 1.0f / (1.0f + lum);
        } else if (tm == 2) {
            const float lw2 = white_point * white_point;
            const float mapped = (lum * (1.0f + lum / lw2)) / (1.0f + lum);
            s = lum > 1e-6f ? mapped / lum : 1.0f;
        }
        for (int k = 0; k < 3; ++k) {
            float m = tm == 0 ? c[k] : c[k] * s;
            m = std::min(std::max(m, 0.0f), 1.0f);  // Vec3A::clamp(ZERO, ONE)
            const float e = std::pow(m, inv_gamma);
            const float v = std::min(e * 255.0f + 0.5f, 255.0f);
            out[3 * i + k] = v > 0.0f ? uint8_t(v) : uint8_t(0);  // Rust `as u8` saturates
        }
    }
    return 0;
}

// ImageTexture::load + sample (src/texture.rs:77-136) at n uv pairs, in f32.
int oracle_texture_sample(const uint8_t* rgb8, uint32_t w, uint32_t h, const float* uv, uint32_t n, float* out) {
    if (!rgb8 || w == 0 || h == 0) return 1;
    Texture<float> t;
    t.load(ar_texture_desc{rgb8, w, h});
    for (uint32_t i = 0; i < n; ++i) {
        const V3<float> c = t.sample(V2<float>{uv[2 * i], uv[2 * i + 1]});
        out[3 * i] = c.x;
        out[3 * i + 1] = c.y;
        out[3 * i + 2] = c.z;
    }
    return 0;
}

// First n f32 draws of the pixel-seeded independent sampler (xoshiro256++).
int oracle_xoshiro_f32(uint32_t px, uint32_t py, uint32_t n, float* out) {
    Sampler s(SAMPLER_XOSHIRO, px, py, 1, 0);
    for (uint32_t i = 0; i < n; ++i) out[i] = s.next_1d();
    return 0;
}

// sin and cos of n FP32 angles through the routine the FP32 oracle samples with.
int oracle_sincos_f32(const float* x, uint64_t n, float* s, float* c) {
    for (uint64_t i = 0; i < n; ++i) sin_cos(x[i], s[i], c[i]);
    return 0;
}

// Structure of the restated reference BVH: node count, leaf count, max depth.
int oracle_blas_stats(void* sp, uint32_t mesh, uint64_t* out3) {
    auto* s = static_cast<OracleScene*>(sp);
    const BuildResult& b = s->precision == 64 ? s->d->meshes[mesh].bvh : s->f->meshes[mesh].bvh;
    uint64_t leaves = 0;
    for (auto& nd : b.nodes) leaves += nd.leaf() ? 1 : 0;
    // depth by explicit stack
    uint64_t maxd = 0;
    if (!b.nodes.empty()) {
        std::vector<std::pair<uint32_t, uint32_t>> st{{0u, 1u}};
        while (!st.empty()) {
            auto [i, d] = st.back();
            st.pop_back();
            maxd = std::max<uint64_t>(maxd, d);
            if (!b.nodes[i].leaf()) {
                st.push_back({b.nodes[i].left_or_start, d + 1});
                st.push_back({b.nodes[i].right_or_end, d + 1});
            }
        }
    }
    out3[0] = b.nodes.size();
    out3[1] = leaves;
    out3[2] = maxd;
    return 0;
}

}  // extern "C"
