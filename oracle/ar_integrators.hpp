// ORACLE — test infrastructure only (see ar_math.hpp header; parity unpinned).
// Restates agent-ray's integrators:
//   PathTracer::li / render        src/integrators/path_tracer.rs:59-205
//   BDPT subpaths, mis_weight, connect_bdpt, connect_bdpt_s1, render
//                                  src/integrators/bidirectional_path_tracer.rs:158-1357
//   ReplaySampler, trace_with_gradients, render, screened_poisson_reconstruct
//                                  src/integrators/gradient_domain_pt.rs:91-630
// Quad area-light support (emission on hit with MIS in PT/GDPT, the t=0 and
// area-light t=1 BDPT strategies) is an EXTENSION, marked where it appears.
#pragma once
#include <atomic>
#include <cstring>
#include "ar_scene.hpp"

namespace oracle {

template <class T> inline T power_heuristic(T a, T b) { T a2 = a * a, b2 = b * b; return a2 / (a2 + b2); }

struct RenderOpts {
    uint32_t sampler = SAMPLER_COUNTER;
    uint32_t threads = 0;
    uint64_t seed = 0;
};

// Row-parallel loop (rayon into_par_iter over rows in the reference).
template <class F>
inline void parallel_rows(uint32_t height, uint32_t threads, F&& f) {
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            for (;;) {
                uint32_t y = next.fetch_add(1);
                if (y >= height) break;
                f(y, t);
            }
        });
    for (auto& th : pool) th.join();
}

// ---------------------------------------------------------------------------
// Path tracer (path_tracer.rs:59-156) + EXTENSION: emitter hits add Le, MIS-
// weighted against light sampling after the first bounce.
// ---------------------------------------------------------------------------
template <class T, class S>
V3<T> pt_li(const Scene<T>& sc, Ray<T> ray, S& sampler, uint32_t max_depth, uint32_t rr_depth) {
    V3<T> L(0, 0, 0), thr(1, 1, 1);
    T prev_pdf = T(0);
    for (uint32_t depth = 0; depth < max_depth; ++depth) {
        ShadingPoint<T> hit;
        if (!sc.intersect(ray, hit)) break;
        V3<T> wo = -ray.d;
        V3<T> wo_l = hit.onb.to_local(wo);
        const Material<T>& m = *hit.mat;
        if (m.emitter >= 0) {  // EXTENSION
            const Light<T>& lt = sc.lights[m.emitter];
            T cos_l = dot(lt.n, wo);
            if (cos_l > T(0)) {
                if (depth == 0 || !sc.ldist.enabled()) {
                    L += thr * lt.intensity;
                } else {
                    T pdf_light = sc.ldist.pmf_of(uint32_t(m.emitter)) * (hit.t * hit.t) / (cos_l * lt.area);
                    T w = power_heuristic(prev_pdf, pdf_light);
                    L += (thr * lt.intensity) * w;
                }
            }
        }
        if (sc.ldist.enabled()) {
            T u_sel = T(sampler.next_1d());
            uint32_t li_idx;
            T sel;
            sc.ldist.sample_index(u_sel, li_idx, sel);
            const Light<T>& light = sc.lights[li_idx];
            V2<T> ul{T(sampler.next_1d()), T(0)};
            ul.y = T(sampler.next_1d());
            LightSample<T> ls = light.sample(hit.p, ul);
            if (ls.valid) {
                V3<T> off = hit.n * T(1e-4f) * signum(dot(ls.wi, hit.n));
                Ray<T> sr = Ray<T>::make(hit.p + off, ls.wi, T(0), ls.dist * (T(1) - T(1e-4f)));
                if (!sc.occluded(sr)) {
                    V3<T> wi_l = hit.onb.to_local(ls.wi);
                    T cos_wi = std::fabs(wi_l.z);
                    if (cos_wi > T(0)) {
                        V3<T> f = m.eval(wi_l, wo_l, hit.uv);
                        if (light.is_delta()) {
                            L += ((thr * f) * cos_wi) * ls.li / sel;
                        } else {
                            T pdf_light = ls.pdf * sel;
                            T pdf_bsdf = m.pdf(wi_l, wo_l);
                            T w = power_heuristic(pdf_light, pdf_bsdf);
                            L += ((((thr * f) * cos_wi) * ls.li) * w) / pdf_light;
                        }
                    }
                }
            }
        }
        T u_sel = T(sampler.next_1d());
        V2<T> ud{T(sampler.next_1d()), T(0)};
        ud.y = T(sampler.next_1d());
        BsdfSample<T> bs = m.sample(wo_l, hit.uv, u_sel, ud);
        if (!bs.valid) break;
        if (bs.pdf == T(0) || bs.f == V3<T>(0, 0, 0)) break;
        T cos_wi = std::fabs(bs.wi.z);
        thr *= (bs.f * cos_wi) / bs.pdf;
        prev_pdf = bs.pdf;
        if (depth + 1 >= rr_depth) {
            T survival = rmin(max_element(thr), T(0.95f));
            if (T(sampler.next_1d()) > survival) break;
            thr /= survival;
        }
        V3<T> wi_w = hit.onb.to_world(bs.wi);
        V3<T> off = hit.n * T(1e-4f) * signum(dot(wi_w, hit.n));
        ray = Ray<T>::make(hit.p + off, wi_w, T(1e-4f), ray_unbounded<T>());
    }
    return L;
}

// PathTracer::render (path_tracer.rs:159-190).  out: W*H*3 (accum / spp).
// moments (optional): W*H*3 per-channel mean of squared per-sample radiance.
template <class T>
void render_pt(const Scene<T>& sc, const Camera<T>& cam, const ar_integrator_cfg& cfg, uint32_t w, uint32_t h,
               const RenderOpts& o, T* out, T* moments) {
    parallel_rows(h, o.threads, [&](uint32_t y, uint32_t) {
        for (uint32_t x = 0; x < w; ++x) {
            Sampler smp(o.sampler, x, y, w, o.seed);
            V3<T> acc(0, 0, 0), acc2(0, 0, 0);
            for (uint32_t s = 0; s < cfg.spp; ++s) {
                smp.start_sample(s);
                T jx = T(smp.next_1d());
                T jy = T(smp.next_1d());
                T u = (T(float(x)) + jx) / T(float(w));
                T v = T(1) - (T(float(y)) + jy) / T(float(h));
                Ray<T> ray = cam.generate_ray({u, v});
                V3<T> Ls = pt_li(sc, ray, smp, cfg.max_depth, cfg.rr_depth);
                acc += Ls;
                acc2 += Ls * Ls;
            }
            size_t i = (size_t(y) * w + x) * 3;
            V3<T> r = acc / T(float(cfg.spp));
            out[i] = r.x; out[i + 1] = r.y; out[i + 2] = r.z;
            if (moments) {
                V3<T> r2 = acc2 / T(float(cfg.spp));
                moments[i] = r2.x; moments[i + 1] = r2.y; moments[i + 2] = r2.z;
            }
        }
    });
}

// ---------------------------------------------------------------------------
// BDPT (bidirectional_path_tracer.rs)
// ---------------------------------------------------------------------------
enum VType : uint8_t { V_CAMERA, V_LIGHT, V_SURFACE };

template <class T>
struct PathVertex {
    VType type;
    V3<T> p, n;
    Onb<T> onb;
    const Material<T>* mat;
    V3<T> thr;
    T pdf_fwd, pdf_rev;
    bool is_delta;
    int32_t light;
    V2<T> uv;  // tex_uv of surface vertices
    bool connectible() const { return type != V_SURFACE || !is_delta; }  // :281-292
};

// :305-314
template <class T>
inline T pdf_sa_to_area(T pdf, V3<T> from, V3<T> to, V3<T> n_to) {
    V3<T> d = to - from;
    T d2 = length_squared(d);
    if (d2 < T(1e-12f)) return T(0);
    V3<T> dir = d / std::sqrt(d2);
    T c = std::fabs(dot(n_to, dir));
    return pdf * c / d2;
}
// :318-328
template <class T>
inline T geometry_term(V3<T> pa, V3<T> na, V3<T> pb, V3<T> nb) {
    V3<T> d = pb - pa;
    T d2 = length_squared(d);
    if (d2 < T(1e-12f)) return T(0);
    V3<T> dir = d / std::sqrt(d2);
    T ca = std::fabs(dot(na, dir));
    T cb = std::fabs(dot(nb, -dir));
    return ca * cb / d2;
}

template <class T, class S>
inline void bdpt_subpath_walk(const Scene<T>& sc, Ray<T> ray, V3<T> thr, T prev_pdf_dir, uint32_t max_depth,
                              uint32_t rr_depth, S& smp, std::vector<PathVertex<T>>& vs) {
    for (uint32_t depth = 0; depth < max_depth; ++depth) {
        ShadingPoint<T> hit;
        if (!sc.intersect(ray, hit)) break;
        T pdf_fwd = pdf_sa_to_area(prev_pdf_dir, vs.back().p, hit.p, hit.n);
        PathVertex<T> v{V_SURFACE, hit.p, hit.n, hit.onb, hit.mat, thr, pdf_fwd, T(0), false, -1, hit.uv};
        vs.push_back(v);
        V3<T> wo = -ray.d;
        V3<T> wo_l = hit.onb.to_local(wo);
        T u_sel = T(smp.next_1d());
        V2<T> ud{T(smp.next_1d()), T(0)};
        ud.y = T(smp.next_1d());
        BsdfSample<T> bs = hit.mat->sample(wo_l, hit.uv, u_sel, ud);
        if (!bs.valid) break;
        if (bs.pdf == T(0) || bs.f == V3<T>(0, 0, 0)) break;
        T cos_wi = std::fabs(bs.wi.z);
        thr *= (bs.f * cos_wi) / bs.pdf;
        prev_pdf_dir = bs.pdf;
        T pdf_rev_dir = hit.mat->pdf(wo_l, bs.wi);
        size_t prev = vs.size() - 2;
        vs[prev].pdf_rev = pdf_sa_to_area(pdf_rev_dir, hit.p, vs[prev].p, vs[prev].n);
        if (depth + 1 >= rr_depth) {
            T survival = rmin(max_element(thr), T(0.95f));
            if (T(smp.next_1d()) > survival || survival <= T(0)) break;
            thr /= survival;
        }
        V3<T> wi_w = hit.onb.to_world(bs.wi);
        V3<T> off = hit.n * T(1e-4f) * signum(dot(wi_w, hit.n));
        ray = Ray<T>::make(hit.p + off, wi_w, T(1e-4f), ray_unbounded<T>());
    }
}

// generate_camera_subpath (:338-437)
template <class T, class S>
void gen_camera_subpath(const Scene<T>& sc, const Camera<T>& cam, const Ray<T>& ray, uint32_t max_depth,
                        uint32_t rr_depth, S& smp, std::vector<PathVertex<T>>& vs) {
    vs.clear();
    PathVertex<T> c{V_CAMERA, cam.origin, ray.d, Onb<T>::from_normal(ray.d), nullptr, V3<T>(1, 1, 1), T(1), T(0), true, -1};
    vs.push_back(c);
    bdpt_subpath_walk(sc, ray, V3<T>(1, 1, 1), cam.pdf_we(ray), max_depth, rr_depth, smp, vs);
}

// generate_light_subpath (:443-559)
template <class T, class S>
void gen_light_subpath(const Scene<T>& sc, uint32_t max_depth, uint32_t rr_depth, S& smp,
                       std::vector<PathVertex<T>>& vs) {
    vs.clear();
    if (!sc.ldist.enabled()) return;
    T u_sel = T(smp.next_1d());
    uint32_t li;
    T sel;
    sc.ldist.sample_index(u_sel, li, sel);
    const Light<T>& light = sc.lights[li];
    V2<T> up{T(smp.next_1d()), T(0)};
    up.y = T(smp.next_1d());
    V2<T> ud{T(smp.next_1d()), T(0)};
    ud.y = T(smp.next_1d());
    EmissionSample<T> es = light.sample_emission(up, ud);
    if (!es.valid) return;
    PathVertex<T> y0{V_LIGHT, es.ray.o, es.n_light, Onb<T>::from_normal(es.n_light), nullptr,
                     es.le / (es.pdf_pos * sel), es.pdf_pos * sel, T(0), light.is_positional_delta(), int32_t(li)};
    vs.push_back(y0);
    if (max_depth == 0) return;
    V3<T> thr = es.le / ((es.pdf_pos * sel) * es.pdf_dir);
    T cos_emit = std::fabs(dot(es.n_light, es.ray.d));
    thr = thr * cos_emit;
    bdpt_subpath_walk(sc, es.ray, thr, es.pdf_dir, max_depth, rr_depth, smp, vs);
}

// mis_weight (:594-770).  EXTENSION: for t == 1 the (s+1, 0) alternative is
// counted when the light is an area light (the reference hard-codes "skip").
template <class T>
T mis_weight(const Scene<T>& sc, const std::vector<PathVertex<T>>& cv, const std::vector<PathVertex<T>>& lv, size_t s,
             size_t t, T pdf_cc, T pdf_cl, uint32_t mode, T beta) {
    if (mode == AR_MIS_UNIFORM) {
        size_t len = s + t, nc = cv.size(), nl = lv.size();
        uint32_t count = 0;
        for (size_t t2 = 0; t2 <= std::min(len, nl); ++t2) {
            size_t s2 = len - t2;
            if (s2 > nc || s2 + t2 < 2) continue;
            if (s2 == 0) continue;
            count++;
        }
        return count == 0 ? T(1) : T(1.0f / float(count));
    }
    if (s + t == 2) return T(1);
    double sum = 0.0;
    const double b = double(float(beta));
    auto pw = [&](double r) { return b == 2.0 ? r * r : std::pow(r, b); };
    auto mis_delta = [](const PathVertex<T>& v) { return v.type == V_SURFACE && v.is_delta; };
    {
        double ri = 1.0;
        if (s >= 1) {
            const auto& v = cv[s - 1];
            ri *= double(pdf_cc) / double(rmax(v.pdf_fwd, T(1e-30f)));
            bool pd = s >= 2 ? mis_delta(cv[s - 2]) : true;
            if (!mis_delta(v) && !pd) sum += pw(std::fabs(ri));
        }
        for (size_t i = s; i-- > 1;) {
            const auto& v = cv[i];
            ri *= double(rmax(v.pdf_rev, T(0))) / double(rmax(v.pdf_fwd, T(1e-30f)));
            bool pd = mis_delta(cv[i - 1]);
            if (!mis_delta(v) && !pd) sum += pw(std::fabs(ri));
        }
    }
    {
        double ri = 1.0;
        if (t >= 1) {
            const auto& v = lv[t - 1];
            ri *= double(pdf_cl) / double(rmax(v.pdf_fwd, T(1e-30f)));
            bool pd;
            if (t >= 2) pd = mis_delta(lv[t - 2]);
            else pd = lv[0].light < 0 || sc.lights[lv[0].light].is_positional_delta();  // EXTENSION
            if (!mis_delta(v) && !pd) sum += pw(std::fabs(ri));
        }
        for (size_t i = t; i-- > 1;) {
            const auto& v = lv[i];
            ri *= double(rmax(v.pdf_rev, T(0))) / double(rmax(v.pdf_fwd, T(1e-30f)));
            bool pd = mis_delta(lv[i - 1]);
            if (!mis_delta(v) && !pd) sum += pw(std::fabs(ri));
        }
    }
    return T(1.0 / (1.0 + sum));
}

// connect_bdpt (:782-1044) for s >= 2, plus the EXTENSION t == 0 case.
template <class T>
bool connect_bdpt(const Scene<T>& sc, const std::vector<PathVertex<T>>& cv, const std::vector<PathVertex<T>>& lv,
                  size_t s, size_t t, uint32_t mode, T beta, V3<T>& out) {
    if (s == 0) return false;
    if (s > cv.size() || t > lv.size()) return false;
    if (t == 0) {  // EXTENSION: the camera subpath ends on an emitter.
        if (s < 2) return false;
        const auto& z = cv[s - 1];
        if (!z.mat || z.mat->emitter < 0 || !sc.ldist.enabled()) return false;
        const Light<T>& lt = sc.lights[z.mat->emitter];
        V3<T> wo = normalize(cv[s - 2].p - z.p);
        if (dot(lt.n, wo) <= T(0)) return false;
        V3<T> c = z.thr * lt.intensity;
        if (max_element(c) <= T(0)) return false;
        T pdf_cc = sc.ldist.pmf_of(uint32_t(z.mat->emitter)) / lt.area;
        T w = mis_weight(sc, cv, lv, s, 0, pdf_cc, T(0), mode, beta);
        out = c * w;
        return true;
    }
    if (s == 1) return false;
    const auto& z = cv[s - 1];
    const auto& y = lv[t - 1];
    if (!z.connectible() || !y.connectible()) return false;
    V3<T> d = y.p - z.p;
    T d2 = length_squared(d);
    if (d2 < T(1e-10f)) return false;
    T dist = std::sqrt(d2);
    V3<T> wi_z = d / dist;
    V3<T> wi_y = -wi_z;
    V3<T> off_z = z.n * T(1e-4f) * signum(dot(wi_z, z.n));
    V3<T> off_y = y.n * T(1e-4f) * signum(dot(wi_y, y.n));
    V3<T> so = z.p + off_z, st = y.p + off_y;
    V3<T> sd = st - so;
    T sdist = length(sd);
    if (sdist < T(1e-6f)) return false;
    Ray<T> sr = Ray<T>::make(so, sd / sdist, T(0), sdist * (T(1) - T(1e-4f)));
    if (sc.occluded(sr)) return false;
    V3<T> wo_z = normalize(cv[s - 2].p - z.p);
    V3<T> wo_zl = z.onb.to_local(wo_z);
    V3<T> f_z = z.mat ? z.mat->eval(z.onb.to_local(wi_z), wo_zl, z.uv) : V3<T>(1, 1, 1);
    if (f_z == V3<T>(0, 0, 0)) return false;
    V3<T> f_y(1, 1, 1);
    if (t != 1 && y.mat) {
        V3<T> wo_y = normalize(lv[t - 2].p - y.p);
        f_y = y.mat->eval(y.onb.to_local(wi_y), y.onb.to_local(wo_y), y.uv);
    }
    if (f_y == V3<T>(0, 0, 0)) return false;
    T g = geometry_term(z.p, z.n, y.p, y.n);
    V3<T> c;
    if (t == 1) {
        const Light<T>& light = sc.lights[y.light];
        if (light.kind == AR_LIGHT_POINT) {
            // :951-967 — the reference re-samples the point light toward z.
            LightSample<T> ls = light.sample(z.p, V2<T>{T(0), T(0)});
            if (!ls.valid) return false;
            V3<T> f_direct = z.mat ? z.mat->eval(z.onb.to_local(ls.wi), wo_zl, z.uv) : V3<T>(1, 1, 1);
            T cos_z = std::fabs(dot(z.n, ls.wi));
            c = ((z.thr * f_direct) * cos_z) * ls.li;
        } else {
            // EXTENSION: connect to the sampled point y0 of the quad light.
            if (dot(y.n, wi_y) <= T(0)) return false;
            c = ((z.thr * f_z) * g) * y.thr;
        }
    } else {
        c = (((z.thr * f_z) * g) * f_y) * y.thr;
    }
    if (max_element(c) <= T(0)) return false;
    T pdf_cc;
    if (t == 1) {
        const Light<T>& light = sc.lights[y.light];
        V3<T> dyz = normalize(z.p - y.p);
        pdf_cc = pdf_sa_to_area(light.pdf_emission_dir(dyz), y.p, z.p, z.n);
    } else if (y.mat) {
        V3<T> wo_y = t >= 2 ? normalize(lv[t - 2].p - y.p) : V3<T>(0, 0, 0);
        V3<T> wiy = normalize(z.p - y.p);
        pdf_cc = pdf_sa_to_area(y.mat->pdf(y.onb.to_local(wiy), y.onb.to_local(wo_y)), y.p, z.p, z.n);
    } else {
        pdf_cc = T(0);
    }
    T pdf_cl;
    if (z.mat) {
        V3<T> wiz = normalize(y.p - z.p);
        pdf_cl = pdf_sa_to_area(z.mat->pdf(z.onb.to_local(wiz), wo_zl), z.p, y.p, y.n);
    } else {
        pdf_cl = T(0);
    }
    T w = mis_weight(sc, cv, lv, s, t, pdf_cc, pdf_cl, mode, beta);
    out = c * w;
    return true;
}

// connect_bdpt_s1 (:1051-1155): light tracing to the camera, splatted.
template <class T>
bool connect_s1(const Scene<T>& sc, const Camera<T>& cam, const std::vector<PathVertex<T>>& cv,
                const std::vector<PathVertex<T>>& lv, size_t t, uint32_t w, uint32_t h, uint32_t mode, T beta,
                V3<T>& out, T& px, T& py) {
    if (t < 2 || lv.size() < t) return false;
    const auto& y = lv[t - 1];
    if (!y.connectible()) return false;
    auto cs = cam.sample_we(y.p, w, h);
    if (!cs.valid) return false;
    V3<T> to_cam = cs.wi;
    T dist = cs.dist;
    V3<T> off = y.n * T(1e-4f) * signum(dot(to_cam, y.n));
    Ray<T> sr = Ray<T>::make(y.p + off, to_cam, T(0), dist * (T(1) - T(1e-4f)));
    if (sc.occluded(sr)) return false;
    V3<T> f_y(1, 1, 1);
    V3<T> wo_y = normalize(lv[t - 2].p - y.p);
    V3<T> wo_yl = y.onb.to_local(wo_y);
    if (y.mat) f_y = y.mat->eval(y.onb.to_local(to_cam), wo_yl, y.uv);
    if (f_y == V3<T>(0, 0, 0)) return false;
    T cos_y = std::fabs(dot(y.n, to_cam));
    T gf = cos_y / (dist * dist);
    V3<T> c = ((y.thr * f_y) * gf) * cs.we;
    if (max_element(c) <= T(0)) return false;
    T pdf_cl = T(0);
    if (y.mat) {
        T pd = y.mat->pdf(y.onb.to_local(to_cam), wo_yl);
        pdf_cl = pdf_sa_to_area(pd, y.p, cam.origin, cv[0].n);
    }
    T wgt = mis_weight(sc, cv, lv, 1, t, T(0), pdf_cl, mode, beta);
    out = c * wgt;
    px = cs.px;
    py = cs.py;
    return true;
}

// BidirectionalPathTracer::render (:1221-1357).
template <class T>
void render_bdpt(const Scene<T>& sc, const Camera<T>& cam, const ar_integrator_cfg& cfg, uint32_t w, uint32_t h,
                 const RenderOpts& o, T* out) {
    uint32_t threads = o.threads ? o.threads : std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::vector<V3<T>>> splats(threads, std::vector<V3<T>>(size_t(w) * h));
    const T beta = T(cfg.mis_beta);
    parallel_rows(h, threads, [&](uint32_t yr, uint32_t tid) {
        std::vector<PathVertex<T>> cv, lv;
        cv.reserve(cfg.max_depth + 1);
        lv.reserve(cfg.max_depth + 1);
        auto& splat = splats[tid];
        for (uint32_t xc = 0; xc < w; ++xc) {
            Sampler smp(o.sampler, xc, yr, w, o.seed);
            V3<T> acc(0, 0, 0);
            for (uint32_t s_ = 0; s_ < cfg.spp; ++s_) {
                smp.start_sample(s_);
                T jx = T(smp.next_1d());
                T jy = T(smp.next_1d());
                T u = (T(float(xc)) + jx) / T(float(w));
                T v = T(1) - (T(float(yr)) + jy) / T(float(h));
                Ray<T> ray = cam.generate_ray({u, v});
                gen_camera_subpath(sc, cam, ray, cfg.max_depth, cfg.rr_depth, smp, cv);
                smp.set_dim(kLightSubpathDim);
                gen_light_subpath(sc, cfg.max_depth, cfg.rr_depth, smp, lv);
                size_t smax = cv.size(), tmax = lv.size();
                size_t limit = size_t(cfg.max_depth) + 2;
                for (size_t t = 0; t <= tmax; ++t) {
                    for (size_t s = 0; s <= smax; ++s) {
                        if (s + t < 2 || s + t > limit || s == 0) continue;
                        V3<T> c;
                        if (s == 1) {
                            T px, py;
                            if (connect_s1(sc, cam, cv, lv, t, w, h, cfg.mis_mode, beta, c, px, py)) {
                                size_t ix = std::min<size_t>(size_t(px), w - 1);
                                size_t iy = std::min<size_t>(size_t(py), h - 1);
                                splat[iy * w + ix] += c;
                            }
                            continue;
                        }
                        if (connect_bdpt(sc, cv, lv, s, t, cfg.mis_mode, beta, c)) acc += c;
                    }
                }
            }
            V3<T> r = acc / T(float(cfg.spp));
            size_t i = (size_t(yr) * w + xc) * 3;
            out[i] = r.x; out[i + 1] = r.y; out[i + 2] = r.z;
        }
    });
    const T inv_spp = T(1.0f / float(cfg.spp));
    for (size_t i = 0; i < size_t(w) * h; ++i) {
        V3<T> sp(0, 0, 0);
        for (auto& sb : splats) sp += sb[i];
        if (!(sp == V3<T>(0, 0, 0))) {
            V3<T> add = sp * inv_spp;
            out[3 * i] += add.x; out[3 * i + 1] += add.y; out[3 * i + 2] += add.z;
        }
    }
}

// ---------------------------------------------------------------------------
// GDPT (gradient_domain_pt.rs)
// ---------------------------------------------------------------------------
// ReplaySampler (:91-161) over the independent sampler (xoshiro mode); in
// counter mode a replay re-reads the same keyed dimensions.
struct ReplaySampler {
    Sampler& inner;
    std::vector<float> tape;
    size_t cursor = 0;
    bool recording = true;
    explicit ReplaySampler(Sampler& s) : inner(s) { tape.reserve(128); }
    void reset_for_new_sample(uint32_t s) {
        tape.clear();
        cursor = 0;
        recording = true;
        inner.start_sample(s);
    }
    void start_replay() {
        recording = false;
        cursor = 0;
        if (inner.kind == SAMPLER_COUNTER) inner.dim = 0;
    }
    float next_1d() {
        if (inner.kind == SAMPLER_COUNTER) return inner.next_1d();
        if (recording) {
            float v = inner.next_1d();
            tape.push_back(v);
            return v;
        }
        float v = cursor < tape.size() ? tape[cursor] : inner.next_1d();
        cursor++;
        return v;
    }
};

// trace_with_gradients (:266-342) -> (base, dx, dy)
template <class T>
void gdpt_trace(const Scene<T>& sc, const Camera<T>& cam, ReplaySampler& rs, uint32_t px, uint32_t py, uint32_t w,
                uint32_t h, uint32_t s, const ar_integrator_cfg& cfg, V3<T>& base, V3<T>& dx, V3<T>& dy) {
    rs.reset_for_new_sample(s);
    T jx = T(rs.next_1d());
    T jy = T(rs.next_1d());
    auto gen = [&](uint32_t x, uint32_t y) {
        T u = (T(float(x)) + jx) / T(float(w));
        T v = T(1) - (T(float(y)) + jy) / T(float(h));
        return cam.generate_ray({u, v});
    };
    base = pt_li(sc, gen(px, py), rs, cfg.max_depth, cfg.rr_depth);
    V3<T> right = base, down = base;
    if (px + 1 < w) {
        rs.start_replay();
        rs.next_1d();
        rs.next_1d();
        right = pt_li(sc, gen(px + 1, py), rs, cfg.max_depth, cfg.rr_depth);
    }
    if (py + 1 < h) {
        rs.start_replay();
        rs.next_1d();
        rs.next_1d();
        down = pt_li(sc, gen(px, py + 1), rs, cfg.max_depth, cfg.rr_depth);
    }
    dx = right - base;
    dy = down - base;
}

// Pass 1 of GradientDomainPathTracer::render (:346-393): primal, dx, dy films.
template <class T>
void render_gdpt_films(const Scene<T>& sc, const Camera<T>& cam, const ar_integrator_cfg& cfg, uint32_t w, uint32_t h,
                       const RenderOpts& o, T* primal, T* gx, T* gy) {
    parallel_rows(h, o.threads, [&](uint32_t y, uint32_t) {
        for (uint32_t x = 0; x < w; ++x) {
            Sampler smp(o.sampler, x, y, w, o.seed);
            ReplaySampler rs(smp);
            V3<T> pa(0, 0, 0), da(0, 0, 0), ya(0, 0, 0);
            for (uint32_t s = 0; s < cfg.spp; ++s) {
                V3<T> b, dx, dy;
                gdpt_trace(sc, cam, rs, x, y, w, h, s, cfg, b, dx, dy);
                pa += b;
                da += dx;
                ya += dy;
            }
            T inv = T(1.0f / float(cfg.spp));
            size_t i = (size_t(y) * w + x) * 3;
            V3<T> a = pa * inv, b = da * inv, c = ya * inv;
            primal[i] = a.x; primal[i + 1] = a.y; primal[i + 2] = a.z;
            gx[i] = b.x; gx[i + 1] = b.y; gx[i + 2] = b.z;
            gy[i] = c.x; gy[i + 1] = c.y; gy[i + 2] = c.z;
        }
    });
}

// screened_poisson_reconstruct (:449-630): RHS = alpha*primal + div G, then
// red-black SOR; result clamped at 0.  Buffers are interleaved RGB (W*H*3).
// neg_div (an extension, off for the reference): RHS = alpha*primal - div G,
// the sign consistent with the stencil for G = I(x+1) - I(x).
template <class T>
void poisson_sor(uint32_t w, uint32_t h, const T* primal, const T* gx, const T* gy, T alpha, uint32_t iters, T omega,
                 T* out, bool neg_div = false) {
    size_t n = size_t(w) * h;
    std::vector<T> img(3 * n), rhs(3 * n);
    for (size_t i = 0; i < 3 * n; ++i) img[i] = primal[i];
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            size_t idx = size_t(y) * w + x;
            for (int c = 0; c < 3; ++c) {
                T div = gx[3 * idx + c];
                if (x > 0) div -= gx[3 * (idx - 1) + c];
                div += gy[3 * idx + c];
                if (y > 0) div -= gy[3 * (idx - w) + c];
                const T a = alpha * primal[3 * idx + c];
                rhs[3 * idx + c] = neg_div ? a - div : a + div;
            }
        }
    for (uint32_t it = 0; it < iters; ++it)
        for (uint32_t parity = 0; parity < 2; ++parity)
            for (uint32_t y = 0; y < h; ++y)
                for (uint32_t x = 0; x < w; ++x) {
                    if (((x + y) & 1u) != parity) continue;
                    size_t idx = size_t(y) * w + x;
                    uint32_t nn = 0;
                    T sum[3] = {T(0), T(0), T(0)};
                    auto addn = [&](size_t j) { for (int c = 0; c < 3; ++c) sum[c] += img[3 * j + c]; nn++; };
                    if (x > 0) addn(idx - 1);
                    if (x + 1 < w) addn(idx + 1);
                    if (y > 0) addn(idx - w);
                    if (y + 1 < h) addn(idx + w);
                    T diag = alpha + T(float(nn));
                    T inv = T(1) / diag;
                    for (int c = 0; c < 3; ++c) {
                        T gs = (rhs[3 * idx + c] + sum[c]) * inv;
                        img[3 * idx + c] = (T(1) - omega) * img[3 * idx + c] + omega * gs;
                    }
                }
    for (size_t i = 0; i < 3 * n; ++i) out[i] = img[i] > T(0) ? img[i] : T(0);
}

// Exact solve of the same screened-Poisson system in FP64 by conjugate
// gradient (the converged reference for the CG solver; not in the crate).
inline void poisson_cg_exact(uint32_t w, uint32_t h, const double* primal, const double* gx, const double* gy,
                             double alpha, double tol, uint32_t max_iters, double* out, double* rel_res) {
    size_t n = size_t(w) * h;
    auto applyA = [&](const std::vector<double>& x, std::vector<double>& y, int c) {
        for (uint32_t yy = 0; yy < h; ++yy)
            for (uint32_t xx = 0; xx < w; ++xx) {
                size_t i = size_t(yy) * w + xx;
                double s = 0;
                int nn = 0;
                if (xx > 0) { s += x[i - 1]; nn++; }
                if (xx + 1 < w) { s += x[i + 1]; nn++; }
                if (yy > 0) { s += x[i - w]; nn++; }
                if (yy + 1 < h) { s += x[i + w]; nn++; }
                y[i] = (alpha + nn) * x[i] - s;
            }
        (void)c;
    };
    double worst = 0;
    for (int c = 0; c < 3; ++c) {
        std::vector<double> b(n), x(n), r(n), p(n), Ap(n);
        for (uint32_t yy = 0; yy < h; ++yy)
            for (uint32_t xx = 0; xx < w; ++xx) {
                size_t i = size_t(yy) * w + xx;
                double div = gx[3 * i + c];
                if (xx > 0) div -= gx[3 * (i - 1) + c];
                div += gy[3 * i + c];
                if (yy > 0) div -= gy[3 * (i - w) + c];
                b[i] = alpha * primal[3 * i + c] + div;
                x[i] = primal[3 * i + c];
            }
        applyA(x, Ap, c);
        double bn = 0, rr = 0;
        for (size_t i = 0; i < n; ++i) { r[i] = b[i] - Ap[i]; p[i] = r[i]; rr += r[i] * r[i]; bn += b[i] * b[i]; }
        bn = std::sqrt(bn);
        if (bn == 0) bn = 1;
        for (uint32_t it = 0; it < max_iters && std::sqrt(rr) / bn > tol; ++it) {
            applyA(p, Ap, c);
            double pAp = 0;
            for (size_t i = 0; i < n; ++i) pAp += p[i] * Ap[i];
            double a = rr / pAp;
            double rr2 = 0;
            for (size_t i = 0; i < n; ++i) { x[i] += a * p[i]; r[i] -= a * Ap[i]; rr2 += r[i] * r[i]; }
            double bb = rr2 / rr;
            rr = rr2;
            for (size_t i = 0; i < n; ++i) p[i] = r[i] + bb * p[i];
        }
        worst = std::max(worst, std::sqrt(rr) / bn);
        for (size_t i = 0; i < n; ++i) out[3 * i + c] = x[i];
    }
    if (rel_res) *rel_res = worst;
}

}  // namespace oracle
