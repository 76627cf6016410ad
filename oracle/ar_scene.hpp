// ORACLE — test infrastructure only (see ar_math.hpp header; parity unpinned).
// Restates the scene layer of agent-ray:
//   Scene / SceneObject / ShadingPoint   src/scene.rs:17-168
//   Onb                                  src/geometry.rs:211-244
//   Bsdf helpers                         src/surfaces.rs:36-83, :109-111
//   Lambertian                           src/surfaces/lambertian.rs:35-64
//   ConductorBsdf + GGX                  src/surfaces/microfacet.rs:14-152
//   DielectricBsdf                       src/surfaces/microfacet.rs:155-307, src/surfaces.rs:86-123
//   ImageTexture                         src/texture.rs:65-151
//   Light / PointLight                   src/lights.rs:14-103, src/lights/point.rs:48-100
//   Uniform/PowerLightDistribution       src/lights.rs:136-235
//   PinholeCamera                        src/cameras.rs:91-248
//   IndependentSampler                   src/sampler.rs:62-95
// plus the quad area-light extension (marked EXTENSION) that the procedural
// scenes need and the reference lacks.
#pragma once
#include <memory>
#include <vector>
#include "../include/agentray.h"
#include "ar_bvh.hpp"

namespace oracle {


// Onb::from_normal (src/geometry.rs:218-232)
template <class T>
struct Onb {
    V3<T> n, t, b;
    static Onb from_normal(V3<T> nin) {
        Onb o;
        o.n = normalize(nin);
        V3<T> a = std::fabs(o.n.x) > T(0.9f) ? V3<T>(0, 1, 0) : V3<T>(1, 0, 0);
        o.b = normalize(cross(o.n, a));
        o.t = cross(o.b, o.n);
        return o;
    }
    V3<T> to_local(V3<T> v) const { return {dot(v, t), dot(v, b), dot(v, n)}; }
    V3<T> to_world(V3<T> v) const { return (t * v.x + b * v.y) + n * v.z; }
};

// ---- BSDFs (local frame, n = +Z) ----
template <class T> inline T cos2_theta(V3<T> v) { return v.z * v.z; }
template <class T> inline T abs_cos_theta(V3<T> v) { return std::fabs(v.z); }
template <class T> inline bool same_hemisphere(V3<T> a, V3<T> b) { return a.z * b.z > T(0); }

// src/surfaces.rs:50-57
template <class T>
inline V3<T> cosine_hemisphere_sample(V2<T> u) {
    T r = std::sqrt(u.x);
    T phi = (T(2) * pi<T>()) * u.y;
    T sp, cp;
    sin_cos(phi, sp, cp);
    T x = r * cp;
    T y = r * sp;
    T z = std::sqrt(rmax((T(1) - x * x) - y * y, T(0)));
    return {x, y, z};
}

// powi(5) as LLVM expands it: t * ((t*t)*(t*t))
template <class T> inline T powi5(T t) { T t2 = t * t; return t * (t2 * t2); }

// src/surfaces.rs:80-83
template <class T>
inline V3<T> fresnel_schlick(T cos_i, V3<T> f0) {
    T c = T(1) - std::fabs(cos_i);
    c = c < T(0) ? T(0) : (c > T(1) ? T(1) : c);
    T t = powi5(c);
    return f0 + (V3<T>(1, 1, 1) - f0) * t;
}

// src/surfaces.rs:109-111: -v + n * 2.0 * v.dot(n)
template <class T> inline V3<T> reflect(V3<T> v, V3<T> n) { return -v + (n * T(2)) * dot(v, n); }

template <class T>
inline T ggx_d(T alpha, V3<T> h) {
    T a2 = alpha * alpha;
    T c2 = cos2_theta(h);
    T denom = c2 * (a2 - T(1)) + T(1);
    return a2 / ((pi<T>() * denom) * denom);
}
template <class T>
inline T ggx_lambda(T alpha, V3<T> v) {
    T c2 = cos2_theta(v);
    if (c2 <= T(0)) return T(INFINITY);
    T a2 = alpha * alpha;
    T tan2 = (T(1) - c2) / c2;
    return (std::sqrt(T(1) + a2 * tan2) - T(1)) * T(0.5f);
}
template <class T>
inline T ggx_g2(T alpha, V3<T> wi, V3<T> wo) { return T(1) / ((T(1) + ggx_lambda(alpha, wi)) + ggx_lambda(alpha, wo)); }
template <class T>
inline V3<T> ggx_sample_wh(T alpha, V3<T> wo, V2<T> u) {
    T a2 = alpha * alpha;
    T c2 = (T(1) - u.x) / ((a2 - T(1)) * u.x + T(1));
    T ch = std::sqrt(rmax(c2, T(0)));
    T sh = std::sqrt(rmax(T(1) - c2, T(0)));
    T phi = (T(2) * pi<T>()) * u.y;
    T sp, cp;
    sin_cos(phi, sp, cp);
    V3<T> h(sh * cp, sh * sp, ch);
    if (h.z * wo.z < T(0)) h = -h;
    return h;
}

// src/surfaces.rs:86-101
template <class T>
inline T fresnel_dielectric(T cos_theta_i, T eta) {
    T ci = cos_theta_i < T(-1) ? T(-1) : (cos_theta_i > T(1) ? T(1) : cos_theta_i);
    if (ci < T(0)) {
        ci = -ci;
        eta = T(1) / eta;
    }
    T sin2_t = (eta * eta) * (T(1) - ci * ci);
    if (sin2_t >= T(1)) return T(1);  // total internal reflection
    T ct = std::sqrt(T(1) - sin2_t);
    T r_par = (eta * ci - ct) / (eta * ci + ct);
    T r_per = (ci - eta * ct) / (ci + eta * ct);
    return T(0.5f) * (r_par * r_par + r_per * r_per);
}

// src/surfaces.rs:115-123: eta * (-v) + n * (eta * cos_i - cos_t), or None on TIR
template <class T>
inline bool refract(V3<T> v, V3<T> n, T eta, V3<T>& out) {
    T cos_i = dot(n, v);
    T sin2_t = (eta * eta) * (T(1) - cos_i * cos_i);
    if (sin2_t >= T(1)) return false;
    T cos_t = std::sqrt(T(1) - sin2_t);
    out = (-v) * eta + n * (eta * cos_i - cos_t);
    return true;
}

// src/texture.rs:139-150 (IEC 61966-2-1), in f32 as the reference decodes
inline float srgb_to_linear(float x) { return x <= 0.04045f ? x / 12.92f : std::pow((x + 0.055f) / 1.055f, 2.4f); }

// ImageTexture (src/texture.rs:65-136): linear texels, bilinear, repeat wrap.
template <class T>
struct Texture {
    std::vector<V3<T>> data;  // row-major, top row first
    uint32_t width = 0, height = 0;

    void load(const ar_texture_desc& d) {
        width = d.width;
        height = d.height;
        data.resize(size_t(width) * height);
        for (size_t i = 0; i < data.size(); ++i)
            data[i] = V3<T>(T(srgb_to_linear(float(d.rgb8[3 * i]) / 255.0f)),
                            T(srgb_to_linear(float(d.rgb8[3 * i + 1]) / 255.0f)),
                            T(srgb_to_linear(float(d.rgb8[3 * i + 2]) / 255.0f)));
    }
    static T wrap01(T x) {  // x.fract().rem_euclid(1.0)
        T f = x - std::trunc(x);
        T r = std::fmod(f, T(1));
        return r < T(0) ? r + T(1) : r;
    }
    V3<T> fetch(int32_t x, int32_t y) const {
        const int32_t w = int32_t(width), h = int32_t(height);
        int32_t xm = x % w, ym = y % h;
        if (xm < 0) xm += w;
        if (ym < 0) ym += h;
        return data[size_t(uint32_t(ym) * width + uint32_t(xm))];
    }
    V3<T> sample(V2<T> uv) const {
        T u = wrap01(uv.x) * T(float(width)) - T(0.5f);
        T v = wrap01(uv.y) * T(float(height)) - T(0.5f);
        T fu = std::floor(u), fv = std::floor(v);
        int32_t x0 = int32_t(fu), y0 = int32_t(fv);
        T tx = u - fu, ty = v - fv;
        V3<T> c00 = fetch(x0, y0), c10 = fetch(x0 + 1, y0), c01 = fetch(x0, y0 + 1), c11 = fetch(x0 + 1, y0 + 1);
        return ((c00 * ((T(1) - tx) * (T(1) - ty)) + c10 * (tx * (T(1) - ty))) + c01 * ((T(1) - tx) * ty)) +
               c11 * (tx * ty);
    }
};

template <class T>
struct BsdfSample {
    V3<T> wi;
    T pdf;
    V3<T> f;
    bool valid;
};

template <class T>
struct Material {
    uint32_t kind;        // ar_material_kind
    int32_t emitter;      // quad light index or -1 (EXTENSION)
    V3<T> albedo, f0;
    T alpha;
    T eta;                // DielectricBsdf interior IOR
    const Texture<T>* tex = nullptr;  // Lambertian ImageTexture albedo, or constant `albedo`

    V3<T> albedo_at(V2<T> uv) const { return tex ? tex->sample(uv) : albedo; }

    // DielectricBsdf (src/surfaces/microfacet.rs:155-307)
    V3<T> refraction_half(V3<T> wi, V3<T> wo, T e) const {
        V3<T> h = -normalize(wo + wi * e);
        if (h.z * wo.z < T(0)) h = -h;
        return h;
    }
    V3<T> dielectric_eval(V3<T> wi, V3<T> wo) const {
        T cos_wo = abs_cos_theta(wo), cos_wi = abs_cos_theta(wi);
        if (cos_wo == T(0) || cos_wi == T(0)) return {};
        T v;
        if (same_hemisphere(wi, wo)) {
            V3<T> h = normalize(wi + wo);
            T f = fresnel_dielectric(std::fabs(dot(wi, h)), eta);
            v = ((f * ggx_d(alpha, h)) * ggx_g2(alpha, wi, wo)) / ((T(4) * cos_wi) * cos_wo);
        } else {
            T e = wo.z > T(0) ? eta : T(1) / eta;
            V3<T> h = refraction_half(wi, wo, e);
            T woh = dot(wo, h), wih = dot(wi, h);
            if (woh == T(0) || wih == T(0)) return {};
            T f = T(1) - fresnel_dielectric(std::fabs(wih), eta);
            T d = ggx_d(alpha, h), g = ggx_g2(alpha, wi, wo);
            T sum = woh + e * wih;
            T denom = sum * sum;  // powi(2)
            if (denom == T(0)) return {};
            T eta2 = e * e;
            v = ((((f * d) * g) * eta2) * std::fabs(woh)) * std::fabs(wih) / ((cos_wi * cos_wo) * denom);
        }
        return V3<T>(v, v, v);
    }
    T dielectric_pdf(V3<T> wi, V3<T> wo) const {
        if (abs_cos_theta(wo) == T(0) || abs_cos_theta(wi) == T(0)) return T(0);
        if (same_hemisphere(wi, wo)) {
            V3<T> h = normalize(wi + wo);
            T whwi = std::fabs(dot(wi, h));
            if (whwi == T(0)) return T(0);
            T f = fresnel_dielectric(std::fabs(dot(wo, h)), eta);
            return ((f * ggx_d(alpha, h)) * abs_cos_theta(h)) / (T(4) * whwi);
        }
        T e = wo.z > T(0) ? eta : T(1) / eta;
        V3<T> h = refraction_half(wi, wo, e);
        T woh = dot(wo, h), wih = dot(wi, h);
        if (woh == T(0) || wih == T(0)) return T(0);
        T sum = woh + e * wih;
        T denom = sum * sum;
        if (denom == T(0)) return T(0);
        T f = T(1) - fresnel_dielectric(std::fabs(woh), eta);
        return (((((f * ggx_d(alpha, h)) * abs_cos_theta(h)) * e) * e) * std::fabs(wih)) / denom;
    }

    V3<T> eval(V3<T> wi, V3<T> wo, V2<T> uv) const {
        if (kind == AR_MATERIAL_DIELECTRIC) return dielectric_eval(wi, wo);
        if (kind == AR_MATERIAL_LAMBERTIAN) {
            if (!same_hemisphere(wi, wo)) return {};
            return albedo_at(uv) * frac_1_pi<T>();
        }
        if (!same_hemisphere(wi, wo)) return {};
        T ci = abs_cos_theta(wi), co = abs_cos_theta(wo);
        if (ci == T(0) || co == T(0)) return {};
        V3<T> h = normalize(wi + wo);
        V3<T> f = fresnel_schlick(std::fabs(dot(wi, h)), f0);
        T d = ggx_d(alpha, h);
        T g = ggx_g2(alpha, wi, wo);
        return f * (d * g / ((T(4) * ci) * co));
    }
    T pdf(V3<T> wi, V3<T> wo) const {
        if (kind == AR_MATERIAL_DIELECTRIC) return dielectric_pdf(wi, wo);
        if (kind == AR_MATERIAL_LAMBERTIAN) {
            if (!same_hemisphere(wi, wo)) return T(0);
            return abs_cos_theta(wi) * frac_1_pi<T>();
        }
        if (!same_hemisphere(wi, wo)) return T(0);
        V3<T> h = normalize(wi + wo);
        T whwi = std::fabs(dot(wi, h));
        if (whwi == T(0)) return T(0);
        return ggx_d(alpha, h) * abs_cos_theta(h) / (T(4) * whwi);
    }
    BsdfSample<T> sample(V3<T> wo, V2<T> uv, T u_sel, V2<T> u) const {
        BsdfSample<T> s{};
        s.valid = false;
        if (kind == AR_MATERIAL_LAMBERTIAN) {
            V3<T> wi = cosine_hemisphere_sample(u);
            if (wo.z < T(0)) wi.z = -wi.z;
            T pdf = abs_cos_theta(wi) * frac_1_pi<T>();
            if (pdf == T(0)) return s;
            s = {wi, pdf, albedo_at(uv) * frac_1_pi<T>(), true};
            return s;
        }
        if (wo.z == T(0)) return s;
        V3<T> h = ggx_sample_wh(alpha, wo, u);
        if (kind == AR_MATERIAL_DIELECTRIC && !(u_sel < fresnel_dielectric(std::fabs(dot(wo, h)), eta))) {
            // refraction lobe (microfacet.rs:248-264)
            T e = wo.z > T(0) ? T(1) / eta : eta;
            V3<T> wi;
            if (!refract(wo, h, e, wi)) return s;
            if (same_hemisphere(wi, wo)) return s;
            T p = pdf(wi, wo);
            if (p == T(0)) return s;
            s = {wi, p, eval(wi, wo, uv), true};
            return s;
        }
        V3<T> wi = reflect(wo, h);
        if (!same_hemisphere(wi, wo)) return s;
        T p = pdf(wi, wo);
        if (p == T(0)) return s;
        s = {wi, p, eval(wi, wo, uv), true};
        return s;
    }
};

// ---- lights ----
template <class T>
struct LightSample {
    V3<T> wi;
    T dist;
    V3<T> li;
    T pdf;
    bool valid;
};
template <class T>
struct EmissionSample {
    Ray<T> ray;
    V3<T> le;
    T pdf_pos, pdf_dir;
    V3<T> n_light;
    bool valid;
};

// src/lights/point.rs:26-32
template <class T>
inline V3<T> uniform_sphere_sample(V2<T> u) {
    T ct = T(1) - T(2) * u.x;
    T st = std::sqrt(rmax(T(1) - ct * ct, T(0)));
    T phi = (T(2) * pi<T>()) * u.y;
    T sp, cp;
    sin_cos(phi, sp, cp);
    return {st * cp, st * sp, ct};
}

template <class T>
struct Light {
    uint32_t kind;
    V3<T> pos, intensity;   // point: position/intensity; quad: corner/radiance
    V3<T> e1, e2, n;        // quad only
    T area;

    bool is_delta() const { return kind == AR_LIGHT_POINT; }
    bool is_positional_delta() const { return kind == AR_LIGHT_POINT; }
    V3<T> power() const {
        if (kind == AR_LIGHT_POINT) return intensity * (T(4) * pi<T>());
        return intensity * (area * pi<T>());  // EXTENSION: Lambertian one-sided emitter
    }
    LightSample<T> sample(V3<T> ref, V2<T> u) const {
        LightSample<T> ls{};
        ls.valid = false;
        if (kind == AR_LIGHT_POINT) {  // point.rs:49-61
            V3<T> off = pos - ref;
            T d2 = length_squared(off);
            T d = std::sqrt(d2);
            if (d < T(1e-6f)) return ls;
            ls = {off / d, d, intensity / d2, T(1), true};
            return ls;
        }
        // EXTENSION: sample the quad uniformly by area, solid-angle pdf.
        V3<T> q = (pos + e1 * u.x) + e2 * u.y;
        V3<T> off = q - ref;
        T d2 = length_squared(off);
        T d = std::sqrt(d2);
        if (d < T(1e-6f)) return ls;
        V3<T> wi = off / d;
        T cos_l = -dot(n, wi);
        if (cos_l <= T(0)) return ls;
        ls = {wi, d, intensity, d2 / (cos_l * area), true};
        return ls;
    }
    EmissionSample<T> sample_emission(V2<T> upos, V2<T> udir) const {
        EmissionSample<T> es{};
        es.valid = false;
        if (kind == AR_LIGHT_POINT) {  // point.rs:71-86
            V3<T> dir = uniform_sphere_sample(udir);
            es.ray = Ray<T>::make(pos, dir, T(1e-4f), ray_unbounded<T>());
            es.le = intensity;
            es.pdf_pos = T(1);
            es.pdf_dir = T(1) / (T(4) * pi<T>());
            es.n_light = dir;
            es.valid = true;
            return es;
        }
        // EXTENSION: uniform point on the quad, cosine-weighted direction about n.
        V3<T> q = (pos + e1 * upos.x) + e2 * upos.y;
        V3<T> local = cosine_hemisphere_sample(udir);
        Onb<T> f = Onb<T>::from_normal(n);
        V3<T> dir = f.to_world(local);
        es.ray = Ray<T>::make(q, dir, T(1e-4f), ray_unbounded<T>());
        es.le = intensity;
        es.pdf_pos = T(1) / area;
        es.pdf_dir = local.z * frac_1_pi<T>();
        es.n_light = n;
        es.valid = es.pdf_dir > T(0);
        return es;
    }
    T pdf_emission_dir(V3<T> dir) const {
        if (kind == AR_LIGHT_POINT) return T(1) / (T(4) * pi<T>());
        T c = dot(n, dir);
        return c > T(0) ? c * frac_1_pi<T>() : T(0);
    }
};

template <class T>
struct LightDist {
    uint32_t kind = AR_LIGHT_DIST_NONE;
    std::vector<float> cdf, pmf;  // f32 as in the reference
    uint32_t n = 0;
    void build(uint32_t k, const std::vector<Light<T>>& lights) {
        kind = k;
        n = uint32_t(lights.size());
        if (kind == AR_LIGHT_DIST_POWER) {
            std::vector<float> w(n);
            for (uint32_t i = 0; i < n; ++i) {
                V3<float> p(lights[i].power());
                w[i] = rmax((0.2126f * p.x + 0.7152f * p.y) + 0.0722f * p.z, 0.0f);
            }
            float total = 0.f;
            for (float x : w) total += x;
            pmf.resize(n);
            cdf.resize(n);
            if (total == 0.0f) {
                float u = 1.0f / float(n);
                for (uint32_t i = 0; i < n; ++i) { pmf[i] = u; cdf[i] = float(i + 1) * u; }
            } else {
                float acc = 0.f;
                for (uint32_t i = 0; i < n; ++i) { pmf[i] = w[i] / total; acc += pmf[i]; cdf[i] = acc; }
                cdf[n - 1] = 1.0f;
            }
        }
    }
    bool enabled() const { return kind != AR_LIGHT_DIST_NONE && n > 0; }
    void sample_index(T u, uint32_t& idx, T& p) const {
        if (kind == AR_LIGHT_DIST_UNIFORM) {
            float uf = float(u);
            float s = uf * float(n);
            uint32_t i = s >= 0.f ? uint32_t(s) : 0u;  // `as usize` saturates
            idx = std::min(i, n - 1);
            p = T(1.0f / float(n));
            return;
        }
        // partition_point(|c| c < u)
        uint32_t lo = 0, hi = n;
        while (lo < hi) {
            uint32_t mid = (lo + hi) / 2;
            if (T(cdf[mid]) < u) lo = mid + 1; else hi = mid;
        }
        idx = std::min(lo, n - 1);
        p = T(pmf[idx]);
    }
    T pmf_of(uint32_t i) const {
        if (kind == AR_LIGHT_DIST_UNIFORM) return T(1.0f / float(n));
        return T(pmf[i]);
    }
};

// ---- camera (src/cameras.rs:91-248) ----
template <class T>
struct Camera {
    V3<T> origin, lower_left, horizontal, vertical, forward;
    T area;
    static Camera from_lookat(const ar_camera_desc& d) {
        // Set up in f32 exactly as the reference does, then widened.
        V3<float> lf(d.lookfrom[0], d.lookfrom[1], d.lookfrom[2]);
        V3<float> la(d.lookat[0], d.lookat[1], d.lookat[2]);
        V3<float> up(d.vup[0], d.vup[1], d.vup[2]);
        const float rads_per_deg = 3.14159265358979323846f / 180.0f;
        float theta = d.vfov_deg * rads_per_deg;
        float h = std::tan(theta / 2.0f);
        float vh = 2.0f * h;
        float vw = d.aspect * vh;
        V3<float> w = normalize(lf - la);
        V3<float> u = normalize(cross(up, w));
        V3<float> v = cross(w, u);
        V3<float> hor = vw * u;
        V3<float> ver = vh * v;
        V3<float> ll = ((lf - hor / 2.0f) - ver / 2.0f) - w;
        Camera c;
        c.origin = V3<T>(lf);
        c.lower_left = V3<T>(ll);
        c.horizontal = V3<T>(hor);
        c.vertical = V3<T>(ver);
        c.forward = V3<T>(-w);
        c.area = T(vw * vh);
        return c;
    }
    Ray<T> generate_ray(V2<T> uv) const {
        V3<T> dir = ((lower_left + uv.x * horizontal) + uv.y * vertical) - origin;
        return Ray<T>::make(origin, dir, T(0.001f), ray_unbounded<T>());
    }
    T pdf_we(const Ray<T>& r) const {
        T c = dot(r.d, forward);
        if (c <= T(0)) return T(0);
        return T(1) / (((area * c) * c) * c);
    }
    struct WeSample { T px, py; V3<T> wi; T dist, we, pdf; bool valid; };
    WeSample sample_we(V3<T> p, uint32_t width, uint32_t height) const {
        WeSample s{};
        s.valid = false;
        V3<T> to_cam = origin - p;
        T d2 = length_squared(to_cam);
        T d = std::sqrt(d2);
        if (d < T(1e-6f)) return s;
        V3<T> wi = to_cam / d;
        V3<T> dir = -wi;
        T ct = dot(dir, forward);
        if (ct <= T(1e-6f)) return s;
        V3<T> right = normalize(horizontal), up = normalize(vertical);
        T vw = length(horizontal), vh = length(vertical);
        V3<T> ds = dir / ct;
        T u = dot(ds, right) / vw + T(0.5f);
        T v = dot(ds, up) / vh + T(0.5f);
        if (u < T(0) || u > T(1) || v < T(0) || v > T(1)) return s;
        T px = u * T(width);
        T py = (T(1) - v) * T(height);
        if (px < T(0) || px >= T(width) || py < T(0) || py >= T(height)) return s;
        T c2 = ct * ct, c4 = c2 * c2, c3 = c2 * ct;
        s = {px, py, wi, d, T(1) / (area * c4), d2 / (area * c3), true};
        return s;
    }
};

// ---- samplers ----
// Xoshiro256++ seeded by SplitMix64: the published algorithms behind rand 0.10
// SmallRng::seed_from_u64 on 64-bit targets, and f32 = (next_u32 >> 8) * 2^-24.
// UNPINNED: rand's source is not under the reference tree; this is a best-
// effort restatement of the published generator.
struct Xoshiro256pp {
    uint64_t s[4];
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    explicit Xoshiro256pp(uint64_t state) {
        const uint64_t phi = 0x9e3779b97f4a7c15ull;
        for (int i = 0; i < 4; ++i) {
            state += phi;
            uint64_t z = state;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            s[i] = z ^ (z >> 31);
        }
    }
    uint64_t next_u64() {
        uint64_t r = rotl(s[0] + s[3], 23) + s[0];
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    float next_f32() { return float(uint32_t(next_u64() >> 32) >> 8) * (1.0f / 16777216.0f); }
};

// SplitMix64 finalizer (Steele, Lea & Flood 2014) — the mixing function of the
// counter-based sampler shared with the GPU kernels.
inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
// Counter-based sampler: u(dim) depends only on (seed, pixel, sample, dim).
inline uint64_t counter_key(uint64_t seed, uint32_t pixel, uint32_t sample) {
    return mix64(seed ^ mix64((uint64_t(pixel) << 32) | uint64_t(sample)));
}
inline float counter_u01(uint64_t key, uint32_t dim) {
    uint64_t z = mix64(key + uint64_t(dim + 1) * 0x9e3779b97f4a7c15ull);
    return float(uint32_t(z >> 40)) * (1.0f / 16777216.0f);
}

enum SamplerKind : uint32_t { SAMPLER_XOSHIRO = 0, SAMPLER_COUNTER = 1 };

// Sampler trait (src/sampler.rs:27-51).  Xoshiro mode reproduces the
// reference IndependentSampler: one stream per pixel across all samples.
// Counter mode keys each (pixel, sample) and indexes dimensions explicitly.
struct Sampler {
    uint32_t kind;
    Xoshiro256pp rng;
    uint64_t seed;
    uint32_t pixel = 0, sample = 0, dim = 0;
    uint64_t key = 0;
    Sampler(uint32_t k, uint32_t px, uint32_t py, uint32_t width, uint64_t sd)
        : kind(k), rng(((uint64_t(py) * 2654435761ull) ^ (uint64_t(px) * 805459861ull)) ^ sd), seed(sd) {
        pixel = py * width + px;
    }
    // start_next_sample: a no-op for the independent sampler.
    void start_sample(uint32_t s) {
        sample = s;
        dim = 0;
        key = counter_key(seed, pixel, sample);
    }
    void set_dim(uint32_t d) {
        if (kind == SAMPLER_COUNTER) dim = d;
    }
    float next_1d() {
        if (kind == SAMPLER_XOSHIRO) return rng.next_f32();
        return counter_u01(key, dim++);
    }
};

// Dimension layout of the counter sampler (shared with the GPU kernels).
constexpr uint32_t kLightSubpathDim = 4096;

// ---- the scene (src/scene.rs:17-168) ----
template <class T>
struct Object {
    uint32_t mesh;
    Mat4<float> xf, inv;
    Mat4<T> invT;
    Mat3<T> nmat;
    std::vector<uint32_t> mats;
    AabbF world;
};

template <class T>
struct ShadingPoint {
    V3<T> p, n;
    V2<T> uv;  // tex_uv (src/scene.rs:54-66)
    Onb<T> onb;
    const Material<T>* mat;
    uint32_t inst, prim;
    T t;
};

template <class T>
struct Scene {
    std::vector<MeshBlas<T>> meshes;
    std::vector<Object<T>> objects;
    std::vector<Material<T>> materials;
    std::vector<Light<T>> lights;
    std::vector<Texture<T>> textures;
    LightDist<T> ldist;
    BuildResult tlas;

    bool load(const ar_scene_desc& d) {
        meshes.resize(d.num_meshes);
        for (uint32_t m = 0; m < d.num_meshes; ++m) {
            const ar_mesh_desc& md = d.meshes[m];
            auto& mb = meshes[m];
            mb.pos.resize(md.num_vertices);
            for (uint32_t i = 0; i < md.num_vertices; ++i)
                mb.pos[i] = V3<T>(T(md.positions[3 * i]), T(md.positions[3 * i + 1]), T(md.positions[3 * i + 2]));
            if (md.normals) {
                mb.nrm.resize(md.num_vertices);
                for (uint32_t i = 0; i < md.num_vertices; ++i)
                    mb.nrm[i] = V3<T>(T(md.normals[3 * i]), T(md.normals[3 * i + 1]), T(md.normals[3 * i + 2]));
            }
            if (md.tex_coords) {
                mb.uv.resize(md.num_vertices);
                for (uint32_t i = 0; i < md.num_vertices; ++i)
                    mb.uv[i] = V2<T>{T(md.tex_coords[2 * i]), T(md.tex_coords[2 * i + 1])};
            }
            mb.idx.assign(md.indices, md.indices + 3 * size_t(md.num_triangles));
            if (md.num_material_slots == 0 || !md.material_slots) mb.slots = {0u};
            else mb.slots.assign(md.material_slots, md.material_slots + md.num_material_slots);
            mb.build();
        }
        objects.resize(d.num_objects);
        for (uint32_t o = 0; o < d.num_objects; ++o) {
            const ar_object_desc& od = d.objects[o];
            auto& ob = objects[o];
            ob.mesh = od.mesh;
            float inv[16];
            if (od.has_inverse) std::copy(od.inv_transform, od.inv_transform + 16, inv);
            else invert4x4_colmajor(od.transform, inv);
            for (int c = 0; c < 4; ++c) {
                ob.xf.c[c] = V3<float>(od.transform[4 * c], od.transform[4 * c + 1], od.transform[4 * c + 2]);
                ob.inv.c[c] = V3<float>(inv[4 * c], inv[4 * c + 1], inv[4 * c + 2]);
                ob.invT.c[c] = V3<T>(ob.inv.c[c]);
            }
            Mat4<T> xfT;
            for (int c = 0; c < 4; ++c) xfT.c[c] = V3<T>(ob.xf.c[c]);
            ob.nmat = normal_matrix(xfT);
            ob.mats.assign(od.materials, od.materials + od.num_materials);
            ob.world = transform_aabb(meshes[ob.mesh].overall, ob.xf);
        }
        textures.resize(d.num_textures);
        for (uint32_t i = 0; i < d.num_textures; ++i) textures[i].load(d.textures[i]);
        materials.resize(d.num_materials);
        for (uint32_t i = 0; i < d.num_materials; ++i) {
            const auto& m = d.materials[i];
            auto& mm = materials[i];
            mm.kind = m.kind;
            mm.emitter = m.emitter_light;
            mm.albedo = V3<T>(T(m.albedo[0]), T(m.albedo[1]), T(m.albedo[2]));
            mm.f0 = V3<T>(T(m.f0[0]), T(m.f0[1]), T(m.f0[2]));
            float a = m.roughness < 1e-3f ? 1e-3f : (m.roughness > 1.0f ? 1.0f : m.roughness);
            mm.alpha = T(a);
            mm.eta = T(m.eta);
            mm.tex = m.albedo_texture >= 0 && uint32_t(m.albedo_texture) < textures.size()
                         ? &textures[m.albedo_texture] : nullptr;
        }
        lights.resize(d.num_lights);
        for (uint32_t i = 0; i < d.num_lights; ++i) {
            const auto& l = d.lights[i];
            auto& ll = lights[i];
            ll.kind = l.kind;
            ll.pos = V3<T>(T(l.position[0]), T(l.position[1]), T(l.position[2]));
            ll.intensity = V3<T>(T(l.intensity[0]), T(l.intensity[1]), T(l.intensity[2]));
            ll.e1 = V3<T>(T(l.edge1[0]), T(l.edge1[1]), T(l.edge1[2]));
            ll.e2 = V3<T>(T(l.edge2[0]), T(l.edge2[1]), T(l.edge2[2]));
            V3<T> c = cross(ll.e1, ll.e2);
            ll.area = length(c);
            ll.n = ll.kind == AR_LIGHT_QUAD ? normalize(c) : V3<T>();
        }
        ldist.build(d.light_distribution, lights);
        std::vector<AabbF> boxes(objects.size());
        for (size_t i = 0; i < objects.size(); ++i) boxes[i] = objects[i].world;
        tlas = build_bvh(boxes);
        return true;
    }

    // TLAS::intersect (src/accel/bvh.rs:413-447)
    Hit<T> tlas_intersect(const Ray<T>& ray, TraversalStats* st) const {
        return traverse(tlas.nodes, tlas.prims, ray, [&](uint32_t inst, T tmax) {
            Hit<T> none{};
            none.valid = false;
            if (st) st->instances++;
            const Object<T>& ob = objects[inst];
            V3<T> lo = ob.invT.transform_point(ray.o);
            V3<T> ldu = ob.invT.transform_vector(ray.d);
            T ds = length(ldu);
            if (ds < T(FLT_EPSILON)) return none;
            Ray<T> lr = Ray<T>::make(lo, ldu, ray.tmin * ds, tmax * ds);
            Hit<T> h = meshes[ob.mesh].intersect(lr, st);
            if (!h.valid) return none;
            h.t = h.t / ds;
            h.inst = inst;
            return h;
        }, st);
    }

    // Scene::intersect (src/scene.rs:142-162)
    bool intersect(const Ray<T>& ray, ShadingPoint<T>& sp) const {
        Hit<T> h = tlas_intersect(ray, nullptr);
        if (!h.valid) return false;
        const Object<T>& ob = objects[h.inst];
        const MeshBlas<T>& m = meshes[ob.mesh];
        sp.p = ray.at(h.t);
        V3<T> nobj = h.n;
        if (!m.nrm.empty()) {
            uint32_t i0 = m.idx[3 * h.prim], i1 = m.idx[3 * h.prim + 1], i2 = m.idx[3 * h.prim + 2];
            T w = (T(1) - h.u) - h.v;
            nobj = normalize((m.nrm[i0] * w + m.nrm[i1] * h.u) + m.nrm[i2] * h.v);
        }
        V3<T> n = normalize(ob.nmat.mul(nobj));
        V3<T> wo = -ray.d;
        if (dot(n, wo) < T(0)) n = -n;
        sp.n = n;
        sp.onb = Onb<T>::from_normal(n);
        if (!m.uv.empty()) {  // tex_coords[i0] * w + tex_coords[i1] * u + tex_coords[i2] * v
            uint32_t i0 = m.idx[3 * h.prim], i1 = m.idx[3 * h.prim + 1], i2 = m.idx[3 * h.prim + 2];
            T w = (T(1) - h.u) - h.v;
            sp.uv = V2<T>{(m.uv[i0].x * w + m.uv[i1].x * h.u) + m.uv[i2].x * h.v,
                          (m.uv[i0].y * w + m.uv[i1].y * h.u) + m.uv[i2].y * h.v};
        } else {
            sp.uv = V2<T>{h.u, h.v};
        }
        uint32_t slot = m.slots.size() == 1 ? m.slots[0] : m.slots[h.prim];
        size_t k = std::min<size_t>(slot, ob.mats.size() - 1);
        sp.mat = &materials[ob.mats[k]];
        sp.inst = h.inst;
        sp.prim = h.prim;
        sp.t = h.t;
        return true;
    }
    // Scene::occluded (src/scene.rs:166-168): closest hit, then is_some().
    bool occluded(const Ray<T>& ray) const { return tlas_intersect(ray, nullptr).valid; }
};

}  // namespace oracle
