// Device shading layer: shading points, BSDFs, lights and the camera.
// Mirrors the reference operation order; translation units that include this
// are compiled with -fmad=false so no multiply is fused into an add (the
// reference Rust/glam code rounds each operation separately).  Sines and
// cosines of sampling angles come from ar_trig.h, which the CPU oracle uses
// too, so both sides draw bit-identical directions.
//   Scene::intersect shading     src/scene.rs:142-162, :55-87
//   Onb                          src/geometry.rs:218-244
//   Lambertian                   src/surfaces/lambertian.rs:35-64
//   ConductorBsdf (GGX)          src/surfaces/microfacet.rs:14-152
//   DielectricBsdf (GGX glass)   src/surfaces/microfacet.rs:155-307, src/surfaces.rs:86-123
//   ImageTexture                 src/texture.rs:65-151
//   PointLight                   src/lights/point.rs:48-100
//   Uniform/PowerLightDistribution src/lights.rs:136-235
//   PinholeCamera                src/cameras.rs:146-248
// Quad lights are the area-light extension shared with the oracle.
#pragma once
#include "ar_device.cuh"
#include "ar_render.hpp"
#include "ar_trig.h"

namespace ar {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;

struct Onb {
    f3 n, t, b;
};
__device__ __forceinline__ Onb onb_from_normal(f3 nin) {
    Onb o;
    o.n = normalize(nin);
    f3 a = fabsf(o.n.x) > 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
    o.b = normalize(cross(o.n, a));
    o.t = cross(o.b, o.n);
    return o;
}
__device__ __forceinline__ f3 to_local(const Onb& o, f3 v) { return mk(dot(v, o.t), dot(v, o.b), dot(v, o.n)); }
__device__ __forceinline__ f3 to_world(const Onb& o, f3 v) { return (o.t * v.x + o.b * v.y) + o.n * v.z; }
__device__ __forceinline__ float signum(float a) { return copysignf(1.0f, a); }

struct Shade {
    f3 p, n;
    Onb onb;
    uint32_t mat;
    uint32_t prim;
    float tu, tv;  // tex_uv (SceneObject::tex_uv, src/scene.rs:54-66)
};

// Scene::intersect post-processing: world shading normal (interpolated vertex
// normal or geometric normal through the normal matrix), face-forwarded
// toward the incoming ray, ONB and material.
__device__ __forceinline__ Shade make_shade(const DevScene& sc, f3 ro, f3 rd, float t, float u, float v, uint32_t slot,
                                           uint32_t inst) {
    Shade s;
    const TriRecord tr = load_tri(sc.tris, slot);
    const ObjectRecord& ob = sc.objects[inst];
    const MeshRecord mr = sc.meshes[ob.mesh];
    s.prim = tr.prim;
    f3 nobj = normalize(cross(mk(tr.e1x, tr.e1y, tr.e1z), mk(tr.e2x, tr.e2y, tr.e2z)));
    if (mr.nrm_offset != kInvalid) {
        const uint32_t* ix = sc.indices + mr.idx_offset + 3 * tr.prim;
        const float* nb = sc.normals + 3 * size_t(mr.nrm_offset);
        f3 n0 = ld3(nb + 3 * size_t(ix[0])), n1 = ld3(nb + 3 * size_t(ix[1])), n2 = ld3(nb + 3 * size_t(ix[2]));
        float w = (1.0f - u) - v;
        nobj = normalize((n0 * w + n1 * u) + n2 * v);
    }
    f3 c0 = mk(ob.nmat[0], ob.nmat[1], ob.nmat[2]), c1 = mk(ob.nmat[3], ob.nmat[4], ob.nmat[5]),
       c2 = mk(ob.nmat[6], ob.nmat[7], ob.nmat[8]);
    f3 n = normalize((c0 * nobj.x + c1 * nobj.y) + c2 * nobj.z);
    f3 wo = -rd;
    if (dot(n, wo) < 0.f) n = -n;
    s.n = n;
    s.onb = onb_from_normal(n);
    s.p = ro + rd * t;
    if (mr.uv_offset != kInvalid) {  // tex_coords[i0] * w + tex_coords[i1] * u + tex_coords[i2] * v
        const uint32_t* ix = sc.indices + mr.idx_offset + 3 * tr.prim;
        const float* tc = sc.texcoords + 2 * size_t(mr.uv_offset);
        const float w = (1.0f - u) - v;
        s.tu = (tc[2 * ix[0]] * w + tc[2 * ix[1]] * u) + tc[2 * ix[2]] * v;
        s.tv = (tc[2 * ix[0] + 1] * w + tc[2 * ix[1] + 1] * u) + tc[2 * ix[2] + 1] * v;
    } else {
        s.tu = u;
        s.tv = v;
    }
    const uint32_t si = mr.num_slots == 1 ? sc.material_slots[mr.slot_offset]
                                          : sc.material_slots[mr.slot_offset + tr.prim];
    const uint32_t k = min(si, ob.num_mats - 1);
    s.mat = sc.material_table[ob.mat_offset + k];
    return s;
}

// ---- BSDF (local frame, n = +Z) ----
__device__ __forceinline__ bool same_hemi(f3 a, f3 b) { return a.z * b.z > 0.f; }
__device__ __forceinline__ f3 cosine_hemisphere(float ux, float uy) {
    float r = sqrtf(ux);
    float phi = (2.0f * kPi) * uy;
    float sp, cp;
    ar_trig::sincos(phi, &sp, &cp);
    float x = r * cp, y = r * sp;
    float z = sqrtf(fmaxf((1.0f - x * x) - y * y, 0.0f));
    return mk(x, y, z);
}
__device__ __forceinline__ float ggx_d(float a, f3 h) {
    float a2 = a * a;
    float c2 = h.z * h.z;
    float den = c2 * (a2 - 1.0f) + 1.0f;
    return a2 / ((kPi * den) * den);
}
__device__ __forceinline__ float ggx_lambda(float a, f3 v) {
    float c2 = v.z * v.z;
    if (c2 <= 0.f) return INFINITY;
    float a2 = a * a;
    float tan2 = (1.0f - c2) / c2;
    return (sqrtf(1.0f + a2 * tan2) - 1.0f) * 0.5f;
}
__device__ __forceinline__ f3 fresnel_schlick(float ci, const float* f0) {
    float c = fminf(fmaxf(1.0f - fabsf(ci), 0.0f), 1.0f);
    float c2 = c * c;
    float t = c * (c2 * c2);
    return mk(f0[0] + (1.0f - f0[0]) * t, f0[1] + (1.0f - f0[1]) * t, f0[2] + (1.0f - f0[2]) * t);
}

struct MatView {
    uint32_t kind;
    int32_t emitter;
    float albedo[3], f0[3];
    float alpha, eta;
};
// ImageTexture::sample (src/texture.rs:97-136): repeat wrap, bilinear.
__device__ __forceinline__ float wrap01(float x) {  // x.fract().rem_euclid(1.0)
    const float f = x - truncf(x);
    const float r = fmodf(f, 1.0f);
    return r < 0.f ? r + 1.0f : r;
}
__device__ __forceinline__ f3 texel(const DevScene& sc, const TextureRecord& t, int32_t x, int32_t y) {
    int32_t xm = x % int32_t(t.width), ym = y % int32_t(t.height);
    if (xm < 0) xm += int32_t(t.width);
    if (ym < 0) ym += int32_t(t.height);
    const float4 c = __ldg(sc.texels + t.offset + uint32_t(ym) * t.width + uint32_t(xm));
    return mk(c.x, c.y, c.z);
}
__device__ __forceinline__ f3 texture_sample(const DevScene& sc, uint32_t ti, float tu, float tv) {
    const TextureRecord t = sc.textures[ti];
    const float u = wrap01(tu) * float(t.width) - 0.5f;
    const float v = wrap01(tv) * float(t.height) - 0.5f;
    const float fu = floorf(u), fv = floorf(v);
    const int32_t x0 = int32_t(fu), y0 = int32_t(fv);
    const float tx = u - fu, ty = v - fv;
    const f3 c00 = texel(sc, t, x0, y0), c10 = texel(sc, t, x0 + 1, y0), c01 = texel(sc, t, x0, y0 + 1),
             c11 = texel(sc, t, x0 + 1, y0 + 1);
    return ((c00 * ((1.0f - tx) * (1.0f - ty)) + c10 * (tx * (1.0f - ty))) + c01 * ((1.0f - tx) * ty)) +
           c11 * (tx * ty);
}

__device__ __forceinline__ MatView load_mat(const DevScene& sc, uint32_t m) {
    const MaterialRecord& r = sc.materials[m];
    MatView v;
    v.kind = r.kind;
    v.emitter = r.emitter;
    for (int k = 0; k < 3; ++k) { v.albedo[k] = r.albedo[k]; v.f0[k] = r.f0[k]; }
    v.alpha = r.alpha;
    v.eta = r.eta;
    return v;
}

// The material at a shading point: a textured Lambertian's albedo is its
// ImageTexture sampled at tex_uv (Lambertian::eval, lambertian.rs:35-41).
__device__ __forceinline__ MatView load_mat_at(const DevScene& sc, uint32_t m, float tu, float tv) {
    MatView v = load_mat(sc, m);
    const int32_t ti = sc.materials[m].tex;
    if (ti >= 0) {
        const f3 a = texture_sample(sc, uint32_t(ti), tu, tv);
        v.albedo[0] = a.x;
        v.albedo[1] = a.y;
        v.albedo[2] = a.z;
    }
    return v;
}

// ---- DielectricBsdf (microfacet.rs:155-307) with fresnel_dielectric and
// refract (surfaces.rs:86-123); operation order as in the reference ----
__device__ __forceinline__ float fresnel_dielectric(float cos_theta_i, float eta) {
    float ci = fminf(fmaxf(cos_theta_i, -1.0f), 1.0f);
    if (ci < 0.0f) {
        ci = -ci;
        eta = 1.0f / eta;
    }
    const float sin2_t = (eta * eta) * (1.0f - ci * ci);
    if (sin2_t >= 1.0f) return 1.0f;
    const float ct = sqrtf(1.0f - sin2_t);
    const float r_par = (eta * ci - ct) / (eta * ci + ct);
    const float r_per = (ci - eta * ct) / (ci + eta * ct);
    return 0.5f * (r_par * r_par + r_per * r_per);
}
__device__ __forceinline__ bool refract_dir(f3 v, f3 n, float eta, f3& out) {
    const float cos_i = dot(n, v);
    const float sin2_t = (eta * eta) * (1.0f - cos_i * cos_i);
    if (sin2_t >= 1.0f) return false;
    const float cos_t = sqrtf(1.0f - sin2_t);
    out = (-v) * eta + n * (eta * cos_i - cos_t);
    return true;
}
__device__ __forceinline__ float ggx_g2(float a, f3 wi, f3 wo) {
    return 1.0f / ((1.0f + ggx_lambda(a, wi)) + ggx_lambda(a, wo));
}
// Refraction half-vector -(wo + wi*eta).normalize(), turned to wo's side.
__device__ __forceinline__ f3 refraction_half(f3 wi, f3 wo, float eta) {
    f3 h = -normalize(wo + wi * eta);
    if (h.z * wo.z < 0.f) h = -h;
    return h;
}
__device__ __forceinline__ f3 dielectric_eval(const MatView& m, f3 wi, f3 wo) {
    const float cos_wo = fabsf(wo.z), cos_wi = fabsf(wi.z);
    if (cos_wo == 0.f || cos_wi == 0.f) return mk(0.f, 0.f, 0.f);
    float v;
    if (same_hemi(wi, wo)) {
        const f3 h = normalize(wi + wo);
        const float f = fresnel_dielectric(fabsf(dot(wi, h)), m.eta);
        v = ((f * ggx_d(m.alpha, h)) * ggx_g2(m.alpha, wi, wo)) / ((4.0f * cos_wi) * cos_wo);
    } else {
        const float eta = wo.z > 0.f ? m.eta : 1.0f / m.eta;
        const f3 h = refraction_half(wi, wo, eta);
        const float woh = dot(wo, h), wih = dot(wi, h);
        if (woh == 0.f || wih == 0.f) return mk(0.f, 0.f, 0.f);
        const float f = 1.0f - fresnel_dielectric(fabsf(wih), m.eta);
        const float d = ggx_d(m.alpha, h), g = ggx_g2(m.alpha, wi, wo);
        const float s = woh + eta * wih;
        const float denom = s * s;
        if (denom == 0.f) return mk(0.f, 0.f, 0.f);
        const float eta2 = eta * eta;
        v = ((((f * d) * g) * eta2) * fabsf(woh)) * fabsf(wih) / ((cos_wi * cos_wo) * denom);
    }
    return mk(v, v, v);
}
__device__ __forceinline__ float dielectric_pdf(const MatView& m, f3 wi, f3 wo) {
    if (fabsf(wo.z) == 0.f || fabsf(wi.z) == 0.f) return 0.f;
    if (same_hemi(wi, wo)) {
        const f3 h = normalize(wi + wo);
        const float whwi = fabsf(dot(wi, h));
        if (whwi == 0.f) return 0.f;
        const float f = fresnel_dielectric(fabsf(dot(wo, h)), m.eta);
        return ((f * ggx_d(m.alpha, h)) * fabsf(h.z)) / (4.0f * whwi);
    }
    const float eta = wo.z > 0.f ? m.eta : 1.0f / m.eta;
    const f3 h = refraction_half(wi, wo, eta);
    const float woh = dot(wo, h), wih = dot(wi, h);
    if (woh == 0.f || wih == 0.f) return 0.f;
    const float s = woh + eta * wih;
    const float denom = s * s;
    if (denom == 0.f) return 0.f;
    const float f = 1.0f - fresnel_dielectric(fabsf(woh), m.eta);
    return (((((f * ggx_d(m.alpha, h)) * fabsf(h.z)) * eta) * eta) * fabsf(wih)) / denom;
}

__device__ __forceinline__ f3 bsdf_eval(const MatView& m, f3 wi, f3 wo) {
    if (m.kind == AR_MATERIAL_DIELECTRIC) return dielectric_eval(m, wi, wo);
    if (!same_hemi(wi, wo)) return mk(0.f, 0.f, 0.f);
    if (m.kind == AR_MATERIAL_LAMBERTIAN) return mk(m.albedo[0] * kInvPi, m.albedo[1] * kInvPi, m.albedo[2] * kInvPi);
    float ci = fabsf(wi.z), co = fabsf(wo.z);
    if (ci == 0.f || co == 0.f) return mk(0.f, 0.f, 0.f);
    f3 h = normalize(wi + wo);
    f3 f = fresnel_schlick(fabsf(dot(wi, h)), m.f0);
    float d = ggx_d(m.alpha, h);
    float g = 1.0f / ((1.0f + ggx_lambda(m.alpha, wi)) + ggx_lambda(m.alpha, wo));
    return f * (d * g / ((4.0f * ci) * co));
}
__device__ __forceinline__ float bsdf_pdf(const MatView& m, f3 wi, f3 wo) {
    if (m.kind == AR_MATERIAL_DIELECTRIC) return dielectric_pdf(m, wi, wo);
    if (!same_hemi(wi, wo)) return 0.f;
    if (m.kind == AR_MATERIAL_LAMBERTIAN) return fabsf(wi.z) * kInvPi;
    f3 h = normalize(wi + wo);
    float whwi = fabsf(dot(wi, h));
    if (whwi == 0.f) return 0.f;
    return ggx_d(m.alpha, h) * fabsf(h.z) / (4.0f * whwi);
}
// Returns false when the reference returns None.  u_sel picks the
// dielectric's lobe (reflection when u_sel < F); the other BSDFs ignore it.
__device__ __forceinline__ bool bsdf_sample(const MatView& m, f3 wo, float u_sel, float ux, float uy, f3& wi,
                                            float& pdf, f3& f) {
    if (m.kind == AR_MATERIAL_LAMBERTIAN) {
        wi = cosine_hemisphere(ux, uy);
        if (wo.z < 0.f) wi.z = -wi.z;
        pdf = fabsf(wi.z) * kInvPi;
        if (pdf == 0.f) return false;
        f = mk(m.albedo[0] * kInvPi, m.albedo[1] * kInvPi, m.albedo[2] * kInvPi);
        return true;
    }
    if (wo.z == 0.f) return false;
    float a2 = m.alpha * m.alpha;
    float c2 = (1.0f - ux) / ((a2 - 1.0f) * ux + 1.0f);
    float ch = sqrtf(fmaxf(c2, 0.f)), sh = sqrtf(fmaxf(1.0f - c2, 0.f));
    float phi = (2.0f * kPi) * uy;
    float sp, cp;
    ar_trig::sincos(phi, &sp, &cp);
    f3 h = mk(sh * cp, sh * sp, ch);
    if (h.z * wo.z < 0.f) h = -h;
    if (m.kind == AR_MATERIAL_DIELECTRIC && !(u_sel < fresnel_dielectric(fabsf(dot(wo, h)), m.eta))) {
        const float eta = wo.z > 0.f ? 1.0f / m.eta : m.eta;
        if (!refract_dir(wo, h, eta, wi)) return false;
        if (same_hemi(wi, wo)) return false;
        pdf = bsdf_pdf(m, wi, wo);
        if (pdf == 0.f) return false;
        f = bsdf_eval(m, wi, wo);
        return true;
    }
    wi = -wo + (h * 2.0f) * dot(wo, h);
    if (!same_hemi(wi, wo)) return false;
    pdf = bsdf_pdf(m, wi, wo);
    if (pdf == 0.f) return false;
    f = bsdf_eval(m, wi, wo);
    return true;
}

// ---- lights ----
struct LightView {
    uint32_t kind;
    float area;
    f3 pos, inten, e1, e2, n;
};
__device__ __forceinline__ LightView load_light(const DevScene& sc, uint32_t i) {
    const LightRecord& r = sc.lights[i];
    LightView l;
    l.kind = r.kind;
    l.area = r.area;
    l.pos = ld3(r.pos);
    l.inten = ld3(r.inten);
    l.e1 = ld3(r.e1);
    l.e2 = ld3(r.e2);
    l.n = ld3(r.n);
    return l;
}
__device__ __forceinline__ bool light_enabled(const DevScene& sc) {
    return sc.light_dist != AR_LIGHT_DIST_NONE && sc.num_lights > 0;
}
__device__ __forceinline__ void light_select(const DevScene& sc, float u, uint32_t& idx, float& pmf) {
    const uint32_t n = sc.num_lights;
    if (sc.light_dist == AR_LIGHT_DIST_UNIFORM) {
        float s = u * float(n);
        uint32_t i = s >= 0.f ? uint32_t(s) : 0u;
        idx = min(i, n - 1);
        pmf = 1.0f / float(n);
        return;
    }
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (sc.light_cdf[mid] < u) lo = mid + 1; else hi = mid;
    }
    idx = min(lo, n - 1);
    pmf = sc.light_pmf[idx];
}
__device__ __forceinline__ float light_pmf_of(const DevScene& sc, uint32_t i) {
    return sc.light_dist == AR_LIGHT_DIST_UNIFORM ? 1.0f / float(sc.num_lights) : sc.light_pmf[i];
}
// Light::sample toward `ref`; false when the reference returns None.
__device__ __forceinline__ bool light_sample(const LightView& l, f3 ref, float ux, float uy, f3& wi, float& dist, f3& li,
                                             float& pdf) {
    if (l.kind == AR_LIGHT_POINT) {
        f3 off = l.pos - ref;
        float d2 = dot(off, off);
        float d = sqrtf(d2);
        if (d < 1e-6f) return false;
        wi = off / d;
        dist = d;
        li = l.inten / d2;
        pdf = 1.0f;
        return true;
    }
    f3 q = (l.pos + l.e1 * ux) + l.e2 * uy;
    f3 off = q - ref;
    float d2 = dot(off, off);
    float d = sqrtf(d2);
    if (d < 1e-6f) return false;
    wi = off / d;
    float cl = -dot(l.n, wi);
    if (cl <= 0.f) return false;
    dist = d;
    li = l.inten;
    pdf = d2 / (cl * l.area);
    return true;
}
__device__ __forceinline__ float light_pdf_emission_dir(const LightView& l, f3 dir) {
    if (l.kind == AR_LIGHT_POINT) return 1.0f / (4.0f * kPi);
    float c = dot(l.n, dir);
    return c > 0.f ? c * kInvPi : 0.f;
}

// ---- camera ----
__device__ __forceinline__ Ray camera_ray(const CameraDev& c, float u, float v) {
    f3 dir = ((ld3(c.ll) + ld3(c.hor) * u) + ld3(c.ver) * v) - ld3(c.o);
    return Ray{ld3(c.o), normalize(dir), 0.001f, FLT_MAX};
}
__device__ __forceinline__ float camera_pdf_we(const CameraDev& c, f3 d) {
    float ct = dot(d, ld3(c.fwd));
    if (ct <= 0.f) return 0.f;
    return 1.0f / (((c.area * ct) * ct) * ct);
}

__device__ __forceinline__ float power_heuristic(float a, float b) {
    float a2 = a * a, b2 = b * b;
    return a2 / (a2 + b2);
}

// Warp-aggregated queue slot allocation; every lane of the warp must call it.
__device__ __forceinline__ uint32_t warp_alloc(uint32_t* counter, bool pred) {
    const uint32_t mask = __ballot_sync(0xffffffffu, pred);
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if (mask) {
        const int leader = __ffs(mask) - 1;
        if (int(lane) == leader) base = atomicAdd(counter, uint32_t(__popc(mask)));
        base = __shfl_sync(0xffffffffu, base, leader);
    }
    return base + uint32_t(__popc(mask & ((1u << lane) - 1u)));
}

}  // namespace ar
