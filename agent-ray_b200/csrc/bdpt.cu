// Wavefront bidirectional path tracer (BidirectionalPathTracer::render,
// src/integrators/bidirectional_path_tracer.rs:1221-1357), batched over jobs.
//
// A batch is a list of segments (job, first sample, count); the samples of all
// segments are traced together.  Stages per batch:
//   generate   camera vertex z0 + primary ray, light vertex y0 + emitted ray
//   [extend -> vertex] x max depth of the batch
//              both subpaths of every sample trace in one wavefront; each hit
//              appends a vertex (area-measure pdf_fwd) and retroactively sets
//              pdf_rev of the previous vertex (:338-559)
//   connect    one thread per sample enumerates the (s, t) strategies with
//              s + t <= max_depth + 2, evaluates the unweighted contribution
//              and the power-heuristic MIS weight (FP64 ratio walk, :594-770)
//              and emits one shadow ray per candidate (:782-1155)
//   shadow     any-hit test; visible contributions go to the job's film (s >= 2:
//              the sample's pixel; s = 1: the projected splat pixel)
// Vertices are stored SoA by (subpath, depth, sample) so each stage reads
// coalesced 16-byte records.  Quad-light strategies (t = 0 and area-light t = 1)
// are the same extension the oracle implements.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "ar_bdpt.hpp"
#include "ar_shading.cuh"

namespace cg = cooperative_groups;

namespace ar {

namespace {

constexpr uint32_t kTypeSurface = 0, kTypeCamera = 1, kTypeLight = 2;

// Layout of the per-batch counter block (max_depth <= 62): rays per bounce,
// shadow count and overflow flag, ray-fetch cursors, then the histogram and
// bucket offsets of the (S, T) sort.
constexpr uint32_t kBdShadowCursor = 127, kBdExtendCursor = 128, kBdBins = 256, kBdHist = 192,
                   kBdOffs = kBdHist + kBdBins, kBdCounts = kBdOffs + kBdBins;

struct BdParams {
    const BdJob* jobs;
    const BdSegment* seg;
    const uint32_t* dyn;  // device: [0] samples in this batch, [1] segments (set per batch)
    uint32_t cap;         // batch capacity: the stride of the per-sample arrays
    uint32_t maxv;        // vertex capacity per subpath
    uint32_t* sjob;     // job of each batch sample
    unsigned long long* sindex;  // global sample index of each batch sample
    float4* va;  // p.xyz, pdf_fwd
    float4* vb;  // n.xyz, pdf_rev
    float4* vc;  // thr.xyz, info (type << 30 | delta << 29 | index)
    float2* vuv; // tex_uv of surface vertices
    float4* sva; // the vertex arrays permuted into the (S, T)-sorted sample
    float4* svb; // order, so the connection kernel's warps read them coalesced
    float4* svc;
    float2* svuv;
    uint8_t* nv; // [sub * cap + si]
    float4* thr; // per subpath, at sub * cap + si: thr.xyz, previous directional pdf
    uint32_t* dim;
    float4* ray_o[2];
    float4* ray_d[2];
    uint32_t* qpath[2];
    float4* hit;
    uint32_t* hit_inst;
    float4* sh_o;
    float4* sh_d;  // dir.xyz, tmax
    float4* sh_c;  // contribution.xyz, pixel bits
    uint32_t* sh_job;
    uint32_t sh_cap;
    uint32_t* counts;  // [0..63]: rays per bounce; [64]: shadow rays; [65]: overflow flag;
                       // [kBdShadowCursor], [kBdExtendCursor + depth]: ray-fetch cursors;
                       // [kBdHist..], [kBdOffs..]: (S, T) histogram and bucket offsets
    uint32_t* order;   // batch samples sorted by (S, T)
};

// Subpath q = 2 si + sub (as carried in the ray queues) -> its slot in the
// per-subpath arrays, camera subpaths first: a warp of camera (or light) rays
// of neighbouring samples reads contiguous records.
__device__ __forceinline__ uint32_t sp_slot(const BdParams& P, uint32_t q) { return (q & 1u) * P.cap + (q >> 1); }

__device__ __forceinline__ size_t vidx(const BdParams& P, uint32_t sub, uint32_t k, uint32_t si) {
    return (size_t(sub) * P.maxv + k) * P.cap + si;
}

struct Vtx {
    f3 p, n, thr;
    float pdf_fwd, pdf_rev;
    uint32_t type, index;
    bool delta;
    bool uv;  // a textured surface vertex: its tex_uv is stored in vuv
};

__device__ __forceinline__ Vtx load_vtx(const BdParams& P, uint32_t sub, uint32_t k, uint32_t si) {
    const size_t i = vidx(P, sub, k, si);
    // read-only where this is called (connection and MIS stages): through the
    // non-coherent path (connection stage -2.5%)
    const float4 a = __ldg(P.va + i), b = __ldg(P.vb + i), c = __ldg(P.vc + i);
    Vtx v;
    v.p = mk(a.x, a.y, a.z);
    v.pdf_fwd = a.w;
    v.n = mk(b.x, b.y, b.z);
    v.pdf_rev = b.w;
    v.thr = mk(c.x, c.y, c.z);
    const uint32_t info = __float_as_uint(c.w);
    v.type = info >> 30;
    v.delta = (info >> 29) & 1u;
    v.uv = (info >> 28) & 1u;
    v.index = info & 0x0fffffffu;
    return v;
}

__device__ __forceinline__ void store_vtx(const BdParams& P, uint32_t sub, uint32_t k, uint32_t si, f3 p, f3 n, f3 thr,
                                          float pdf_fwd, uint32_t type, bool delta, uint32_t index, bool uv = false,
                                          float tu = 0.f, float tv = 0.f) {
    const size_t i = vidx(P, sub, k, si);
    P.va[i] = make_float4(p.x, p.y, p.z, pdf_fwd);
    P.vb[i] = make_float4(n.x, n.y, n.z, 0.f);
    P.vc[i] = make_float4(thr.x, thr.y, thr.z,
                          __uint_as_float((type << 30) | (delta ? (1u << 29) : 0u) | (uv ? (1u << 28) : 0u) |
                                          (index & 0x0fffffffu)));
    if (uv) P.vuv[i] = make_float2(tu, tv);
}

// The material of surface vertex (sub, k) of sample si, with a textured
// albedo sampled at the vertex's tex_uv (read only for textured materials).
__device__ __forceinline__ MatView vtx_mat(const BdParams& P, const BdJob& J, const Vtx& v, uint32_t sub, uint32_t k,
                                           uint32_t si) {
    if (!v.uv) return load_mat(J.sc, v.index);
    const float2 uv = __ldg(P.vuv + vidx(P, sub, k, si));
    return load_mat_at(J.sc, v.index, uv.x, uv.y);
}

// pdf_solid_angle_to_area (:305-314) and geometry_term (:318-328)
__device__ __forceinline__ float pdf_sa_to_area(float pdf, f3 from, f3 to, f3 n_to) {
    const f3 d = to - from;
    const float d2 = dot(d, d);
    if (d2 < 1e-12f) return 0.f;
    const f3 dir = d / sqrtf(d2);
    return pdf * fabsf(dot(n_to, dir)) / d2;
}
__device__ __forceinline__ float geometry_term(f3 pa, f3 na, f3 pb, f3 nb) {
    const f3 d = pb - pa;
    const float d2 = dot(d, d);
    if (d2 < 1e-12f) return 0.f;
    const f3 dir = d / sqrtf(d2);
    return fabsf(dot(na, dir)) * fabsf(dot(nb, -dir)) / d2;
}

__device__ __forceinline__ f3 uniform_sphere(float ux, float uy) {
    const float ct = 1.0f - 2.0f * ux;
    const float st = sqrtf(fmaxf(1.0f - ct * ct, 0.0f));
    const float phi = (2.0f * kPi) * uy;
    float sp, cp;
    ar_trig::sincos(phi, &sp, &cp);
    return mk(st * cp, st * sp, ct);
}

__device__ __forceinline__ bool mis_delta(const Vtx& v) { return v.type == kTypeSurface && v.delta; }

// mis_weight (:594-770) with the area-light extension for the t == 1 step.
__device__ __noinline__ float mis_weight(const BdParams& P, const BdJob& J, uint32_t si, uint32_t S, uint32_t T, uint32_t s,
                            uint32_t t, float pdf_cc, float pdf_cl) {
    if (J.mis_mode == AR_MIS_UNIFORM) {
        const uint32_t len = s + t;
        uint32_t count = 0;
        for (uint32_t t2 = 0; t2 <= min(len, T); ++t2) {
            const uint32_t s2 = len - t2;
            if (s2 > S || s2 + t2 < 2 || s2 == 0) continue;
            count++;
        }
        return count == 0 ? 1.0f : 1.0f / float(count);
    }
    if (s + t == 2) return 1.0f;
    const double beta = double(J.mis_beta);
    auto pw = [&](double r) { return beta == 2.0 ? r * r : pow(r, beta); };
    double sum = 0.0;
    {
        double ri = 1.0;
        if (s >= 1) {
            const Vtx v = load_vtx(P, 0, s - 1, si);
            ri *= double(pdf_cc) / double(fmaxf(v.pdf_fwd, 1e-30f));
            const bool pd = s >= 2 ? mis_delta(load_vtx(P, 0, s - 2, si)) : true;
            if (!mis_delta(v) && !pd) sum += pw(fabs(ri));
        }
        for (uint32_t i = s; i-- > 1;) {
            const Vtx v = load_vtx(P, 0, i, si);
            ri *= double(fmaxf(v.pdf_rev, 0.f)) / double(fmaxf(v.pdf_fwd, 1e-30f));
            const bool pd = mis_delta(load_vtx(P, 0, i - 1, si));
            if (!mis_delta(v) && !pd) sum += pw(fabs(ri));
        }
    }
    {
        double ri = 1.0;
        if (t >= 1) {
            const Vtx v = load_vtx(P, 1, t - 1, si);
            ri *= double(pdf_cl) / double(fmaxf(v.pdf_fwd, 1e-30f));
            bool pd;
            if (t >= 2) {
                pd = mis_delta(load_vtx(P, 1, t - 2, si));
            } else {
                const Vtx y0 = load_vtx(P, 1, 0, si);
                pd = J.sc.lights[y0.index].kind == AR_LIGHT_POINT;
            }
            if (!mis_delta(v) && !pd) sum += pw(fabs(ri));
        }
        for (uint32_t i = t; i-- > 1;) {
            const Vtx v = load_vtx(P, 1, i, si);
            ri *= double(fmaxf(v.pdf_rev, 0.f)) / double(fmaxf(v.pdf_fwd, 1e-30f));
            const bool pd = mis_delta(load_vtx(P, 1, i - 1, si));
            if (!mis_delta(v) && !pd) sum += pw(fabs(ri));
        }
    }
    return float(1.0 / (1.0 + sum));
}

// Prefix form of the reference ratio walk for the power heuristic with
// beta = 2 and no delta surface vertex (the only BSDFs here are Lambertian and
// GGX).  With q_i = pdf_rev(z_i) / pdf_fwd(z_i) the camera-side terms of
// strategy (s, t) are r1^2 (1 + q_{s-1}^2 + (q_{s-1} q_{s-2})^2 + ...), where
// r1 = pdf_connect_cam / pdf_fwd(z_{s-1}); the bracket C_s obeys C_1 = 1,
// C_s = 1 + q_{s-1}^2 C_{s-1}.  The light side is symmetric (D_t), and its
// t = 1 term counts only for area lights.  Same sums as mis_weight, in FP64.
constexpr uint32_t kMisCache = 16;
struct MisCache {
    double C[kMisCache], D[kMisCache];
    float fwd_cam[kMisCache], fwd_light[kMisCache];
    bool fast;
};

__device__ void build_mis_cache(const BdParams& P, const BdJob& J, uint32_t si, uint32_t S, uint32_t T, MisCache& mc) {
    mc.fast = J.mis_mode == AR_MIS_POWER && J.mis_beta == 2.0f && S <= kMisCache && T <= kMisCache;
    if (!mc.fast) return;
    double c = 1.0;
    for (uint32_t s = 1; s <= S; ++s) {
        const Vtx v = load_vtx(P, 0, s - 1, si);
        if (v.type == kTypeSurface && v.delta) mc.fast = false;
        mc.fwd_cam[s - 1] = v.pdf_fwd;
        if (s >= 2) {
            const double q = double(fmaxf(v.pdf_rev, 0.f)) / double(fmaxf(v.pdf_fwd, 1e-30f));
            c = 1.0 + q * q * c;
        }
        mc.C[s - 1] = c;  // C_s (s >= 1) with q_{s-1} taken from z[s-1]
    }
    double d = 1.0;
    for (uint32_t t = 1; t <= T; ++t) {
        const Vtx v = load_vtx(P, 1, t - 1, si);
        if (v.type == kTypeSurface && v.delta) mc.fast = false;
        mc.fwd_light[t - 1] = v.pdf_fwd;
        if (t >= 2) {
            const double q = double(fmaxf(v.pdf_rev, 0.f)) / double(fmaxf(v.pdf_fwd, 1e-30f));
            d = 1.0 + q * q * d;
        }
        mc.D[t - 1] = d;
    }
}

__device__ __forceinline__ float mis_weight_cached(const BdParams& P, const BdJob& J, const MisCache& mc, uint32_t si,
                                                   uint32_t S, uint32_t T, uint32_t s, uint32_t t, float pdf_cc,
                                                   float pdf_cl, bool light_is_point) {
    if (!mc.fast) return mis_weight(P, J, si, S, T, s, t, pdf_cc, pdf_cl);
    if (s + t == 2) return 1.0f;
    double sum = 0.0;
    if (s >= 2) {
        const double r = double(pdf_cc) / double(fmaxf(mc.fwd_cam[s - 1], 1e-30f));
        sum += r * r * mc.C[s - 1];
    }
    if (t >= 2 || (t == 1 && !light_is_point)) {
        const double r = double(pdf_cl) / double(fmaxf(mc.fwd_light[t - 1], 1e-30f));
        sum += r * r * mc.D[t - 1];
    }
    return float(1.0 / (1.0 + sum));
}

__device__ __forceinline__ void film_add(const BdJob& J, uint32_t pix, f3 v) {
    if (J.film64) {
        double* f = static_cast<double*>(J.film) + 3 * size_t(pix);
        atomicAdd(f, double(v.x));
        atomicAdd(f + 1, double(v.y));
        atomicAdd(f + 2, double(v.z));
    } else {
        float* f = static_cast<float*>(J.film) + 3 * size_t(pix);
        atomicAdd(f, v.x);
        atomicAdd(f + 1, v.y);
        atomicAdd(f + 2, v.z);
    }
}

__device__ __forceinline__ void push_shadow(const BdParams& P, uint32_t job, f3 o, f3 d, float tmax, f3 c,
                                            uint32_t pix) {
    cg::coalesced_group g = cg::coalesced_threads();
    uint32_t base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(&P.counts[64], g.size());
    base = g.shfl(base, 0);
    const uint32_t slot = base + g.thread_rank();
    if (slot >= P.sh_cap) {
        atomicExch(&P.counts[65], 1u);
        return;
    }
    st_once(P.sh_o + slot, make_float4(o.x, o.y, o.z, 0.f));
    st_once(P.sh_d + slot, make_float4(d.x, d.y, d.z, tmax));
    st_once(P.sh_c + slot, make_float4(c.x, c.y, c.z, __uint_as_float(pix)));
    st_once(P.sh_job + slot, job);
}

__global__ void __launch_bounds__(256) k_bd_generate(BdParams P) {
    const uint32_t ns = P.dyn[0], nseg = P.dyn[1];
    // Threads [0, ns) start the camera subpaths of samples 0..ns-1, threads
    // [ns, 2 ns) their light subpaths: a warp's 32 rays are all camera rays of
    // neighbouring pixels, or all light rays, and every later bounce keeps the
    // queue order, so the extension warps stay coherent.  q = 2 si + sub names
    // the subpath in the per-subpath arrays.
    for (uint32_t base = blockIdx.x * blockDim.x; base < 2 * ns; base += gridDim.x * blockDim.x) {
        const uint32_t idx = base + threadIdx.x;
        bool live = idx < 2 * ns;
        const uint32_t sub = idx >= ns ? 1u : 0u, si = idx - sub * ns, q = 2 * si + sub;
        Ray r{};
        if (live) {
            uint32_t lo = 0, hi = nseg;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (P.seg[mid].offset <= si) lo = mid; else hi = mid;
            }
            const BdSegment sg = P.seg[lo];
            const BdJob& J = P.jobs[sg.job];
            const unsigned long long g = sg.sample_begin + (si - sg.offset);
            const uint32_t npix = J.width * J.height;
            const uint32_t pixel = uint32_t(g % npix), sample = uint32_t(g / npix);
            const uint64_t key = counter_key(J.seed, pixel, sample);
            if (sub == 0) {
                P.sjob[si] = sg.job;
                P.sindex[si] = g;
                const float jx = counter_u01(key, 0), jy = counter_u01(key, 1);
                const uint32_t px = pixel % J.width, py = pixel / J.width;
                r = camera_ray(J.cam, (float(px) + jx) / float(J.width), 1.0f - (float(py) + jy) / float(J.height));
                store_vtx(P, 0, 0, si, ld3(J.cam.o), r.d, mk(1.f, 1.f, 1.f), 1.0f, kTypeCamera, true, 0);
                P.nv[si] = 1;
                P.thr[si] = make_float4(1.f, 1.f, 1.f, camera_pdf_we(J.cam, r.d));
                P.dim[si] = 2;
            } else if (light_enabled(J.sc)) {
                uint32_t d = kLightSubpathDim;
                const float u_sel = counter_u01(key, d++);
                const float upx = counter_u01(key, d++), upy = counter_u01(key, d++);
                const float udx = counter_u01(key, d++), udy = counter_u01(key, d++);
                uint32_t li;
                float sel;
                light_select(J.sc, u_sel, li, sel);
                const LightView L = load_light(J.sc, li);
                f3 o, dir, nl;
                float pdf_pos, pdf_dir;
                bool ok = true;
                if (L.kind == AR_LIGHT_POINT) {
                    dir = uniform_sphere(udx, udy);
                    o = L.pos;
                    pdf_pos = 1.0f;
                    pdf_dir = 1.0f / (4.0f * kPi);
                    nl = dir;
                } else {
                    o = (L.pos + L.e1 * upx) + L.e2 * upy;
                    const f3 local = cosine_hemisphere(udx, udy);
                    dir = to_world(onb_from_normal(L.n), local);
                    pdf_pos = 1.0f / L.area;
                    pdf_dir = local.z * kInvPi;
                    nl = L.n;
                    ok = pdf_dir > 0.f;
                }
                if (ok) {
                    r = Ray{o, normalize(dir), 1e-4f, FLT_MAX};
                    const float pp = pdf_pos * sel;
                    store_vtx(P, 1, 0, si, o, nl, L.inten / pp, pp, kTypeLight, L.kind == AR_LIGHT_POINT, li);
                    P.nv[P.cap + si] = 1;
                    f3 thr = L.inten / (pp * pdf_dir);
                    thr = thr * fabsf(dot(nl, r.d));
                    P.thr[P.cap + si] = make_float4(thr.x, thr.y, thr.z, pdf_dir);
                    P.dim[P.cap + si] = d;
                } else {
                    P.nv[P.cap + si] = 0;
                    live = false;
                }
            } else {
                P.nv[P.cap + si] = 0;
                live = false;
            }
            if (J.max_depth == 0) live = false;
        }
        const uint32_t slot = warp_alloc(&P.counts[0], live);
        if (!live) continue;
        P.ray_o[0][slot] = make_float4(r.o.x, r.o.y, r.o.z, r.tmin);
        P.ray_d[0][slot] = make_float4(r.d.x, r.d.y, r.d.z, r.tmax);
        P.qpath[0][slot] = q;
    }
}

__global__ void AR_TRAVERSAL_BOUNDS k_bd_extend(const __grid_constant__ BdParams P, uint32_t depth, int* err) {
    const uint32_t n = P.counts[depth];
    const int b = depth & 1;
    run_traversal<false>(
        &P.counts[kBdExtendCursor + depth], n, err,
        [&](uint32_t j, const DevScene*& s, Ray& r) {
            const float4 a = P.ray_o[b][j], d = P.ray_d[b][j];
            s = &P.jobs[P.sjob[P.qpath[b][j] >> 1]].sc;
            r = Ray{mk(a.x, a.y, a.z), mk(d.x, d.y, d.z), a.w, d.w};
        },
        [&](uint32_t j, const HitRec& h) {
            P.hit[j] = make_float4(h.t, h.u, h.v, __uint_as_float(h.slot));
            P.hit_inst[j] = h.inst;
        });
}

// One bounce of both subpaths (:368-434, :498-556).  <= 64 registers, as
// k_shade: latency-bound, faster at double occupancy despite spills.
__global__ void __launch_bounds__(256, 4) k_bd_vertex(BdParams P, uint32_t depth) {
    const uint32_t n = P.counts[depth];
    const int b = depth & 1;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t j = base + threadIdx.x;
        bool cont = false;
        uint32_t q = 0;
        f3 no, nd;
        if (j < n) {
            q = P.qpath[b][j];
            const uint32_t si = q >> 1, sub = q & 1u;
            const BdJob& J = P.jobs[P.sjob[si]];
            const float4 h = P.hit[j];
            const uint32_t slot = __float_as_uint(h.w);
            if (slot != kInvalid) {
                const float4 ro4 = P.ray_o[b][j], rd4 = P.ray_d[b][j];
                const f3 ro = mk(ro4.x, ro4.y, ro4.z), rd = mk(rd4.x, rd4.y, rd4.z);
                const Shade s = make_shade(J.sc, ro, rd, h.x, h.y, h.z, slot, P.hit_inst[j]);
                const MatView m = load_mat_at(J.sc, s.mat, s.tu, s.tv);
                const uint32_t spi = sp_slot(P, q);
                const float4 t4 = P.thr[spi];
                f3 thr = mk(t4.x, t4.y, t4.z);
                const uint32_t k = P.nv[sub * P.cap + si];  // index of the new vertex
                const size_t pi = vidx(P, sub, k - 1, si);
                const float4 pa = P.va[pi], pb = P.vb[pi];
                const f3 prev_p = mk(pa.x, pa.y, pa.z), prev_n = mk(pb.x, pb.y, pb.z);
                const float pdf_fwd = pdf_sa_to_area(t4.w, prev_p, s.p, s.n);
                store_vtx(P, sub, k, si, s.p, s.n, thr, pdf_fwd, kTypeSurface, false, s.mat,
                          J.sc.materials[s.mat].tex >= 0, s.tu, s.tv);
                P.nv[sub * P.cap + si] = uint8_t(k + 1);
                const unsigned long long g = P.sindex[si];
                const uint32_t npix = J.width * J.height;
                const uint64_t key = counter_key(J.seed, uint32_t(g % npix), uint32_t(g / npix));
                uint32_t d = P.dim[spi];
                const f3 wo_l = to_local(s.onb, -rd);
                const float usel = counter_u01(key, d++);
                const float ux = counter_u01(key, d++), uy = counter_u01(key, d++);
                f3 wi, f;
                float pdf;
                if (bsdf_sample(m, wo_l, usel, ux, uy, wi, pdf, f) && pdf != 0.f && !is_zero(f)) {
                    thr = thr * ((f * fabsf(wi.z)) / pdf);
                    const float pdf_rev_dir = bsdf_pdf(m, wo_l, wi);
                    P.vb[pi].w = pdf_sa_to_area(pdf_rev_dir, s.p, prev_p, prev_n);
                    bool alive = true;
                    if (depth + 1 >= J.rr_depth) {
                        const float survival = fminf(max3(thr), 0.95f);
                        if (counter_u01(key, d++) > survival || survival <= 0.f) alive = false;
                        else thr = thr / survival;
                    }
                    if (alive && depth + 1 < J.max_depth) {
                        const f3 wi_w = to_world(s.onb, wi);
                        no = s.p + (s.n * 1e-4f) * signum(dot(wi_w, s.n));
                        nd = normalize(wi_w);
                        P.thr[spi] = make_float4(thr.x, thr.y, thr.z, pdf);
                        P.dim[spi] = d;
                        cont = true;
                    }
                }
            }
        }
        const uint32_t rs = warp_alloc(&P.counts[depth + 1], cont);
        if (cont) {
            P.ray_o[b ^ 1][rs] = make_float4(no.x, no.y, no.z, 1e-4f);
            P.ray_d[b ^ 1][rs] = make_float4(nd.x, nd.y, nd.z, FLT_MAX);
            P.qpath[b ^ 1][rs] = q;
        }
    }
}

// Out-of-line BSDF bodies for the connection kernel: its warps diverge
// across strategies, and one copy of each body keeps the instruction
// footprint small.  Same arithmetic as the inline forms.
__device__ __noinline__ f3 bsdf_eval_ool(const MatView& m, f3 wi, f3 wo) { return bsdf_eval(m, wi, wo); }
__device__ __noinline__ float bsdf_pdf_ool(const MatView& m, f3 wi, f3 wo) { return bsdf_pdf(m, wi, wo); }

// connect_bdpt for s >= 2 (:782-1044) + the t == 0 extension.  Emits a shadow
// ray with the MIS-weighted contribution, or deposits directly when t == 0.
// Camera-side data of strategy (s, *): z = z[s-1] and its shading frame.
struct CamSide {
    Vtx z;
    f3 zp_p;
    Onb oz;
    MatView mz;
    f3 wo_zl;
};

__device__ __forceinline__ CamSide cam_side(const BdParams& P, const BdJob& J, uint32_t si, uint32_t s) {
    CamSide c;
    c.z = load_vtx(P, 0, s - 1, si);
    c.zp_p = load_vtx(P, 0, s - 2, si).p;
    c.oz = onb_from_normal(c.z.n);
    c.mz = vtx_mat(P, J, c.z, 0, s - 1, si);
    c.wo_zl = to_local(c.oz, normalize(c.zp_p - c.z.p));
    return c;
}

__device__ void connect_general(const BdParams& P, const BdJob& J, uint32_t job, uint32_t si, uint32_t S, uint32_t T,
                                const MisCache& mc, bool lpt, const CamSide& cs, uint32_t s, uint32_t t,
                                uint32_t pix) {
    const Vtx& z = cs.z;
    if (t == 0) {
        const MatView& mz = cs.mz;
        if (mz.emitter < 0 || !light_enabled(J.sc)) return;
        const LightView lt = load_light(J.sc, uint32_t(mz.emitter));
        const f3 wo = normalize(cs.zp_p - z.p);
        if (dot(lt.n, wo) <= 0.f) return;
        const f3 c = z.thr * lt.inten;
        if (max3(c) <= 0.f) return;
        const float pdf_cc = light_pmf_of(J.sc, uint32_t(mz.emitter)) / lt.area;
        const float w = mis_weight_cached(P, J, mc, si, S, T, s, 0, pdf_cc, 0.f, lpt);
        film_add(J, pix, (c * w) * J.inv_spp);
        return;
    }
    const Vtx y = load_vtx(P, 1, t - 1, si);
    if (y.type == kTypeSurface && y.delta) return;
    const f3 d = y.p - z.p;
    const float d2 = dot(d, d);
    if (d2 < 1e-10f) return;
    const float dist = sqrtf(d2);
    const f3 wi_z = d / dist;
    const f3 wi_y = -wi_z;
    const f3 so = z.p + (z.n * 1e-4f) * signum(dot(wi_z, z.n));
    const f3 st = y.p + (y.n * 1e-4f) * signum(dot(wi_y, y.n));
    const f3 sd = st - so;
    const float sdist = length(sd);
    if (sdist < 1e-6f) return;
    const Onb& oz = cs.oz;
    const MatView& mz = cs.mz;
    const f3& wo_zl = cs.wo_zl;
    const f3 f_z = bsdf_eval_ool(mz, to_local(oz, wi_z), wo_zl);
    if (is_zero(f_z)) return;
    f3 f_y = mk(1.f, 1.f, 1.f);
    Onb oy;
    MatView my;
    f3 wo_yl = mk(0.f, 0.f, 0.f);
    if (t != 1) {
        oy = onb_from_normal(y.n);
        my = vtx_mat(P, J, y, 1, t - 1, si);
        const Vtx yp = load_vtx(P, 1, t - 2, si);
        wo_yl = to_local(oy, normalize(yp.p - y.p));
        f_y = bsdf_eval_ool(my, to_local(oy, wi_y), wo_yl);
    }
    if (is_zero(f_y)) return;
    const float g = geometry_term(z.p, z.n, y.p, y.n);
    f3 c;
    if (t == 1) {
        const LightView L = load_light(J.sc, y.index);
        if (L.kind == AR_LIGHT_POINT) {
            // :951-967 — re-sample the point light toward z
            f3 lwi, lrad;
            float ldist, lpdf;
            if (!light_sample(L, z.p, 0.f, 0.f, lwi, ldist, lrad, lpdf)) return;
            const f3 f_direct = bsdf_eval_ool(mz, to_local(oz, lwi), wo_zl);
            c = ((z.thr * f_direct) * fabsf(dot(z.n, lwi))) * lrad;
        } else {
            if (dot(y.n, wi_y) <= 0.f) return;
            c = ((z.thr * f_z) * g) * y.thr;
        }
    } else {
        c = (((z.thr * f_z) * g) * f_y) * y.thr;
    }
    if (max3(c) <= 0.f) return;
    float pdf_cc;
    if (t == 1) {
        const LightView L = load_light(J.sc, y.index);
        pdf_cc = pdf_sa_to_area(light_pdf_emission_dir(L, normalize(z.p - y.p)), y.p, z.p, z.n);
    } else {
        const f3 wiy = normalize(z.p - y.p);
        pdf_cc = pdf_sa_to_area(bsdf_pdf_ool(my, to_local(oy, wiy), wo_yl), y.p, z.p, z.n);
    }
    const float pdf_cl = pdf_sa_to_area(bsdf_pdf_ool(mz, to_local(oz, normalize(y.p - z.p)), wo_zl), z.p, y.p, y.n);
    const float w = mis_weight_cached(P, J, mc, si, S, T, s, t, pdf_cc, pdf_cl, lpt);
    push_shadow(P, job, so, normalize(sd / sdist), sdist * (1.0f - 1e-4f), c * w, pix);
}

// connect_bdpt_s1 (:1051-1155): light tracing to the pinhole, splatted.
__device__ void connect_s1(const BdParams& P, const BdJob& J, uint32_t job, uint32_t si, uint32_t S, uint32_t T, const MisCache& mc, bool lpt,
                           uint32_t t) {
    const Vtx y = load_vtx(P, 1, t - 1, si);
    if (y.type == kTypeSurface && y.delta) return;
    // PinholeCamera::sample_we (src/cameras.rs:175-240)
    const f3 co = ld3(J.cam.o);
    const f3 to_cam0 = co - y.p;
    const float d2 = dot(to_cam0, to_cam0);
    const float dist = sqrtf(d2);
    if (dist < 1e-6f) return;
    const f3 wi = to_cam0 / dist;
    const f3 dir = -wi;
    const float ct = dot(dir, ld3(J.cam.fwd));
    if (ct <= 1e-6f) return;
    const f3 ds = dir / ct;
    const float u = dot(ds, ld3(J.cam.right)) / J.cam.vw + 0.5f;
    const float v = dot(ds, ld3(J.cam.up)) / J.cam.vh + 0.5f;
    if (u < 0.f || u > 1.f || v < 0.f || v > 1.f) return;
    const float px = u * float(J.width);
    const float py = (1.0f - v) * float(J.height);
    if (px < 0.f || px >= float(J.width) || py < 0.f || py >= float(J.height)) return;
    const float c2 = ct * ct, c4 = c2 * c2;
    const float we = 1.0f / (J.cam.area * c4);
    const Onb oy = onb_from_normal(y.n);
    const MatView my = vtx_mat(P, J, y, 1, t - 1, si);
    const Vtx yp = load_vtx(P, 1, t - 2, si);
    const f3 wo_yl = to_local(oy, normalize(yp.p - y.p));
    const f3 f_y = bsdf_eval_ool(my, to_local(oy, wi), wo_yl);
    if (is_zero(f_y)) return;
    const float gf = fabsf(dot(y.n, wi)) / (dist * dist);
    const f3 c = ((y.thr * f_y) * gf) * we;
    if (max3(c) <= 0.f) return;
    const Vtx z0 = load_vtx(P, 0, 0, si);
    const float pdf_cl = pdf_sa_to_area(bsdf_pdf_ool(my, to_local(oy, wi), wo_yl), y.p, co, z0.n);
    const float w = mis_weight_cached(P, J, mc, si, S, T, 1, t, 0.f, pdf_cl, lpt);
    const uint32_t ix = min(uint32_t(px), J.width - 1), iy = min(uint32_t(py), J.height - 1);
    const f3 o = y.p + (y.n * 1e-4f) * signum(dot(wi, y.n));
    push_shadow(P, job, o, normalize(wi), dist * (1.0f - 1e-4f), c * w, iy * J.width + ix);
}

// Counting sort of the batch samples by their subpath lengths (S, T), so the
// warps of the connection kernel run strategy loops of equal trip counts.
__device__ __forceinline__ uint32_t bd_sort_key(const BdParams& P, uint32_t si) {
    const uint32_t S = P.nv[si], T = P.nv[P.cap + si];
    return min(S, 15u) * 16u + min(T, 15u);
}

__global__ void __launch_bounds__(256) k_bd_hist(BdParams P) {
    __shared__ uint32_t h[kBdBins];
    const uint32_t ns = P.dyn[0];
    h[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t si = blockIdx.x * 256 + threadIdx.x; si < ns; si += gridDim.x * 256)
        atomicAdd(&h[bd_sort_key(P, si)], 1u);
    __syncthreads();
    if (h[threadIdx.x]) atomicAdd(&P.counts[kBdHist + threadIdx.x], h[threadIdx.x]);
}

__global__ void __launch_bounds__(256) k_bd_scan(BdParams P) {
    __shared__ uint32_t h[kBdBins];
    h[threadIdx.x] = P.counts[kBdHist + threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (uint32_t k = 0; k < kBdBins; ++k) {
            const uint32_t c = h[k];
            h[k] = acc;
            acc += c;
        }
    }
    __syncthreads();
    P.counts[kBdOffs + threadIdx.x] = h[threadIdx.x];
}

// Chunks of 256 samples, one chunk per block at a time (the loop trip count is
// the same for every thread of a block, so the barriers are uniform).
__global__ void __launch_bounds__(256) k_bd_scatter(BdParams P) {
    __shared__ uint32_t h[kBdBins], base[kBdBins];
    const uint32_t ns = P.dyn[0];
    for (uint32_t chunk = blockIdx.x * 256; chunk < ns; chunk += gridDim.x * 256) {
        h[threadIdx.x] = 0;
        __syncthreads();
        const uint32_t si = chunk + threadIdx.x;
        const bool live = si < ns;
        uint32_t key = 0, rank = 0;
        if (live) {
            key = bd_sort_key(P, si);
            rank = atomicAdd(&h[key], 1u);
        }
        __syncthreads();
        if (h[threadIdx.x]) base[threadIdx.x] = atomicAdd(&P.counts[kBdOffs + threadIdx.x], h[threadIdx.x]);
        __syncthreads();
        if (live) P.order[base[key] + rank] = si;
        __syncthreads();
    }
}

// Copies every sample's vertices to its sorted position oi (reads scattered,
// writes coalesced), so k_bd_connect, whose thread oi handles sample
// order[oi], reads vertex k of 32 consecutive samples as one contiguous block.
// One thread per (depth k, position oi), oi fastest: a warp copies depth k of
// 32 consecutive positions, and many independent copies are in flight.
__global__ void __launch_bounds__(256) k_bd_permute(BdParams P) {
    const uint32_t ns = P.dyn[0];
    const uint64_t total = uint64_t(ns) * P.maxv;
    for (uint64_t w = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; w < total;
         w += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t k = uint32_t(w / ns), oi = uint32_t(w - uint64_t(k) * ns);
        const uint32_t si = P.order[oi];
        for (uint32_t sub = 0; sub < 2; ++sub) {
            if (k >= P.nv[sub * P.cap + si]) continue;
            const size_t from = vidx(P, sub, k, si), to = vidx(P, sub, k, oi);
            P.sva[to] = P.va[from];
            P.svb[to] = P.vb[from];
            const float4 c = P.vc[from];
            P.svc[to] = c;
            if ((__float_as_uint(c.w) >> 28) & 1u) P.svuv[to] = P.vuv[from];  // textured vertices only
        }
    }
}

// One thread per sample: the MIS prefix sums are built once, then the
// strategies run camera-vertex-major so each z's frame is computed once.
__global__ void __launch_bounds__(128) k_bd_connect(BdParams P) {
    // P.va/vb/vc are the sorted copies here (see bdpt_run_batch): vertex
    // records of sample order[oi] are read at index oi; the per-sample arrays
    // (job, lengths, global index) stay indexed by the sample itself.
    const uint32_t ns = P.dyn[0];
    for (uint32_t oi = blockIdx.x * blockDim.x + threadIdx.x; oi < ns; oi += gridDim.x * blockDim.x) {
        const uint32_t si = P.order[oi];
        const uint32_t job = P.sjob[si];
        const BdJob& J = P.jobs[job];
        const uint32_t S = P.nv[si], T = P.nv[P.cap + si];
        const uint32_t pix = uint32_t(P.sindex[si] % (J.width * J.height));
        const uint32_t limit = J.max_depth + 2;
        MisCache mc;
        build_mis_cache(P, J, oi, S, T, mc);
        bool lpt = false;
        if (T >= 1) lpt = J.sc.lights[load_vtx(P, 1, 0, oi).index].kind == AR_LIGHT_POINT;
        if (S >= 1)
            for (uint32_t t = 2; t <= T && 1 + t <= limit; ++t) connect_s1(P, J, job, oi, S, T, mc, lpt, t);
        for (uint32_t s = 2; s <= S; ++s) {
            const CamSide cs = cam_side(P, J, oi, s);
            for (uint32_t t = 0; t <= T && s + t <= limit; ++t) connect_general(P, J, job, oi, S, T, mc, lpt, cs, s, t, pix);
        }
    }
}

__global__ void AR_TRAVERSAL_BOUNDS k_bd_shadow(const __grid_constant__ BdParams P, int* err) {
    const uint32_t n = min(P.counts[64], P.sh_cap);
    run_traversal<true>(
        &P.counts[kBdShadowCursor], n, err,
        [&](uint32_t m, const DevScene*& s, Ray& r) {
            const float4 a = ld_once(P.sh_o + m), d = ld_once(P.sh_d + m);
            s = &P.jobs[ld_once(P.sh_job + m)].sc;
            r = Ray{mk(a.x, a.y, a.z), mk(d.x, d.y, d.z), 0.f, d.w};
        },
        [&](uint32_t m, const HitRec& h) {
            if (h.slot == kInvalid) {
                const BdJob& J = P.jobs[ld_once(P.sh_job + m)];
                const float4 c = ld_once(P.sh_c + m);
                film_add(J, __float_as_uint(c.w), mk(c.x, c.y, c.z) * J.inv_spp);
            }
        });
}

__global__ void k_bd_count(const uint32_t* counts, uint32_t max_depth, unsigned long long* stats, int* err) {
    if (threadIdx.x == 0) {
        unsigned long long ext = 0;
        for (uint32_t d = 0; d < max_depth; ++d) ext += counts[d];
        // atomics: batches of one render may run on two streams at once
        atomicAdd(&stats[0], (unsigned long long)counts[0]);
        atomicAdd(&stats[1], ext);
        atomicAdd(&stats[2], (unsigned long long)counts[64]);
        if (counts[65]) atomicExch(err, 4);
    }
}

template <class T>
T* carve(char*& cur, size_t n) {
    cur = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(cur) + 255) & ~uintptr_t(255));
    T* p = reinterpret_cast<T*>(cur);
    cur += n * sizeof(T);
    return p;
}

uint32_t max_pairs_for(uint32_t max_depth) {
    const uint32_t maxv = max_depth + 1;
    uint32_t n = 0;
    for (uint32_t t = 0; t <= maxv; ++t)
        for (uint32_t s = 1; s <= maxv; ++s)
            if (s + t >= 2 && s + t <= max_depth + 2) n++;
    return n;
}

}  // namespace

struct BdptBatcher {
    ar_context* ctx;
    uint32_t max_depth_cap, batch;
    DevBuf mem, jobs_d, seg_d;
    BdParams P{};
    BdJob* jobs_h = nullptr;      // pinned staging
    BdSegment* seg_h = nullptr;   // pinned staging
    uint32_t* dyn_h = nullptr;    // pinned staging: samples, segments of the batch
    uint32_t* dyn_d = nullptr;
    cudaEvent_t staged = nullptr;
    // The stage sequence of a batch captured as one CUDA graph per max depth
    // (the kernels read the batch's size from dyn_d, so a graph serves every
    // batch of that depth), replayed on captured_stream.
    cudaGraphExec_t graphs[63] = {};
    cudaStream_t captured_stream = nullptr;
};

size_t bdpt_batch_bytes(uint32_t max_depth, uint32_t batch) {
    const size_t maxv = max_depth + 1;
    const size_t per_sample = 2 * 2 * maxv * 56 + 2 + 2 * (16 + 4) + 2 * 2 * (32 + 4) + 2 * 20 + 4 + 8 +
                              size_t(max_pairs_for(max_depth)) * 52 + 4;
    return per_sample * batch + 64 * 1024;
}

BdptBatcher* bdpt_create(ar_context* ctx, uint32_t max_depth_cap, uint32_t batch) {
    AR_REQUIRE(max_depth_cap <= 62, AR_ERR_INVALID_ARGUMENT, "BDPT max_depth must be <= 62");
    auto b = std::make_unique<BdptBatcher>();
    b->ctx = ctx;
    b->max_depth_cap = max_depth_cap;
    b->batch = batch;
    b->mem.alloc(bdpt_batch_bytes(max_depth_cap, batch));
    b->jobs_d.alloc(kMaxBdptJobs * sizeof(BdJob));
    b->seg_d.alloc(kMaxBdptJobs * sizeof(BdSegment));
    AR_CUDA(cudaMallocHost(&b->jobs_h, kMaxBdptJobs * sizeof(BdJob)));
    AR_CUDA(cudaMallocHost(&b->seg_h, kMaxBdptJobs * sizeof(BdSegment)));
    AR_CUDA(cudaMallocHost(&b->dyn_h, 4 * sizeof(uint32_t)));
    AR_CUDA(cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming));
    AR_CUDA(cudaEventRecord(b->staged, ctx->stream));
    char* cur = b->mem.as<char>();
    BdParams& P = b->P;
    const uint32_t maxv = max_depth_cap + 1;
    P.maxv = maxv;
    const size_t nvtx = size_t(2) * maxv * batch;
    P.va = carve<float4>(cur, nvtx);
    P.vb = carve<float4>(cur, nvtx);
    P.vc = carve<float4>(cur, nvtx);
    P.vuv = carve<float2>(cur, nvtx);
    P.sva = carve<float4>(cur, nvtx);
    P.svb = carve<float4>(cur, nvtx);
    P.svc = carve<float4>(cur, nvtx);
    P.svuv = carve<float2>(cur, nvtx);
    P.nv = carve<uint8_t>(cur, 2 * size_t(batch));
    P.thr = carve<float4>(cur, 2 * size_t(batch));
    P.dim = carve<uint32_t>(cur, 2 * size_t(batch));
    for (int k = 0; k < 2; ++k) {
        P.ray_o[k] = carve<float4>(cur, 2 * size_t(batch));
        P.ray_d[k] = carve<float4>(cur, 2 * size_t(batch));
        P.qpath[k] = carve<uint32_t>(cur, 2 * size_t(batch));
    }
    P.hit = carve<float4>(cur, 2 * size_t(batch));
    P.hit_inst = carve<uint32_t>(cur, 2 * size_t(batch));
    P.sjob = carve<uint32_t>(cur, batch);
    P.sindex = carve<unsigned long long>(cur, batch);
    P.sh_cap = uint32_t(std::min<uint64_t>(uint64_t(max_pairs_for(max_depth_cap)) * batch, 0xFFFFFFF0ull));
    P.sh_o = carve<float4>(cur, P.sh_cap);
    P.sh_d = carve<float4>(cur, P.sh_cap);
    P.sh_c = carve<float4>(cur, P.sh_cap);
    P.sh_job = carve<uint32_t>(cur, P.sh_cap);
    P.counts = carve<uint32_t>(cur, kBdCounts);
    P.order = carve<uint32_t>(cur, batch);
    b->dyn_d = carve<uint32_t>(cur, 4);
    P.dyn = b->dyn_d;
    P.cap = batch;
    P.jobs = b->jobs_d.as<BdJob>();
    P.seg = b->seg_d.as<BdSegment>();
    return b.release();
}

void bdpt_destroy(BdptBatcher* b) {
    if (!b) return;
    for (auto& g : b->graphs)
        if (g) cudaGraphExecDestroy(g);
    if (b->jobs_h) cudaFreeHost(b->jobs_h);
    if (b->seg_h) cudaFreeHost(b->seg_h);
    if (b->dyn_h) cudaFreeHost(b->dyn_h);
    if (b->staged) cudaEventDestroy(b->staged);
    delete b;
}

uint32_t bdpt_batch_capacity(const BdptBatcher* b) { return b->batch; }
uint32_t bdpt_max_depth_cap(const BdptBatcher* b) { return b->max_depth_cap; }

// The stages of one batch whose jobs reach `max_depth` bounces, on stream
// `s`; grids are sized for the batch capacity (the kernels loop over the
// batch's own size, read from P.dyn).  Returns the number of kernels.
static uint32_t launch_batch(BdptBatcher* b, uint32_t max_depth, cudaStream_t s) {
    ar_context* ctx = b->ctx;
    const BdParams& P = b->P;
    int* err = ctx->err_flag.as<int>();
    const int wide = ctx->num_sms * 8;
    AR_CUDA(cudaMemsetAsync(P.counts, 0, kBdCounts * sizeof(uint32_t), s));
    {
        KernelScope ks(ctx->prof, s, "bdpt_generate");
        k_bd_generate<<<std::max(1, int(std::min<uint64_t>((2ull * b->batch + 255) / 256, wide))), 256, 0, s>>>(P);
    }
    for (uint32_t d = 0; d < max_depth; ++d) {
        {
            KernelScope ks(ctx->prof, s, "bdpt_extend");
            k_bd_extend<<<ctx->num_sms * int(ctx->trav_blocks_per_sm), 128, 0, s>>>(P, d, err);
        }
        {
            KernelScope ks(ctx->prof, s, "bdpt_vertex");
            k_bd_vertex<<<wide, 256, 0, s>>>(P, d);
        }
    }
    const int g = std::max(1, int(std::min<uint64_t>((b->batch + 255) / 256, wide)));
    {
        KernelScope ks(ctx->prof, s, "bdpt_sort");
        k_bd_hist<<<g, 256, 0, s>>>(P);
        k_bd_scan<<<1, 256, 0, s>>>(P);
        k_bd_scatter<<<g, 256, 0, s>>>(P);
    }
    {
        KernelScope ks(ctx->prof, s, "bdpt_permute");
        k_bd_permute<<<g, 256, 0, s>>>(P);
    }
    {
        KernelScope ks(ctx->prof, s, "bdpt_connect");
        BdParams Pc = P;
        Pc.va = P.sva;
        Pc.vb = P.svb;
        Pc.vc = P.svc;
        Pc.vuv = P.svuv;
        k_bd_connect<<<std::max(1, int(std::min<uint64_t>((b->batch + 127) / 128, ctx->num_sms * 16))), 128, 0,
                       s>>>(Pc);
    }
    {
        KernelScope ks(ctx->prof, s, "bdpt_shadow");
        k_bd_shadow<<<ctx->num_sms * int(ctx->trav_blocks_per_sm), 128, 0, s>>>(P, err);
    }
    k_bd_count<<<1, 32, 0, s>>>(P.counts, max_depth, ctx->stats_d.as<unsigned long long>(), err);
    AR_CUDA(cudaGetLastError());
    // generate, (extend, vertex) per depth, hist/scan/scatter, permute,
    // connect, shadow, count
    return 2 * max_depth + 8;
}

uint32_t bdpt_run_batch(BdptBatcher* b, const std::vector<BdJob>& jobs, const std::vector<BdSegment>& segs,
                        cudaStream_t stream) {
    ar_context* ctx = b->ctx;
    cudaStream_t st = stream ? stream : ctx->stream;
    AR_REQUIRE(!segs.empty() && segs.size() <= kMaxBdptJobs && jobs.size() <= kMaxBdptJobs, AR_ERR_INVALID_ARGUMENT,
               "bad BDPT batch");
    uint32_t nsamples = 0, max_depth = 0;
    for (const auto& s : segs) nsamples = std::max(nsamples, s.offset + s.nsamples);
    for (const auto& j : jobs) {
        AR_REQUIRE(j.max_depth <= b->max_depth_cap, AR_ERR_INVALID_ARGUMENT, "job max_depth above the batch capacity");
        max_depth = std::max(max_depth, j.max_depth);
    }
    AR_REQUIRE(nsamples <= b->batch, AR_ERR_INVALID_ARGUMENT, "batch too large");
    AR_CUDA(cudaEventSynchronize(b->staged));  // staging buffers free again
    std::copy(jobs.begin(), jobs.end(), b->jobs_h);
    std::copy(segs.begin(), segs.end(), b->seg_h);
    b->dyn_h[0] = nsamples;
    b->dyn_h[1] = uint32_t(segs.size());
    AR_CUDA(cudaMemcpyAsync(b->jobs_d.ptr, b->jobs_h, jobs.size() * sizeof(BdJob), cudaMemcpyHostToDevice,
                            st));
    AR_CUDA(cudaMemcpyAsync(b->seg_d.ptr, b->seg_h, segs.size() * sizeof(BdSegment), cudaMemcpyHostToDevice,
                            st));
    AR_CUDA(cudaMemcpyAsync(b->dyn_d, b->dyn_h, 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    AR_CUDA(cudaEventRecord(b->staged, st));
    if (ctx->prof.on) return launch_batch(b, max_depth, st);  // per-stage timing
    if (b->captured_stream != st) {
        for (auto& g : b->graphs)
            if (g) cudaGraphExecDestroy(g);
        for (auto& g : b->graphs) g = nullptr;
        b->captured_stream = st;
    }
    cudaGraphExec_t& ge = b->graphs[max_depth];
    if (!ge) {
        cudaGraph_t graph;
        AR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            launch_batch(b, max_depth, st);
        } catch (...) {
            cudaStreamEndCapture(st, &graph);
            throw;
        }
        AR_CUDA(cudaStreamEndCapture(st, &graph));
        const cudaError_t e = cudaGraphInstantiate(&ge, graph, 0);
        cudaGraphDestroy(graph);
        AR_CUDA(e);
    }
    AR_CUDA(cudaGraphLaunch(ge, st));
    return 2 * max_depth + 8;
}

BdJob make_bdpt_job(const ar_scene* sc, const CameraDev& cam, const ar_integrator_cfg& cfg, uint32_t w, uint32_t h,
                    void* film) {
    BdJob J{};
    J.sc = sc->view;
    J.cam = cam;
    J.width = w;
    J.height = h;
    J.spp = cfg.spp;
    J.max_depth = cfg.max_depth;
    J.rr_depth = cfg.rr_depth;
    J.mis_mode = cfg.mis_mode;
    J.mis_beta = cfg.mis_beta;
    J.film64 = cfg.film_precision == AR_FILM_F64 ? 1u : 0u;
    J.seed = cfg.seed;
    J.inv_spp = 1.0f / float(cfg.spp);
    J.film = film;
    return J;
}

// Single-job BDPT render (the plain path): consecutive batches of one job.
void render_bdpt_film(ar_context* ctx, const ar_scene* sc, const CameraDev& cam, const ar_integrator_cfg& cfg,
                      uint32_t w, uint32_t h, void* film) {
    AR_REQUIRE(cfg.max_depth <= 62, AR_ERR_INVALID_ARGUMENT, "max_depth must be <= 62");
    const uint64_t npix = uint64_t(w) * h;
    const uint32_t s0 = ctx->range_end ? ctx->range_begin : 0u, s1 = ctx->range_end ? ctx->range_end : cfg.spp;
    const uint64_t first = npix * s0, total = npix * (s1 - s0);
    const size_t budget = ctx->bdpt_budget;
    const size_t per = bdpt_batch_bytes(cfg.max_depth, 1024) / 1024 + 1;
    const uint32_t batch = uint32_t(std::max<uint64_t>(1024, std::min<uint64_t>(total, budget / per)));
    const auto fits = [&](const BdptBatcher* b) {
        return b && bdpt_max_depth_cap(b) >= cfg.max_depth && bdpt_batch_capacity(b) >= batch;
    };
    if (!fits(ctx->bdpt)) {
        AR_CUDA(cudaStreamSynchronize(ctx->stream));
        bdpt_destroy(ctx->bdpt);
        ctx->bdpt = nullptr;
        ctx->bdpt = bdpt_create(ctx, std::max(cfg.max_depth, 10u), batch);
    }
    const uint32_t cap = bdpt_batch_capacity(ctx->bdpt);
    // Renders of two or more batches alternate them over two lanes (the
    // context stream and a second stream, each with its own batch buffers):
    // one batch's stage tails overlap the other's work.  Profiling keeps one
    // lane so that the per-stage times do not overlap.
    const bool two_lanes = total > cap && !ctx->prof.on;
    if (two_lanes) {
        if (!ctx->lane_stream) {
            AR_CUDA(cudaStreamCreateWithFlags(&ctx->lane_stream, cudaStreamNonBlocking));
            for (cudaEvent_t& e : ctx->lane_ev) AR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        if (!fits(ctx->bdpt2) || bdpt_batch_capacity(ctx->bdpt2) < cap) {
            AR_CUDA(cudaStreamSynchronize(ctx->lane_stream));
            bdpt_destroy(ctx->bdpt2);
            ctx->bdpt2 = nullptr;
            ctx->bdpt2 = bdpt_create(ctx, bdpt_max_depth_cap(ctx->bdpt), cap);
        }
    }
    const bool f64 = cfg.film_precision == AR_FILM_F64;
    AR_CUDA(cudaMemsetAsync(film, 0, size_t(w) * h * 3 * (f64 ? sizeof(double) : sizeof(float)), ctx->stream));
    AR_CUDA(cudaMemsetAsync(ctx->stats_d.ptr, 0, 8 * sizeof(uint64_t), ctx->stream));
    if (two_lanes) {  // fork: the second lane starts after the clears
        AR_CUDA(cudaEventRecord(ctx->lane_ev[0], ctx->stream));
        AR_CUDA(cudaStreamWaitEvent(ctx->lane_stream, ctx->lane_ev[0], 0));
    }
    const std::vector<BdJob> jobs{make_bdpt_job(sc, cam, cfg, w, h, film)};
    uint64_t batches = 0;
    for (uint64_t begin = 0; begin < total; begin += cap, ++batches) {
        const uint32_t n = uint32_t(std::min<uint64_t>(cap, total - begin));
        if (two_lanes && (batches & 1))
            bdpt_run_batch(ctx->bdpt2, jobs, {BdSegment{0, 0, n, 0, first + begin}}, ctx->lane_stream);
        else
            bdpt_run_batch(ctx->bdpt, jobs, {BdSegment{0, 0, n, 0, first + begin}});
    }
    if (two_lanes) {  // join: the context stream waits for the second lane
        AR_CUDA(cudaEventRecord(ctx->lane_ev[1], ctx->lane_stream));
        AR_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->lane_ev[1], 0));
    }
    AR_CUDA(cudaMemcpyAsync(ctx->stats_h, ctx->stats_d.ptr, 8 * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                            ctx->stream));
    ctx->stats_pending = true;
    ctx->last_stats.path_samples = total;
    ctx->last_stats.extend_launches = batches * cfg.max_depth;
    ctx->last_stats.shadow_launches = batches;
}

}  // namespace ar
