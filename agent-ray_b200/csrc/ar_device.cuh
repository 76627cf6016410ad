// Device-side math, sampler and BVH8 traversal for the light-transport kernels.
//
// Parity-critical arithmetic (ray normalisation, instance transforms and the
// Möller–Trumbore test) uses explicitly rounded intrinsics so that no multiply
// is fused into an add: the reference (Rust + glam SSE2) computes these with
// separate roundings, and the closest-hit t/u/v must match it bit for bit.
#pragma once
#include <cfloat>
#include <cstdint>
#include "ar_types.h"

// Traversal kernels: 128 threads, at least 8 blocks per SM (<= 64 registers),
// i.e. half the SM's warps resident to hide node-fetch latency.
#ifndef AR_TRAVERSAL_MIN_BLOCKS
#define AR_TRAVERSAL_MIN_BLOCKS 8
#endif
#define AR_TRAVERSAL_BOUNDS __launch_bounds__(128, AR_TRAVERSAL_MIN_BLOCKS)
// Traversal steps a lane runs between two ray-fetch rounds of its warp.
#ifndef AR_TRAVERSAL_STEPS
#define AR_TRAVERSAL_STEPS 4
#endif
// Resident blocks per SM under AR_TRAVERSAL_BOUNDS: the persistent grid of a ray-fetch launch.
constexpr int kTraversalBlocksPerSm = AR_TRAVERSAL_MIN_BLOCKS;

namespace ar {

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator*(float s, f3 a) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float length(f3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ f3 normalize(f3 a) { return a * (1.0f / length(a)); }
__device__ __forceinline__ float max3(f3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
__device__ __forceinline__ bool is_zero(f3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }

// ---- exactly rounded (no contraction) variants: reference arithmetic order ----
__device__ __forceinline__ f3 sub_rn(f3 a, f3 b) {
    return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}
__device__ __forceinline__ f3 add_rn(f3 a, f3 b) {
    return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)};
}
__device__ __forceinline__ f3 scale_rn(f3 a, float s) {
    return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)};
}
// glam dot3: (x*x' + y*y') + z*z'
__device__ __forceinline__ float dot_rn(f3 a, f3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ f3 cross_rn(f3 a, f3 b) {
    return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
// glam normalize: v * (1 / sqrt(dot(v, v)))
__device__ __forceinline__ f3 normalize_rn(f3 a) {
    return scale_rn(a, __fdiv_rn(1.0f, __fsqrt_rn(dot_rn(a, a))));
}
__device__ __forceinline__ f3 ld3(const float* p) { return {p[0], p[1], p[2]}; }

// Queue records that a stage touches once (batched rays and their hits, shadow
// queues): loaded and stored evict-first, so that streaming them through L2
// does not push out the BVH and the traversal stacks, which every ray reuses
// (measured: closest hit on the 1M-triangle soup +0.5%, BDPT +1.3%).
template <class T>
__device__ __forceinline__ T ld_once(const T* p) {
    return __ldcs(p);
}
template <class T>
__device__ __forceinline__ void st_once(T* p, T v) {
    __stcs(p, v);
}

// ---- counter-based sampler (SplitMix64 finalizer, Steele et al. 2014) ----
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t counter_key(uint64_t seed, uint32_t pixel, uint32_t sample) {
    return mix64(seed ^ mix64((uint64_t(pixel) << 32) | uint64_t(sample)));
}
__device__ __forceinline__ float counter_u01(uint64_t key, uint32_t dim) {
    uint64_t z = mix64(key + uint64_t(dim + 1) * 0x9e3779b97f4a7c15ull);
    return float(uint32_t(z >> 40)) * (1.0f / 16777216.0f);
}
constexpr uint32_t kLightSubpathDim = 4096;

// ---- traversal ----
struct Ray {
    f3 o, d;
    float tmin, tmax;
};

struct HitRec {
    float t, u, v;
    uint32_t slot;  // triangle record index (leaf order), kInvalid on miss
    uint32_t inst;  // SceneObject index
};

// Ray::new applied to a world ray (direction normalised as glam does).
__device__ __forceinline__ Ray make_ray(f3 o, f3 d, float tmin, float tmax) { return {o, normalize_rn(d), tmin, tmax}; }

// Triangle::hit (src/geometry.rs:172-206) with the reference's operation order.
__device__ __forceinline__ bool tri_test(const TriRecord& tr, f3 o, f3 d, float tmin, float tmax, float& t, float& u,
                                         float& v) {
    f3 v0 = mk(tr.v0x, tr.v0y, tr.v0z), e1 = mk(tr.e1x, tr.e1y, tr.e1z), e2 = mk(tr.e2x, tr.e2y, tr.e2z);
    f3 h = cross_rn(d, e2);
    float a = dot_rn(e1, h);
    if (fabsf(a) < 1e-8f) return false;
    float f = __fdiv_rn(1.0f, a);
    f3 s = sub_rn(o, v0);
    float uu = __fmul_rn(f, dot_rn(s, h));
    if (uu < 0.0f || uu > 1.0f) return false;
    f3 q = cross_rn(s, e1);
    float vv = __fmul_rn(f, dot_rn(d, q));
    if (vv < 0.0f || __fadd_rn(uu, vv) > 1.0f) return false;
    float tt = __fmul_rn(f, dot_rn(e2, q));
    if (tt < tmin || tt > tmax) return false;
    t = tt;
    u = uu;
    v = vv;
    return true;
}

__device__ __forceinline__ TriRecord load_tri(const TriRecord* tris, uint32_t i) {
    const float4* p = reinterpret_cast<const float4*>(tris + i);
    float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    TriRecord r;
    r.v0x = a.x; r.v0y = a.y; r.v0z = a.z; r.prim = __float_as_uint(a.w);
    r.e1x = b.x; r.e1y = b.y; r.e1z = b.z; r.object_local = __float_as_uint(b.w);
    r.e2x = c.x; r.e2y = c.y; r.e2z = c.z; r.pad = __float_as_uint(c.w);
    return r;
}

// Per-ray constants of the slab test.
struct RayPre {
    f3 o, inv;
    uint32_t oct;  // bit k set when direction k is negative
    float tmin;
};
__device__ __forceinline__ RayPre precompute(f3 o, f3 d, float tmin) {
    RayPre r;
    r.o = o;
    const float eps = 1e-20f;
    // The reciprocals only cull child boxes, which the builder quantised
    // outward, so the hardware approximation serves (t, u, v and the hit
    // itself come from the exactly rounded triangle test); every parity test
    // gives the same hits, and ray setup and instance entry get cheaper
    // (measured +0.9% closest hit on the soup, +2.4% PT, +1.6% BDPT).
    r.inv.x = __fdividef(1.0f, fabsf(d.x) > eps ? d.x : copysignf(eps, d.x));
    r.inv.y = __fdividef(1.0f, fabsf(d.y) > eps ? d.y : copysignf(eps, d.y));
    r.inv.z = __fdividef(1.0f, fabsf(d.z) > eps ? d.z : copysignf(eps, d.z));
    // the octant follows the reciprocal's sign, -0.0 included (its reciprocal
    // is -1e20): near and far planes must swap exactly when inv is negative
    r.oct = (signbit(d.x) ? 1u : 0u) | (signbit(d.y) ? 2u : 0u) | (signbit(d.z) ? 4u : 0u);
    r.tmin = tmin;
    return r;
}

__device__ __forceinline__ uint32_t byte_of(uint32_t w, uint32_t i) { return (w >> (8 * i)) & 0xffu; }
// Packed pairs of f32 (Blackwell's f32x2 arithmetic: one instruction per
// pair, each half rounded exactly as the scalar instruction would).
__device__ __forceinline__ uint64_t f2_pack(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(uint64_t v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ uint64_t f2_fma(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ uint64_t f2_add(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
// max / min of three (NaN operands ignored, as fmaxf / fminf do)
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
// Byte j of w as the float 2^23 + byte: the bits 0x4B0000qq encode 2^23 + qq,
// and subtracting 2^23 afterwards is exact (a byte-permute and an add
// instead of an I2F).
__device__ __forceinline__ float biased_byte(uint32_t w, uint32_t j) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7650u + j));
}

// Intersects the 8 children of node `ni`.  Outputs the node group (bits 8..15:
// internal-child hits in traversal order i, bits 0..7: imask) and the leaf
// primitive hit mask relative to tri_base.  Each child's six slab distances
// come from three packed multiply-adds, each half the scalar
// fmaf(byte, a, b) of the same operands (measured against the scalar form:
// served-scene traversal stages -2%, two children per pair instead of the
// (x, y) / (near z, far z) pairs used here: -0.3..+0.5%, more spills).
__device__ __forceinline__ void intersect_node(const WideNode* nodes, uint32_t ni, const RayPre& r, float tmax,
                                               uint32_t& child_base, uint32_t& node_bits, uint32_t& tri_base,
                                               uint32_t& tri_bits) {
    const uint4* np = reinterpret_cast<const uint4*>(nodes + ni);
    uint4 w0 = __ldg(np), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
    const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
    const uint32_t ex = w0.w & 0xffu, ey = (w0.w >> 8) & 0xffu, ez = (w0.w >> 16) & 0xffu;
    const uint32_t imask = w0.w >> 24;
    const float ax = __uint_as_float(ex << 23) * r.inv.x;
    const float ay = __uint_as_float(ey << 23) * r.inv.y;
    const float az = __uint_as_float(ez << 23) * r.inv.z;
    const float bx = (px - r.o.x) * r.inv.x;
    const float by = (py - r.o.y) * r.inv.y;
    const float bz = (pz - r.o.z) * r.inv.z;
    // pairs: (x, y) of the near and of the far planes, and (near z, far z)
    const uint64_t AXY = f2_pack(ax, ay), BXY = f2_pack(bx, by), AZZ = f2_pack(az, az), BZZ = f2_pack(bz, bz);
    const uint64_t UNBIAS = f2_pack(-8388608.0f, -8388608.0f);
    child_base = w1.x;
    tri_base = w1.y;
    // near/far plane bytes per axis, chosen by the ray octant
    const bool nx = r.oct & 1u, ny = r.oct & 2u, nz = r.oct & 4u;
    uint32_t nb = 0, tb = 0;
    const float tfar_limit = tmax * 1.0000004f;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const uint32_t meta = half ? w1.w : w1.z;
        const uint32_t lox = half ? w2.y : w2.x, loy = half ? w2.w : w2.z, loz = half ? w3.y : w3.x;
        const uint32_t hix = half ? w3.w : w3.z, hiy = half ? w4.y : w4.x, hiz = half ? w4.w : w4.z;
        const uint32_t nxw = nx ? hix : lox, fxw = nx ? lox : hix;
        const uint32_t nyw = ny ? hiy : loy, fyw = ny ? loy : hiy;
        const uint32_t nzw = nz ? hiz : loz, fzw = nz ? loz : hiz;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float tnx, tny, tfx, tfy, tnz, tfz;
            f2_unpack(f2_fma(f2_add(f2_pack(biased_byte(nxw, j), biased_byte(nyw, j)), UNBIAS), AXY, BXY), tnx, tny);
            f2_unpack(f2_fma(f2_add(f2_pack(biased_byte(fxw, j), biased_byte(fyw, j)), UNBIAS), AXY, BXY), tfx, tfy);
            f2_unpack(f2_fma(f2_add(f2_pack(biased_byte(nzw, j), biased_byte(fzw, j)), UNBIAS), AZZ, BZZ), tnz, tfz);
            const float tn = fmax3(tnx, tny, fmaxf(tnz, r.tmin));
            const float tf = fmin3(tfx, tfy, fminf(tfz, tfar_limit));
            const uint32_t s = uint32_t(half * 4 + j);
            if (tn <= tf) {
                const uint32_t m = byte_of(meta, j);
                if (imask & (1u << s)) {
                    nb |= 1u << (s ^ r.oct);
                } else if (m) {
                    const uint32_t cnt = m >> 5, off = m & 31u;
                    tb |= ((1u << cnt) - 1u) << off;
                }
            }
        }
    }
    node_bits = (nb << 8) | imask;
    tri_bits = tb;
}

// Two-level closest-hit / any-hit traversal (TLAS::intersect + BLASAccel::intersect,
// src/accel/bvh.rs:247-296, :413-447) as a resumable state machine.  One
// stack serves both levels: entering an instance pushes a marker so that
// popping it restores the world ray.  start() loads a ray, step() performs one
// node visit with its leaf tests and the stack work up to the next node, and
// returns true when the ray is done; stack overflow or a runaway loop sets *err and
// ends the ray.  Kernels drive it with dynamic ray fetch (run_traversal
// below): a lane whose ray finishes takes the next ray at once, so a warp is
// not held by its slowest ray.
template <bool kAnyHit>
struct Traverser {
    static constexpr uint32_t kNodeGroup = 0x80000000u, kMarker = 0x40000000u;
    const DevScene* sc;
    // World ray: its direction and t_max; its origin and t_min live in wpre
    // (closest hit, which keeps the world ray's precompute to restore on
    // instance exit) or in wo/wtmin (any hit, which recomputes it).  Inside an
    // instance the local ray is pre.o / ld / pre.tmin.
    f3 wd, wo, ld;
    float wtmin, wtmax;
    RayPre pre, wpre;
    HitRec hit;
    float ds, best_l, bu, bv;
    uint32_t cur_inst, best_l_slot, node, guard;
    uint2 group;
    int sp;
    bool in_blas, visit;

    __device__ __forceinline__ void start(const DevScene* s, const Ray& r) {
        sc = s;
        wd = r.d;
        wtmax = r.tmax;
        if (kAnyHit) {
            wo = r.o;
            wtmin = r.tmin;
        }
        hit.t = r.tmax;
        hit.slot = kInvalid;
        hit.inst = kInvalid;
        hit.u = hit.v = 0.f;
        pre = precompute(r.o, r.d, r.tmin);
        if (!kAnyHit) wpre = pre;
        in_blas = false;
        ds = 1.f;
        cur_inst = kInvalid;
        best_l = bu = bv = 0.f;
        best_l_slot = kInvalid;
        group = make_uint2(0, 0);
        node = s->tlas_root;
        visit = node != kInvalid;
        sp = 0;
        guard = 0;
    }

    // One step = one node visit (with its leaf tests) followed by the stack
    // work that leads to the next node to visit, so every active lane of a
    // warp intersects a node in every step.  Returns true when the ray is
    // finished (or failed: *err set).  `stack` is the caller's local array
    // (kept out of the struct so that the scalar state stays in registers).
    __device__ __forceinline__ bool step(int* err, uint2* stack) {
        if (++guard > (1u << 22)) { atomicExch(err, 3); return true; }
        if (visit) {
            uint32_t cb, nbits, tbase, tbits;
            intersect_node(sc->nodes, node, pre, in_blas ? best_l : (kAnyHit ? wtmax : hit.t), cb, nbits, tbase, tbits);
            group = make_uint2(cb, nbits | kNodeGroup);
            if (tbits) {
                if (in_blas) {
                    while (tbits) {
                        const uint32_t b = __ffs(tbits) - 1;
                        tbits &= tbits - 1;
                        const TriRecord tr = load_tri(sc->tris, tbase + b);
                        float t, u, v;
                        if (tri_test(tr, pre.o, ld, pre.tmin, best_l, t, u, v) && t < best_l) {
                            if (kAnyHit) {
                                if (__fdiv_rn(t, ds) < wtmax) {
                                    hit.t = t;
                                    hit.slot = tbase + b;
                                    hit.inst = cur_inst;
                                    return true;
                                }
                            } else {
                                best_l = t;
                                best_l_slot = tbase + b;
                                bu = u;
                                bv = v;
                            }
                        }
                    }
                } else {
                    // TLAS leaves: resume the node group after the instances.
                    if ((group.y >> 8) & 0xffu) {
                        if (sp >= kTraversalStack) { atomicExch(err, 1); return true; }
                        stack[sp++] = group;
                    }
                    group = make_uint2(0, 0);
                    if (sp >= kTraversalStack) { atomicExch(err, 1); return true; }
                    stack[sp++] = make_uint2(tbase, tbits);  // leaf group (instances)
                }
            }
        }
        // Find the next node: the nearest child of the current group, else
        // pop (node groups, instance exits and entries) until one is found.
        // Every pass pops one entry, so the loop ends within sp passes.
        for (;;) {
            if ((group.y & kNodeGroup) && ((group.y >> 8) & 0xffu)) {
                const uint32_t hits = (group.y >> 8) & 0xffu;
                const uint32_t i = __ffs(hits) - 1;
                const uint32_t s = i ^ pre.oct;
                const uint32_t imask = group.y & 0xffu;
                node = group.x + __popc(imask & ((1u << s) - 1u));
                group.y &= ~(1u << (8 + i));
                if ((group.y >> 8) & 0xffu) {
                    if (sp >= kTraversalStack) { atomicExch(err, 1); return true; }
                    stack[sp++] = group;
                }
                group = make_uint2(0, 0);
                visit = true;
                return false;
            }
            if (sp == 0) {
                visit = false;
                return true;
            }
            const uint2 e = stack[--sp];
            if (e.y & kNodeGroup) {
                group = e;
                continue;
            }
            group = make_uint2(0, 0);
            if (e.y & kMarker) {
                // Leave the instance: convert the local best back to world t.
                if (!kAnyHit && best_l_slot != kInvalid) {
                    const float tw = __fdiv_rn(best_l, ds);
                    if (tw < hit.t) {
                        hit.t = tw;
                        hit.slot = best_l_slot;
                        hit.inst = cur_inst;
                        hit.u = bu;
                        hit.v = bv;
                    }
                }
                in_blas = false;
                // (any-hit recomputes: keeping the copy costs its kernel more than it saves)
                pre = kAnyHit ? precompute(wo, wd, wtmin) : wpre;
                continue;
            }
            // Instance leaf group: enter the next instance.
            uint32_t bits = e.y;
            const uint32_t b = __ffs(bits) - 1;
            bits &= bits - 1;
            if (bits) stack[sp++] = make_uint2(e.x, bits);
            const InstanceRecord* ir = sc->instances + (e.x + b);
            const float4* ip = reinterpret_cast<const float4*>(ir);
            const float4 m0 = __ldg(ip), m1 = __ldg(ip + 1), m2 = __ldg(ip + 2);
            const uint4 m3 = __ldg(reinterpret_cast<const uint4*>(ip + 3));
            if (!m3.z) continue;  // mesh without triangles
            const f3 c0 = mk(m0.x, m0.y, m0.z), c1 = mk(m0.w, m1.x, m1.y), c2 = mk(m1.z, m1.w, m2.x),
                     c3 = mk(m2.y, m2.z, m2.w);
            // glam transform_point3a / transform_vector3a: ((c0*x + c1*y) + c2*z) + c3
            const f3 w_o = kAnyHit ? wo : wpre.o;
            const f3 lo = add_rn(c3, add_rn(add_rn(scale_rn(c0, w_o.x), scale_rn(c1, w_o.y)), scale_rn(c2, w_o.z)));
            const f3 ldu = add_rn(add_rn(scale_rn(c0, wd.x), scale_rn(c1, wd.y)), scale_rn(c2, wd.z));
            const float scale = __fsqrt_rn(dot_rn(ldu, ldu));
            if (scale < FLT_EPSILON) continue;
            ds = scale;
            ld = normalize_rn(ldu);
            const float ltmin = __fmul_rn(kAnyHit ? wtmin : wpre.tmin, ds);
            best_l = __fmul_rn(kAnyHit ? wtmax : hit.t, ds);
            best_l_slot = kInvalid;
            cur_inst = m3.y;
            in_blas = true;
            pre = precompute(lo, ld, ltmin);
            if (sp >= kTraversalStack) { atomicExch(err, 1); return true; }
            stack[sp++] = make_uint2(0, kMarker);
            node = m3.x;
            visit = true;
            return false;
        }
    }
};

// Persistent traversal with dynamic ray fetch.  Every lane of the warp calls
// this (warp-uniform loop).  `counter` hands out ray indices in [0, n) (reset
// to 0 before the launch); load(i, scene, ray) fetches ray i and its scene;
// store(i, hit) writes the result.
template <bool kAnyHit, class Load, class Store>
__device__ __forceinline__ void run_traversal(uint32_t* counter, uint32_t n, int* err, Load load, Store store) {
    Traverser<kAnyHit> tr;
    uint2 stack[kTraversalStack];
    int cur = -1;
    bool more = true;
    const uint32_t lane = threadIdx.x & 31u;
    for (;;) {
        const bool need = more && cur < 0;
        const uint32_t mask = __ballot_sync(0xffffffffu, need);
        if (mask) {
            const int leader = __ffs(mask) - 1;
            uint32_t base = 0;
            if (int(lane) == leader) base = atomicAdd(counter, uint32_t(__popc(mask)));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                const uint32_t idx = base + __popc(mask & ((1u << lane) - 1u));
                if (idx < n) {
                    const DevScene* s;
                    Ray r;
                    load(idx, s, r);
                    tr.start(s, r);
                    cur = int(idx);
                } else {
                    more = false;
                }
            }
        }
        if (!__any_sync(0xffffffffu, cur >= 0)) break;
        if (cur >= 0) {
            for (int k = 0; k < AR_TRAVERSAL_STEPS; ++k) {
                if (tr.step(err, stack)) {
                    store(uint32_t(cur), tr.hit);
                    cur = -1;
                    break;
                }
            }
        }
    }
}

}  // namespace ar
