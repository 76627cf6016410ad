// ORACLE — test infrastructure only (see ar_math.hpp header; parity unpinned).
// Restates agent-ray's geometry and two-level SAH BVH:
//   Ray::new                     src/geometry.rs:12-20
//   AABB::{surface_area,intersect} src/geometry.rs:54-98
//   Triangle::hit (Möller–Trumbore) src/geometry.rs:172-206
//   BVHNode / sah_split / build_recursive / traverse_bvh   src/accel/bvh.rs:32-296
//   BLASAccel / TLAS / Instance   src/accel/bvh.rs:306-447
//   TriangleMesh BLASPrimitive impl src/primitives/mesh.rs:81-116
#pragma once
#include <algorithm>
#include <numeric>
#include <thread>
#include <vector>
#include "ar_math.hpp"

namespace oracle {

template <class T>
struct Ray {
    V3<T> o, d;
    T tmin, tmax;
    // Ray::new normalises the direction (src/geometry.rs:12-20).
    static Ray make(V3<T> o, V3<T> d, T tmin, T tmax) { return Ray{o, normalize(d), tmin, tmax}; }
    V3<T> at(T t) const { return o + d * t; }
};

struct AabbF {
    V3<float> mn, mx;
    static AabbF empty() {
        return {V3<float>(INFINITY, INFINITY, INFINITY), V3<float>(-INFINITY, -INFINITY, -INFINITY)};
    }
    AabbF uni(const AabbF& b) const { return {vmin(mn, b.mn), vmax(mx, b.mx)}; }
    // src/geometry.rs:54-57
    float surface_area() const {
        V3<float> d = vmax(mx - mn, V3<float>(0.f, 0.f, 0.f));
        return 2.0f * ((d.x * d.y + d.y * d.z) + d.z * d.x);
    }
    V3<float> centroid() const { return (mn + mx) * 0.5f; }
};

// AABB::intersect (src/geometry.rs:86-98) in precision T.
template <class T>
inline bool aabb_intersect(const AabbF& b, const Ray<T>& r) {
    V3<T> inv = V3<T>(T(1), T(1), T(1)) / r.d;
    V3<T> t0 = (V3<T>(b.mn) - r.o) * inv;
    V3<T> t1 = (V3<T>(b.mx) - r.o) * inv;
    V3<T> tminv = vmin(t0, t1);
    V3<T> tmaxv = vmax(t0, t1);
    T tmin = rmax(max_element(tminv), r.tmin);
    T tmax = rmin(min_element(tmaxv), r.tmax);
    return tmin <= tmax;
}

template <class T>
struct Hit {
    uint32_t inst, prim;
    V3<T> n;  // object-space geometric normal
    T u, v, t;
    bool valid;
};

// Triangle::hit (src/geometry.rs:172-206).  v0, e1 = v1 - v0, e2 = v2 - v0.
template <class T>
inline bool triangle_hit(V3<T> v0, V3<T> e1, V3<T> e2, const Ray<T>& r, T tmax, T& t_out, T& u_out, T& v_out) {
    V3<T> h = cross(r.d, e2);
    T a = dot(e1, h);
    if (std::fabs(a) < T(1e-8f)) return false;
    T f = T(1) / a;
    V3<T> s = r.o - v0;
    T u = f * dot(s, h);
    if (u < T(0) || u > T(1)) return false;
    V3<T> q = cross(s, e1);
    T v = f * dot(r.d, q);
    if (v < T(0) || u + v > T(1)) return false;
    T t = f * dot(e2, q);
    if (t < r.tmin || t > tmax) return false;
    t_out = t;
    u_out = u;
    v_out = v;
    return true;
}

struct BNode {
    AabbF box;
    uint32_t left_or_start, right_or_end, count;  // count > 0: leaf
    bool leaf() const { return count > 0; }
};

constexpr size_t kMaxLeafSize = 4;        // src/accel/bvh.rs:58
constexpr int kMaxParallelDepth = 3;      // the reference forks rayon tasks to depth 8; scheduling only

struct BuildResult {
    std::vector<BNode> nodes;
    std::vector<uint32_t> prims;
};

// sah_split (src/accel/bvh.rs:71-150): full sweep of all n-1 splits on the
// three axes after a centroid sort, C_trav = 1, C_isect = 1, leaf cost n.
inline bool sah_split(const std::vector<AabbF>& all, std::vector<uint32_t>& idx, size_t& split_out) {
    const size_t n = idx.size();
    std::vector<AabbF> pa(n);
    for (size_t i = 0; i < n; ++i) pa[i] = all[idx[i]];
    AabbF parent = AabbF::empty();
    for (auto& b : pa) parent = parent.uni(b);
    float parent_sa = parent.surface_area();
    if (parent_sa < FLT_EPSILON) return false;
    const float c_trav = 1.0f;
    float best_cost = float(n);
    int best_axis = -1;
    size_t best_k = 0;
    std::vector<uint32_t> sorted(n);
    std::iota(sorted.begin(), sorted.end(), 0u);
    std::vector<float> cen(n);
    std::vector<AabbF> prefix(n), suffix(n);
    for (int axis = 0; axis < 3; ++axis) {
        for (size_t i = 0; i < n; ++i) cen[i] = pa[i].centroid()[axis];
        std::sort(sorted.begin(), sorted.end(), [&](uint32_t a, uint32_t b) { return cen[a] < cen[b]; });
        prefix[0] = pa[sorted[0]];
        for (size_t i = 1; i < n; ++i) prefix[i] = prefix[i - 1].uni(pa[sorted[i]]);
        suffix[n - 1] = pa[sorted[n - 1]];
        for (size_t i = n - 1; i-- > 0;) suffix[i] = suffix[i + 1].uni(pa[sorted[i]]);
        for (size_t k = 1; k < n; ++k) {
            float cost = c_trav + (prefix[k - 1].surface_area() * float(k) + suffix[k].surface_area() * float(n - k)) / parent_sa;
            if (cost < best_cost) {
                best_cost = cost;
                best_axis = axis;
                best_k = k;
            }
        }
    }
    if (best_axis < 0) return false;
    if (best_axis != 2) {
        for (size_t i = 0; i < n; ++i) cen[i] = pa[i].centroid()[best_axis];
        std::sort(sorted.begin(), sorted.end(), [&](uint32_t a, uint32_t b) { return cen[a] < cen[b]; });
    }
    std::vector<uint32_t> old = idx;
    for (size_t i = 0; i < n; ++i) idx[i] = old[sorted[i]];
    split_out = best_k;
    return true;
}

// build_recursive + merge (src/accel/bvh.rs:157-236): preorder layout, root at
// index 0, left subtree next, then the right subtree; prims in leaf order.
inline BuildResult build_recursive(const std::vector<AabbF>& all, std::vector<uint32_t> idx, int depth) {
    const size_t n = idx.size();
    AabbF box = AabbF::empty();
    for (uint32_t i : idx) box = box.uni(all[i]);
    size_t split = 0;
    bool do_split = n > kMaxLeafSize && sah_split(all, idx, split);
    BuildResult res;
    if (!do_split) {
        res.nodes.push_back({box, 0u, 0u, uint32_t(n)});
        res.prims = std::move(idx);
        return res;
    }
    std::vector<uint32_t> right(idx.begin() + split, idx.end());
    idx.resize(split);
    BuildResult L, R;
    if (depth < kMaxParallelDepth) {
        std::thread th([&] { L = build_recursive(all, std::move(idx), depth + 1); });
        R = build_recursive(all, std::move(right), depth + 1);
        th.join();
    } else {
        L = build_recursive(all, std::move(idx), depth + 1);
        R = build_recursive(all, std::move(right), depth + 1);
    }
    const uint32_t lnodes = uint32_t(L.nodes.size());
    const uint32_t lprims = uint32_t(L.prims.size());
    res.nodes.reserve(1 + L.nodes.size() + R.nodes.size());
    res.nodes.push_back({box, 1u, 1u + lnodes, 0u});
    for (auto nd : L.nodes) {
        if (nd.leaf()) nd.left_or_start += 0;
        else { nd.left_or_start += 1; nd.right_or_end += 1; }
        res.nodes.push_back(nd);
    }
    for (auto nd : R.nodes) {
        if (nd.leaf()) nd.left_or_start += lprims;
        else { nd.left_or_start += 1 + lnodes; nd.right_or_end += 1 + lnodes; }
        res.nodes.push_back(nd);
    }
    res.prims = std::move(L.prims);
    res.prims.insert(res.prims.end(), R.prims.begin(), R.prims.end());
    return res;
}

inline BuildResult build_bvh(const std::vector<AabbF>& boxes) {
    if (boxes.empty()) return {};
    std::vector<uint32_t> idx(boxes.size());
    std::iota(idx.begin(), idx.end(), 0u);
    return build_recursive(boxes, std::move(idx), 0);
}

struct TraversalStats {
    uint64_t nodes = 0;      // nodes popped and AABB-tested
    uint64_t tris = 0;       // triangle tests
    uint64_t instances = 0;  // instance (TLAS leaf) entries
};

// traverse_bvh (src/accel/bvh.rs:247-296): stack[64], pop, AABB test against the
// current best t, leaf loop accepting only strictly closer hits, push right
// then left (no near-first ordering).
template <class T, class LeafFn>
inline Hit<T> traverse(const std::vector<BNode>& nodes, const std::vector<uint32_t>& prims, const Ray<T>& ray,
                       LeafFn&& leaf, TraversalStats* st) {
    Hit<T> best{};
    best.valid = false;
    if (nodes.empty()) return best;
    uint32_t stack[64];
    int sp = 0;
    T tmax = ray.tmax;
    stack[sp++] = 0;
    while (sp > 0) {
        const BNode& nd = nodes[stack[--sp]];
        if (st) st->nodes++;
        Ray<T> probe = ray;
        probe.tmax = tmax;
        if (!aabb_intersect(nd.box, probe)) continue;
        if (nd.leaf()) {
            for (uint32_t i = nd.left_or_start; i < nd.left_or_start + nd.count; ++i) {
                Hit<T> h = leaf(prims[i], tmax);
                if (h.valid && h.t < tmax) {
                    tmax = h.t;
                    best = h;
                }
            }
        } else {
            if (sp + 2 > 64) break;  // debug_assert in the reference
            stack[sp++] = nd.right_or_end;
            stack[sp++] = nd.left_or_start;
        }
    }
    return best;
}

// A mesh with its BLAS (BLASAccel::build over TriangleMesh, bvh.rs:326-344).
template <class T>
struct MeshBlas {
    std::vector<V3<T>> pos;
    std::vector<V3<T>> nrm;  // empty if absent
    std::vector<V2<T>> uv;   // tex_coords, empty if absent
    std::vector<uint32_t> idx;
    std::vector<uint32_t> slots;
    BuildResult bvh;
    AabbF overall;

    uint32_t ntri() const { return uint32_t(idx.size() / 3); }
    void build() {
        std::vector<AabbF> boxes(ntri());
        for (uint32_t p = 0; p < ntri(); ++p) {
            // primitive_aabb is computed on the f32 positions (mesh.rs:81-94)
            V3<float> v0(pos[idx[3 * p]]), v1(pos[idx[3 * p + 1]]), v2(pos[idx[3 * p + 2]]);
            boxes[p] = {vmin(vmin(v0, v1), v2), vmax(vmax(v0, v1), v2)};
        }
        bvh = build_bvh(boxes);
        overall = bvh.nodes.empty() ? AabbF::empty() : bvh.nodes[0].box;
    }
    // intersect_primitive (mesh.rs:96-116)
    Hit<T> intersect_prim(uint32_t p, const Ray<T>& r, T tmax) const {
        Hit<T> h{};
        h.valid = false;
        V3<T> v0 = pos[idx[3 * p]], v1 = pos[idx[3 * p + 1]], v2 = pos[idx[3 * p + 2]];
        V3<T> e1 = v1 - v0, e2 = v2 - v0;
        T t, u, v;
        if (!triangle_hit(v0, e1, e2, r, tmax, t, u, v)) return h;
        h.valid = true;
        h.inst = 0;
        h.prim = p;
        h.n = normalize(cross(e1, e2));
        h.u = u;
        h.v = v;
        h.t = t;
        return h;
    }
    Hit<T> intersect(const Ray<T>& r, TraversalStats* st) const {
        return traverse(bvh.nodes, bvh.prims, r, [&](uint32_t p, T tm) {
            if (st) st->tris++;
            return intersect_prim(p, r, tm);
        }, st);
    }
};

// AABB::transform (src/geometry.rs:66-84) of the BLAS box by the f32 transform.
inline AabbF transform_aabb(const AabbF& b, const Mat4<float>& m) {
    V3<float> cs[8] = {
        {b.mn.x, b.mn.y, b.mn.z}, {b.mx.x, b.mn.y, b.mn.z}, {b.mn.x, b.mx.y, b.mn.z}, {b.mx.x, b.mx.y, b.mn.z},
        {b.mn.x, b.mn.y, b.mx.z}, {b.mx.x, b.mn.y, b.mx.z}, {b.mn.x, b.mx.y, b.mx.z}, {b.mx.x, b.mx.y, b.mx.z}};
    AabbF r = AabbF::empty();
    for (auto& c : cs) {
        V3<float> tc = m.transform_point(c);
        r.mn = vmin(r.mn, tc);
        r.mx = vmax(r.mx, tc);
    }
    return r;
}

}  // namespace oracle
