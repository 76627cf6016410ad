// Scene upload and acceleration-structure assembly (Scene::new / SceneObject::new,
// src/scene.rs:125-139, :29-35; BLASAccel::build / TLAS::build, src/accel/bvh.rs).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <array>
#include <cstring>
#include <memory>

#include "ar_internal.hpp"

namespace ar {

void DevBuf::alloc(size_t n) {
    free();
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
        ptr = nullptr;
        throw ArError{e == cudaErrorMemoryAllocation ? AR_ERR_OUT_OF_MEMORY : AR_ERR_CUDA,
                      std::string("cudaMalloc: ") + cudaGetErrorString(e)};
    }
    bytes = n;
}

void DevBuf::free() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

void Workspace::ensure(size_t b) {
    if (buf.bytes >= b) return;
    buf.alloc(b + b / 4);
}

namespace {

template <class T>
void upload(DevBuf& d, const std::vector<T>& h) {
    d.alloc(std::max<size_t>(16, h.size() * sizeof(T)));
    if (!h.empty()) AR_CUDA(cudaMemcpy(d.ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
}

struct V3f {
    float x, y, z;
};
inline V3f mulf(V3f a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3f addv(V3f a, V3f b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline float dotf(V3f a, V3f b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3f crossf(V3f a, V3f b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3f col(const float* m, int c) { return {m[4 * c], m[4 * c + 1], m[4 * c + 2]}; }

// glam transform_point3a order: ((c0*x + c1*y) + c2*z) + c3
inline V3f xf_point(const float* m, V3f p) {
    V3f r = mulf(col(m, 0), p.x);
    r = addv(mulf(col(m, 1), p.y), r);
    r = addv(mulf(col(m, 2), p.z), r);
    return addv(col(m, 3), r);
}

void invert4x4(const float* m, float* out) {
    double a[16];
    for (int i = 0; i < 16; ++i) a[i] = m[i];
    double inv[16];
    inv[0] = a[5] * a[10] * a[15] - a[5] * a[11] * a[14] - a[9] * a[6] * a[15] + a[9] * a[7] * a[14] + a[13] * a[6] * a[11] - a[13] * a[7] * a[10];
    inv[4] = -a[4] * a[10] * a[15] + a[4] * a[11] * a[14] + a[8] * a[6] * a[15] - a[8] * a[7] * a[14] - a[12] * a[6] * a[11] + a[12] * a[7] * a[10];
    inv[8] = a[4] * a[9] * a[15] - a[4] * a[11] * a[13] - a[8] * a[5] * a[15] + a[8] * a[7] * a[13] + a[12] * a[5] * a[11] - a[12] * a[7] * a[9];
    inv[12] = -a[4] * a[9] * a[14] + a[4] * a[10] * a[13] + a[8] * a[5] * a[14] - a[8] * a[6] * a[13] - a[12] * a[5] * a[10] + a[12] * a[6] * a[9];
    inv[1] = -a[1] * a[10] * a[15] + a[1] * a[11] * a[14] + a[9] * a[2] * a[15] - a[9] * a[3] * a[14] - a[13] * a[2] * a[11] + a[13] * a[3] * a[10];
    inv[5] = a[0] * a[10] * a[15] - a[0] * a[11] * a[14] - a[8] * a[2] * a[15] + a[8] * a[3] * a[14] + a[12] * a[2] * a[11] - a[12] * a[3] * a[10];
    inv[9] = -a[0] * a[9] * a[15] + a[0] * a[11] * a[13] + a[8] * a[1] * a[15] - a[8] * a[3] * a[13] - a[12] * a[1] * a[11] + a[12] * a[3] * a[9];
    inv[13] = a[0] * a[9] * a[14] - a[0] * a[10] * a[13] - a[8] * a[1] * a[14] + a[8] * a[2] * a[13] + a[12] * a[1] * a[10] - a[12] * a[2] * a[9];
    inv[2] = a[1] * a[6] * a[15] - a[1] * a[7] * a[14] - a[5] * a[2] * a[15] + a[5] * a[3] * a[14] + a[13] * a[2] * a[7] - a[13] * a[3] * a[6];
    inv[6] = -a[0] * a[6] * a[15] + a[0] * a[7] * a[14] + a[4] * a[2] * a[15] - a[4] * a[3] * a[14] - a[12] * a[2] * a[7] + a[12] * a[3] * a[6];
    inv[10] = a[0] * a[5] * a[15] - a[0] * a[7] * a[13] - a[4] * a[1] * a[15] + a[4] * a[3] * a[13] + a[12] * a[1] * a[7] - a[12] * a[3] * a[5];
    inv[14] = -a[0] * a[5] * a[14] + a[0] * a[6] * a[13] + a[4] * a[1] * a[14] - a[4] * a[2] * a[13] - a[12] * a[1] * a[6] + a[12] * a[2] * a[5];
    inv[3] = -a[1] * a[6] * a[11] + a[1] * a[7] * a[10] + a[5] * a[2] * a[11] - a[5] * a[3] * a[10] - a[9] * a[2] * a[7] + a[9] * a[3] * a[6];
    inv[7] = a[0] * a[6] * a[11] - a[0] * a[7] * a[10] - a[4] * a[2] * a[11] + a[4] * a[3] * a[10] + a[8] * a[2] * a[7] - a[8] * a[3] * a[6];
    inv[11] = -a[0] * a[5] * a[11] + a[0] * a[7] * a[9] + a[4] * a[1] * a[11] - a[4] * a[3] * a[9] - a[8] * a[1] * a[7] + a[8] * a[3] * a[5];
    inv[15] = a[0] * a[5] * a[10] - a[0] * a[6] * a[9] - a[4] * a[1] * a[10] + a[4] * a[2] * a[9] + a[8] * a[1] * a[6] - a[8] * a[2] * a[5];
    double det = a[0] * inv[0] + a[1] * inv[4] + a[2] * inv[8] + a[3] * inv[12];
    AR_REQUIRE(det != 0.0 && std::isfinite(det), AR_ERR_INVALID_ARGUMENT, "object transform is singular");
    double id = 1.0 / det;
    for (int i = 0; i < 16; ++i) out[i] = float(inv[i] * id);
}

}  // namespace

void build_scene_accel(ar_scene* s, const ar_accel_opts* o) {
    auto t0 = std::chrono::steady_clock::now();
    s->accel = o ? *o : ar_accel_opts{};
    BuildOptions bo;
    if (o) {
        if (o->max_leaf_size) bo.max_leaf = o->max_leaf_size;
        if (o->sah_bins) bo.bins = o->sah_bins;
        if (o->bvh_width) bo.width = o->bvh_width;
        if (o->sah_node_cost > 0.f) bo.node_cost = o->sah_node_cost;
        bo.threads = o->build_threads;
    }
    std::vector<WideNode> nodes;
    std::vector<TriRecord> tris;
    std::vector<uint32_t> blas_root(s->meshes.size(), kInvalid);
    std::vector<PrimBox> blas_box(s->meshes.size());
    uint32_t max_blas_depth = 0;
    uint64_t blas_nodes = 0;
    for (size_t m = 0; m < s->meshes.size(); ++m) {
        const auto& mh = s->meshes[m];
        if (mh.ntri == 0) continue;
        std::vector<PrimBox> boxes(mh.ntri);
        for (uint32_t p = 0; p < mh.ntri; ++p) {
            const float* v0 = &mh.pos[3 * size_t(mh.idx[3 * size_t(p)])];
            const float* v1 = &mh.pos[3 * size_t(mh.idx[3 * size_t(p) + 1])];
            const float* v2 = &mh.pos[3 * size_t(mh.idx[3 * size_t(p) + 2])];
            for (int k = 0; k < 3; ++k) {
                boxes[p].mn[k] = std::min(std::min(v0[k], v1[k]), v2[k]);
                boxes[p].mx[k] = std::max(std::max(v0[k], v1[k]), v2[k]);
            }
        }
        WideBuild wb = build_wide_bvh(boxes, bo);
        const uint32_t node_off = uint32_t(nodes.size());
        const uint32_t tri_off = uint32_t(tris.size());
        for (auto n : wb.nodes) {
            n.child_base += node_off;
            n.tri_base += tri_off;
            nodes.push_back(n);
        }
        PrimBox all;
        for (int k = 0; k < 3; ++k) { all.mn[k] = INFINITY; all.mx[k] = -INFINITY; }
        for (uint32_t p : wb.prim_order) {
            const float* v0 = &mh.pos[3 * size_t(mh.idx[3 * size_t(p)])];
            const float* v1 = &mh.pos[3 * size_t(mh.idx[3 * size_t(p) + 1])];
            const float* v2 = &mh.pos[3 * size_t(mh.idx[3 * size_t(p) + 2])];
            TriRecord tr{};
            tr.v0x = v0[0]; tr.v0y = v0[1]; tr.v0z = v0[2];
            tr.prim = p;
            tr.e1x = v1[0] - v0[0]; tr.e1y = v1[1] - v0[1]; tr.e1z = v1[2] - v0[2];
            tr.e2x = v2[0] - v0[0]; tr.e2y = v2[1] - v0[1]; tr.e2z = v2[2] - v0[2];
            tr.object_local = uint32_t(m);
            tris.push_back(tr);
            for (int k = 0; k < 3; ++k) {
                all.mn[k] = std::min(all.mn[k], boxes[p].mn[k]);
                all.mx[k] = std::max(all.mx[k], boxes[p].mx[k]);
            }
        }
        blas_root[m] = node_off;
        blas_box[m] = all;
        max_blas_depth = std::max(max_blas_depth, wb.depth);
        blas_nodes += wb.nodes.size();
    }
    // TLAS over the world boxes of objects with non-empty meshes.
    std::vector<PrimBox> inst_boxes;
    std::vector<uint32_t> inst_obj;
    std::vector<std::array<float, 16>> invs(s->objects.size());
    for (size_t i = 0; i < s->objects.size(); ++i) {
        const auto& od = s->objects[i];
        if (od.has_inverse) std::memcpy(invs[i].data(), od.inv_transform, sizeof(float) * 16);
        else invert4x4(od.transform, invs[i].data());
        if (blas_root[od.mesh] == kInvalid) continue;
        const PrimBox& b = blas_box[od.mesh];
        PrimBox w;
        for (int k = 0; k < 3; ++k) { w.mn[k] = INFINITY; w.mx[k] = -INFINITY; }
        for (int c = 0; c < 8; ++c) {
            V3f p{(c & 1) ? b.mx[0] : b.mn[0], (c & 2) ? b.mx[1] : b.mn[1], (c & 4) ? b.mx[2] : b.mn[2]};
            V3f q = xf_point(od.transform, p);
            const float qq[3] = {q.x, q.y, q.z};
            for (int k = 0; k < 3; ++k) { w.mn[k] = std::min(w.mn[k], qq[k]); w.mx[k] = std::max(w.mx[k], qq[k]); }
        }
        inst_boxes.push_back(w);
        inst_obj.push_back(uint32_t(i));
    }
    std::vector<InstanceRecord> inst_rec;
    uint32_t tlas_root = kInvalid, tlas_depth = 0;
    uint64_t tlas_nodes = 0;
    if (!inst_boxes.empty()) {
        // Single-instance TLAS leaves: a hit TLAS leaf group is pushed on the
        // traversal stack with its instance mask in the entry's flag word,
        // whose top two bits mark node groups and instance exits, so a node's
        // instance mask must stay below bit 30 (8 leaves of up to 4 would
        // reach bit 31).  One instance per leaf also tests every instance's
        // own box in its parent's 8-wide node test (measured no slower).
        BuildOptions tbo = bo;
        tbo.max_leaf = 1;
        WideBuild tb = build_wide_bvh(inst_boxes, tbo);
        const uint32_t node_off = uint32_t(nodes.size());
        for (auto n : tb.nodes) {
            n.child_base += node_off;
            nodes.push_back(n);
        }
        tlas_root = node_off;
        tlas_depth = tb.depth;
        tlas_nodes = tb.nodes.size();
        for (uint32_t k : tb.prim_order) {
            const uint32_t obj = inst_obj[k];
            InstanceRecord r{};
            for (int c = 0; c < 4; ++c)
                for (int j = 0; j < 3; ++j) r.c[3 * c + j] = invs[obj][4 * c + j];
            r.blas_root = blas_root[s->objects[obj].mesh];
            r.object = obj;
            r.valid_blas = 1;
            inst_rec.push_back(r);
        }
    }
    const uint32_t worst_stack = tlas_depth + max_blas_depth + 4;
    AR_REQUIRE(worst_stack <= uint32_t(kTraversalStack), AR_ERR_UNSUPPORTED,
               "BVH too deep for the traversal stack (" + std::to_string(worst_stack) + " entries)");
    upload(s->nodes, nodes);
    upload(s->tris, tris);
    upload(s->instances, inst_rec);
    s->view.nodes = s->nodes.as<WideNode>();
    s->view.tris = s->tris.as<TriRecord>();
    s->view.instances = s->instances.as<InstanceRecord>();
    s->view.tlas_root = tlas_root;
    s->view.num_instances = uint32_t(inst_rec.size());
    s->stats.num_blas_nodes = blas_nodes;
    s->stats.num_tlas_nodes = tlas_nodes;
    s->stats.num_instances = inst_rec.size();
    s->stats.max_stack_depth = worst_stack;
    s->stats.build_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void create_scene(ar_context* ctx, const ar_scene_desc* d, ar_scene** out) {
    AR_REQUIRE(ctx && d && out, AR_ERR_INVALID_ARGUMENT, "null argument");
    AR_CUDA(cudaSetDevice(ctx->device));
    auto s = std::make_unique<ar_scene>();
    s->device = ctx->device;
    AR_REQUIRE(d->num_meshes == 0 || d->meshes, AR_ERR_INVALID_ARGUMENT, "meshes is null");
    AR_REQUIRE(d->num_objects == 0 || d->objects, AR_ERR_INVALID_ARGUMENT, "objects is null");
    AR_REQUIRE(d->num_materials > 0 && d->materials, AR_ERR_INVALID_ARGUMENT, "scene needs at least one material");
    AR_REQUIRE(d->num_lights == 0 || d->lights, AR_ERR_INVALID_ARGUMENT, "lights is null");
    AR_REQUIRE(d->num_materials < (1u << 28) && d->num_lights < (1u << 28), AR_ERR_INVALID_ARGUMENT,
               "at most 2^28 - 1 materials and lights (BDPT vertices pack the index in 28 bits)");
    AR_REQUIRE(d->light_distribution <= AR_LIGHT_DIST_POWER, AR_ERR_INVALID_ARGUMENT, "bad light distribution");
    // meshes
    std::vector<uint32_t> indices, slots;
    std::vector<float> normals, texcoords;
    std::vector<MeshRecord> mrec(d->num_meshes);
    uint64_t ntri_total = 0;
    s->meshes.resize(d->num_meshes);
    for (uint32_t m = 0; m < d->num_meshes; ++m) {
        const ar_mesh_desc& md = d->meshes[m];
        AR_REQUIRE(md.num_triangles == 0 || (md.indices && md.positions), AR_ERR_INVALID_ARGUMENT,
                   "mesh " + std::to_string(m) + " lacks positions/indices");
        auto& mh = s->meshes[m];
        mh.ntri = md.num_triangles;
        mh.pos.assign(md.positions, md.positions + 3 * size_t(md.num_vertices));
        mh.idx.assign(md.indices, md.indices + 3 * size_t(md.num_triangles));
        for (uint32_t v : mh.idx)
            AR_REQUIRE(v < md.num_vertices, AR_ERR_INVALID_ARGUMENT, "mesh " + std::to_string(m) + ": index out of range");
        AR_REQUIRE(md.num_material_slots == 1 || md.num_material_slots == md.num_triangles || md.num_material_slots == 0,
                   AR_ERR_INVALID_ARGUMENT, "material_slots must have 1 or num_triangles entries");
        mrec[m].idx_offset = uint32_t(indices.size());
        indices.insert(indices.end(), mh.idx.begin(), mh.idx.end());
        if (md.normals) {
            mh.has_normals = true;
            mrec[m].nrm_offset = uint32_t(normals.size() / 3);
            normals.insert(normals.end(), md.normals, md.normals + 3 * size_t(md.num_vertices));
        } else {
            mrec[m].nrm_offset = kInvalid;
        }
        if (md.tex_coords) {
            mrec[m].uv_offset = uint32_t(texcoords.size() / 2);
            texcoords.insert(texcoords.end(), md.tex_coords, md.tex_coords + 2 * size_t(md.num_vertices));
        } else {
            mrec[m].uv_offset = kInvalid;
        }
        mrec[m].slot_offset = uint32_t(slots.size());
        if (md.num_material_slots == 0 || !md.material_slots) {
            slots.push_back(0);
            mrec[m].num_slots = 1;
        } else {
            slots.insert(slots.end(), md.material_slots, md.material_slots + md.num_material_slots);
            mrec[m].num_slots = md.num_material_slots;
        }
        ntri_total += md.num_triangles;
    }
    // objects
    std::vector<ObjectRecord> orec(d->num_objects);
    std::vector<uint32_t> mat_table;
    s->objects.assign(d->objects, d->objects + d->num_objects);
    for (uint32_t i = 0; i < d->num_objects; ++i) {
        const ar_object_desc& od = d->objects[i];
        AR_REQUIRE(od.mesh < d->num_meshes, AR_ERR_INVALID_ARGUMENT, "object mesh index out of range");
        AR_REQUIRE(od.num_materials > 0 && od.materials, AR_ERR_INVALID_ARGUMENT, "object needs a material table");
        for (uint32_t k = 0; k < od.num_materials; ++k)
            AR_REQUIRE(od.materials[k] < d->num_materials, AR_ERR_INVALID_ARGUMENT, "material index out of range");
        s->objects[i].materials = nullptr;
        // Mat3::from_mat4(t).inverse().transpose() as glam computes it in f32:
        // columns (y x z, z x x, x x y) / det(z . (x x y)).
        V3f x = col(od.transform, 0), y = col(od.transform, 1), z = col(od.transform, 2);
        V3f t0 = crossf(y, z), t1 = crossf(z, x), t2 = crossf(x, y);
        float det = dotf(z, t2);
        float inv_det = 1.0f / det;
        V3f c0 = mulf(t0, inv_det), c1 = mulf(t1, inv_det), c2 = mulf(t2, inv_det);
        float nm[9] = {c0.x, c0.y, c0.z, c1.x, c1.y, c1.z, c2.x, c2.y, c2.z};
        std::memcpy(orec[i].nmat, nm, sizeof(nm));
        orec[i].mesh = od.mesh;
        orec[i].mat_offset = uint32_t(mat_table.size());
        orec[i].num_mats = od.num_materials;
        mat_table.insert(mat_table.end(), od.materials, od.materials + od.num_materials);
    }
    // materials
    s->materials_h.resize(d->num_materials);
    for (uint32_t i = 0; i < d->num_materials; ++i) {
        const auto& m = d->materials[i];
        AR_REQUIRE(m.kind <= AR_MATERIAL_DIELECTRIC, AR_ERR_INVALID_ARGUMENT, "unknown material kind");
        AR_REQUIRE(m.kind != AR_MATERIAL_DIELECTRIC || m.eta > 0.f, AR_ERR_INVALID_ARGUMENT,
                   "dielectric eta must be positive");
        AR_REQUIRE(m.emitter_light < int32_t(d->num_lights), AR_ERR_INVALID_ARGUMENT, "emitter_light out of range");
        if (m.emitter_light >= 0)
            AR_REQUIRE(d->lights[m.emitter_light].kind == AR_LIGHT_QUAD, AR_ERR_INVALID_ARGUMENT,
                       "emitter_light must name a quad light");
        MaterialRecord r{};
        r.kind = m.kind;
        r.emitter = m.emitter_light;
        for (int k = 0; k < 3; ++k) { r.albedo[k] = m.albedo[k]; r.f0[k] = m.f0[k]; }
        r.alpha = std::min(1.0f, std::max(1e-3f, m.roughness));
        r.eta = m.eta;
        AR_REQUIRE(m.albedo_texture < int32_t(d->num_textures), AR_ERR_INVALID_ARGUMENT,
                   "albedo_texture out of range");
        r.tex = m.kind == AR_MATERIAL_LAMBERTIAN ? std::max<int32_t>(m.albedo_texture, -1) : -1;
        s->materials_h[i] = r;
    }
    // lights + distribution (src/lights.rs:171-235)
    s->lights_h.resize(d->num_lights);
    std::vector<float> weights(d->num_lights);
    const float pi = 3.14159265358979323846f;
    for (uint32_t i = 0; i < d->num_lights; ++i) {
        const auto& l = d->lights[i];
        AR_REQUIRE(l.kind <= AR_LIGHT_QUAD, AR_ERR_INVALID_ARGUMENT, "unknown light kind");
        LightRecord r{};
        r.kind = l.kind;
        for (int k = 0; k < 3; ++k) {
            r.pos[k] = l.position[k];
            r.inten[k] = l.intensity[k];
            r.e1[k] = l.edge1[k];
            r.e2[k] = l.edge2[k];
        }
        V3f p;
        if (l.kind == AR_LIGHT_QUAD) {
            V3f c = crossf({l.edge1[0], l.edge1[1], l.edge1[2]}, {l.edge2[0], l.edge2[1], l.edge2[2]});
            r.area = std::sqrt(dotf(c, c));
            AR_REQUIRE(r.area > 0.f, AR_ERR_INVALID_ARGUMENT, "degenerate quad light");
            V3f n = mulf(c, 1.0f / r.area);
            r.n[0] = n.x; r.n[1] = n.y; r.n[2] = n.z;
            p = mulf({l.intensity[0], l.intensity[1], l.intensity[2]}, r.area * pi);
        } else {
            p = mulf({l.intensity[0], l.intensity[1], l.intensity[2]}, 4.0f * pi);
        }
        weights[i] = std::max((0.2126f * p.x + 0.7152f * p.y) + 0.0722f * p.z, 0.0f);
        s->lights_h[i] = r;
    }
    s->light_dist = d->num_lights ? d->light_distribution : AR_LIGHT_DIST_NONE;
    if (s->light_dist == AR_LIGHT_DIST_POWER) {
        const uint32_t n = d->num_lights;
        float total = 0.f;
        for (float w : weights) total += w;
        s->pmf_h.resize(n);
        s->cdf_h.resize(n);
        if (total == 0.0f) {
            float u = 1.0f / float(n);
            for (uint32_t i = 0; i < n; ++i) { s->pmf_h[i] = u; s->cdf_h[i] = float(i + 1) * u; }
        } else {
            float acc = 0.f;
            for (uint32_t i = 0; i < n; ++i) { s->pmf_h[i] = weights[i] / total; acc += s->pmf_h[i]; s->cdf_h[i] = acc; }
            s->cdf_h[n - 1] = 1.0f;
        }
    }
    // ImageTexture::load (src/texture.rs:77-94): sRGB bytes -> linear f32
    AR_REQUIRE(d->num_textures == 0 || d->textures, AR_ERR_INVALID_ARGUMENT, "textures is null");
    std::vector<float4> texels;
    std::vector<TextureRecord> trec(d->num_textures);
    for (uint32_t t = 0; t < d->num_textures; ++t) {
        const ar_texture_desc& td = d->textures[t];
        AR_REQUIRE(td.rgb8 && td.width > 0 && td.height > 0, AR_ERR_INVALID_ARGUMENT, "empty texture");
        AR_REQUIRE(uint64_t(td.width) * td.height < (1ull << 28), AR_ERR_INVALID_ARGUMENT, "texture too large");
        AR_REQUIRE(texels.size() + uint64_t(td.width) * td.height < (1ull << 31), AR_ERR_INVALID_ARGUMENT,
                   "textures too large in total (texel offsets are 32-bit)");
        trec[t] = TextureRecord{uint32_t(texels.size()), td.width, td.height, 0};
        const auto lin = [](uint8_t b) {
            const float x = float(b) / 255.0f;
            return x <= 0.04045f ? x / 12.92f : std::pow((x + 0.055f) / 1.055f, 2.4f);
        };
        for (size_t i = 0; i < size_t(td.width) * td.height; ++i)
            texels.push_back(make_float4(lin(td.rgb8[3 * i]), lin(td.rgb8[3 * i + 1]), lin(td.rgb8[3 * i + 2]), 0.f));
    }
    upload(s->texcoords, texcoords);
    upload(s->texels, texels);
    upload(s->textures, trec);
    upload(s->indices, indices);
    upload(s->normals, normals);
    upload(s->slots, slots);
    upload(s->meshes_d, mrec);
    upload(s->objects_d, orec);
    upload(s->mat_table, mat_table);
    upload(s->materials, s->materials_h);
    upload(s->lights, s->lights_h);
    upload(s->light_cdf, s->cdf_h);
    upload(s->light_pmf, s->pmf_h);
    s->view.objects = s->objects_d.as<ObjectRecord>();
    s->view.meshes = s->meshes_d.as<MeshRecord>();
    s->view.indices = s->indices.as<uint32_t>();
    s->view.normals = s->normals.as<float>();
    s->view.texcoords = s->texcoords.as<float>();
    s->view.texels = s->texels.as<float4>();
    s->view.textures = s->textures.as<TextureRecord>();
    s->view.material_slots = s->slots.as<uint32_t>();
    s->view.material_table = s->mat_table.as<uint32_t>();
    s->view.materials = s->materials.as<MaterialRecord>();
    s->view.lights = s->lights.as<LightRecord>();
    s->view.light_cdf = s->light_cdf.as<float>();
    s->view.light_pmf = s->light_pmf.as<float>();
    s->view.num_lights = d->num_lights;
    s->view.light_dist = s->light_dist;
    s->stats.num_triangles = ntri_total;
    build_scene_accel(s.get(), nullptr);
    size_t bytes = 0;
    for (DevBuf* b : {&s->nodes, &s->tris, &s->instances, &s->objects_d, &s->meshes_d, &s->indices, &s->normals,
                      &s->slots, &s->mat_table, &s->materials, &s->lights, &s->light_cdf, &s->light_pmf,
                      &s->texcoords, &s->texels, &s->textures})
        bytes += b->bytes;
    s->stats.device_bytes = bytes;
    *out = s.release();
}

}  // namespace ar
