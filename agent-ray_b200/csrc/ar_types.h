// Device-visible data layout of a scene in HBM (shared by host and device code).
//
// Wide BVH node (80 bytes, five 16-byte words so one node is five coalesced
// 128-bit loads): 8 children with 8-bit quantised boxes on a per-node grid.
//   word0: origin px, py, pz (f32), packed biased exponents ex|ey<<8|ez<<16|imask<<24
//   word1: child_base, tri_base, meta[0..3], meta[4..7]
//   word2: qlo_x[0..7], qlo_y[0..7]
//   word3: qlo_z[0..7], qhi_x[0..7]
//   word4: qhi_y[0..7], qhi_z[0..7]
// Child slot s holds: meta[s] == 0 -> empty; imask bit s set -> internal child
// at child_base + popc(imask & ((1<<s)-1)); otherwise a leaf of
// (meta[s] >> 5) primitives starting at tri_base + (meta[s] & 31).
// Slots are assigned by octant (bit k of s set: child lies on the + side of
// axis k), so traversal visits slot (i ^ ray_octant) for i = 0..7, an
// approximately front-to-back order with no sorting.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define AR_HD __host__ __device__
#else
#define AR_HD
#endif

namespace ar {

struct alignas(16) WideNode {
    float px, py, pz;
    uint32_t exps;  // ex | ey << 8 | ez << 16 | imask << 24
    uint32_t child_base, tri_base;
    uint8_t meta[8];
    uint8_t qlo_x[8], qlo_y[8], qlo_z[8];
    uint8_t qhi_x[8], qhi_y[8], qhi_z[8];
};
static_assert(sizeof(WideNode) == 80, "wide node is 80 bytes");

// Triangle in BLAS leaf order: v0 (w = original prim id bits), e1 = v1 - v0,
// e2 = v2 - v0, precomputed in f32 exactly as Triangle::new does.
struct alignas(16) TriRecord {
    float v0x, v0y, v0z;
    uint32_t prim;
    float e1x, e1y, e1z;
    uint32_t object_local;  // unused padding
    float e2x, e2y, e2z;
    uint32_t pad;
};
static_assert(sizeof(TriRecord) == 48, "triangle record is 48 bytes");

// TLAS leaf entry: world->local transform columns (xyz of c0..c3) + BLAS root.
struct alignas(16) InstanceRecord {
    float c[12];
    uint32_t blas_root;   // node index of the mesh BLAS root
    uint32_t object;      // SceneObject index (RayHit::instance_id)
    uint32_t valid_blas;  // 0 when the mesh has no triangles
    uint32_t pad;
};
static_assert(sizeof(InstanceRecord) == 64, "instance record is 64 bytes");

struct alignas(16) ObjectRecord {
    float nmat[9];        // normal matrix columns (inverse-transpose of the linear part)
    uint32_t mesh;
    uint32_t mat_offset;  // into material_table
    uint32_t num_mats;
};

struct alignas(16) MeshRecord {
    uint32_t idx_offset;   // into indices (3 per triangle, original order)
    uint32_t nrm_offset;   // into normals (3 floats per vertex), 0xFFFFFFFF when absent
    uint32_t slot_offset;  // into material_slots
    uint32_t num_slots;
    uint32_t uv_offset;    // into texcoords (2 floats per vertex), 0xFFFFFFFF when absent
};

struct alignas(16) MaterialRecord {
    uint32_t kind;
    int32_t emitter;
    float albedo[3];
    float f0[3];
    float alpha;
    float eta;  // dielectric interior IOR
    int32_t tex;  // Lambertian albedo texture, -1: constant albedo
    float pad;
};

// ImageTexture (src/texture.rs:65-151) texels [offset, offset + width * height)
// of DevScene::texels, linear RGB, row-major from the top row.
struct TextureRecord {
    uint32_t offset, width, height, pad;
};

struct alignas(16) LightRecord {
    uint32_t kind;
    float area;
    float pad0[2];
    float pos[4];    // point: position;  quad: corner
    float inten[4];  // point: intensity; quad: radiance
    float e1[4], e2[4], n[4];
};

// Read-only view of a device-resident scene, passed by value to kernels.
struct DevScene {
    const WideNode* nodes;
    const TriRecord* tris;
    const InstanceRecord* instances;  // in TLAS leaf order
    const ObjectRecord* objects;
    const MeshRecord* meshes;
    const uint32_t* indices;
    const float* normals;
    const uint32_t* material_slots;
    const uint32_t* material_table;
    const MaterialRecord* materials;
    const LightRecord* lights;
    const float* light_cdf;
    const float* light_pmf;
    const float* texcoords;
    const float4* texels;
    const TextureRecord* textures;
    uint32_t tlas_root;       // 0xFFFFFFFF: empty scene
    uint32_t num_lights;
    uint32_t light_dist;      // ar_light_distribution
    uint32_t num_instances;
};

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr int kTraversalStack = 32;

}  // namespace ar
