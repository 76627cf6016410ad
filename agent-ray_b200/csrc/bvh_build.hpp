// Host-side acceleration-structure builder: binned SAH binary BVH collapsed
// into the 8-wide quantised layout of ar_types.h.
//
// Replaces BLASAccel::build / TLAS::build (src/accel/bvh.rs:326-411).  The
// reference builds a binary full-sweep SAH tree for a scalar CPU traversal;
// here the tree is re-shaped for the GPU (8 children per 80-byte node, leaves
// of at most 3 primitives, octant-ordered slots).  Closest-hit results do not
// depend on tree shape except for exact ties in t.
#pragma once
#include <cstdint>
#include <vector>
#include "ar_types.h"

namespace ar {

struct PrimBox {
    float mn[3], mx[3];
};

struct BuildOptions {
    uint32_t max_leaf = 3;  // 1..4
    uint32_t bins = 32;
    uint32_t threads = 0;   // 0: all hardware threads
    uint32_t width = 8;     // children per wide node, 2..8
    float node_cost = 0.5f; // SAH: a node visit relative to one triangle test
};

struct WideBuild {
    std::vector<WideNode> nodes;      // nodes[0] is the root; child_base/tri_base are build-local
    std::vector<uint32_t> prim_order; // leaf-order primitive ids (tri_base indexes this)
    uint32_t depth = 0;               // number of wide levels
};

// Builds the wide BVH over `boxes`.  An empty input yields an empty build.
WideBuild build_wide_bvh(const std::vector<PrimBox>& boxes, const BuildOptions& opts);

}  // namespace ar
