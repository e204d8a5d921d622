// Shadow-ray BVH (no reference counterpart): a second acceleration structure
// over the same triangles and instances, used only for the query "is there a
// hit nearer than the light" (the visibility test of _evaluateLightSample,
// ris_direct_light_integrator.cpp:628-658, and of the MIS integrator's NEE,
// mis_direct_light_integrator.cpp:140-151).
//
// The answer of that query does not depend on the tree: the reference walks its
// midpoint-split trees and compares the closest hit with the light distance,
// and a hit exists below the limit exactly when some triangle test (the same
// IntersectTriangle arithmetic in the same instance space) returns one. So this
// structure is built for speed: binned-SAH binary trees collapsed to 4 children
// per node, each node holding its children's boxes (tested together, before
// descending), triangles in leaf order. Closest hits keep walking the
// reference-order trees, whose tie-breaks they need.
//
// The same trees answer closest-hit queries with the reference's result: every
// triangle record carries its index in the reference's BLAS triangle order, and
// every instance its position in the reference TLAS's leaf order; among hits at
// equal distance the walk keeps the smallest (instance position, triangle
// index), which is the one the reference's left-first walks find first
// (bvh.cpp:262-304, scene.cpp:414-510, strict `<` on t).
//
// Node record: 28 floats = 7 float4
//   [0] min.x of children 0..3   [1] max.x   [2] min.y   [3] max.y
//   [4] min.z                    [5] max.z   [6] child codes (int bits)
// child code: >= 0 inner node index (absolute); < 0 leaf: ~((first << 2) | (count - 1)),
// first = absolute triangle index (BLAS, count 1..4) or instance index (TLAS, count 1).
// An empty slot has min = +FLT_MAX, max = -FLT_MAX (no ray hits it).
// Nodes: the TLAS region first (its root is node 0; room for a rebuild over the
// same instances), then every mesh's BLAS. Triangles: 12 floats each, the
// tri_geo record (v0, e1 = v1 - v0, e2 = v2 - v0) the reference-order walk
// tests, with float 9 holding (as int bits) the triangle's index in its mesh's
// reference BLAS order.
#pragma once

#include <string>
#include <vector>

#include "../../../include/hdrestir.h"
#include "../device/sh4_layout.h"

namespace hdr {

struct FlatScene;

struct ShadowBvh {
    std::vector<float> nodes;
    std::vector<float> tris;
    std::vector<int> inst_root;  // per instance: its mesh's BLAS root node, or -1 (no triangles)
    std::vector<int> inst_rank;  // per instance: its position in the reference TLAS's leaf order
    int tlas_capacity = 0;       // nodes reserved for the TLAS at the front of `nodes`
    int tlas_depth = 0, blas_depth = 0;
    bool ok = false;             // false: not built (the scene is walked with the reference trees)
};

// Builds the BLAS of every mesh over its triangles in the reference's BLAS order
// (the flat scene's tri_geo records when the host built them, else a host
// build of the reference's tree for the order) and the TLAS over the instances'
// world boxes (instances whose mesh has no triangles are left out). Returns
// false only on error; out.ok stays false when the trees would need more than
// kSh4Stack stack entries.
bool build_shadow_bvh(const hdr_scene_desc &desc, const FlatScene &flat, ShadowBvh &out, std::string &err);

// inst_rank from the reference TLAS's instance order (tlas_inst: instance per leaf slot).
void shadow_ranks(const std::vector<int> &tlas_inst, int num_instances, std::vector<int> &rank);

// Rebuilds the TLAS part of `nodes` (into the first tlas_capacity nodes) over new
// instance boxes; returns false when it does not fit the reserved room or the
// stack bound.
bool rebuild_shadow_tlas(const std::vector<float> &inst_bounds, const std::vector<int> &inst_root, int blas_depth,
                         std::vector<float> &tlas_nodes, int tlas_capacity, int &tlas_depth);

}  // namespace hdr
