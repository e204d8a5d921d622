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
// Node record: 28 floats = 7 float4
//   [0] min.x of children 0..3   [1] max.x   [2] min.y   [3] max.y
//   [4] min.z                    [5] max.z   [6] child codes (int bits)
// child code: >= 0 inner node index (absolute); < 0 leaf: ~((first << 2) | (count - 1)),
// first = absolute triangle index (BLAS, count 1..4) or instance index (TLAS, count 1).
// An empty slot has min = +FLT_MAX, max = -FLT_MAX (no ray hits it).
// Nodes: the TLAS region first (its root is node 0; room for a rebuild over the
// same instances), then every mesh's BLAS. Triangles: 12 floats each, the
// tri_geo record (v0, e1 = v1 - v0, e2 = v2 - v0) the closest-hit walk tests.
#pragma once

#include <string>
#include <vector>

#include "../../../include/hdrestir.h"
#include "../device/sh4_layout.h"

namespace hdr {

struct ShadowBvh {
    std::vector<float> nodes;
    std::vector<float> tris;
    std::vector<int> inst_root;  // per instance: its mesh's BLAS root node, or -1 (no triangles)
    int tlas_capacity = 0;       // nodes reserved for the TLAS at the front of `nodes`
    int tlas_depth = 0, blas_depth = 0;
    bool ok = false;             // false: not built (the scene is walked with the reference trees)
};

// Builds the BLAS of every mesh and the TLAS over the instances' world boxes
// (6 floats per instance: min.xyz, max.xyz; instances whose mesh has no
// triangles are left out). Returns false (and leaves out.ok false) when the
// trees would need more than kSh4Stack stack entries.
bool build_shadow_bvh(const hdr_scene_desc &desc, const std::vector<float> &inst_bounds, ShadowBvh &out,
                      std::string &err);

// Rebuilds the TLAS part of `nodes` (into the first tlas_capacity nodes) over new
// instance boxes; returns false when it does not fit the reserved room or the
// stack bound.
bool rebuild_shadow_tlas(const std::vector<float> &inst_bounds, const std::vector<int> &inst_root, int blas_depth,
                         std::vector<float> &tlas_nodes, int tlas_capacity, int &tlas_depth);

}  // namespace hdr
