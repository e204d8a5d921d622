// Host-side scene preparation: the acceleration structures and tables the
// kernels read, laid out as 16-byte records.
//
// The builders restate the reference's host builders so the device traverses
// the SAME trees in the same order (closest-hit ties resolve identically):
//   BLAS  BVH::Build / _Subdivide           renderContext/bvh.cpp:66-208
//   TLAS  Scene::_BuildTLAS / _SubdivideTLAS scene/scene.cpp:333-407
//   instances (transform, inverse, bounds)   scene/scene.cpp:187-222, 101-116
//   mesh-subset bounds                       hydra/hd_restir_mesh.cpp:523-529
//   dome CDF                                 scene/dome_light.cpp:21-83
#pragma once

#include <stdint.h>
#include <string>
#include <vector>

#include "../../../include/hdrestir.h"
#include "../device/bvh_layout.h"
#include "../device/gf.cuh"
#include "../device/tri_setup.cuh"

namespace hdr {

struct Range3 {  // GfRange3f semantics (default = empty)
    V3 mn{3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    V3 mx{-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    void set_empty() { *this = Range3{}; }
    void extend(V3 p) {
        if (p.x < mn.x) mn.x = p.x;
        if (p.y < mn.y) mn.y = p.y;
        if (p.z < mn.z) mn.z = p.z;
        if (p.x > mx.x) mx.x = p.x;
        if (p.y > mx.y) mx.y = p.y;
        if (p.z > mx.z) mx.z = p.z;
    }
    bool empty() const { return mn.x > mx.x || mn.y > mx.y || mn.z > mx.z; }
    V3 size() const { return mx - mn; }
};

struct BlasNode {  // BVHNode (bvh.h:15-20)
    Range3 bounds;
    int left = 0;
    int count = 0;
};

struct Blas {
    std::vector<BlasNode> nodes;
    std::vector<BlasTriangle> tris;
    Range3 range;  // MeshSubset::range
    int max_depth = 0;
};

struct TlasNode {
    Range3 bounds;
    int left = 0;
    int count = 0;
};

struct HostInstance {
    int mesh = 0, material = -1, light = -1;
    float xf[16];
    float inv[16];
    Range3 bounds;
    V3 centroid;
};

// Flattened device-ready arrays (all float4-sized records, little-endian
// int fields stored bitwise in float slots).
struct FlatScene {
    std::vector<float> blas4;       // wide BLAS nodes, all meshes (node indices relative to the mesh base)
    std::vector<float> blas_roots;  // 8 floats per mesh: root min.xyz, root code | root max.xyz, 0
    std::vector<float> tlas4;       // wide TLAS nodes
    float tlas_root[8] = {};        // root min.xyz, root code | root max.xyz, 0
    int max_blas4_depth = 0, max_tlas4_depth = 0;
    std::vector<float> blas_nodes;  // 8 floats per node: min.xyz,left | max.xyz,count
    std::vector<float> tri_geo;     // 12 floats per tri: v0.xyz,e1.x | e1.yz,e2.xy | e2.z,0,0,0
    std::vector<float> tri_attr;    // 36 floats per tri (see scene_build.cpp)
    std::vector<float> instances;   // 32 floats per instance
    std::vector<float> tlas_nodes;  // 8 floats per node
    std::vector<int> tlas_inst;
    std::vector<float> mesh_ranges; // 6 floats per mesh: MeshSubset::range min.xyz, max.xyz
    std::vector<float> inst_bounds; // 6 floats per instance: world box min.xyz, max.xyz
    std::vector<int> mesh_tri_base, mesh_tri_count;  // per mesh: its triangle records in tri_geo
    std::vector<float> materials;   // kMaterialFloats per material
    std::vector<float> textures;    // every material texture's RGB texels, back to back
    std::vector<float> lights;      // kLightFloats per light
    std::vector<float> dome_pixels, dome_row_cdf, dome_col_cdf;
    int dome_width = 0, dome_height = 0;
    float dome_total_lum = 0.0f;
    int env_light = -1;
    int num_instances = 0, num_lights = 0, num_materials = 0;
    int max_blas_depth = 0, max_tlas_depth = 0;
    size_t num_triangles = 0, num_blas_nodes = 0;
};

constexpr int kMaterialFloats = 48;
constexpr int kLightFloats = 48;

// A mesh's BLAS built elsewhere (the device build): what the instance records need.
struct ExternalBlas {
    int num_nodes = 0, num_tris = 0, max_depth = 0;
};

Range3 mesh_range(const hdr_mesh_desc &mesh);
Blas build_blas(const hdr_mesh_desc &mesh);
// ext (one per mesh, or null): the BLAS trees and triangle records are not built
// here; blas_nodes, tri_geo, tri_attr, blas4 and blas_roots stay empty and the
// instance records take their node and triangle bases from ext's counts.
bool build_flat_scene(const hdr_scene_desc &desc, FlatScene &out, std::string &err,
                      const ExternalBlas *ext = nullptr);

}  // namespace hdr
