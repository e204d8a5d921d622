// Reference scene prims from an hdr_scene_desc — TEST INFRASTRUCTURE.
//
// What the Hydra prims hand the reference's Scene, made from a scene description
// the way the render delegate would: one mesh subset per instance (its BVH built
// by the reference's BVH::Build from the mesh's arrays, as HdRestirMesh does,
// hydra/hd_restir_mesh.cpp:505-531), PreviewSurfaceParams per material (textures
// registered in the HioImage stand-in under a path the material names),
// LightFactoryInput per light. The calls go to a sink with Scene's input
// methods (the reference's Scene, or a scene hand-off forwarding to one).
#pragma once

#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "../include/hdrestir.h"
#include "light_factory.h"
#include "preview_surface_params.h"
#include "pxr/imaging/hio/image.h"
#include "sceneInterface/mesh.h"

namespace refprims {

using namespace Restir;

class RefMesh final : public IMesh {
  public:
    VtVec3fArray points, colors, normals;
    VtVec2fArray uvs;
    std::vector<MeshSubset> subsets;
    GfMatrix4f transform{1.0f};
    SdfPath id, instancer;
    const VtVec3fArray &GetPoints() const override { return points; }
    const GfMatrix4f &GetTransform() const override { return transform; }
    bool IsVisible() const override { return true; }
    const VtVec3fArray &GetColors() const override { return colors; }
    const VtVec2fArray &GetUVs() const override { return uvs; }
    const VtVec3fArray &GetNormals() const override { return normals; }
    const std::vector<MeshSubset> &GetSubsets() const override { return subsets; }
    const SdfPath &GetInstancerId() const override { return instancer; }
    const SdfPath &GetId() const override { return id; }
};

inline std::string path_of(const char *prefix, int i) {
    char b[64];
    std::snprintf(b, sizeof(b), "/%s%08d", prefix, i);
    return b;
}

struct RefPrims {
    std::vector<std::unique_ptr<RefMesh>> meshes;
    std::string error;
};

// Hands the prims of `d` to `sink` (AddMesh, SetMaterialParams, SetLightFactoryInput),
// naming them "/mesh%08d", "/mat%08d", "/light%08d" so SdfPath order is index order.
// Returns false (prims.error set) for what the harness does not model.
template <class Sink>
bool Populate(const hdr_scene_desc *d, Sink &sink, RefPrims &prims) {
    // one reference BVH per desc mesh, copied into every instance subset
    std::vector<MeshSubset> protos((size_t)d->num_meshes);
    std::vector<VtVec3fArray> proto_points((size_t)d->num_meshes), proto_normals((size_t)d->num_meshes),
        proto_colors((size_t)d->num_meshes);
    std::vector<VtVec2fArray> proto_uvs((size_t)d->num_meshes);
    for (int mi = 0; mi < d->num_meshes; ++mi) {
        const hdr_mesh_desc &m = d->meshes[mi];
        VtVec3fArray pts((size_t)m.num_points);
        for (int i = 0; i < m.num_points; ++i) pts[i] = GfVec3f(m.points[3 * i], m.points[3 * i + 1], m.points[3 * i + 2]);
        VtVec3iArray idx((size_t)m.num_triangles);
        for (int i = 0; i < m.num_triangles; ++i) idx[i] = GfVec3i(m.indices[3 * i], m.indices[3 * i + 1], m.indices[3 * i + 2]);
        VtVec2fArray uvs((size_t)m.num_uvs);
        for (int i = 0; i < m.num_uvs; ++i) uvs[i] = GfVec2f(m.uvs[2 * i], m.uvs[2 * i + 1]);
        VtVec3fArray nrm((size_t)m.num_normals), col((size_t)m.num_colors);
        for (int i = 0; i < m.num_normals; ++i) nrm[i] = GfVec3f(m.normals[3 * i], m.normals[3 * i + 1], m.normals[3 * i + 2]);
        for (int i = 0; i < m.num_colors; ++i) col[i] = GfVec3f(m.colors[3 * i], m.colors[3 * i + 1], m.colors[3 * i + 2]);
        MeshSubset &s = protos[mi];
        s.indices = idx;
        // HdRestirMesh::_rebuildSubsetsIfNeeded (hydra/hd_restir_mesh.cpp:516-531)
        if (!idx.empty() && !pts.empty()) {
            s.bvh.Build(pts, idx, uvs, nrm, col, std::vector<int>());
            s.range.SetEmpty();
            for (const auto &t : idx) {
                s.range.ExtendBy(pts[t[0]]);
                s.range.ExtendBy(pts[t[1]]);
                s.range.ExtendBy(pts[t[2]]);
            }
        }
        proto_points[mi] = pts;
        proto_uvs[mi] = uvs;
        proto_normals[mi] = nrm;
        proto_colors[mi] = col;
    }
    for (int k = 0; k < d->num_materials; ++k) {
        const hdr_material_desc &p = d->materials[k];
        PreviewSurfaceParams q;
        q.DiffuseColor = GfVec3f(p.diffuse_color[0], p.diffuse_color[1], p.diffuse_color[2]);
        q.Metallic = p.metallic;
        q.Roughness = p.roughness;
        q.SpecularColor = GfVec3f(p.specular_color[0], p.specular_color[1], p.specular_color[2]);
        q.Specular = p.specular;
        q.Opacity = p.opacity;
        q.Ior = p.ior;
        q.Transmission = p.transmission;
        q.TransmissionColor = GfVec3f(p.transmission_color[0], p.transmission_color[1], p.transmission_color[2]);
        q.TransmissionDepth = p.transmission_depth;
        q.TransmissionScatter = GfVec3f(p.transmission_scatter[0], p.transmission_scatter[1], p.transmission_scatter[2]);
        q.EmissionColor = GfVec3f(p.emission_color[0], p.emission_color[1], p.emission_color[2]);
        q.Emission = p.emission;
        q.Coat = p.coat;
        q.CoatColor = GfVec3f(p.coat_color[0], p.coat_color[1], p.coat_color[2]);
        q.CoatRoughness = p.coat_roughness;
        q.CoatIor = p.coat_ior;
        q.Sheen = p.sheen;
        q.SheenColor = GfVec3f(p.sheen_color[0], p.sheen_color[1], p.sheen_color[2]);
        q.SheenRoughness = p.sheen_roughness;
        q.Subsurface = p.subsurface;
        q.SubsurfaceColor = GfVec3f(p.subsurface_color[0], p.subsurface_color[1], p.subsurface_color[2]);
        q.ThinWalled = p.thin_walled != 0;
        // textures: registered in the HioImage stand-in under a path the material names; the
        // reference's own ImageTextureSamplerFactory loads them from there
        SdfAssetPath *slots[4] = {&q.DiffuseTexture, &q.MetallicTexture, &q.RoughnessTexture, &q.NormalTexture};
        for (int t = 0; t < 4; ++t) {
            if (!p.textures[t] || p.tex_width[t] <= 0 || p.tex_height[t] <= 0) continue;
            const std::string path = "mem://" + path_of("mat", k) + "/tex" + std::to_string(t);
            HioImage::Register(path, p.tex_width[t], p.tex_height[t], p.textures[t]);
            *slots[t] = SdfAssetPath(path);
        }
        sink.SetMaterialParams(SdfPath(path_of("mat", k)), q);
    }
    for (int i = 0; i < d->num_instances; ++i) {
        const hdr_instance_desc &in = d->instances[i];
        if (in.light >= 0) {
            prims.error = "light-linked geometry is not supported by the reference harness";
            return false;
        }
        auto m = std::make_unique<RefMesh>();
        m->id = SdfPath(path_of("mesh", i));
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) m->transform[r][c] = in.transform[4 * r + c];
        m->points = proto_points[in.mesh];
        m->uvs = proto_uvs[in.mesh];
        m->normals = proto_normals[in.mesh];
        m->colors = proto_colors[in.mesh];
        MeshSubset s = protos[in.mesh];
        s.materialId = in.material >= 0 ? SdfPath(path_of("mat", in.material)) : SdfPath();
        m->subsets.push_back(std::move(s));
        sink.AddMesh(m->id, m.get());
        prims.meshes.push_back(std::move(m));
    }
    for (int k = 0; k < d->num_lights; ++k) {
        const hdr_light_desc &L = d->lights[k];
        LightFactoryInput li;
        li.Id = SdfPath(path_of("light", k));
        li.Type = (LightType)L.type;
        li.Params.Color = GfVec3f(L.color[0], L.color[1], L.color[2]);
        li.Params.Intensity = L.intensity;
        li.Params.Exposure = L.exposure;
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) li.Params.Transform[r][c] = L.transform[4 * r + c];
        li.Params.Width = L.width;
        li.Params.Height = L.height;
        li.Params.ShapingConeAngle = L.shaping_cone_angle;
        li.Params.ShapingConeSoftness = L.shaping_cone_softness;
        if (L.texture && L.tex_width > 0 && L.tex_height > 0) {
            const std::string tex = "mem://" + li.Id.GetString();
            HioImage::Register(tex, L.tex_width, L.tex_height, L.texture);
            li.Params.TextureFile = SdfAssetPath(tex);
        }
        sink.SetLightFactoryInput(li.Id, li);
    }
    return true;
}

}  // namespace refprims
