// Scene hand-off for the reference renderer: the inputs the reference's Scene
// receives (Scene::AddMesh / AddInstancer / SetMaterialParams /
// SetLightFactoryInput, scene/scene.cpp:50-92) turned into the hdr_scene_desc
// that hdr_scene_upload builds the device scene from, in the order
// Scene::BuildRenderState (scene.cpp:118-271) builds its render state:
//   lights     every light input, in SdfPath order (the order of GetLights(), so
//              light-selection indices agree);
//   materials  every PreviewSurfaceParams, in SdfPath order;
//   instances  meshes in SdfPath order, invisible ones skipped; a mesh with an
//              instancer gives one instance per instancer transform and subset
//              (GfMatrix4f(instancer transform) * mesh transform), otherwise one
//              per subset (mesh transform); a subset's material is looked up by
//              its materialId (none: DefaultMaterial). Instance indices are the
//              reference's MeshInstance indices, so PrimId / MatId agree.
// Each distinct (mesh, subset) becomes one hdr_mesh_desc: the mesh's points, the
// subset's triangles and the mesh's uvs / normals / colours (the BVH the
// reference builds for the subset from the same arrays, bvh.cpp:66-179). A mesh
// with several subsets and face-varying primvars keeps per-subset primvar arrays
// inside HdRestirMesh that IMesh does not expose: give them with
// SetSubsetPrimvars, or Build reports the mesh.
//
// Header-only, compiled inside the reference tree next to scene/scene.h. A
// maintainer wraps or replaces the Scene calls of the Hydra prims with these
// (the optional Scene pointer receives every call too), and calls Upload where
// the renderer calls Scene::BuildRenderState.
#pragma once

#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "hdrestir.h"
#include "scene.h"

namespace Restir::B200 {

class SceneHandoff {
  public:
    // Decodes a texture asset to RGB floats as ImageTextureSamplerFactory does
    // (scene/image_texture_sampler.cpp:14-123): linear, or sRGB-decoded when
    // linear is false. Returns false when the asset cannot be read (no texture).
    using TextureLoader =
        std::function<bool(const SdfAssetPath &asset, bool linear, std::vector<float> &rgb, int &width, int &height)>;

    explicit SceneHandoff(Scene *forward = nullptr) : _forward{forward} {}

    void AddMesh(const SdfPath &id, IMesh *mesh) {
        _meshes[id] = mesh;
        if (_forward) _forward->AddMesh(id, mesh);
    }
    void RemoveMesh(const SdfPath &id) {
        _meshes.erase(id);
        if (_forward) _forward->RemoveMesh(id);
    }
    void AddInstancer(const SdfPath &id, IInstancer *instancer) {
        _instancers[id] = instancer;
        if (_forward) _forward->AddInstancer(id, instancer);
    }
    void RemoveInstancer(const SdfPath &id) {
        _instancers.erase(id);
        if (_forward) _forward->RemoveInstancer(id);
    }
    void SetMaterialParams(const SdfPath &id, const PreviewSurfaceParams &params) {
        _materials[id] = params;
        if (_forward) _forward->SetMaterialParams(id, params);
    }
    void RemoveMaterialParams(const SdfPath &id) {
        _materials.erase(id);
        if (_forward) _forward->RemoveMaterialParams(id);
    }
    void SetLightFactoryInput(const SdfPath &id, const LightFactoryInput &input) {
        _lights[id] = input;
        if (_forward) _forward->SetLightFactoryInput(id, input);
    }
    void RemoveLightFactoryInput(const SdfPath &id) {
        _lights.erase(id);
        if (_forward) _forward->RemoveLightFactoryInput(id);
    }
    void SetTextureLoader(TextureLoader loader) { _loader = std::move(loader); }
    // The per-corner (3 per subset triangle) or per-point primvars HdRestirMesh built
    // subset `subset` of mesh `id`'s BVH from; empty arrays fall back to the mesh's own.
    void SetSubsetPrimvars(const SdfPath &id, size_t subset, VtVec2fArray uvs, VtVec3fArray normals,
                           VtVec3fArray colors) {
        _subsetPrimvars[{id, subset}] = Primvars{std::move(uvs), std::move(normals), std::move(colors)};
    }

    // Scene::BuildRenderState: the forward Scene builds its render state, then the
    // descriptor of the same state is built and uploaded to `ctx`.
    void BuildRenderState(const SceneBuildRenderStateConfig &config, const IRenderJob &job, hdr_ctx *ctx) {
        if (_forward) _forward->BuildRenderState(config, job);
        _config = config;
        Upload(ctx);
    }
    void Upload(hdr_ctx *ctx) {
        const hdr_scene_desc &d = Build();
        if (hdr_scene_upload(ctx, &d) != HDR_OK)
            throw std::runtime_error(std::string("[hdrestir-b200] hdr_scene_upload: ") + hdr_last_error());
    }

    // The descriptor of the current inputs; its arrays live in this object until the
    // next Build. Throws std::runtime_error for a mesh whose subset primvars IMesh
    // cannot give (see SetSubsetPrimvars).
    const hdr_scene_desc &Build() {
        _store = std::make_unique<Store>();
        Store &s = *_store;
        // lights: the order of Scene::GetLights() (scene.cpp:158-172)
        std::map<SdfPath, int> light_index;
        s.lights.reserve(_lights.size());
        s.light_texels.reserve(_lights.size());
        for (const auto &[id, in] : _lights) {
            hdr_light_desc L{};
            L.type = static_cast<int32_t>(in.Type);
            for (int k = 0; k < 3; ++k) L.color[k] = in.Params.Color[k];
            L.intensity = in.Params.Intensity;
            L.exposure = in.Params.Exposure;
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c) L.transform[4 * r + c] = in.Params.Transform[r][c];
            L.width = in.Params.Width;
            L.height = in.Params.Height;
            L.shaping_cone_angle = in.Params.ShapingConeAngle;
            L.shaping_cone_softness = in.Params.ShapingConeSoftness;
            s.light_texels.emplace_back();
            // the dome reads its file as linear RGB floats (DomeLight::Prepare, dome_light.cpp:35-47)
            if (!in.Params.TextureFile.GetAssetPath().empty() && _loader &&
                _loader(in.Params.TextureFile, true, s.light_texels.back(), L.tex_width, L.tex_height))
                L.texture = s.light_texels.back().data();
            light_index[id] = (int)s.lights.size();
            s.lights.push_back(L);
        }
        // materials, in SdfPath order
        std::map<SdfPath, int> material_index;
        s.materials.reserve(_materials.size());
        s.material_texels.reserve(4 * _materials.size());
        for (const auto &[id, p] : _materials) {
            material_index[id] = (int)s.materials.size();
            s.materials.push_back(MaterialDesc(p, s));
        }
        // instances (appendMeshInstance, scene.cpp:174-238)
        std::map<std::pair<const IMesh *, size_t>, int> mesh_index;
        for (const auto &[id, mesh] : _meshes) {
            if (!mesh || !mesh->IsVisible()) continue;
            const auto &subsets = mesh->GetSubsets();
            const auto lit = light_index.find(mesh->GetId());
            const int light = lit == light_index.end() ? -1 : lit->second;
            auto add = [&](size_t si, const GfMatrix4f &xf) {
                const auto key = std::make_pair(static_cast<const IMesh *>(mesh), si);
                auto mit = mesh_index.find(key);
                if (mit == mesh_index.end()) mit = mesh_index.emplace(key, MeshDescOf(id, *mesh, si, s)).first;
                hdr_instance_desc in{};
                in.mesh = mit->second;
                const auto matit = material_index.find(subsets[si].materialId);
                in.material = matit == material_index.end() ? -1 : matit->second;
                in.light = light;
                for (int r = 0; r < 4; ++r)
                    for (int c = 0; c < 4; ++c) in.transform[4 * r + c] = xf[r][c];
                s.instances.push_back(in);
            };
            if (!mesh->GetInstancerId().IsEmpty()) {
                const auto it = _instancers.find(mesh->GetInstancerId());
                if (it != _instancers.end() && it->second != nullptr) {
                    const VtMatrix4dArray transforms{it->second->ComputeInstanceTransforms(mesh->GetId())};
                    for (const auto &t : transforms)
                        for (size_t si = 0; si < subsets.size(); ++si) add(si, GfMatrix4f(t) * mesh->GetTransform());
                }
                continue;
            }
            for (size_t si = 0; si < subsets.size(); ++si) add(si, mesh->GetTransform());
        }
        s.desc.meshes = s.meshes.data();
        s.desc.num_meshes = (int32_t)s.meshes.size();
        s.desc.instances = s.instances.data();
        s.desc.num_instances = (int32_t)s.instances.size();
        s.desc.materials = s.materials.data();
        s.desc.num_materials = (int32_t)s.materials.size();
        s.desc.lights = s.lights.data();
        s.desc.num_lights = (int32_t)s.lights.size();
        // SceneBuildRenderStateConfig (scene.cpp:248-268): the physical sky as the environment
        s.desc.enable_physical_sky = _config.EnablePhysicalSky ? 1 : 0;
        s.desc.physical_sky_time = _config.PhysicalSkyTime;
        return s.desc;
    }

  private:
    struct Primvars {
        VtVec2fArray uvs;
        VtVec3fArray normals, colors;
    };
    struct MeshArrays {
        std::vector<float> points, uvs, normals, colors;
        std::vector<int32_t> indices;
    };
    struct Store {
        hdr_scene_desc desc{};
        std::vector<hdr_mesh_desc> meshes;
        std::vector<std::unique_ptr<MeshArrays>> arrays;
        std::vector<hdr_instance_desc> instances;
        std::vector<hdr_material_desc> materials;
        std::vector<hdr_light_desc> lights;
        std::vector<std::vector<float>> material_texels, light_texels;
    };

    template <class V>
    static void flat(const V &arr, int n, std::vector<float> &out) {
        out.resize(arr.size() * (size_t)n);
        for (size_t i = 0; i < arr.size(); ++i)
            for (int k = 0; k < n; ++k) out[i * (size_t)n + (size_t)k] = arr[i][k];
    }

    // one (mesh, subset): the reference's BVH inputs for it (hd_restir_mesh.cpp:505-531)
    int MeshDescOf(const SdfPath &id, const IMesh &mesh, size_t si, Store &s) {
        const auto &subsets = mesh.GetSubsets();
        const MeshSubset &sub = subsets[si];
        auto a = std::make_unique<MeshArrays>();
        flat(mesh.GetPoints(), 3, a->points);
        a->indices.resize(sub.indices.size() * 3);
        for (size_t t = 0; t < sub.indices.size(); ++t)
            for (int k = 0; k < 3; ++k) a->indices[3 * t + (size_t)k] = sub.indices[t][k];
        VtVec2fArray uvs = mesh.GetUVs();
        VtVec3fArray normals = mesh.GetNormals(), colors = mesh.GetColors();
        const auto pv = _subsetPrimvars.find({id, si});
        if (pv != _subsetPrimvars.end()) {
            if (!pv->second.uvs.empty()) uvs = pv->second.uvs;
            if (!pv->second.normals.empty()) normals = pv->second.normals;
            if (!pv->second.colors.empty()) colors = pv->second.colors;
        } else if (subsets.size() > 1) {
            // face-varying arrays of the whole mesh: HdRestirMesh split them per subset
            size_t total = 0;
            for (const MeshSubset &x : subsets) total += x.indices.size();
            const size_t np = mesh.GetPoints().size();
            const bool corner = (uvs.size() == 3 * total && uvs.size() != np) ||
                                (normals.size() == 3 * total && normals.size() != np) ||
                                (colors.size() == 3 * total && colors.size() != np);
            if (corner)
                throw std::runtime_error("[hdrestir-b200] mesh " + id.GetString() +
                                         ": face-varying primvars over several subsets; give them per subset "
                                         "(SceneHandoff::SetSubsetPrimvars)");
        }
        flat(uvs, 2, a->uvs);
        flat(normals, 3, a->normals);
        flat(colors, 3, a->colors);
        hdr_mesh_desc m{};
        m.points = a->points.data();
        m.num_points = (int32_t)(a->points.size() / 3);
        m.indices = a->indices.data();
        m.num_triangles = (int32_t)(a->indices.size() / 3);
        m.uvs = a->uvs.empty() ? nullptr : a->uvs.data();
        m.num_uvs = (int32_t)(a->uvs.size() / 2);
        m.normals = a->normals.empty() ? nullptr : a->normals.data();
        m.num_normals = (int32_t)(a->normals.size() / 3);
        m.colors = a->colors.empty() ? nullptr : a->colors.data();
        m.num_colors = (int32_t)(a->colors.size() / 3);
        s.arrays.push_back(std::move(a));
        s.meshes.push_back(m);
        return (int)s.meshes.size() - 1;
    }

    // PreviewSurfaceParams field for field (materials/preview_surface_params.h:12-52); the
    // textures decoded by the loader (the diffuse one sRGB-decoded, the others linear)
    hdr_material_desc MaterialDesc(const PreviewSurfaceParams &p, Store &s) {
        hdr_material_desc m{};
        auto c3 = [](float *d, const GfVec3f &v) {
            for (int k = 0; k < 3; ++k) d[k] = v[k];
        };
        c3(m.diffuse_color, p.DiffuseColor);
        m.metallic = p.Metallic;
        m.roughness = p.Roughness;
        c3(m.specular_color, p.SpecularColor);
        m.specular = p.Specular;
        m.opacity = p.Opacity;
        m.ior = p.Ior;
        m.transmission = p.Transmission;
        c3(m.transmission_color, p.TransmissionColor);
        m.transmission_depth = p.TransmissionDepth;
        c3(m.transmission_scatter, p.TransmissionScatter);
        c3(m.emission_color, p.EmissionColor);
        m.emission = p.Emission;
        m.coat = p.Coat;
        c3(m.coat_color, p.CoatColor);
        m.coat_roughness = p.CoatRoughness;
        m.coat_ior = p.CoatIor;
        m.sheen = p.Sheen;
        c3(m.sheen_color, p.SheenColor);
        m.sheen_roughness = p.SheenRoughness;
        m.subsurface = p.Subsurface;
        c3(m.subsurface_color, p.SubsurfaceColor);
        c3(m.subsurface_radius, p.SubsurfaceRadius);
        m.subsurface_scale = p.SubsurfaceScale;
        m.subsurface_anisotropy = p.SubsurfaceAnisotropy;
        m.thin_walled = p.ThinWalled ? 1 : 0;
        m.diffuse_roughness = p.DiffuseRoughness;
        const SdfAssetPath *tex[4] = {&p.DiffuseTexture, &p.MetallicTexture, &p.RoughnessTexture, &p.NormalTexture};
        for (int k = 0; k < 4; ++k) {
            if (tex[k]->GetAssetPath().empty() || !_loader) continue;
            s.material_texels.emplace_back();
            int w = 0, h = 0;
            if (_loader(*tex[k], k != HDR_TEX_DIFFUSE, s.material_texels.back(), w, h) && w > 0 && h > 0) {
                m.textures[k] = s.material_texels.back().data();
                m.tex_width[k] = w;
                m.tex_height[k] = h;
            }
        }
        return m;
    }

    Scene *_forward;
    SceneBuildRenderStateConfig _config{};  // of the last BuildRenderState
    TextureLoader _loader;
    std::map<SdfPath, IMesh *> _meshes;
    std::map<SdfPath, IInstancer *> _instancers;
    std::map<SdfPath, PreviewSurfaceParams> _materials;
    std::map<SdfPath, LightFactoryInput> _lights;
    std::map<std::pair<SdfPath, size_t>, Primvars> _subsetPrimvars;
    std::unique_ptr<Store> _store;
};

}  // namespace Restir::B200
