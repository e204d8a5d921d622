// hdr_material_from_network: the material network of a Hydra material mapped to
// PreviewSurface parameters, as HdRestirMaterial::Sync does on the host before
// Scene::SetMaterialParams (hydra/hd_restir_material.cpp:22-424).
//
// The walk starts at the surface terminal ("mtlx:surface", else "surface", else
// "outputs:surface", else the first terminal by name) and visits every node
// upstream of it once, depth first, inputs in name order. Each node's
// parameters (in name order, so a later name overrides an earlier one that sets
// the same field) are applied by shader family:
//   UsdPreviewSurface                      diffuseColor, metallic, roughness,
//                                          specularColor, opacity, ior, emissiveColor
//                                          (which also sets emission to 1)
//   standard_surface (ND_standard_surface_surfaceshader, StandardSurface) and
//   open_pbr_surface (ND_open_pbr_surface_surfaceshader)
//                                          their weights and colours; diffuse
//                                          colour = base colour x base weight
//                                          (defaults 0.8 and 1)
//   image nodes (UsdUVTexture, ND_image*)  an asset-valued "file" or "texcoord"
//                                          becomes a texture of the surface input
//                                          the connection chain started from
// A parameter counts only when it holds the type the reference tests for.
// Texture slots hold asset paths; the host decodes them (as the reference's
// ImageTextureSamplerFactory does) into hdr_material_desc.textures. The result
// is that of a material's first Sync (the reference keeps a material's earlier
// parameters across later syncs; a caller that wants that passes the earlier
// result's fields back through a network of its own).
#include <algorithm>
#include <cstddef>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "../../../include/hdrestir.h"

namespace hdr {
hdr_status set_last_error(hdr_status st, const char *fmt, ...);
}

namespace {

// PreviewSurfaceParams defaults (materials/preview_surface_params.h:12-52)
void preview_defaults(hdr_material_desc &m) {
    std::memset(&m, 0, sizeof(m));
    auto set3 = [](float *v, float a) { v[0] = v[1] = v[2] = a; };
    set3(m.diffuse_color, 1.0f);
    m.metallic = 0.0f;
    m.roughness = 0.5f;
    set3(m.specular_color, 1.0f);
    m.specular = 1.0f;
    m.opacity = 1.0f;
    m.ior = 1.5f;
    m.transmission = 0.0f;
    set3(m.transmission_color, 1.0f);
    m.transmission_depth = 0.0f;
    set3(m.transmission_scatter, 0.0f);
    set3(m.emission_color, 1.0f);
    m.emission = 0.0f;
    m.coat = 0.0f;
    set3(m.coat_color, 1.0f);
    m.coat_roughness = 0.1f;
    m.coat_ior = 1.5f;
    m.sheen = 0.0f;
    set3(m.sheen_color, 1.0f);
    m.sheen_roughness = 0.3f;
    m.subsurface = 0.0f;
    set3(m.subsurface_color, 1.0f);
    set3(m.subsurface_radius, 1.0f);
    m.subsurface_scale = 1.0f;
    m.subsurface_anisotropy = 0.0f;
    m.thin_walled = 0;
    m.diffuse_roughness = 0.0f;
}

enum Target { kNone, kF, kF3, kBool, kBase, kBaseColor, kEmissive };

struct Rule {
    const char *name;
    int type;      // HDR_MTL_* the parameter must hold
    Target what;
    size_t field;  // offset into hdr_material_desc (kF, kF3, kBool)
};

#define F(field) offsetof(hdr_material_desc, field)

// UsdPreviewSurface (hd_restir_material.cpp:47-81)
const Rule kPreview[] = {
    {"diffuseColor", HDR_MTL_FLOAT3, kF3, F(diffuse_color)}, {"metallic", HDR_MTL_FLOAT, kF, F(metallic)},
    {"roughness", HDR_MTL_FLOAT, kF, F(roughness)},          {"specularColor", HDR_MTL_FLOAT3, kF3, F(specular_color)},
    {"opacity", HDR_MTL_FLOAT, kF, F(opacity)},              {"ior", HDR_MTL_FLOAT, kF, F(ior)},
    {"emissiveColor", HDR_MTL_FLOAT3, kEmissive, 0},
};

// standard_surface (hd_restir_material.cpp:82-212)
const Rule kStandard[] = {
    {"base", HDR_MTL_FLOAT, kBase, 0},
    {"base_weight", HDR_MTL_FLOAT, kBase, 0},
    {"base_color", HDR_MTL_FLOAT3, kBaseColor, 0},
    {"metalness", HDR_MTL_FLOAT, kF, F(metallic)},
    {"specular", HDR_MTL_FLOAT, kF, F(specular)},
    {"specular_weight", HDR_MTL_FLOAT, kF, F(specular)},
    {"specular_color", HDR_MTL_FLOAT3, kF3, F(specular_color)},
    {"specular_roughness", HDR_MTL_FLOAT, kF, F(roughness)},
    {"roughness", HDR_MTL_FLOAT, kF, F(roughness)},
    {"opacity", HDR_MTL_FLOAT, kF, F(opacity)},
    {"ior", HDR_MTL_FLOAT, kF, F(ior)},
    {"transmission", HDR_MTL_FLOAT, kF, F(transmission)},
    {"transmission_weight", HDR_MTL_FLOAT, kF, F(transmission)},
    {"transmission_color", HDR_MTL_FLOAT3, kF3, F(transmission_color)},
    {"transmission_depth", HDR_MTL_FLOAT, kF, F(transmission_depth)},
    {"transmission_scatter", HDR_MTL_FLOAT3, kF3, F(transmission_scatter)},
    {"subsurface", HDR_MTL_FLOAT, kF, F(subsurface)},
    {"subsurface_weight", HDR_MTL_FLOAT, kF, F(subsurface)},
    {"subsurface_color", HDR_MTL_FLOAT3, kF3, F(subsurface_color)},
    {"subsurface_radius", HDR_MTL_FLOAT3, kF3, F(subsurface_radius)},
    {"subsurface_scale", HDR_MTL_FLOAT, kF, F(subsurface_scale)},
    {"subsurface_anisotropy", HDR_MTL_FLOAT, kF, F(subsurface_anisotropy)},
    {"sheen", HDR_MTL_FLOAT, kF, F(sheen)},
    {"sheen_weight", HDR_MTL_FLOAT, kF, F(sheen)},
    {"sheen_color", HDR_MTL_FLOAT3, kF3, F(sheen_color)},
    {"sheen_roughness", HDR_MTL_FLOAT, kF, F(sheen_roughness)},
    {"coat", HDR_MTL_FLOAT, kF, F(coat)},
    {"coat_weight", HDR_MTL_FLOAT, kF, F(coat)},
    {"coat_color", HDR_MTL_FLOAT3, kF3, F(coat_color)},
    {"coat_roughness", HDR_MTL_FLOAT, kF, F(coat_roughness)},
    {"coat_IOR", HDR_MTL_FLOAT, kF, F(coat_ior)},
    {"coat_ior", HDR_MTL_FLOAT, kF, F(coat_ior)},
    {"thin_walled", HDR_MTL_BOOL, kBool, F(thin_walled)},
    {"diffuse_roughness", HDR_MTL_FLOAT, kF, F(diffuse_roughness)},
    {"emission", HDR_MTL_FLOAT, kF, F(emission)},
    {"emission_weight", HDR_MTL_FLOAT, kF, F(emission)},
    {"emission_color", HDR_MTL_FLOAT3, kF3, F(emission_color)},
};

// open_pbr_surface (hd_restir_material.cpp:213-329)
const Rule kOpenPbr[] = {
    {"base_weight", HDR_MTL_FLOAT, kBase, 0},
    {"base_color", HDR_MTL_FLOAT3, kBaseColor, 0},
    {"base_metalness", HDR_MTL_FLOAT, kF, F(metallic)},
    {"specular_weight", HDR_MTL_FLOAT, kF, F(specular)},
    {"specular_color", HDR_MTL_FLOAT3, kF3, F(specular_color)},
    {"specular_roughness", HDR_MTL_FLOAT, kF, F(roughness)},
    {"geometry_opacity", HDR_MTL_FLOAT, kF, F(opacity)},
    {"specular_ior", HDR_MTL_FLOAT, kF, F(ior)},
    {"transmission_weight", HDR_MTL_FLOAT, kF, F(transmission)},
    {"transmission_color", HDR_MTL_FLOAT3, kF3, F(transmission_color)},
    {"transmission_depth", HDR_MTL_FLOAT, kF, F(transmission_depth)},
    {"transmission_scatter", HDR_MTL_FLOAT3, kF3, F(transmission_scatter)},
    {"subsurface_weight", HDR_MTL_FLOAT, kF, F(subsurface)},
    {"subsurface_color", HDR_MTL_FLOAT3, kF3, F(subsurface_color)},
    {"subsurface_radius", HDR_MTL_FLOAT3, kF3, F(subsurface_radius)},
    {"subsurface_radius_scale", HDR_MTL_FLOAT, kF, F(subsurface_scale)},
    {"subsurface_anisotropy", HDR_MTL_FLOAT, kF, F(subsurface_anisotropy)},
    {"fuzz_weight", HDR_MTL_FLOAT, kF, F(sheen)},
    {"fuzz_color", HDR_MTL_FLOAT3, kF3, F(sheen_color)},
    {"fuzz_roughness", HDR_MTL_FLOAT, kF, F(sheen_roughness)},
    {"coat_weight", HDR_MTL_FLOAT, kF, F(coat)},
    {"coat_color", HDR_MTL_FLOAT3, kF3, F(coat_color)},
    {"coat_roughness", HDR_MTL_FLOAT, kF, F(coat_roughness)},
    {"coat_ior", HDR_MTL_FLOAT, kF, F(coat_ior)},
    {"geometry_thin_walled", HDR_MTL_BOOL, kBool, F(thin_walled)},
    {"emission_luminance", HDR_MTL_FLOAT, kF, F(emission)},
    {"emission_color", HDR_MTL_FLOAT3, kF3, F(emission_color)},
};
#undef F

template <size_t N>
bool in(const std::string &s, const char *const (&names)[N]) {
    for (const char *n : names)
        if (s == n) return true;
    return false;
}

const char *const kStandardIds[] = {"ND_standard_surface_surfaceshader", "standard_surface", "StandardSurface"};
const char *const kOpenPbrIds[] = {"ND_open_pbr_surface_surfaceshader", "open_pbr_surface"};
const char *const kImageIds[] = {"UsdUVTexture",     "ND_image_color3",  "ND_image",         "ND_image_float",
                                 "ND_image_vector2", "ND_image_vector3", "ND_image_vector4", "ND_image_color4"};
// surface inputs whose upstream image nodes become each texture slot (hd_restir_material.cpp:330-406);
// an emission chain fills the diffuse slot only while it is empty
const char *const kDiffuseInputs[] = {"diffuseColor", "base_color", "base"};
const char *const kMetallicInputs[] = {"metalness", "base_metalness"};
const char *const kRoughnessInputs[] = {"specular_roughness", "roughness"};
const char *const kEmissionInputs[] = {"emissiveColor", "emission_color", "emission", "emission_luminance"};

struct Walk {
    std::map<std::string, const hdr_mtl_node *> nodes;
    std::set<std::string> visited;
    hdr_material_desc *out;
    hdr_mtl_textures *tex;

    void set_texture(int slot, const char *path) {
        if (!tex) return;
        std::strncpy(tex->path[slot], path, sizeof(tex->path[slot]) - 1);
        tex->path[slot][sizeof(tex->path[slot]) - 1] = '\0';
    }

    template <size_t N>
    void apply(const std::vector<const hdr_mtl_param *> &params, const Rule (&rules)[N], bool weighted) {
        float base = 1.0f, base_color[3] = {0.8f, 0.8f, 0.8f};
        char *o = reinterpret_cast<char *>(out);
        for (const hdr_mtl_param *p : params) {
            for (const Rule &r : rules) {
                if (p->type != r.type || std::strcmp(p->name, r.name) != 0) continue;
                switch (r.what) {
                    case kF: std::memcpy(o + r.field, &p->value[0], sizeof(float)); break;
                    case kF3: std::memcpy(o + r.field, p->value, 3 * sizeof(float)); break;
                    case kBool: {
                        const int32_t b = p->value[0] != 0.0f ? 1 : 0;
                        std::memcpy(o + r.field, &b, sizeof(b));
                        break;
                    }
                    case kBase: base = p->value[0]; break;
                    case kBaseColor: std::memcpy(base_color, p->value, sizeof(base_color)); break;
                    case kEmissive:
                        std::memcpy(out->emission_color, p->value, 3 * sizeof(float));
                        out->emission = 1.0f;
                        break;
                    default: break;
                }
            }
        }
        if (weighted)  // GfVec3f * float: each component rounded once (the double product is exact)
            for (int k = 0; k < 3; ++k) out->diffuse_color[k] = (float)((double)base_color[k] * (double)base);
    }

    void image(const std::vector<const hdr_mtl_param *> &params, const std::string &target) {
        int slot = -1;
        bool only_if_empty = false;
        if (in(target, kDiffuseInputs))
            slot = HDR_TEX_DIFFUSE;
        else if (in(target, kMetallicInputs))
            slot = HDR_TEX_METALLIC;
        else if (in(target, kRoughnessInputs))
            slot = HDR_TEX_ROUGHNESS;
        else if (in(target, kEmissionInputs))
            slot = HDR_TEX_DIFFUSE, only_if_empty = true;
        else if (target == "normal")
            slot = HDR_TEX_NORMAL;
        if (slot < 0) return;
        for (const hdr_mtl_param *p : params) {
            if (p->type != HDR_MTL_ASSET || !p->asset) continue;
            if (std::strcmp(p->name, "file") != 0 && std::strcmp(p->name, "texcoord") != 0) continue;
            if (only_if_empty && tex && tex->path[HDR_TEX_DIFFUSE][0] != '\0') continue;
            set_texture(slot, p->asset);
        }
    }

    void visit(const std::string &path, const std::string &target) {
        if (!visited.insert(path).second) return;
        const auto it = nodes.find(path);
        if (it == nodes.end()) return;
        const hdr_mtl_node &node = *it->second;
        const std::string id = node.shader_id ? node.shader_id : "";
        std::vector<const hdr_mtl_param *> params;
        for (int i = 0; i < node.num_params; ++i)
            if (node.params[i].name) params.push_back(&node.params[i]);
        std::stable_sort(params.begin(), params.end(), [](const hdr_mtl_param *a, const hdr_mtl_param *b) {
            return std::strcmp(a->name, b->name) < 0;
        });
        if (id == "UsdPreviewSurface")
            apply(params, kPreview, false);
        else if (in(id, kStandardIds))
            apply(params, kStandard, true);
        else if (in(id, kOpenPbrIds))
            apply(params, kOpenPbr, true);
        else if (in(id, kImageIds))
            image(params, target);
        // upstream, inputs in name order; a chain keeps the surface input it started from
        std::vector<const hdr_mtl_connection *> inputs;
        for (int i = 0; i < node.num_inputs; ++i)
            if (node.inputs[i].input && node.inputs[i].upstream_node) inputs.push_back(&node.inputs[i]);
        std::stable_sort(inputs.begin(), inputs.end(), [](const hdr_mtl_connection *a, const hdr_mtl_connection *b) {
            return std::strcmp(a->input, b->input) < 0;
        });
        for (const hdr_mtl_connection *c : inputs) visit(c->upstream_node, target.empty() ? c->input : target);
    }
};

}  // namespace

extern "C" hdr_status hdr_material_from_network(const hdr_mtl_network *net, hdr_material_desc *out,
                                                hdr_mtl_textures *textures) {
    if (!net || !out) return hdr::set_last_error(HDR_EINVAL, "NULL argument");
    if (net->num_nodes < 0 || net->num_terminals < 0 || (net->num_nodes > 0 && !net->nodes) ||
        (net->num_terminals > 0 && !net->terminals))
        return hdr::set_last_error(HDR_EINVAL, "bad node or terminal array");
    preview_defaults(*out);
    if (textures) std::memset(textures, 0, sizeof(*textures));
    Walk w{{}, {}, out, textures};
    for (int i = 0; i < net->num_nodes; ++i)
        if (net->nodes[i].path) w.nodes.emplace(net->nodes[i].path, &net->nodes[i]);
    // the surface terminal (hd_restir_material.cpp:446-466)
    std::map<std::string, std::string> terminals;
    for (int i = 0; i < net->num_terminals; ++i)
        if (net->terminals[i].name && net->terminals[i].upstream_node)
            terminals.emplace(net->terminals[i].name, net->terminals[i].upstream_node);
    const char *const priority[] = {"mtlx:surface", "surface", "outputs:surface"};
    const std::string *start = nullptr;
    for (const char *t : priority) {
        const auto it = terminals.find(t);
        if (it != terminals.end()) {
            start = &it->second;
            break;
        }
    }
    if (!start && !terminals.empty()) start = &terminals.begin()->second;
    if (start) w.visit(*start, std::string());
    return HDR_OK;
}
