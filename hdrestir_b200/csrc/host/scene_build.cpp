// Host-side scene preparation (see scene_build.h for the reference map).
// Compiled with -ffp-contract=off: the values computed here (centroids,
// bounds, tangent frames, light frames) must round exactly like the
// reference's host code.
#include "scene_build.h"

#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <utility>

namespace hdr {

namespace {

inline float as_float(int i) {
    float f;
    std::memcpy(&f, &i, 4);
    return f;
}

struct BlasBuilder {
    Blas &b;
    void subdivide(int node_idx, int start, int end, int depth) {
        if (depth > b.max_depth) b.max_depth = depth;
        BlasNode &node = b.nodes[node_idx];
        node.bounds.set_empty();
        for (int i = start; i < end; ++i) {
            node.bounds.extend(b.tris[i].v0);
            node.bounds.extend(b.tris[i].v1);
            node.bounds.extend(b.tris[i].v2);
        }
        const int count = end - start;
        if (count <= 4) {
            node.left = -start - 1;
            node.count = count;
            return;
        }
        const V3 size = node.bounds.size();
        int axis = 0;
        if (size.y > size.x) axis = 1;
        if (comp(size, 2) > comp(size, axis)) axis = 2;
        const float split = comp(node.bounds.mn, axis) + comp(size, axis) * 0.5f;
        int i = start, j = end - 1;
        while (i <= j) {
            if (comp(b.tris[i].centroid, axis) < split) {
                i++;
            } else {
                std::swap(b.tris[i], b.tris[j]);
                j--;
            }
        }
        const int left_count = i - start;
        if (left_count == 0 || left_count == count) i = start + count / 2;
        const int left_idx = (int)b.nodes.size();
        b.nodes.push_back(BlasNode());
        b.nodes.push_back(BlasNode());
        b.nodes[node_idx].left = left_idx;
        b.nodes[node_idx].count = 0;
        subdivide(left_idx, start, i, depth + 1);
        subdivide(left_idx + 1, i, end, depth + 1);
    }
};

struct TlasBuilder {
    std::vector<TlasNode> &nodes;
    std::vector<int> &idx;
    const std::vector<HostInstance> &inst;
    int max_depth = 0;
    void subdivide(int node_idx, int start, int end, int depth) {
        if (depth > max_depth) max_depth = depth;
        const int left_idx = (int)nodes.size();
        nodes.push_back(TlasNode{});
        nodes.push_back(TlasNode{});
        nodes[node_idx].left = left_idx;
        nodes[node_idx].count = 0;
        nodes[node_idx].bounds.set_empty();
        for (int i = start; i < end; ++i) {
            const Range3 &bb = inst[idx[i]].bounds;
            nodes[node_idx].bounds.extend(bb.mn);
            nodes[node_idx].bounds.extend(bb.mx);
        }
        const int count = end - start;
        if (count <= 2) {
            nodes[node_idx].left = -start - 1;
            nodes[node_idx].count = count;
            return;
        }
        const V3 size = nodes[node_idx].bounds.size();
        int axis = 0;
        if (size.y > size.x) axis = 1;
        if (comp(size, 2) > comp(size, axis)) axis = 2;
        const float split = comp(nodes[node_idx].bounds.mn, axis) + comp(size, axis) * 0.5f;
        int i = start, j = end - 1;
        while (i <= j) {
            if (comp(inst[idx[i]].centroid, axis) < split) {
                ++i;
            } else {
                std::swap(idx[i], idx[j]);
                --j;
            }
        }
        if (i == start || i == end) i = start + count / 2;
        subdivide(left_idx, start, i, depth + 1);
        subdivide(left_idx + 1, i, end, depth + 1);
    }
};

// Scene::_TransformBounds (scene.cpp:101-116)
Range3 transform_bounds(const Range3 &b, const float *m) {
    if (b.empty()) return b;
    const V3 mn = b.mn, mx = b.mx;
    const V3 corners[8] = {{mn.x, mn.y, mn.z}, {mx.x, mn.y, mn.z}, {mn.x, mx.y, mn.z}, {mx.x, mx.y, mn.z},
                           {mn.x, mn.y, mx.z}, {mx.x, mn.y, mx.z}, {mn.x, mx.y, mx.z}, {mx.x, mx.y, mx.z}};
    Range3 r;
    for (const V3 &c : corners) r.extend(m4f_transform(m, c));
    return r;
}

void put_node(std::vector<float> &dst, const Range3 &r, int left, int count) {
    const float rec[8] = {r.mn.x, r.mn.y, r.mn.z, as_float(left), r.mx.x, r.mx.y, r.mx.z, as_float(count)};
    dst.insert(dst.end(), rec, rec + 8);
}

// Collapse of a binary tree (children of an inner node at left and left+1, a
// leaf when left < 0) into 4-wide nodes over the SAME boxes: the slots of the
// wide node made for binary node n are n's grandchildren, or n's child itself
// when that child is a leaf, in left-to-right order. Only the boxes of the
// odd-depth nodes are dropped. Every tree here is built bottom-up as the union
// of its children's boxes, and the slab test is monotone under box inclusion
// (the rounded products (bound - o) * inv are monotone in bound), so a child's
// box passes only if its parent's passes and enters no earlier. The dropped
// test therefore never rejects a ray its children would keep, nor culls one by
// entry distance that its children would not, and a depth-first walk of the
// wide tree tests the same leaves in the same order with the same running
// closest t as the binary walk.
template <class Node>
struct WideBuilder {
    const std::vector<Node> &nodes;
    int leaf_tag, inner_tag, count_bits;
    std::vector<float> out;
    int max_depth = 0;
    bool overflow = false;

    int leaf_code(const Node &n) const {
        const long long start = -(long long)n.left - 1;
        const long long payload = (start << count_bits) | (long long)(n.count - 1);
        const int count = n.count, max_count = 1 << count_bits;
        if (count < 1 || count > max_count || payload >= (1ll << 28)) return -2;
        return (int)(payload << kWideTagBits) | leaf_tag;
    }
    int code_of(int idx, int depth) {
        const Node &n = nodes[(size_t)idx];
        if (n.left < 0) return leaf_code(n);
        const int w = emit(idx, depth);
        if (w >= (1 << 28)) return -2;
        return (w << kWideTagBits) | inner_tag;
    }
    // returns the wide-node index of inner binary node idx
    int emit(int idx, int depth) {
        if (depth > max_depth) max_depth = depth;
        const int w = (int)(out.size() / kWideNodeFloats);
        out.resize(out.size() + kWideNodeFloats, 0.0f);
        int slot_node[4];
        int ns = 0;
        const Node &n = nodes[(size_t)idx];
        for (int c = 0; c < 2; ++c) {
            const int ci = n.left + c;
            const Node &ch = nodes[(size_t)ci];
            if (ch.left < 0) {
                slot_node[ns++] = ci;
            } else {
                slot_node[ns++] = ch.left;
                slot_node[ns++] = ch.left + 1;
            }
        }
        int codes[4] = {-1, -1, -1, -1};
        for (int k = 0; k < ns; ++k) {
            codes[k] = code_of(slot_node[k], depth + 1);
            if (codes[k] == -2) overflow = true;
        }
        float *r = &out[(size_t)w * kWideNodeFloats];
        for (int k = 0; k < 4; ++k) {
            Range3 b;  // empty slot: min > max, never passes the slab test
            if (k < ns) b = nodes[(size_t)slot_node[k]].bounds;
            r[0 + k] = b.mn.x;
            r[4 + k] = b.mn.y;
            r[8 + k] = b.mn.z;
            r[12 + k] = b.mx.x;
            r[16 + k] = b.mx.y;
            r[20 + k] = b.mx.z;
            r[24 + k] = as_float(codes[k]);
        }
        return w;
    }
    // root entry: {min.xyz, code, max.xyz, 0}
    void root(float rec[8]) {
        const Node &n = nodes[0];
        const int code = code_of(0, 1);
        if (code == -2) overflow = true;
        const float r[8] = {n.bounds.mn.x, n.bounds.mn.y, n.bounds.mn.z, as_float(code),
                            n.bounds.mx.x, n.bounds.mx.y, n.bounds.mx.z, 0.0f};
        std::memcpy(rec, r, sizeof(r));
    }
};

}  // namespace

// MeshSubset::range over the referenced points (hd_restir_mesh.cpp:523-529)
Range3 mesh_range(const hdr_mesh_desc &m) {
    Range3 r;
    for (int i = 0; i < m.num_triangles; ++i) {
        for (int k = 0; k < 3; ++k) {
            const int p = m.indices[3 * i + k];
            if (p >= 0 && p < m.num_points) r.extend(V3{m.points[3 * p], m.points[3 * p + 1], m.points[3 * p + 2]});
        }
    }
    return r;
}

Blas build_blas(const hdr_mesh_desc &m) {
    Blas b;
    b.range = mesh_range(m);
    if (m.num_triangles <= 0 || m.num_points <= 0) return b;
    b.tris.reserve((size_t)m.num_triangles);
    for (int i = 0; i < m.num_triangles; ++i) {
        BlasTriangle t;
        if (make_triangle(m, i, t)) b.tris.push_back(t);
    }
    if (b.tris.empty()) return b;
    b.nodes.reserve((size_t)m.num_triangles * 2);
    b.nodes.push_back(BlasNode());
    BlasBuilder bb{b};
    bb.subdivide(0, 0, (int)b.tris.size(), 1);
    return b;
}

bool build_flat_scene(const hdr_scene_desc &desc, FlatScene &out, std::string &err, const ExternalBlas *ext) {
    out = FlatScene{};
    if (desc.num_meshes < 0 || desc.num_instances < 0 || desc.num_materials < 0 || desc.num_lights < 0) {
        err = "negative count in hdr_scene_desc";
        return false;
    }
    // ---- BLAS per mesh
    std::vector<int> node_base(desc.num_meshes), tri_base(desc.num_meshes), blas_ok(desc.num_meshes);
    std::vector<int> wide_base(desc.num_meshes);
    std::vector<Range3> ranges(desc.num_meshes);
    for (int mi = 0; mi < desc.num_meshes; ++mi) {
        const hdr_mesh_desc &m = desc.meshes[mi];
        if ((m.num_points > 0 && !m.points) || (m.num_triangles > 0 && !m.indices) || (m.num_uvs > 0 && !m.uvs) ||
            (m.num_normals > 0 && !m.normals) || (m.num_colors > 0 && !m.colors)) {
            err = "mesh " + std::to_string(mi) + ": NULL array with non-zero count";
            return false;
        }
        if (ext) {  // the trees and triangle records are built elsewhere (on the device)
            const ExternalBlas &e = ext[mi];
            ranges[mi] = mesh_range(m);
            const Range3 &r = ranges[mi];
            const float r6[6] = {r.mn.x, r.mn.y, r.mn.z, r.mx.x, r.mx.y, r.mx.z};
            out.mesh_ranges.insert(out.mesh_ranges.end(), r6, r6 + 6);
            node_base[mi] = (int)out.num_blas_nodes;
            tri_base[mi] = (int)out.num_triangles;
            out.mesh_tri_base.push_back((int)out.num_triangles);
            out.mesh_tri_count.push_back(e.num_tris);
            blas_ok[mi] = e.num_nodes > 0 ? 1 : 0;
            wide_base[mi] = 0;
            if (e.max_depth > out.max_blas_depth) out.max_blas_depth = e.max_depth;
            out.num_blas_nodes += (size_t)e.num_nodes;
            out.num_triangles += (size_t)e.num_tris;
            continue;
        }
        Blas b = build_blas(m);
        ranges[mi] = b.range;
        const float r6[6] = {b.range.mn.x, b.range.mn.y, b.range.mn.z, b.range.mx.x, b.range.mx.y, b.range.mx.z};
        out.mesh_ranges.insert(out.mesh_ranges.end(), r6, r6 + 6);
        node_base[mi] = (int)out.num_blas_nodes;
        tri_base[mi] = (int)out.num_triangles;
        out.mesh_tri_base.push_back((int)out.num_triangles);
        out.mesh_tri_count.push_back((int)b.tris.size());
        blas_ok[mi] = b.nodes.empty() ? 0 : 1;
        if (b.max_depth > out.max_blas_depth) out.max_blas_depth = b.max_depth;
        for (const BlasNode &n : b.nodes) put_node(out.blas_nodes, n.bounds, n.left, n.count);
        wide_base[mi] = (int)(out.blas4.size() / kWideNodeFloats);
        float root[8] = {0.0f, 0.0f, 0.0f, as_float(-1), 0.0f, 0.0f, 0.0f, 0.0f};
        if (!b.nodes.empty()) {
            WideBuilder<BlasNode> wb{b.nodes, kWTagBlasLeaf, kWTagBlasNode, kBlasLeafCountBits, {}};
            wb.root(root);
            if (wb.overflow) {
                err = "mesh " + std::to_string(mi) + ": too many triangles for the wide BVH encoding";
                return false;
            }
            if (wb.max_depth > out.max_blas4_depth) out.max_blas4_depth = wb.max_depth;
            out.blas4.insert(out.blas4.end(), wb.out.begin(), wb.out.end());
        }
        out.blas_roots.insert(out.blas_roots.end(), root, root + 8);
        for (const BlasTriangle &t : b.tris) {
            float g[kTriGeoFloats], a[kTriAttrFloats];
            pack_triangle(t, g, a);
            out.tri_geo.insert(out.tri_geo.end(), g, g + kTriGeoFloats);
            out.tri_attr.insert(out.tri_attr.end(), a, a + kTriAttrFloats);
        }
        out.num_blas_nodes += b.nodes.size();
        out.num_triangles += b.tris.size();
    }
    // ---- instances (appendMeshInstance, scene.cpp:187-222)
    std::vector<HostInstance> inst((size_t)desc.num_instances);
    for (int ii = 0; ii < desc.num_instances; ++ii) {
        const hdr_instance_desc &d = desc.instances[ii];
        if (d.mesh < 0 || d.mesh >= desc.num_meshes) {
            err = "instance " + std::to_string(ii) + ": mesh index out of range";
            return false;
        }
        if (d.material < -1 || d.material >= desc.num_materials || d.light < -1 || d.light >= desc.num_lights) {
            err = "instance " + std::to_string(ii) + ": material/light index out of range";
            return false;
        }
        HostInstance &h = inst[ii];
        h.mesh = d.mesh;
        h.material = d.material;
        h.light = d.light;
        std::memcpy(h.xf, d.transform, sizeof(h.xf));
        gf_inverse4f(h.xf, h.inv);
        h.bounds = transform_bounds(ranges[d.mesh], h.xf);
        h.centroid = (h.bounds.mn + h.bounds.mx) * 0.5f;
        const float b6[6] = {h.bounds.mn.x, h.bounds.mn.y, h.bounds.mn.z, h.bounds.mx.x, h.bounds.mx.y, h.bounds.mx.z};
        out.inst_bounds.insert(out.inst_bounds.end(), b6, b6 + 6);
        float rec[32];
        std::memcpy(rec, h.inv, sizeof(h.inv));
        const float *T = h.xf;
        const float r4[16] = {T[0], T[1], T[2], as_float(node_base[d.mesh]), T[4], T[5], T[6], as_float(tri_base[d.mesh]),
                              T[8], T[9], T[10], as_float(d.material), as_float(d.light), as_float(blas_ok[d.mesh]),
                              as_float(wide_base[d.mesh]), as_float(d.mesh)};
        std::memcpy(rec + 16, r4, sizeof(r4));
        out.instances.insert(out.instances.end(), rec, rec + 32);
    }
    out.num_instances = desc.num_instances;
    // ---- TLAS (scene.cpp:333-407)
    if (desc.num_instances > 0) {
        std::vector<TlasNode> nodes;
        std::vector<int> idx((size_t)desc.num_instances);
        for (int i = 0; i < desc.num_instances; ++i) idx[i] = i;
        nodes.reserve((size_t)desc.num_instances * 2);
        nodes.push_back(TlasNode{});
        TlasBuilder tb{nodes, idx, inst};
        tb.subdivide(0, 0, desc.num_instances, 1);
        out.max_tlas_depth = tb.max_depth;
        for (const TlasNode &n : nodes) put_node(out.tlas_nodes, n.bounds, n.left, n.count);
        out.tlas_inst = idx;
        WideBuilder<TlasNode> wt{nodes, kWTagTlasLeaf, kWTagTlasNode, kTlasLeafCountBits, {}};
        wt.root(out.tlas_root);
        if (wt.overflow) {
            err = "too many instances for the wide TLAS encoding";
            return false;
        }
        out.max_tlas4_depth = wt.max_depth;
        out.tlas4 = std::move(wt.out);
    }
    // ---- materials: PreviewSurfaceMaterial::GetClosure inputs (preview_surface.cpp:61-127)
    out.num_materials = desc.num_materials;
    out.materials.assign((size_t)desc.num_materials * kMaterialFloats, 0.0f);
    // one copy per distinct texel array, as ImageTextureSamplerFactory loads each path once
    // (image_texture_sampler.cpp:14-33)
    std::map<std::tuple<const float *, int, int>, int> texture_offsets;
    for (int i = 0; i < desc.num_materials; ++i) {
        const hdr_material_desc &p = desc.materials[i];
        float *r = &out.materials[(size_t)i * kMaterialFloats];
        const V3 emission = V3{p.emission_color[0], p.emission_color[1], p.emission_color[2]} * p.emission;
        const float v[40] = {p.diffuse_color[0], p.diffuse_color[1], p.diffuse_color[2], p.metallic,
                             p.specular_color[0], p.specular_color[1], p.specular_color[2], p.specular,
                             emission.x, emission.y, emission.z, std::max(0.001f, p.roughness),
                             p.transmission_color[0], p.transmission_color[1], p.transmission_color[2], p.transmission,
                             p.coat_color[0], p.coat_color[1], p.coat_color[2], p.coat,
                             p.sheen_color[0], p.sheen_color[1], p.sheen_color[2], p.sheen,
                             p.subsurface_color[0], p.subsurface_color[1], p.subsurface_color[2], p.subsurface,
                             p.ior, p.opacity, p.transmission_depth, as_float(p.thin_walled),
                             p.coat_roughness, p.coat_ior, p.sheen_roughness, p.roughness,
                             0.0f, 0.0f, 0.0f, 0.0f};
        std::memcpy(r, v, sizeof(v));
        // textures (preview_surface.cpp:68-95): float offset into `textures` (-1 = none), width, height
        for (int k = 0; k < 4; ++k) {
            int off = -1;
            const int w = p.tex_width[k], h = p.tex_height[k];
            const auto known = texture_offsets.find(std::make_tuple(p.textures[k], w, h));
            if (p.textures[k] && w > 0 && h > 0 && known != texture_offsets.end()) {
                off = known->second;
            } else if (p.textures[k] && w > 0 && h > 0) {
                const size_t n = (size_t)w * (size_t)h * 3;
                if (out.textures.size() + n > (size_t)0x7fffffff || (size_t)w * (size_t)h > (size_t)0x7fffffff / 3) {
                    err = "material " + std::to_string(i) + ": textures exceed 2^31 floats";
                    return false;
                }
                off = (int)out.textures.size();
                out.textures.insert(out.textures.end(), p.textures[k], p.textures[k] + n);
                texture_offsets[std::make_tuple(p.textures[k], w, h)] = off;
            }
            r[36 + k] = as_float(off);
            r[40 + k] = as_float(off >= 0 ? w : 0);
            r[44 + k] = as_float(off >= 0 ? h : 0);
        }
    }
    // ---- lights (rect_light.cpp, point_light.cpp, distant_light.cpp, dome_light.cpp)
    out.num_lights = desc.num_lights;
    out.lights.assign((size_t)desc.num_lights * kLightFloats, 0.0f);
    for (int i = 0; i < desc.num_lights; ++i) {
        const hdr_light_desc &L = desc.lights[i];
        if (L.type < HDR_LIGHT_DISTANT || L.type > HDR_LIGHT_TRIANGLE) {
            err = "light " + std::to_string(i) + ": unknown type";
            return false;
        }
        if (!(L.temperature >= 0.0f) || !std::isfinite(L.temperature)) {
            err = "light " + std::to_string(i) + ": temperature must be finite and >= 0";
            return false;
        }
        float *r = &out.lights[(size_t)i * kLightFloats];
        float M[16];
        for (int k = 0; k < 16; ++k) M[k] = (float)L.transform[k];  // GfMatrix4f(GfMatrix4d)
        const float eff = L.intensity * std::exp2(L.exposure);       // LightParams::EffectiveIntensity
        const V3 color = V3{L.color[0], L.color[1], L.color[2]} * eff;
        const V3 lnormal = normalized(m4f_transform_dir(M, V3{0.0f, 0.0f, -1.0f}));
        const float area = L.type == HDR_LIGHT_TRIANGLE ? 0.5f * (L.width * L.height) : L.width * L.height;
        const float cone_rad = L.shaping_cone_angle * (float)(3.14159265358979323846 / 180.0);
        const float cos_cone = std::cos(cone_rad);
        const float cos_inner = std::cos(cone_rad * (1.0f - L.shaping_cone_softness));
        const int is_delta = (L.type == HDR_LIGHT_POINT || L.type == HDR_LIGHT_DISTANT) ? 1 : 0;
        const float head[16] = {as_float(L.type), as_float(is_delta), L.width, L.height,
                                color.x, color.y, color.z, area,
                                lnormal.x, lnormal.y, lnormal.z, L.shaping_cone_angle,
                                cos_cone, cos_inner, L.shaping_cone_softness, L.temperature};
        std::memcpy(r, head, sizeof(head));
        std::memcpy(r + 16, M, sizeof(M));
        // light params color & intensity kept separately for the dome's CompMult
        r[32] = L.color[0];
        r[33] = L.color[1];
        r[34] = L.color[2];
        r[35] = eff;
        if (L.type == HDR_LIGHT_DOME) {
            if (out.env_light < 0) out.env_light = i;
            if (L.texture && L.tex_width > 0 && L.tex_height > 0 && out.dome_width == 0) {
                // DomeLight::Prepare (dome_light.cpp:21-83)
                const int W = L.tex_width, H = L.tex_height;
                out.dome_width = W;
                out.dome_height = H;
                out.dome_pixels.assign(L.texture, L.texture + (size_t)W * H * 3);
                std::vector<float> &row = out.dome_row_cdf;
                std::vector<float> &col = out.dome_col_cdf;
                row.assign((size_t)H + 1, 0.0f);
                col.assign((size_t)H * (W + 1), 0.0f);
                const float *px = out.dome_pixels.data();
                float total = 0.0f;
                for (int y = 0; y < H; ++y) {
                    float row_lum = 0.0f;
                    const float sin_theta = std::sin(3.14159265358979323846 * (float)(y + 0.5f) / (float)H);
                    for (int x = 0; x < W; ++x) {
                        const size_t idx = (size_t)(y * W + x) * 3;
                        float lum = 0.2126f * px[idx] + 0.7152f * px[idx + 1] + 0.0722f * px[idx + 2];
                        lum *= sin_theta;
                        row_lum += lum;
                        col[(size_t)y * (W + 1) + x + 1] = col[(size_t)y * (W + 1) + x] + lum;
                    }
                    if (row_lum > 0)
                        for (int x = 0; x <= W; ++x) col[(size_t)y * (W + 1) + x] /= row_lum;
                    total += row_lum;
                    row[y + 1] = row[y] + row_lum;
                }
                if (total > 0)
                    for (int y = 0; y <= H; ++y) row[y] /= total;
                out.dome_total_lum = total;
            }
        }
    }
    return true;
}

}  // namespace hdr
