// Shadow-ray BVH builder (see shadow_bvh.h).
#include "shadow_bvh.h"

#include "scene_build.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "../device/tri_setup.cuh"

namespace hdr {

namespace {

struct PrimBox {
    float lo[3], hi[3], c[3];
};

struct BNode {  // binary SAH node: inner (left >= 0: children left, left + 1) or leaf (prims first..first+count)
    float lo[3], hi[3];
    int left = -1, first = 0, count = 0;
};

inline float half_area(const float *lo, const float *hi) {
    const float x = hi[0] - lo[0], y = hi[1] - lo[1], z = hi[2] - lo[2];
    return (x < 0.0f || y < 0.0f || z < 0.0f) ? 0.0f : x * y + y * z + z * x;
}

inline void grow(float *lo, float *hi, const float *a, const float *b) {
    for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], a[k]);
        hi[k] = std::max(hi[k], b[k]);
    }
}

// Binned SAH (16 bins per axis over the centroid bounds), leaves of at most
// max_leaf primitives. order[] is permuted into leaf order.
void build_binary(const std::vector<PrimBox> &prims, int max_leaf, std::vector<BNode> &nodes, std::vector<int> &order) {
    constexpr int kBins = 16;
    const int n = (int)prims.size();
    order.resize((size_t)n);
    for (int i = 0; i < n; ++i) order[(size_t)i] = i;
    nodes.clear();
    nodes.reserve((size_t)std::max(1, 2 * n / std::max(1, max_leaf / 2)));
    nodes.emplace_back();
    struct Task {
        int node, start, end;
    };
    std::vector<Task> todo{{0, 0, n}};
    while (!todo.empty()) {
        const Task t = todo.back();
        todo.pop_back();
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int i = t.start; i < t.end; ++i) {
            const PrimBox &p = prims[(size_t)order[(size_t)i]];
            grow(lo, hi, p.lo, p.hi);
            grow(clo, chi, p.c, p.c);
        }
        BNode &nd = nodes[(size_t)t.node];
        std::memcpy(nd.lo, lo, sizeof(lo));
        std::memcpy(nd.hi, hi, sizeof(hi));
        const int count = t.end - t.start;
        if (count <= max_leaf) {
            nd.left = -1;
            nd.first = t.start;
            nd.count = count;
            continue;
        }
        float best = FLT_MAX;
        int best_axis = -1, best_bin = 0;
        for (int ax = 0; ax < 3; ++ax) {
            const float extent = chi[ax] - clo[ax];
            if (!(extent > 0.0f)) continue;
            const float scale = kBins / extent;
            int bc[kBins] = {};
            float blo[kBins][3], bhi[kBins][3];
            for (int b = 0; b < kBins; ++b)
                for (int k = 0; k < 3; ++k) blo[b][k] = FLT_MAX, bhi[b][k] = -FLT_MAX;
            for (int i = t.start; i < t.end; ++i) {
                const PrimBox &p = prims[(size_t)order[(size_t)i]];
                const int b = std::min(kBins - 1, std::max(0, (int)((p.c[ax] - clo[ax]) * scale)));
                ++bc[b];
                grow(blo[b], bhi[b], p.lo, p.hi);
            }
            float r_area[kBins];
            int r_count[kBins];
            float alo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, ahi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
            int acc = 0;
            for (int b = kBins - 1; b > 0; --b) {
                acc += bc[b];
                if (bc[b]) grow(alo, ahi, blo[b], bhi[b]);
                r_area[b] = half_area(alo, ahi);
                r_count[b] = acc;
            }
            for (int k = 0; k < 3; ++k) alo[k] = FLT_MAX, ahi[k] = -FLT_MAX;
            acc = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                acc += bc[b];
                if (bc[b]) grow(alo, ahi, blo[b], bhi[b]);
                if (!acc || !r_count[b + 1]) continue;
                const float cost = half_area(alo, ahi) * (float)acc + r_area[b + 1] * (float)r_count[b + 1];
                if (cost < best) {
                    best = cost;
                    best_axis = ax;
                    best_bin = b + 1;
                }
            }
        }
        int mid = (t.start + t.end) / 2;
        if (best_axis >= 0) {
            const float scale = kBins / (chi[best_axis] - clo[best_axis]);
            auto in_left = [&](int pi) {
                const int b = std::min(kBins - 1, std::max(0, (int)((prims[(size_t)pi].c[best_axis] - clo[best_axis]) * scale)));
                return b < best_bin;
            };
            const int m = (int)(std::partition(order.begin() + t.start, order.begin() + t.end, in_left) - order.begin());
            if (m > t.start && m < t.end) mid = m;
        }
        const int l = (int)nodes.size();
        nodes.emplace_back();
        nodes.emplace_back();
        nodes[(size_t)t.node].left = l;
        nodes[(size_t)t.node].count = 0;
        todo.push_back({l + 1, mid, t.end});
        todo.push_back({l, t.start, mid});
    }
}

inline float bits_float(int v) {
    float f;
    std::memcpy(&f, &v, sizeof(f));
    return f;
}

// Collapses a binary tree into 4-wide records appended to `out`. leaf_code(node)
// gives a binary leaf's child code. Returns the depth of the emitted subtree.
struct Collapser {
    const std::vector<BNode> &bn;
    std::vector<float> &out;
    size_t limit;  // maximum nodes in `out` (the TLAS region), 0 = none
    bool overflow = false;
    template <class LeafCode>
    int emit(int b, LeafCode &&leaf_code, int &index) {
        int ch[4], nch = 0;
        if (bn[(size_t)b].left < 0) {
            ch[nch++] = b;  // a tree that is one leaf: a root with a single child
        } else {
            ch[nch++] = bn[(size_t)b].left;
            ch[nch++] = bn[(size_t)b].left + 1;
            while (nch < 4) {  // open the inner child with the largest surface area
                int pick = -1;
                float area = -1.0f;
                for (int k = 0; k < nch; ++k) {
                    const BNode &c = bn[(size_t)ch[k]];
                    if (c.left >= 0 && half_area(c.lo, c.hi) > area) {
                        area = half_area(c.lo, c.hi);
                        pick = k;
                    }
                }
                if (pick < 0) break;
                const int x = ch[pick];
                ch[pick] = bn[(size_t)x].left;
                ch[nch++] = bn[(size_t)x].left + 1;
            }
        }
        index = (int)(out.size() / kSh4NodeFloats);
        if (limit && (size_t)index >= limit) {
            overflow = true;
            return 0;
        }
        out.resize(out.size() + kSh4NodeFloats);
        float rec[kSh4NodeFloats];
        for (int k = 0; k < 4; ++k) {
            rec[k] = rec[8 + k] = rec[16 + k] = FLT_MAX;
            rec[4 + k] = rec[12 + k] = rec[20 + k] = -FLT_MAX;
            rec[24 + k] = bits_float(-1);
        }
        int depth = 0;
        for (int k = 0; k < nch; ++k) {
            const BNode &c = bn[(size_t)ch[k]];
            rec[k] = c.lo[0], rec[4 + k] = c.hi[0];
            rec[8 + k] = c.lo[1], rec[12 + k] = c.hi[1];
            rec[16 + k] = c.lo[2], rec[20 + k] = c.hi[2];
            int code;
            if (c.left < 0) {
                code = leaf_code(ch[k]);
            } else {
                int idx = 0;
                depth = std::max(depth, emit(ch[k], leaf_code, idx));
                code = idx;
            }
            rec[24 + k] = bits_float(code);
        }
        std::memcpy(&out[(size_t)index * kSh4NodeFloats], rec, sizeof(rec));
        return depth + 1;
    }
};

}  // namespace

bool rebuild_shadow_tlas(const std::vector<float> &inst_bounds, const std::vector<int> &inst_root, int blas_depth,
                         std::vector<float> &tlas_nodes, int tlas_capacity, int &tlas_depth) {
    std::vector<PrimBox> prims;
    std::vector<int> prim_inst;
    for (size_t i = 0; i < inst_root.size(); ++i) {
        if (inst_root[i] < 0) continue;
        PrimBox p;
        for (int k = 0; k < 3; ++k) {
            p.lo[k] = inst_bounds[6 * i + k];
            p.hi[k] = inst_bounds[6 * i + 3 + k];
            p.c[k] = 0.5f * (p.lo[k] + p.hi[k]);
        }
        prims.push_back(p);
        prim_inst.push_back((int)i);
    }
    tlas_nodes.clear();
    tlas_depth = 0;
    if (!prims.empty()) {
        std::vector<BNode> bn;
        std::vector<int> order;
        build_binary(prims, 1, bn, order);
        Collapser col{bn, tlas_nodes, (size_t)tlas_capacity};
        int root = 0;
        tlas_depth = col.emit(
            0, [&](int b) { return ~((prim_inst[(size_t)order[(size_t)bn[(size_t)b].first]] << 2) | 0); }, root);
        if (col.overflow) return false;
    } else {  // nothing to hit: a root whose slots are all empty
        tlas_nodes.resize(kSh4NodeFloats);
        for (int k = 0; k < 4; ++k) {
            tlas_nodes[k] = tlas_nodes[8 + k] = tlas_nodes[16 + k] = FLT_MAX;
            tlas_nodes[4 + k] = tlas_nodes[12 + k] = tlas_nodes[20 + k] = -FLT_MAX;
            tlas_nodes[24 + k] = bits_float(-1);
        }
        tlas_depth = 1;
    }
    // a walk holds at most 1 + 3 entries per level it has descended
    return 1 + 3 * (tlas_depth + blas_depth) <= kSh4Stack;
}

void shadow_ranks(const std::vector<int> &tlas_inst, int num_instances, std::vector<int> &rank) {
    rank.assign((size_t)std::max(0, num_instances), 0x7fffffff);
    for (size_t k = 0; k < tlas_inst.size(); ++k) {
        const int i = tlas_inst[k];
        if (i >= 0 && i < num_instances && rank[(size_t)i] == 0x7fffffff) rank[(size_t)i] = (int)k;
    }
}

bool build_shadow_bvh(const hdr_scene_desc &desc, const FlatScene &flat, ShadowBvh &out, std::string &err) {
    out = ShadowBvh{};
    const int n_inst = desc.num_instances;
    out.tlas_capacity = std::max(1, n_inst);
    out.nodes.assign((size_t)out.tlas_capacity * kSh4NodeFloats, 0.0f);
    std::vector<int> mesh_root((size_t)std::max(0, desc.num_meshes), -1);
    const bool host_geo = !flat.tri_geo.empty() || flat.num_triangles == 0;
    for (int mi = 0; mi < desc.num_meshes; ++mi) {
        // the mesh's triangle records in the reference's BLAS order
        std::vector<float> geo;
        if (host_geo) {
            const size_t b = (size_t)flat.mesh_tri_base[(size_t)mi], n = (size_t)flat.mesh_tri_count[(size_t)mi];
            geo.assign(flat.tri_geo.begin() + (long)(b * kTriGeoFloats),
                       flat.tri_geo.begin() + (long)((b + n) * kTriGeoFloats));
        } else {  // the BLAS was built on the device: the host build gives the same order
            const Blas blas = build_blas(desc.meshes[mi]);
            geo.resize(blas.tris.size() * kTriGeoFloats);
            float a[kTriAttrFloats];
            for (size_t t = 0; t < blas.tris.size(); ++t) pack_triangle(blas.tris[t], &geo[t * kTriGeoFloats], a);
        }
        const size_t nt = geo.size() / kTriGeoFloats;
        if (nt == 0) continue;
        std::vector<PrimBox> prims(nt);
        for (size_t t = 0; t < nt; ++t) {
            const float *g = &geo[t * kTriGeoFloats];
            const float v[3][3] = {{g[0], g[1], g[2]},
                                   {g[0] + g[3], g[1] + g[4], g[2] + g[5]},
                                   {g[0] + g[6], g[1] + g[7], g[2] + g[8]}};
            PrimBox &p = prims[t];
            for (int k = 0; k < 3; ++k) p.lo[k] = FLT_MAX, p.hi[k] = -FLT_MAX;
            // vertices v0 + e1 / v0 + e2 may round: widen the box by a relative ulp margin
            for (const auto &x : v) grow(p.lo, p.hi, x, x);
            for (int k = 0; k < 3; ++k) {
                const float m = (std::fabs(p.lo[k]) + std::fabs(p.hi[k])) * 2.4e-7f + 1e-30f;
                p.lo[k] -= m;
                p.hi[k] += m;
                p.c[k] = 0.5f * (p.lo[k] + p.hi[k]);
            }
        }
        std::vector<BNode> bn;
        std::vector<int> order;
        build_binary(prims, 4, bn, order);
        Collapser col{bn, out.nodes, 0};
        int root = 0;
        const size_t tri_base = out.tris.size() / kTriGeoFloats;
        if (tri_base + nt >= ((size_t)1 << 27)) {  // leaf entries: (first << 4) | ... fits 31 bits
            err = "too many triangles for the shadow BVH encoding";
            return false;
        }
        // leaf triangles go to `tris` in leaf order as the collapse meets them, each
        // with its reference-order index in float 9
        const int depth = col.emit(
            0,
            [&](int b) {
                const BNode &lf = bn[(size_t)b];
                const int first = (int)(out.tris.size() / kTriGeoFloats);
                for (int q = 0; q < lf.count; ++q) {
                    const int t = order[(size_t)(lf.first + q)];
                    const float *g = &geo[(size_t)t * kTriGeoFloats];
                    float rec[kTriGeoFloats];
                    std::memcpy(rec, g, sizeof(rec));
                    rec[9] = bits_float(t);
                    rec[10] = rec[11] = 0.0f;
                    out.tris.insert(out.tris.end(), rec, rec + kTriGeoFloats);
                }
                return ~((first << 2) | (lf.count - 1));
            },
            root);
        mesh_root[(size_t)mi] = root;
        out.blas_depth = std::max(out.blas_depth, depth);
    }
    out.inst_root.assign((size_t)std::max(0, n_inst), -1);
    for (int i = 0; i < n_inst; ++i) {
        const int mesh = desc.instances[i].mesh;
        if (mesh >= 0 && mesh < desc.num_meshes) out.inst_root[(size_t)i] = mesh_root[(size_t)mesh];
    }
    shadow_ranks(flat.tlas_inst, n_inst, out.inst_rank);
    std::vector<float> tlas;
    const bool fits = rebuild_shadow_tlas(flat.inst_bounds, out.inst_root, out.blas_depth, tlas, out.tlas_capacity,
                                          out.tlas_depth);
    if (!fits) return true;  // not an error: the reference trees serve these queries too
    std::memcpy(out.nodes.data(), tlas.data(), tlas.size() * sizeof(float));
    out.ok = true;
    return true;
}

}  // namespace hdr
