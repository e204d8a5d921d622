// Per-triangle data of BVH::Build (bvh.cpp:81-179) and the packed records the
// kernels read, shared by the host scene builder and the device BLAS build so
// both give the same bits.
#pragma once

#include <string.h>

#include "../../../include/hdrestir.h"
#include "gf.cuh"

namespace hdr {

struct BlasTriangle {  // BVHTriangle (bvh.h:22-31)
    V3 v0, v1, v2;
    V2 uv0, uv1, uv2;
    V3 n0, n1, n2;
    V3 c0, c1, c2;
    V3 dpdu, dpdv;
    V3 centroid;
    int material = -1;
};

// Triangle records: tri_geo is 12 floats (v0.xyz, e1.x | e1.yz, e2.xy | e2.z, 0, 0, 0),
// tri_attr 36 floats (geometric normal + smooth flag, corner normals / uvs / colours,
// dpdu + material, dpdv).
constexpr int kTriGeoFloats = 12, kTriAttrFloats = 36;

HDR_HD float int_bits_float(int v) {
#if defined(__CUDA_ARCH__)
    return __int_as_float(v);
#else
    float f;
    memcpy(&f, &v, sizeof(f));
    return f;
#endif
}

// false when a corner index is outside the points (the triangle is skipped)
HDR_HD bool make_triangle(const hdr_mesh_desc &m, int i, BlasTriangle &tri) {
    const int ntri = m.num_triangles;
    const int i0 = m.indices[3 * i + 0], i1 = m.indices[3 * i + 1], i2 = m.indices[3 * i + 2];
    const int np = m.num_points;
    if (i0 < 0 || i0 >= np || i1 < 0 || i1 >= np || i2 < 0 || i2 >= np) return false;
    const float *pts = m.points;
    tri.v0 = V3{pts[3 * i0], pts[3 * i0 + 1], pts[3 * i0 + 2]};
    tri.v1 = V3{pts[3 * i1], pts[3 * i1 + 1], pts[3 * i1 + 2]};
    tri.v2 = V3{pts[3 * i2], pts[3 * i2 + 1], pts[3 * i2 + 2]};

    const float *uv = m.uvs;
    if (m.num_uvs > 0) {
        if (m.num_uvs == ntri * 3) {
            tri.uv0 = V2{uv[2 * (i * 3 + 0)], uv[2 * (i * 3 + 0) + 1]};
            tri.uv1 = V2{uv[2 * (i * 3 + 1)], uv[2 * (i * 3 + 1) + 1]};
            tri.uv2 = V2{uv[2 * (i * 3 + 2)], uv[2 * (i * 3 + 2) + 1]};
        } else {
            tri.uv0 = (i0 < m.num_uvs) ? V2{uv[2 * i0], uv[2 * i0 + 1]} : V2{0.0f, 0.0f};
            tri.uv1 = (i1 < m.num_uvs) ? V2{uv[2 * i1], uv[2 * i1 + 1]} : V2{0.0f, 0.0f};
            tri.uv2 = (i2 < m.num_uvs) ? V2{uv[2 * i2], uv[2 * i2 + 1]} : V2{0.0f, 0.0f};
        }
    } else {
        tri.uv0 = tri.uv1 = tri.uv2 = V2{0.0f, 0.0f};
    }

    // per-corner when the array has 3 entries per triangle, else per point with `dflt` past its end
    auto corner3 = [&](const float *a, int n, V3 dflt, V3 &c0, V3 &c1, V3 &c2) {
        if (n == ntri * 3) {
            c0 = V3{a[9 * i + 0], a[9 * i + 1], a[9 * i + 2]};
            c1 = V3{a[9 * i + 3], a[9 * i + 4], a[9 * i + 5]};
            c2 = V3{a[9 * i + 6], a[9 * i + 7], a[9 * i + 8]};
        } else {
            c0 = (i0 < n) ? V3{a[3 * i0], a[3 * i0 + 1], a[3 * i0 + 2]} : dflt;
            c1 = (i1 < n) ? V3{a[3 * i1], a[3 * i1 + 1], a[3 * i1 + 2]} : dflt;
            c2 = (i2 < n) ? V3{a[3 * i2], a[3 * i2 + 1], a[3 * i2 + 2]} : dflt;
        }
    };
    if (m.num_normals > 0)
        corner3(m.normals, m.num_normals, V3{0.0f, 1.0f, 0.0f}, tri.n0, tri.n1, tri.n2);
    else
        tri.n0 = tri.n1 = tri.n2 = V3{0.0f, 0.0f, 0.0f};
    if (m.num_colors > 0)
        corner3(m.colors, m.num_colors, V3{1.0f, 1.0f, 1.0f}, tri.c0, tri.c1, tri.c2);
    else
        tri.c0 = tri.c1 = tri.c2 = V3{1.0f, 1.0f, 1.0f};

    const V3 edge1 = tri.v1 - tri.v0;
    const V3 edge2 = tri.v2 - tri.v0;
    const V2 duv1{tri.uv1.x - tri.uv0.x, tri.uv1.y - tri.uv0.y};
    const V2 duv2{tri.uv2.x - tri.uv0.x, tri.uv2.y - tri.uv0.y};
    float f = duv1.x * duv2.y - duv2.x * duv1.y;
    if (fabsf(f) > 1e-8f) {
        f = 1.0f / f;
        tri.dpdu = (edge1 * duv2.y - edge2 * duv1.y) * f;
        tri.dpdv = (edge2 * duv1.x - edge1 * duv2.x) * f;
        tri.dpdu = normalized(tri.dpdu);
        tri.dpdv = normalized(tri.dpdv);
    } else {
        const V3 n = normalized(cross(edge1, edge2));
        const V3 up = fabsf(n.y) < 0.999f ? V3{0, 1, 0} : V3{1, 0, 0};
        tri.dpdu = normalized(cross(up, n));
        tri.dpdv = normalized(cross(n, tri.dpdu));
    }
    tri.material = (i < m.num_material_indices && m.material_indices) ? m.material_indices[i] : -1;
    tri.centroid = div_d(tri.v0 + tri.v1 + tri.v2, 3.0);
    return true;
}

HDR_HD void pack_triangle(const BlasTriangle &t, float *geo, float *attr) {
    const V3 e1 = t.v1 - t.v0, e2 = t.v2 - t.v0;
    const float g[kTriGeoFloats] = {t.v0.x, t.v0.y, t.v0.z, e1.x, e1.y, e1.z, e2.x, e2.y, e2.z, 0.0f, 0.0f, 0.0f};
    for (int k = 0; k < kTriGeoFloats; ++k) geo[k] = g[k];
    // geometric normal of bvh.cpp:277 and the smooth-normal switch of bvh.cpp:281
    const V3 ng = normalized(cross(t.v1 - t.v0, t.v2 - t.v0));
    const float smooth = (length_sq(t.n0) > 1e-6f) ? 1.0f : 0.0f;
    const float a[kTriAttrFloats] = {
        ng.x,    ng.y,    ng.z,    smooth,  t.n0.x,   t.n0.y,   t.n0.z,   t.uv0.x,  t.n1.x,
        t.n1.y,  t.n1.z,  t.uv0.y, t.n2.x,  t.n2.y,   t.n2.z,   t.uv1.x,  t.c0.x,   t.c0.y,
        t.c0.z,  t.uv1.y, t.c1.x,  t.c1.y,  t.c1.z,   t.uv2.x,  t.c2.x,   t.c2.y,   t.c2.z,
        t.uv2.y, t.dpdu.x, t.dpdu.y, t.dpdu.z, int_bits_float(t.material), t.dpdv.x, t.dpdv.y, t.dpdv.z, 0.0f};
    for (int k = 0; k < kTriAttrFloats; ++k) attr[k] = a[k];
}

}  // namespace hdr
