/*
 * CPU oracle — TEST INFRASTRUCTURE (see orc_core.h). RNG, spectra, scene
 * build and scene query, restated from the reference.
 */
#include "orc_core.h"

#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------------
 * 4x4 inverse by cofactors in double. The reference calls OpenUSD's
 * GfMatrix4d/4f::GetInverse (scene.cpp:208, raycast_pass.cpp:86-87); OpenUSD
 * is not vendored, so this is the Gf semantics every component here agrees
 * on (singular -> scale FLT_MAX).
 * ------------------------------------------------------------------------- */
void orc_inverse4d(const double *m, double *o) {
    double s0 = m[0] * m[5] - m[4] * m[1], s1 = m[0] * m[6] - m[4] * m[2], s2 = m[0] * m[7] - m[4] * m[3];
    double s3 = m[1] * m[6] - m[5] * m[2], s4 = m[1] * m[7] - m[5] * m[3], s5 = m[2] * m[7] - m[6] * m[3];
    double c5 = m[10] * m[15] - m[14] * m[11], c4 = m[9] * m[15] - m[13] * m[11], c3 = m[9] * m[14] - m[13] * m[10];
    double c2 = m[8] * m[15] - m[12] * m[11], c1 = m[8] * m[14] - m[12] * m[10], c0 = m[8] * m[13] - m[12] * m[9];
    double det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
    if (!(fabs(det) > 0.0)) {
        memset(o, 0, 16 * sizeof(double));
        o[0] = o[5] = o[10] = 3.402823466e+38;
        o[15] = 1.0;
        return;
    }
    double r = 1.0 / det;
    o[0] = (m[5] * c5 - m[6] * c4 + m[7] * c3) * r;
    o[1] = (-m[1] * c5 + m[2] * c4 - m[3] * c3) * r;
    o[2] = (m[13] * s5 - m[14] * s4 + m[15] * s3) * r;
    o[3] = (-m[9] * s5 + m[10] * s4 - m[11] * s3) * r;
    o[4] = (-m[4] * c5 + m[6] * c2 - m[7] * c1) * r;
    o[5] = (m[0] * c5 - m[2] * c2 + m[3] * c1) * r;
    o[6] = (-m[12] * s5 + m[14] * s2 - m[15] * s1) * r;
    o[7] = (m[8] * s5 - m[10] * s2 + m[11] * s1) * r;
    o[8] = (m[4] * c4 - m[5] * c2 + m[7] * c0) * r;
    o[9] = (-m[0] * c4 + m[1] * c2 - m[3] * c0) * r;
    o[10] = (m[12] * s4 - m[13] * s2 + m[15] * s0) * r;
    o[11] = (-m[8] * s4 + m[9] * s2 - m[11] * s0) * r;
    o[12] = (-m[4] * c3 + m[5] * c1 - m[6] * c0) * r;
    o[13] = (m[0] * c3 - m[1] * c1 + m[2] * c0) * r;
    o[14] = (-m[12] * s3 + m[13] * s1 - m[14] * s0) * r;
    o[15] = (m[8] * s3 - m[9] * s1 + m[10] * s0) * r;
}

/* ---------------------------------------------------------------------------
 * std::mt19937_64 (the algorithm fixed by the C++ standard) and libstdc++'s
 * generate_canonical<float, 24>: float(y) * 2^-64, clamped below 1.
 * core/rng.h:13-55
 * ------------------------------------------------------------------------- */
void orc_rng_seed(orc_rng *r, uint32_t seed) {
    r->mt[0] = (uint64_t)seed;
    for (int i = 1; i < 312; ++i) r->mt[i] = 6364136223846793005ULL * (r->mt[i - 1] ^ (r->mt[i - 1] >> 62)) + (uint64_t)i;
    r->idx = 312;
}

static void orc_rng_twist(orc_rng *r) {
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL, A = 0xB5026F5AA96619E9ULL;
    uint64_t *mt = r->mt;
    for (int k = 0; k < 312; ++k) {
        uint64_t y = (mt[k] & UM) | (mt[(k + 1) % 312] & LM);
        mt[k] = mt[(k + 156) % 312] ^ (y >> 1) ^ ((y & 1ULL) ? A : 0ULL);
    }
    r->idx = 0;
}

uint64_t orc_rng_u64(orc_rng *r) {
    if (r->idx >= 312) orc_rng_twist(r);
    uint64_t y = r->mt[r->idx++];
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= (y >> 43);
    return y;
}

float orc_rng_float(orc_rng *r) {
    float f = (float)orc_rng_u64(r) / 18446744073709551616.0f;
    return (f >= 1.0f) ? nextafterf(1.0f, 0.0f) : f;
}

/* ---------------------------------------------------------------------------
 * Spectra: core/spectrum.h:24-37, core/spectrum.cpp:4-109
 * ------------------------------------------------------------------------- */
olambda orc_sample_wavelengths(float u) {
    olambda w;
    w.l[0] = 360.0f + u * (830.0f - 360.0f);
    for (int i = 1; i < 4; ++i) {
        w.l[i] = w.l[0] + ((float)i * (830.0f - 360.0f) / 4);
        if (w.l[i] > 830.0f) w.l[i] -= (830.0f - 360.0f);
    }
    return w;
}

static float xfit(float w) {
    float t1 = (w - 442.0f) * ((w < 442.0f) ? 0.0624f : 0.0374f);
    float t2 = (w - 599.8f) * ((w < 599.8f) ? 0.0264f : 0.0323f);
    float t3 = (w - 501.1f) * ((w < 501.1f) ? 0.0490f : 0.0382f);
    return 0.362f * expf(-0.5f * t1 * t1) + 1.056f * expf(-0.5f * t2 * t2) - 0.065f * expf(-0.5f * t3 * t3);
}
static float yfit(float w) {
    float t1 = (w - 568.8f) * ((w < 568.8f) ? 0.0213f : 0.0247f);
    float t2 = (w - 530.9f) * ((w < 530.9f) ? 0.0613f : 0.0322f);
    return 0.821f * expf(-0.5f * t1 * t1) + 0.286f * expf(-0.5f * t2 * t2);
}
static float zfit(float w) {
    float t1 = (w - 437.0f) * ((w < 437.0f) ? 0.0845f : 0.0278f);
    float t2 = (w - 459.0f) * ((w < 459.0f) ? 0.0385f : 0.0725f);
    return 1.217f * expf(-0.5f * t1 * t1) + 0.681f * expf(-0.5f * t2 * t2);
}

ov3 orc_spectrum_to_rgb(ospec s, const olambda *w) {
    float X = 0.0f, Y = 0.0f, Z = 0.0f;
    float weight = (830.0f - 360.0f) / 4;
    weight /= 106.856f;
    for (int i = 0; i < 4; ++i) {
        float l = w->l[i], v = s.v[i];
        X += v * xfit(l);
        Y += v * yfit(l);
        Z += v * zfit(l);
    }
    X *= weight;
    Y *= weight;
    Z *= weight;
    float r = 3.2404542f * X - 1.5371385f * Y - 0.4985314f * Z;
    float g = -0.9692660f * X + 1.8760108f * Y + 0.0415560f * Z;
    float b = 0.0556434f * X - 0.2040259f * Y + 1.0572252f * Z;
    r /= 1.198185f;
    g /= 0.950366f;
    b /= 0.907827f;
    return V(omax(0.0f, r), omax(0.0f, g), omax(0.0f, b));
}

static float gauss(float x, float c, float sigma) {
    float t = (x - c) / sigma;
    return expf(-0.5f * t * t);
}

ospec orc_rgb_to_spectrum(ov3 rgb, const olambda *w) {
    ospec s;
    float white = omin(rgb.x, omin(rgb.y, rgb.z));
    ov3 rem = V(rgb.x - white, rgb.y - white, rgb.z - white);
    for (int i = 0; i < 4; ++i) {
        float l = w->l[i];
        float val = white;
        val += rem.x * gauss(l, 615.0f, 20.0f) * 1.295f;
        val += rem.y * gauss(l, 540.0f, 20.0f) * 1.556f;
        val += rem.z * gauss(l, 460.0f, 20.0f) * 1.382f;
        s.v[i] = omax(0.0f, val);
    }
    return s;
}

float orc_spectrum_luminance(ospec s, const olambda *w) {
    ov3 c = orc_spectrum_to_rgb(s, w);
    return omax(0.0f, 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z);
}

/* ---------------------------------------------------------------------------
 * BLAS build: BVH::Build / _Subdivide (renderContext/bvh.cpp:66-208)
 * ------------------------------------------------------------------------- */
static void range_empty(ov3 *mn, ov3 *mx) {
    *mn = V(3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f);
    *mx = V(-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f);
}
static void range_extend(ov3 *mn, ov3 *mx, ov3 p) {
    if (p.x < mn->x) mn->x = p.x;
    if (p.y < mn->y) mn->y = p.y;
    if (p.z < mn->z) mn->z = p.z;
    if (p.x > mx->x) mx->x = p.x;
    if (p.y > mx->y) mx->y = p.y;
    if (p.z > mx->z) mx->z = p.z;
}
static int range_is_empty(ov3 mn, ov3 mx) { return mn.x > mx.x || mn.y > mx.y || mn.z > mx.z; }

static int push_node(onode **nodes, int *n, int *cap) {
    if (*n == *cap) {
        *cap = *cap ? *cap * 2 : 64;
        *nodes = (onode *)realloc(*nodes, (size_t)*cap * sizeof(onode));
    }
    memset(&(*nodes)[*n], 0, sizeof(onode));
    range_empty(&(*nodes)[*n].mn, &(*nodes)[*n].mx);
    return (*n)++;
}

static void blas_subdivide(oblas *b, int ni, int start, int end) {
    onode *node = &b->nodes[ni];
    range_empty(&node->mn, &node->mx);
    for (int i = start; i < end; ++i) {
        range_extend(&node->mn, &node->mx, b->tris[i].v0);
        range_extend(&node->mn, &node->mx, b->tris[i].v1);
        range_extend(&node->mn, &node->mx, b->tris[i].v2);
    }
    int count = end - start;
    if (count <= 4) {
        node->left = -start - 1;
        node->count = count;
        return;
    }
    ov3 size = vsub(node->mx, node->mn);
    int axis = 0;
    if (size.y > size.x) axis = 1;
    if (size.z > vcomp(size, axis)) axis = 2;
    float split = vcomp(node->mn, axis) + vcomp(size, axis) * 0.5f;
    int i = start, j = end - 1;
    while (i <= j) {
        if (vcomp(b->tris[i].centroid, axis) < split) {
            i++;
        } else {
            otri t = b->tris[i];
            b->tris[i] = b->tris[j];
            b->tris[j] = t;
            j--;
        }
    }
    int left_count = i - start;
    if (left_count == 0 || left_count == count) i = start + count / 2;
    int li = push_node(&b->nodes, &b->n_nodes, &b->cap_nodes);
    push_node(&b->nodes, &b->n_nodes, &b->cap_nodes);
    b->nodes[ni].left = li;
    b->nodes[ni].count = 0;
    blas_subdivide(b, li, start, i);
    blas_subdivide(b, li + 1, i, end);
}

static void blas_build(oblas *b, const hdr_mesh_desc *m) {
    memset(b, 0, sizeof(*b));
    range_empty(&b->range_mn, &b->range_mx);
    for (int i = 0; i < m->num_triangles; ++i)
        for (int k = 0; k < 3; ++k) {
            int p = m->indices[3 * i + k];
            if (p >= 0 && p < m->num_points)
                range_extend(&b->range_mn, &b->range_mx, V(m->points[3 * p], m->points[3 * p + 1], m->points[3 * p + 2]));
        }
    if (m->num_triangles <= 0 || m->num_points <= 0) return;
    b->tris = (otri *)calloc((size_t)m->num_triangles, sizeof(otri));
    int nt = m->num_triangles, np = m->num_points;
    for (int i = 0; i < nt; ++i) {
        int i0 = m->indices[3 * i], i1 = m->indices[3 * i + 1], i2 = m->indices[3 * i + 2];
        if (i0 < 0 || i0 >= np || i1 < 0 || i1 >= np || i2 < 0 || i2 >= np) continue;
        otri t;
        memset(&t, 0, sizeof(t));
#define PT(k) V(m->points[3 * (k)], m->points[3 * (k) + 1], m->points[3 * (k) + 2])
        t.v0 = PT(i0);
        t.v1 = PT(i1);
        t.v2 = PT(i2);
#undef PT
        if (m->num_uvs > 0) {
            const float *u = m->uvs;
            if (m->num_uvs == nt * 3) {
                t.uv0 = (ov2){u[6 * i], u[6 * i + 1]};
                t.uv1 = (ov2){u[6 * i + 2], u[6 * i + 3]};
                t.uv2 = (ov2){u[6 * i + 4], u[6 * i + 5]};
            } else {
                t.uv0 = i0 < m->num_uvs ? (ov2){u[2 * i0], u[2 * i0 + 1]} : (ov2){0, 0};
                t.uv1 = i1 < m->num_uvs ? (ov2){u[2 * i1], u[2 * i1 + 1]} : (ov2){0, 0};
                t.uv2 = i2 < m->num_uvs ? (ov2){u[2 * i2], u[2 * i2 + 1]} : (ov2){0, 0};
            }
        }
#define A3(a, k) V((a)[3 * (k)], (a)[3 * (k) + 1], (a)[3 * (k) + 2])
        if (m->num_normals > 0) {
            if (m->num_normals == nt * 3) {
                t.n0 = A3(m->normals, 3 * i);
                t.n1 = A3(m->normals, 3 * i + 1);
                t.n2 = A3(m->normals, 3 * i + 2);
            } else {
                t.n0 = i0 < m->num_normals ? A3(m->normals, i0) : V(0, 1, 0);
                t.n1 = i1 < m->num_normals ? A3(m->normals, i1) : V(0, 1, 0);
                t.n2 = i2 < m->num_normals ? A3(m->normals, i2) : V(0, 1, 0);
            }
        }
        if (m->num_colors > 0) {
            if (m->num_colors == nt * 3) {
                t.c0 = A3(m->colors, 3 * i);
                t.c1 = A3(m->colors, 3 * i + 1);
                t.c2 = A3(m->colors, 3 * i + 2);
            } else {
                t.c0 = i0 < m->num_colors ? A3(m->colors, i0) : V(1, 1, 1);
                t.c1 = i1 < m->num_colors ? A3(m->colors, i1) : V(1, 1, 1);
                t.c2 = i2 < m->num_colors ? A3(m->colors, i2) : V(1, 1, 1);
            }
        } else {
            t.c0 = t.c1 = t.c2 = V(1, 1, 1);
        }
#undef A3
        ov3 e1 = vsub(t.v1, t.v0), e2 = vsub(t.v2, t.v0);
        ov2 d1 = {t.uv1.x - t.uv0.x, t.uv1.y - t.uv0.y}, d2 = {t.uv2.x - t.uv0.x, t.uv2.y - t.uv0.y};
        float f = d1.x * d2.y - d2.x * d1.y;
        if (fabsf(f) > 1e-8f) {
            f = 1.0f / f;
            t.dpdu = vnorm(vmulf(vsub(vmulf(e1, d2.y), vmulf(e2, d1.y)), f));
            t.dpdv = vnorm(vmulf(vsub(vmulf(e2, d1.x), vmulf(e1, d2.x)), f));
        } else {
            ov3 n = vnorm(vcross(e1, e2));
            ov3 up = fabsf(n.y) < 0.999f ? V(0, 1, 0) : V(1, 0, 0);
            t.dpdu = vnorm(vcross(up, n));
            t.dpdv = vnorm(vcross(n, t.dpdu));
        }
        t.material = (m->material_indices && i < m->num_material_indices) ? m->material_indices[i] : -1;
        t.centroid = vdivd(vadd(vadd(t.v0, t.v1), t.v2), 3.0);
        b->tris[b->n_tris++] = t;
    }
    if (b->n_tris == 0) return;
    push_node(&b->nodes, &b->n_nodes, &b->cap_nodes);
    blas_subdivide(b, 0, 0, b->n_tris);
}

/* ---------------------------------------------------------------------------
 * TLAS build: Scene::_BuildTLAS / _SubdivideTLAS (scene/scene.cpp:333-407)
 * ------------------------------------------------------------------------- */
static void tlas_subdivide(orc_scene *s, int ni, int start, int end) {
    int li = push_node(&s->tlas, &s->n_tlas, &s->cap_tlas);
    push_node(&s->tlas, &s->n_tlas, &s->cap_tlas);
    onode *node = &s->tlas[ni];
    node->left = li;
    node->count = 0;
    range_empty(&node->mn, &node->mx);
    for (int i = start; i < end; ++i) {
        const oinst *in = &s->inst[s->tlas_idx[i]];
        range_extend(&node->mn, &node->mx, in->bmn);
        range_extend(&node->mn, &node->mx, in->bmx);
    }
    int count = end - start;
    if (count <= 2) {
        node->left = -start - 1;
        node->count = count;
        return;
    }
    ov3 size = vsub(node->mx, node->mn);
    int axis = 0;
    if (size.y > size.x) axis = 1;
    if (size.z > vcomp(size, axis)) axis = 2;
    float split = vcomp(node->mn, axis) + vcomp(size, axis) * 0.5f;
    int i = start, j = end - 1;
    while (i <= j) {
        if (vcomp(s->inst[s->tlas_idx[i]].centroid, axis) < split) {
            ++i;
        } else {
            int t = s->tlas_idx[i];
            s->tlas_idx[i] = s->tlas_idx[j];
            s->tlas_idx[j] = t;
            --j;
        }
    }
    if (i == start || i == end) i = start + count / 2;
    tlas_subdivide(s, li, start, i);
    tlas_subdivide(s, li + 1, i, end);
}

/* DomeLight::Prepare (scene/dome_light.cpp:21-83) */
static void dome_prepare(olight *L, const hdr_light_desc *d) {
    if (!d->texture || d->tex_width <= 0 || d->tex_height <= 0) return;
    int W = d->tex_width, H = d->tex_height;
    L->w = W;
    L->h = H;
    L->pixels = (float *)malloc((size_t)W * H * 3 * sizeof(float));
    memcpy(L->pixels, d->texture, (size_t)W * H * 3 * sizeof(float));
    L->row_cdf = (float *)calloc((size_t)H + 1, sizeof(float));
    L->col_cdf = (float *)calloc((size_t)H * (W + 1), sizeof(float));
    float total = 0.0f;
    for (int y = 0; y < H; ++y) {
        float row = 0.0f;
        float sin_t = (float)sin(3.14159265358979323846 * (float)(y + 0.5f) / (float)H);
        for (int x = 0; x < W; ++x) {
            size_t idx = (size_t)(y * W + x) * 3;
            float lum = 0.2126f * L->pixels[idx] + 0.7152f * L->pixels[idx + 1] + 0.0722f * L->pixels[idx + 2];
            lum *= sin_t;
            row += lum;
            L->col_cdf[(size_t)y * (W + 1) + x + 1] = L->col_cdf[(size_t)y * (W + 1) + x] + lum;
        }
        if (row > 0)
            for (int x = 0; x <= W; ++x) L->col_cdf[(size_t)y * (W + 1) + x] /= row;
        total += row;
        L->row_cdf[y + 1] = L->row_cdf[y] + row;
    }
    if (total > 0)
        for (int y = 0; y <= H; ++y) L->row_cdf[y] /= total;
    L->total_lum = total;
}

orc_scene *orc_scene_create(const hdr_scene_desc *d) {
    orc_scene *s = (orc_scene *)calloc(1, sizeof(orc_scene));
    s->n_mesh = d->num_meshes;
    s->blas = (oblas *)calloc((size_t)(d->num_meshes > 0 ? d->num_meshes : 1), sizeof(oblas));
    for (int i = 0; i < d->num_meshes; ++i) blas_build(&s->blas[i], &d->meshes[i]);
    s->n_inst = d->num_instances;
    s->inst = (oinst *)calloc((size_t)(d->num_instances > 0 ? d->num_instances : 1), sizeof(oinst));
    for (int i = 0; i < d->num_instances; ++i) {
        /* appendMeshInstance (scene.cpp:187-222) */
        const hdr_instance_desc *id = &d->instances[i];
        oinst *in = &s->inst[i];
        in->mesh = id->mesh;
        in->material = id->material;
        in->light = id->light;
        memcpy(in->xf, id->transform, sizeof(in->xf));
        double md[16], od[16];
        for (int k = 0; k < 16; ++k) md[k] = (double)in->xf[k];
        orc_inverse4d(md, od);
        for (int k = 0; k < 16; ++k) in->inv[k] = (float)od[k];
        /* Scene::_TransformBounds (scene.cpp:101-116) */
        const oblas *b = &s->blas[id->mesh];
        range_empty(&in->bmn, &in->bmx);
        if (!range_is_empty(b->range_mn, b->range_mx)) {
            ov3 mn = b->range_mn, mx = b->range_mx;
            ov3 c[8] = {V(mn.x, mn.y, mn.z), V(mx.x, mn.y, mn.z), V(mn.x, mx.y, mn.z), V(mx.x, mx.y, mn.z),
                        V(mn.x, mn.y, mx.z), V(mx.x, mn.y, mx.z), V(mn.x, mx.y, mx.z), V(mx.x, mx.y, mx.z)};
            for (int k = 0; k < 8; ++k) range_extend(&in->bmn, &in->bmx, m4f_xform(in->xf, c[k]));
        } else {
            in->bmn = b->range_mn;
            in->bmx = b->range_mx;
        }
        in->centroid = vmulf(vadd(in->bmn, in->bmx), 0.5f);
    }
    if (s->n_inst > 0) {
        s->tlas_idx = (int *)malloc((size_t)s->n_inst * sizeof(int));
        for (int i = 0; i < s->n_inst; ++i) s->tlas_idx[i] = i;
        push_node(&s->tlas, &s->n_tlas, &s->cap_tlas);
        tlas_subdivide(s, 0, 0, s->n_inst);
    }
    s->n_mat = d->num_materials;
    s->mat = (hdr_material_desc *)calloc((size_t)(d->num_materials > 0 ? d->num_materials : 1), sizeof(hdr_material_desc));
    if (d->num_materials > 0) memcpy(s->mat, d->materials, (size_t)d->num_materials * sizeof(hdr_material_desc));
    for (int i = 0; i < d->num_materials; ++i) /* the texels are copied: the scene outlives the caller's arrays */
        for (int k = 0; k < 4; ++k) {
            hdr_material_desc *m = &s->mat[i];
            if (!m->textures[k] || m->tex_width[k] <= 0 || m->tex_height[k] <= 0) {
                m->textures[k] = NULL;
                continue;
            }
            const size_t n = (size_t)m->tex_width[k] * (size_t)m->tex_height[k] * 3;
            float *copy = (float *)malloc(n * sizeof(float));
            memcpy(copy, m->textures[k], n * sizeof(float));
            m->textures[k] = copy;
        }
    s->n_lights = d->num_lights;
    s->lights = (olight *)calloc((size_t)(d->num_lights > 0 ? d->num_lights : 1), sizeof(olight));
    s->env = -1;
    for (int i = 0; i < d->num_lights; ++i) {
        const hdr_light_desc *ld = &d->lights[i];
        olight *L = &s->lights[i];
        L->type = ld->type;
        memcpy(L->color, ld->color, sizeof(L->color));
        L->intensity = ld->intensity;
        L->exposure = ld->exposure;
        memcpy(L->xf, ld->transform, sizeof(L->xf));
        L->width = ld->width;
        L->height = ld->height;
        L->cone_angle = ld->shaping_cone_angle;
        L->cone_softness = ld->shaping_cone_softness;
        L->temperature = ld->temperature;
        if (L->type == HDR_LIGHT_DOME) {
            if (s->env < 0) {
                s->env = i;
                dome_prepare(L, ld);
            }
        }
    }
    s->sky = d->enable_physical_sky != 0;
    if (s->sky) {
        s->sun_dir = orc_sky_sun_direction(d->physical_sky_time);
        s->sun_dir_n = vnorm(s->sun_dir);
        s->sun_lit = orc_sky_sun_color(s->sun_dir, &s->sun_color);
    }
    return s;
}

/* ---- PhysicalSky (scene/physical_sky.cpp:14-208) ---------------------------- */
#define SKY_RP 6371e3f  /* planet radius */
#define SKY_RA 6471e3f  /* atmosphere radius */
#define SKY_HR 7994.0f
#define SKY_HM 1200.0f
#define SKY_BM 21e-6f
static ov3 sky_br(void) { return V(5.5e-6f, 13.0e-6f, 22.4e-6f); }
static ov3 sky_o(void) { return V(0.0f, SKY_RP + 100.0f, 0.0f); }

/* RaySphereIntersect (physical_sky.cpp:14-23): near and far distances, (1e5, -1e5) on a miss */
static void sky_sphere(ov3 r0, ov3 rd, float sr, float *t0, float *t1) {
    float a = vdot(rd, rd);
    float b = 2.0f * vdot(rd, r0);
    float c = vdot(r0, r0) - (sr * sr);
    float d = (b * b) - 4.0f * a * c;
    if (d < 0.0f) {
        *t0 = 1e5f;
        *t1 = -1e5f;
        return;
    }
    *t0 = (-b - sqrtf(d)) / (2.0f * a);
    *t1 = (-b + sqrtf(d)) / (2.0f * a);
}
static ov3 sky_att(float r, float m) {
    ov3 tau = vadd(vmulf(sky_br(), r), vmulf(V(SKY_BM * 1.1f, SKY_BM * 1.1f, SKY_BM * 1.1f), m));
    return V(expf(-tau.x), expf(-tau.y), expf(-tau.z));
}

/* The scene's sky along n directions (rgb into out) and its sun (direction, colour);
 * -1 without a sky, else whether the sun gives a sample (the reference harness's ref_sky) */
int orc_scene_sky(const orc_scene *s, const float *dirs, int n, float *out, float *sun) {
    if (!s->sky) return -1;
    for (int i = 0; i < n; ++i) {
        ov3 c = orc_sky_sample(s->sun_dir_n, V(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
        out[3 * i] = c.x, out[3 * i + 1] = c.y, out[3 * i + 2] = c.z;
    }
    if (!s->sun_lit) return 0;
    sun[0] = s->sun_dir.x, sun[1] = s->sun_dir.y, sun[2] = s->sun_dir.z;
    sun[3] = s->sun_color.x, sun[4] = s->sun_color.y, sun[5] = s->sun_color.z;
    return 1;
}

/* Scene::BuildRenderState's sun (scene.cpp:249-253) */
ov3 orc_sky_sun_direction(float hour) {
    float a = (hour - 12.0f) / 12.0f * (float)M_PI;
    return vnorm(V(sinf(a) * cosf(0.5f), cosf(a), sinf(a) * sinf(0.5f)));
}

/* GetSunTransmittance (:172-206) and SampleDirect (:161-169) */
int orc_sky_sun_color(ov3 sun, ov3 *color) {
    if (sun.y < -0.05f) return 0;
    ov3 tr = V(0.0f, 0.0f, 0.0f);
    if (!(sun.y < 0.0f)) {
        ov3 o = sky_o();
        float t0, t1;
        sky_sphere(o, sun, SKY_RA, &t0, &t1);
        float step = t1 / 16.0f, t = 0.0f, r = 0.0f, m = 0.0f;
        for (int j = 0; j < 16; ++j) {
            float mid = t + step * 0.5f;
            float h = vlen(vadd(o, vmulf(sun, mid))) - SKY_RP;
            if (h < 0.0f) break;
            r += expf(-h / SKY_HR) * step;
            m += expf(-h / SKY_HM) * step;
            t += step;
        }
        tr = sky_att(r, m);
    }
    *color = vmulf(tr, 20.0f);
    return !(color->x <= 0.0f && color->y <= 0.0f && color->z <= 0.0f);
}

/* Sample (:29-159): the sky radiance along rd; sun_n is the sun direction normalised again */
ov3 orc_sky_sample(ov3 sun_n, ov3 rd) {
    ov3 dir = vnorm(rd), o = sky_o(), br = sky_br();
    float a0, a1, p0, p1;
    sky_sphere(o, dir, SKY_RA, &a0, &a1);
    if (a1 < 0.0f) return V(0.0f, 0.0f, 0.0f);
    float tmin = omax(0.0f, a0), tmax = a1;
    sky_sphere(o, dir, SKY_RP, &p0, &p1);
    if (p0 >= 0.0f && p0 < tmax) tmax = p0;
    float step = (tmax - tmin) / 16.0f, t = tmin, odr = 0.0f, odm = 0.0f;
    ov3 tr_ = V(0.0f, 0.0f, 0.0f), tm_ = V(0.0f, 0.0f, 0.0f);
    float mu = vdot(dir, sun_n);
    float phr = 3.0f / (16.0f * (float)M_PI) * (1.0f + mu * mu);
    float g = 0.76f;
    float phm = 3.0f / (8.0f * (float)M_PI) * ((1.0f - g * g) * (1.0f + mu * mu)) /
                ((2.0f + g * g) * powf(1.0f + g * g - 2.0f * g * mu, 1.5f));
    for (int i = 0; i < 16; ++i) {
        float mid = t + step * 0.5f;
        ov3 p = vadd(o, vmulf(dir, mid));
        float h = vlen(p) - SKY_RP;
        if (h < 0.0f) break;
        float hr = expf(-h / SKY_HR) * step, hm = expf(-h / SKY_HM) * step;
        odr += hr;
        odm += hm;
        float s0, s1, q0, q1;
        sky_sphere(p, sun_n, SKY_RA, &s0, &s1);
        float sstep = s1 / 8.0f, st = 0.0f, sr = 0.0f, sm = 0.0f;
        sky_sphere(p, sun_n, SKY_RP, &q0, &q1);
        if (!(q0 > 0.0f)) {
            for (int j = 0; j < 8; ++j) {
                float smid = st + sstep * 0.5f;
                float sh = vlen(vadd(p, vmulf(sun_n, smid))) - SKY_RP;
                if (sh < 0.0f) break;
                sr += expf(-sh / SKY_HR) * sstep;
                sm += expf(-sh / SKY_HM) * sstep;
                st += sstep;
            }
            ov3 at = sky_att(odr + sr, odm + sm);
            tr_ = vadd(tr_, vmulf(at, hr));
            tm_ = vadd(tm_, vmulf(at, hm));
        }
        t += step;
    }
    ov3 si = V(20.0f, 20.0f, 20.0f);
    ov3 col = vcmul(vadd(vmulf(vcmul(tr_, br), phr), vmulf(vmulf(tm_, SKY_BM), phm)), si);
    if (p0 >= 0.0f && p0 < tmax + step) col = vmulf(col, 0.5f);
    if (acosf(oclamp(mu, -1.0f, 1.0f)) < 0.00465f && p0 < 0.0f)
        col = vadd(col, vmulf(vcmul(si, sky_att(odr, odm)), 10.0f));
    return col;
}

void orc_scene_destroy(orc_scene *s) {
    if (!s) return;
    for (int i = 0; i < s->n_mesh; ++i) {
        free(s->blas[i].nodes);
        free(s->blas[i].tris);
    }
    for (int i = 0; i < s->n_lights; ++i) {
        free(s->lights[i].pixels);
        free(s->lights[i].row_cdf);
        free(s->lights[i].col_cdf);
    }
    free(s->blas);
    free(s->inst);
    free(s->tlas);
    free(s->tlas_idx);
    for (int i = 0; i < s->n_mat; ++i)
        for (int k = 0; k < 4; ++k) free((void *)s->mat[i].textures[k]);
    free(s->mat);
    free(s->lights);
    free(s);
}

/* ---------------------------------------------------------------------------
 * Scene query
 * ------------------------------------------------------------------------- */
/* IntersectTriangle (bvh.cpp:8-30); the determinant test is in double */
static int tri_hit(ov3 o, ov3 d, ov3 v0, ov3 v1, ov3 v2, float *t, float *u, float *v) {
    ov3 e1 = vsub(v1, v0), e2 = vsub(v2, v0);
    ov3 p = vcross(d, e2);
    float det = vdot(e1, p);
    if ((double)fabsf(det) < 1e-8) return 0;
    float inv = 1.0f / det;
    ov3 tv = vsub(o, v0);
    float uu = vdot(tv, p) * inv;
    if (uu < 0.0f || uu > 1.0f) return 0;
    ov3 q = vcross(tv, e1);
    float vv = vdot(d, q) * inv;
    if (vv < 0.0f || uu + vv > 1.0f) return 0;
    *t = vdot(e2, q) * inv;
    *u = uu;
    *v = vv;
    return (double)*t > 1e-4;
}

/* IntersectAABB: bvh.cpp:32-64 (thresholds in double) and scene.cpp:16-47 (in float) */
static int aabb_hit(ov3 o, ov3 d, ov3 mn, ov3 mx, float *tmin_out, int dbl) {
    if (range_is_empty(mn, mx)) return 0;
    float tmin = -1e30f, tmax = 1e30f;
    for (int i = 0; i < 3; ++i) {
        float di = vcomp(d, i), oi = vcomp(o, i), lo = vcomp(mn, i), hi = vcomp(mx, i);
        int small = dbl ? ((double)fabsf(di) < 1e-8) : (fabsf(di) < 1e-8f);
        if (small) {
            if (oi < lo || oi > hi) return 0;
        } else {
            float inv = 1.0f / di;
            float t1 = (lo - oi) * inv, t2 = (hi - oi) * inv;
            if (t1 > t2) {
                float tt = t1;
                t1 = t2;
                t2 = tt;
            }
            tmin = omax(tmin, t1);
            tmax = omin(tmax, t2);
            if (tmin > tmax) return 0;
        }
    }
    *tmin_out = tmin;
    return dbl ? (tmax > 0 && (double)tmax > 1e-4) : (tmax > 0.0f && tmax > 1e-4f);
}

typedef struct {
    float t, u, v;
    int tri;
} blas_best;

/* BVH::_IntersectNode (bvh.cpp:250-305): recursive, left before right */
static int blas_node(const oblas *b, int ni, ov3 o, ov3 d, blas_best *best) {
    const onode *n = &b->nodes[ni];
    float ta;
    if (!aabb_hit(o, d, n->mn, n->mx, &ta, 1)) return 0;
    if (ta > best->t) return 0;
    if (n->left < 0) {
        int hit = 0, start = -n->left - 1;
        for (int i = 0; i < n->count; ++i) {
            const otri *tr = &b->tris[start + i];
            float tt, uu, vv;
            if (tri_hit(o, d, tr->v0, tr->v1, tr->v2, &tt, &uu, &vv)) {
                if (tt < best->t) {
                    best->t = tt;
                    best->u = uu;
                    best->v = vv;
                    best->tri = start + i;
                    hit = 1;
                }
            }
        }
        return hit;
    }
    int hl = blas_node(b, n->left, o, d, best);
    int hr = blas_node(b, n->left + 1, o, d, best);
    return hl || hr;
}

/* Scene::Intersect + IntersectScene (scene.cpp:409-535) */
int orc_intersect(const orc_scene *s, ov3 o, ov3 d, ohit *out) {
    if (s->n_tlas == 0) return 0;
    int stack[64], sp = 0;
    stack[sp++] = 0;
    float best_t = 1e30f;
    int best_inst = -1, best_tri = -1;
    float best_u = 0, best_v = 0;
    while (sp > 0) {
        const onode *n = &s->tlas[stack[--sp]];
        float ta = 0.0f;
        if (!aabb_hit(o, d, n->mn, n->mx, &ta, 0) || ta > best_t) continue;
        if (n->left < 0) {
            int start = -n->left - 1;
            for (int i = 0; i < n->count; ++i) {
                int ii = s->tlas_idx[start + i];
                const oinst *in = &s->inst[ii];
                const oblas *b = &s->blas[in->mesh];
                if (b->n_nodes == 0) continue;
                ov3 oo = m4f_xform(in->inv, o), od = m4f_xdir(in->inv, d);
                blas_best bb = {best_t, 0, 0, -1};
                if (!blas_node(b, 0, oo, od, &bb)) continue;
                if (bb.t >= best_t) continue;
                best_t = bb.t;
                best_inst = ii;
                best_tri = bb.tri;
                best_u = bb.u;
                best_v = bb.v;
            }
        } else {
            if (sp + 2 > 64) return 0;
            stack[sp++] = n->left + 1;
            stack[sp++] = n->left;
        }
    }
    if (best_inst < 0) return 0;
    /* hit attributes: bvh.cpp:276-292, scene.cpp:466-503, 525-534 */
    const oinst *in = &s->inst[best_inst];
    const otri *tr = &s->blas[in->mesh].tris[best_tri];
    float u = best_u, v = best_v, w = 1.0f - u - v;
    ov3 normal = vnorm(vcross(vsub(tr->v1, tr->v0), vsub(tr->v2, tr->v0)));
    ov2 uv = {tr->uv0.x * w + tr->uv1.x * u + tr->uv2.x * v, tr->uv0.y * w + tr->uv1.y * u + tr->uv2.y * v};
    ov3 sn = normal;
    if (vdot(tr->n0, tr->n0) > 1e-6f) sn = vnorm(vadd(vadd(vmulf(tr->n0, w), vmulf(tr->n1, u)), vmulf(tr->n2, v)));
    ov3 color = vadd(vadd(vmulf(tr->c0, w), vmulf(tr->c1, u)), vmulf(tr->c2, v));
    out->normal = vnorm(m4f_xdir(in->xf, normal));
    out->smooth_normal = vnorm(m4f_xdir(in->xf, sn));
    out->dpdu = vnorm(m4f_xdir(in->xf, tr->dpdu));
    out->dpdv = vnorm(m4f_xdir(in->xf, tr->dpdv));
    out->uv = uv;
    out->albedo = color;
    if (in->material >= 0) {
        const hdr_material_desc *m = &s->mat[in->material];
        out->albedo = V(m->diffuse_color[0], m->diffuse_color[1], m->diffuse_color[2]);
    }
    out->position = vadd(o, vmulf(d, best_t));
    out->depth = best_t;
    out->prim = best_inst;
    out->mat = best_inst;
    out->tri = best_tri;
    return 1;
}
