/*
 * CPU oracle for the hdRestir light-transport hot path — TEST INFRASTRUCTURE.
 *
 * A plain-C restatement of the reference's CPU algorithm, used only by the
 * tests, smoke() and bench.py's CPU-baseline leg to check and time the CUDA
 * passes. Nothing in the product links or calls it. It follows the reference
 * source structure (full std::mt19937_64 state per pixel, candidate lists,
 * recursive BLAS traversal) rather than the device design, and each function
 * cites the reference file:line it restates (paths relative to the reference
 * project root). Parity is pinned by comparing this restatement with the
 * reference's own sources compiled in place (oracle/_ref) and with the golden
 * vectors under tests/golden.
 *
 * Floating point: compiled with -O2 -ffp-contract=off (no FMA), IEEE float in
 * source order, like the reference built with g++ on x86-64.
 */
#ifndef HDR_ORACLE_CORE_H
#define HDR_ORACLE_CORE_H

#include <math.h>
#include <stdint.h>
#include <stddef.h>

#include "../include/hdrestir.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Gf-style vectors (OpenUSD GfVec3f semantics) ------------------------ */
typedef struct { float x, y, z; } ov3;
typedef struct { float x, y; } ov2;

static inline float omax(float a, float b) { return (a < b) ? b : a; } /* std::max */
static inline float omin(float a, float b) { return (b < a) ? b : a; } /* std::min */
static inline float oclamp(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
static inline int oclampi(int v, int lo, int hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
static inline ov3 V(float x, float y, float z) { ov3 r = {x, y, z}; return r; }
static inline ov3 vadd(ov3 a, ov3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline ov3 vsub(ov3 a, ov3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline ov3 vneg(ov3 a) { return V(-a.x, -a.y, -a.z); }
static inline ov3 vmulf(ov3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline ov3 vcmul(ov3 a, ov3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
/* GfVec3f *= double / GfVec3f / double (multiply by the double reciprocal) */
static inline ov3 vmuld(ov3 a, double s) {
    return V((float)((double)a.x * s), (float)((double)a.y * s), (float)((double)a.z * s));
}
static inline ov3 vdivd(ov3 a, double s) { return vmuld(a, 1.0 / s); }
static inline float vdot(ov3 a, ov3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline ov3 vcross(ov3 a, ov3 b) {
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float vlen(ov3 a) { return sqrtf(vdot(a, a)); }
/* GfVec3f::GetNormalized(eps = 1e-10) */
static inline ov3 vnorm(ov3 a) {
    float l = vlen(a);
    return vdivd(a, (double)((l > 1e-10f) ? l : 1e-10f));
}
static inline float vcomp(ov3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

/* GfMatrix4f::Transform (row vector, GfProject) / TransformDir */
static inline ov3 m4f_xform(const float *m, ov3 v) {
    float x = v.x * m[0] + v.y * m[4] + v.z * m[8] + m[12];
    float y = v.x * m[1] + v.y * m[5] + v.z * m[9] + m[13];
    float z = v.x * m[2] + v.y * m[6] + v.z * m[10] + m[14];
    float w = v.x * m[3] + v.y * m[7] + v.z * m[11] + m[15];
    float inv = (w != 0.0f) ? 1.0f / w : 1.0f;
    return V(inv * x, inv * y, inv * z);
}
static inline ov3 m4f_xdir(const float *m, ov3 v) {
    return V(v.x * m[0] + v.y * m[4] + v.z * m[8], v.x * m[1] + v.y * m[5] + v.z * m[9],
             v.x * m[2] + v.y * m[6] + v.z * m[10]);
}
void orc_inverse4d(const double *m, double *out);

/* ---- std::mt19937_64 + uniform_real_distribution<float> (core/rng.h) ------ */
typedef struct {
    uint64_t mt[312];
    int idx;
} orc_rng;
void orc_rng_seed(orc_rng *r, uint32_t seed);
uint64_t orc_rng_u64(orc_rng *r);
float orc_rng_float(orc_rng *r);

/* ---- spectra (core/spectrum.h, core/spectrum.cpp) ------------------------ */
typedef struct { float v[4]; } ospec;
typedef struct { float l[4]; } olambda;
olambda orc_sample_wavelengths(float u);
ov3 orc_spectrum_to_rgb(ospec s, const olambda *w);
ospec orc_rgb_to_spectrum(ov3 rgb, const olambda *w);
float orc_spectrum_luminance(ospec s, const olambda *w);
static inline ospec S1(float v) { ospec s = {{v, v, v, v}}; return s; }
static inline ospec smul(ospec a, ospec b) {
    ospec r = {{a.v[0] * b.v[0], a.v[1] * b.v[1], a.v[2] * b.v[2], a.v[3] * b.v[3]}};
    return r;
}
static inline ospec sadd(ospec a, ospec b) {
    ospec r = {{a.v[0] + b.v[0], a.v[1] + b.v[1], a.v[2] + b.v[2], a.v[3] + b.v[3]}};
    return r;
}
static inline ospec smulf(ospec a, float s) {
    ospec r = {{a.v[0] * s, a.v[1] * s, a.v[2] * s, a.v[3] * s}};
    return r;
}

/* ---- scene ----------------------------------------------------------------- */
typedef struct {
    ov3 v0, v1, v2;
    ov2 uv0, uv1, uv2;
    ov3 n0, n1, n2, c0, c1, c2, dpdu, dpdv, centroid;
    int material;
} otri;

typedef struct {
    ov3 mn, mx; /* GfRange3f */
    int left, count;
} onode;

typedef struct {
    onode *nodes;
    int n_nodes, cap_nodes;
    otri *tris;
    int n_tris;
    ov3 range_mn, range_mx;
} oblas;

typedef struct {
    int mesh, material, light;
    float xf[16], inv[16];
    ov3 bmn, bmx, centroid;
} oinst;

typedef struct {
    int type;
    float color[3], intensity, exposure;
    double xf[16];
    float width, height, cone_angle, cone_softness;
    float temperature; /* extension: blackbody emission in kelvin, 0 = the colour */
    float *pixels;
    int w, h;
    float *row_cdf, *col_cdf;
    float total_lum;
} olight;

typedef struct orc_scene {
    oblas *blas;
    int n_mesh;
    oinst *inst;
    int n_inst;
    onode *tlas;
    int n_tlas, cap_tlas;
    int *tlas_idx;
    hdr_material_desc *mat;
    int n_mat;
    olight *lights;
    int n_lights;
    int env; /* first dome light index or -1 (the environment unless sky) */
    /* PhysicalSky (scene/physical_sky.cpp) as the environment (scene.cpp:248-256): its
     * sun is light index n_lights, outside the light sampler */
    int sky;
    ov3 sun_dir, sun_dir_n, sun_color;
    int sun_lit; /* SampleDirect gives a sample */
} orc_scene;

/* HitRecord (core/hit_record.h:15-27) plus the triangle index */
typedef struct {
    ov3 position, normal, smooth_normal, dpdu, dpdv;
    ov2 uv;
    ov3 albedo;
    float depth;
    int prim, mat, tri;
} ohit;

orc_scene *orc_scene_create(const hdr_scene_desc *d);
void orc_scene_destroy(orc_scene *s);
/* PhysicalSky (scene/physical_sky.cpp): the sun for an hour of the day, its colour
 * (0 when SampleDirect gives none), and the sky radiance along a direction */
ov3 orc_sky_sun_direction(float hour);
int orc_sky_sun_color(ov3 sun, ov3 *color);
ov3 orc_sky_sample(ov3 sun_n, ov3 rd);
/* Scene::IntersectScene (scene/scene.cpp:515-535) */
int orc_intersect(const orc_scene *s, ov3 o, ov3 d, ohit *out);

#ifdef __cplusplus
}
#endif
#endif
