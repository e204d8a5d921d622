// Materials on the device.
//   BSDFClosure                  core/shading_types.h:18-42
//   PreviewSurface GetClosure    materials/preview_surface.cpp:61-127 (textures out of scope)
//   PreviewSurface SampleBounce  materials/preview_surface.cpp:129-381
//   DefaultMaterial              materials/default_material.cpp:55-86
//   GGXBsdf::Eval / Pdf          materials/ggx.cpp:20-67
//   shading helpers              materials/shading_helpers.h:20-145
// Random numbers are drawn in the order the reference binary draws them:
// g++ evaluates call arguments right to left, so in
// SampleGGX(rng.NextFloat(), rng.NextFloat(), r) the SECOND parameter
// receives the first draw (same for SampleCosineHemisphere).
#pragma once

// HDR_TEXTURES 0 compiles closures without the texture overrides: the translation
// unit's kernels then serve scenes without textures only (the host picks them by
// DeviceScene::has_textures).
#ifndef HDR_TEXTURES
#define HDR_TEXTURES 1
#endif

#include "rng.cuh"
#include "spectrum.cuh"
#include "traverse.cuh"

namespace hdr {

struct Closure {
    V3 base_color, emission, normal, specular_color, coat_color, sheen_color, subsurface_color, transmission_color;
    float metallic, roughness, ior, specular, transmission, transmission_depth, coat, coat_roughness, coat_ior, sheen,
        sheen_roughness, subsurface, opacity;
    bool thin_walled;
    bool is_default;  // DefaultMaterial: cosine-only SampleBounce
};

// BoundTextureSampler::Sample (scene/image_texture_sampler.h:41-68): bilinear, u wrapped,
// v wrapped and flipped, texel (x, y) at (y * width + x) * 3. Corner indices are clamped to
// the texture, which changes nothing for a finite uv (the reference has no defined texel
// for a non-finite one).
__device__ __forceinline__ V3 texture_sample(const float *tex, int w, int h, V2 uv) {
    const float u = uv.x - floorf(uv.x);
    const float v = 1.0f - (uv.y - floorf(uv.y));
    const float px = u * (float)(w - 1);
    const float py = v * (float)(h - 1);
    const int x0 = sclampi((int)floorf(px), 0, w - 1);
    const int y0 = sclampi((int)floorf(py), 0, h - 1);
    const int x1 = smini(x0 + 1, w - 1);
    const int y1 = smini(y0 + 1, h - 1);
    const float fx = px - (float)x0;
    const float fy = py - (float)y0;
    auto texel = [&](int x, int y) {
        const float *t = tex + (size_t)((y * w + x) * 3);
        return V3{__ldg(t), __ldg(t + 1), __ldg(t + 2)};
    };
    return (texel(x0, y0) * (1 - fx) + texel(x1, y0) * fx) * (1 - fy) +
           (texel(x0, y1) * (1 - fx) + texel(x1, y1) * fx) * fy;
}

struct TexturedParams {
    V3 base_color;
    float metallic, roughness;
    V3 normal;
};

// The texture overrides of PreviewSurfaceMaterial::GetClosure (preview_surface.cpp:68-95);
// out of line so the kernels of untextured scenes keep their registers.
static __device__ __forceinline__ TexturedParams apply_textures(const float *textures, int4 off, int4 tw, int4 th, V2 uv,
                                                      V3 smooth_normal, V3 dpdu, V3 dpdv, TexturedParams p) {
    if (off.x >= 0) p.base_color = cmul(p.base_color, texture_sample(textures + off.x, tw.x, th.x, uv));
    if (off.y >= 0) p.metallic = texture_sample(textures + off.y, tw.y, th.y, uv).x;
    if (off.z >= 0) p.roughness = texture_sample(textures + off.z, tw.z, th.z, uv).x;
    if (off.w >= 0) {  // tangent-space normal map
        V3 nt = texture_sample(textures + off.w, tw.w, th.w, uv);
        nt = nt * 2.0f - v3s(1.0f);
        const V3 n = smooth_normal;
        V3 t = dpdu, b = dpdv;
        t = normalized(t - n * dot(t, n));
        b = normalized(b - n * dot(b, n) - t * dot(b, t));
        if (dot(cross(n, t), b) < 0.0f) b = -b;
        p.normal = normalized(t * nt.x + b * nt.y + n * nt.z);
    }
    return p;
}

__device__ __forceinline__ Closure get_closure(const DeviceScene &s, const Hit &h) {
    Closure c;
    if (h.material < 0) {  // DefaultMaterial::GetClosure + BSDFClosure defaults
        c.base_color = h.albedo;
        c.emission = v3s(0.0f);
        c.normal = h.normal;
        c.specular_color = v3s(1.0f);
        c.coat_color = v3s(1.0f);
        c.sheen_color = v3s(1.0f);
        c.subsurface_color = V3{0.7f, 0.2f, 0.2f};
        c.transmission_color = v3s(1.0f);
        c.metallic = 0.0f;
        c.roughness = 1.0f;
        c.ior = 1.5f;
        c.specular = 0.5f;
        c.transmission = 0.0f;
        c.transmission_depth = 0.0f;
        c.coat = 0.0f;
        c.coat_roughness = 0.0f;
        c.coat_ior = 1.5f;
        c.sheen = 0.0f;
        c.sheen_roughness = 0.3f;
        c.subsurface = 0.0f;
        c.opacity = 1.0f;
        c.thin_walled = false;
        c.is_default = true;
        return c;
    }
    const float4 *m = s.materials + 12 * h.material;
    const float4 m0 = __ldg(m), m1 = __ldg(m + 1), m2 = __ldg(m + 2), m3 = __ldg(m + 3), m4 = __ldg(m + 4);
    const float4 m5 = __ldg(m + 5), m6 = __ldg(m + 6), m7 = __ldg(m + 7), m8 = __ldg(m + 8);
    c.base_color = V3{m0.x, m0.y, m0.z};
    c.metallic = m0.w;
    c.specular_color = V3{m1.x, m1.y, m1.z};
    c.specular = m1.w;
    c.emission = V3{m2.x, m2.y, m2.z};
    c.roughness = m2.w;
    c.transmission_color = V3{m3.x, m3.y, m3.z};
    c.transmission = m3.w;
    c.coat_color = V3{m4.x, m4.y, m4.z};
    c.coat = m4.w;
    c.sheen_color = V3{m5.x, m5.y, m5.z};
    c.sheen = m5.w;
    c.subsurface_color = V3{m6.x, m6.y, m6.z};
    c.subsurface = m6.w;
    c.ior = m7.x;
    c.opacity = m7.y;
    c.transmission_depth = m7.z;
    c.thin_walled = fbits(m7.w) != 0;
    c.coat_roughness = m8.x;
    c.coat_ior = m8.y;
    c.sheen_roughness = m8.z;
    c.normal = h.smooth_normal;
    c.is_default = false;
#if HDR_TEXTURES
    if (!s.has_textures) return c;
    const float4 m9 = __ldg(m + 9);  // texture offsets, -1 = none
    const int4 off = make_int4(fbits(m9.x), fbits(m9.y), fbits(m9.z), fbits(m9.w));
    if ((off.x & off.y & off.z & off.w) != -1) {
        const float4 m10 = __ldg(m + 10), m11 = __ldg(m + 11);
        const TexturedParams t = apply_textures(
            s.textures, off, make_int4(fbits(m10.x), fbits(m10.y), fbits(m10.z), fbits(m10.w)),
            make_int4(fbits(m11.x), fbits(m11.y), fbits(m11.z), fbits(m11.w)), h.uv, h.smooth_normal, h.dpdu,
            h.dpdv, TexturedParams{c.base_color, c.metallic, c.roughness, c.normal});
        c.base_color = t.base_color;
        c.metallic = t.metallic;
        c.roughness = t.roughness;
        c.normal = t.normal;
    }
#endif
    return c;
}

// FresnelDielectric (shading_helpers.h:47-61)
__device__ __forceinline__ float fresnel_dielectric(float cos_i, float ior) {
    cos_i = sclampf(cos_i, -1.0f, 1.0f);
    float eta_i = 1.0f, eta_t = ior;
    if (cos_i > 0) {
        const float t = eta_i;
        eta_i = eta_t;
        eta_t = t;
    }
    const float sin_t = eta_i / eta_t * sqrtf(smaxf(0.0f, 1.0f - cos_i * cos_i));
    if (sin_t >= 1.0f) return 1.0f;
    const float cos_t = sqrtf(smaxf(0.0f, 1.0f - sin_t * sin_t));
    cos_i = fabsf(cos_i);
    const float r_parl = ((eta_t * cos_i) - (eta_i * cos_t)) / ((eta_t * cos_i) + (eta_i * cos_t));
    const float r_perp = ((eta_i * cos_i) - (eta_t * cos_t)) / ((eta_i * cos_i) + (eta_t * cos_t));
    return (r_parl * r_parl + r_perp * r_perp) / 2.0f;
}

// x^5 for the Schlick terms (the reference's std::pow(x, 5.0f)). x*x is exact
// in double and x^4, x^5 are rounded once each there, so the float result is
// the correctly rounded x^5 except within ~2^-50 of a rounding boundary.
HDR_HD float hdr_pow5(float x) {
    const double xd = (double)x;
    const double x2 = xd * xd;
    return (float)(x2 * x2 * xd);
}

// The terms of GGXBsdf::Eval and ::Pdf (ggx.cpp:20-67) that depend only on the
// closure, the normal and wo, each with the reference's expression: a surface
// computes them once and reuses them for every light direction it evaluates.
struct GgxFixed {
    float n_v, alpha2, k_g, one_minus_k_g, g_v, reflect_prob, diff_w;
    V3 F0, one_minus_F0, diff;
};
__device__ __forceinline__ GgxFixed ggx_fixed(const Closure &c, V3 n, V3 wo) {
    GgxFixed g;
    g.n_v = smaxf(0.001f, dot(n, wo));
    const float alpha = smaxf(0.001f, c.roughness * c.roughness);
    g.alpha2 = alpha * alpha;
    g.k_g = alpha / 2.0f;
    g.one_minus_k_g = 1.0f - g.k_g;
    g.g_v = g.n_v / (g.n_v * g.one_minus_k_g + g.k_g);
    g.F0 = c.specular_color * (1.0f - c.metallic) * 0.04f + c.base_color * c.metallic;
    g.one_minus_F0 = v3s(1.0f) - g.F0;
    const V3 fd = c.base_color * (1.0f - c.subsurface) + c.subsurface_color * c.subsurface;
    g.diff = div_d(fd * (1.0f - c.metallic) * (1.0f - c.transmission), (double)kPiF);
    float reflect_prob = fresnel_dielectric(g.n_v, c.ior) * c.specular;
    if (c.metallic > 0.0f) reflect_prob = smaxf(reflect_prob, c.metallic);
    g.reflect_prob = reflect_prob;
    g.diff_w = (1.0f - reflect_prob) * (1.0f - c.transmission);
    return g;
}
// GGXBsdf::Eval with the surface's fixed terms
__device__ __forceinline__ V3 ggx_eval_f(const GgxFixed &g, V3 n, V3 wo, V3 wi) {
    const V3 h = normalized(wo + wi);
    const float n_l = smaxf(0.001f, dot(n, wi));
    const float n_h = smaxf(0.001f, dot(n, h));
    const float l_h = smaxf(0.001f, dot(wi, h));
    const float denom = n_h * n_h * (g.alpha2 - 1.0f) + 1.0f;
    const float D = g.alpha2 / (kPiF * denom * denom);
    const float g_l = n_l / (n_l * g.one_minus_k_g + g.k_g);
    const float G = g_l * g.g_v;
    const V3 F = g.F0 + g.one_minus_F0 * hdr_pow5(1.0f - l_h);
    const V3 spec = div_d(F * D * G, (double)(4.0f * n_l * g.n_v));
    return g.diff + spec;
}
// GGXBsdf::Pdf with the surface's fixed terms
__device__ __forceinline__ float ggx_pdf_f(const GgxFixed &g, V3 n, V3 wo, V3 wi) {
    const V3 h = normalized(wo + wi);
    const float n_l = smaxf(0.001f, dot(n, wi));
    const float n_h = smaxf(0.001f, dot(n, h));
    const float l_h = smaxf(0.001f, dot(wi, h));
    const float denom = n_h * n_h * (g.alpha2 - 1.0f) + 1.0f;
    const float D = g.alpha2 / (kPiF * denom * denom);
    const float diff_pdf = n_l / kPiF;
    const float spec_pdf = (D * n_h) / (4.0f * l_h);
    return g.reflect_prob * spec_pdf + g.diff_w * diff_pdf;
}

// GGXBsdf::Eval (ggx.cpp:20-44)
__device__ __forceinline__ V3 ggx_eval(const Closure &c, V3 n, V3 wo, V3 wi) {
    const V3 h = normalized(wo + wi);
    const float n_l = smaxf(0.001f, dot(n, wi));
    const float n_v = smaxf(0.001f, dot(n, wo));
    const float n_h = smaxf(0.001f, dot(n, h));
    const float l_h = smaxf(0.001f, dot(wi, h));
    const float alpha = smaxf(0.001f, c.roughness * c.roughness);
    const float alpha2 = alpha * alpha;
    const float denom = n_h * n_h * (alpha2 - 1.0f) + 1.0f;
    const float D = alpha2 / (kPiF * denom * denom);
    const float k_g = alpha / 2.0f;
    const float g_l = n_l / (n_l * (1.0f - k_g) + k_g);
    const float g_v = n_v / (n_v * (1.0f - k_g) + k_g);
    const float G = g_l * g_v;
    const V3 F0 = c.specular_color * (1.0f - c.metallic) * 0.04f + c.base_color * c.metallic;
    const V3 F = F0 + (v3s(1.0f) - F0) * hdr_pow5(1.0f - l_h);
    const V3 spec = div_d(F * D * G, (double)(4.0f * n_l * n_v));
    const V3 fd = c.base_color * (1.0f - c.subsurface) + c.subsurface_color * c.subsurface;
    const V3 diff = div_d(fd * (1.0f - c.metallic) * (1.0f - c.transmission), (double)kPiF);
    return diff + spec;
}

// GGXBsdf::Pdf (ggx.cpp:46-67)
__device__ __forceinline__ float ggx_pdf(const Closure &c, V3 n, V3 wo, V3 wi) {
    const V3 h = normalized(wo + wi);
    const float n_l = smaxf(0.001f, dot(n, wi));
    const float n_v = smaxf(0.001f, dot(n, wo));
    const float n_h = smaxf(0.001f, dot(n, h));
    const float l_h = smaxf(0.001f, dot(wi, h));
    const float alpha = smaxf(0.001f, c.roughness * c.roughness);
    const float alpha2 = alpha * alpha;
    const float denom = n_h * n_h * (alpha2 - 1.0f) + 1.0f;
    const float D = alpha2 / (kPiF * denom * denom);
    float reflect_prob = fresnel_dielectric(n_v, c.ior) * c.specular;
    if (c.metallic > 0.0f) reflect_prob = smaxf(reflect_prob, c.metallic);
    const float diff_pdf = n_l / kPiF;
    const float spec_pdf = (D * n_h) / (4.0f * l_h);
    return reflect_prob * spec_pdf + (1.0f - reflect_prob) * (1.0f - c.transmission) * diff_pdf;
}

// SampleGGX (shading_helpers.h:32-40)
__device__ __forceinline__ V3 sample_ggx(float u1, float u2, float roughness) {
    const float alpha = smaxf(0.001f, roughness * roughness);
    const float alpha2 = alpha * alpha;
    const float phi = 2.0f * kPiF * u1;
    const float cos_t = sqrtf((1.0f - u2) / (1.0f + (alpha2 - 1.0f) * u2));
    const float sin_t = sqrtf(smaxf(0.0f, 1.0f - cos_t * cos_t));
    return V3{sin_t * HDR_COSF(phi), cos_t, sin_t * HDR_SINF(phi)};
}
// SampleCosineHemisphere (shading_helpers.h:25-30), y-up
__device__ __forceinline__ V3 sample_cosine_y(float u1, float u2) {
    const float r = sqrtf(u1);
    const float theta = 2.0f * kPiF * u2;
    return V3{r * HDR_COSF(theta), sqrtf(1.0f - u1), r * HDR_SINF(theta)};
}
// AlignToNormal (shading_helpers.h:42-48)
__device__ __forceinline__ V3 align_to_normal(V3 s, V3 n) {
    const V3 up = fabsf(n.y) < 0.999f ? V3{0.0f, 1.0f, 0.0f} : V3{1.0f, 0.0f, 0.0f};
    const V3 t = normalized(cross(up, n));
    const V3 b = cross(n, t);
    return s.x * t + s.y * n + s.z * b;
}
// GGXPdf (shading_helpers.h:64-71)
__device__ __forceinline__ float ggx_half_pdf(V3 h, V3 n, float alpha) {
    const float cos_h = smaxf(0.0f, dot(h, n));
    const float a2 = alpha * alpha;
    const float denom = cos_h * cos_h * (a2 - 1.0f) + 1.0f;
    return a2 / (kPiF * denom * denom) * cos_h;
}
// GGXReflectionWeight (shading_helpers.h:75-91)
__device__ __forceinline__ float ggx_reflection_weight(float n_v, float n_l, float v_h, float n_h, float alpha) {
    n_v = smaxf(0.001f, n_v);
    n_l = smaxf(0.001f, n_l);
    v_h = smaxf(0.001f, v_h);
    n_h = smaxf(0.001f, n_h);
    alpha = smaxf(0.001f, alpha);
    const float a2 = alpha * alpha;
    const float g1v = 2.0f * n_v / (n_v + sqrtf(a2 + (1.0f - a2) * n_v * n_v));
    const float g1l = 2.0f * n_l / (n_l + sqrtf(a2 + (1.0f - a2) * n_l * n_l));
    const float w = (g1v * g1l * v_h) / (n_v * n_h);
    return sminf(w, 10.0f);
}

// PowerHeuristic(f, nf, g, ng, h, nh) (shading_helpers.h:118-130) and the 2-argument form
__device__ __forceinline__ float power_heuristic3(float f, int nf, float g, int ng, float h, int nh) {
    const float f2 = f * f;
    const float g2 = g * g;
    const float h2 = h * h;
    const float denom = (float)nf * f2 + (float)ng * g2 + ((float)nh * h2 + 0.0f);
    return denom > 0.0f ? f2 / denom : 0.0f;
}
__device__ __forceinline__ float power_heuristic2(float f, float g) {
    const float f2 = f * f;
    const float g2 = g * g;
    return f2 / (f2 + g2);
}

// BeerAbsorption (shading_helpers.h:133-145)
__device__ __forceinline__ void beer_absorption(Spec &tp, const Closure &c, float t, bool inside,
                                                const SpectralCtx &sc) {
    if (inside && c.transmission_depth > 0.0f && !c.thin_walled) {
        const Spec ts = rgb_to_spectrum(c.transmission_color, sc.up);
        for (int i = 0; i < 4; ++i) {
            const float sigma_a = -HDR_LOGF(smaxf(ts.v[i], 1e-4f)) / c.transmission_depth;
            tp.v[i] *= HDR_EXPF(-sigma_a * t);
        }
    }
}

// BsdfBounceSample / BounceSampleResult (shading_types.h:59-75)
struct Bounce {
    bool ok;  // false: BounceSampleError (max bounces reached)
    V3 origin, dir;
    Spec tmul;      // ThroughputMul
    Spec integrand; // ThroughputIntegrandMul
    float pdf;      // BsdfPdf.value (always solid angle)
    bool impossible_nee;
    bool skip_roulette;
};

struct BounceState {
    int refl, refr;
};

// DefaultMaterial::SampleBounce (default_material.cpp:66-86): ONB of Duff et al. 2017, z-up cosine sample.
__device__ __forceinline__ Bounce sample_bounce_default(const Closure &c, V3 sn, V3 hit_pos, const SpectralCtx &sc,
                                                        MtStream &rng) {
    const float sign = (sn.z >= 0.0f) ? 1.0f : -1.0f;
    const float a = -1.0f / (sign + sn.z);
    const float bb = sn.x * sn.y * a;
    const V3 t{1.0f + sign * sn.x * sn.x * a, sign * bb, -sign * sn.x};
    const V3 b{bb, sign + sn.y * sn.y * a, -sn.y};
    const float u2 = rng.next_float();  // right-to-left argument evaluation
    const float u1 = rng.next_float();
    const float sin_t = sqrtf(u1);
    const float phi = 2.0f * kPiF * u2;
    const V3 wl{sin_t * HDR_COSF(phi), sin_t * HDR_SINF(phi), sqrtf(smaxf(0.0f, 1.0f - u1))};
    const V3 wi = wl.x * t + wl.y * b + wl.z * sn;
    const float n_l = wl.z;
    const float raw = n_l / kPiF;
    const float safe = smaxf(raw, 1e-6f);
    const float scale = raw / safe;
    Bounce r;
    r.ok = true;
    r.origin = hit_pos + sn * 1e-4f;
    r.dir = wi;
    const Spec base = rgb_to_spectrum(c.base_color, sc.up);
    r.tmul = base * scale;
    r.integrand = base * (n_l / kPiF);
    r.pdf = safe;
    r.impossible_nee = false;
    r.skip_roulette = false;
    return r;
}

// A GGX-lobe reflection shared by the coat, sheen and base lobes (preview_surface.cpp:140-176 etc.)
__device__ __forceinline__ Bounce ggx_lobe_bounce(V3 ray_dir, V3 sn, V3 hit_pos, V3 h, float alpha, V3 tint,
                                                  const SpectralCtx &sc) {
    V3 refl = normalized(ray_dir - 2.0f * dot(ray_dir, h) * h);
    if (dot(refl, sn) < 0) refl = normalized(ray_dir - 2.0f * dot(ray_dir, sn) * sn);
    const float cos_h = smaxf(0.f, dot(refl, h));
    const float n_v = smaxf(0.f, dot(sn, -ray_dir));
    const float n_l = smaxf(0.f, dot(sn, refl));
    const float n_h = smaxf(0.f, dot(sn, h));
    const float pdf = cos_h > 0.f ? ggx_half_pdf(h, sn, alpha) / (4.f * cos_h) : 0.f;
    const float w = ggx_reflection_weight(n_v, n_l, cos_h, n_h, alpha);
    Bounce r;
    r.ok = true;
    r.origin = hit_pos + sn * 1e-4f;
    r.dir = refl;
    r.tmul = rgb_to_spectrum(tint, sc.up) * w;
    r.integrand = r.tmul * pdf;
    r.pdf = pdf;
    r.impossible_nee = false;
    r.skip_roulette = false;
    return r;
}

__device__ __forceinline__ Bounce bounce_error() {
    Bounce r;
    r.ok = false;
    r.origin = r.dir = v3s(0.0f);
    r.tmul = r.integrand = spec(0.0f);
    r.pdf = 0.0f;
    r.impossible_nee = false;
    r.skip_roulette = false;
    return r;
}

__device__ __forceinline__ Bounce specular_bounce(V3 origin, V3 dir, Spec tmul, bool skip_roulette) {
    Bounce r;
    r.ok = true;
    r.origin = origin;
    r.dir = dir;
    r.tmul = tmul;
    r.integrand = spec(0.0f);
    r.pdf = 0.0f;
    r.impossible_nee = true;
    r.skip_roulette = skip_roulette;
    return r;
}

// HDR_BOUNCE_INLINE: how the including kernels take sample_bounce and the RIS
// pass's direct-light estimate and BSDF-connection evaluation (a call keeps the
// closure, surface, spectral context and random stream it is given in local
// memory).
#ifndef HDR_BOUNCE_INLINE
#define HDR_BOUNCE_INLINE inline
#endif
// IMaterial::SampleBounce dispatch
__device__ HDR_BOUNCE_INLINE Bounce sample_bounce(const Closure &c, V3 sn, bool inside, V3 hit_pos, V3 ray_dir, int max_refl,
                                int max_refr, BounceState &st, const SpectralCtx &sc, MtStream &rng) {
    if (c.is_default) return sample_bounce_default(c, sn, hit_pos, sc, rng);
    // --- coat (preview_surface.cpp:136-196)
    if (c.coat > 0.0f && !inside) {
        const float coat_f = c.coat * fresnel_dielectric(dot(ray_dir, sn), c.coat_ior);
        if (rng.next_float() < coat_f) {
            if (st.refl >= max_refl) return bounce_error();
            ++st.refl;
            if (c.coat_roughness > 0.0f) {
                const float u2 = rng.next_float();
                const float u1 = rng.next_float();
                const V3 h = align_to_normal(sample_ggx(u1, u2, c.coat_roughness), sn);
                Bounce r = ggx_lobe_bounce(ray_dir, sn, hit_pos, h, c.coat_roughness * c.coat_roughness,
                                           c.coat_color, sc);
                r.skip_roulette = true;
                return r;
            }
            const V3 refl = normalized(ray_dir - 2.0f * dot(ray_dir, sn) * sn);
            return specular_bounce(hit_pos + sn * 1e-4f, refl, rgb_to_spectrum(c.coat_color, sc.up), true);
        }
    }
    // --- sheen (preview_surface.cpp:198-256)
    if (c.sheen > 0.0f && !inside) {
        const float cos_t = smaxf(0.0f, dot(-ray_dir, sn));
        const float sheen_f = c.sheen * hdr_pow5(1.0f - cos_t);
        if (rng.next_float() < sheen_f) {
            if (st.refl >= max_refl) return bounce_error();
            ++st.refl;
            if (c.sheen_roughness > 0.0f) {
                const float u2 = rng.next_float();
                const float u1 = rng.next_float();
                const V3 h = align_to_normal(sample_ggx(u1, u2, c.sheen_roughness), sn);
                Bounce r = ggx_lobe_bounce(ray_dir, sn, hit_pos, h, c.sheen_roughness * c.sheen_roughness,
                                           c.sheen_color, sc);
                r.skip_roulette = true;
                return r;
            }
            const V3 refl = normalized(ray_dir - 2.0f * dot(ray_dir, sn) * sn);
            return specular_bounce(hit_pos + sn * 1e-4f, refl, rgb_to_spectrum(c.sheen_color, sc.up), true);
        }
    }
    // --- dispersion on lambda0 (preview_surface.cpp:258-264)
    float local_ior = c.ior;
    {
        const float C = 10000.0f;
        const float B = local_ior - C / (589.3f * 589.3f);
        local_ior = B + C / (sc.lambda.l[0] * sc.lambda.l[0]);
    }
    const float fres = fresnel_dielectric(dot(ray_dir, sn), local_ior);
    float reflect_prob = fres * c.specular;
    if (c.metallic > 0.0f) reflect_prob = smaxf(reflect_prob, c.metallic);
    const float rv = rng.next_float();
    if (rv < reflect_prob) {
        // --- reflection (preview_surface.cpp:275-320)
        if (st.refl >= max_refl) return bounce_error();
        ++st.refl;
        const V3 tint = c.specular_color * (1.0f - c.metallic) + c.base_color * c.metallic;
        if (c.roughness > 0.0f) {
            const float u2 = rng.next_float();
            const float u1 = rng.next_float();
            const V3 h = align_to_normal(sample_ggx(u1, u2, c.roughness), sn);
            V3 refl = normalized(ray_dir - 2.0f * dot(ray_dir, h) * h);
            if (dot(refl, sn) < 0) refl = normalized(ray_dir - 2.0f * dot(ray_dir, sn) * sn);
            const float cos_h = smaxf(0.f, dot(refl, h));
            const float n_v = smaxf(0.f, dot(sn, -ray_dir));
            const float n_l = smaxf(0.f, dot(sn, refl));
            const float n_h = smaxf(0.f, dot(sn, h));
            const float alpha = c.roughness * c.roughness;
            const float cond_pdf = cos_h > 0.f ? ggx_half_pdf(h, sn, alpha) / (4.f * cos_h) : 0.f;
            const float w = ggx_reflection_weight(n_v, n_l, cos_h, n_h, alpha);
            Bounce r;
            r.ok = true;
            r.origin = hit_pos + sn * 1e-4f;
            r.dir = refl;
            r.tmul = rgb_to_spectrum(tint, sc.up) * w;
            r.integrand = r.tmul * cond_pdf;
            r.pdf = ggx_pdf(c, sn, -ray_dir, refl);
            r.impossible_nee = false;
            r.skip_roulette = false;
            return r;
        }
        const V3 refl = normalized(ray_dir - 2.0f * dot(ray_dir, sn) * sn);
        return specular_bounce(hit_pos + sn * 1e-4f, refl, rgb_to_spectrum(tint, sc.up), false);
    }
    const float remaining = (rv - reflect_prob) / (1.0f - reflect_prob);
    if (c.transmission > 1e-6f && remaining < c.transmission) {
        // --- refraction / total internal reflection (preview_surface.cpp:322-361)
        float eta_i = 1.0f, eta_t = local_ior;
        if (inside) {
            const float t = eta_i;
            eta_i = eta_t;
            eta_t = t;
        }
        const float eta = eta_i / eta_t;
        const V3 n = sn;
        const float cos_i = dot(ray_dir, n);
        const float k = 1.0f - eta * eta * (1.0f - cos_i * cos_i);
        if (k >= 0) {
            if (st.refr >= max_refr) return bounce_error();
            ++st.refr;
            V3 refr = normalized(eta * ray_dir - (eta * cos_i + sqrtf(k)) * n);
            if (c.roughness > 0.0f) {
                const float u2 = rng.next_float();
                const float u1 = rng.next_float();
                const V3 h = align_to_normal(sample_ggx(u1, u2, c.roughness), n);
                const float cos_ih = dot(ray_dir, h);
                const float k_h = 1.0f - eta * eta * (1.0f - cos_ih * cos_ih);
                if (k_h >= 0.0f)
                    refr = normalized(eta * ray_dir - (eta * cos_ih + sqrtf(k_h)) * h);
                else
                    refr = normalized(ray_dir - 2.0f * cos_ih * h);
            }
            return specular_bounce(hit_pos - n * 1e-4f, refr, rgb_to_spectrum(c.transmission_color, sc.up), false);
        }
        if (st.refl >= max_refl) return bounce_error();
        ++st.refl;
        const V3 refl = normalized(ray_dir - 2.0f * cos_i * sn);
        return specular_bounce(hit_pos + sn * 1e-4f, refl, spec(1.0f), false);
    }
    // --- diffuse (preview_surface.cpp:362-380)
    const float u2 = rng.next_float();
    const float u1 = rng.next_float();
    const V3 dir = align_to_normal(sample_cosine_y(u1, u2), sn);
    const float n_l = smaxf(0.0f, dot(sn, dir));
    const float raw = n_l / kPiF;
    const float safe = smaxf(raw, 1e-6f);
    const float scale = raw / safe;
    const V3 fd = c.base_color * (1.0f - c.subsurface) + c.subsurface_color * c.subsurface;
    const Spec fds = rgb_to_spectrum(fd, sc.up);
    Bounce r;
    r.ok = true;
    r.origin = hit_pos + sn * 1e-4f;
    r.dir = dir;
    r.tmul = fds * scale;
    r.integrand = fds * (n_l / kPiF);
    r.pdf = safe;
    r.impossible_nee = false;
    r.skip_roulette = false;
    return r;
}

// The draws of sample_bounce without the bounce itself, for callers that only
// need the stream to end where the sampling would have left it. Every branch
// that decides how many numbers are drawn depends on the surface alone, so a
// surface computes those quantities once (same expressions as sample_bounce)
// and each call only draws and compares.
struct BounceDraws {
    bool is_default, coat_on, coat_rough, sheen_on, sheen_rough, rough, trans_on, refract_ok;
    float coat_f, sheen_f, reflect_prob, transmission;
};
__device__ __forceinline__ BounceDraws bounce_draws_of(const Closure &c, V3 sn, bool inside, V3 ray_dir,
                                                       const SpectralCtx &sc) {
    BounceDraws d;
    d.is_default = c.is_default;
    d.coat_on = c.coat > 0.0f && !inside;
    d.coat_f = d.coat_on ? c.coat * fresnel_dielectric(dot(ray_dir, sn), c.coat_ior) : 0.0f;
    d.coat_rough = c.coat_roughness > 0.0f;
    d.sheen_on = c.sheen > 0.0f && !inside;
    d.sheen_f = d.sheen_on ? c.sheen * hdr_pow5(1.0f - smaxf(0.0f, dot(-ray_dir, sn))) : 0.0f;
    d.sheen_rough = c.sheen_roughness > 0.0f;
    float local_ior = c.ior;
    {
        const float C = 10000.0f;
        const float B = local_ior - C / (589.3f * 589.3f);
        local_ior = B + C / (sc.lambda.l[0] * sc.lambda.l[0]);
    }
    float reflect_prob = fresnel_dielectric(dot(ray_dir, sn), local_ior) * c.specular;
    if (c.metallic > 0.0f) reflect_prob = smaxf(reflect_prob, c.metallic);
    d.reflect_prob = reflect_prob;
    d.rough = c.roughness > 0.0f;
    d.trans_on = c.transmission > 1e-6f;
    d.transmission = c.transmission;
    float eta_i = 1.0f, eta_t = local_ior;
    if (inside) {
        const float t = eta_i;
        eta_i = eta_t;
        eta_t = t;
    }
    const float eta = eta_i / eta_t;
    const float cos_i = dot(ray_dir, sn);
    d.refract_ok = 1.0f - eta * eta * (1.0f - cos_i * cos_i) >= 0;
    return d;
}
__device__ __forceinline__ void bounce_draws(const BounceDraws &d, int max_refl, int max_refr, BounceState &st,
                                             MtStream &rng) {
    if (d.is_default) {
        (void)rng.next_raw();
        (void)rng.next_raw();
        return;
    }
    if (d.coat_on && rng.next_float() < d.coat_f) {
        if (st.refl >= max_refl) return;
        ++st.refl;
        if (d.coat_rough) {
            (void)rng.next_raw();
            (void)rng.next_raw();
        }
        return;
    }
    if (d.sheen_on && rng.next_float() < d.sheen_f) {
        if (st.refl >= max_refl) return;
        ++st.refl;
        if (d.sheen_rough) {
            (void)rng.next_raw();
            (void)rng.next_raw();
        }
        return;
    }
    const float rv = rng.next_float();
    if (rv < d.reflect_prob) {
        if (st.refl >= max_refl) return;
        ++st.refl;
        if (d.rough) {
            (void)rng.next_raw();
            (void)rng.next_raw();
        }
        return;
    }
    const float remaining = (rv - d.reflect_prob) / (1.0f - d.reflect_prob);
    if (d.trans_on && remaining < d.transmission) {
        if (d.refract_ok) {
            if (st.refr >= max_refr) return;
            ++st.refr;
            if (d.rough) {
                (void)rng.next_raw();
                (void)rng.next_raw();
            }
            return;
        }
        if (st.refl < max_refl) ++st.refl;
        return;
    }
    (void)rng.next_raw();
    (void)rng.next_raw();
}

}  // namespace hdr
