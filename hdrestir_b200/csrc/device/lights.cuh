// Lights and the uniform light sampler on the device.
//   LightSample / ILight            sceneInterface/light_interface.h:15-49
//   RectLight                       scene/rect_light.cpp:14-46
//   PointLight (cone shaping)       scene/point_light.cpp:16-61
//   DistantLight                    scene/distant_light.cpp:10-23
//   DomeLight (CDF sampling, pdf)   scene/dome_light.cpp:85-148
//   UniformLightSampler             lighting_core/uniform_light_sampler.cpp:12-52
//   Pdf::ConvertTo                  math/pdf.h:13-28
// Per-light constants that depend only on the light (frame, colour x
// intensity, cone cosines) are evaluated once on the host with the reference's
// own expressions, so the device only does the per-sample arithmetic.
// Light record (12 float4): [0] type, delta, width, height | [1] colour*intensity, area |
// [2] -z axis normal, cone angle | [3] cos cone, cos inner, softness, - |
// [4..7] GfMatrix4f(transform) | [8] params colour, effective intensity.
#pragma once

#include "rng.cuh"
#include "sky.cuh"
#include "spectrum.cuh"
#include "traverse.cuh"

// HDR_SKY 0 compiles the light code without the physical sky, for kernels whose
// launchers never take a scene with it (the wavefront forms): they keep the
// registers they had without it.
#ifndef HDR_SKY
#define HDR_SKY 1
#endif
// HDR_BLACKBODY 0 likewise leaves out the blackbody emission extension.
#ifndef HDR_BLACKBODY
#define HDR_BLACKBODY 1
#endif

namespace hdr {

// the scene renders under the physical sky (and this build has its code)
__device__ __forceinline__ bool sky_on(const DeviceScene &s) { return HDR_SKY && s.sky; }

constexpr int kLightDistant = 0, kLightDome = 1, kLightRect = 2, kLightPoint = 3;
constexpr int kLightTriangle = 4;  // extension: HDR_LIGHT_TRIANGLE

struct LightSampleD {  // LightSample
    V3 dir, color, normal;
    float dist;
    float pdf;
    bool pdf_solid_angle;
};

__device__ __forceinline__ int light_type(const DeviceScene &s, int li) { return fbits(__ldg(&s.lights[12 * li].x)); }

// Extension (hdr_light_desc.temperature > 0): blackbody emission. Planck's law
// B(l, T) = 2hc^2 / l^5 / (exp(c2 / (l T)) - 1), c2 = hc / k, divided by its value at
// Wien's peak l_max = b / T, where c2 / (l_max T) = c2 / b: (l_max / l)^5 (e^(c2/b) - 1) /
// (exp(c2 / (l T)) - 1), at the wavelength l in nm.
__device__ __forceinline__ float blackbody_normalized(float lambda_nm, float kelvin) {
    const float c2 = 1.4387769e-2f, wien_b = 2.8977721e-3f;  // m K
    const float l = lambda_nm * 1e-9f, lmax = wien_b / kelvin;
    const float r = lmax / l;
    const float peak_den = 142.32490f;  // e^(c2 / b) - 1, c2 / b = 4.9651141
    return (r * r * r * r * r) * peak_den / expm1f(c2 / (l * kelvin));
}
// The spectral emission of scene light li whose sample carries the colour rgb: the
// colour upsampled as the reference does, or the blackbody spectrum times the light's
// effective intensity (record float 35) for a light with a temperature (record float 15).
__device__ __forceinline__ Spec light_emission(const DeviceScene &s, int li, V3 rgb, const SpectralCtx &sc) {
    if (HDR_BLACKBODY && s.blackbody && li >= 0 && li < s.num_lights) {
        const float kelvin = __ldg(&s.lights[12 * li + 3]).w;
        if (kelvin > 0.0f) {
            const float eff = __ldg(&s.lights[12 * li + 8]).w;
            Spec e;
#pragma unroll
            for (int i = 0; i < 4; ++i) e.v[i] = eff * blackbody_normalized(sc.lambda.l[i], kelvin);
            return e;
        }
    }
    return rgb_to_spectrum(rgb, sc.up);
}
// ILight::IsDeltaLight; light index num_lights is the physical sky's sun (a delta light)
__device__ __forceinline__ bool light_is_delta(const DeviceScene &s, int li) {
    return li >= s.num_lights || fbits(__ldg(&s.lights[12 * li].y)) != 0;
}

// ---- PhysicalSky as a light (physical_sky.cpp:161-187) ----------------------
// SampleLight: the sun, the same sample for every point (no random numbers).
__device__ __forceinline__ bool sky_sun_sample(const DeviceScene &s, LightSampleD &ls) {
    if (!sky_on(s) || s.sky_sun.w == 0.0f) return false;
    const V3 d{s.sky_sun.x, s.sky_sun.y, s.sky_sun.z};
    ls = LightSampleD{d, V3{s.sky_sun_color.x, s.sky_sun_color.y, s.sky_sun_color.z}, -d, 1e30f, 1.0f, true};
    return true;
}
__device__ __forceinline__ int sky_light_index(const DeviceScene &s) { return s.num_lights; }

// Pdf::ConvertTo(SolidAngle, dist2, cosY)
__device__ __forceinline__ float pdf_to_solid_angle(float value, bool solid, float dist2, float cos_y) {
    if (solid) return value;
    return value * dist2 / cos_y;
}

// ---- DomeLight --------------------------------------------------------------
__device__ __forceinline__ int lower_bound_f(const float *a, int n, float v) {  // std::lower_bound index
    int lo = 0, len = n;
    while (len > 0) {
        const int half = len >> 1;
        if (__ldg(&a[lo + half]) < v) {
            lo += half + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    return lo;
}
__device__ __forceinline__ V3 dome_pixel(const DeviceScene &s, int x, int y) {
    const size_t idx = (size_t)(y * s.dome_width + x) * 3;
    return V3{__ldg(&s.dome_pixels[idx]), __ldg(&s.dome_pixels[idx + 1]), __ldg(&s.dome_pixels[idx + 2])};
}
// texel lookup of DomeLight::Sample / EvalPdf (dome_light.cpp:117-148)
__device__ __forceinline__ void dome_xy(const DeviceScene &s, V3 dir, int &x, int &y) {
    const double kPi = 3.14159265358979323846;
    const float theta = acosf(sclampf(dir.y, -1.0f, 1.0f));
    float phi = atan2f(dir.z, dir.x);
    if (phi < 0) phi = (float)((double)phi + 2.0 * kPi);
    x = sclampi((int)((double)phi / (2.0 * kPi) * (double)s.dome_width), 0, s.dome_width - 1);
    y = sclampi((int)((double)theta / kPi * (double)s.dome_height), 0, s.dome_height - 1);
}
__device__ __forceinline__ float dome_lum_pdf(const DeviceScene &s, V3 texel) {
    const float lum = 0.2126f * texel.x + 0.7152f * texel.y + 0.0722f * texel.z;
    return smaxf(lum / (s.dome_total_lum * (kPiF / (float)s.dome_height) * (2.0f * kPiF / (float)s.dome_width)),
                 1e-6f);
}
// Scene::GetEnvironment (scene.cpp:248-268): the physical sky when enabled, else
// the first dome light, else none.
__device__ __forceinline__ bool env_present(const DeviceScene &s) { return sky_on(s) || s.env_light >= 0; }
// The environment's light index in a candidate (the dome's; the sky has none)
__device__ __forceinline__ int env_light_index(const DeviceScene &s) { return sky_on(s) ? -1 : s.env_light; }
// IEnvironment::Sample (miss radiance)
__device__ __forceinline__ V3 env_radiance(const DeviceScene &s, V3 dir) {
    if (sky_on(s)) return sky_radiance(V3{s.sky_sun_n.x, s.sky_sun_n.y, s.sky_sun_n.z}, dir);
    if (s.env_light < 0 || s.dome_width <= 0) return v3s(0.0f);
    int x, y;
    dome_xy(s, dir, x, y);
    const float4 p = __ldg(&s.lights[12 * s.env_light + 8]);
    return cmul(dome_pixel(s, x, y), V3{p.x, p.y, p.z}) * p.w;
}
// IEnvironment::EvalPdf(dir): the dome's importance-sampling pdf; the sky's is 0
// (IEnvironment's default, sceneInterface/environment.h:19-24)
__device__ __forceinline__ float env_pdf(const DeviceScene &s, V3 dir) {
    if (sky_on(s) || s.env_light < 0 || s.dome_width <= 0 || s.dome_total_lum <= 0.f) return 0.f;
    int x, y;
    dome_xy(s, dir, x, y);
    return dome_lum_pdf(s, dome_pixel(s, x, y));
}

// ILight::SampleLight
__device__ inline bool sample_light(const DeviceScene &s, int li, V3 hit_pos, MtStream &rng, LightSampleD &ls) {
    const float4 *p = s.lights + 12 * li;
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    const int type = fbits(a.x);
    const V3 color{b.x, b.y, b.z};
    const V3 lnormal{c.x, c.y, c.z};
    if (type == kLightRect || type == kLightTriangle) {
        float u = rng.next_float();
        float v = rng.next_float();
        if (type == kLightTriangle && u + v > 1.0f) {  // the lower-left half of the unit square, folded
            u = 1.0f - u;
            v = 1.0f - v;
        }
        u -= 0.5f;
        v -= 0.5f;
        float m[16];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float4 r = __ldg(p + 4 + k);
            m[4 * k] = r.x, m[4 * k + 1] = r.y, m[4 * k + 2] = r.z, m[4 * k + 3] = r.w;
        }
        const V3 lpos = m4f_transform(m, V3{u * a.z, v * a.w, 0.0f});
        const V3 to_light = lpos - hit_pos;
        const float dist = length(to_light);
        const V3 ldir = div_d(to_light, (double)dist);
        const float area = type == kLightTriangle ? 0.5f * (a.z * a.w) : a.z * a.w;
        if (area <= 0.0f) return false;
        const float cos_l = smaxf(0.0f, dot(lnormal, -ldir));
        if (cos_l <= 0.0f) return false;
        if (color.x <= 0.0f && color.y <= 0.0f && color.z <= 0.0f) return false;
        ls = LightSampleD{ldir, color, lnormal, dist, 1.f / area, false};
        return true;
    }
    if (type == kLightPoint) {
        const float4 r3 = __ldg(p + 7);
        const V3 lpos{r3.x, r3.y, r3.z};  // GfMatrix4f::ExtractTranslation
        const V3 to_light = lpos - hit_pos;
        const float dist = length(to_light);
        const V3 ldir = div_d(to_light, (double)dist);
        V3 lcol = color;
        if (c.w < 180.0f) {
            const float cos_t = dot(lnormal, -ldir);
            if (cos_t <= d.x) {
                lcol = v3s(0.0f);
            } else if (d.z > 0.0f) {
                if (cos_t < d.y) {
                    float f = (cos_t - d.x) / (d.y - d.x);
                    f = f * f * (3.0f - 2.0f * f);
                    lcol = lcol * f;
                }
            }
        }
        if (lcol.x <= 0.0f && lcol.y <= 0.0f && lcol.z <= 0.0f) return false;
        ls = LightSampleD{ldir, lcol, -ldir, dist, 1.f, true};
        return true;
    }
    if (type == kLightDistant) {
        if (color.x <= 0.0f && color.y <= 0.0f && color.z <= 0.0f) return false;
        ls = LightSampleD{lnormal, color, -lnormal, 1e30f, 1.f, true};
        return true;
    }
    // dome (dome_light.cpp:85-115)
    if (s.dome_width <= 0 || li != s.env_light) return false;
    const float u1 = rng.next_float();
    const float u2 = rng.next_float();
    const int W = s.dome_width, H = s.dome_height;
    const int y = sclampi(lower_bound_f(s.dome_row_cdf, H + 1, u1) - 1, 0, H - 1);
    const float *col = s.dome_col_cdf + (size_t)y * (W + 1);
    const int x = sclampi(lower_bound_f(col, W + 1, u2) - 1, 0, W - 1);
    const double kPi = 3.14159265358979323846;
    const float theta = (float)(kPi * (double)(float)(y + 0.5f) / (double)(float)H);
    const float phi = (float)(2.0 * kPi * (double)(float)(x + 0.5f) / (double)(float)W);
    const V3 ldir{HDR_SINF(theta) * HDR_COSF(phi), HDR_COSF(theta), HDR_SINF(theta) * HDR_SINF(phi)};
    const V3 tex = dome_pixel(s, x, y);
    const float4 pc = __ldg(p + 8);
    const V3 lcol = cmul(tex, V3{pc.x, pc.y, pc.z}) * pc.w;
    float pdf = 1.0f;
    if (s.dome_total_lum > 0) pdf = dome_lum_pdf(s, tex);
    if (lcol.x <= 0.0f && lcol.y <= 0.0f && lcol.z <= 0.0f) return false;
    ls = LightSampleD{ldir, lcol, -ldir, 1e30f, pdf, true};
    return true;
}

// Number of random numbers SampleLight consumes (for replaying a stream).
__device__ __forceinline__ int light_sample_draws(const DeviceScene &s, int li) {
    const int type = light_type(s, li);
    if (type == kLightRect || type == kLightTriangle) return 2;
    if (type == kLightDome) return (s.dome_width > 0 && li == s.env_light) ? 2 : 0;
    return 0;
}

// ILight::EvalPdf(hitPos, dir, dist, lightNormal)
__device__ __forceinline__ void light_eval_pdf(const DeviceScene &s, int li, V3 dir, float &value, bool &solid) {
    const float4 a = __ldg(&s.lights[12 * li]);
    const int type = fbits(a.x);
    if (type == kLightRect || type == kLightTriangle) {
        const float area = type == kLightTriangle ? 0.5f * (a.z * a.w) : a.z * a.w;
        value = area <= 0.f ? 0.f : 1.f / area;
        solid = false;
    } else if (type == kLightDome) {
        value = env_pdf(s, dir);
        solid = true;
    } else {
        value = 0.f;
        solid = false;
    }
}

// UniformLightSampler::ProposeCandidate: light index, then SampleLight, pdf x 1/L.
__device__ __forceinline__ bool propose_candidate(const DeviceScene &s, V3 hit_pos, MtStream &rng, int &li,
                                                  LightSampleD &ls) {
    const int L = s.num_lights;
    if (L <= 0) return false;
    const float u = rng.next_float();
    unsigned long long idx = (unsigned long long)(u * (float)L);
    if (idx > (unsigned long long)(L - 1)) idx = (unsigned long long)(L - 1);
    li = (int)idx;
    if (!sample_light(s, li, hit_pos, rng, ls)) return false;
    ls.pdf *= 1.0f / (float)L;
    return true;
}
// The draws of ProposeCandidate without the sample itself.
__device__ __forceinline__ void skip_propose_candidate(const DeviceScene &s, MtStream &rng) {
    const int L = s.num_lights;
    if (L <= 0) return;
    const float u = rng.next_float();
    unsigned long long idx = (unsigned long long)(u * (float)L);
    if (idx > (unsigned long long)(L - 1)) idx = (unsigned long long)(L - 1);
    const int n = light_sample_draws(s, (int)idx);
    for (int k = 0; k < n; ++k) (void)rng.next_raw();
}
// UniformLightSampler::EvalPdf: every scene light is in the sampler's set.
__device__ __forceinline__ float light_select_pdf(const DeviceScene &s) {
    return s.num_lights <= 0 ? 0.0f : 1.0f / (float)s.num_lights;
}
// UniformLightSampler::EvalPdf(*environment): the dome is a scene light, the
// physical sky is not (so it gets a technique of its own)
__device__ __forceinline__ float env_select_pdf(const DeviceScene &s) {
    return (sky_on(s) || s.env_light < 0) ? 0.0f : light_select_pdf(s);
}

// The RIS technique split (ris_direct_light_integrator.cpp:89-99): light-sampler
// NEE, sky NEE when the environment is outside the sampler, BSDF.
__device__ __forceinline__ void ris_technique_split(const DeviceScene &s, int n, int &n_nee, int &n_sky,
                                                    int &n_bsdf) {
    const bool sep = env_present(s) && env_select_pdf(s) <= 0.0f;
    const int n_tech = sep ? 3 : 2;
    n_nee = smaxi(1, n / n_tech);
    n_sky = sep ? n / n_tech : 0;
    n_bsdf = smaxi(0, n - n_nee - n_sky);
}

}  // namespace hdr
