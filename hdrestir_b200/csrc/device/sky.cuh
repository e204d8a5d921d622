// PhysicalSky (scene/physical_sky.h:14-51, physical_sky.cpp:14-208): a
// single-scattering Rayleigh + Mie atmosphere over a 6371 km planet, seen from
// 100 m above the ground, lit by one sun. The environment of a scene built with
// SceneBuildRenderStateConfig::EnablePhysicalSky (scene.cpp:248-256): misses
// see Sample(dir); the sun is a delta light outside the light sampler, offered
// by the RIS pass's sky technique and the path tracer's separate environment
// technique.
// The arithmetic is the reference's float expressions in its order (GfVec3f *
// float products, dots left to right, no contraction); expf / powf / acosf are
// CUDA's on the device, so radiance agrees with the reference within a few ulp.
// The sun's direction and colour depend on the scene only and are computed on
// the host (sky_sun_setup) with the host's libm, as the reference computes them.
#pragma once

#include "gf.cuh"

namespace hdr {

namespace sky {
constexpr float kPlanetR = 6371e3f;
constexpr float kAtmosR = 6471e3f;
constexpr float kViewHeight = 100.0f;
constexpr float kHr = 7994.0f;   // Rayleigh scale height
constexpr float kHm = 1200.0f;   // Mie scale height
constexpr float kBetaM = 21e-6f;
constexpr float kMieG = 0.76f;
constexpr float kSunIntensity = 20.0f;
constexpr float kSunAngularRadius = 0.00465f;

HDR_HD V3 beta_r() { return V3{5.5e-6f, 13.0e-6f, 22.4e-6f}; }
HDR_HD V3 origin() { return V3{0.0f, kPlanetR + kViewHeight, 0.0f}; }

// the (near, far) distances of a ray against a sphere about the planet centre;
// (1e5, -1e5) when it misses
HDR_HD V2 ray_sphere(V3 r0, V3 rd, float sr) {
    const float a = dot(rd, rd);
    const float b = 2.0f * dot(rd, r0);
    const float c = dot(r0, r0) - (sr * sr);
    const float d = (b * b) - 4.0f * a * c;
    if (d < 0.0f) return V2{1e5f, -1e5f};
    return V2{(-b - hdr_sqrtf(d)) / (2.0f * a), (-b + hdr_sqrtf(d)) / (2.0f * a)};
}

// exp(-tau) per channel of the optical depths (Rayleigh r, Mie m) along a path
HDR_HD V3 attenuation(float r, float m) {
    const V3 tau = beta_r() * r + v3s(kBetaM * 1.1f) * m;
    return V3{expf(-tau.x), expf(-tau.y), expf(-tau.z)};
}
}  // namespace sky

// PhysicalSky::GetSunTransmittance (physical_sky.cpp:172-206): the sun's light
// through the atmosphere to the viewer, 16 steps.
HDR_HD V3 sky_sun_transmittance(V3 sun_dir) {
    if (sun_dir.y < 0.0f) return v3s(0.0f);
    const V3 o = sky::origin();
    const float t_max = sky::ray_sphere(o, sun_dir, sky::kAtmosR).y;
    const float step = t_max / 16.0f;
    float t = 0.0f, odr = 0.0f, odm = 0.0f;
    for (int j = 0; j < 16; ++j) {
        const float mid = t + step * 0.5f;
        const float h = length(o + sun_dir * mid) - sky::kPlanetR;
        if (h < 0.0f) break;
        odr += expf(-h / sky::kHr) * step;
        odm += expf(-h / sky::kHm) * step;
        t += step;
    }
    return sky::attenuation(odr, odm);
}

// The sun of Scene::BuildRenderState (scene.cpp:249-253) and
// PhysicalSky::SampleDirect (physical_sky.cpp:161-169): its direction for the
// sky's hour, and its colour, or none (returns false) when it is set or black.
HDR_HD V3 sky_sun_direction(float hour) {
    const float a = (hour - 12.0f) / 12.0f * kPiF;
    return normalized(V3{sinf(a) * cosf(0.5f), cosf(a), sinf(a) * sinf(0.5f)});
}
HDR_HD bool sky_sun_color(V3 sun_dir, V3 &color) {
    if (sun_dir.y < -0.05f) return false;
    color = sky_sun_transmittance(sun_dir) * sky::kSunIntensity;
    return !(color.x <= 0.0f && color.y <= 0.0f && color.z <= 0.0f);
}

// PhysicalSky::Sample (physical_sky.cpp:29-159): radiance seen along ray_dir.
// sun_n: the sun direction normalised again, as Sample normalises it.
HDR_HD V3 sky_radiance(V3 sun_n, V3 ray_dir) {
    const V3 dir = normalized(ray_dir);
    const V3 o = sky::origin();
    const V2 ia = sky::ray_sphere(o, dir, sky::kAtmosR);
    if (ia.y < 0.0f) return v3s(0.0f);
    const float t_min = smaxf(0.0f, ia.x);
    float t_max = ia.y;
    const V2 ip = sky::ray_sphere(o, dir, sky::kPlanetR);
    if (ip.x >= 0.0f && ip.x < t_max) t_max = ip.x;
    const float step = (t_max - t_min) / 16.0f;
    const V3 br = sky::beta_r();
    float t = t_min, odr = 0.0f, odm = 0.0f;
    V3 tot_r = v3s(0.0f), tot_m = v3s(0.0f);
    const float mu = dot(dir, sun_n);
    const float phase_r = 3.0f / (16.0f * kPiF) * (1.0f + mu * mu);
    const float g = sky::kMieG;
    const float phase_m = 3.0f / (8.0f * kPiF) * ((1.0f - g * g) * (1.0f + mu * mu)) /
                          ((2.0f + g * g) * powf(1.0f + g * g - 2.0f * g * mu, 1.5f));
    for (int i = 0; i < 16; ++i) {
        const float mid = t + step * 0.5f;
        const V3 p = o + dir * mid;
        const float h = length(p) - sky::kPlanetR;
        if (h < 0.0f) break;
        const float hr = expf(-h / sky::kHr) * step;
        const float hm = expf(-h / sky::kHm) * step;
        odr += hr;
        odm += hm;
        // light path from p to the sun: 8 steps, none when the planet is in the way
        const float sun_t_max = sky::ray_sphere(p, sun_n, sky::kAtmosR).y;
        const float sun_step = sun_t_max / 8.0f;
        float st = 0.0f, sodr = 0.0f, sodm = 0.0f;
        const bool shadowed = sky::ray_sphere(p, sun_n, sky::kPlanetR).x > 0.0f;
        if (!shadowed) {
            for (int j = 0; j < 8; ++j) {
                const float smid = st + sun_step * 0.5f;
                const float sh = length(p + sun_n * smid) - sky::kPlanetR;
                if (sh < 0.0f) break;
                sodr += expf(-sh / sky::kHr) * sun_step;
                sodm += expf(-sh / sky::kHm) * sun_step;
                st += sun_step;
            }
            const V3 att = sky::attenuation(odr + sodr, odm + sodm);
            tot_r = tot_r + att * hr;
            tot_m = tot_m + att * hm;
        }
        t += step;
    }
    const V3 sun_i = v3s(sky::kSunIntensity);
    V3 color = cmul(cmul(tot_r, br) * phase_r + tot_m * sky::kBetaM * phase_m, sun_i);
    if (ip.x >= 0.0f && ip.x < t_max + step) color = color * 0.5f;
    if (acosf(sclampf(mu, -1.0f, 1.0f)) < sky::kSunAngularRadius && ip.x < 0.0f)
        color = color + cmul(sun_i, sky::attenuation(odr, odm)) * 10.0f;
    return color;
}

}  // namespace hdr
