/*
 * CPU oracle — TEST INFRASTRUCTURE (see orc_core.h). Materials, lights,
 * direct-light integrators, path integrator and the passes, restated from the
 * reference. Candidate lists are materialised like the reference's
 * std::vector<OptionalRisLightCandidate>.
 */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "orc_api.h"

#define OPI 3.14159265358979323846f /* (float)M_PI */

/* ---- BSDFClosure (core/shading_types.h:18-42) ---------------------------- */
typedef struct {
    ov3 base, emission, normal, spec_col, coat_col, sheen_col, sss_col, trans_col;
    float metallic, roughness, ior, specular, transmission, trans_depth, coat, coat_rough, coat_ior, sheen,
        sheen_rough, subsurface, opacity;
    int thin, is_default;
} oclosure;

/* BoundTextureSampler::Sample (scene/image_texture_sampler.h:41-68): bilinear, u wrapped,
 * v wrapped and flipped; (1 - fx) etc. are float, each product rounds once. */
static ov3 tex_sample(const float *px, int w, int h, ov2 uv) {
    const float u = uv.x - floorf(uv.x);
    const float v = 1.0f - (uv.y - floorf(uv.y));
    const float fxp = u * (float)(w - 1);
    const float fyp = v * (float)(h - 1);
    const int x0 = (int)floorf(fxp), y0 = (int)floorf(fyp);
    const int x1 = x0 + 1 < w - 1 ? x0 + 1 : w - 1;
    const int y1 = y0 + 1 < h - 1 ? y0 + 1 : h - 1;
    const float fx = fxp - (float)x0, fy = fyp - (float)y0;
#define TX(x, y) V(px[((y) * w + (x)) * 3], px[((y) * w + (x)) * 3 + 1], px[((y) * w + (x)) * 3 + 2])
    const ov3 top = vadd(vmulf(TX(x0, y0), 1 - fx), vmulf(TX(x1, y0), fx));
    const ov3 bot = vadd(vmulf(TX(x0, y1), 1 - fx), vmulf(TX(x1, y1), fx));
#undef TX
    return vadd(vmulf(top, 1 - fy), vmulf(bot, fy));
}

/* PreviewSurfaceMaterial::GetClosure (preview_surface.cpp:61-127, textures at 68-95) /
 * DefaultMaterial::GetClosure (default_material.cpp:55-64) */
static oclosure closure_of(const orc_scene *s, const ohit *h) {
    oclosure c;
    int mi = s->inst[h->mat].material;
    if (mi < 0) {
        c.base = h->albedo;
        c.emission = V(0, 0, 0);
        c.normal = h->normal;
        c.spec_col = V(1, 1, 1);
        c.coat_col = V(1, 1, 1);
        c.sheen_col = V(1, 1, 1);
        c.sss_col = V(0.7f, 0.2f, 0.2f);
        c.trans_col = V(1, 1, 1);
        c.metallic = 0.0f;
        c.roughness = 1.0f;
        c.ior = 1.5f;
        c.specular = 0.5f;
        c.transmission = 0.0f;
        c.trans_depth = 0.0f;
        c.coat = 0.0f;
        c.coat_rough = 0.0f;
        c.coat_ior = 1.5f;
        c.sheen = 0.0f;
        c.sheen_rough = 0.3f;
        c.subsurface = 0.0f;
        c.opacity = 1.0f;
        c.thin = 0;
        c.is_default = 1;
        return c;
    }
    const hdr_material_desc *p = &s->mat[mi];
#define C3(a) V((a)[0], (a)[1], (a)[2])
    c.base = C3(p->diffuse_color);
    c.emission = vmulf(C3(p->emission_color), p->emission);
    c.normal = h->smooth_normal;
    c.spec_col = C3(p->specular_color);
    c.coat_col = C3(p->coat_color);
    c.sheen_col = C3(p->sheen_color);
    c.sss_col = C3(p->subsurface_color);
    c.trans_col = C3(p->transmission_color);
#undef C3
    c.metallic = p->metallic;
    c.roughness = omax(0.001f, p->roughness);
    c.ior = p->ior;
    c.specular = p->specular;
    c.transmission = p->transmission;
    c.trans_depth = p->transmission_depth;
    c.coat = p->coat;
    c.coat_rough = p->coat_roughness;
    c.coat_ior = p->coat_ior;
    c.sheen = p->sheen;
    c.sheen_rough = p->sheen_roughness;
    c.subsurface = p->subsurface;
    c.opacity = p->opacity;
    c.thin = p->thin_walled != 0;
    c.is_default = 0;
    if (p->textures[HDR_TEX_DIFFUSE])
        c.base = vcmul(c.base, tex_sample(p->textures[0], p->tex_width[0], p->tex_height[0], h->uv));
    if (p->textures[HDR_TEX_METALLIC])
        c.metallic = tex_sample(p->textures[1], p->tex_width[1], p->tex_height[1], h->uv).x;
    if (p->textures[HDR_TEX_ROUGHNESS])
        c.roughness = tex_sample(p->textures[2], p->tex_width[2], p->tex_height[2], h->uv).x;
    if (p->textures[HDR_TEX_NORMAL]) {
        ov3 nt = tex_sample(p->textures[3], p->tex_width[3], p->tex_height[3], h->uv);
        nt = vsub(vmulf(nt, 2.0f), V(1.0f, 1.0f, 1.0f));
        const ov3 n = h->smooth_normal;
        ov3 t = h->dpdu, b = h->dpdv;
        t = vnorm(vsub(t, vmulf(n, vdot(t, n))));
        b = vnorm(vsub(vsub(b, vmulf(n, vdot(b, n))), vmulf(t, vdot(b, t))));
        if (vdot(vcross(n, t), b) < 0.0f) b = vneg(b);
        c.normal = vnorm(vadd(vadd(vmulf(t, nt.x), vmulf(b, nt.y)), vmulf(n, nt.z)));
    }
    return c;
}

/* ---- shading helpers (materials/shading_helpers.h) ----------------------- */
static float fresnel(float ci, float ior) {
    ci = oclamp(ci, -1.0f, 1.0f);
    float ei = 1.0f, et = ior;
    if (ci > 0) {
        float t = ei;
        ei = et;
        et = t;
    }
    float st = ei / et * sqrtf(omax(0.0f, 1.0f - ci * ci));
    if (st >= 1.0f) return 1.0f;
    float ct = sqrtf(omax(0.0f, 1.0f - st * st));
    ci = fabsf(ci);
    float rpa = ((et * ci) - (ei * ct)) / ((et * ci) + (ei * ct));
    float rpe = ((ei * ci) - (et * ct)) / ((ei * ci) + (et * ct));
    return (rpa * rpa + rpe * rpe) / 2.0f;
}
static ov3 sample_ggx(float u1, float u2, float r) {
    float a = omax(0.001f, r * r), a2 = a * a;
    float phi = 2.0f * OPI * u1;
    float ct = sqrtf((1.0f - u2) / (1.0f + (a2 - 1.0f) * u2));
    float st = sqrtf(omax(0.0f, 1.0f - ct * ct));
    return V(st * cosf(phi), ct, st * sinf(phi));
}
static ov3 sample_cos_y(float u1, float u2) {
    float r = sqrtf(u1), th = 2.0f * OPI * u2;
    return V(r * cosf(th), sqrtf(1.0f - u1), r * sinf(th));
}
static ov3 align(ov3 s, ov3 n) {
    ov3 up = fabsf(n.y) < 0.999f ? V(0, 1, 0) : V(1, 0, 0);
    ov3 t = vnorm(vcross(up, n));
    ov3 b = vcross(n, t);
    return vadd(vadd(vmulf(t, s.x), vmulf(n, s.y)), vmulf(b, s.z));
}
static float ggx_half_pdf(ov3 h, ov3 n, float a) {
    float ch = omax(0.f, vdot(h, n)), a2 = a * a, den = ch * ch * (a2 - 1.f) + 1.f;
    return a2 / (OPI * den * den) * ch;
}
static float ggx_refl_w(float nv, float nl, float vh, float nh, float a) {
    nv = omax(0.001f, nv);
    nl = omax(0.001f, nl);
    vh = omax(0.001f, vh);
    nh = omax(0.001f, nh);
    a = omax(0.001f, a);
    float a2 = a * a;
    float g1v = 2.0f * nv / (nv + sqrtf(a2 + (1.0f - a2) * nv * nv));
    float g1l = 2.0f * nl / (nl + sqrtf(a2 + (1.0f - a2) * nl * nl));
    return omin((g1v * g1l * vh) / (nv * nh), 10.0f);
}
static float ph3(float f, int nf, float g, int ng, float h, int nh) {
    float f2 = f * f, g2 = g * g, h2 = h * h;
    float den = (float)nf * f2 + (float)ng * g2 + ((float)nh * h2 + 0.0f);
    return den > 0.0f ? f2 / den : 0.0f;
}
static float ph2(float f, float g) {
    float f2 = f * f, g2 = g * g;
    return f2 / (f2 + g2);
}
static void beer(ospec *tp, const oclosure *c, float t, int inside, const olambda *w) {
    if (inside && c->trans_depth > 0.0f && !c->thin) {
        ospec ts = orc_rgb_to_spectrum(c->trans_col, w);
        for (int i = 0; i < 4; ++i) {
            float sa = -logf(omax(ts.v[i], 1e-4f)) / c->trans_depth;
            tp->v[i] *= expf(-sa * t);
        }
    }
}

/* ---- GGXBsdf::Eval / Pdf (materials/ggx.cpp:20-67) ----------------------- */
static ov3 ggx_eval(const oclosure *c, ov3 n, ov3 wo, ov3 wi) {
    ov3 h = vnorm(vadd(wo, wi));
    float nl = omax(0.001f, vdot(n, wi)), nv = omax(0.001f, vdot(n, wo));
    float nh = omax(0.001f, vdot(n, h)), lh = omax(0.001f, vdot(wi, h));
    float a = omax(0.001f, c->roughness * c->roughness), a2 = a * a;
    float den = nh * nh * (a2 - 1.0f) + 1.0f;
    float D = a2 / (OPI * den * den);
    float k = a / 2.0f;
    float G = (nl / (nl * (1.0f - k) + k)) * (nv / (nv * (1.0f - k) + k));
    ov3 F0 = vadd(vmulf(vmulf(c->spec_col, 1.0f - c->metallic), 0.04f), vmulf(c->base, c->metallic));
    ov3 F = vadd(F0, vmulf(vsub(V(1, 1, 1), F0), powf(1.0f - lh, 5.0f)));
    ov3 spec = vdivd(vmulf(vmulf(F, D), G), (double)(4.0f * nl * nv));
    ov3 fd = vadd(vmulf(c->base, 1.0f - c->subsurface), vmulf(c->sss_col, c->subsurface));
    ov3 diff = vdivd(vmulf(vmulf(fd, 1.0f - c->metallic), 1.0f - c->transmission), (double)OPI);
    return vadd(diff, spec);
}
static float ggx_pdf(const oclosure *c, ov3 n, ov3 wo, ov3 wi) {
    ov3 h = vnorm(vadd(wo, wi));
    float nl = omax(0.001f, vdot(n, wi)), nv = omax(0.001f, vdot(n, wo));
    float nh = omax(0.001f, vdot(n, h)), lh = omax(0.001f, vdot(wi, h));
    float a = omax(0.001f, c->roughness * c->roughness), a2 = a * a;
    float den = nh * nh * (a2 - 1.0f) + 1.0f;
    float D = a2 / (OPI * den * den);
    float rp = fresnel(nv, c->ior) * c->specular;
    if (c->metallic > 0.0f) rp = omax(rp, c->metallic);
    float dpdf = nl / OPI, spdf = (D * nh) / (4.0f * lh);
    return rp * spdf + (1.0f - rp) * (1.0f - c->transmission) * dpdf;
}

/* ---- SampleBounce ---------------------------------------------------------- */
typedef struct {
    int ok;
    ov3 o, d;
    ospec tmul, integ;
    float pdf;
    int impossible, skip_roulette;
} obounce;

/* a helper mirroring the argument evaluation of the reference binary:
 * f(rng.NextFloat(), rng.NextFloat()) receives its SECOND argument first (g++
 * evaluates call arguments right to left; pinned by the golden vectors) */
static void draw_pair(orc_rng *r, float *u1, float *u2) {
    *u2 = orc_rng_float(r);
    *u1 = orc_rng_float(r);
}

static obounce bounce_err(void) {
    obounce b;
    memset(&b, 0, sizeof(b));
    b.ok = 0;
    return b;
}

/* DefaultMaterial::SampleBounce (default_material.cpp:66-86) */
static obounce sb_default(const oclosure *c, ov3 n, ov3 p, const olambda *w, orc_rng *r) {
    float sign = (n.z >= 0.0f) ? 1.0f : -1.0f;
    float a = -1.0f / (sign + n.z);
    float bb = n.x * n.y * a;
    ov3 t = V(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    ov3 b = V(bb, sign + n.y * n.y * a, -n.y);
    float u1, u2;
    draw_pair(r, &u1, &u2);
    float st = sqrtf(u1), phi = 2.0f * OPI * u2;
    ov3 wl = V(st * cosf(phi), st * sinf(phi), sqrtf(omax(0.0f, 1.0f - u1)));
    ov3 wi = vadd(vadd(vmulf(t, wl.x), vmulf(b, wl.y)), vmulf(n, wl.z));
    float nl = wl.z, raw = nl / OPI, safe = omax(raw, 1e-6f), sc = raw / safe;
    obounce o;
    memset(&o, 0, sizeof(o));
    o.ok = 1;
    o.o = vadd(p, vmulf(n, 1e-4f));
    o.d = wi;
    ospec base = orc_rgb_to_spectrum(c->base, w);
    o.tmul = smulf(base, sc);
    o.integ = smulf(base, nl / OPI);
    o.pdf = safe;
    return o;
}

static obounce lobe_refl(ov3 rd, ov3 n, ov3 p, ov3 h, float alpha, ov3 tint, const olambda *w, int skip_rr) {
    ov3 rf = vnorm(vsub(rd, vmulf(h, 2.0f * vdot(rd, h))));
    if (vdot(rf, n) < 0) rf = vnorm(vsub(rd, vmulf(n, 2.0f * vdot(rd, n))));
    float ch = omax(0.f, vdot(rf, h)), nv = omax(0.f, vdot(n, vneg(rd))), nl = omax(0.f, vdot(n, rf)),
          nh = omax(0.f, vdot(n, h));
    float pdf = ch > 0.f ? ggx_half_pdf(h, n, alpha) / (4.f * ch) : 0.f;
    float gw = ggx_refl_w(nv, nl, ch, nh, alpha);
    obounce o;
    memset(&o, 0, sizeof(o));
    o.ok = 1;
    o.o = vadd(p, vmulf(n, 1e-4f));
    o.d = rf;
    o.tmul = smulf(orc_rgb_to_spectrum(tint, w), gw);
    o.integ = smulf(o.tmul, pdf);
    o.pdf = pdf;
    o.skip_roulette = skip_rr;
    return o;
}

static obounce spec_bounce(ov3 o_, ov3 d, ospec tmul, int skip_rr) {
    obounce o;
    memset(&o, 0, sizeof(o));
    o.ok = 1;
    o.o = o_;
    o.d = d;
    o.tmul = tmul;
    o.integ = S1(0.0f);
    o.pdf = 0.0f;
    o.impossible = 1;
    o.skip_roulette = skip_rr;
    return o;
}

/* PreviewSurfaceMaterial::SampleBounce (preview_surface.cpp:129-381) */
static obounce sample_bounce(const oclosure *c, ov3 n, int inside, ov3 p, ov3 rd, int max_refl, int max_refr,
                             int *refl, int *refr, const olambda *w, orc_rng *r) {
    if (c->is_default) return sb_default(c, n, p, w, r);
    if (c->coat > 0.0f && !inside) {
        float cf = c->coat * fresnel(vdot(rd, n), c->coat_ior);
        if (orc_rng_float(r) < cf) {
            if (*refl >= max_refl) return bounce_err();
            ++*refl;
            if (c->coat_rough > 0.0f) {
                float u1, u2;
                draw_pair(r, &u1, &u2);
                ov3 h = align(sample_ggx(u1, u2, c->coat_rough), n);
                return lobe_refl(rd, n, p, h, c->coat_rough * c->coat_rough, c->coat_col, w, 1);
            }
            ov3 rf = vnorm(vsub(rd, vmulf(n, 2.0f * vdot(rd, n))));
            return spec_bounce(vadd(p, vmulf(n, 1e-4f)), rf, orc_rgb_to_spectrum(c->coat_col, w), 1);
        }
    }
    if (c->sheen > 0.0f && !inside) {
        float ct = omax(0.0f, vdot(vneg(rd), n));
        float sf = c->sheen * powf(1.0f - ct, 5.0f);
        if (orc_rng_float(r) < sf) {
            if (*refl >= max_refl) return bounce_err();
            ++*refl;
            if (c->sheen_rough > 0.0f) {
                float u1, u2;
                draw_pair(r, &u1, &u2);
                ov3 h = align(sample_ggx(u1, u2, c->sheen_rough), n);
                return lobe_refl(rd, n, p, h, c->sheen_rough * c->sheen_rough, c->sheen_col, w, 1);
            }
            ov3 rf = vnorm(vsub(rd, vmulf(n, 2.0f * vdot(rd, n))));
            return spec_bounce(vadd(p, vmulf(n, 1e-4f)), rf, orc_rgb_to_spectrum(c->sheen_col, w), 1);
        }
    }
    float lior = c->ior;
    {
        float C = 10000.0f;
        float B = lior - C / (589.3f * 589.3f);
        lior = B + C / (w->l[0] * w->l[0]);
    }
    float rp = fresnel(vdot(rd, n), lior) * c->specular;
    if (c->metallic > 0.0f) rp = omax(rp, c->metallic);
    float rv = orc_rng_float(r);
    if (rv < rp) {
        if (*refl >= max_refl) return bounce_err();
        ++*refl;
        ov3 tint = vadd(vmulf(c->spec_col, 1.0f - c->metallic), vmulf(c->base, c->metallic));
        if (c->roughness > 0.0f) {
            float u1, u2;
            draw_pair(r, &u1, &u2);
            ov3 h = align(sample_ggx(u1, u2, c->roughness), n);
            obounce o = lobe_refl(rd, n, p, h, c->roughness * c->roughness, tint, w, 0);
            o.pdf = ggx_pdf(c, n, vneg(rd), o.d);
            return o;
        }
        ov3 rf = vnorm(vsub(rd, vmulf(n, 2.0f * vdot(rd, n))));
        return spec_bounce(vadd(p, vmulf(n, 1e-4f)), rf, orc_rgb_to_spectrum(tint, w), 0);
    }
    float rem = (rv - rp) / (1.0f - rp);
    if (c->transmission > 1e-6f && rem < c->transmission) {
        float ei = 1.0f, et = lior;
        if (inside) {
            float t = ei;
            ei = et;
            et = t;
        }
        float eta = ei / et;
        float ci = vdot(rd, n);
        float k = 1.0f - eta * eta * (1.0f - ci * ci);
        if (k >= 0) {
            if (*refr >= max_refr) return bounce_err();
            ++*refr;
            ov3 rdir = vnorm(vsub(vmulf(rd, eta), vmulf(n, eta * ci + sqrtf(k))));
            if (c->roughness > 0.0f) {
                float u1, u2;
                draw_pair(r, &u1, &u2);
                ov3 h = align(sample_ggx(u1, u2, c->roughness), n);
                float cih = vdot(rd, h);
                float kh = 1.0f - eta * eta * (1.0f - cih * cih);
                if (kh >= 0.0f)
                    rdir = vnorm(vsub(vmulf(rd, eta), vmulf(h, eta * cih + sqrtf(kh))));
                else
                    rdir = vnorm(vsub(rd, vmulf(h, 2.0f * cih)));
            }
            return spec_bounce(vsub(p, vmulf(n, 1e-4f)), rdir, orc_rgb_to_spectrum(c->trans_col, w), 0);
        }
        if (*refl >= max_refl) return bounce_err();
        ++*refl;
        ov3 rf = vnorm(vsub(rd, vmulf(n, 2.0f * ci)));
        return spec_bounce(vadd(p, vmulf(n, 1e-4f)), rf, S1(1.0f), 0);
    }
    float u1, u2;
    draw_pair(r, &u1, &u2);
    ov3 dir = align(sample_cos_y(u1, u2), n);
    float nl = omax(0.0f, vdot(n, dir)), raw = nl / OPI, safe = omax(raw, 1e-6f), sc = raw / safe;
    ov3 fd = vadd(vmulf(c->base, 1.0f - c->subsurface), vmulf(c->sss_col, c->subsurface));
    ospec fs = orc_rgb_to_spectrum(fd, w);
    obounce o;
    memset(&o, 0, sizeof(o));
    o.ok = 1;
    o.o = vadd(p, vmulf(n, 1e-4f));
    o.d = dir;
    o.tmul = smulf(fs, sc);
    o.integ = smulf(fs, nl / OPI);
    o.pdf = safe;
    return o;
}

/* ---- lights ---------------------------------------------------------------- */
typedef struct {
    ov3 dir, color, normal;
    float dist, pdf;
    int solid;
} olsample;

static void light_matrix(const olight *L, float *m) {
    for (int k = 0; k < 16; ++k) m[k] = (float)L->xf[k];
}
static ov3 light_color(const olight *L) {
    return vmulf(V(L->color[0], L->color[1], L->color[2]), L->intensity * exp2f(L->exposure));
}
/* Extension: blackbody emission (hdr_light_desc.temperature > 0), Planck's law divided by its
 * value at Wien's peak: (lmax / l)^5 (e^(c2/b) - 1) / (exp(c2 / (l T)) - 1); else the colour
 * upsampled as the reference does. */
static float blackbody_normalized(float lambda_nm, float kelvin) {
    const float c2 = 1.4387769e-2f, wien_b = 2.8977721e-3f;
    const float l = lambda_nm * 1e-9f, lmax = wien_b / kelvin;
    const float r = lmax / l;
    return (r * r * r * r * r) * 142.32490f / expm1f(c2 / (l * kelvin));
}
static ospec light_emission(const orc_scene *s, int li, ov3 rgb, const olambda *w) {
    if (li >= 0 && li < s->n_lights && s->lights[li].temperature > 0.0f) {
        const olight *L = &s->lights[li];
        const float eff = L->intensity * exp2f(L->exposure);
        ospec e;
        for (int i = 0; i < 4; ++i) e.v[i] = eff * blackbody_normalized(w->l[i], L->temperature);
        return e;
    }
    return orc_rgb_to_spectrum(rgb, w);
}
static int is_delta(const olight *L) { return L->type == HDR_LIGHT_POINT || L->type == HDR_LIGHT_DISTANT; }
/* ILight::IsDeltaLight by index: n_lights is the physical sky's sun (a delta light) */
static int light_delta(const orc_scene *s, int li) { return li >= s->n_lights || is_delta(&s->lights[li]); }
/* Scene::GetEnvironment: the physical sky, else the first dome, else none */
static int has_env(const orc_scene *s) { return s->sky || s->env >= 0; }

static void dome_xy(const olight *L, ov3 d, int *x, int *y) {
    const double PI = 3.14159265358979323846;
    float th = acosf(oclamp(d.y, -1.0f, 1.0f));
    float ph = atan2f(d.z, d.x);
    if (ph < 0) ph = (float)((double)ph + 2.0 * PI);
    *x = oclampi((int)((double)ph / (2.0 * PI) * L->w), 0, L->w - 1);
    *y = oclampi((int)((double)th / PI * L->h), 0, L->h - 1);
}
static float dome_pdf_lum(const olight *L, ov3 t) {
    float lum = 0.2126f * t.x + 0.7152f * t.y + 0.0722f * t.z;
    return omax(lum / (L->total_lum * (OPI / (float)L->h) * (2.0f * OPI / (float)L->w)), 1e-6f);
}
/* DomeLight::Sample / EvalPdf (dome_light.cpp:117-148) */
static ov3 env_sample(const orc_scene *s, ov3 d) {
    if (s->sky) return orc_sky_sample(s->sun_dir_n, d);
    if (s->env < 0) return V(0, 0, 0);
    const olight *L = &s->lights[s->env];
    if (!L->pixels) return V(0, 0, 0);
    int x, y;
    dome_xy(L, d, &x, &y);
    const float *p = &L->pixels[(size_t)(y * L->w + x) * 3];
    return vmulf(vcmul(V(p[0], p[1], p[2]), V(L->color[0], L->color[1], L->color[2])),
                 L->intensity * exp2f(L->exposure));
}
static float env_pdf(const orc_scene *s, ov3 d) {
    if (s->sky || s->env < 0) return 0.f; /* the sky: IEnvironment's default 0 */
    const olight *L = &s->lights[s->env];
    if (!L->pixels || L->total_lum <= 0.f) return 0.f;
    int x, y;
    dome_xy(L, d, &x, &y);
    const float *p = &L->pixels[(size_t)(y * L->w + x) * 3];
    return dome_pdf_lum(L, V(p[0], p[1], p[2]));
}
static int lower_bound(const float *a, int n, float v) {
    int lo = 0, len = n;
    while (len > 0) {
        int half = len / 2;
        if (a[lo + half] < v) {
            lo += half + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    return lo;
}

/* ILight::SampleLight: rect_light.cpp:14-37, point_light.cpp:16-55,
 * distant_light.cpp:10-17, dome_light.cpp:85-115 */
static int sample_light(const orc_scene *s, int li, ov3 hp, orc_rng *r, olsample *ls) {
    const olight *L = &s->lights[li];
    float m[16];
    light_matrix(L, m);
    if (L->type == HDR_LIGHT_RECT || L->type == HDR_LIGHT_TRIANGLE) {
        float u = orc_rng_float(r);
        float v = orc_rng_float(r);
        if (L->type == HDR_LIGHT_TRIANGLE && u + v > 1.0f) { /* extension: the folded half square */
            u = 1.0f - u;
            v = 1.0f - v;
        }
        u -= 0.5f;
        v -= 0.5f;
        ov3 lp = m4f_xform(m, V(u * L->width, v * L->height, 0.0f));
        ov3 tl = vsub(lp, hp);
        float dist = vlen(tl);
        ov3 ld = vdivd(tl, (double)dist);
        float area = L->type == HDR_LIGHT_TRIANGLE ? 0.5f * (L->width * L->height) : L->width * L->height;
        if (area <= 0.0f) return 0;
        ov3 ln = vnorm(m4f_xdir(m, V(0, 0, -1)));
        float cl = omax(0.0f, vdot(ln, vneg(ld)));
        if (cl <= 0.0f) return 0;
        ov3 col = light_color(L);
        if (col.x <= 0.0f && col.y <= 0.0f && col.z <= 0.0f) return 0;
        ls->dir = ld;
        ls->color = col;
        ls->normal = ln;
        ls->dist = dist;
        ls->pdf = 1.f / area;
        ls->solid = 0;
        return 1;
    }
    if (L->type == HDR_LIGHT_POINT) {
        ov3 lp = V(m[12], m[13], m[14]);
        ov3 tl = vsub(lp, hp);
        float dist = vlen(tl);
        ov3 ld = vdivd(tl, (double)dist);
        ov3 col = light_color(L);
        float cone = L->cone_angle;
        if (cone < 180.0f) {
            ov3 ln = vnorm(m4f_xdir(m, V(0, 0, -1)));
            float ct = vdot(ln, vneg(ld));
            float rad = cone * (float)(3.14159265358979323846 / 180.0);
            float cc = cosf(rad);
            if (ct <= cc) {
                col = V(0, 0, 0);
            } else {
                float soft = L->cone_softness;
                if (soft > 0.0f) {
                    float ci = cosf(rad * (1.0f - soft));
                    if (ct < ci) {
                        float f = (ct - cc) / (ci - cc);
                        f = f * f * (3.0f - 2.0f * f);
                        col = vmulf(col, f);
                    }
                }
            }
        }
        if (col.x <= 0.0f && col.y <= 0.0f && col.z <= 0.0f) return 0;
        ls->dir = ld;
        ls->color = col;
        ls->normal = vneg(ld);
        ls->dist = dist;
        ls->pdf = 1.f;
        ls->solid = 1;
        return 1;
    }
    if (L->type == HDR_LIGHT_DISTANT) {
        ov3 ld = vnorm(m4f_xdir(m, V(0, 0, -1)));
        ov3 col = light_color(L);
        if (col.x <= 0.0f && col.y <= 0.0f && col.z <= 0.0f) return 0;
        ls->dir = ld;
        ls->color = col;
        ls->normal = vneg(ld);
        ls->dist = 1e30f;
        ls->pdf = 1.f;
        ls->solid = 1;
        return 1;
    }
    /* dome */
    if (!L->pixels) return 0;
    float u1 = orc_rng_float(r);
    float u2 = orc_rng_float(r);
    int y = oclampi(lower_bound(L->row_cdf, L->h + 1, u1) - 1, 0, L->h - 1);
    int x = oclampi(lower_bound(&L->col_cdf[(size_t)y * (L->w + 1)], L->w + 1, u2) - 1, 0, L->w - 1);
    const double PI = 3.14159265358979323846;
    float th = (float)(PI * (float)(y + 0.5f) / (float)L->h);
    float ph = (float)(2.0f * PI * (float)(x + 0.5f) / (float)L->w);
    ov3 ld = V(sinf(th) * cosf(ph), cosf(th), sinf(th) * sinf(ph));
    const float *p = &L->pixels[(size_t)(y * L->w + x) * 3];
    ov3 tex = V(p[0], p[1], p[2]);
    ov3 col = vmulf(vcmul(tex, V(L->color[0], L->color[1], L->color[2])), L->intensity * exp2f(L->exposure));
    float pdf = 1.0f;
    if (L->total_lum > 0) pdf = dome_pdf_lum(L, tex);
    if (col.x <= 0.0f && col.y <= 0.0f && col.z <= 0.0f) return 0;
    ls->dir = ld;
    ls->color = col;
    ls->normal = vneg(ld);
    ls->dist = 1e30f;
    ls->pdf = pdf;
    ls->solid = 1;
    return 1;
}

/* ILight::EvalPdf(hitPos, dir, dist, lightNormal) */
static void light_eval_pdf(const orc_scene *s, int li, ov3 d, float *val, int *solid) {
    const olight *L = &s->lights[li];
    if (L->type == HDR_LIGHT_RECT || L->type == HDR_LIGHT_TRIANGLE) {
        float a = L->type == HDR_LIGHT_TRIANGLE ? 0.5f * (L->width * L->height) : L->width * L->height;
        *val = a <= 0.f ? 0.f : 1.f / a;
        *solid = 0;
    } else if (L->type == HDR_LIGHT_DOME) {
        *val = (li == s->env) ? env_pdf(s, d) : 0.f;
        *solid = 1;
    } else {
        *val = 0.f;
        *solid = 0;
    }
}

static float pdf_sa(float v, int solid, float d2, float cy) { return solid ? v : v * d2 / cy; }

/* UniformLightSampler (lighting_core/uniform_light_sampler.cpp:12-52) */
static int propose(const orc_scene *s, ov3 hp, orc_rng *r, int *li, olsample *ls) {
    size_t L = (size_t)s->n_lights;
    if (L == 0) return 0;
    size_t idx = (size_t)(orc_rng_float(r) * (float)L);
    if (idx > L - 1u) idx = L - 1u;
    *li = (int)idx;
    if (!sample_light(s, *li, hp, r, ls)) return 0;
    ls->pdf *= 1.0f / (float)L;
    return 1;
}
static float select_pdf(const orc_scene *s) { return s->n_lights == 0 ? 0.0f : 1.0f / (float)s->n_lights; }
/* UniformLightSampler::EvalPdf(*environment): the dome is a scene light, the sky is not */
static float env_sel(const orc_scene *s) { return (s->sky || s->env < 0) ? 0.0f : select_pdf(s); }
/* PhysicalSky::SampleLight (physical_sky.cpp:171-178): the sun, no random numbers */
static int sky_sun(const orc_scene *s, olsample *ls) {
    if (!s->sky || !s->sun_lit) return 0;
    ls->dir = s->sun_dir;
    ls->color = s->sun_color;
    ls->normal = vneg(s->sun_dir);
    ls->dist = 1e30f;
    ls->pdf = 1.0f;
    ls->solid = 1;
    return 1;
}

/* ---- shading point --------------------------------------------------------- */
typedef struct {
    ov3 ro, rd;
    ohit hit;
    oclosure c;
    ov3 sn;
    int inside;
} osurf;

typedef struct {
    obounce b;
    int has_hit;
    ohit hit;
} oconn;

static int occluded(const orc_scene *s, ov3 o, ov3 d, float dist) {
    ohit h;
    return orc_intersect(s, o, d, &h) && h.depth < dist - 1e-3f;
}

/* Detail::SampleBounceWithConnection (direct_light_integrator_interface.h:18-40) */
static oconn bounce_with_connection(const orc_scene *s, const osurf *sf, int mr, int mt, int *refl, int *refr,
                                    const olambda *w, orc_rng *r) {
    oconn c;
    memset(&c, 0, sizeof(c));
    c.b = sample_bounce(&sf->c, sf->sn, sf->inside, sf->hit.position, sf->rd, mr, mt, refl, refr, w, r);
    if (c.b.ok) c.has_hit = orc_intersect(s, c.b.o, c.b.d, &c.hit);
    return c;
}

static int hit_light(const orc_scene *s, const ohit *h) { return s->inst[h->prim].light; } /* GetLightAtHit */

/* ---- MisDirectLightIntegrator (mis_direct_light_integrator.cpp) ----------- */
/* _evaluateNEE (:80-120): the radiance a light sample adds, 0 (returns 0) when it
 * cannot or is occluded; *pn / *bp: its NEE and BSDF pdfs */
static int mis_nee(const orc_scene *s, const osurf *sf, int li, const olsample *ls, const olambda *w, ospec *rad,
                   float *pn, float *bp) {
    float nl = vdot(sf->sn, ls->dir);
    if (nl <= 0.0f) return 0;
    float d2 = ls->dist * ls->dist;
    float cy = omax(0.0f, vdot(vneg(ls->dir), ls->normal));
    if (cy <= 0.0f && !light_delta(s, li)) return 0;
    *pn = pdf_sa(ls->pdf, ls->solid, d2, omax(cy, 1e-6f));
    if (*pn <= 0.0f) return 0;
    if (occluded(s, vadd(sf->hit.position, vmulf(sf->sn, 1e-4f)), ls->dir, ls->dist)) return 0;
    ov3 wo = vneg(sf->rd);
    *bp = ggx_pdf(&sf->c, sf->sn, wo, ls->dir);
    ov3 bv = ggx_eval(&sf->c, sf->sn, wo, ls->dir);
    *rad = smulf(smul(orc_rgb_to_spectrum(bv, w), light_emission(s, li, ls->color, w)), nl / *pn);
    return 1;
}

static ospec mis_li(const orc_scene *s, const osurf *sf, const oconn *cn, const olambda *w, orc_rng *r) {
    ospec total = S1(0.0f);
    int use_bsdf = cn != NULL;
    /* _integrateNEE :122-178; the physical sky is outside the sampler: a technique of its own */
    int separate = has_env(s) && env_sel(s) <= 0.0f;
    int li;
    olsample ls;
    if (propose(s, sf->hit.position, r, &li, &ls)) {
        ospec rad;
        float pn, bp;
        if (mis_nee(s, sf, li, &ls, w, &rad, &pn, &bp)) {
            float mw = (light_delta(s, li) || !use_bsdf) ? 1.0f : (separate ? ph3(pn, 1, 0.0f, 1, bp, 1) : ph2(pn, bp));
            total = sadd(total, smulf(rad, mw));
        }
    }
    if (separate && sky_sun(s, &ls)) { /* the sun: a delta light, weight 1 */
        ospec rad;
        float pn, bp;
        if (mis_nee(s, sf, s->n_lights, &ls, w, &rad, &pn, &bp)) total = sadd(total, smulf(rad, 1.0f));
    }
    if (!cn) return total;
    /* _integrateBSDFConnection :180-248 */
    const obounce *b = &cn->b;
    if (b->impossible || b->pdf <= 0.0f) {
        if (!cn->has_hit) return sadd(total, smul(orc_rgb_to_spectrum(env_sample(s, b->d), w), b->tmul));
        oclosure hc = closure_of(s, &cn->hit);
        return sadd(total, smul(orc_rgb_to_spectrum(hc.emission, w), b->tmul));
    }
    float ps = 0.0f, pe = 0.0f;
    ospec rad;
    if (!cn->has_hit) {
        if (!has_env(s)) return total;
        rad = orc_rgb_to_spectrum(env_sample(s, b->d), w);
        float sel = env_sel(s), ep = env_pdf(s, b->d);
        ps = sel * ep;
        pe = sel <= 0.0f ? ep : 0.0f;
    } else {
        oclosure hc = closure_of(s, &cn->hit);
        rad = orc_rgb_to_spectrum(hc.emission, w);
        int hl = hit_light(s, &cn->hit);
        if (hl >= 0) {
            float sel = select_pdf(s);
            if (sel > 0.0f) {
                ov3 off = vsub(cn->hit.position, b->o);
                float d2 = vdot(off, off);
                float cy = omax(0.0f, vdot(vneg(b->d), cn->hit.normal));
                if (cy > 0.0f) {
                    float av;
                    int so;
                    light_eval_pdf(s, hl, b->d, &av, &so);
                    ps = sel * pdf_sa(av, so, d2, cy);
                }
            }
        }
    }
    if (ps + pe <= 0.0f) return sadd(total, smul(rad, b->tmul));
    float mw = ph3(b->pdf, 1, ps, 1, pe, 1);
    return sadd(total, smul(smulf(rad, mw), b->tmul));
}

/* ---- RisDirectLightIntegrator (restir/ris_direct_light_integrator.cpp) ---- */
typedef struct {
    int valid, has_lc, light;
    olsample ls;
    int origin;
    ospec tp;
    double ris_weight, target;
    int vis_tested;
} ocand;

typedef struct {
    ospec emission, tmul;
    float p_nee, p_bsdf;
    int use_mis, vis_tested;
} ocontrib;

static ocand cand_none(void) {
    ocand c;
    memset(&c, 0, sizeof(c));
    c.vis_tested = 1;
    c.light = -1;
    return c;
}

/* _evaluateLightSample (:628-673) */
static ocontrib eval_light_sample(const orc_scene *s, const osurf *sf, int li, const olsample *ls, int skip,
                                  const olambda *w) {
    ov3 wo = vneg(sf->rd);
    float nl = vdot(sf->sn, ls->dir);
    float d2 = ls->dist * ls->dist;
    float cy = omax(0.0f, vdot(vneg(ls->dir), ls->normal));
    float pn = pdf_sa(ls->pdf, ls->solid, d2, omax(cy, 1e-6f));
    float pb = ggx_pdf(&sf->c, sf->sn, wo, ls->dir);
    ov3 bv = ggx_eval(&sf->c, sf->sn, wo, ls->dir);
    int delta = light_delta(s, li);
    ocontrib r = {S1(0), S1(0), pn, pb, !delta, 1};
    if (nl <= 0.0f || pn <= 0.0f || (cy <= 0.0f && !delta)) return r;
    r.tmul = orc_rgb_to_spectrum(vmulf(bv, nl), w);
    if (skip) {
        r.emission = light_emission(s, li, ls->color, w);
        r.vis_tested = 0;
        return r;
    }
    if (occluded(s, vadd(sf->hit.position, vmulf(sf->sn, 1e-4f)), ls->dir, ls->dist)) return r;
    r.emission = light_emission(s, li, ls->color, w);
    return r;
}

/* _evaluateBSDFConnection (:693-780) */
static ocontrib eval_bsdf_connection(const orc_scene *s, const osurf *sf, const oconn *cn, int n_sky,
                                     const olambda *w) {
    const obounce *b = &cn->b;
    ocontrib r = {S1(0), b->integ, 0.0f, b->pdf, 0, 1};
    if (b->impossible || b->pdf <= 0.0f) {
        if (!cn->has_hit) {
            if (has_env(s)) r.emission = orc_rgb_to_spectrum(env_sample(s, b->d), w);
            return r;
        }
        r.emission = orc_rgb_to_spectrum(closure_of(s, &cn->hit).emission, w);
        return r;
    }
    if (!cn->has_hit) {
        if (!has_env(s)) return r;
        float sel = env_sel(s), ep = env_pdf(s, b->d);
        float pn = sel > 0.0f ? sel * ep : (n_sky > 0 ? ep : 0.0f);
        r.emission = orc_rgb_to_spectrum(env_sample(s, b->d), w);
        r.p_nee = pn;
        r.use_mis = pn > 0.0f;
        return r;
    }
    float pn = 0.f;
    r.emission = orc_rgb_to_spectrum(closure_of(s, &cn->hit).emission, w);
    int hl = hit_light(s, &cn->hit);
    if (hl >= 0) {
        float sel = select_pdf(s);
        ov3 off = vsub(cn->hit.position, b->o);
        float d2 = vdot(off, off);
        float cy = omax(0.0f, vdot(vneg(b->d), cn->hit.normal));
        if (cy > 0.0f && sel > 0.0f) {
            float av;
            int so;
            light_eval_pdf(s, hl, b->d, &av, &so);
            pn = sel * pdf_sa(av, so, d2, cy);
        }
    }
    r.p_nee = pn;
    r.use_mis = pn > 0.0f;
    return r;
}

static ospec reeval(const orc_scene *s, const osurf *sf, int li, const olsample *ls, const olambda *w) {
    ov3 wo = vneg(sf->rd);
    float nl = vdot(sf->sn, ls->dir);
    float d2 = ls->dist * ls->dist;
    float cy = omax(0.0f, vdot(vneg(ls->dir), ls->normal));
    float pn = pdf_sa(ls->pdf, ls->solid, d2, omax(cy, 1e-6f));
    if (nl <= 0.0f || pn <= 0.0f || (cy <= 0.0f && !light_delta(s, li))) return S1(0.0f);
    ov3 bv = ggx_eval(&sf->c, sf->sn, wo, ls->dir);
    return smul(light_emission(s, li, ls->color, w), orc_rgb_to_spectrum(vmulf(bv, nl), w));
}

/* per-pixel RIS trace records for parity tests */
static ospec ris_li(const orc_scene *s, const osurf *sf, const oconn *cn, const olambda *w, orc_rng *r,
                    int primary, const orc_ris_params *p, orc_reservoir *res, orc_pixel_trace *tr) {
    int N = p->candidate_count;
    /* technique split (:89-99): sky NEE when the environment is outside the light sampler */
    int sep = has_env(s) && env_sel(s) <= 0.0f;
    int n_tech = sep ? 3 : 2;
    int n_nee = N / n_tech > 1 ? N / n_tech : 1, n_sky = sep ? N / n_tech : 0;
    int n_bsdf = N - n_nee - n_sky;
    if (n_bsdf < 0) n_bsdf = 0;
    int cap = n_nee + n_sky + n_bsdf + 1;
    ocand *all = (ocand *)malloc((size_t)cap * sizeof(ocand));
    int n = 0;
    /* _generateNEECandidates (:553-626) */
    for (int i = 0; i < n_nee; ++i) {
        int li;
        olsample ls;
        ocand c = cand_none();
        if (propose(s, sf->hit.position, r, &li, &ls)) {
            ocontrib nee = eval_light_sample(s, sf, li, &ls, p->skip_visibility, w);
            ospec contrib = smul(nee.emission, nee.tmul);
            float target = orc_spectrum_luminance(contrib, w);
            float mis = nee.use_mis ? ph3(nee.p_nee, n_nee, 0.0f, n_sky, nee.p_bsdf, n_bsdf) : 1.0f;
            c.valid = 1;
            c.has_lc = 1;
            c.light = li;
            c.ls = ls;
            c.origin = 0;
            c.tp = contrib;
            c.ris_weight = (mis * target) / ((double)nee.p_nee + 1e-9);
            c.target = (double)target;
            c.vis_tested = nee.vis_tested;
            if (tr && tr->n_nee_idx < ORC_MAX_TRACE) tr->nee_light[tr->n_nee_idx++] = li;
        } else if (tr && tr->n_nee_idx < ORC_MAX_TRACE) {
            tr->nee_light[tr->n_nee_idx++] = -1;
        }
        all[n++] = c;
    }
    /* sky NEE (:445-475): the physical sky's SampleLight, the sun */
    for (int i = 0; i < n_sky; ++i) {
        olsample ls;
        ocand c = cand_none();
        if (sky_sun(s, &ls)) {
            ocontrib nee = eval_light_sample(s, sf, s->n_lights, &ls, p->skip_visibility, w);
            ospec contrib = smul(nee.emission, nee.tmul);
            float target = orc_spectrum_luminance(contrib, w);
            float mis = nee.use_mis ? ph3(nee.p_nee, n_sky, 0.0f, n_nee, nee.p_bsdf, n_bsdf) : 1.0f;
            c.valid = 1;
            c.has_lc = 1;
            c.light = s->n_lights;
            c.ls = ls;
            c.origin = 1;
            c.tp = contrib;
            c.ris_weight = (mis * target) / ((double)nee.p_nee + 1e-9);
            c.target = (double)target;
            c.vis_tested = nee.vis_tested;
        }
        all[n++] = c;
    }
    /* _generateBSDFSamplingCandidates (:396-551) */
    int first = n;
    if (cn && cn->b.pdf > 0.0f) {
        ocontrib bc = eval_bsdf_connection(s, sf, cn, n_sky, w);
        ospec contrib = smul(bc.emission, bc.tmul);
        double target = (double)orc_spectrum_luminance(contrib, w);
        float ps = bc.p_nee, pk = 0.0f;
        if (!cn->has_hit && (!has_env(s) || env_sel(s) <= 0.0f)) {
            ps = 0.0f;
            pk = bc.p_nee;
        }
        double mis = (double)ph3(bc.p_bsdf, n_bsdf, ps, n_nee, pk, n_sky);
        ocand c = cand_none();
        c.valid = 1;
        c.tp = contrib;
        c.ris_weight = mis * target / ((double)bc.p_bsdf + 1e-9);
        c.target = target;
        all[n++] = c;
    }
    int to_gen = n_bsdf - (n - first);
    for (int i = 0; i < to_gen; ++i) {
        int refl = 0, refr = 0;
        oconn sc = bounce_with_connection(s, sf, 1, 1, &refl, &refr, w, r);
        ocand c = cand_none();
        if (!sc.b.ok) {
            all[n++] = c;
            continue;
        }
        if (!sc.has_hit) {
            if (!has_env(s)) {
                all[n++] = c;
                continue;
            }
            ov3 wi = sc.b.d;
            ov3 env_rgb = env_sample(s, wi);
            ospec em = orc_rgb_to_spectrum(env_rgb, w);
            float pb = sc.b.pdf, sel = env_sel(s), ep = env_pdf(s, wi);
            float ps = sel * ep, pk = (sel <= 0.0f && n_sky > 0) ? ep : 0.0f, pn = ps + pk;
            double target = (double)orc_spectrum_luminance(smul(em, sc.b.integ), w);
            double mis = (double)ph3(pb, n_bsdf, ps, n_nee, pk, n_sky);
            c.valid = 1;
            c.has_lc = pn > 0.0f;
            c.light = s->sky ? -1 : s->env;
            c.ls.dir = wi;
            c.ls.color = env_rgb;
            c.ls.normal = vneg(wi);
            c.ls.dist = 1e30f;
            c.ls.pdf = pn;
            c.ls.solid = 1;
            c.origin = 2;
            c.tp = smul(em, sc.b.integ);
            c.ris_weight = mis * target / ((double)pb + 1e-9);
            c.target = target;
            all[n++] = c;
            continue;
        }
        int hl = hit_light(s, &sc.hit);
        if (hl < 0) {
            all[n++] = c;
            continue;
        }
        ocontrib bc = eval_bsdf_connection(s, sf, &sc, n_sky, w);
        ospec contrib = smul(bc.emission, bc.tmul);
        double target = (double)orc_spectrum_luminance(contrib, w);
        double mis = (double)ph3(bc.p_bsdf, n_bsdf, bc.p_nee, n_nee, 0.0f, n_sky);
        float av;
        int so;
        light_eval_pdf(s, hl, sc.b.d, &av, &so);
        av *= select_pdf(s);
        c.valid = 1;
        c.has_lc = 1;
        c.light = hl;
        c.ls.dir = sc.b.d;
        c.ls.color = closure_of(s, &sc.hit).emission;
        c.ls.normal = sc.hit.normal;
        c.ls.dist = sc.hit.depth;
        c.ls.pdf = av;
        c.ls.solid = so;
        c.origin = 2;
        c.tp = contrib;
        c.ris_weight = mis * target / ((double)bc.p_bsdf + 1e-9);
        c.target = target;
        all[n++] = c;
    }
    ospec out = S1(0.0f);
    if (p->use_reservoir && primary) {
        /* reservoir branch (:267-331), WeightedReservoir (reservoir.h:69-161) */
        ocand chosen = cand_none();
        float wsum = 0.0f;
        int m = 0;
        for (int i = 0; i < n; ++i) {
            ++m;
            if (!all[i].valid) continue;
            float wt = (float)all[i].ris_weight;
            if (wt <= 0.0f) continue;
            wsum += wt;
            if (orc_rng_float(r) <= wt / wsum) chosen = all[i];
        }
        if (res->has_sample && res->has_lc) {
            olsample pls = {V(res->dir[0], res->dir[1], res->dir[2]), V(res->color[0], res->color[1], res->color[2]),
                            V(res->normal[0], res->normal[1], res->normal[2]), res->dist, res->pdf,
                            res->pdf_solid};
            ospec re = reeval(s, sf, res->light, &pls, w);
            float pc = orc_spectrum_luminance(re, w);
            float pg = (float)res->target;
            if (pg > 0.0f) {
                int pm = res->m;
                float pw = res->wsum;
                if (p->m_cap > 0) { /* extension (no reference counterpart) */
                    int capm = p->m_cap * n;
                    if (pm > capm) {
                        pw *= (float)capm / (float)pm;
                        pm = capm;
                    }
                }
                float mw = pw * (pc / pg);
                m += pm;
                if (mw > 0.0f) {
                    wsum += mw;
                    if (orc_rng_float(r) <= mw / wsum) {
                        chosen = cand_none();
                        chosen.valid = 1;
                        chosen.has_lc = 1;
                        chosen.light = res->light;
                        chosen.ls = pls;
                        chosen.origin = res->origin;
                        chosen.tp = re;
                        chosen.target = (double)pc;
                        chosen.vis_tested = res->vis_tested;
                    }
                }
            }
        }
        /* Finalize (reservoir.h:108-125) */
        float W = 0.0f;
        if (chosen.valid && m > 0) {
            float ph = (float)chosen.target;
            if (ph > 0.0f) {
                int frames = m / (n > 1 ? n : 1);
                if (frames < 1) frames = 1;
                W = wsum / ((float)frames * ph);
                if (!isfinite(W)) W = 0.0f;
            }
        }
        if (chosen.valid && !chosen.vis_tested && chosen.has_lc) {
            ocontrib nee = eval_light_sample(s, sf, chosen.light, &chosen.ls, 0, w);
            chosen.tp = smul(nee.emission, nee.tmul);
            chosen.vis_tested = 1;
        }
        res->has_sample = chosen.valid;
        res->has_lc = chosen.has_lc;
        res->light = chosen.light;
        res->dir[0] = chosen.ls.dir.x, res->dir[1] = chosen.ls.dir.y, res->dir[2] = chosen.ls.dir.z;
        res->color[0] = chosen.ls.color.x, res->color[1] = chosen.ls.color.y, res->color[2] = chosen.ls.color.z;
        res->normal[0] = chosen.ls.normal.x, res->normal[1] = chosen.ls.normal.y, res->normal[2] = chosen.ls.normal.z;
        res->dist = chosen.ls.dist;
        res->pdf = chosen.ls.pdf;
        res->pdf_solid = chosen.ls.solid;
        res->origin = chosen.origin;
        memcpy(res->tp, chosen.tp.v, sizeof(res->tp));
        res->target = (float)chosen.target;
        res->vis_tested = chosen.vis_tested;
        res->wsum = wsum;
        res->m = m;
        res->w = W;
        if (chosen.valid && W > 0.0f) out = smulf(chosen.tp, W);
    } else {
        /* standard RIS (:333-361), RIS::RandomIndexFromWeights (random_index.h:27-63) */
        double ws = 0.0;
        for (int i = 0; i < n; ++i)
            if (all[i].valid && all[i].ris_weight > 0.0) ws += all[i].ris_weight;
        if (ws > 0.0) {
            double rem = (double)orc_rng_float(r) * ws;
            int ch = -1;
            for (int i = 0; i < n; ++i) {
                double wt = all[i].valid ? all[i].ris_weight : 0.0;
                if (wt <= 0.0) continue;
                rem -= wt;
                if (rem <= 0.0) {
                    ch = i;
                    break;
                }
            }
            if (ch >= 0 && all[ch].valid) {
                float W = (float)(ws / all[ch].target);
                ospec tp = all[ch].tp;
                if (!all[ch].vis_tested && all[ch].has_lc) {
                    ocontrib nee = eval_light_sample(s, sf, all[ch].light, &all[ch].ls, 0, w);
                    tp = smul(nee.emission, nee.tmul);
                }
                out = smulf(tp, W);
                if (tr) tr->ris_choice = ch;
            }
        }
    }
    if (tr) tr->n_candidates = n;
    free(all);
    return out;
}

/* ---- PathIntegrator (integrators/path_integrator.cpp:48-209) ------------- */
static osurf make_surf(ov3 ro, ov3 rd, const ohit *h, const oclosure *c, int inside) {
    osurf sf;
    sf.ro = ro;
    sf.rd = rd;
    sf.hit = *h;
    sf.c = *c;
    sf.inside = inside;
    sf.sn = inside ? vneg(c->normal) : c->normal;
    return sf;
}

static ospec direct(const orc_scene *s, const osurf *sf, const oconn *cn, const olambda *w, orc_rng *r, int primary,
                    const orc_frame_params *fp, orc_reservoir *res, orc_pixel_trace *tr) {
    if (fp->ris) return ris_li(s, sf, cn, w, r, primary, &fp->ris_params, res, primary ? tr : NULL);
    return mis_li(s, sf, cn, w, r);
}

static ospec path_li(const orc_scene *s, ov3 ro, ov3 rd, int has, ohit hit, const olambda *w, orc_rng *r,
                     const orc_frame_params *fp, orc_reservoir *res, orc_pixel_trace *tr) {
    const orc_path_params *pp = &fp->path;
    ospec tp = S1(1.0f);
    while (has) {
        oclosure c = closure_of(s, &hit);
        if (!pp->enable_subsurface) c.subsurface = 0.0f;
        if (c.opacity >= 0.999f || orc_rng_float(r) <= c.opacity) {
            int inside = vdot(c.normal, rd) > 0.0f;
            beer(&tp, &c, hit.depth, inside, w);
            osurf sf0 = make_surf(ro, rd, &hit, &c, inside);
            /* _li (:92-209) */
            ospec total = orc_rgb_to_spectrum(sf0.c.emission, w);
            ospec t2 = S1(1.0f);
            int refl = 0, refr = 0;
            oconn first = bounce_with_connection(s, &sf0, pp->max_refl, pp->max_refr, &refl, &refr, w, r);
            total = sadd(total, direct(s, &sf0, first.b.ok ? &first : NULL, w, r, 1, fp, res, tr));
            if (first.b.ok) {
                t2 = smul(t2, first.b.tmul);
                ov3 cro = first.b.o, crd = first.b.d;
                int hn = first.has_hit;
                ohit nx = first.hit;
                for (int bounce = 1; bounce < pp->max_depth; ++bounce) {
                    if (!hn) break;
                    ohit bh = nx;
                    oclosure bc = closure_of(s, &bh);
                    if (!pp->enable_subsurface) bc.subsurface = 0.0f;
                    if (bc.opacity < 0.999f && orc_rng_float(r) > bc.opacity) {
                        cro = vadd(bh.position, vmulf(crd, 1e-4f));
                        hn = orc_intersect(s, cro, crd, &nx);
                        --bounce;
                        continue;
                    }
                    int in2 = vdot(bc.normal, crd) > 0.0f;
                    beer(&t2, &bc, bh.depth, in2, w);
                    osurf sf = make_surf(cro, crd, &bh, &bc, in2);
                    oconn cn = bounce_with_connection(s, &sf, pp->max_refl, pp->max_refr, &refl, &refr, w, r);
                    total = sadd(total, smul(t2, direct(s, &sf, cn.b.ok ? &cn : NULL, w, r, 0, fp, res, tr)));
                    if (!cn.b.ok) break;
                    t2 = smul(t2, cn.b.tmul);
                    cro = cn.b.o;
                    crd = cn.b.d;
                    hn = cn.has_hit;
                    nx = cn.hit;
                    if (cn.b.skip_roulette) continue;
                    if (bounce > 3) {
                        float pr = oclamp(omax(omax(omax(t2.v[0], t2.v[1]), t2.v[2]), t2.v[3]) * pp->roulette, 0.0f,
                                          1.0f);
                        if (orc_rng_float(r) > pr) break;
                        t2 = smulf(t2, 1.0f / pr);
                    }
                }
            }
            return smul(tp, total);
        }
        has = orc_intersect(s, vadd(hit.position, vmulf(rd, 1e-4f)), rd, &hit);
    }
    if (has_env(s) && pp->render_ibl_background) return orc_rgb_to_spectrum(env_sample(s, rd), w);
    return S1(0.0f);
}

/* ---- camera (scene/camera_ray.cpp:10-76) ---------------------------------- */
static void m4d_xform(const double *m, const double *v, double *o) {
    double x = v[0] * m[0] + v[1] * m[4] + v[2] * m[8] + m[12];
    double y = v[0] * m[1] + v[1] * m[5] + v[2] * m[9] + m[13];
    double z = v[0] * m[2] + v[1] * m[6] + v[2] * m[10] + m[14];
    double w = v[0] * m[3] + v[1] * m[7] + v[2] * m[11] + m[15];
    double inv = (w != 0.0) ? 1.0 / w : 1.0;
    o[0] = inv * x;
    o[1] = inv * y;
    o[2] = inv * z;
}
static ov3 d2f(const double *v) { return V((float)v[0], (float)v[1], (float)v[2]); }

void orc_camera_ray(const hdr_camera *cam, const double *iv, const double *ip, float px, float py, orc_rng *r,
                    float *o6) {
    float nx = (2.0f * px / cam->width) - 1.0f;
    float ny = (2.0f * py / cam->height) - 1.0f;
    if (cam->has_params && cam->lens_distortion != 0.0f) {
        float r2 = nx * nx + ny * ny;
        float f = 1.0f + cam->lens_distortion * r2;
        nx *= f;
        ny *= f;
    }
    double zero[3] = {0, 0, 0}, t[3], ndc[3] = {nx, ny, -1.0};
    m4d_xform(iv, zero, t);
    ov3 origin = d2f(t);
    m4d_xform(ip, ndc, t);
    ov3 near_cam = d2f(t);
    ov3 ro, rd;
    if (!(cam->has_params && cam->enable_dof)) {
        double nc[3] = {near_cam.x, near_cam.y, near_cam.z};
        m4d_xform(iv, nc, t);
        ov3 nw = d2f(t);
        ro = origin;
        rd = vnorm(vsub(nw, origin));
    } else {
        const double PI = 3.14159265358979323846;
        float ap = (cam->focal_length / 10.0f) / (2.0f * cam->f_stop);
        float lu, lv;
        if (cam->bokeh_blades < 3) {
            float rr = sqrtf(orc_rng_float(r));
            float th = (float)(2.0f * PI * orc_rng_float(r));
            lu = rr * cosf(th);
            lv = rr * sinf(th);
        } else {
            float th = (float)(2.0f * PI * orc_rng_float(r));
            float rr = sqrtf(orc_rng_float(r));
            float sa = (float)(2.0f * PI / (float)cam->bokeh_blades);
            float sec = floorf(th / sa);
            float ais = th - sec * sa;
            float d = cosf(sa / 2.0f) / cosf(sa / 2.0f - ais);
            lu = rr * d * cosf(th);
            lv = rr * d * sinf(th);
        }
        lu *= ap;
        lv *= ap;
        ov3 fc = vmulf(near_cam, cam->focus_distance);
        double lc[3] = {lu, lv, 0.0}, fcd[3] = {fc.x, fc.y, fc.z};
        m4d_xform(iv, lc, t);
        ov3 lw = d2f(t);
        m4d_xform(iv, fcd, t);
        ov3 fw = d2f(t);
        ro = lw;
        rd = vnorm(vsub(fw, lw));
    }
    o6[0] = ro.x, o6[1] = ro.y, o6[2] = ro.z, o6[3] = rd.x, o6[4] = rd.y, o6[5] = rd.z;
}

/* ---- passes ----------------------------------------------------------------- */
static float exposure_mult(const hdr_camera *cam) {
    if (!(cam->has_params && cam->enable_exposure)) return 1.0f;
    float sf = omax(cam->f_stop, 0.1f);
    return (cam->iso / 100.0f) * cam->shutter_speed / (sf * sf) * 100.0f;
}

static void fill_texel(hdr_gbuffer_texel *t, int has, const ohit *h) {
    memset(t, 0, sizeof(*t));
    if (!has) {
        t->depth = 3.402823466e+38f;
        t->prim_id = -1;
        t->tri_id = -1;
        return;
    }
    t->position[0] = h->position.x, t->position[1] = h->position.y, t->position[2] = h->position.z;
    t->depth = h->depth;
    t->normal[0] = h->normal.x, t->normal[1] = h->normal.y, t->normal[2] = h->normal.z;
    t->prim_id = h->prim;
    t->smooth_normal[0] = h->smooth_normal.x, t->smooth_normal[1] = h->smooth_normal.y;
    t->smooth_normal[2] = h->smooth_normal.z;
    t->tri_id = h->tri;
    t->albedo[0] = h->albedo.x, t->albedo[1] = h->albedo.y, t->albedo[2] = h->albedo.z;
    t->hit = 1;
    t->uv[0] = h->uv.x, t->uv[1] = h->uv.y;
    t->dpdu[0] = h->dpdu.x, t->dpdu[1] = h->dpdu.y, t->dpdu[2] = h->dpdu.z;
    t->dpdv[0] = h->dpdv.x, t->dpdv[1] = h->dpdv.y, t->dpdv[2] = h->dpdv.z;
}

static void texel_to_hit(const orc_scene *s, const hdr_gbuffer_texel *t, ohit *h) {
    h->position = V(t->position[0], t->position[1], t->position[2]);
    h->normal = V(t->normal[0], t->normal[1], t->normal[2]);
    h->smooth_normal = V(t->smooth_normal[0], t->smooth_normal[1], t->smooth_normal[2]);
    h->dpdu = V(t->dpdu[0], t->dpdu[1], t->dpdu[2]);
    h->dpdv = V(t->dpdv[0], t->dpdv[1], t->dpdv[2]);
    h->uv.x = t->uv[0], h->uv.y = t->uv[1];
    h->albedo = V(t->albedo[0], t->albedo[1], t->albedo[2]);
    h->depth = t->depth;
    h->prim = t->prim_id;
    h->mat = t->prim_id;
    h->tri = t->tri_id;
    (void)s;
}

typedef struct {
    const orc_scene *s;
    const hdr_camera *cam;
    double iv[16], ip[16];
    int frame;
    const orc_frame_params *fp;
    hdr_gbuffer_texel *gbuf;
    float *color;
    orc_reservoir *res;
    orc_pixel_trace *trace;
    int y0, y1, pass;
} job;

static void *run_rows(void *arg) {
    job *j = (job *)arg;
    const hdr_camera *cam = j->cam;
    for (int y = j->y0; y < j->y1; ++y)
        for (int x = 0; x < cam->width; ++x) {
            size_t i = (size_t)y * cam->width + x;
            uint32_t seed = (uint32_t)i ^ (uint32_t)((unsigned long long)j->frame * 12345ULL);
            orc_rng r;
            orc_rng_seed(&r, seed);
            float ray[6];
            if (j->pass == 0) { /* RaycastPass (raycast_pass.cpp:108-157) */
                orc_camera_ray(cam, j->iv, j->ip, (float)x + 0.5f, (float)y + 0.5f, &r, ray);
                ohit h;
                int has = orc_intersect(j->s, V(ray[0], ray[1], ray[2]), V(ray[3], ray[4], ray[5]), &h);
                fill_texel(&j->gbuf[i], has, &h);
                continue;
            }
            /* IntegrationPass (integration_pass.cpp:205-244) */
            float px = (float)x + orc_rng_float(&r);
            float py = (float)y + orc_rng_float(&r);
            orc_camera_ray(cam, j->iv, j->ip, px, py, &r, ray);
            olambda w = orc_sample_wavelengths(orc_rng_float(&r));
            ohit h;
            int has = j->gbuf[i].prim_id >= 0;
            if (has) texel_to_hit(j->s, &j->gbuf[i], &h);
            orc_pixel_trace *tr = j->trace ? &j->trace[i] : NULL;
            if (tr) memset(tr, 0, sizeof(*tr)), tr->ris_choice = -1;
            ospec L = path_li(j->s, V(ray[0], ray[1], ray[2]), V(ray[3], ray[4], ray[5]), has, h, &w, &r, j->fp,
                              j->res ? &j->res[i] : NULL, tr);
            ov3 c = orc_spectrum_to_rgb(L, &w);
            c = vmulf(c, exposure_mult(cam));
            if (tr) {
                memcpy(tr->L, L.v, sizeof(tr->L));
                memcpy(tr->lambda, w.l, sizeof(tr->lambda));
                tr->draws = -1;
            }
            j->color[4 * i] = c.x, j->color[4 * i + 1] = c.y, j->color[4 * i + 2] = c.z, j->color[4 * i + 3] = 1.0f;
        }
    return NULL;
}

/* rows [base->y0, base->y1) split over threads in interleaved strips of 4 rows */
static void *run_strips(void *arg);
typedef struct {
    job base;
    int t, threads;
} strip_job;
static void *run_strips(void *arg) {
    strip_job *sj = (strip_job *)arg;
    for (int y = sj->base.y0 + 4 * sj->t; y < sj->base.y1; y += 4 * sj->threads) {
        job j = sj->base;
        j.y0 = y;
        j.y1 = y + 4 < sj->base.y1 ? y + 4 : sj->base.y1;
        run_rows(&j);
    }
    return NULL;
}

static void run_pass(job *base, int threads) {
    int H = base->y1 - base->y0;
    if (H <= 0) return;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    if (threads > 1) {
        pthread_t th[256];
        strip_job sj[256];
        for (int t = 0; t < threads; ++t) {
            sj[t].base = *base;
            sj[t].t = t;
            sj[t].threads = threads;
            pthread_create(&th[t], NULL, run_strips, &sj[t]);
        }
        for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
        return;
    }
    run_rows(base);
}

void orc_raycast_band(const orc_scene *s, const hdr_camera *cam, int frame, hdr_gbuffer_texel *gbuf, int y0,
                      int y1, int threads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.s = s;
    j.cam = cam;
    orc_inverse4d(cam->view, j.iv);
    orc_inverse4d(cam->proj, j.ip);
    j.frame = frame;
    j.gbuf = gbuf;
    j.pass = 0;
    j.y0 = y0;
    j.y1 = y1;
    run_pass(&j, threads);
}

void orc_raycast(const orc_scene *s, const hdr_camera *cam, int frame, hdr_gbuffer_texel *gbuf, int threads) {
    orc_raycast_band(s, cam, frame, gbuf, 0, cam->height, threads);
}

void orc_integrate_band(const orc_scene *s, const hdr_camera *cam, int frame, const orc_frame_params *fp,
                        hdr_gbuffer_texel *gbuf, float *color, orc_reservoir *res, orc_pixel_trace *trace, int y0,
                        int y1, int threads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.s = s;
    j.cam = cam;
    orc_inverse4d(cam->view, j.iv);
    orc_inverse4d(cam->proj, j.ip);
    j.frame = frame;
    j.fp = fp;
    j.gbuf = gbuf;
    j.color = color;
    j.res = res;
    j.trace = trace;
    j.pass = 1;
    j.y0 = y0;
    j.y1 = y1;
    run_pass(&j, threads);
}

void orc_integrate(const orc_scene *s, const hdr_camera *cam, int frame, const orc_frame_params *fp,
                   hdr_gbuffer_texel *gbuf, float *color, orc_reservoir *res, orc_pixel_trace *trace, int threads) {
    orc_integrate_band(s, cam, frame, fp, gbuf, color, res, trace, 0, cam->height, threads);
}

/* AccumulationPass::_execute (passes/accumulation_pass.cpp:22-139): firefly
 * clamp in place, row-major; accum += Color; Color = accum / (frame+1). */
void orc_accumulate(float *color, float *accum, int width, int height, int frame, int firefly) {
    if (firefly) {
        for (int y = 0; y < height; ++y)
            for (int x = 0; x < width; ++x) {
                float *c = &color[4 * ((size_t)y * width + x)];
                float lum = 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2];
                float mx = 0.0f;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (dx == 0 && dy == 0) continue;
                        int nx = oclampi(x + dx, 0, width - 1), ny = oclampi(y + dy, 0, height - 1);
                        const float *q = &color[4 * ((size_t)ny * width + nx)];
                        mx = omax(mx, 0.2126f * q[0] + 0.7152f * q[1] + 0.0722f * q[2]);
                    }
                float thr = mx * 4.0f + 0.5f;
                if (lum > thr && lum > 0.0f) {
                    float sc = thr / lum;
                    c[0] *= sc;
                    c[1] *= sc;
                    c[2] *= sc;
                }
            }
    }
    float inv = 1.0f / (float)(frame + 1);
    size_t n = (size_t)width * height * 4;
    for (size_t i = 0; i < n; ++i) {
        accum[i] += color[i];
        color[i] = accum[i] * inv;
    }
}

/* GpuAccumulationPass's shader (gpu_functions/shaders/accumulation.slang:55-97):
 * the same firefly rule, but every pixel clamps against the unclamped input
 * (colorIn), then acc = accum + colour, out = acc * invN. Metrics off. */
void orc_accumulate_shader(float *color, float *accum, int width, int height, int frame, int firefly) {
    size_t n = (size_t)width * height;
    float *out = (float *)malloc(n * 4 * sizeof(float));
    float inv = 1.0f / (float)(frame + 1);
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            size_t i = (size_t)y * width + x;
            float c[4] = {color[4 * i], color[4 * i + 1], color[4 * i + 2], color[4 * i + 3]};
            if (firefly) {
                float mx = 0.0f;
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if (dx == 0 && dy == 0) continue;
                        int nx = oclampi(x + dx, 0, width - 1), ny = oclampi(y + dy, 0, height - 1);
                        const float *q = &color[4 * ((size_t)ny * width + nx)];
                        mx = omax(mx, 0.2126f * q[0] + 0.7152f * q[1] + 0.0722f * q[2]);
                    }
                float thr = mx * 4.0f + 0.5f;
                float lum = 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2];
                if (lum > thr && lum > 0.0f) {
                    float sc = thr / lum;
                    c[0] *= sc;
                    c[1] *= sc;
                    c[2] *= sc;
                }
            }
            for (int k = 0; k < 4; ++k) {
                accum[4 * i + k] += c[k];
                out[4 * i + k] = accum[4 * i + k] * inv;
            }
        }
    memcpy(color, out, n * 4 * sizeof(float));
    free(out);
}

/* WeightedReservoir::Update + Finalize (restir/reservoir.h:76-125) for one
 * candidate with the given weight and target function; returns W. The draw
 * comes from Rng{777} as in tests/test_reservoir.cpp:67-76. */
float orc_reservoir_known_answer(float weight, float phat, int candidates_per_frame) {
    orc_rng r;
    orc_rng_seed(&r, 777u);
    int m = 0, chosen = 0;
    float wsum = 0.0f, chosen_phat = 0.0f;
    ++m;
    if (weight > 0.0f) {
        wsum += weight;
        if (orc_rng_float(&r) <= weight / wsum) {
            chosen = 1;
            chosen_phat = phat;
        }
    }
    if (!chosen || m <= 0) return 0.0f;
    if (chosen_phat <= 0.0f) return 0.0f;
    int cpf = candidates_per_frame > 1 ? candidates_per_frame : 1;
    int frames = m / cpf;
    if (frames < 1) frames = 1;
    float w = wsum / ((float)frames * chosen_phat);
    return isfinite(w) ? w : 0.0f;
}

void orc_rng_floats(const uint32_t *seeds, int n, int count, float *out) {
    for (int k = 0; k < n; ++k) {
        orc_rng r;
        orc_rng_seed(&r, seeds[k]);
        for (int j = 0; j < count; ++j) out[(size_t)k * count + j] = orc_rng_float(&r);
    }
}

void orc_trace_rays(const orc_scene *s, const float *rays, const float *tmax, int n, int any_hit,
                    hdr_gbuffer_texel *out) {
    for (int k = 0; k < n; ++k) {
        ov3 o = V(rays[6 * k], rays[6 * k + 1], rays[6 * k + 2]), d = V(rays[6 * k + 3], rays[6 * k + 4], rays[6 * k + 5]);
        ohit h;
        int has = orc_intersect(s, o, d, &h);
        if (any_hit) {
            float lim = tmax ? tmax[k] : 3.402823466e+38f;
            int occ = has && h.depth < lim;
            memset(&out[k], 0, sizeof(out[k]));
            out[k].depth = occ ? h.depth : 3.402823466e+38f;
            out[k].prim_id = occ ? h.prim : -1;
            out[k].tri_id = occ ? h.tri : -1;
            out[k].hit = occ;
        } else {
            fill_texel(&out[k], has, &h);
        }
    }
}
