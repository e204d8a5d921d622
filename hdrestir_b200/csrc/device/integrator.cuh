// Integrators on the device.
//   PathIntegrator::Li / _li                 integrators/path_integrator.cpp:48-209
//   SampleBounceWithConnection              integrators/direct_light_integrator_interface.h:18-40
//   MisDirectLightIntegrator                integrators/mis_direct_light_integrator.cpp:37-271
//   RisDirectLightIntegrator (RIS, ReSTIR)  restir/ris_direct_light_integrator.cpp:84-634
//   WeightedReservoir                       restir/reservoir.h:69-161
//   RIS::RandomIndexFromWeights             restir/random_index.h:27-63
//
// One thread integrates one pixel. Candidate generation keeps only the running
// reservoir (no per-candidate arrays): the reference draws all candidate
// samples first and the reservoir-update numbers after them, so the kernel
// first replays the sampling decisions alone (no rays) to find where the
// update numbers start, then generates the candidates for real while a second
// cursor on the same stream supplies the update numbers. Both cursors must end
// where the reference's single stream would; a mismatch raises kErrRngDesync.
#pragma once

#include "frame.cuh"
#include "lights.cuh"
#include "material.cuh"

namespace hdr {

constexpr unsigned kErrRngDesync = 4u;
constexpr unsigned kErrRisCapacity = 8u;
constexpr int kMaxPlainRisCandidates = 64;

struct Surface {  // RayIntersection with its ShadingPoint
    V3 ray_o, ray_d;
    Hit hit;
    Closure c;
    V3 sn;  // shading normal
    bool inside;
    GgxFixed g;  // GGX terms of (c, sn, -ray_d), shared by every light direction evaluated here
};

struct Connection {  // BsdfBounceConnection
    Bounce b;
    bool has_hit;
    Hit hit;
};

// Scene::IntersectScene -> optional<HitRecord>
__device__ __forceinline__ bool intersect(const DeviceScene &s, V3 o, V3 d, Hit &h, unsigned &err) {
    HitId id;
    if (!trace_ray<false>(s, o, d, 0.0f, id, err)) return false;
    h = make_hit(s, o, d, id);
    return true;
}
// "shadowHit && shadowHit->Depth < limit"
__device__ __forceinline__ bool occluded(const DeviceScene &s, V3 o, V3 d, float limit, unsigned &err) {
    return shadow_ray(s, o, d, limit, err);
}

// The same query behind a call: kernels that cast a shadow ray only on a rare
// path keep the traversal's registers out of their hot loop. Returns the answer
// in bit 0 and the error bits shifted up by one. (Each translation unit gets its
// own copy: the library is compiled without device linking.)
__device__ __noinline__ static unsigned occluded_call(const DeviceScene *s, V3 o, V3 d, float limit) {
    unsigned e = 0;
    const bool occ = occluded(*s, o, d, limit, e);
    return (occ ? 1u : 0u) | (e << 1);
}

// Where the integrators get ray results from. Every ray a pixel casts has a
// slot: closest-hit slot 0 is the path's bounce ray, closest-hit slot 1 + k
// the k-th generated BSDF candidate, shadow slot j the j-th NEE candidate.
// TraceNow traverses at the call (one thread per pixel); TracedResults reads
// what the wavefront trace kernels wrote for the pixel's slots.
struct TraceNow {
    const DeviceScene *s;
    __device__ __forceinline__ bool fresh_bsdf_empty() const { return false; }
    __device__ __forceinline__ bool shadow(int, V3 o, V3 d, float limit, unsigned &err) const {
        return occluded(*s, o, d, limit, err);
    }
    __device__ __forceinline__ bool closest(int, V3 o, V3 d, Hit &h, unsigned &err) const {
        return intersect(*s, o, d, h, err);
    }
    __device__ __forceinline__ bool winner_shadow(V3 o, V3 d, float limit, unsigned &err) const {
        return occluded(*s, o, d, limit, err);
    }
};

struct TracedResults {
    const DeviceScene *s;
    const float4 *hits;        // this pixel's closest-hit slots: t, instance bits, triangle bits, u
    const float *hit_v;        // and v
    const unsigned char *occ;  // this pixel's shadow slots
    int trace_level;           // kTrace*: which closest-hit slots were cast (the others cannot matter)
    float4 *q_winner;          // non-null: the winner's shadow ray is queued (answer fixed up later)
    int *winner_count;
    int pixel;
    // Every generated BSDF candidate is invalid whatever it samples: its ray was
    // not cast because the scene has no light geometry and no environment.
    __device__ __forceinline__ bool fresh_bsdf_empty() const { return trace_level < kTraceAllBsdfRays; }
    __device__ __forceinline__ bool shadow(int slot, V3, V3, float, unsigned &) const { return occ[slot] != 0; }
    __device__ __forceinline__ bool closest(int slot, V3 o, V3 d, Hit &h, unsigned &) const {
        if (trace_level < (slot > 0 ? kTraceAllBsdfRays : kTraceBounceRay)) return false;
        const float4 r = hits[slot];
        const HitId id{r.x, fbits(r.y), fbits(r.z), r.w, hit_v[slot]};
        if (id.inst < 0) return false;
        h = make_hit(*s, o, d, id);
        return true;
    }
    // The winner's visibility test (skipVisibility, or a sample taken from history): queued for
    // the shadow kernel and answered "visible" here; a pixel whose ray turns out occluded is
    // fixed up afterwards (its throughput is then 0, as the test on the spot would have made it).
    // Without a queue the ray is cast on the spot.
    __device__ __forceinline__ bool winner_shadow(V3 o, V3 d, float limit, unsigned &err) const {
        if (q_winner) {
            const int k = atomicAdd(winner_count, 1);
            q_winner[2 * (size_t)k] = make_float4(o.x, o.y, o.z, __int_as_float(pixel));
            q_winner[2 * (size_t)k + 1] = make_float4(d.x, d.y, d.z, limit);
            return false;
        }
        const unsigned r = occluded_call(s->dev, o, d, limit);
        err |= r >> 1;
        return (r & 1u) != 0;
    }
};

__device__ __forceinline__ Surface make_surface(const DeviceScene &s, V3 ro, V3 rd, const Hit &h, const Closure &c,
                                                bool inside) {
    Surface sf;
    sf.ray_o = ro;
    sf.ray_d = rd;
    sf.hit = h;
    sf.c = c;
    sf.inside = inside;
    sf.sn = inside ? -c.normal : c.normal;
    sf.g = ggx_fixed(c, sf.sn, -rd);
    return sf;
}

// GBuffer texel -> HitRecord (the "GBuffer" input of IntegrationPass, integration_pass.cpp:184)
__device__ inline bool load_gbuffer_hit(const DeviceScene &s, const GBufferView &gb, size_t i, Hit &h) {
    const float4 a = gb.pos_depth[i], b = gb.normal_prim[i], c = gb.smooth_tri[i], d = gb.albedo_uv[i];
    h.prim = fbits(b.w);
    if (h.prim < 0) return false;
    h.position = V3{a.x, a.y, a.z};
    h.depth = a.w;
    h.normal = V3{b.x, b.y, b.z};
    h.smooth_normal = V3{c.x, c.y, c.z};
    h.tri = fbits(c.w);
    h.albedo = V3{d.x, d.y, d.z};
    if (s.has_textures) {  // a texture lookup needs uv.y and the tangents (the only readers of them)
        const float4 e = gb.aux0[i], f = gb.aux1[i];
        h.uv = V2{d.w, e.x};
        h.dpdu = V3{e.y, e.z, e.w};
        h.dpdv = V3{f.x, f.y, f.z};
    } else {
        h.uv = V2{d.w, 0.0f};
        h.dpdu = h.dpdv = v3s(0.0f);
    }
    const float4 r = __ldg(&s.instances[8 * h.prim + 6]);
    const float4 r7 = __ldg(&s.instances[8 * h.prim + 7]);
    h.material = fbits(r.w);
    h.light = fbits(r7.x);
    return true;
}

// Detail::SampleBounceWithConnection
template <class RP>
__device__ __forceinline__ Connection sample_bounce_with_connection(const RP &rp, int slot, const Surface &sf,
                                                                    int max_refl, int max_refr, BounceState &st,
                                                                    const SpectralCtx &sc, MtStream &rng,
                                                                    unsigned &err) {
    Connection cn;
    cn.b = sample_bounce(sf.c, sf.sn, sf.inside, sf.hit.position, sf.ray_d, max_refl, max_refr, st, sc, rng);
    cn.has_hit = false;
    if (cn.b.ok) cn.has_hit = rp.closest(slot, cn.b.origin, cn.b.dir, cn.hit, err);
    return cn;
}

// ============================================================================
// MisDirectLightIntegrator (PathTracePass)
// ============================================================================
// _evaluateNEE (mis_direct_light_integrator.cpp:70-120) up to its shadow ray:
// the light sample's draws and what it adds to the vertex if the ray from
// (o, d) reaches `limit` unoccluded (`add` = radiance x MIS weight of
// _integrateNEE, :122-178). cast = false: no shadow ray, nothing added.
struct MisNeePart {
    bool cast;
    V3 o, d;
    float limit;
    Spec add;
};

__device__ inline MisNeePart mis_nee_part(const DeviceScene &s, const Surface &sf, bool has_conn,
                                          const SpectralCtx &sc, MtStream &rng) {
    MisNeePart r;
    r.cast = false;
    r.add = spec(0.0f);
    // a dome environment is a scene light and so part of the sampler; the physical
    // sky is not, and gets its own technique (mis_sky_part)
    int li;
    LightSampleD ls;
    if (!propose_candidate(s, sf.hit.position, rng, li, ls)) return r;
    const float n_l = dot(sf.sn, ls.dir);
    if (n_l <= 0.0f) return r;
    const bool delta = light_is_delta(s, li);
    const float dist2 = ls.dist * ls.dist;
    const float cos_y = smaxf(0.0f, dot(-ls.dir, ls.normal));
    if (cos_y <= 0.0f && !delta) return r;
    const float p_nee = pdf_to_solid_angle(ls.pdf, ls.pdf_solid_angle, dist2, smaxf(cos_y, 1e-6f));
    if (p_nee <= 0.0f) return r;
    const V3 wo = -sf.ray_d;
    const float bpdf = ggx_pdf_f(sf.g, sf.sn, wo, ls.dir);
    const V3 bval = ggx_eval_f(sf.g, sf.sn, wo, ls.dir);
    const Spec radiance = rgb_to_spectrum(bval, sc.up) * light_emission(s, li, ls.color, sc) * (n_l / p_nee);
    const bool separate_env = env_present(s) && env_select_pdf(s) <= 0.0f;
    const float w = (delta || !has_conn) ? 1.0f
                    : separate_env       ? power_heuristic3(p_nee, 1, 0.0f, 1, bpdf, 1)
                                         : power_heuristic2(p_nee, bpdf);
    r.cast = true;
    r.o = sf.hit.position + sf.sn * 1e-4f;
    r.d = ls.dir;
    r.limit = ls.dist - 1e-3f;
    r.add = radiance * w;
    return r;
}

// The separate environment technique of _integrateNEE (:153-176): the physical
// sky's sun (its SampleLight draws nothing), with what it adds if unoccluded.
__device__ inline MisNeePart mis_sky_part(const DeviceScene &s, const Surface &sf, const SpectralCtx &sc) {
    MisNeePart r;
    r.cast = false;
    r.add = spec(0.0f);
    LightSampleD ls;
    if (!(env_present(s) && env_select_pdf(s) <= 0.0f) || !sky_sun_sample(s, ls)) return r;
    const float n_l = dot(sf.sn, ls.dir);
    if (n_l <= 0.0f) return r;
    const float dist2 = ls.dist * ls.dist;
    const float cos_y = smaxf(0.0f, dot(-ls.dir, ls.normal));
    const float p_nee = pdf_to_solid_angle(ls.pdf, ls.pdf_solid_angle, dist2, smaxf(cos_y, 1e-6f));
    if (p_nee <= 0.0f) return r;
    const V3 wo = -sf.ray_d;
    const V3 bval = ggx_eval_f(sf.g, sf.sn, wo, ls.dir);
    // the sun is a delta light: MIS weight 1
    const Spec radiance = rgb_to_spectrum(bval, sc.up) * rgb_to_spectrum(ls.color, sc.up) * (n_l / p_nee);
    r.cast = true;
    r.o = sf.hit.position + sf.sn * 1e-4f;
    r.d = ls.dir;
    r.limit = ls.dist - 1e-3f;
    r.add = radiance;
    return r;
}

// _integrateBSDFConnection (:180-248) added to what the NEE part gave (`total`).
__device__ inline Spec mis_conn_part(const DeviceScene &s, Spec total, bool has_conn, const Connection &cn,
                                     const SpectralCtx &sc) {
    if (!has_conn) return total;
    // _integrateBSDFConnection (:180-248)
    const Bounce &b = cn.b;
    if (b.impossible_nee || b.pdf <= 0.0f) {
        if (!cn.has_hit) return total + rgb_to_spectrum(env_radiance(s, b.dir), sc.up) * b.tmul;
        const Closure hc = get_closure(s, cn.hit);
        return total + rgb_to_spectrum(hc.emission, sc.up) * b.tmul;
    }
    float p_sampler = 0.0f, p_env = 0.0f;
    Spec radiance;
    if (!cn.has_hit) {
        if (!env_present(s)) return total;
        radiance = rgb_to_spectrum(env_radiance(s, b.dir), sc.up);
        const float sel = env_select_pdf(s);
        const float epdf = env_pdf(s, b.dir);
        p_sampler = sel * epdf;
        p_env = sel <= 0.0f ? epdf : 0.0f;
    } else {
        const Closure hc = get_closure(s, cn.hit);
        radiance = rgb_to_spectrum(hc.emission, sc.up);
        if (cn.hit.light >= 0) {
            const float sel = light_select_pdf(s);
            if (sel > 0.0f) {
                const V3 off = cn.hit.position - b.origin;
                const float dist2 = dot(off, off);
                const float cos_y = smaxf(0.0f, dot(-b.dir, cn.hit.normal));
                if (cos_y > 0.0f) {
                    float av;
                    bool solid;
                    light_eval_pdf(s, cn.hit.light, b.dir, av, solid);
                    p_sampler = sel * pdf_to_solid_angle(av, solid, dist2, cos_y);
                }
            }
        }
    }
    if (p_sampler + p_env <= 0.0f) return total + radiance * b.tmul;
    const float w = power_heuristic3(b.pdf, 1, p_sampler, 1, p_env, 1);
    return total + radiance * w * b.tmul;
}


// MisDirectLightIntegrator::Li (per-bounce form, :250-269) = _integrateNEE + _integrateBSDFConnection
__device__ HDR_BOUNCE_INLINE Spec mis_direct_li(const DeviceScene &s, const Surface &sf, bool has_conn, const Connection &cn,
                                     const SpectralCtx &sc, MtStream &rng, unsigned &err) {
    const MisNeePart nee = mis_nee_part(s, sf, has_conn, sc, rng);
    Spec total = spec(0.0f);
    if (nee.cast && !occluded(s, nee.o, nee.d, nee.limit, err)) total = total + nee.add;
    if (sky_on(s)) {  // the physical sky's sun, after the sampler's candidate
        const MisNeePart sun = mis_sky_part(s, sf, sc);
        if (sun.cast && !occluded(s, sun.o, sun.d, sun.limit, err)) total = total + sun.add;
    }
    return mis_conn_part(s, total, has_conn, cn, sc);
}

// ============================================================================
// RisDirectLightIntegrator
// ============================================================================
struct Cand {  // optional<RISLightCandidate>
    bool valid;
    bool has_lc;  // Candidate (LightCandidate) engaged
    int light;
    LightSampleD ls;
    int origin;   // CandidateOrigin: 0 NEE, 1 SkyNEE, 2 BSDF
    Spec tp;      // Throughput
    double ris_weight;
    float target; // targetFunction (always a float value)
    bool vis_tested;
};

__device__ __forceinline__ Cand cand_none() {
    Cand c;
    c.valid = false;
    c.has_lc = false;
    c.light = -1;
    c.ls = LightSampleD{v3s(0.0f), v3s(0.0f), v3s(0.0f), 1e30f, 0.0f, false};
    c.origin = 0;
    c.tp = spec(0.0f);
    c.ris_weight = 0.0;
    c.target = 0.0f;
    c.vis_tested = true;
    return c;
}

struct RisStrategy {  // SamplingStrategy
    int n_nee, n_sky, n_bsdf;
    bool skip_vis;
};

struct RisContrib {  // RisDirectLightIntegrator::MISContrib
    Spec emission, tmul;
    float p_nee, p_bsdf;
    bool use_mis;
    bool vis_tested;
};

// _evaluateLightSample (:628-673). shadow_slot < 0: the winner's own test.
template <class RP>
__device__ inline RisContrib ris_evaluate_light_sample(const DeviceScene &s, const RP &rp, int shadow_slot,
                                                       const Surface &sf, int li, const LightSampleD &ls,
                                                       bool skip_vis, const SpectralCtx &sc, unsigned &err) {
    const V3 wo = -sf.ray_d;
    const float n_l = dot(sf.sn, ls.dir);
    const float dist2 = ls.dist * ls.dist;
    const float cos_y = smaxf(0.0f, dot(-ls.dir, ls.normal));
    const float p_nee = pdf_to_solid_angle(ls.pdf, ls.pdf_solid_angle, dist2, smaxf(cos_y, 1e-6f));
    const float p_bsdf = ggx_pdf_f(sf.g, sf.sn, wo, ls.dir);
    const V3 bval = ggx_eval_f(sf.g, sf.sn, wo, ls.dir);
    const bool delta = light_is_delta(s, li);
    RisContrib r{spec(0.0f), spec(0.0f), p_nee, p_bsdf, !delta, true};
    if (n_l <= 0.0f || p_nee <= 0.0f || (cos_y <= 0.0f && !delta)) return r;
    r.tmul = rgb_to_spectrum(bval * n_l, sc.up);
    if (skip_vis) {
        r.emission = light_emission(s, li, ls.color, sc);
        r.vis_tested = false;
        return r;
    }
    const V3 so = sf.hit.position + sf.sn * 1e-4f;
    const float lim = ls.dist - 1e-3f;
    const bool occ = shadow_slot >= 0 ? rp.shadow(shadow_slot, so, ls.dir, lim, err) : rp.winner_shadow(so, ls.dir, lim, err);
    if (occ) return r;
    r.emission = light_emission(s, li, ls.color, sc);
    return r;
}

// The shadow ray _evaluateLightSample would cast for a fresh NEE sample, or
// false when its early-outs (or skipVisibility) mean none is cast.
__device__ __forceinline__ bool ris_nee_shadow_ray(const DeviceScene &s, const Surface &sf, int li,
                                                   const LightSampleD &ls, bool skip_vis, V3 &o, V3 &d,
                                                   float &limit) {
    const float n_l = dot(sf.sn, ls.dir);
    const float dist2 = ls.dist * ls.dist;
    const float cos_y = smaxf(0.0f, dot(-ls.dir, ls.normal));
    const float p_nee = pdf_to_solid_angle(ls.pdf, ls.pdf_solid_angle, dist2, smaxf(cos_y, 1e-6f));
    const bool delta = light_is_delta(s, li);
    if (n_l <= 0.0f || p_nee <= 0.0f || (cos_y <= 0.0f && !delta) || skip_vis) return false;
    o = sf.hit.position + sf.sn * 1e-4f;
    d = ls.dir;
    limit = ls.dist - 1e-3f;
    return true;
}

// _reEvaluateForTemporalReuse (:675-691)
__device__ inline Spec ris_reevaluate(const DeviceScene &s, const Surface &sf, int li, const LightSampleD &ls,
                               const SpectralCtx &sc) {
    const V3 wo = -sf.ray_d;
    const float n_l = dot(sf.sn, ls.dir);
    const float dist2 = ls.dist * ls.dist;
    const float cos_y = smaxf(0.0f, dot(-ls.dir, ls.normal));
    const float p_nee = pdf_to_solid_angle(ls.pdf, ls.pdf_solid_angle, dist2, smaxf(cos_y, 1e-6f));
    if (n_l <= 0.0f || p_nee <= 0.0f || (cos_y <= 0.0f && !light_is_delta(s, li))) return spec(0.0f);
    const V3 bval = ggx_eval_f(sf.g, sf.sn, wo, ls.dir);
    return light_emission(s, li, ls.color, sc) * rgb_to_spectrum(bval * n_l, sc.up);
}

// _evaluateBSDFConnection (:693-780); HDR_BOUNCE_INLINE as sample_bounce
__device__ HDR_BOUNCE_INLINE RisContrib ris_evaluate_bsdf_connection(const DeviceScene &s, const Surface &sf, const Connection &cn,
                                                   const RisStrategy &strat, const SpectralCtx &sc) {
    const Bounce &b = cn.b;
    RisContrib r{spec(0.0f), b.integrand, 0.0f, b.pdf, false, true};
    if (b.impossible_nee || b.pdf <= 0.0f) {
        if (!cn.has_hit) {
            if (env_present(s)) r.emission = rgb_to_spectrum(env_radiance(s, b.dir), sc.up);
            return r;
        }
        r.emission = rgb_to_spectrum(get_closure(s, cn.hit).emission, sc.up);
        return r;
    }
    if (!cn.has_hit) {
        if (!env_present(s)) return r;
        const float sel = env_select_pdf(s);
        const float epdf = env_pdf(s, b.dir);
        const float p_nee = sel > 0.0f ? sel * epdf : (strat.n_sky > 0 ? epdf : 0.0f);
        r.emission = rgb_to_spectrum(env_radiance(s, b.dir), sc.up);
        r.p_nee = p_nee;
        r.use_mis = p_nee > 0.0f;
        return r;
    }
    float p_nee = 0.f;
    r.emission = rgb_to_spectrum(get_closure(s, cn.hit).emission, sc.up);
    if (cn.hit.light >= 0) {
        const float sel = light_select_pdf(s);
        const V3 off = cn.hit.position - b.origin;
        const float dist2 = dot(off, off);
        const float cos_y = smaxf(0.0f, dot(-b.dir, cn.hit.normal));
        if (cos_y > 0.0f && sel > 0.0f) {
            float av;
            bool solid;
            light_eval_pdf(s, cn.hit.light, b.dir, av, solid);
            p_nee = sel * pdf_to_solid_angle(av, solid, dist2, cos_y);
        }
    }
    r.p_nee = p_nee;
    r.use_mis = p_nee > 0.0f;
    return r;
}

template <class RP>
struct RisCtx {
    const DeviceScene *s;
    const RP *rp;
    const Surface *sf;
    const SpectralCtx *sc;
    RisStrategy strat;
    bool has_conn;
    const Connection *conn;
    bool conn_cand;  // the caller's connection becomes candidate #0 (its pdf > 0)
    int n_total;     // allCandidates.size()
    int max_refl, max_refr;
};

// Candidate j of allCandidates: NEE (sampler), then sky NEE, then BSDF.
// kFull = false only advances the stream exactly like the full generation.
// HDR_CANDIDATE_INLINE: how the including kernels take it (a call returns the
// candidate through local memory, about 20 stores and loads per candidate).
#ifndef HDR_CANDIDATE_INLINE
#define HDR_CANDIDATE_INLINE
#endif
template <bool kFull, class RP>
__device__ HDR_CANDIDATE_INLINE Cand ris_candidate(const RisCtx<RP> &x, int j, MtStream &rng, unsigned &err) {
    const DeviceScene &s = *x.s;
    const Surface &sf = *x.sf;
    const SpectralCtx &sc = *x.sc;
    Cand c = cand_none();
    if (j < x.strat.n_nee) {
        // _generateNEECandidates (:553-589)
        if (!kFull) {
            skip_propose_candidate(s, rng);
            return c;
        }
        int li;
        LightSampleD ls;
        if (!propose_candidate(s, sf.hit.position, rng, li, ls)) return c;
        const RisContrib nee = ris_evaluate_light_sample(s, *x.rp, j, sf, li, ls, x.strat.skip_vis, sc, err);
        const Spec contribution = nee.emission * nee.tmul;
        const float target = spectrum_luminance(contribution, sc.cie);
        const float mis = nee.use_mis ? power_heuristic3(nee.p_nee, x.strat.n_nee, 0.0f, x.strat.n_sky, nee.p_bsdf,
                                                         x.strat.n_bsdf)
                                      : 1.0f;
        c.valid = true;
        c.has_lc = true;
        c.light = li;
        c.ls = ls;
        c.origin = 0;
        c.tp = contribution;
        c.ris_weight = (double)(mis * target) / ((double)nee.p_nee + 1e-9);
        c.target = target;
        c.vis_tested = nee.vis_tested;
        return c;
    }
    j -= x.strat.n_nee;
    if (j < x.strat.n_sky) {
        // sky NEE (:445-475): the environment outside the light sampler is the physical
        // sky, whose SampleLight is the sun and draws nothing; every sky candidate is
        // the same sample, so they share one shadow slot (index n_nee of the pixel's)
        if (!kFull) return c;
        LightSampleD ls;
        if (!sky_sun_sample(s, ls)) return c;
        const int li = sky_light_index(s);
        const RisContrib nee =
            ris_evaluate_light_sample(s, *x.rp, x.strat.n_nee, sf, li, ls, x.strat.skip_vis, sc, err);
        const Spec contribution = nee.emission * nee.tmul;
        const float target = spectrum_luminance(contribution, sc.cie);
        const float mis = nee.use_mis ? power_heuristic3(nee.p_nee, x.strat.n_sky, 0.0f, x.strat.n_nee, nee.p_bsdf,
                                                         x.strat.n_bsdf)
                                      : 1.0f;
        c.valid = true;
        c.has_lc = true;
        c.light = li;
        c.ls = ls;
        c.origin = 1;
        c.tp = contribution;
        c.ris_weight = (double)(mis * target) / ((double)nee.p_nee + 1e-9);
        c.target = target;
        c.vis_tested = nee.vis_tested;
        return c;
    }
    j -= x.strat.n_sky;
    // _generateBSDFSamplingCandidates (:396-551)
    if (x.conn_cand && j == 0) {
        if (!kFull) return c;
        const RisContrib bc = ris_evaluate_bsdf_connection(s, sf, *x.conn, x.strat, sc);
        const Spec contribution = bc.emission * bc.tmul;
        const double target = (double)spectrum_luminance(contribution, sc.cie);
        float p_sampler = bc.p_nee, p_sky = 0.0f;
        if (!x.conn->has_hit && (!env_present(s) || env_select_pdf(s) <= 0.0f)) {
            p_sampler = 0.0f;
            p_sky = bc.p_nee;
        }
        const double mis =
            (double)power_heuristic3(bc.p_bsdf, x.strat.n_bsdf, p_sampler, x.strat.n_nee, p_sky, x.strat.n_sky);
        c.valid = true;
        c.has_lc = false;
        c.origin = 0;
        c.tp = contribution;
        c.ris_weight = mis * target / ((double)bc.p_bsdf + 1e-9);
        c.target = (float)target;
        c.vis_tested = true;
        return c;
    }
    BounceState st{0, 0};
    if (!kFull) {
        (void)sample_bounce(sf.c, sf.sn, sf.inside, sf.hit.position, sf.ray_d, 1, 1, st, sc, rng);
        return c;
    }
    const int fresh = j - (x.conn_cand ? 1 : 0);  // index among the generated BSDF candidates
    const Connection cn = sample_bounce_with_connection(*x.rp, 1 + fresh, sf, 1, 1, st, sc, rng, err);
    if (!cn.b.ok) return c;
    if (!cn.has_hit) {
        if (!env_present(s)) return c;
        const Spec env_tp = cn.b.integrand;
        const V3 wi = cn.b.dir;
        const V3 env_rgb = env_radiance(s, wi);
        const Spec env_em = rgb_to_spectrum(env_rgb, sc.up);
        const float p_bsdf = cn.b.pdf;
        const float sel = env_select_pdf(s);
        const float epdf = env_pdf(s, wi);
        const float p_sampler = sel * epdf;
        const float p_sky = (sel <= 0.0f && x.strat.n_sky > 0) ? epdf : 0.0f;
        const float p_nee = p_sampler + p_sky;
        const double target = (double)spectrum_luminance(env_em * env_tp, sc.cie);
        const double mis =
            (double)power_heuristic3(p_bsdf, x.strat.n_bsdf, p_sampler, x.strat.n_nee, p_sky, x.strat.n_sky);
        c.valid = true;
        c.has_lc = p_nee > 0.0f;
        c.light = env_light_index(s);
        c.ls = LightSampleD{wi, env_rgb, -wi, 1e30f, p_nee, true};
        c.origin = 2;
        c.tp = env_em * env_tp;
        c.ris_weight = mis * target / ((double)p_bsdf + 1e-9);
        c.target = (float)target;
        c.vis_tested = true;
        return c;
    }
    if (cn.hit.light < 0) return c;  // GetLightAtHit == nullptr
    const RisContrib bc = ris_evaluate_bsdf_connection(s, sf, cn, x.strat, sc);
    const Spec contribution = bc.emission * bc.tmul;
    const double target = (double)spectrum_luminance(contribution, sc.cie);
    const double mis =
        (double)power_heuristic3(bc.p_bsdf, x.strat.n_bsdf, bc.p_nee, x.strat.n_nee, 0.0f, x.strat.n_sky);
    const V3 wi = cn.b.dir;
    float av;
    bool solid;
    light_eval_pdf(s, cn.hit.light, wi, av, solid);
    av *= light_select_pdf(s);
    c.valid = true;
    c.has_lc = true;
    c.light = cn.hit.light;
    c.ls = LightSampleD{wi, get_closure(s, cn.hit).emission, cn.hit.normal, cn.hit.depth, av, solid};
    c.origin = 2;
    c.tp = contribution;
    c.ris_weight = mis * target / ((double)bc.p_bsdf + 1e-9);
    c.target = (float)target;
    c.vis_tested = true;
    return c;
}

struct Reservoir {  // WeightedReservoir<RISLightCandidate>
    Cand chosen;    // chosen.valid == ChosenSample engaged
    float wsum;
    int m;
    float w;
};

__device__ __forceinline__ void reservoir_update(Reservoir &r, const Cand &c, float weight, MtStream &rng) {
    ++r.m;
    if (weight <= 0.0f) return;
    r.wsum += weight;
    if (rng.next_float() <= weight / r.wsum) r.chosen = c;
}

__device__ __forceinline__ void reservoir_finalize(Reservoir &r, int cpf) {
    if (!r.chosen.valid || r.m <= 0) {
        r.w = 0.0f;
        return;
    }
    const float phat = r.chosen.target;
    if (phat <= 0.0f) {
        r.w = 0.0f;
        return;
    }
    const int frames = smaxi(1, r.m / smaxi(1, cpf));
    r.w = r.wsum / ((float)frames * phat);
    if (!isfinite(r.w)) r.w = 0.0f;
}

__device__ __forceinline__ void reservoir_load(const ReservoirView &v, size_t i, Reservoir &r) {
    const float4 a = v.dir_dist[i], b = v.color_pdf[i], c = v.normal_phat[i], d = v.throughput[i];
    const float4 e = v.wsum_w_m_meta[i];
    const unsigned meta = (unsigned)fbits(e.w);
    r.wsum = e.x;
    r.w = e.y;
    r.m = fbits(e.z);
    Cand &k = r.chosen;
    k.valid = (meta & kResHasSample) != 0;
    k.has_lc = (meta & kResHasCandidate) != 0;
    k.vis_tested = (meta & kResVisTested) != 0;
    k.origin = (int)((meta >> kResOriginShift) & 3u);
    k.light = (int)(meta >> kResLightShift) - 1;
    k.ls = LightSampleD{V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, V3{c.x, c.y, c.z}, a.w, b.w,
                        (meta & kResPdfSolidAngle) != 0};
    k.tp = Spec{{d.x, d.y, d.z, d.w}};
    k.target = c.w;
    k.ris_weight = 0.0;
}

__device__ __forceinline__ void reservoir_store(const ReservoirView &v, size_t i, const Reservoir &r) {
    const Cand &k = r.chosen;
    unsigned meta = 0;
    if (k.valid) meta |= kResHasSample;
    if (k.has_lc) meta |= kResHasCandidate;
    if (k.vis_tested) meta |= kResVisTested;
    if (k.ls.pdf_solid_angle) meta |= kResPdfSolidAngle;
    meta |= ((unsigned)k.origin & 3u) << kResOriginShift;
    meta |= ((unsigned)(k.light + 1) & 0xFFFFFFu) << kResLightShift;
    v.dir_dist[i] = make_float4(k.ls.dir.x, k.ls.dir.y, k.ls.dir.z, k.ls.dist);
    v.color_pdf[i] = make_float4(k.ls.color.x, k.ls.color.y, k.ls.color.z, k.ls.pdf);
    v.normal_phat[i] = make_float4(k.ls.normal.x, k.ls.normal.y, k.ls.normal.z, k.target);
    v.throughput[i] = make_float4(k.tp.v[0], k.tp.v[1], k.tp.v[2], k.tp.v[3]);
    v.wsum_w_m_meta[i] = make_float4(r.wsum, r.w, __int_as_float(r.m), __int_as_float((int)meta));
}

struct RisRun {
    int candidate_count;
    bool use_reservoir;
    bool skip_vis;
    int m_cap;       // extension: 0 = unbounded (reference)
    ReprojD reproj;  // extension: mode 0 = the reference's same-pixel history
};

// The previous frame's reservoir for a hit point at p (ReprojD mode 1): the
// pixel p projected to with the previous camera, if that pixel saw the same
// surface point (within 2 % of its depth). Its light sample is moved to p
// (same point on the light, direction and distance from p) and marked
// untested, so a winner taken from it gets a shadow ray from here.
__device__ __forceinline__ bool reprojected_history(const ReprojD &rj, V3 p, Reservoir &out) {
    if (rj.mode != 1) return false;
    const D3 c = m4d_transform(rj.view, f3_to_d(p));
    const D3 ndc = m4d_transform(rj.proj, c);
    if (!(fabs(ndc.x) <= 1.0) || !(fabs(ndc.y) <= 1.0)) return false;
    const int ix = (int)floor((ndc.x + 1.0) * 0.5 * (double)rj.width);
    const int iy = (int)floor((ndc.y + 1.0) * 0.5 * (double)rj.height);
    if (ix < 0 || iy < 0 || ix >= rj.width || iy >= rj.height) return false;
    const size_t q = (size_t)iy * (size_t)rj.width + (size_t)ix;
    const float4 pp = rj.prev_pos[q];
    const V3 prev_p{pp.x, pp.y, pp.z};
    if (!(pp.w < 3.0e38f) || !(length(prev_p - p) <= 0.02f * pp.w)) return false;
    reservoir_load(rj.prev, q, out);
    LightSampleD &ls = out.chosen.ls;
    if (out.chosen.valid && out.chosen.has_lc && !ls.pdf_solid_angle) {
        const V3 v = (prev_p + ls.dir * ls.dist) - p;
        const float dist = length(v);
        if (!(dist > 0.0f)) return false;
        ls.dir = v * (1.0f / dist);
        ls.dist = dist;
    }
    out.chosen.vis_tested = false;
    return true;
}

// RisDirectLightIntegrator::Li, per-bounce form (:230-361). primary == (callId.id < callId.stride).
// gen_end: the stream state right after candidate generation when the caller
// already knows it (the wavefront generate kernel saved it); NULL replays the
// sampling decisions to find it.
template <class RP>
__device__ HDR_BOUNCE_INLINE Spec ris_direct_li(const DeviceScene &s, const RP &rp, const Surface &sf, bool has_conn,
                                     const Connection &cn, const SpectralCtx &sc, MtStream &rng, bool primary,
                                     const RisRun &run, const ReservoirView &rv, size_t pixel,
                                     const MtStream *gen_end_state, unsigned &err) {
    // technique split (:89-99): a dome environment is a scene light, covered by the
    // sampler; the physical sky is not and gets the sky technique
    RisCtx<RP> x;
    x.s = &s;
    x.rp = &rp;
    x.sf = &sf;
    x.sc = &sc;
    ris_technique_split(s, run.candidate_count, x.strat.n_nee, x.strat.n_sky, x.strat.n_bsdf);
    x.strat.skip_vis = run.skip_vis;
    x.has_conn = has_conn;
    x.conn = &cn;
    x.conn_cand = has_conn && cn.b.pdf > 0.0f;
    const int n_fresh = x.strat.n_bsdf - (x.conn_cand ? 1 : 0);
    x.n_total = x.strat.n_nee + x.strat.n_sky + (x.conn_cand ? 1 : 0) + smaxi(0, n_fresh);
    // When the generated BSDF candidates (the last ones) are all invalid and the
    // stream state after generation is known, they are counted as misses and the
    // stream jumps to that state instead of replaying their samples.
    const bool skip_fresh = gen_end_state != nullptr && rp.fresh_bsdf_empty();
    const int n_eval = skip_fresh ? x.n_total - smaxi(0, n_fresh) : x.n_total;

    if (run.use_reservoir && primary) {
        // ---- reservoir branch (:267-331)
        MtStream upd = rng;
        if (gen_end_state) {
            upd = *gen_end_state;
            upd.spill = rng.spill;
        } else {  // replay the sampling draws to find the first update draw
            for (int j = 0; j < x.n_total; ++j) (void)ris_candidate<false>(x, j, upd, err);
        }
        const uint32_t gen_end = upd.k;
        Reservoir r;
        r.chosen = cand_none();
        r.wsum = 0.0f;
        r.m = 0;
        r.w = 0.0f;
        for (int j = 0; j < n_eval; ++j) {
            const Cand c = ris_candidate<true>(x, j, rng, err);
            if (c.valid)
                reservoir_update(r, c, (float)c.ris_weight, upd);
            else
                ++r.m;  // CountMiss
        }
        if (skip_fresh) {
            r.m += x.n_total - n_eval;  // CountMiss of each generated BSDF candidate
        } else if (rng.k != gen_end) {
            err |= kErrRngDesync;
        }
        rng = upd;
        // temporal reuse (:284-305)
        Reservoir prev;
        bool have_prev = true;
        if (run.reproj.mode == 0)
            reservoir_load(rv, pixel, prev);
        else
            have_prev = reprojected_history(run.reproj, sf.hit.position, prev);
        if (have_prev && prev.chosen.valid && prev.chosen.has_lc) {
            const Spec reeval = ris_reevaluate(s, sf, prev.chosen.light, prev.chosen.ls, sc);
            const float phat_curr = spectrum_luminance(reeval, sc.cie);
            const float phat_gen = prev.chosen.target;
            if (phat_gen > 0.0f) {
                prev.chosen.target = phat_curr;
                prev.chosen.tp = reeval;
                if (run.m_cap > 0) {  // extension: bound the history (M-cap)
                    const int cap = run.m_cap * x.n_total;
                    if (prev.m > cap) {
                        prev.wsum *= (float)cap / (float)prev.m;
                        prev.m = cap;
                    }
                }
                const float mw = prev.wsum * (phat_curr / phat_gen);
                // Merge (:157-166)
                r.m += prev.m;
                if (mw > 0.0f) {
                    r.wsum += mw;
                    if (rng.next_float() <= mw / r.wsum) r.chosen = prev.chosen;
                }
            }
        }
        reservoir_finalize(r, x.n_total);
        // winner visibility (:309-321)
        if (r.chosen.valid && !r.chosen.vis_tested && r.chosen.has_lc) {
            const RisContrib nee =
                ris_evaluate_light_sample(s, rp, -1, sf, r.chosen.light, r.chosen.ls, false, sc, err);
            r.chosen.tp = nee.emission * nee.tmul;
            r.chosen.vis_tested = true;
        }
        reservoir_store(rv, pixel, r);
        if (!r.chosen.valid || r.w <= 0.0f) return spec(0.0f);
        return r.chosen.tp * r.w;
    }

    // ---- standard RIS (:333-361): RandomIndexFromWeights over stored weights
    if (x.n_total > kMaxPlainRisCandidates) {
        err |= kErrRisCapacity;
        return spec(0.0f);
    }
    const MtStream start = rng;
    double weights[kMaxPlainRisCandidates];
    double wsum = 0.0;
    for (int j = 0; j < n_eval; ++j) {
        const Cand c = ris_candidate<true>(x, j, rng, err);
        const double w = c.valid ? c.ris_weight : 0.0;
        weights[j] = w;
        if (w > 0.0) wsum += w;
    }
    if (skip_fresh) {  // the generated BSDF candidates weigh nothing; the stream continues after them
        for (int j = n_eval; j < x.n_total; ++j) weights[j] = 0.0;
        uint64_t *const spill = rng.spill;
        rng = *gen_end_state;
        rng.spill = spill;
    }
    if (wsum <= 0.0) return spec(0.0f);
    double remaining = (double)rng.next_float() * wsum;
    int chosen = -1;
    for (int j = 0; j < x.n_total; ++j) {
        const double w = weights[j];
        if (w <= 0.0) continue;
        remaining -= w;
        if (remaining <= 0.0) {
            chosen = j;
            break;
        }
    }
    if (chosen < 0) return spec(0.0f);
    // rebuild the winner from its own draws (a second pass over the same stream)
    MtStream replay = start;
    for (int j = 0; j < chosen; ++j) (void)ris_candidate<false>(x, j, replay, err);
    const Cand c = ris_candidate<true>(x, chosen, replay, err);
    if (!c.valid) return spec(0.0f);
    const float W = (float)(wsum / (double)c.target);
    Spec tp = c.tp;
    if (!c.vis_tested && c.has_lc) {
        const RisContrib nee = ris_evaluate_light_sample(s, rp, -1, sf, c.light, c.ls, false, sc, err);
        tp = nee.emission * nee.tmul;
    }
    return tp * W;
}

// ============================================================================
// PathIntegrator (integrators/path_integrator.cpp:48-209)
// ============================================================================
template <bool kRis, class RP>
__device__ __forceinline__ Spec direct_li(const DeviceScene &s, const RP &rp, const Surface &sf, bool has_conn,
                                          const Connection &cn, const SpectralCtx &sc, MtStream &rng, bool primary,
                                          const RisRun &ris, const ReservoirView &rv, size_t pixel,
                                          const MtStream *gen_end_state, unsigned &err) {
    if (kRis) return ris_direct_li(s, rp, sf, has_conn, cn, sc, rng, primary, ris, rv, pixel, gen_end_state, err);
    return mis_direct_li(s, sf, has_conn, cn, sc, rng, err);
}

// The bounce loop of _li (:114-207) from vertex `first_bounce` on: `next` is
// that vertex's hit (of the ray ro, rd), tp and total the path so far. Later
// vertices query the scene on the spot.
template <bool kRis>
__device__ Spec path_li_continue(const DeviceScene &s, Spec total, Spec tp, V3 ro, V3 rd, bool has_next, Hit next,
                                 BounceState st, const SpectralCtx &sc, MtStream &rng, const PathRun &pr,
                                 const RisRun &ris, const ReservoirView &rv, size_t pixel, int first_bounce,
                                 unsigned &err) {
    const TraceNow now{&s};
    for (int bounce = first_bounce; bounce < pr.max_depth; ++bounce) {
        if (!has_next) break;
        const Hit bh = next;
        Closure c = get_closure(s, bh);
        if (!pr.enable_subsurface) c.subsurface = 0.0f;
        if (c.opacity < 0.999f && rng.next_float() > c.opacity) {
            ro = bh.position + rd * 1e-4f;
            has_next = intersect(s, ro, rd, next, err);
            --bounce;
            continue;
        }
        const bool inside = dot(c.normal, rd) > 0.0f;
        beer_absorption(tp, c, bh.depth, inside, sc);
        const Surface sf = make_surface(s, ro, rd, bh, c, inside);
        const Connection cn = sample_bounce_with_connection(now, 0, sf, pr.max_refl, pr.max_refr, st, sc, rng, err);
        total = total + tp * direct_li<kRis>(s, now, sf, cn.b.ok, cn, sc, rng, false, ris, rv, pixel, nullptr, err);
        if (!cn.b.ok) break;
        tp = tp * cn.b.tmul;
        ro = cn.b.origin;
        rd = cn.b.dir;
        has_next = cn.has_hit;
        next = cn.hit;
        if (cn.b.skip_roulette) continue;
        if (bounce > 3) {
            const float p = sclampf(spec_max(tp) * pr.roulette, 0.0f, 1.0f);
            if (rng.next_float() > p) break;
            tp = tp * (1.0f / p);
        }
    }
    return total;
}

// _li (:92-209). Later bounces query the scene directly (they only run in the
// one-thread-per-pixel form). kDirectOnly: the caller guarantees maxDepth 1
// (the wavefront form), so the later-bounce loop is not compiled.
template <bool kRis, class RP, bool kDirectOnly = false>
__device__ Spec path_li_shaded(const DeviceScene &s, const RP &rp, const Surface &sf0, const SpectralCtx &sc,
                               MtStream &rng, const PathRun &pr, const RisRun &ris, const ReservoirView &rv,
                               size_t pixel, const MtStream *gen_end_state, unsigned &err) {
    Spec total = rgb_to_spectrum(sf0.c.emission, sc.up);
    Spec tp = spec(1.0f);
    BounceState st{0, 0};
    const Connection first = sample_bounce_with_connection(rp, 0, sf0, pr.max_refl, pr.max_refr, st, sc, rng, err);
    total = total + direct_li<kRis>(s, rp, sf0, first.b.ok, first, sc, rng, true, ris, rv, pixel, gen_end_state, err);
    if (!first.b.ok) return total;
    if (kDirectOnly) return total;  // maxDepth 1: the loop below would not run
    tp = tp * first.b.tmul;
    return path_li_continue<kRis>(s, total, tp, first.b.origin, first.b.dir, first.has_hit, first.hit, st, sc, rng, pr,
                                  ris, rv, pixel, 1, err);
}

// PathIntegrator::Li (:48-90): opacity skip at the GBuffer hit, Beer, then _li.
// kDirectOnly also means an opaque scene (opacity >= 0.999 everywhere, checked
// at upload), where the skip never triggers and never draws.
template <bool kRis, class RP, bool kDirectOnly = false>
__device__ Spec path_li(const DeviceScene &s, const RP &rp, V3 ray_o, V3 ray_d, bool has_hit, Hit hit,
                        const SpectralCtx &sc, MtStream &rng, const PathRun &pr, const RisRun &ris,
                        const ReservoirView &rv, size_t pixel, const MtStream *gen_end_state, unsigned &err) {
    Spec tp = spec(1.0f);
    while (has_hit) {
        Closure c = get_closure(s, hit);
        if (!pr.enable_subsurface) c.subsurface = 0.0f;
        if (kDirectOnly || c.opacity >= 0.999f || rng.next_float() <= c.opacity) {
            const bool inside = dot(c.normal, ray_d) > 0.0f;
            beer_absorption(tp, c, hit.depth, inside, sc);
            const Surface sf = make_surface(s, ray_o, ray_d, hit, c, inside);
            return tp * path_li_shaded<kRis, RP, kDirectOnly>(s, rp, sf, sc, rng, pr, ris, rv, pixel, gen_end_state,
                                                              err);
        }
        has_hit = intersect(s, hit.position + ray_d * 1e-4f, ray_d, hit, err);
    }
    if (env_present(s) && pr.render_ibl_background) return rgb_to_spectrum(env_radiance(s, ray_d), sc.up);
    return spec(0.0f);
}

}  // namespace hdr
