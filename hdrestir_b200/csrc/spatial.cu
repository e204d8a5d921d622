// Spatial reuse of ReSTIR reservoirs: an extension with no reference
// counterpart (the reference reuses only the same pixel's reservoir of the
// previous frame, ris_direct_light_integrator.cpp:267-331). It runs after the
// wavefront resampling pass when hdr_ris_params.spatial_neighbors > 0; with 0
// nothing here runs and the images are the reference's.
//
// Per pixel, after the temporal merge, up to `neighbours` pixels within
// `radius` are picked at random. A neighbour whose GBuffer surface is similar
// (normals within ~25 degrees, depth within 10 %) offers its reservoir: its
// light sample is moved to this pixel (the point on the light is kept, the
// direction and distance are recomputed from this pixel's hit point), its
// target function is evaluated here, and it is merged with the weight the
// reference's temporal merge uses, WSum * p̂_here / p̂_there, adding its
// CandidateCount (capped by m_cap like the temporal history). A sample taken
// from a neighbour gets a shadow ray from this pixel; if occluded it lights
// nothing this frame. W and the colour are then recomputed as the resampling
// pass computes them: Color = Beer * (emission + Throughput * W).
//
// The merged reservoirs are written to a second buffer (neighbours read the
// first), which the host copies back, so the next frame's temporal reuse
// starts from them. Random numbers come from a hash of pixel, frame and step
// (PCG hash, Jarzynski and Olano, "Hash Functions for GPU Rendering", JCGT
// 2020), not from the pixel's MT stream, whose draws the reference defines.
#include "device/integrator.cuh"
#include "device/pixel.cuh"

namespace hdr {
namespace {

__device__ __forceinline__ uint32_t pcg_hash(uint32_t v) {
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

struct HashStream {
    uint32_t s;
    __device__ __forceinline__ float next() {
        s = pcg_hash(s);
        return (float)(s >> 8) * (1.0f / 16777216.0f);  // [0, 1)
    }
};

__device__ __forceinline__ bool similar_surface(const Hit &a, const Hit &b) {
    return dot(a.normal, b.normal) >= 0.9f && fabsf(a.depth - b.depth) <= 0.1f * a.depth;
}

__device__ __forceinline__ void copy_record(const ReservoirView &in, const ReservoirView &out, size_t i) {
    out.dir_dist[i] = in.dir_dist[i];
    out.color_pdf[i] = in.color_pdf[i];
    out.normal_phat[i] = in.normal_phat[i];
    out.throughput[i] = in.throughput[i];
    out.wsum_w_m_meta[i] = in.wsum_w_m_meta[i];
}

template <int kThreads>
__global__ void __launch_bounds__(kThreads) ris_spatial_kernel(DeviceScene s, CameraD cam, int frame_arg,
                                                               PathRun pr, int cpf, int m_cap, int neighbours,
                                                               float radius, GBufferView gb, ReservoirView in,
                                                               ReservoirView out, float4 *color, float4 *q_winner,
                                                               int *winner_count, unsigned *err) {
    const int frame_index = live_frame(cam, frame_arg);
    MtStream rng;
    PixelStart ps;
    if (!pixel_start<kThreads>(s, cam, frame_index, gb, rng, nullptr, ps)) return;
    const size_t i = ps.i;
    if (!ps.has_hit) {  // background pixel: the resampling pass left no reservoir to merge
        copy_record(in, out, i);
        return;
    }
    Closure c = get_closure(s, ps.hit);
    if (!pr.enable_subsurface) c.subsurface = 0.0f;
    const bool inside = dot(c.normal, ps.ray.d) > 0.0f;
    Spec beer = spec(1.0f);
    beer_absorption(beer, c, ps.hit.depth, inside, ps.sc);
    const Surface sf = make_surface(s, ps.ray.o, ps.ray.d, ps.hit, c, inside);

    Reservoir r;
    reservoir_load(in, i, r);
    const int x = (int)(i % (size_t)cam.width), y = (int)(i / (size_t)cam.width);
    HashStream h{pcg_hash((uint32_t)i ^ pcg_hash((uint32_t)frame_index + 0x9e3779b9u))};
    bool shifted = false;
    unsigned e = 0;
    for (int k = 0; k < neighbours; ++k) {
        const float rr = radius * sqrtf(h.next());
        const float th = 6.2831853f * h.next();
        const int qx = x + __float2int_rn(rr * cosf(th)), qy = y + __float2int_rn(rr * sinf(th));
        if (qx < 0 || qy < 0 || qx >= cam.width || qy >= cam.height || (qx == x && qy == y)) continue;
        const size_t q = (size_t)qy * (size_t)cam.width + (size_t)qx;
        Hit hq;
        if (!load_gbuffer_hit(s, gb, q, hq) || !similar_surface(ps.hit, hq)) continue;
        Reservoir n;
        reservoir_load(in, q, n);
        if (m_cap > 0 && n.m > m_cap * cpf) {  // bound the neighbour's history like the temporal one
            n.wsum *= (float)(m_cap * cpf) / (float)n.m;
            n.m = m_cap * cpf;
        }
        r.m += n.m;
        if (!n.chosen.valid || !n.chosen.has_lc || !(n.chosen.target > 0.0f)) continue;
        LightSampleD ls = n.chosen.ls;
        if (!ls.pdf_solid_angle) {  // a point on the light: the direction from here
            const V3 v = (hq.position + ls.dir * ls.dist) - ps.hit.position;
            const float dist = length(v);
            if (!(dist > 0.0f)) continue;
            ls.dir = v * (1.0f / dist);
            ls.dist = dist;
        }
        const Spec f = ris_reevaluate(s, sf, n.chosen.light, ls, ps.sc);
        const float phat = spectrum_luminance(f, ps.sc.cie);
        const float mw = n.wsum * (phat / n.chosen.target);
        if (!(mw > 0.0f) || !isfinite(mw)) continue;
        r.wsum += mw;
        if (h.next() <= mw / r.wsum) {
            r.chosen = n.chosen;
            r.chosen.ls = ls;
            r.chosen.target = phat;
            r.chosen.tp = f;
            r.chosen.vis_tested = false;
            shifted = true;
        }
    }
    reservoir_finalize(r, cpf);
    if (shifted && r.chosen.valid && r.w > 0.0f) {  // the moved sample's visibility from this pixel
        const V3 so = sf.hit.position + sf.sn * 1e-4f;
        if (q_winner) {  // queued; an occluded pixel is fixed up after the shadow kernel
            const int k = atomicAdd(winner_count, 1);
            q_winner[2 * (size_t)k] = make_float4(so.x, so.y, so.z, __int_as_float((int)i));
            q_winner[2 * (size_t)k + 1] =
                make_float4(r.chosen.ls.dir.x, r.chosen.ls.dir.y, r.chosen.ls.dir.z, r.chosen.ls.dist - 1e-3f);
        } else {
            const unsigned oc = occluded_call(s.dev, so, r.chosen.ls.dir, r.chosen.ls.dist - 1e-3f);
            e |= oc >> 1;
            if (oc & 1u) r.chosen.tp = spec(0.0f);
        }
        r.chosen.vis_tested = true;
    }
    reservoir_store(out, i, r);
    const Spec direct = (r.chosen.valid && r.w > 0.0f) ? r.chosen.tp * r.w : spec(0.0f);
    const Spec L = beer * (rgb_to_spectrum(c.emission, ps.sc.up) + direct);
    V3 rgb = spectrum_to_rgb(L, ps.sc.cie);
    if (cam.p.has_params && cam.p.enable_exposure) rgb = rgb * cam.p.exposure_mult;
    color[i] = make_float4(rgb.x, rgb.y, rgb.z, 1.0f);
    if (e) atomicOr(err, e);
}

}  // namespace

int launch_ris_spatial(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                       GBufferView gb, ReservoirView in, ReservoirView out, float4 *color, float4 *q_winner,
                       int *winner_count, unsigned *err, cudaStream_t st) {
    PathRun pr{};
    pr.max_depth = p.max_depth;
    pr.enable_subsurface = p.enable_subsurface != 0;
    // allCandidates.size(): NEE + generated BSDF (+ the connection, which replaces one of them)
    const int n_nee = p.candidate_count / 2 > 1 ? p.candidate_count / 2 : 1;
    const int cpf = n_nee + (p.candidate_count - n_nee > 0 ? p.candidate_count - n_nee : 0);
    const float radius = p.spatial_radius > 0.0f ? p.spatial_radius : 30.0f;
    ris_spatial_kernel<256><<<tile_blocks(cam.width, cam.height), 256, 0, st>>>(
        s, cam, frame_index, pr, cpf, p.m_cap, p.spatial_neighbors, radius, gb, in, out, color, q_winner,
        winner_count, err);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

}  // namespace hdr
