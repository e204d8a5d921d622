// RaycastPass (passes/raycast_pass.cpp:57-162) and the scene-query / RNG
// kernels exposed for direct testing.
#include "device/frame.cuh"

namespace hdr {

__device__ __forceinline__ void write_gbuffer(const GBufferView &gb, size_t i, bool has, const Hit &h) {
    if (has) {
        gb.pos_depth[i] = make_float4(h.position.x, h.position.y, h.position.z, h.depth);
        gb.normal_prim[i] = make_float4(h.normal.x, h.normal.y, h.normal.z, __int_as_float(h.prim));
        gb.smooth_tri[i] = make_float4(h.smooth_normal.x, h.smooth_normal.y, h.smooth_normal.z, __int_as_float(h.tri));
        gb.albedo_uv[i] = make_float4(h.albedo.x, h.albedo.y, h.albedo.z, h.uv.x);
        gb.aux0[i] = make_float4(h.uv.y, h.dpdu.x, h.dpdu.y, h.dpdu.z);
        gb.aux1[i] = make_float4(h.dpdv.x, h.dpdv.y, h.dpdv.z, 0.0f);
    } else {
        gb.pos_depth[i] = make_float4(0.0f, 0.0f, 0.0f, 3.402823466e+38f);
        gb.normal_prim[i] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
        gb.smooth_tri[i] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
        gb.albedo_uv[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        gb.aux0[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        gb.aux1[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

__global__ void __launch_bounds__(256) raycast_kernel(DeviceScene s, CameraD cam, int frame_arg, GBufferView gb,
                                                      AovView aov, unsigned *err) {
    const int frame_index = live_frame(cam, frame_arg);
    int x, y;
    if (!tile_pixel(cam.width, cam.height, x, y)) return;
    const size_t i = (size_t)y * (size_t)cam.width + (size_t)x;
    const float px = (float)x + 0.5f, py = (float)y + 0.5f;
    MtStream rng;  // the raycast pass draws at most 2 numbers (thin lens): no spill state
    rng.init((uint32_t)i ^ (uint32_t)((unsigned long long)frame_index * 12345ULL), nullptr);
    const RayF ray = camera_ray(cam, px, py, rng);
    unsigned e = 0;
    HitId hid;
    const bool has = trace_ray<false>(s, ray.o, ray.d, 0.0f, hid, e);
    Hit h;
    if (has) h = make_hit(s, ray.o, ray.d, hid);
    write_gbuffer(gb, i, has, h);
    if (aov.depth) aov.depth[i] = has ? h.depth : 1.0f;
    if (aov.albedo) {
        aov.albedo[3 * i] = has ? h.albedo.x : 0.0f;
        aov.albedo[3 * i + 1] = has ? h.albedo.y : 0.0f;
        aov.albedo[3 * i + 2] = has ? h.albedo.z : 0.0f;
    }
    if (aov.normal) {
        aov.normal[3 * i] = has ? h.normal.x : 0.0f;
        aov.normal[3 * i + 1] = has ? h.normal.y : 0.0f;
        aov.normal[3 * i + 2] = has ? h.normal.z : 0.0f;
    }
    if (e) atomicOr(err, e);
}

// hdr_gbuffer_texel = 6 float4 (see include/hdrestir.h)
__global__ void trace_rays_kernel(DeviceScene s, const float *rays, const float *tmax, int n, int any_hit,
                                  float4 *out, unsigned *err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const V3 o{rays[6 * k], rays[6 * k + 1], rays[6 * k + 2]};
    const V3 d{rays[6 * k + 3], rays[6 * k + 4], rays[6 * k + 5]};
    unsigned e = 0;
    HitId hid;
    float4 *t = out + 6 * (size_t)k;
    if (any_hit) {
        const float lim = tmax ? tmax[k] : 3.402823466e+38f;
        const bool occ = shadow_ray(s, o, d, lim, e);
        t[0] = make_float4(0.0f, 0.0f, 0.0f, 3.402823466e+38f);
        t[1] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
        t[2] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
        t[3] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(occ ? 1 : 0));
        t[4] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        t[5] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else {
        const bool has = trace_ray<false>(s, o, d, 0.0f, hid, e);
        if (has) {
            const Hit h = make_hit(s, o, d, hid);
            t[0] = make_float4(h.position.x, h.position.y, h.position.z, h.depth);
            t[1] = make_float4(h.normal.x, h.normal.y, h.normal.z, __int_as_float(h.prim));
            t[2] = make_float4(h.smooth_normal.x, h.smooth_normal.y, h.smooth_normal.z, __int_as_float(h.tri));
            t[3] = make_float4(h.albedo.x, h.albedo.y, h.albedo.z, __int_as_float(1));
            t[4] = make_float4(h.uv.x, h.uv.y, h.dpdu.x, h.dpdu.y);
            t[5] = make_float4(h.dpdu.z, h.dpdv.x, h.dpdv.y, h.dpdv.z);
        } else {
            t[0] = make_float4(0.0f, 0.0f, 0.0f, 3.402823466e+38f);
            t[1] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
            t[2] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
            t[3] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(0));
            t[4] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            t[5] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
    if (e) atomicOr(err, e);
}

__global__ void rng_floats_kernel(const uint32_t *seeds, int n, int count, float *out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint64_t spill[312];
    MtStream rng;
    rng.init(seeds[k], spill);
    for (int j = 0; j < count; ++j) out[(size_t)k * count + j] = rng.next_float();
}

void launch_raycast(const DeviceScene &s, const CameraD &cam, int frame_index, GBufferView gb, AovView aov,
                    unsigned *err, cudaStream_t st) {
    raycast_kernel<<<tile_blocks(cam.width, cam.height), 256, 0, st>>>(s, cam, frame_index, gb, aov, err);
}

// Per-ray traversal work of one walk (hdr_trace_stats): nodes popped, leaves
// entered, triangles tested, and the answer.
__global__ void trace_stats_kernel(DeviceScene s, const float *rays, const float *tmax, int n, int mode, int4 *out,
                                   unsigned *err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const V3 o{rays[6 * k], rays[6 * k + 1], rays[6 * k + 2]};
    const V3 d{rays[6 * k + 3], rays[6 * k + 4], rays[6 * k + 5]};
    const float lim = tmax ? tmax[k] : 3.402823466e+38f;
    unsigned e = 0;
    CountStats st;
    HitId h;
    bool r = false;
    switch (mode) {
        case 0: r = trace_ray_binary<false>(s, o, d, 0.0f, h, e, st); break;
        case 1: r = trace_ray_wide<false>(s, o, d, 0.0f, h, e, st); break;
        case 2: r = trace_ray_binary<true>(s, o, d, lim, h, e, st) && h.t < lim; break;
        case 3: r = trace_ray_wide<true>(s, o, d, lim, h, e, st) && h.t < lim; break;
        case 4: r = shadow4_ray(s, o, d, lim, e, st); break;
        default: r = closest4_ray(s, o, d, h, e, st); break;
    }
    out[k] = make_int4(st.pops, st.leaves, st.tris, r ? 1 : 0);
    if (e) atomicOr(err, e);
}

void launch_trace_stats(const DeviceScene &s, const float *rays, const float *tmax, int n, int mode, int4 *out,
                        unsigned *err, cudaStream_t st) {
    trace_stats_kernel<<<(n + 127) / 128, 128, 0, st>>>(s, rays, tmax, n, mode, out, err);
}

void launch_trace_rays(const DeviceScene &s, const float *rays, const float *tmax, int n, int any_hit, float4 *out,
                       unsigned *err, cudaStream_t st) {
    trace_rays_kernel<<<(n + 127) / 128, 128, 0, st>>>(s, rays, tmax, n, any_hit, out, err);
}

void launch_rng_floats(const uint32_t *seeds, int n, int count, float *out, cudaStream_t st) {
    rng_floats_kernel<<<(n + 127) / 128, 128, 0, st>>>(seeds, n, count, out);
}

}  // namespace hdr
