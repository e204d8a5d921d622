// Per-pixel prologue of the wavefront RIS kernels: the pixel's stream, jittered
// camera ray, wavelengths and GBuffer hit (integration_pass.cpp:210-233).
#pragma once

#include "camera.cuh"
#include "integrator.cuh"

namespace hdr {

struct PixelStart {
    size_t i;
    RayF ray;
    SpectralCtx sc;
    Hit hit;
    bool has_hit;
};

template <int kThreads = 256>
__device__ __forceinline__ bool pixel_start(const DeviceScene &s, const CameraD &cam, int frame_index,
                                            const GBufferView &gb, MtStream &rng, uint64_t *spill, PixelStart &ps) {
    int x, y;
    if (!tile_pixel<kThreads>(cam.width, cam.height, x, y)) return false;
    ps.i = (size_t)y * (size_t)cam.width + (size_t)x;
    rng.init((uint32_t)ps.i ^ (uint32_t)((unsigned long long)frame_index * 12345ULL), spill);
    const float px = (float)x + rng.next_float();
    const float py = (float)y + rng.next_float();
    ps.ray = camera_ray(cam, px, py, rng);
    ps.sc = make_spectral_ctx(rng.next_float());
    ps.has_hit = load_gbuffer_hit(s, gb, ps.i, ps.hit);
    return true;
}

}  // namespace hdr
