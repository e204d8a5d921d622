// IntegrationPass::_execute (passes/integration_pass.cpp:157-252) for the two
// integration passes: PathTracePass (MIS direct light) and RISPathTracePass
// (RIS / ReSTIR direct light). One thread per pixel:
//   seed = uint32(i) ^ uint32(frameIndex * 12345)      (:210-211)
//   jittered camera ray (2 draws [+2 thin lens])       (:212-224)
//   wavelengths (1 draw)                               (:226)
//   PathIntegrator::Li on the GBuffer hit              (:231-233)
//   Color = SpectrumToRGB [x exposure], alpha 1        (:238-243)
#include "device/integrator.cuh"

namespace hdr {

template <bool kRis>
__global__ void __launch_bounds__(256) integrate_kernel(DeviceScene s, CameraD cam, int frame_index, PathRun pr,
                                                        RisRun ris, GBufferView gb, ReservoirView rv, float4 *color,
                                                        unsigned *err) {
    int x, y;
    if (!tile_pixel(cam.width, cam.height, x, y)) return;
    const size_t i = (size_t)y * (size_t)cam.width + (size_t)x;
    uint64_t spill[312];
    MtStream rng;
    rng.init((uint32_t)i ^ (uint32_t)((unsigned long long)frame_index * 12345ULL), spill);
    const float px = (float)x + rng.next_float();
    const float py = (float)y + rng.next_float();
    const RayF ray = camera_ray(cam, px, py, rng);
    const SpectralCtx sc = make_spectral_ctx(rng.next_float());
    unsigned e = 0;
    Hit h;
    const bool has = load_gbuffer_hit(s, gb, i, h);
    const TraceNow now{&s};
    const Spec L = path_li<kRis>(s, now, ray.o, ray.d, has, h, sc, rng, pr, ris, rv, i, nullptr, e);
    V3 rgb = spectrum_to_rgb(L, sc.cie);
    if (cam.p.has_params && cam.p.enable_exposure) rgb = rgb * cam.p.exposure_mult;
    color[i] = make_float4(rgb.x, rgb.y, rgb.z, 1.0f);
    if (e) atomicOr(err, e);
}

static PathRun make_path_run(int max_depth, int subsurface, int max_refl, int max_refr, int ibl, float roulette) {
    PathRun pr;
    pr.max_depth = max_depth;
    pr.enable_subsurface = subsurface != 0;
    pr.max_refl = max_refl;
    pr.max_refr = max_refr;
    pr.render_ibl_background = ibl != 0;
    pr.roulette = roulette;
    return pr;
}

void launch_ris_path_trace(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                           GBufferView gb, ReservoirView res, float4 *color, unsigned *err, cudaStream_t st) {
    const PathRun pr = make_path_run(p.max_depth, p.enable_subsurface, p.max_refl, p.max_refr,
                                     p.render_ibl_background, p.roulette);
    RisRun ris;
    ris.candidate_count = p.candidate_count;
    ris.use_reservoir = p.use_reservoir != 0;
    ris.skip_vis = p.skip_visibility != 0;
    ris.m_cap = p.m_cap;
    integrate_kernel<true><<<tile_blocks(cam.width, cam.height), 256, 0, st>>>(s, cam, frame_index, pr, ris, gb, res,
                                                                             color, err);
}

void launch_path_trace(const DeviceScene &s, const CameraD &cam, int frame_index, const PathParamsD &p,
                       GBufferView gb, float4 *color, unsigned *err, cudaStream_t st) {
    const PathRun pr = make_path_run(p.max_depth, p.enable_subsurface, p.max_refl, p.max_refr,
                                     p.render_ibl_background, p.roulette);
    RisRun ris{};
    ReservoirView rv{};
    integrate_kernel<false><<<tile_blocks(cam.width, cam.height), 256, 0, st>>>(s, cam, frame_index, pr, ris, gb, rv,
                                                                              color, err);
}

}  // namespace hdr
