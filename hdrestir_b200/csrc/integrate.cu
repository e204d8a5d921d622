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
__device__ __forceinline__ void integrate_pixel(const DeviceScene &s, const CameraD &cam, int frame_index,
                                                const PathRun &pr, const RisRun &ris, const GBufferView &gb,
                                                const ReservoirView &rv, float4 *color, int x, int y, unsigned &e) {
    const size_t i = (size_t)y * (size_t)cam.width + (size_t)x;
    uint64_t spill[312];
    MtStream rng;
    rng.init((uint32_t)i ^ (uint32_t)((unsigned long long)frame_index * 12345ULL), spill);
    const float px = (float)x + rng.next_float();
    const float py = (float)y + rng.next_float();
    const RayF ray = camera_ray(cam, px, py, rng);
    const SpectralCtx sc = make_spectral_ctx(rng.next_float());
    Hit h;
    const bool has = load_gbuffer_hit(s, gb, i, h);
    const TraceNow now{&s};
    const Spec L = path_li<kRis>(s, now, ray.o, ray.d, has, h, sc, rng, pr, ris, rv, i, nullptr, e);
    V3 rgb = spectrum_to_rgb(L, sc.cie);
    if (cam.p.has_params && cam.p.enable_exposure) rgb = rgb * cam.p.exposure_mult;
    color[i] = make_float4(rgb.x, rgb.y, rgb.z, 1.0f);
}

template <bool kRis>
__global__ void __launch_bounds__(256) integrate_kernel(DeviceScene s, CameraD cam, int frame_arg, PathRun pr,
                                                        RisRun ris, GBufferView gb, ReservoirView rv, float4 *color,
                                                        unsigned *err) {
    int x, y;
    if (!tile_pixel(cam.width, cam.height, x, y)) return;
    unsigned e = 0;
    integrate_pixel<kRis>(s, cam, live_frame(cam, frame_arg), pr, ris, gb, rv, color, x, y, e);
    if (e) atomicOr(err, e);
}

// Batched PathTracePass: the 16x16 tiles of every image of the batch in one
// grid; a block finds its image by binary search over the images' first tiles.
__global__ void __launch_bounds__(256) path_trace_batch_kernel(DeviceScene s, const PtJobD *__restrict__ jobs,
                                                               int n_jobs) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {  // last job whose tile_begin <= blockIdx.x
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&jobs[mid].tile_begin) <= (int)blockIdx.x)
            lo = mid;
        else
            hi = mid - 1;
    }
    const PtJobD &j = jobs[lo];
    int x, y;
    if (!tile_pixel(j.cam.width, j.cam.height, x, y, (int)blockIdx.x - j.tile_begin)) return;
    unsigned e = 0;
    const RisRun ris{};
    const ReservoirView rv{};
    integrate_pixel<false>(s, j.cam, j.frame_index, j.pr, ris, j.gb, rv, j.color, x, y, e);
    if (e) atomicOr(j.err, e);
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
    ris.reproj = p.reproj;
    integrate_kernel<true><<<tile_blocks(cam.width, cam.height), 256, 0, st>>>(s, cam, frame_index, pr, ris, gb, res,
                                                                             color, err);
}

PathRun path_run_of(const PathParamsD &p) {
    return make_path_run(p.max_depth, p.enable_subsurface, p.max_refl, p.max_refr, p.render_ibl_background,
                         p.roulette);
}

void launch_path_trace_batch(const DeviceScene &s, const PtJobD *jobs, int n_jobs, int total_tiles,
                             cudaStream_t st) {
    path_trace_batch_kernel<<<total_tiles, 256, 0, st>>>(s, jobs, n_jobs);
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
