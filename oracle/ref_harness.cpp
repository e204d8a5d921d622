// Harness around the reference's own hot-path sources, compiled in place
// against the shim headers (oracle/shim) — TEST INFRASTRUCTURE.
//
// Builds a Restir::Scene from an hdr_scene_desc the way the Hydra adapter
// feeds it (one mesh subset per instance, PreviewSurface params per material,
// LightFactoryInput per light), runs the reference passes RaycastPass ->
// PathTracePass | RISPathTracePass -> AccumulationPass with the persistent
// buffer store of RenderPipeline::Execute (pipeline/render_pipeline.cpp:24-40),
// and exports GBuffer, Color and "__ris_reservoir" through a C interface for
// the parity tests and the CPU baseline. Nothing here is part of the product.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../include/hdrestir.h"
#include "pxr/base/work/loops.h"
#include "accumulation_pass.h"
#include "denoiser.h"
#include "hydra/hd_restir_render_buffer.h"
#include "upscale_pass.h"
#include "ref_prims.h"
#include "path_trace_pass.h"
#include "pxr/imaging/hio/image.h"
#include "raycast_pass.h"
#include "render_context.h"
#include "reservoir.h"
#include "restir/output_names.h"
#include "ris_direct_light_integrator.h"
#include "ris_path_trace_pass.h"
#include "rng.h"
#include "scene.h"

using namespace Restir;

// Material textures load through the reference's own ImageTextureSamplerFactory
// (scene/image_texture_sampler.cpp, compiled in), reading the HioImage stand-in,
// where this harness registers each material's texels.

using refprims::path_of;
using refprims::RefMesh;


struct ref_params {
    int32_t pipeline;  // 0 PathTracer, 1 RIS
    int32_t candidate_count, use_reservoir, skip_visibility;
    int32_t max_depth, enable_subsurface, max_refl, max_refr, render_ibl_background;
    float roulette;
    int32_t firefly, accumulate;
    int32_t resolution_level;
};

struct ref_reservoir {  // same layout as the C oracle's orc_reservoir
    int32_t has_sample, has_lc, light, origin, vis_tested, pdf_solid, m;
    float dir[3], color[3], normal[3];
    float dist, pdf, target, wsum, w;
    float tp[4];
};

struct RefScene {
    Scene scene;
    std::vector<std::unique_ptr<RefMesh>> meshes;
    FrameBuffersMap store;
    size_t store_pixels = 0;  // frame size the persistent buffers in `store` were made for
    std::unordered_map<const ILight *, int> light_index;
    std::string error;
};

extern "C" {

RefScene *ref_create(const hdr_scene_desc *d) {
    auto *rs = new RefScene();
    try {
        refprims::RefPrims prims;
        if (!refprims::Populate(d, rs->scene, prims)) {
            rs->error = prims.error;
            delete rs;
            return nullptr;
        }
        for (auto &m : prims.meshes) rs->meshes.push_back(std::move(m));
        SceneBuildRenderStateConfig config{};
        config.EnablePhysicalSky = d->enable_physical_sky != 0;
        config.PhysicalSkyTime = d->physical_sky_time;
        rs->scene.BuildRenderState(config, GetMainThreadRenderJob());
        const auto lights = rs->scene.GetLights();
        for (size_t k = 0; k < lights.size(); ++k) rs->light_index[lights[k]] = (int)k;
        // the physical sky's sun is the light after the scene's own (it is not one of them)
        if (const PhysicalSky *sky = rs->scene.GetPhysicalSky()) rs->light_index[sky] = (int)lights.size();
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_create: %s\n", e.what());
        delete rs;
        return nullptr;
    }
    return rs;
}

void ref_destroy(RefScene *rs) { delete rs; }

void ref_clear_persistent(RefScene *rs) {
    rs->store.Clear();
    rs->store_pixels = 0;
}

static void texel_from_hit(hdr_gbuffer_texel &t, const std::optional<HitRecord> &h) {
    std::memset(&t, 0, sizeof(t));
    t.tri_id = -1;
    if (!h) {
        t.depth = 3.402823466e+38f;
        t.prim_id = -1;
        return;
    }
    for (int i = 0; i < 3; ++i) {
        t.position[i] = h->Position[i];
        t.normal[i] = h->Normal[i];
        t.smooth_normal[i] = h->SmoothNormal[i];
        t.albedo[i] = h->Albedo[i];
        t.dpdu[i] = h->Dpdu[i];
        t.dpdv[i] = h->Dpdv[i];
    }
    t.depth = h->Depth;
    t.prim_id = h->PrimId;
    t.hit = 1;
    t.uv[0] = h->Uv[0];
    t.uv[1] = h->Uv[1];
}

// One frame through the reference passes. Outputs may be NULL; sizes are
// RenderedWidth x RenderedHeight of the chosen resolution level.
//
// tile_row_stride > 0 renders a bounded sample of the frame for CPU timing: the
// passes' 16x16 tile loops (WorkParallelForN over the tiles) run only the tile
// rows tile_row_offset, +stride, +2 stride, ... of the real frame (the shim's
// loop selection); every other pixel keeps a miss in "GBuffer" and zero in
// "Color", and the persistent store carries those rows' reservoirs from frame
// to frame like any frame's. times (if not NULL) receives the wall seconds of
// RaycastPass + the integration pass [0] and of AccumulationPass [1] (the full
// frame: it loops over every pixel on one thread), and [2] the tile rows run.
static int render_frame(RefScene *rs, const hdr_camera *cam, int frame_index, const ref_params *p,
                        hdr_gbuffer_texel *gbuf_out, float *color_out, ref_reservoir *res_out, int tile_row_stride,
                        int tile_row_offset, double *times) {
    try {
        GfMatrix4d view, proj;
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) view[r][c] = cam->view[4 * r + c], proj[r][c] = cam->proj[4 * r + c];
        std::optional<CameraParams> cp;
        if (cam->has_params) {
            CameraParams q;
            q.enableDoF = cam->enable_dof != 0;
            q.enableExposure = cam->enable_exposure != 0;
            q.focalLength = cam->focal_length;
            q.fStop = cam->f_stop;
            q.focusDistance = cam->focus_distance;
            q.bokehBlades = cam->bokeh_blades;
            q.lensDistortion = cam->lens_distortion;
            q.iso = cam->iso;
            q.shutterSpeed = cam->shutter_speed;
            cp = q;
        }
        Rng rng{static_cast<std::uint32_t>(frame_index)};
        RenderContext ctx{
            .scene = &rs->scene,
            .viewMatrix = view,
            .projMatrix = proj,
            .frame = CameraFrame{.windowWidth = cam->width, .windowHeight = cam->height,
                                 .resolutionLevel = p->resolution_level, .visibleMinX = 0, .visibleMinY = 0,
                                 .visibleMaxX = cam->width, .visibleMaxY = cam->height},
            .frameIndex = frame_index,
            .rng = rng,
            .buffers = FrameBuffersMap{},
            .OutputNames = {"Color"},
            .cameraParams = cp,
        };
        PathTracePassSettings settings;
        settings.EnableSubsurface = p->enable_subsurface != 0;
        settings.MaxReflectionBounces = p->max_refl;
        settings.MaxRefractionBounces = p->max_refr;
        settings.RenderIblBackground = p->render_ibl_background != 0;
        settings.RouletteAggressiveness = p->roulette;
        RaycastPass raycast{};
        std::unique_ptr<RenderPass> integ;
        if (p->pipeline == 1)
            integ = std::make_unique<RISPathTracePass>(p->candidate_count, p->use_reservoir != 0,
                                                       p->skip_visibility != 0, settings, p->max_depth);
        else
            integ = std::make_unique<PathTracePass>(settings, p->max_depth);
        AccumulationPass accum{p->firefly != 0};
        // A new frame size makes the renderer mark its integrand dirty and clear the
        // persistent buffers (renderer.cpp:401-406); the passes index them by pixel.
        if (rs->store_pixels != ctx.frame.PixelCount()) {
            rs->store.Clear();
            rs->store_pixels = ctx.frame.PixelCount();
        }
        // the sampled tile rows (the passes tile the rendered frame by 16x16)
        const int tiles_x = (ctx.frame.RenderedWidth() + 15) / 16, tiles_y = (ctx.frame.RenderedHeight() + 15) / 16;
        WorkShimSelection &sel = WorkShimSelected();
        sel = WorkShimSelection{};
        int rows_run = tiles_y;
        if (tile_row_stride > 0) {
            sel.total = (size_t)tiles_x * (size_t)tiles_y;
            rows_run = 0;
            for (int ty = tile_row_offset % tile_row_stride; ty < tiles_y; ty += tile_row_stride, ++rows_run)
                sel.ranges.emplace_back((size_t)ty * tiles_x, (size_t)(ty + 1) * tiles_x);
        }
        // RenderPipeline::Execute (pipeline/render_pipeline.cpp:24-40)
        ctx.buffers.InjectFrom(rs->store);
        const auto t0 = std::chrono::steady_clock::now();
        raycast.Execute(ctx);
        integ->Execute(ctx);
        const auto t1 = std::chrono::steady_clock::now();
        sel = WorkShimSelection{};
        if (p->accumulate) accum.Execute(ctx);
        const auto t2 = std::chrono::steady_clock::now();
        ctx.buffers.ExtractPersistentTo(rs->store);
        if (times) {
            times[0] = std::chrono::duration<double>(t1 - t0).count();
            times[1] = std::chrono::duration<double>(t2 - t1).count();
            times[2] = rows_run;
        }

        const size_t n = ctx.frame.PixelCount();
        if (gbuf_out) {
            auto g = ctx.buffers.Get<std::optional<HitRecord>>("GBuffer");
            for (size_t i = 0; i < n; ++i) texel_from_hit(gbuf_out[i], g[i]);
        }
        if (color_out) {
            auto c = ctx.buffers.Get<GfVec4f>("Color");
            for (size_t i = 0; i < n; ++i)
                for (int k = 0; k < 4; ++k) color_out[4 * i + k] = c[i][k];
        }
        if (res_out && rs->store.Has(kReservoirBufferName)) {
            using ResT = WeightedReservoir<RisDirectLightIntegrator::Candidate>;
            auto rb = rs->store.GetFrameBuffer(kReservoirBufferName).As<ResT>();
            for (size_t i = 0; i < n; ++i) {
                const ResT &r = rb[i];
                ref_reservoir &o = res_out[i];
                std::memset(&o, 0, sizeof(o));
                o.light = -1;
                o.m = r.CandidateCount;
                o.wsum = r.WSum;
                o.w = r.W;
                if (!r.ChosenSample) continue;
                const auto &cs = *r.ChosenSample;
                o.has_sample = 1;
                o.origin = (int)cs.Origin;
                o.vis_tested = cs.VisibilityTested ? 1 : 0;
                o.target = (float)cs.targetFunction;
                for (int k = 0; k < 4; ++k) o.tp[k] = cs.Throughput[k];
                if (cs.Candidate) {
                    const LightCandidate &lc = *cs.Candidate;
                    o.has_lc = 1;
                    auto it = rs->light_index.find(lc.Light.get());
                    o.light = it == rs->light_index.end() ? -2 : it->second;
                    for (int k = 0; k < 3; ++k) {
                        o.dir[k] = lc.Ls.Dir[k];
                        o.color[k] = lc.Ls.Color[k];
                        o.normal[k] = lc.Ls.LightNormal[k];
                    }
                    o.dist = lc.Ls.Dist;
                    o.pdf = lc.Ls.Pdf.value;
                    o.pdf_solid = lc.Ls.Pdf.space == PdfSpace::SolidAngle ? 1 : 0;
                }
            }
        }
        return (int)n;
    } catch (const std::exception &e) {
        WorkShimSelected() = WorkShimSelection{};
        std::fprintf(stderr, "ref_render_frame: %s\n", e.what());
        return -1;
    }
}

int ref_render_frame(RefScene *rs, const hdr_camera *cam, int frame_index, const ref_params *p,
                     hdr_gbuffer_texel *gbuf_out, float *color_out, ref_reservoir *res_out) {
    return render_frame(rs, cam, frame_index, p, gbuf_out, color_out, res_out, 0, 0, nullptr);
}

// A timed sample of one frame (see render_frame): the chosen tile rows through
// RaycastPass and the integration pass, then AccumulationPass over the frame.
int ref_render_frame_sampled(RefScene *rs, const hdr_camera *cam, int frame_index, const ref_params *p,
                             int tile_row_stride, int tile_row_offset, float *color_out, double *times) {
    return render_frame(rs, cam, frame_index, p, nullptr, color_out, nullptr, tile_row_stride, tile_row_offset,
                        times);
}

int ref_trace_rays(RefScene *rs, const float *rays, int n, hdr_gbuffer_texel *out) {
    for (int k = 0; k < n; ++k) {
        const GfVec3f o(rays[6 * k], rays[6 * k + 1], rays[6 * k + 2]);
        const GfVec3f d(rays[6 * k + 3], rays[6 * k + 4], rays[6 * k + 5]);
        texel_from_hit(out[k], rs->scene.IntersectScene(o, d));
    }
    return n;
}

void ref_rng_floats(const uint32_t *seeds, int n, int count, float *out) {
    for (int k = 0; k < n; ++k) {
        Rng r{seeds[k]};
        for (int j = 0; j < count; ++j) out[(size_t)k * count + j] = r.NextFloat();
    }
}

// WeightedReservoir known answers of tests/test_reservoir.cpp, run on the
// reference type itself: returns W of (weight 6, p-hat 3, one candidate).
float ref_reservoir_known_answer(float weight, float phat, int candidates_per_frame) {
    struct S {
        int id;
        float targetFunction;
    };
    WeightedReservoir<S> r{};
    Rng rng{777u};
    r.Update(S{0, phat}, weight, rng);
    r.Finalize(candidates_per_frame);
    return r.W;
}

// UpscalePass::_execute on one named buffer ("Color" RGBA, "Albedo" / "Normal"
// RGB, "Depth" float, as GetOutputDataType types them): src holds the frame at
// `level` (RenderedWidth x RenderedHeight floats), dst receives window_w x
// window_h pixels. Returns the components per pixel, or -1.
int ref_upscale(const char *name, const float *src, int window_w, int window_h, int level, float *dst) {
    static Scene empty_scene;
    const GfMatrix4d ident(1.0);
    Rng rng{0u};
    RenderContext ctx{
        .scene = &empty_scene,
        .viewMatrix = ident,
        .projMatrix = ident,
        .frame = CameraFrame{.windowWidth = window_w, .windowHeight = window_h, .resolutionLevel = level,
                             .visibleMinX = 0, .visibleMinY = 0, .visibleMaxX = window_w, .visibleMaxY = window_h},
        .frameIndex = 0,
        .rng = rng,
        .buffers = FrameBuffersMap{},
        .OutputNames = {name},
        .cameraParams = std::nullopt,
    };
    int comps = 0;
    switch (GetOutputDataType(name)) {
        case OutputDataType::Color4: comps = 4; break;
        case OutputDataType::Vec3: comps = 3; break;
        case OutputDataType::Float1: comps = 1; break;
        default: return -1;
    }
    const size_t n_src = ctx.frame.PixelCount();
    ctx.buffers.Add(name, sizeof(float) * comps, n_src);
    std::memcpy(ctx.buffers.GetFrameBuffer(name).Data(), src, n_src * comps * sizeof(float));
    UpscalePass pass{{name}};
    pass.Execute(ctx);
    const FrameBuffer &out = ctx.buffers.GetFrameBuffer(name);
    std::memcpy(dst, out.Data(), out.SizeBytes());
    return comps;
}

// Denoiser::Run without OIDN (the chromaticity blur alone, alpha kept) on an
// RGBA float frame, in place.
void ref_denoise(float *rgba, int width, int height, int chromaticity_blur) {
    Denoiser::Config cfg;
    cfg.EnableChromaticityBlur = chromaticity_blur != 0;
    Denoiser::Run(gsl::span<pxr::GfVec4f>{reinterpret_cast<pxr::GfVec4f *>(rgba), (size_t)width * (size_t)height},
                  width, height, cfg);
}

// AccumulationPass::Execute on a caller frame: "Color" (width x height RGBA
// floats, in place) and the persistent "__accum_color" (accum, in and out), as
// RenderPipeline::Execute hands them to the pass from frame to frame.
void ref_accumulate(float *color, float *accum, int width, int height, int frame_index, int firefly) {
    static Scene empty_scene;
    const GfMatrix4d ident(1.0);
    Rng rng{0u};
    RenderContext ctx{
        .scene = &empty_scene,
        .viewMatrix = ident,
        .projMatrix = ident,
        .frame = CameraFrame{.windowWidth = width, .windowHeight = height, .resolutionLevel = 0,
                             .visibleMinX = 0, .visibleMinY = 0, .visibleMaxX = width, .visibleMaxY = height},
        .frameIndex = frame_index,
        .rng = rng,
        .buffers = FrameBuffersMap{},
        .OutputNames = {"Color"},
        .cameraParams = std::nullopt,
    };
    const size_t n = ctx.frame.PixelCount();
    ctx.buffers.Add(kColorOutputName, sizeof(GfVec4f), n);
    std::memcpy(ctx.buffers.GetFrameBuffer(kColorOutputName).Data(), color, n * sizeof(GfVec4f));
    ctx.buffers.AddOrGetPersistent(kAccumColorBuf, sizeof(GfVec4f), n);
    std::memcpy(ctx.buffers.GetFrameBuffer(kAccumColorBuf).Data(), accum, n * sizeof(GfVec4f));
    AccumulationPass pass{firefly != 0};
    pass.Execute(ctx);
    std::memcpy(color, ctx.buffers.GetFrameBuffer(kColorOutputName).Data(), n * sizeof(GfVec4f));
    std::memcpy(accum, ctx.buffers.GetFrameBuffer(kAccumColorBuf).Data(), n * sizeof(GfVec4f));
}

// HdRestirRenderBuffer::CopyFromFrameBuffer + Resolve (hydra/hd_restir_render_buffer.cpp:
// 46-73, 113-148, 176-186) on a float frame buffer of `pixels` x src_components:
// the render buffer is allocated with `format` (the HdFormat of the shim:
// component type x 4 + components - 1), filled from the frame buffer and
// resolved; dst receives Map()'s bytes. Returns the bytes written, or -1.
int ref_resolve(const float *src, int pixels, int src_components, int format, unsigned char *dst) {
    HdRestirRenderBuffer rb{SdfPath("/renderBuffer")};
    if (!rb.Allocate(GfVec3i(pixels, 1, 1), (HdFormat)format, false)) return -1;
    FrameBuffer fb{"Color", sizeof(float) * (size_t)src_components, (size_t)pixels};
    std::memcpy(fb.Data(), src, sizeof(float) * (size_t)src_components * (size_t)pixels);
    rb.CopyFromFrameBuffer(fb);
    rb.Resolve();
    const size_t bytes = HdDataSizeOfFormat((HdFormat)format) * (size_t)pixels;
    std::memcpy(dst, rb.Map(), bytes);
    rb.Unmap();
    return (int)bytes;
}

const char *ref_version(void) { return "hdRestir reference sources compiled in place with the oracle shim"; }

// The scene's PhysicalSky (Scene::BuildRenderState with EnablePhysicalSky): Sample()
// along each of n directions (xyz) into out (rgb), and SampleDirect's sun into
// sun (direction, colour). Returns -1 without a sky, else whether the sun gave a sample.
int ref_sky(RefScene *rs, const float *dirs, int n, float *out, float *sun) {
    const PhysicalSky *sky = rs->scene.GetPhysicalSky();
    if (!sky) return -1;
    for (int i = 0; i < n; ++i) {
        const GfVec3f c = sky->Sample(GfVec3f(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
        for (int k = 0; k < 3; ++k) out[3 * i + k] = c[k];
    }
    const auto s = sky->SampleDirect();
    if (!s) return 0;
    for (int k = 0; k < 3; ++k) sun[k] = s->Dir[k], sun[3 + k] = s->Color[k];
    return 1;
}

}  // extern "C"
