// Drop-in check — TEST INFRASTRUCTURE. Runs the reference's own RenderPipeline
// (pipeline/render_pipeline.cpp) with the GPU passes of
// hdrestir_b200/integration/gpu_passes.h in place of the CPU passes, exactly
// as a maintainer would wire them in, and returns the final
// "Color" the renderer would resolve. Built with the reference sources in place
// (oracle/Makefile, target ref-gpu) and linked against libhdrestir_b200.so.
#include <cstdio>
#include <memory>

#include "gpu_passes.h"
#include "render_pipeline.h"
#include "scene.h"

using namespace Restir;

struct ref_gpu_params {
    int32_t pipeline;  // 0 PathTracer, 1 RIS
    int32_t candidate_count, use_reservoir, skip_visibility, max_depth;
    int32_t firefly;
    int32_t resolution_level;  // > 0: render at ceil(window / 2^level) and end with the upscale pass
};

extern "C" int refgpu_render(const hdr_scene_desc *desc, const hdr_camera *cam, int frames, const ref_gpu_params *p,
                             float *color_out) {
    try {
        auto dev = std::make_shared<B200::DeviceContext>(0);
        dev->UploadScene(*desc);
        RenderPipeline pipe{"GPU"};
        PathTracePassSettings settings{};
        pipe.Add(std::make_unique<B200::GpuRaycastPass>(dev));
        if (p->pipeline == 1)
            pipe.Add(std::make_unique<B200::GpuRISPathTracePass>(dev, p->candidate_count, p->use_reservoir != 0,
                                                                 p->skip_visibility != 0, settings, p->max_depth));
        else
            pipe.Add(std::make_unique<B200::GpuPathTracePass>(dev, settings, p->max_depth));
        pipe.Add(std::make_unique<B200::GpuAccumulationPassB200>(dev, p->firefly != 0));
        if (p->resolution_level > 0)
            pipe.Add(std::make_unique<B200::GpuUpscalePass>(dev, std::vector<std::string>{"Color"}));
        GfMatrix4d view, proj;
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) view[r][c] = cam->view[4 * r + c], proj[r][c] = cam->proj[4 * r + c];
        std::size_t n = 0;
        static Scene unused_cpu_scene;  // the GPU passes read the device scene only
        for (int f = 0; f < frames; ++f) {
            Rng rng{static_cast<std::uint32_t>(f)};
            RenderContext ctx{
                .scene = &unused_cpu_scene,
                .viewMatrix = view,
                .projMatrix = proj,
                .frame = CameraFrame{.windowWidth = cam->width, .windowHeight = cam->height,
                                     .resolutionLevel = p->resolution_level,
                                     .visibleMinX = 0, .visibleMinY = 0, .visibleMaxX = cam->width,
                                     .visibleMaxY = cam->height},
                .frameIndex = f,
                .rng = rng,
                .buffers = FrameBuffersMap{},
                .OutputNames = {"Color"},
                .cameraParams = std::nullopt,
            };
            pipe.Execute(ctx);
            auto color = ctx.buffers.Get<GfVec4f>(kColorOutputName);
            n = color.size();
            if (f == frames - 1)
                for (std::size_t i = 0; i < n; ++i)
                    for (int k = 0; k < 4; ++k) color_out[4 * i + k] = color[i][k];
        }
        return (int)n;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "refgpu_render: %s\n", e.what());
        return -1;
    }
}
