// GPU passes for the reference renderer's RenderPipeline, on the hdrestir
// C ABI (include/hdrestir.h). Header-only; compiled inside the reference tree
// next to passes/raycast_pass.h etc., with -I for include/ and this directory.
//
// They implement the reference's pass interface (passes/render_pass.h:13-48,
// HasStaticPassIo) with the same names, inputs and outputs as the CPU passes
// they replace:
//   GpuRaycastPass          <- RaycastPass       (passes/raycast_pass.h)
//   GpuRISPathTracePass     <- RISPathTracePass  (restir_passes/ris_path_trace_pass.h)
//   GpuPathTracePass        <- PathTracePass     (passes/path_trace_pass.h)
//   GpuAccumulationPassB200 <- AccumulationPass / GpuAccumulationPass
//   GpuUpscalePass          <- UpscalePass       (passes/upscale_pass.h)
// Frame buffers stay on the device between passes and frames; the last pass
// copies "Color" into ctx.buffers so the renderer's AOV resolve
// (renderer.cpp:462-475) finds it where the CPU pipeline leaves it.
// Errors surface as std::runtime_error, like the reference's GPU pass.
#pragma once

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "hdrestir.h"
#include "passes/output_names.h"
#include "path_integrator.h"
#include "render_context.h"
#include "render_pass.h"

namespace Restir::B200 {

inline void Check(hdr_status st, const char *what) {
    if (st != HDR_OK) throw std::runtime_error(std::string("[hdrestir-b200] ") + what + ": " + hdr_last_error());
}

// One device context per pipeline instance (a ctx owns a stream and the device
// frame buffers). The caller uploads the scene whenever Scene::BuildRenderState
// would rebuild it.
class DeviceContext {
  public:
    explicit DeviceContext(int device = 0) {
        hdr_ctx_desc d{};
        d.device = device;
        Check(hdr_ctx_create(&_ctx, &d), "hdr_ctx_create");
    }
    ~DeviceContext() { hdr_ctx_destroy(_ctx); }
    DeviceContext(const DeviceContext &) = delete;
    DeviceContext &operator=(const DeviceContext &) = delete;
    void UploadScene(const hdr_scene_desc &desc) { Check(hdr_scene_upload(_ctx, &desc), "hdr_scene_upload"); }
    void ClearPersistentBuffers() { Check(hdr_clear_persistent(_ctx), "hdr_clear_persistent"); }
    hdr_ctx *Get() const noexcept { return _ctx; }

  private:
    hdr_ctx *_ctx{nullptr};
};

// RenderContext -> hdr_camera (camera matrices, CameraFrame size, CameraParams)
inline hdr_camera MakeCamera(const RenderContext &ctx) {
    hdr_camera c{};
    for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 4; ++k) {
            c.view[4 * r + k] = ctx.viewMatrix[r][k];
            c.proj[4 * r + k] = ctx.projMatrix[r][k];
        }
    c.width = ctx.frame.RenderedWidth();
    c.height = ctx.frame.RenderedHeight();
    if (ctx.cameraParams) {
        const CameraParams &p = *ctx.cameraParams;
        c.has_params = 1;
        c.enable_dof = p.enableDoF;
        c.enable_exposure = p.enableExposure;
        c.focal_length = p.focalLength;
        c.f_stop = p.fStop;
        c.focus_distance = p.focusDistance;
        c.bokeh_blades = p.bokehBlades;
        c.lens_distortion = p.lensDistortion;
        c.iso = p.iso;
        c.shutter_speed = p.shutterSpeed;
    }
    return c;
}

inline hdr_path_settings MakePathSettings(const PathTracePassSettings &s, int maxDepth) {
    return hdr_path_settings{maxDepth, s.EnableSubsurface ? 1 : 0, s.MaxReflectionBounces, s.MaxRefractionBounces,
                             s.RenderIblBackground ? 1 : 0, s.RouletteAggressiveness};
}

class GpuRaycastPass final : public RenderPass {
  public:
    explicit GpuRaycastPass(std::shared_ptr<DeviceContext> dev, std::vector<std::string> requestedOutputs = {})
        : RenderPass{"GpuRaycastPass"}, _dev{std::move(dev)}, _requested{std::move(requestedOutputs)} {}
    static std::vector<std::string> StaticInputs() { return {}; }
    static std::vector<std::string> StaticOutputs() {
        return {std::string{kGBufferOutputName}, std::string{kDepthOutputName}, std::string{kAlbedoOutputName},
                std::string{kNormalOutputName}};
    }
    std::vector<std::string> Inputs() const override { return {}; }
    std::vector<std::string> Outputs() const override {
        std::vector<std::string> out{std::string{kGBufferOutputName}};
        for (const auto &n : _requested)
            if (n == kDepthOutputName || n == kAlbedoOutputName || n == kNormalOutputName) out.push_back(n);
        return out;
    }

  protected:
    void _execute(RenderContext &ctx) override {
        uint32_t mask = 0;
        for (const auto &n : Outputs()) {
            if (n == kDepthOutputName) mask |= HDR_AOV_DEPTH;
            if (n == kAlbedoOutputName) mask |= HDR_AOV_ALBEDO;
            if (n == kNormalOutputName) mask |= HDR_AOV_NORMAL;
        }
        const hdr_camera cam = MakeCamera(ctx);
        Check(hdr_raycast(_dev->Get(), &cam, ctx.frameIndex, mask), "hdr_raycast");
    }

  private:
    std::shared_ptr<DeviceContext> _dev;
    std::vector<std::string> _requested;
};

class GpuRISPathTracePass final : public RenderPass {
  public:
    GpuRISPathTracePass(std::shared_ptr<DeviceContext> dev, int candidateCount = 16, bool useReservoir = true,
                        bool skipVisibility = false, PathTracePassSettings settings = {}, int maxDepth = 32)
        : RenderPass{"GpuRISPathTracePass"}, _dev{std::move(dev)} {
        _p.path = MakePathSettings(settings, maxDepth);
        _p.candidate_count = candidateCount;
        _p.use_reservoir = useReservoir ? 1 : 0;
        _p.skip_visibility = skipVisibility ? 1 : 0;
    }
    static std::vector<std::string> StaticInputs() { return {std::string{kGBufferOutputName}}; }
    static std::vector<std::string> StaticOutputs() { return {std::string{kColorOutputName}}; }
    std::vector<std::string> Inputs() const override { return StaticInputs(); }
    std::vector<std::string> Outputs() const override { return StaticOutputs(); }

  protected:
    void _execute(RenderContext &ctx) override {
        const hdr_camera cam = MakeCamera(ctx);
        Check(hdr_ris_path_trace(_dev->Get(), &cam, ctx.frameIndex, &_p), "hdr_ris_path_trace");
    }

  private:
    std::shared_ptr<DeviceContext> _dev;
    hdr_ris_params _p{};
};

class GpuPathTracePass final : public RenderPass {
  public:
    GpuPathTracePass(std::shared_ptr<DeviceContext> dev, PathTracePassSettings settings = {}, int maxDepth = 32)
        : RenderPass{"GpuPathTracePass"}, _dev{std::move(dev)}, _s{MakePathSettings(settings, maxDepth)} {}
    static std::vector<std::string> StaticInputs() { return {std::string{kGBufferOutputName}}; }
    static std::vector<std::string> StaticOutputs() { return {std::string{kColorOutputName}}; }
    std::vector<std::string> Inputs() const override { return StaticInputs(); }
    std::vector<std::string> Outputs() const override { return StaticOutputs(); }

  protected:
    void _execute(RenderContext &ctx) override {
        const hdr_camera cam = MakeCamera(ctx);
        Check(hdr_path_trace(_dev->Get(), &cam, ctx.frameIndex, &_s), "hdr_path_trace");
    }

  private:
    std::shared_ptr<DeviceContext> _dev;
    hdr_path_settings _s;
};

// Accumulation on the device, then "Color" handed to the host FrameBuffersMap.
class GpuAccumulationPassB200 final : public RenderPass {
  public:
    explicit GpuAccumulationPassB200(std::shared_ptr<DeviceContext> dev, bool enableFireflyFilter = true)
        : RenderPass{"GpuAccumulationPass"}, _dev{std::move(dev)}, _firefly{enableFireflyFilter} {}
    static std::vector<std::string> StaticInputs() { return {std::string{kColorOutputName}}; }
    static std::vector<std::string> StaticOutputs() { return {std::string{kColorOutputName}}; }
    std::vector<std::string> Inputs() const override { return StaticInputs(); }
    std::vector<std::string> Outputs() const override { return StaticOutputs(); }

  protected:
    void _execute(RenderContext &ctx) override {
        Check(hdr_accumulate(_dev->Get(), ctx.frameIndex, _firefly ? 1 : 0, HDR_ACCUM_PARITY), "hdr_accumulate");
        const std::size_t count = ctx.frame.PixelCount();
        ctx.buffers.Add(kColorOutputName, sizeof(GfVec4f), count);
        FrameBuffer &fb = ctx.buffers.GetFrameBuffer(kColorOutputName);
        Check(hdr_download(_dev->Get(), "Color", fb.Data(), fb.SizeBytes()), "hdr_download(Color)");
    }

  private:
    std::shared_ptr<DeviceContext> _dev;
    bool _firefly;
};

// UpscalePass on the device: the named buffers the GPU passes left at the frame's
// rendered size are upscaled in HBM and handed to ctx.buffers at window size.
class GpuUpscalePass final : public RenderPass {
  public:
    explicit GpuUpscalePass(std::shared_ptr<DeviceContext> dev, std::vector<std::string> outputNames = {})
        : RenderPass{"UpscalePass"}, _dev{std::move(dev)}, _outputNames{std::move(outputNames)} {}
    static std::vector<std::string> StaticInputs() {
        return {std::string{kColorOutputName}, std::string{kDepthOutputName}, std::string{kAlbedoOutputName},
                std::string{kNormalOutputName}};
    }
    static std::vector<std::string> StaticOutputs() { return StaticInputs(); }
    std::vector<std::string> Inputs() const override { return _outputNames; }
    std::vector<std::string> Outputs() const override { return _outputNames; }

  protected:
    void _execute(RenderContext &ctx) override {
        if (!ctx.frame.NeedsUpscale()) return;
        const int sw = ctx.frame.RenderedWidth(), sh = ctx.frame.RenderedHeight();
        const int dw = ctx.frame.windowWidth, dh = ctx.frame.windowHeight;
        for (const std::string &name : Outputs()) {
            int comps = 0;
            switch (GetOutputDataType(name)) {
                case OutputDataType::Color4: comps = 4; break;
                case OutputDataType::Vec3: comps = 3; break;
                case OutputDataType::Float1: comps = 1; break;
                default: continue;
            }
            std::size_t have = 0;
            if (hdr_buffer_size(_dev->Get(), name.c_str(), &have) != HDR_OK) continue;  // not produced this frame
            Check(hdr_upscale(_dev->Get(), name.c_str(), comps, sw, sh, dw, dh), "hdr_upscale");
            ctx.buffers.Add(name, sizeof(float) * comps, (std::size_t)dw * (std::size_t)dh);
            FrameBuffer &fb = ctx.buffers.GetFrameBuffer(name);
            Check(hdr_download(_dev->Get(), name.c_str(), fb.Data(), fb.SizeBytes()), "hdr_download");
        }
        ctx.frame.MarkUpscaled();
    }

  private:
    std::shared_ptr<DeviceContext> _dev;
    std::vector<std::string> _outputNames;
};

}  // namespace Restir::B200
