// Drop-in check — TEST INFRASTRUCTURE. Runs the reference's own RenderPipeline
// (pipeline/render_pipeline.cpp) with the GPU passes of
// hdrestir_b200/integration/gpu_passes.h in place of the CPU passes, exactly
// as a maintainer would wire them in, and returns the final
// "Color" the renderer would resolve. Built with the reference sources in place
// (oracle/Makefile, target ref-gpu) and linked against libhdrestir_b200.so.
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <memory>

#include "gpu_passes.h"
#include "ref_prims.h"
#include "render_pipeline.h"
#include "scene.h"
#include "scene_handoff.h"

using namespace Restir;

struct ref_gpu_params {
    int32_t pipeline;  // 0 PathTracer, 1 RIS
    int32_t candidate_count, use_reservoir, skip_visibility, max_depth;
    int32_t firefly;
    int32_t resolution_level;  // > 0: render at ceil(window / 2^level) and end with the upscale pass
};

namespace {

// Decodes a texture of the HioImage stand-in as ImageTextureSamplerFactory does
// for the harness's registered linear texels (test scenes use the linear variant).
bool load_registered(const SdfAssetPath &asset, bool, std::vector<float> &rgb, int &w, int &h) {
    HioImageSharedPtr img = HioImage::OpenForReading(asset.GetResolvedPath());
    if (!img) return false;
    w = img->GetWidth();
    h = img->GetHeight();
    rgb.assign((size_t)w * h * 3, 0.0f);
    HioImage::StorageSpec spec;
    spec.format = HioFormatFloat32Vec3;
    spec.width = w;
    spec.height = h;
    spec.data = rgb.data();
    return img->Read(spec);
}

int render(std::shared_ptr<B200::DeviceContext> dev, Scene *cpu_scene, const hdr_camera *cam, int frames,
           const ref_gpu_params *p, float *color_out);

}  // namespace

// The scene reaches the device only through the reference's Scene inputs: the
// harness's prims call AddMesh / SetMaterialParams / SetLightFactoryInput on a
// scene hand-off that forwards each call to a reference Scene, and
// BuildRenderState builds both that Scene's render state and the device scene.
// The frames render with that Scene in the RenderContext.
extern "C" int refgpu_render_scene(const hdr_scene_desc *desc, const hdr_camera *cam, int frames,
                                   const ref_gpu_params *p, float *color_out) {
    try {
        auto dev = std::make_shared<B200::DeviceContext>(0);
        Scene scene;
        B200::SceneHandoff handoff(&scene);
        handoff.SetTextureLoader(load_registered);
        refprims::RefPrims prims;
        if (!refprims::Populate(desc, handoff, prims)) {
            std::fprintf(stderr, "refgpu_render_scene: %s\n", prims.error.c_str());
            return -1;
        }
        handoff.BuildRenderState(SceneBuildRenderStateConfig{}, GetMainThreadRenderJob(), dev->Get());
        return render(dev, &scene, cam, frames, p, color_out);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "refgpu_render_scene: %s\n", e.what());
        return -1;
    }
}

extern "C" int refgpu_render(const hdr_scene_desc *desc, const hdr_camera *cam, int frames, const ref_gpu_params *p,
                             float *color_out) {
    try {
        auto dev = std::make_shared<B200::DeviceContext>(0);
        dev->UploadScene(*desc);
        static Scene unused_cpu_scene;  // the GPU passes read the device scene only
        return render(dev, &unused_cpu_scene, cam, frames, p, color_out);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "refgpu_render: %s\n", e.what());
        return -1;
    }
}

namespace {
int render(std::shared_ptr<B200::DeviceContext> dev, Scene *cpu_scene, const hdr_camera *cam, int frames,
           const ref_gpu_params *p, float *color_out) {
    {
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
        for (int f = 0; f < frames; ++f) {
            Rng rng{static_cast<std::uint32_t>(f)};
            RenderContext ctx{
                .scene = cpu_scene,
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
    }
}
}  // namespace

namespace {
template <class T>
bool same(const T *a, const T *b, size_t n) {
    return n == 0 || (a && b && std::memcmp(a, b, n * sizeof(T)) == 0);
}
}  // namespace

// The scene hand-off's descriptor against the one the prims were made from
// (host only): instance by instance, the same mesh arrays, transform, material
// and light link; materials and lights field for field. Returns 0 when equal,
// else the 1-based number of the first check that failed.
extern "C" int refgpu_handoff_compare(const hdr_scene_desc *d) {
    try {
        B200::SceneHandoff handoff;
        handoff.SetTextureLoader(load_registered);
        refprims::RefPrims prims;
        if (!refprims::Populate(d, handoff, prims)) return -1;
        const hdr_scene_desc &h = handoff.Build();
        if (h.num_instances != d->num_instances || h.num_materials != d->num_materials || h.num_lights != d->num_lights)
            return 1;
        for (int i = 0; i < d->num_instances; ++i) {
            const hdr_instance_desc &a = d->instances[i], &b = h.instances[i];
            if (a.material != b.material || a.light != b.light || !same(a.transform, b.transform, 16)) return 2;
            const hdr_mesh_desc &ma = d->meshes[a.mesh], &mb = h.meshes[b.mesh];
            if (ma.num_points != mb.num_points || ma.num_triangles != mb.num_triangles || ma.num_uvs != mb.num_uvs ||
                ma.num_normals != mb.num_normals || ma.num_colors != mb.num_colors)
                return 3;
            if (!same(ma.points, mb.points, 3 * (size_t)ma.num_points) ||
                !same(ma.indices, mb.indices, 3 * (size_t)ma.num_triangles) ||
                !same(ma.uvs, mb.uvs, 2 * (size_t)ma.num_uvs) || !same(ma.normals, mb.normals, 3 * (size_t)ma.num_normals) ||
                !same(ma.colors, mb.colors, 3 * (size_t)ma.num_colors))
                return 4;
        }
        for (int k = 0; k < d->num_materials; ++k) {
            const hdr_material_desc &a = d->materials[k], &b = h.materials[k];
            if (std::memcmp(&a, &b, offsetof(hdr_material_desc, textures)) != 0) return 5;
            for (int t = 0; t < 4; ++t) {
                const bool ta = a.textures[t] && a.tex_width[t] > 0 && a.tex_height[t] > 0;
                const bool tb = b.textures[t] != nullptr;
                if (ta != tb) return 6;
                if (ta && (a.tex_width[t] != b.tex_width[t] || a.tex_height[t] != b.tex_height[t] ||
                           !same(a.textures[t], b.textures[t], 3 * (size_t)a.tex_width[t] * a.tex_height[t])))
                    return 7;
            }
        }
        for (int k = 0; k < d->num_lights; ++k) {
            const hdr_light_desc &a = d->lights[k], &b = h.lights[k];
            if (a.type != b.type || !same(a.color, b.color, 3) || a.intensity != b.intensity ||
                a.exposure != b.exposure || !same(a.transform, b.transform, 16) || a.width != b.width ||
                a.height != b.height || a.shaping_cone_angle != b.shaping_cone_angle ||
                a.shaping_cone_softness != b.shaping_cone_softness)
                return 8;
            const bool ta = a.texture && a.tex_width > 0 && a.tex_height > 0;
            if (ta != (b.texture != nullptr) ||
                (ta && !same(a.texture, b.texture, 3 * (size_t)a.tex_width * a.tex_height)))
                return 9;
        }
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "refgpu_handoff_compare: %s\n", e.what());
        return -2;
    }
}
