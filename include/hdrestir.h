/*
 * hdrestir.h — C ABI of the B200 (sm_100a) light-transport passes.
 *
 * The reference renderer (hdRestir) runs its per-pixel light transport as CPU
 * RenderPasses behind `RenderPass::Execute/_execute` (source/passes/render_pass.h:13-42).
 * Its only GPU boundary is pass-granular too (GpuAccumulationPass,
 * source/gpu_passes/gpu_accumulation_pass.h). This header is the same boundary
 * for every pass on the hot path: plain C, plain pointers and sizes, no C++ or
 * torch types, integer status codes and a thread-local error string. A pass
 * wrapper on the host (C++ RenderPass subclass, ctypes, cgo, …) forwards its
 * `_execute(RenderContext&)` to one call here; device buffers keep the
 * reference's frame-buffer names ("GBuffer", "Color", "__accum_color",
 * "__ris_reservoir", …; source/passes/output_names.h:10-40,
 * source/restir/output_names.h:10) and stay resident on the GPU between frames.
 *
 * Threading: one hdr_ctx per pipeline instance; calls on one ctx are
 * serialised by an internal mutex and run on the ctx's own CUDA stream.
 * Errors never throw across the ABI.
 */
#ifndef HDRESTIR_B200_H
#define HDRESTIR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HDR_ABI_VERSION 1

/* Status codes. The reference reports failures with exceptions
 * (gpu_accumulation_kernel.cpp:63-109) and DBG_ASSERT/Expects; across this ABI
 * they become integers plus hdr_last_error(). */
typedef enum hdr_status {
    HDR_OK = 0,
    HDR_EINVAL = 1,      /* bad argument, size or name */
    HDR_ENOMEM = 2,      /* device or host allocation failed, or HBM budget exceeded */
    HDR_ECANCELLED = 3,  /* the cancel word was set (IRenderJob::IsCancelled, render_job.h:9-37) */
    HDR_ETIMEOUT = 4,    /* a bounded device wait gave up */
    HDR_ECUDA = 5,       /* a CUDA runtime call failed */
    HDR_ENOSCENE = 6,    /* pass called before hdr_scene_upload */
    HDR_EDEVICE = 7      /* a kernel reported an internal limit (e.g. traversal stack) */
} hdr_status;

typedef struct hdr_ctx hdr_ctx;

/* ---------------------------------------------------------------------------
 * Scene description (host memory, copied at upload).
 * Mirrors what Scene::BuildRenderState consumes (scene/scene.cpp:118-271):
 * mesh subsets (one BLAS each, BVH::Build inputs, renderContext/bvh.h:44-45),
 * instances (appendMeshInstance, scene.cpp:187-222), PreviewSurface params
 * (materials/preview_surface_params.h:12-52) and lights
 * (sceneInterface/scene_interface.h:24-29, light_params.h).
 * ------------------------------------------------------------------------- */
typedef struct hdr_mesh_desc {
    const float *points;          /* xyz per point */
    int32_t num_points;
    const int32_t *indices;       /* 3 point indices per triangle */
    int32_t num_triangles;
    const float *uvs;             /* 2 per entry; per corner when num_uvs == 3*num_triangles, else per point */
    int32_t num_uvs;
    const float *normals;         /* 3 per entry; same per-corner/per-point rule */
    int32_t num_normals;
    const float *colors;          /* 3 per entry; same rule */
    int32_t num_colors;
    const int32_t *material_indices; /* per triangle (BVHTriangle::materialIndex), may be NULL */
    int32_t num_material_indices;
} hdr_mesh_desc;

typedef struct hdr_instance_desc {
    int32_t mesh;        /* index into hdr_scene_desc.meshes */
    int32_t material;    /* index into materials, -1 = DefaultMaterial (default_material.cpp:55-64) */
    int32_t light;       /* light whose geometry this instance is (Scene::GetLightAtHit), -1 = none */
    int32_t reserved;
    float transform[16]; /* GfMatrix4f, row-major, row-vector convention (translation in row 3) */
} hdr_instance_desc;

typedef struct hdr_material_desc { /* PreviewSurfaceParams field for field */
    float diffuse_color[3];
    float metallic;
    float roughness;
    float specular_color[3];
    float specular;
    float opacity;
    float ior;
    float transmission;
    float transmission_color[3];
    float transmission_depth;
    float transmission_scatter[3];
    float emission_color[3];
    float emission;
    float coat;
    float coat_color[3];
    float coat_roughness;
    float coat_ior;
    float sheen;
    float sheen_color[3];
    float sheen_roughness;
    float subsurface;
    float subsurface_color[3];
    float subsurface_radius[3];
    float subsurface_scale;
    float subsurface_anisotropy;
    int32_t thin_walled;
    float diffuse_roughness;
    /* PreviewSurfaceParams DiffuseTexture / MetallicTexture / RoughnessTexture /
     * NormalTexture (materials/preview_surface_params.h:48-51), indexed by HDR_TEX_*,
     * as the RGB f32 texels ImageTextureSamplerFactory decodes for them
     * (scene/image_texture_sampler.cpp:14-123): width*height*3 floats, row 0 first;
     * the diffuse texture in its sRGB-decoded variant (Linear = false), the other
     * three linear. NULL (or a zero size) = no texture, the parameter is used. */
    const float *textures[4];
    int32_t tex_width[4], tex_height[4];
} hdr_material_desc;

enum { HDR_TEX_DIFFUSE = 0, HDR_TEX_METALLIC = 1, HDR_TEX_ROUGHNESS = 2, HDR_TEX_NORMAL = 3 };

/* ---------------------------------------------------------------------------
 * Material networks (HdRestirMaterial::Sync, hydra/hd_restir_material.cpp:22-424):
 * a Hydra material network (UsdPreviewSurface, MaterialX standard_surface or
 * open_pbr_surface, image nodes) mapped to the PreviewSurface parameters the
 * passes shade with. Plain-C view of an HdMaterialNetwork2.
 * ------------------------------------------------------------------------- */
enum { HDR_MTL_FLOAT = 0, HDR_MTL_FLOAT3 = 1, HDR_MTL_BOOL = 2, HDR_MTL_ASSET = 3 };

typedef struct hdr_mtl_param {  /* one entry of HdMaterialNode2::parameters */
    const char *name;
    int32_t type;                /* HDR_MTL_*: the type the VtValue holds (others are skipped) */
    float value[3];              /* FLOAT: [0]; FLOAT3: [0..2]; BOOL: [0] != 0 */
    const char *asset;           /* ASSET: the SdfAssetPath's asset path */
} hdr_mtl_param;

typedef struct hdr_mtl_connection {  /* HdMaterialNode2::inputConnections, one upstream node each */
    const char *input;
    const char *upstream_node;   /* node path */
} hdr_mtl_connection;

typedef struct hdr_mtl_node {
    const char *path;            /* SdfPath of the node */
    const char *shader_id;       /* the shader identifier the Sdr registry resolves (else the node type id) */
    const hdr_mtl_param *params;
    int32_t num_params;
    const hdr_mtl_connection *inputs;
    int32_t num_inputs;
} hdr_mtl_node;

typedef struct hdr_mtl_terminal {   /* HdMaterialNetwork2::terminals */
    const char *name;            /* "mtlx:surface", "surface", ... */
    const char *upstream_node;
} hdr_mtl_terminal;

typedef struct hdr_mtl_network {
    const hdr_mtl_node *nodes;
    int32_t num_nodes;
    const hdr_mtl_terminal *terminals;
    int32_t num_terminals;
} hdr_mtl_network;

typedef struct hdr_mtl_textures {  /* asset paths per HDR_TEX_* slot ("" = none) */
    char path[4][1024];
} hdr_mtl_textures;

/* LightType order of scene/light_factory.h */
/* HDR_LIGHT_TRIANGLE: extension, no reference counterpart (the reference has no emissive-geometry
 * light): an emissive triangle, the half of the rect of the same width, height and transform
 * below its diagonal, with local corners (-w/2, -h/2), (w/2, -h/2), (-w/2, h/2); the transform
 * (affine) places any triangle. One-sided and sampled uniformly over its area like the rect, whose
 * convention it follows: the area is w * h / 2 in local units. */
enum { HDR_LIGHT_DISTANT = 0, HDR_LIGHT_DOME = 1, HDR_LIGHT_RECT = 2, HDR_LIGHT_POINT = 3, HDR_LIGHT_TRIANGLE = 4 };

typedef struct hdr_light_desc {
    int32_t type;
    float color[3];
    float intensity;
    float exposure;
    double transform[16];        /* GfMatrix4d row-major */
    float width, height;
    float shaping_cone_angle;    /* degrees, 180 = no cone */
    float shaping_cone_softness;
    const float *texture;        /* dome: RGB f32, tex_width*tex_height*3 (the decoded TextureFile) */
    int32_t tex_width, tex_height;
    float temperature;           /* extension, no reference counterpart: > 0 makes a rect, triangle,
                                    point or distant light emit a blackbody spectrum of this many
                                    kelvin (Planck's law at the sampled wavelengths, 1 at its peak)
                                    times intensity * 2^exposure, in place of its colour; 0 = colour */
} hdr_light_desc;

typedef struct hdr_scene_desc {
    const hdr_mesh_desc *meshes;
    int32_t num_meshes;
    const hdr_instance_desc *instances;
    int32_t num_instances;
    const hdr_material_desc *materials;
    int32_t num_materials;
    const hdr_light_desc *lights;
    int32_t num_lights;
    /* SceneBuildRenderStateConfig (sceneInterface/scene_interface.h:30-34): with
     * enable_physical_sky the environment is PhysicalSky (scene/physical_sky.cpp),
     * its sun set from physical_sky_time (hours, 12 = noon; scene.cpp:248-256),
     * instead of the first dome light. The sky is not one of the scene's lights: the
     * RIS pass then splits its candidates over three techniques and the path tracer
     * adds a sun sample per vertex. Zero-initialised descriptors leave it off. */
    int32_t enable_physical_sky;
    float physical_sky_time;
} hdr_scene_desc;

/* ---------------------------------------------------------------------------
 * Per-frame inputs
 * ------------------------------------------------------------------------- */
typedef struct hdr_camera {
    double view[16];             /* RenderContext::viewMatrix (GfMatrix4d row-major) */
    double proj[16];             /* RenderContext::projMatrix */
    int32_t width, height;       /* CameraFrame::RenderedWidth/Height */
    int32_t has_params;          /* RenderContext::cameraParams engaged (else pinhole) */
    int32_t enable_dof;          /* CameraParams (scene/camera_params.h:8-20) */
    int32_t enable_exposure;
    float focal_length;
    float f_stop;
    float focus_distance;
    int32_t bokeh_blades;
    float lens_distortion;
    float iso;
    float shutter_speed;
} hdr_camera;

/* PathTracePassSettings (integrators/path_integrator.h:12-19) + maxDepth */
typedef struct hdr_path_settings {
    int32_t max_depth;
    int32_t enable_subsurface;
    int32_t max_reflection_bounces;
    int32_t max_refraction_bounces;
    int32_t render_ibl_background;
    float roulette_aggressiveness;
} hdr_path_settings;

/* RisDirectLightIntegrator::MakeFactory(candidateCount, useReservoir, skipVisibility)
 * (restir/ris_direct_light_integrator.h:73-74). The fields after skip_visibility
 * are extensions with no reference counterpart; zero keeps reference behaviour. */
typedef struct hdr_ris_params {
    hdr_path_settings path;
    int32_t candidate_count;
    int32_t use_reservoir;
    int32_t skip_visibility;
    int32_t m_cap;               /* 0 = unbounded CandidateCount (reservoir.h:147-155) */
    int32_t spatial_neighbors;   /* 0 = temporal-only, same-pixel reuse; 1..64 = after the temporal
                                    merge, merge that many random neighbours' reservoirs (spatial
                                    reuse; wavefront form only: maxDepth 1, opaque scene) */
    float spatial_radius;        /* neighbour radius in pixels; 0 = 30 */
    uint32_t flags;              /* HDR_RIS_* execution options; 0 = defaults */
    int32_t reserved;
} hdr_ris_params;

/* hdr_ris_params.flags. Neither changes the image.
 * TRACE_ALL_RAYS: also cast the rays whose result cannot matter: those of
 *   generated BSDF candidates in scenes without light geometry or environment,
 *   and the path's bounce ray when, besides, no material emits.
 * ONE_KERNEL: integrate each pixel in one thread that casts its own rays,
 *   instead of the generate / trace / shade wavefront.
 * REPROJECT (extension; changes the image, no reference counterpart): for a
 *   moving camera, take a pixel's temporal history from where its hit point was
 *   in the previous frame of this ctx (same surface point within 2 % of depth),
 *   move the history's light sample to the new hit point and test its
 *   visibility again. Without it the reference's same-pixel history is used
 *   (the reference's renderer clears the reservoirs when the camera moves). */
enum { HDR_RIS_TRACE_ALL_RAYS = 1, HDR_RIS_ONE_KERNEL = 2, HDR_RIS_REPROJECT = 4 };

/* AOV selection for hdr_raycast (RaycastPass requestedOutputs, raycast_pass.cpp:39-55) */
enum { HDR_AOV_DEPTH = 1, HDR_AOV_ALBEDO = 2, HDR_AOV_NORMAL = 4 };

/* Accumulation firefly semantics. PARITY reproduces AccumulationPass's in-place
 * row-major clamp (accumulation_pass.cpp:22-60); SHADER reproduces
 * accumulation.slang:55-81, which clamps against the unclamped input. */
enum { HDR_ACCUM_PARITY = 0, HDR_ACCUM_SHADER = 1 };

/* Device GBuffer texel returned by hdr_download("GBuffer"): the fields of
 * std::optional<HitRecord> (core/hit_record.h:15-27) plus the triangle index. */
typedef struct hdr_gbuffer_texel {
    float position[3];
    float depth;
    float normal[3];
    int32_t prim_id;             /* == MatId == instance index (scene.cpp:531-533) */
    float smooth_normal[3];
    int32_t tri_id;              /* BLAS triangle index (new field, -1 on miss) */
    float albedo[3];
    int32_t hit;                 /* optional engaged */
    float uv[2];
    float dpdu[3];
    float dpdv[3];
} hdr_gbuffer_texel;

/* ---------------------------------------------------------------------------
 * Context
 * ------------------------------------------------------------------------- */
/* hdr_ctx_desc.flags */
#define HDR_CTX_TIMINGS 1u        /* record per-pass CUDA-event timings (hdr_pass_times) */
#define HDR_CTX_WIDE_BVH 2u      /* walk the 4-wide collapse of the reference's binary trees
                                    instead of the trees node by node (identical results; for
                                    A/B timing) */
#define HDR_CTX_LANE_PER_RAY 8u  /* wavefront trace kernels keep each lane on one ray until it is
                                    done instead of refilling idle lanes (for A/B timing) */
#define HDR_CTX_PT_ONE_KERNEL 32u /* PathTracePass in one thread per pixel (rays cast on the spot)
                                     instead of the wavefront form; same image (for A/B checks) */
#define HDR_CTX_UNPHASED 16u     /* wavefront trace kernels step each lane's whole walk every
                                    iteration instead of serving leaves, instance entries and ray
                                    starts in their own phases (for A/B timing) */
#define HDR_CTX_SPLIT_STACK 64u  /* phased binary walk keeps its deeper stack entries in local
                                    memory even when the scene's trees are shallow enough for a
                                    shared-memory-only stack; same results (for A/B checks) */
#define HDR_CTX_DEVICE_BUILD 128u /* hdr_scene_upload builds each mesh's BVH (BVH::Build,
                                     renderContext/bvh.cpp:66-208) and triangle records on the
                                     device instead of the host: the same trees, node order and
                                     triangle order, bit for bit. Binary trees only: not with
                                     HDR_CTX_WIDE_BVH, and the scene cannot be shared into a
                                     wide-walk ctx. Its scratch (about 0.5 KB per triangle while
                                     building) is outside the ctx's HBM budget. */
#define HDR_CTX_REFERENCE_SHADOWS 512u /* every ray walks the reference's own trees instead of the
                                     4-wide SAH trees built at upload over the same triangles
                                     (shadow queries: the closest-hit walk stopped below the light
                                     distance). The answers agree: the same triangle test in the
                                     same instance space, conservative boxes, and closest-hit ties
                                     broken in the reference's walk order. */
#define HDR_CTX_SAH_CLOSEST 1024u /* closest hits walk the 4-wide SAH trees (ties broken in the
                                     reference's walk order) WITHOUT the check below: the
                                     reference's answer except where the reference's own rounded
                                     box tests cull the nearest hit (coplanar surfaces): about 1e-3
                                     of random rays in config 1's scene, 5e-6 in config 2's.
                                     By default closest hits also walk the SAH trees, and each
                                     hit is checked against the reference walk: every box on the
                                     way down to it in the reference's own trees must pass the
                                     reference's slab test no farther than the hit; a ray that
                                     fails the check walks the reference's trees. The answer is
                                     then the reference's bit for bit. */
#define HDR_CTX_REFERENCE_CLOSEST 2048u /* closest hits walk the reference's trees only (for A/B
                                     checks; same answers as the default) */
#define HDR_CTX_RECORD_LIGHTS 256u /* diagnostic, no reference counterpart: the wavefront
                                     hdr_ris_path_trace records the light index each NEE candidate
                                     selected (UniformLightSampler::ProposeCandidate,
                                     lighting_core/uniform_light_sampler.cpp:22-35; -1 where the
                                     proposal failed or the pixel has no hit) in
                                     "__ris_nee_lights": width*height x (candidate_count/2, at least
                                     1) int32, pixel-major. Not recorded by batched or one-kernel
                                     frames. */

typedef struct hdr_ctx_desc {
    int32_t device;              /* CUDA ordinal */
    uint32_t flags;              /* HDR_CTX_* bits */
    size_t hbm_budget_bytes;     /* 0 = unlimited; allocations past it fail with HDR_ENOMEM */
} hdr_ctx_desc;

/* Replaces the LightRHI device/kernel setup of Gpu::AccumulationKernel
 * (gpu_functions/gpu_accumulation_kernel.cpp:63-192) for all passes. */
hdr_status hdr_ctx_create(hdr_ctx **out, const hdr_ctx_desc *desc);
void hdr_ctx_destroy(hdr_ctx *ctx);
int hdr_abi_version(void);
/* Thread-local text of the last failure on this thread ("" if none). */
const char *hdr_last_error(void);

/* HdRestirMaterial::Sync's network walk (hydra/hd_restir_material.cpp:22-424), host only:
 * from the surface terminal ("mtlx:surface", else "surface", else "outputs:surface",
 * else the first by name) every upstream node once, depth first, inputs and parameters
 * in name order; UsdPreviewSurface, standard_surface and open_pbr_surface parameters set
 * the PreviewSurface fields (diffuse = base_color x base weight for the MaterialX
 * surfaces), image nodes give the texture slot of the surface input their chain starts
 * from. out starts from the PreviewSurfaceParams defaults (a material's first Sync); its
 * texture pointers stay NULL: textures (may be NULL) receives the asset paths, which the
 * host decodes into out->textures. */
hdr_status hdr_material_from_network(const hdr_mtl_network *net, hdr_material_desc *out,
                                     hdr_mtl_textures *textures);

/* Uploads and builds the device scene: BLAS per mesh (BVH::Build,
 * renderContext/bvh.cpp:66-241), instances and TLAS (Scene::_BuildTLAS,
 * scene/scene.cpp:333-407), materials, lights, dome CDF (DomeLight::Prepare,
 * scene/dome_light.cpp:21-83). Replaces the per-frame Scene::BuildRenderState:
 * the scene stays resident until the next upload. */
hdr_status hdr_scene_upload(hdr_ctx *ctx, const hdr_scene_desc *scene);

/* No reference counterpart (the reference builds a Scene per delegate). dst
 * renders src's resident scene without a second copy in HBM; both must be on
 * one device. The memory lives until the last context holding it uploads
 * another scene or is destroyed. Required for hdr_ris_path_trace_batch. */
hdr_status hdr_scene_share(hdr_ctx *dst, hdr_ctx *src);

/* Moved instances: HdRestirMesh::Sync taking a dirty transform
 * (hydra/hd_restir_mesh.cpp:160-162) followed by the TLAS rebuild of
 * Scene::BuildRenderState (scene/scene.cpp:118-244, 333-407), on the device.
 * `transforms` holds num_instances row-major 4x4 floats (the layout of
 * hdr_instance_desc.transform), in device memory when transforms_on_device is
 * non-zero (read on the ctx stream), else host memory. The instance records and
 * the binary TLAS are rebuilt in place: the images equal those of a fresh
 * hdr_scene_upload with these transforms, bit for bit. num_instances must be the
 * uploaded scene's; the ctx must walk the binary trees (no HDR_CTX_WIDE_BVH) and
 * hold the scene alone (not shared through hdr_scene_share), and afterwards the
 * scene cannot be shared into a wide-walk ctx. Synchronises the ctx stream (the
 * new TLAS depth sizes the traversal stack). A TLAS too deep for the traversal
 * stack fails with HDR_EINVAL and leaves the ctx without a scene. */
hdr_status hdr_scene_set_instance_transforms(hdr_ctx *ctx, const float *transforms, int32_t num_instances,
                                             int32_t transforms_on_device);

/* No reference counterpart (inspection and tests): a copy of one of the resident
 * scene's device arrays, by its DeviceScene field name ("blas_nodes", "tri_geo",
 * "tri_attr", "instances", "tlas_nodes", "tlas_inst", "materials", "lights", ...).
 * *size (if not NULL) receives the array's bytes; with dst NULL nothing is copied,
 * else bytes must equal that size. */
hdr_status hdr_scene_array(hdr_ctx *ctx, const char *name, void *dst, size_t bytes, size_t *size);

/* RaycastPass::_execute (passes/raycast_pass.cpp:57-162): GBuffer (+AOVs). */
hdr_status hdr_raycast(hdr_ctx *ctx, const hdr_camera *cam, int32_t frame_index, uint32_t aov_mask);

/* RISPathTracePass (restir_passes/ris_path_trace_pass.h:12-28) = IntegrationPass::_execute
 * (passes/integration_pass.cpp:157-252) with PathIntegrator + RisDirectLightIntegrator:
 * reads GBuffer and "__ris_reservoir", writes "Color" and the reservoirs. */
hdr_status hdr_ris_path_trace(hdr_ctx *ctx, const hdr_camera *cam, int32_t frame_index,
                              const hdr_ris_params *params);

/* Batched RISPathTracePass, no reference counterpart: n images (one ctx each,
 * all sharing one resident scene through hdr_scene_share, each after its own
 * hdr_raycast) in one wavefront frame. Every image's generate kernel appends
 * its rays to one queue, one closest-hit and one shadow launch trace them all,
 * then each image is resampled into its own "Color" and "__ris_reservoir".
 * Each image's results are those of hdr_ris_path_trace on its ctx. Images
 * that cannot take the wavefront form (max_depth > 1, non-opaque scene,
 * HDR_RIS_ONE_KERNEL) or do not share the scene are rendered one after
 * another instead. The work runs on ctxs[0]'s stream; the other ctxs' streams
 * are ordered before and after it. A context may appear only once. The shared
 * ray queues and result slots belong to the resident scene (grow-only, outside
 * the contexts' HBM budgets), so batches of changing images allocate nothing once
 * they are large enough; batches on one scene are ordered by an event. */
hdr_status hdr_ris_path_trace_batch(hdr_ctx *const *ctxs, int32_t n, const hdr_camera *cams,
                                    const int32_t *frame_indices, const hdr_ris_params *params);

/* Batched PathTracePass, no reference counterpart: n images (one ctx each,
 * sharing one resident scene, each after its own hdr_raycast) in one launch
 * over all their tiles. Each image's "Color" is that of hdr_path_trace on its
 * ctx. Images that do not share the scene are rendered one after another.
 * With one set of path settings for all images and an opaque scene, every
 * wavefront round traces all images' live paths together. The path planes,
 * ray queues and job table belong to the resident scene, like the RIS batch's
 * queues (grow-only, outside the contexts' HBM budgets; batches on one scene
 * ordered by an event); the call does not wait for the device. */
hdr_status hdr_path_trace_batch(hdr_ctx *const *ctxs, int32_t n, const hdr_camera *cams,
                                const int32_t *frame_indices, const hdr_path_settings *settings);

/* ---------------------------------------------------------------------------
 * Render-job server (no reference counterpart; the reference renders one job
 * per Hydra delegate). Scenes are uploaded once and shared; jobs are admitted
 * first-in first-out while the estimate of their frame buffers fits the HBM
 * budget; each hdr_server_step advances admitted jobs by one frame (all of
 * them, or up to step_pixels of them by priority: least remaining work, less
 * a credit that grows with the work served since the job arrived), with the
 * RIS jobs of one scene traced in one batched launch and path-traced jobs
 * side by side on their own streams. Accumulation follows GpuAccumulationPass
 * (HDR_ACCUM_SHADER). HDR_SERVER_SERIAL runs one job at a time, each frame
 * alone (the plain per-frame pipeline). A job's image is the
 * same in both modes. Calls on one server are serialised by its mutex.
 * ------------------------------------------------------------------------- */
typedef struct hdr_server hdr_server;
#define HDR_SERVER_SERIAL 1u

typedef struct hdr_server_desc {
    int32_t device;
    uint32_t flags;            /* HDR_SERVER_* */
    size_t hbm_budget_bytes;   /* admission budget for the jobs' frame buffers, 0 = unlimited */
    int32_t max_batch;         /* images per batched RIS launch, 0 = 64 */
    int64_t step_pixels;       /* pixels rendered per step, 0 = every admitted job; the jobs with the
                                  lowest key go first: remaining work (frames left x pixels) less
                                  age_weight x the pixels the server rendered since the job's submission */
    float age_weight;          /* 0 = 0.5; negative = no credit (least remaining work first). The credit
                                  keeps early large jobs from waiting behind every later small one */
} hdr_server_desc;

enum { HDR_JOB_PATH_TRACER = 0, HDR_JOB_RIS = 1 };
enum { HDR_JOB_QUEUED = 0, HDR_JOB_RUNNING = 1, HDR_JOB_DONE = 2, HDR_JOB_FAILED = 3 };

typedef struct hdr_job_desc {
    int32_t scene;             /* id from hdr_server_add_scene */
    int32_t pipeline;          /* HDR_JOB_PATH_TRACER or HDR_JOB_RIS */
    int32_t frames;            /* frames to accumulate (samples per pixel), >= 1 */
    int32_t firefly;           /* AccumulationPass firefly filter */
    hdr_camera camera;         /* static over the job's frames */
    hdr_ris_params ris;        /* RIS settings; ris.path also configures the PathTracer pipeline */
} hdr_job_desc;

hdr_status hdr_server_create(hdr_server **out, const hdr_server_desc *desc);
void hdr_server_destroy(hdr_server *server);
hdr_status hdr_server_add_scene(hdr_server *server, const hdr_scene_desc *scene, int32_t *scene_id);
hdr_status hdr_server_submit(hdr_server *server, const hdr_job_desc *job, int64_t *job_id);
/* Admits what fits, renders one frame of every admitted job, and returns the
 * number of jobs that finished (DONE or FAILED) in this step. */
hdr_status hdr_server_step(hdr_server *server, int32_t *jobs_finished);
hdr_status hdr_server_job_state(hdr_server *server, int64_t job_id, int32_t *state, int32_t *frames_done);
/* Copies a finished job's "Color" (width*height RGBA f32; rgba may be NULL to
 * discard it) and frees the job. */
hdr_status hdr_server_take_result(hdr_server *server, int64_t job_id, float *rgba, size_t bytes);
/* Up to cap ids of jobs that finished (DONE or FAILED) since the last call. */
hdr_status hdr_server_drain_finished(hdr_server *server, int64_t *ids, int32_t cap, int32_t *n);
hdr_status hdr_server_load(hdr_server *server, int32_t *queued, int32_t *running, size_t *bytes_in_use);

/* PathTracePass (passes/path_trace_pass.h:12-39) with MisDirectLightIntegrator. */
hdr_status hdr_path_trace(hdr_ctx *ctx, const hdr_camera *cam, int32_t frame_index,
                          const hdr_path_settings *settings);

/* AccumulationPass::_execute (passes/accumulation_pass.cpp:64-139) and
 * GpuAccumulationPass (accumulation.slang:39-97): optional firefly clamp,
 * "__accum_color" += "Color", "Color" = accum / (frame_index+1). Enqueued on the
 * ctx stream; neither mode reads back or waits (parity mode checks the in-place
 * order and, where it differs, clamps in that order, all on the device). */
hdr_status hdr_accumulate(hdr_ctx *ctx, int32_t frame_index, int32_t firefly, int32_t mode);

/* No reference counterpart. hdr_accumulate on caller-owned device planes
 * (color, accum: width*height RGBA f32, 16-byte aligned, on the current
 * device) that allocates nothing: the firefly scratch is a fixed static device
 * array (32 MiB, held on every GPU that loads it until the process exits,
 * outside any HBM budget), so frames above 2,097,152 pixels with firefly != 0
 * are rejected (HDR_EINVAL). For callers that may not allocate device memory
 * while they accumulate. The first call on a device (and in a new context on
 * it) resolves the scratch's address (make it before any stream capture);
 * accum must be zero before frame 0; calls that overlap on one device race on
 * the shared scratch. Neither mode reads back or waits for the stream.
 * stream: a cudaStream_t (NULL = default). */
hdr_status hdr_accumulate_noalloc(float *color, float *accum, int32_t width, int32_t height, int32_t frame_index,
                                  int32_t firefly, int32_t mode, void *stream);

/* RenderPipeline::ClearPersistentBuffers (pipeline/render_pipeline.cpp:42-45):
 * zeroes "__accum_color" and "__ris_reservoir". */
hdr_status hdr_clear_persistent(hdr_ctx *ctx);

/* Copies a named device buffer to host memory (bytes must equal the buffer size,
 * query it with hdr_buffer_size). Names: "GBuffer" (hdr_gbuffer_texel),
 * "Color" (RGBA f32), "Depth" (f32), "Albedo"/"Normal" (RGB f32),
 * "__accum_color" (RGBA f32), "__ris_reservoir" (5 planes of width*height
 * float4: light dir + dist, light colour + pdf, light normal + target
 * function, throughput, then WSum, W, candidate count and flag bits). */
hdr_status hdr_download(hdr_ctx *ctx, const char *name, void *dst, size_t bytes);
/* hdr_download without waiting (no reference counterpart): the buffer as the ctx stream has it
 * now is copied to dst (pinned host memory for the copy to overlap) on a separate copy stream,
 * while later passes run. dst may be read after hdr_download_wait; a second call first lets the
 * previous copy finish on the device. Not for "GBuffer". */
hdr_status hdr_download_async(hdr_ctx *ctx, const char *name, void *dst, size_t bytes);
/* Waits for the last hdr_download_async; later work on the ctx stream is ordered after it. */
hdr_status hdr_download_wait(hdr_ctx *ctx);

/* Component formats of a Hydra render buffer (HdFormat component types). */
enum { HDR_FMT_FLOAT32 = 0, HDR_FMT_FLOAT16 = 1, HDR_FMT_UNORM8 = 2, HDR_FMT_SNORM8 = 3, HDR_FMT_INT32 = 4 };
/* HdRestirRenderBuffer::CopyFromFrameBuffer (hydra/hd_restir_render_buffer.cpp:46-73,113-148)
 * on the device: the named float frame buffer (src_components floats per pixel: "Color" 4,
 * "Depth" 1, "Albedo" / "Normal" 3) into dst_components components of component_format per
 * pixel. As in the reference, a source pixel of the destination pixel's size is copied as
 * bytes; otherwise each component is converted as _WriteOutput does (components the source
 * lacks are 0). (For a multi-component source of another size the reference's conversion
 * stops at a precondition of FrameBuffer::As; here it converts component by component.) dst is device memory on this ctx's GPU when dst_on_device
 * (ordered on the ctx stream; hdr_synchronize waits for it), else host memory (filled
 * before the call returns). dst_bytes must be exactly the converted image's size. */
hdr_status hdr_resolve(hdr_ctx *ctx, const char *name, int32_t src_components, int32_t component_format,
                       int32_t dst_components, void *dst, size_t dst_bytes, int32_t dst_on_device);

/* UpscalePass::_execute (passes/upscale_pass.cpp:13-95) on one named float buffer of this ctx:
 * its src_w x src_h pixels of `components` floats (the frame's RenderedWidth/Height at its
 * resolution level) become dst_w x dst_h (the window), each taking the source pixel
 * (min(src_w - 1, x * src_w / dst_w), min(src_h - 1, y * src_h / dst_h)). The buffer keeps its
 * name at the new size. */
hdr_status hdr_upscale(hdr_ctx *ctx, const char *name, int32_t components, int32_t src_w, int32_t src_h,
                       int32_t dst_w, int32_t dst_h);
/* Denoiser::Run without OIDN (passes/denoiser.cpp:54-96,164-201) on the named RGBA float buffer
 * of width x height pixels, in place: with chromaticity_blur, each pixel keeps its luma and takes
 * the 3x3 mean chroma; alpha is kept. chromaticity_blur = 0 leaves the image as it is, like the
 * reference without OIDN. */
hdr_status hdr_denoise(hdr_ctx *ctx, const char *name, int32_t width, int32_t height, int32_t chromaticity_blur);
hdr_status hdr_upload(hdr_ctx *ctx, const char *name, const void *src, size_t bytes);
hdr_status hdr_buffer_size(hdr_ctx *ctx, const char *name, size_t *bytes);
/* hdr_clear_persistent without giving the memory back (no reference counterpart): the
 * persistent buffers are zeroed in stream order, which a freshly created buffer also is, so the
 * next frame starts without history. No device-wide synchronisation (cudaFree has one). */
hdr_status hdr_zero_persistent(hdr_ctx *ctx);

/* Waits for all work queued on the ctx stream. */
hdr_status hdr_synchronize(hdr_ctx *ctx);

/* Host-visible cancel word polled between launches and by long device loops
 * (the IRenderJob::IsCancelled poll of scene.cpp:422-423). NULL detaches. */
hdr_status hdr_set_cancel(hdr_ctx *ctx, const volatile int32_t *flag);

/* Scene::IntersectScene (scene.cpp:515-535) on caller rays: rays = n x
 * (ox,oy,oz,dx,dy,dz) f32 host array; out = n x hdr_gbuffer_texel.
 * any_hit != 0: the shadow query "closest hit nearer than tmax" (per-ray
 * limit, NULL = +inf) as the passes cast it; only `hit` is meaningful. */
hdr_status hdr_trace_rays(hdr_ctx *ctx, const float *rays, const float *tmax, int32_t n,
                          int32_t any_hit, hdr_gbuffer_texel *out);

/* Schedule of the wavefront trace kernels (no reference counterpart; no effect
 * on results). node_quorum: node steps continue while this many lanes of a
 * warp step nodes (1..32); blocks_per_sm: persistent blocks per SM (1..64).
 * trace_ms: device time of the two trace kernels (autotune output).
 * shade_shape: launch shape of the resampling kernel: 0 = 256 threads with the
 * register file of one block per SM, 1 (default) = 256 threads for two blocks,
 * 2 / 3 = 128 threads for three / four blocks (no effect on results).
 * shadow_shape: register budget of the shadow-BVH walk kernel: 0 = 64 registers
 * (8 resident blocks of 128 threads), 1 (default) = 80 (6 blocks), 2 = 90 (5 blocks). */
typedef struct hdr_trace_tuning {
    int32_t node_quorum;
    int32_t blocks_per_sm;
    float trace_ms;
    int32_t shade_shape;
    int32_t shadow_shape;
    float shade_ms;         /* hdr_autotune_frame: the resampling kernel's time at shade_shape */
} hdr_trace_tuning;
hdr_status hdr_get_trace_tuning(hdr_ctx *ctx, hdr_trace_tuning *out);
hdr_status hdr_set_trace_tuning(hdr_ctx *ctx, const hdr_trace_tuning *tuning);
/* Autotuner: reruns the trace kernels of the last wavefront hdr_ris_path_trace
 * (they only read its ray queues and rewrite the same hit / occlusion slots)
 * over a grid of schedules (node quorum x blocks per SM, and the shadow-BVH
 * walk's register budget), keeps the fastest in the ctx and returns it. */
hdr_status hdr_autotune_trace(hdr_ctx *ctx, hdr_trace_tuning *best);
/* Autotuner over a whole frame: renders one hdr_ris_path_trace frame in the
 * wavefront form (max_depth 1, opaque scene, no HDR_RIS_ONE_KERNEL; else
 * HDR_EINVAL) and tunes while it renders. After the generate kernel has filled
 * the ray queues, the trace kernels run once per trace schedule (as
 * hdr_autotune_trace), then the resampling kernel runs once per launch shape,
 * each time from a copy of the reservoirs it merges into and with the winner
 * queue emptied. Every run writes the same bytes, so the frame's buffers are
 * those of hdr_ris_path_trace. The fastest schedule and shape stay in the ctx
 * and are returned in *best (may be NULL) with their times. The closest-hit
 * queue needs no tuning: it holds a slot only for the rays the frame casts
 * (none when BSDF-candidate rays cannot change the image). Takes about 150
 * trace runs and 8 resampling runs; synchronises the ctx stream. */
hdr_status hdr_autotune_frame(hdr_ctx *ctx, const hdr_camera *cam, int32_t frame_index,
                              const hdr_ris_params *params, hdr_trace_tuning *best);

/* Diagnostic, no reference counterpart: the work one traversal form does per
 * ray. walk: 0 closest hit on the binary trees, 1 closest hit on their 4-wide
 * collapse, 2 shadow query on the binary trees, 3 shadow query on the 4-wide
 * collapse, 4 shadow query on the 4-wide SAH trees, 5 closest hit on them
 * (for 4 and 5: stack entries popped, leaves and instances entered, triangles
 * tested). out = n x int32[4]: nodes popped, leaves entered, triangles tested,
 * answer (hit / occluded). */
hdr_status hdr_trace_stats(hdr_ctx *ctx, const float *rays, const float *tmax, int32_t n, int32_t walk,
                           int32_t *out);

/* Restir::Rng (core/rng.h:10-56) on the device: for each seed, the first
 * `count` NextFloat() values of std::mt19937_64(seed) mapped through
 * uniform_real_distribution<float>. out = n_seeds x count floats. */
hdr_status hdr_rng_floats(hdr_ctx *ctx, const uint32_t *seeds, int32_t n_seeds, int32_t count,
                          float *out);

/* Average device time (ms) and number of calls of each pass since the last
 * reset, measured with CUDA events on the ctx stream when flag bit 0 is set
 * (the replacement for the reference's METRICS_ENABLED pass timers,
 * core/metrics_on_buffers.h): [0] raycast, [1] integrate, [2] accumulate,
 * and for the wavefront form of hdr_ris_path_trace its kernels [3] generate,
 * [4] trace closest, [5] trace shadow, [6] shade (n <= 7).
 * reset != 0 clears the sums after reading them. */
hdr_status hdr_pass_times(hdr_ctx *ctx, float *avg_ms, int32_t *counts, int32_t n, int32_t reset);

/* Device-time regions on the ctx stream (4 slots): begin records a start event,
 * end records a stop event; hdr_region_elapsed waits for the stop event and
 * returns the milliseconds between them. */
hdr_status hdr_region_begin(hdr_ctx *ctx, int32_t slot);
hdr_status hdr_region_end(hdr_ctx *ctx, int32_t slot);
hdr_status hdr_region_elapsed(hdr_ctx *ctx, int32_t slot, float *ms);

/* Number of this library's kernels launched on the ctx so far. */
hdr_status hdr_launch_count(hdr_ctx *ctx, uint64_t *count);

/* No reference counterpart. Frame buffers (and the batch calls' queues) come from
 * one stream-ordered memory pool per device, so allocating and freeing them never
 * synchronises the device; freed memory stays in the pool for later frames. This
 * returns the pool's unused memory beyond keep_bytes to the device (it waits for
 * work that frees memory; call it between jobs, not per frame). */
hdr_status hdr_trim_frame_memory(int32_t device, size_t keep_bytes);

/* ---------------------------------------------------------------------------
 * A frame's pass chain as one CUDA graph. No reference counterpart: the
 * reference's RenderPipeline::Execute (pipeline/render_pipeline.cpp:24-40)
 * calls its passes one by one, and the calls here do the same by default.
 *
 * Between hdr_graph_begin and hdr_graph_end the pass calls on ctx
 * (hdr_raycast, hdr_ris_path_trace, hdr_path_trace, hdr_accumulate,
 * hdr_zero_persistent, hdr_denoise, hdr_resolve into device memory) are
 * recorded from the ctx stream instead of run: they check their arguments,
 * update the ctx's host-side state (frame size, reprojection history) and
 * return. The recorded passes must render one frame index; their kernels read
 * it from device memory, so the record replays for any frame.
 * hdr_graph_end makes the record the ctx's executable graph: the first one is
 * instantiated, a later one with the same launches (other camera or parameter
 * values) updates it in place (cudaGraphExecUpdate), and one with other
 * launches replaces it. hdr_graph_launch(ctx, frame_index) stores frame_index
 * (-1: the recorded one) where the recorded kernels read it and runs the graph
 * on the ctx stream: the results are those of the recorded calls made eagerly
 * with that frame index, every other argument (camera included) as recorded.
 * So a static camera's progressive frames are recorded once and replayed with
 * two launches per frame; a moving camera records each frame again.
 *
 * While recording: every buffer a recorded pass uses must already exist at its
 * size (run the same passes once eagerly first), else the pass fails with
 * HDR_EINVAL; pass timing (flag bit 0) is not taken; calls that wait for the
 * device, copy to or from the host, allocate or free (hdr_download*,
 * hdr_upload, hdr_synchronize, hdr_region_*, hdr_pass_times, hdr_scene_*,
 * hdr_clear_persistent, hdr_upscale, the batch calls, hdr_trace_*,
 * hdr_autotune_trace, hdr_rng_floats, hdr_graph_launch) fail with HDR_EINVAL and
 * leave the recording intact. A recorded pass that fails marks the recording,
 * and hdr_graph_end then discards it (HDR_EINVAL) and keeps the previous graph.
 * hdr_ctx_destroy drops an unfinished recording. */
hdr_status hdr_graph_begin(hdr_ctx *ctx);
hdr_status hdr_graph_end(hdr_ctx *ctx);
hdr_status hdr_graph_launch(hdr_ctx *ctx, int32_t frame_index);
/* The executable graph's kernel launches per replay, and how many times
 * hdr_graph_end instantiated a graph and updated one in place (any may be NULL). */
hdr_status hdr_graph_info(hdr_ctx *ctx, int32_t *kernels, int32_t *instantiations, int32_t *updates);

#ifdef __cplusplus
}
#endif
#endif /* HDRESTIR_B200_H */
