// Device frame-buffer views shared by the pass kernels and their launchers.
// Every per-pixel buffer is a structure of float4 planes so a warp's loads and
// stores are 16-byte vectors over consecutive pixels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "camera.cuh"
#include "traverse.cuh"

namespace hdr {

// "GBuffer" (std::optional<HitRecord> per pixel, raycast_pass.cpp:60-61)
struct GBufferView {
    float4 *pos_depth;    // position.xyz, depth
    float4 *normal_prim;  // normal.xyz, prim id bits (-1 = no hit)
    float4 *smooth_tri;   // smooth normal.xyz, triangle id bits
    float4 *albedo_uv;    // albedo.xyz, uv.x
    float4 *aux0;         // uv.y, dpdu.xyz
    float4 *aux1;         // dpdv.xyz, 0
};

struct AovView {       // optional RaycastPass AOVs
    float *depth;      // f32 x P   (miss = 1)
    float *albedo;     // f32x3 x P (miss = 0)
    float *normal;     // f32x3 x P (miss = 0)
};

// Persistent "__ris_reservoir": WeightedReservoir<RISLightCandidate> per pixel
// (restir/reservoir.h:69-161, ris_direct_light_integrator.h:26-43).
struct ReservoirView {
    float4 *dir_dist;       // Ls.Dir.xyz, Ls.Dist
    float4 *color_pdf;      // Ls.Color.xyz, Ls.Pdf.value
    float4 *normal_phat;    // Ls.LightNormal.xyz, targetFunction
    float4 *throughput;     // Throughput (4 wavelengths)
    float4 *wsum_w_m_meta;  // WSum, W, CandidateCount bits, meta bits
};
// meta bits
constexpr unsigned kResHasSample = 1u << 0;     // ChosenSample engaged
constexpr unsigned kResHasCandidate = 1u << 1;  // ChosenSample->Candidate engaged
constexpr unsigned kResVisTested = 1u << 2;     // VisibilityTested
constexpr unsigned kResPdfSolidAngle = 1u << 3; // Ls.Pdf.space == SolidAngle
constexpr unsigned kResOriginShift = 4;         // CandidateOrigin (2 bits)
constexpr unsigned kResLightShift = 8;          // light index (24 bits)

// Temporal reuse across camera motion (extension, no reference counterpart;
// the reference's renderer resets its reservoirs when the camera moves). Mode 0
// is the reference's same-pixel reuse; mode 1 takes the history from where the
// pixel's hit point was in the previous frame's image; mode 2 has no history.
struct ReprojD {
    int mode;
    int width, height;         // previous frame's image
    double view[16], proj[16];  // previous frame's camera (GfMatrix4d row-major)
    const float4 *prev_pos;    // previous frame's GBuffer position.xyz, depth
    ReservoirView prev;        // previous frame's reservoirs
};

struct RisParamsD {
    int candidate_count;
    int use_reservoir;
    int skip_visibility;
    int max_depth;
    int enable_subsurface;
    int max_refl, max_refr;
    int render_ibl_background;
    float roulette;
    int m_cap;
    int spatial_neighbors;
    float spatial_radius;
    ReprojD reproj;
};

// PathTracePassSettings + maxDepth as the integrators read them
// (integrators/path_integrator.h:12-19)
struct PathRun {
    int max_depth;
    bool enable_subsurface;
    int max_refl, max_refr;
    bool render_ibl_background;
    float roulette;
};

struct PathParamsD {
    int max_depth;
    int enable_subsurface;
    int max_refl, max_refr;
    int render_ibl_background;
    float roulette;
};

// Scratch of the wavefront RISPathTracePass (per frame, not persistent).
struct WaveBuffers {
    float4 *q_closest;    // 2 per entry: origin.xyz + slot bits | direction.xyz
    float4 *q_shadow;     // 2 per entry: origin.xyz + slot bits | direction.xyz + distance limit
    int *counts;          // [0] closest-hit queue length, [1] shadow queue length (8 ints)
    int *fix;             // one per closest-hit queue entry: entries whose checked SAH hit the reference walk
                          // redoes (nullptr exactly when the queue has no entries)
    float4 *hits;         // pixels * n_closest: t, instance bits, triangle bits, u
    float *hit_v;         // pixels * n_closest
    unsigned char *occ;   // pixels * n_shadow
    uint4 *rng_state;     // 3 planes of pixels: stream state at the end of candidate generation
    unsigned char *done;  // pixels: 1 = no GBuffer hit, colour already written
    size_t pixels;
    int n_closest, n_shadow;
    // added to the result slots the generate kernel writes into the queues: a
    // batch of images shares one queue and one result array (0 for one image,
    // whose hits / hit_v / occ then start at its own slot 0)
    int slot_base_closest, slot_base_shadow;
    // winner visibility queued for the shadow kernel instead of cast on the spot
    // (nullptr: on the spot): 2 float4 per entry like q_shadow, slot = pixel;
    // counts[4] entries queued, counts[5] handed out; answers in occ_winner[pixel]
    float4 *q_winner;
    unsigned char *occ_winner;
    // diagnostic (nullptr: off): pixels * n_shadow light indices the NEE
    // candidates selected (UniformLightSampler::ProposeCandidate), -1 where the
    // proposal failed or the pixel has no hit
    int *nee_light;
};

// Returns the number of kernels launched, or -1 on a launch error.
// How the wavefront trace kernels run. mode: kTraceLanePerRay keeps each lane
// on one ray until it is done (default: lanes take the next queued ray as soon
// as theirs is finished); kTraceUnphased steps every lane's whole walk each
// iteration instead of serving leaves, instance entries and ray starts in
// separate phases; kTraceSplitStack keeps the binary walk's split shared/local
// stack on scenes shallow enough for the shared-memory-only one. node_quorum: the phased kernels keep stepping nodes while
// this many lanes of a warp do. Grid: sm_count x blocks_per_sm persistent blocks.
constexpr int kTraceLanePerRay = 1, kTraceUnphased = 2, kTraceSplitStack = 4;
constexpr int kShadowShapes = 3;
struct TraceTuning {
    int mode = 0;
    int node_quorum = 12;  // best for the SAH-tree walks (16 for the reference-tree ones)
    int blocks_per_sm = 16;
    int sm_count = 148;
    int shade_shape = 1;  // ris_shade launch shape, 0 .. kShadeShapes - 1 (256 x 2: fastest at 1080p)
    int shadow_shape = 1; // shadow-BVH walk register budget, 0 .. kShadowShapes - 1: 64 / 80 / 90 registers
};
// ris_shade launch shapes: (threads per block, minimum resident blocks per SM)
// = (256, 1), (256, 2), (128, 3), (128, 4)
constexpr int kShadeShapes = 4;
// The trace kernels over the queues of the last ris_generate: closest hits, then
// shadow queries; with checked SAH closest hits (s.sh4_closest == 2) also the
// check and the reference walk of the entries it rejected (counts[6..7], wb.fix).
// They read the queue counts and reset nothing but their own fetch counters' use,
// so the caller zeroes counts[2..3] before a rerun; returns the launches, -1 on error.
// The shadow-ray queue q over the shadow BVH when the scene has it (s.sh4), else the
// phased walk of the reference trees; *count rays, *fetch the hand-out counter.
int launch_shadow_queue(const DeviceScene &s, const float4 *q, const int *count, int *fetch, unsigned char *occ,
                        const TraceTuning &tune, unsigned *err, cudaStream_t st);
int launch_wave_trace(const DeviceScene &s, WaveBuffers wb, const TraceTuning &tune, unsigned *err, cudaStream_t st,
                      cudaEvent_t *ev_begin = nullptr, cudaEvent_t *ev_end = nullptr);
// Spatial reuse (extension, spatial.cu): merges up to p.spatial_neighbors
// neighbours' reservoirs of `in` into `out` and rewrites the colour. With a
// winner queue (q_winner, counts[4]) the shadow rays of moved samples are
// queued for launch_winner_visibility instead of cast in the kernel.
int launch_ris_spatial(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                       GBufferView gb, ReservoirView in, ReservoirView out, float4 *color, float4 *q_winner,
                       int *winner_count, unsigned *err, cudaStream_t st);
// The queued winner shadow rays (wb.q_winner, counts[4] / [5]) traced, then the
// pixels found occluded fixed up in rv and color.
int launch_winner_visibility(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                             GBufferView gb, ReservoirView rv, WaveBuffers wb, float4 *color, unsigned *err,
                             cudaStream_t st, const TraceTuning &tune);
// Render-buffer conversion (resolve.cu): kResolve* are the HDR_FMT_* values.
constexpr int kResolveFloat32 = 0, kResolveFloat16 = 1, kResolveUNorm8 = 2, kResolveSNorm8 = 3, kResolveInt32 = 4;
int launch_resolve(const float *src, int src_comps, int format, int dst_comps, void *dst, size_t pixels,
                   int sm_count, cudaStream_t st);
// Post passes (post.cu): UpscalePass's nearest-pixel upscale and the
// Denoiser's chromaticity blur.
int launch_upscale(const float *src, float *dst, int comps, int src_w, int src_h, int dst_w, int dst_h, int sm_count,
                   cudaStream_t st);
int launch_chroma_blur(const float4 *src, float4 *dst, int w, int h, int sm_count, cudaStream_t st);
// Moved instances (tlas.cu): the n instance records rewritten from the n row-major
// transforms xf (device memory), their world boxes and centres into bounds (9
// floats each), then the binary TLAS rebuilt into tlas_nodes / tlas_inst as the
// host scene builder builds it. info (device, 4 ints): nodes, maximum depth,
// capacity overflow, an empty visited box. Returns the launches, -1 on error.
int launch_tlas_rebuild(const float *xf, float4 *instances, const float *mesh_ranges, float *bounds, int n,
                        float4 *tlas_nodes, int cap_nodes, int *tlas_inst, int4 *stack, int cap_stack, int *info,
                        cudaStream_t st);
// Which closest-hit rays of a pixel the wavefront RIS pass casts (trace_level).
// Without light geometry and environment no generated BSDF candidate can
// contribute, and without emissive materials either, neither can the
// connection candidate (the path's bounce ray): their weights are the same
// whatever the rays hit, so those rays are not cast.
constexpr int kTraceNoBsdfRays = 0, kTraceBounceRay = 1, kTraceAllBsdfRays = 2;
// The three stages of the wavefront RIS pass on their own (a batch of images
// runs every image's generate, one trace over their shared queues, then every
// image's shade). Return the launches, -1 on a launch error.
int launch_ris_generate(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                        GBufferView gb, WaveBuffers wb, float4 *color, int trace_level, unsigned *err,
                        cudaStream_t st);
int launch_ris_shade(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                     GBufferView gb, ReservoirView rv, WaveBuffers wb, float4 *color, int trace_level, unsigned *err,
                     cudaStream_t st, const TraceTuning &tune);
// ev_begin / ev_end (4 events each, or null): recorded around the generate,
// trace-closest, trace-shadow and shade launches for per-kernel device times.
int launch_ris_wavefront(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                         GBufferView gb, ReservoirView rv, WaveBuffers wb, float4 *color, int trace_level,
                         unsigned *err, cudaStream_t st, const TraceTuning &tune, cudaEvent_t *ev_begin = nullptr,
                         cudaEvent_t *ev_end = nullptr);
// The same launchers with the closures' texture overrides compiled in
// (wavefront_tex.cu); the ones above leave them out, for scenes without textures.
namespace textured {
int launch_shadow_queue(const DeviceScene &s, const float4 *q, const int *count, int *fetch, unsigned char *occ,
                        const TraceTuning &tune, unsigned *err, cudaStream_t st);
int launch_wave_trace(const DeviceScene &s, WaveBuffers wb, const TraceTuning &tune, unsigned *err, cudaStream_t st,
                      cudaEvent_t *ev_begin = nullptr, cudaEvent_t *ev_end = nullptr);
int launch_winner_visibility(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                             GBufferView gb, ReservoirView rv, WaveBuffers wb, float4 *color, unsigned *err,
                             cudaStream_t st, const TraceTuning &tune);
int launch_ris_generate(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                        GBufferView gb, WaveBuffers wb, float4 *color, int trace_level, unsigned *err,
                        cudaStream_t st);
int launch_ris_shade(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                     GBufferView gb, ReservoirView rv, WaveBuffers wb, float4 *color, int trace_level, unsigned *err,
                     cudaStream_t st, const TraceTuning &tune);
int launch_ris_wavefront(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                         GBufferView gb, ReservoirView rv, WaveBuffers wb, float4 *color, int trace_level,
                         unsigned *err, cudaStream_t st, const TraceTuning &tune, cudaEvent_t *ev_begin = nullptr,
                         cudaEvent_t *ev_end = nullptr);
}  // namespace textured

void launch_raycast(const DeviceScene &s, const CameraD &cam, int frame_index, GBufferView gb, AovView aov,
                    unsigned *err, cudaStream_t st);
void launch_trace_rays(const DeviceScene &s, const float *rays, const float *tmax, int n, int any_hit,
                       float4 *out /* 6 float4 per ray: hdr_gbuffer_texel */, unsigned *err, cudaStream_t st);
void launch_trace_stats(const DeviceScene &s, const float *rays, const float *tmax, int n, int mode, int4 *out,
                        unsigned *err, cudaStream_t st);
void launch_rng_floats(const uint32_t *seeds, int n, int count, float *out, cudaStream_t st);
void launch_ris_path_trace(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                           GBufferView gb, ReservoirView res, float4 *color, unsigned *err, cudaStream_t st);
// Per-path state of the wavefront PathTracePass (pathtrace.cu), one entry
// per pixel, plus its ray queues and hit slots (slot = pixel index).
struct PtBuffers {
    uint4 *rng;             // 3 planes: stream state between kernels
    float4 *tp, *total;     // throughput and running radiance of _li (4 wavelengths)
    float4 *outer;          // PathIntegrator::Li's throughput (primary Beer), applied at the end
    float4 *ray_o, *ray_d;  // the current vertex's incoming ray; ray_o.w: the wavelength draw
    float4 *b_origin_pdf, *b_dir, *b_tmul;  // the vertex's BSDF sample
    float4 *nee_add;        // the vertex's NEE term, added if its shadow ray is unoccluded
    int4 *state;            // BounceState refl, refr; flags; spare
    int *active[2];         // live-path lists (ping-pong)
    int *counts;            // [0..3] queue lengths and fetch counters, [4..5] active-list lengths
    int *fix;               // WaveBuffers::fix of the closest-hit queue
    float4 *q_closest, *q_shadow, *hits;
    float *hit_v;
    unsigned char *occ;
    size_t pixels;
};

// One image of a batched PathTracePass launch (a table in device memory).
struct PtJobD {
    CameraD cam;
    GBufferView gb;
    float4 *color;
    unsigned *err;
    PathRun pr;
    int frame_index;
    int tile_begin;    // first tile of this image in the batch grid
    int pixel_begin;   // first path of this image in the wavefront planes
};
PathRun path_run_of(const PathParamsD &p);
// Wavefront PathTracePass over n images (jobs[k].tile_begin / pixel_begin
// laid out by the caller; all with the same PathRun). One image: the job goes
// by value and `table` may be null; several: `table` is a device copy of jobs.
int launch_path_trace_wavefront(const DeviceScene &s, const PtJobD *jobs, int n_jobs, const PtJobD *table,
                                int total_tiles, PtBuffers B, const TraceTuning &tune, unsigned *err,
                                cudaStream_t st);
void launch_path_trace_batch(const DeviceScene &s, const PtJobD *jobs, int n_jobs, int total_tiles,
                             cudaStream_t st);
void launch_path_trace(const DeviceScene &s, const CameraD &cam, int frame_index, const PathParamsD &p,
                       GBufferView gb, float4 *color, unsigned *err, cudaStream_t st);
// Returns the number of kernels launched, or -1 with the CUDA error in *err.
// frame_slot (non-null in a pass recorded into a graph) holds the frame index.
int launch_accumulate(float4 *color, float4 *accum, float4 *scratch, int *flag_dev, int width, int height,
                      int frame_index, int firefly, int mode, cudaStream_t st, cudaError_t *err,
                      const int *frame_slot = nullptr);

// Pixel of thread t in a 16x16 tile: each warp covers an 8x4 sub-tile so the
// rays it traces start close together.
template <int kThreads = 256>
__device__ __forceinline__ bool tile_pixel(int width, int height, int &x, int &y, int tile = -1) {
    constexpr int kTileH = kThreads / 16;  // tiles 16 pixels wide, one 8x4 patch per warp
    const int tiles_x = (width + 15) >> 4;
    if (tile < 0) tile = blockIdx.x;
    const int tx = tile % tiles_x, ty = tile / tiles_x;
    const int t = threadIdx.x;
    const int w = t >> 5, lane = t & 31;
    x = (tx << 4) + ((w & 1) << 3) + (lane & 7);
    y = ty * kTileH + ((w >> 1) << 2) + (lane >> 3);
    return x < width && y < height;
}
template <int kThreads = 256>
inline int tile_blocks(int width, int height) {
    constexpr int kTileH = kThreads / 16;
    return ((width + 15) >> 4) * ((height + kTileH - 1) / kTileH);
}

}  // namespace hdr
