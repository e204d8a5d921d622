// C ABI of the device passes (declared in include/hdrestir.h).
//
// One hdr_ctx owns a CUDA stream, the resident device scene and the named
// device frame buffers. The reference moves its named host buffers in and out
// of a FrameBuffersMap per pipeline run (core/frame_buffer_map.cpp:76-101);
// here the same names stay resident on the GPU and only cross to the host on
// hdr_download / hdr_upload.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hdrestir.h"
#include "device/blas_build.h"
#include "device/frame.cuh"
#include "device/sky.cuh"
#include "host/scene_build.h"
#include "host/shadow_bvh.h"

namespace {

thread_local std::string g_last_error;

hdr_status fail(hdr_status st, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

#define HDR_CUDA(call)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(HDR_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));       \
    } while (0)

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
};

// Stores the frame index a recorded graph renders (hdr_graph_launch); the
// recorded kernels read it from the slot.
__global__ void set_frame_slot_kernel(int *slot, int value) { *slot = value; }

}  // namespace

namespace hdr {
// Sets hdr_last_error() for entry points defined in other translation units.
hdr_status set_last_error(hdr_status st, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}
}  // namespace hdr

// The device memory of one uploaded scene. Contexts hold it by shared_ptr so
// several can render the same resident scene (hdr_scene_share); the memory is
// freed when the last holder lets go, after that holder's stream is idle.
struct SceneStore {
    int device = 0;
    std::vector<void *> ptrs;
    size_t bytes = 0;
    // the scene descriptor in device memory: [wide + 2 * sh4 + 4 * sh4_closest] (binary / wide
    // walk of the reference trees; shadow and closest-hit queries on the 4-wide SAH trees)
    const hdr::DeviceScene *desc_dev = nullptr;
    // hdr_scene_set_instance_transforms: what the device rebuild of the instances and the TLAS needs
    int num_instances = 0, max_blas_depth = 0;
    int tlas_capacity = 0;          // TLAS nodes the upload reserved (4 per instance)
    bool blas_proper = true;        // no BLAS node box is empty (the TLAS is checked at each build)
    bool wide_stale = false;        // the wide TLAS no longer matches the binary one
    float *mesh_ranges = nullptr;   // 6 floats per mesh
    float *inst_bounds = nullptr;   // 9 floats per instance: world box, centre
    float *xf_staging = nullptr;    // 16 floats per instance
    int4 *tlas_stack = nullptr;     // num_instances + 2 entries
    int *tlas_info = nullptr;       // 4 ints
    // shadow-ray BVH (host/shadow_bvh.h): present when sh4 is true; the TLAS part is
    // rebuilt on the host when instances move
    bool sh4 = false;
    // the reference trees' parent links for exact SAH closest hits (closest_mode 2); they
    // describe the uploaded TLAS, so moving instances on the device clears this
    bool ref_links = false;
    std::vector<int> sh4_inst_root;
    int sh4_tlas_capacity = 0, sh4_blas_depth = 0;
    // the scene's arrays by DeviceScene field name, for hdr_scene_array
    std::map<std::string, std::pair<const void *, size_t>> arrays;
    // hdr_ris_path_trace_batch's shared ray queues and result slots: one grow-only set per
    // resident scene, whichever context leads a batch, so batches of changing images (a
    // server's steps) allocate nothing once the set is large enough. batch_done orders the
    // batches that use it across the leads' streams.
    std::mutex batch_mu;
    std::map<std::string, std::pair<void *, size_t>> batch_bufs;
    cudaEvent_t batch_done = nullptr;
    // hdr_path_trace_batch's path planes, queues and job table likewise ("pt_*" in batch_bufs,
    // batches ordered by pt_done); the job table goes up from one of two pinned host buffers,
    // each reused once its last copy (pt_copied) has run
    cudaEvent_t pt_done = nullptr;
    void *pt_table_host[2] = {nullptr, nullptr};
    size_t pt_table_cap[2] = {0, 0};
    cudaEvent_t pt_copied[2] = {nullptr, nullptr};
    int pt_slot = 0;
    ~SceneStore() {
        if (ptrs.empty() && batch_bufs.empty()) return;
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        for (cudaEvent_t ev : {batch_done, pt_done, pt_copied[0], pt_copied[1]})
            if (ev) {
                cudaEventSynchronize(ev);
                cudaEventDestroy(ev);
            }
        for (void *h : pt_table_host)
            if (h) cudaFreeHost(h);
        // pool memory (stream-ordered); every batch that used it has finished (events above)
        for (auto &kv : batch_bufs) cudaFreeAsync(kv.second.first, nullptr);
        for (void *p : ptrs) cudaFree(p);
        cudaSetDevice(prev);
    }
};

// timing slots: 0 raycast, 1 integrate, 2 accumulate, then the wavefront
// kernels 3 ris_generate, 4 trace_closest, 5 trace_shadow, 6 ris_shade
constexpr int kTimeSlots = 7;
constexpr int kSlotWaveFirst = 3;

struct hdr_ctx {
    int device = 0;
    uint32_t flags = 0;
    size_t budget = 0;
    size_t allocated = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;

    // resident scene (scene_store owns the memory; the fields below describe it)
    std::shared_ptr<SceneStore> scene_store;
    size_t scene_bytes_accounted = 0;  // part of `allocated` this ctx uploaded for its scene
    hdr::DeviceScene scene{};
    bool has_scene = false;
    bool scene_opaque = true;          // every material has opacity >= 0.999 (no stochastic pass-through)
    bool scene_light_geometry = false; // some instance is a light's geometry (GetLightAtHit can succeed)
    bool scene_emissive = false;       // some material emits
    // camera of the last RIS frame with HDR_RIS_REPROJECT (its hit points are in "__prev_pos_depth")
    bool reproj_valid = false;
    int reproj_w = 0, reproj_h = 0;
    double reproj_view[16] = {}, reproj_proj[16] = {};

    // named frame buffers
    std::map<std::string, DevBuf> buffers;
    int width = 0, height = 0;

    unsigned *d_err = nullptr;
    int *d_flag = nullptr;
    // per timing slot (raycast, integrate, accumulate, then the four wavefront
    // kernels): one start/stop event pair; the previous pair is folded into the
    // running sums when the slot is reused
    cudaEvent_t ev_start[kTimeSlots] = {};
    cudaEvent_t ev_stop[kTimeSlots] = {};
    bool ev_pending[kTimeSlots] = {};
    double pass_sum_ms[kTimeSlots] = {};
    int pass_count[kTimeSlots] = {};
    float pass_last_ms[kTimeSlots] = {};
    cudaEvent_t region_ev[4][2] = {};
    const volatile int32_t *cancel = nullptr;
    uint64_t launches = 0;
    // wavefront trace schedule, and the queues of the last wavefront frame (for hdr_autotune_trace)
    hdr::TraceTuning tune;
    hdr::WaveBuffers last_wave{};
    bool have_wave = false;
    cudaEvent_t sync_ev = nullptr;  // orders this ctx's stream against a batch's lead stream
    // hdr_download_async: a snapshot of the buffer on the ctx stream, copied to the host on a
    // copy stream while the ctx stream goes on (created at the first call)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_ready = nullptr, copy_done = nullptr;
    // hdr_graph_begin / hdr_graph_end / hdr_graph_launch: while `recording`, the pass calls
    // are captured from the ctx stream instead of run; graph_exec is the executable chain
    bool recording = false;
    bool rec_failed = false;      // a pass failed while recording: its work is missing from the record
    uint64_t rec_launches0 = 0;   // `launches` when the recording began
    // the recorded passes read their frame index from d_frame_slot (device memory), which
    // hdr_graph_launch sets; every pass of one recording renders the same frame index
    int *d_frame_slot = nullptr;
    bool rec_has_frame = false, graph_has_frame = false;
    int32_t rec_frame = 0, graph_frame = 0;
    uint64_t graph_kernels = 0;   // kernel launches one replay of graph_exec makes
    cudaGraphExec_t graph_exec = nullptr;
    int32_t graph_instantiations = 0, graph_updates = 0;
    // hdr_autotune_frame: the wavefront RIS frame in progress searches the trace schedules and
    // resampling launch shapes, reporting into tune_out
    bool tune_frame = false;
    hdr_trace_tuning *tune_out = nullptr;
};

namespace {

hdr_status dev_alloc(hdr_ctx *c, DevBuf &b, size_t bytes) {
    if (c->budget && c->allocated + bytes > c->budget)
        return fail(HDR_ENOMEM, "allocation of %zu bytes exceeds the HBM budget (%zu of %zu in use)", bytes,
                    c->allocated, c->budget);
    void *p = nullptr;
    if (bytes) {
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) return fail(HDR_ENOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
    b.ptr = p;
    b.bytes = bytes;
    c->allocated += bytes;
    return HDR_OK;
}

void dev_free(hdr_ctx *c, DevBuf &b) {
    if (b.ptr) cudaFree(b.ptr);
    c->allocated -= b.bytes;
    b = DevBuf{};
}

// Frame buffers and batch buffers come from one stream-ordered memory pool per
// device (cudaMallocFromPoolAsync / cudaFreeAsync): allocating or freeing one
// orders itself on a stream and never synchronises the device, which cudaMalloc
// and cudaFree may (a server creating and retiring job contexts would otherwise
// stall every job in flight). Freed memory stays mapped in the pool for the next
// allocations (no release threshold): giving physical memory back at a
// synchronisation point waits for the device, which stalled a server's steps for
// up to 0.7 s. hdr_trim_frame_memory returns it; the pools live until the process
// exits.
cudaMemPool_t frame_pool(int device) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[device] = p;
    return p;
}

// A frame buffer of ctx c, allocated and freed in order on the ctx stream (another
// stream that uses it is ordered after the ctx stream's work and before its later work).
hdr_status frame_alloc(hdr_ctx *c, DevBuf &b, size_t bytes) {
    if (c->budget && c->allocated + bytes > c->budget)
        return fail(HDR_ENOMEM, "allocation of %zu bytes exceeds the HBM budget (%zu of %zu in use)", bytes,
                    c->allocated, c->budget);
    void *p = nullptr;
    if (bytes) {
        cudaMemPool_t pool = frame_pool(c->device);
        if (!pool) return fail(HDR_ECUDA, "cannot create the frame-buffer memory pool on device %d", c->device);
        const cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, c->stream);
        if (e != cudaSuccess) return fail(HDR_ENOMEM, "frame buffer of %zu bytes: %s", bytes, cudaGetErrorString(e));
    }
    b.ptr = p;
    b.bytes = bytes;
    c->allocated += bytes;
    return HDR_OK;
}

void frame_free(hdr_ctx *c, DevBuf &b) {
    if (b.ptr) cudaFreeAsync(b.ptr, c->stream);
    c->allocated -= b.bytes;
    b = DevBuf{};
}

// FrameBuffersMap::Add / AddOrGetPersistent: create (zeroed) or resize keeping
// the prefix; a same-size request returns the existing buffer untouched.
hdr_status ensure_buffer(hdr_ctx *c, const char *name, size_t bytes, void **out) {
    auto it = c->buffers.find(name);
    if (it != c->buffers.end() && it->second.bytes == bytes) {
        *out = it->second.ptr;
        return HDR_OK;
    }
    if (c->recording)
        return fail(HDR_EINVAL, "buffer '%s' does not exist at %zu bytes: a recorded pass cannot allocate (run the "
                    "same passes once outside hdr_graph_begin / hdr_graph_end first)", name, bytes);
    DevBuf nb;
    hdr_status st = frame_alloc(c, nb, bytes);
    if (st != HDR_OK) return st;
    if (bytes) HDR_CUDA(cudaMemsetAsync(nb.ptr, 0, bytes, c->stream));
    if (it != c->buffers.end()) {
        const size_t keep = std::min(bytes, it->second.bytes);
        if (keep) HDR_CUDA(cudaMemcpyAsync(nb.ptr, it->second.ptr, keep, cudaMemcpyDeviceToDevice, c->stream));
        HDR_CUDA(cudaStreamSynchronize(c->stream));
        frame_free(c, it->second);
        it->second = nb;
    } else {
        c->buffers[name] = nb;
    }
    *out = nb.ptr;
    return HDR_OK;
}

// Per-frame scratch: reused while large enough, replaced (not copied) when it
// must grow; every frame writes what it reads, so contents are not kept.
hdr_status ensure_scratch(hdr_ctx *c, const char *name, size_t bytes, void **out) {
    auto it = c->buffers.find(name);
    if (it != c->buffers.end() && it->second.bytes >= bytes) {
        *out = it->second.ptr;
        return HDR_OK;
    }
    if (c->recording)
        return fail(HDR_EINVAL, "scratch '%s' is smaller than %zu bytes: a recorded pass cannot allocate (run the "
                    "same passes once outside hdr_graph_begin / hdr_graph_end first)", name, bytes);
    if (it != c->buffers.end()) {
        HDR_CUDA(cudaStreamSynchronize(c->stream));
        frame_free(c, it->second);
        c->buffers.erase(it);
    }
    DevBuf nb;
    hdr_status st = frame_alloc(c, nb, std::max<size_t>(bytes, 16));
    if (st != HDR_OK) return st;
    c->buffers[name] = nb;
    *out = nb.ptr;
    return HDR_OK;
}

// A batch buffer of the scene store (batch_mu held): kept while large enough; grown
// with a quarter of headroom. The old one is freed and the new one allocated in
// order on `stream` (the batch's lead stream), after `done` (the event every batch
// using the buffer records): no host wait and no device synchronisation. Its bytes
// count toward the scene's memory.
hdr_status ensure_batch_scratch(SceneStore *store, const char *name, size_t bytes, void **out,
                                cudaEvent_t done, cudaStream_t stream) {
    auto it = store->batch_bufs.find(name);
    if (it != store->batch_bufs.end() && it->second.second >= bytes) {
        *out = it->second.first;
        return HDR_OK;
    }
    if (it != store->batch_bufs.end()) {
        if (done) HDR_CUDA(cudaStreamWaitEvent(stream, done, 0));
        HDR_CUDA(cudaFreeAsync(it->second.first, stream));
        store->bytes -= it->second.second;
        store->batch_bufs.erase(it);
    }
    const size_t want = std::max<size_t>(16, bytes + bytes / 4);
    void *p = nullptr;
    cudaMemPool_t pool = frame_pool(store->device);
    if (!pool) return fail(HDR_ECUDA, "cannot create the frame-buffer memory pool on device %d", store->device);
    const cudaError_t e = cudaMallocFromPoolAsync(&p, want, pool, stream);
    if (e != cudaSuccess) return fail(HDR_ENOMEM, "batch buffer of %zu bytes: %s", want, cudaGetErrorString(e));
    store->batch_bufs[name] = {p, want};
    store->bytes += want;
    *out = p;
    return HDR_OK;
}

void *find_buffer(hdr_ctx *c, const char *name, size_t *bytes) {
    auto it = c->buffers.find(name);
    if (it == c->buffers.end()) return nullptr;
    if (bytes) *bytes = it->second.bytes;
    return it->second.ptr;
}

hdr_status check_cancel(hdr_ctx *c) {
    if (c->cancel && *c->cancel) return fail(HDR_ECANCELLED, "render job cancelled");
    return HDR_OK;
}

// Calls that wait for the device, read back to the host, allocate or free, or
// order other streams cannot be recorded into a graph: they fail while the ctx
// records (checked before they touch the stream, so the recording stays valid).
hdr_status check_not_recording(const hdr_ctx *c, const char *what) {
    if (c->recording)
        return fail(HDR_EINVAL, "%s cannot run while the ctx records a graph (between hdr_graph_begin and "
                    "hdr_graph_end)", what);
    return HDR_OK;
}
#define HDR_NOT_RECORDING(c, what)                                   \
    do {                                                             \
        hdr_status s_ = check_not_recording((c), (what));            \
        if (s_ != HDR_OK) return s_;                                 \
    } while (0)

// A pass recorded into a graph renders the recording's frame index, read from the
// ctx's frame slot at run time (so hdr_graph_launch can replay it for any frame):
// the first recorded pass fixes that index, the others must give the same one.
hdr_status record_frame_index(hdr_ctx *c, int32_t frame_index, hdr::CameraD *cam) {
    if (!c->recording) return HDR_OK;
    if (c->rec_has_frame && c->rec_frame != frame_index)
        return fail(HDR_EINVAL, "recorded passes render one frame index (%d), not %d", c->rec_frame, frame_index);
    c->rec_has_frame = true;
    c->rec_frame = frame_index;
    if (cam) cam->frame_slot = c->d_frame_slot;
    return HDR_OK;
}

hdr_status check_camera(const hdr_camera *cam) {
    if (!cam) return fail(HDR_EINVAL, "camera is NULL");
    if (cam->width <= 0 || cam->height <= 0 || (int64_t)cam->width * cam->height > (int64_t)1 << 28)
        return fail(HDR_EINVAL, "bad frame size %dx%d", cam->width, cam->height);
    return HDR_OK;
}

// RenderContext camera -> device: inverses as the passes compute them
// (raycast_pass.cpp:86-87), exposure as GetExposureMultiplier (camera_params.h:22-31).
hdr::CameraD make_camera(const hdr_camera *cam) {
    hdr::CameraD d{};
    hdr::gf_inverse4d(cam->view, d.inv_view);
    hdr::gf_inverse4d(cam->proj, d.inv_proj);
    d.width = cam->width;
    d.height = cam->height;
    d.p.has_params = cam->has_params;
    d.p.enable_dof = cam->enable_dof;
    d.p.enable_exposure = cam->enable_exposure;
    d.p.focal_length = cam->focal_length;
    d.p.f_stop = cam->f_stop;
    d.p.focus_distance = cam->focus_distance;
    d.p.bokeh_blades = cam->bokeh_blades;
    d.p.lens_distortion = cam->lens_distortion;
    d.p.iso = cam->iso;
    d.p.shutter_speed = cam->shutter_speed;
    float mult = 1.0f;
    if (cam->has_params && cam->enable_exposure) {
        const float safe = std::max(cam->f_stop, 0.1f);
        mult = (cam->iso / 100.0f) * cam->shutter_speed / (safe * safe) * 100.0f;
    }
    d.p.exposure_mult = mult;
    return d;
}

constexpr size_t kGbPlanes = 6;
constexpr size_t kResPlanes = 5;

hdr_status gbuffer_view(hdr_ctx *c, size_t count, bool create, hdr::GBufferView &gb) {
    void *p = nullptr;
    if (create) {
        hdr_status st = ensure_buffer(c, "GBuffer", count * kGbPlanes * sizeof(float4), &p);
        if (st != HDR_OK) return st;
    } else {
        size_t bytes = 0;
        p = find_buffer(c, "GBuffer", &bytes);
        if (!p || bytes != count * kGbPlanes * sizeof(float4))
            return fail(HDR_EINVAL, "GBuffer must be present (produced by RaycastPass) for %zu pixels", count);
    }
    float4 *b = (float4 *)p;
    gb = hdr::GBufferView{b, b + count, b + 2 * count, b + 3 * count, b + 4 * count, b + 5 * count};
    return HDR_OK;
}

hdr_status fold_pass_time(hdr_ctx *c, int slot) {
    if (!c->ev_pending[slot]) return HDR_OK;
    HDR_CUDA(cudaEventSynchronize(c->ev_stop[slot]));
    float ms = 0.0f;
    HDR_CUDA(cudaEventElapsedTime(&ms, c->ev_start[slot], c->ev_stop[slot]));
    c->pass_last_ms[slot] = ms;
    c->pass_sum_ms[slot] += ms;
    c->pass_count[slot] += 1;
    c->ev_pending[slot] = false;
    return HDR_OK;
}
// Pass timing (HDR_CTX_TIMINGS) waits for the slot's previous events, so it is
// not taken while passes are being recorded into a graph.
bool timing_on(const hdr_ctx *c) { return (c->flags & 1u) && !c->recording && !c->tune_frame; }
hdr_status begin_pass(hdr_ctx *c, int slot) {
    if (timing_on(c)) {
        hdr_status st = fold_pass_time(c, slot);
        if (st != HDR_OK) return st;
        HDR_CUDA(cudaEventRecord(c->ev_start[slot], c->stream));
    }
    return HDR_OK;
}
hdr_status end_pass(hdr_ctx *c, int slot) {
    HDR_CUDA(cudaGetLastError());
    if (timing_on(c)) {
        HDR_CUDA(cudaEventRecord(c->ev_stop[slot], c->stream));
        c->ev_pending[slot] = true;
    }
    return HDR_OK;
}

hdr_status read_device_error(hdr_ctx *c) {
    unsigned e = 0;
    HDR_CUDA(cudaMemcpyAsync(&e, c->d_err, sizeof(e), cudaMemcpyDeviceToHost, c->stream));
    HDR_CUDA(cudaStreamSynchronize(c->stream));
    if (e) {
        HDR_CUDA(cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), c->stream));
        return fail(HDR_EDEVICE, "device traversal stack limit reached (error bits 0x%x)", e);
    }
    return HDR_OK;
}

}  // namespace

extern "C" {

int hdr_abi_version(void) { return HDR_ABI_VERSION; }

const char *hdr_last_error(void) { return g_last_error.c_str(); }

hdr_status hdr_ctx_create(hdr_ctx **out, const hdr_ctx_desc *desc) {
    if (!out) return fail(HDR_EINVAL, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    HDR_CUDA(cudaGetDeviceCount(&ndev));
    const int dev = desc ? desc->device : 0;
    if (dev < 0 || dev >= ndev) return fail(HDR_EINVAL, "device %d not present (%d devices)", dev, ndev);
    if (desc && (desc->flags & HDR_CTX_DEVICE_BUILD) && (desc->flags & HDR_CTX_WIDE_BVH))
        return fail(HDR_EINVAL, "HDR_CTX_DEVICE_BUILD builds the binary trees only (no HDR_CTX_WIDE_BVH)");
    HDR_CUDA(cudaSetDevice(dev));
    hdr_ctx *c = new hdr_ctx();
    c->device = dev;
    c->flags = desc ? desc->flags : 0;
    c->budget = desc ? desc->hbm_budget_bytes : 0;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    cudaMemPool_t pool = e == cudaSuccess ? frame_pool(dev) : nullptr;
    if (e == cudaSuccess && !pool) e = cudaErrorMemoryAllocation;
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(&c->d_err, 64, pool, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_err, 0, 64, c->stream);
    for (int k = 0; k < kTimeSlots && e == cudaSuccess; ++k) {
        e = cudaEventCreate(&c->ev_start[k]);
        if (e == cudaSuccess) e = cudaEventCreate(&c->ev_stop[k]);
    }
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
        e = cudaEventCreate(&c->region_ev[k][0]);
        if (e == cudaSuccess) e = cudaEventCreate(&c->region_ev[k][1]);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->sync_ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        hdr_ctx_destroy(c);
        return fail(HDR_ECUDA, "context setup: %s", cudaGetErrorString(e));
    }
    c->d_flag = (int *)((char *)c->d_err + 32);
    c->d_frame_slot = (int *)((char *)c->d_err + 48);
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0)
        c->tune.sm_count = sms;
    c->tune.mode = ((c->flags & HDR_CTX_LANE_PER_RAY) ? hdr::kTraceLanePerRay : 0) |
                   ((c->flags & HDR_CTX_UNPHASED) ? hdr::kTraceUnphased : 0) |
                   ((c->flags & HDR_CTX_SPLIT_STACK) ? hdr::kTraceSplitStack : 0);
    *out = c;
    return HDR_OK;
}

void hdr_ctx_destroy(hdr_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->recording) {  // an unfinished recording is dropped
        cudaGraph_t g = nullptr;
        if (cudaStreamEndCapture(c->stream, &g) == cudaSuccess && g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
        c->recording = false;
    }
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);  // a read-back may still use a buffer
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    c->scene_store.reset();
    for (auto &kv : c->buffers) frame_free(c, kv.second);
    if (c->d_err) cudaFreeAsync(c->d_err, c->stream);
    for (int k = 0; k < kTimeSlots; ++k) {
        if (c->ev_start[k]) cudaEventDestroy(c->ev_start[k]);
        if (c->ev_stop[k]) cudaEventDestroy(c->ev_stop[k]);
    }
    for (auto &pair : c->region_ev)
        for (auto &e : pair)
            if (e) cudaEventDestroy(e);
    if (c->sync_ev) cudaEventDestroy(c->sync_ev);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->copy_ready) cudaEventDestroy(c->copy_ready);
    if (c->copy_done) cudaEventDestroy(c->copy_done);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

namespace {
// True when no node box of the flat scene's BLAS trees is empty (min > max on an axis).
bool empty_box(const float *lo, const float *hi) { return lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]; }
bool wide_boxes_proper(const std::vector<float> &w) {
    for (size_t k = 0; k + hdr::kWideNodeFloats <= w.size(); k += hdr::kWideNodeFloats) {
        const float *n = w.data() + k;
        for (int j = 0; j < 4; ++j) {
            int code;
            std::memcpy(&code, &n[24 + j], sizeof(code));
            const float lo[3] = {n[j], n[4 + j], n[8 + j]}, hi[3] = {n[12 + j], n[16 + j], n[20 + j]};
            if (code >= 0 && empty_box(lo, hi)) return false;
        }
    }
    return true;
}
bool blas_boxes_proper(const hdr::FlatScene &f) {
    for (size_t k = 0; k + 8 <= f.blas_nodes.size(); k += 8)
        if (empty_box(&f.blas_nodes[k], &f.blas_nodes[k + 4])) return false;
    if (!wide_boxes_proper(f.blas4)) return false;
    for (size_t k = 0; k + 8 <= f.blas_roots.size(); k += 8) {
        int code;
        std::memcpy(&code, &f.blas_roots[k + 3], sizeof(code));
        if (code >= 0 && empty_box(&f.blas_roots[k], &f.blas_roots[k + 4])) return false;
    }
    return true;
}
// The same for the TLAS, over the nodes a walk can reach: the two children
// every TLAS leaf allocates (scene.cpp:344-349) keep their default empty boxes
// but are never visited.
bool tlas_boxes_proper(const hdr::FlatScene &f) {
    if (f.tlas_nodes.empty()) return true;
    std::vector<int> todo{0};
    while (!todo.empty()) {
        const int n = todo.back();
        todo.pop_back();
        const float *rec = &f.tlas_nodes[8 * (size_t)n];
        if (empty_box(rec, rec + 4)) return false;
        int left;
        std::memcpy(&left, &rec[3], sizeof(left));
        if (left < 0) continue;
        todo.push_back(left);
        todo.push_back(left + 1);
    }
    if (!wide_boxes_proper(f.tlas4)) return false;
    int root;
    std::memcpy(&root, &f.tlas_root[3], sizeof(root));
    return !(root >= 0 && empty_box(&f.tlas_root[0], &f.tlas_root[4]));
}
}  // namespace

namespace {
// Parent links of the reference trees, for checking a closest hit found on the
// 4-wide SAH trees against the reference's own walk (exact SAH closest hits):
// per TLAS node its parent, per instance its TLAS leaf, per BLAS node (all meshes,
// mesh-local indices) its parent, per triangle record its mesh-local leaf. Only
// nodes a walk can reach are linked (-1 elsewhere). Needs the host-built trees.
// The check's path records: per TLAS node and per BLAS node, 8 floats (32 B, one
// sector): the node's box min, its parent's index bits (-1 at a root), its box max, 0.
struct RefLinks {
    std::vector<float> tlas_path, blas_path;
    std::vector<int> inst_leaf, tri_leaf;
};
void set_path_record(std::vector<float> &path, size_t n, const float *rec, int parent) {
    float *p = &path[8 * n];
    p[0] = rec[0];
    p[1] = rec[1];
    p[2] = rec[2];
    std::memcpy(&p[3], &parent, sizeof(int));
    p[4] = rec[4];
    p[5] = rec[5];
    p[6] = rec[6];
    p[7] = 0.0f;
}
int float_bits(float v) {
    int i;
    std::memcpy(&i, &v, sizeof(i));
    return i;
}
// The TLAS half of the links: a path record per node (n_tlas of the 8-float nodes)
// and each instance's leaf, from a walk of the tree as it is now. False when the
// tree does not fit the records or names an instance outside the scene.
bool tlas_links(const float *nodes, size_t n_tlas, const int *tlas_inst, size_t n_tlas_inst, int num_instances,
                std::vector<float> &path, std::vector<int> &inst_leaf) {
    std::vector<int> parent(n_tlas, -1);
    inst_leaf.assign((size_t)num_instances, -1);
    std::vector<int> todo{0};
    while (!todo.empty()) {
        const int n = todo.back();
        todo.pop_back();
        const float *rec = &nodes[8 * (size_t)n];
        const int left = float_bits(rec[3]), count = float_bits(rec[7]);
        if (left >= 0) {
            for (int ch : {left, left + 1}) {
                if ((size_t)ch >= n_tlas) return false;
                parent[(size_t)ch] = n;
                todo.push_back(ch);
            }
        } else {
            const int first = -left - 1;
            for (int k = 0; k < count; ++k) {
                if (first < 0 || (size_t)(first + k) >= n_tlas_inst) return false;
                const int ii = tlas_inst[(size_t)(first + k)];
                if (ii < 0 || ii >= num_instances) return false;
                inst_leaf[(size_t)ii] = n;
            }
        }
    }
    path.assign(8 * n_tlas, 0.0f);
    for (size_t n = 0; n < n_tlas; ++n) set_path_record(path, n, &nodes[8 * n], parent[n]);
    return true;
}
// blas_nodes: every mesh's BLAS nodes (8 floats each, the host build's or a copy of the device
// build's); n_tri: the triangle records.
bool build_ref_links(const hdr::FlatScene &f, const std::vector<float> &blas_nodes, size_t n_tri, RefLinks &L) {
    if (blas_nodes.empty() || f.tlas_nodes.empty() || f.num_instances <= 0) return false;
    const size_t n_tlas = f.tlas_nodes.size() / 8, n_blas = blas_nodes.size() / 8;
    std::vector<int> blas_parent(n_blas, -1);
    L.tri_leaf.assign(n_tri, -1);
    auto ibits = float_bits;
    if (!tlas_links(f.tlas_nodes.data(), n_tlas, f.tlas_inst.data(), f.tlas_inst.size(), f.num_instances, L.tlas_path,
                    L.inst_leaf))
        return false;
    std::vector<int> todo;
    std::vector<char> done_mesh(n_blas + 1, 0);
    for (int i = 0; i < f.num_instances; ++i) {  // each mesh's tree once, from its instances' bases
        const float *ir = &f.instances[32 * (size_t)i];
        const int node_base = ibits(ir[19]), tri_base = ibits(ir[23]), blas_ok = ibits(ir[29]);
        if (!blas_ok || node_base < 0 || (size_t)node_base >= n_blas || done_mesh[(size_t)node_base]) continue;
        done_mesh[(size_t)node_base] = 1;
        todo.assign(1, 0);
        while (!todo.empty()) {
            const int m = todo.back();
            todo.pop_back();
            const size_t g = (size_t)node_base + (size_t)m;
            if (g >= n_blas) return false;
            const float *rec = &blas_nodes[8 * g];
            const int left = ibits(rec[3]), count = ibits(rec[7]);
            if (left >= 0) {
                for (int ch : {left, left + 1}) {
                    if ((size_t)node_base + (size_t)ch >= n_blas) return false;
                    blas_parent[(size_t)node_base + (size_t)ch] = m;
                    todo.push_back(ch);
                }
            } else {
                const int first = -left - 1;
                for (int q = 0; q < count; ++q) {
                    const size_t t = (size_t)tri_base + (size_t)(first + q);
                    if (t >= n_tri) return false;
                    L.tri_leaf[t] = m;
                }
            }
        }
    }
    L.blas_path.assign(8 * n_blas, 0.0f);
    for (size_t n = 0; n < n_blas; ++n) set_path_record(L.blas_path, n, &blas_nodes[8 * n], blas_parent[n]);
    return true;
}

// The device copies of a scene descriptor, one per (wide, sh4, closest mode), each
// pointing at itself; a ctx's DeviceScene::dev is the copy of its own walk choices.
constexpr int kDescCopies = 12;
int desc_index(const hdr::DeviceScene &s) { return s.wide + 2 * s.sh4 + 4 * s.sh4_closest; }
void fill_desc_copies(const hdr::DeviceScene &s, const hdr::DeviceScene *base, hdr::DeviceScene *copies, bool sh4) {
    for (int w = 0; w < kDescCopies; ++w) {
        copies[w] = s;
        copies[w].wide = w & 1;
        copies[w].sh4 = (w >> 1) & (sh4 ? 1 : 0);
        copies[w].sh4_closest = copies[w].sh4 ? (w >> 2) : 0;
        copies[w].dev = base + w;
    }
}

// How closest hits walk (DeviceScene::sh4_closest): 0 the reference's trees, 1 the 4-wide
// SAH trees alone (HDR_CTX_SAH_CLOSEST), 2 the SAH trees with each hit checked against
// the reference walk's box tests (the default where the shadow BVH and the links exist;
// flags that select a form of the reference walk for A/B checks keep walk 0).
int closest_mode(uint32_t flags, bool sh4, bool links) {
    if (!sh4) return 0;
    if (flags & HDR_CTX_SAH_CLOSEST) return 1;
    const uint32_t reference_forms = HDR_CTX_REFERENCE_CLOSEST | HDR_CTX_WIDE_BVH | HDR_CTX_LANE_PER_RAY |
                                     HDR_CTX_UNPHASED | HDR_CTX_SPLIT_STACK;
    if (flags & reference_forms) return 0;
    return links ? 2 : 0;
}

// Which closest-hit rays the wavefront RIS pass casts (hdr::kTrace*).
int ris_trace_level(const hdr_ctx *c, const hdr_ris_params *p) {
    if ((p->flags & HDR_RIS_TRACE_ALL_RAYS) || c->scene_light_geometry || c->scene.env_light >= 0 || c->scene.sky)
        return hdr::kTraceAllBsdfRays;
    return c->scene_emissive ? hdr::kTraceBounceRay : hdr::kTraceNoBsdfRays;
}
// Closest-hit slots per pixel of the wavefront RIS queues: only the rays the trace
// level casts get one (the resampling kernel reads no other slot), so a frame whose
// BSDF-candidate rays cannot matter holds no closest-hit queue at all (1.8 GB at
// 1920x1080 with 16 BSDF candidates).
int closest_slots(int trace_level, int n_bsdf) {
    return trace_level >= hdr::kTraceAllBsdfRays ? 1 + n_bsdf : (trace_level >= hdr::kTraceBounceRay ? 1 : 0);
}
}  // namespace

hdr_status hdr_scene_upload(hdr_ctx *c, const hdr_scene_desc *desc) {
    if (!c || !desc) return fail(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_scene_upload");
    HDR_CUDA(cudaSetDevice(c->device));
    const bool device_build = (c->flags & HDR_CTX_DEVICE_BUILD) != 0;
    // HDR_CTX_DEVICE_BUILD: every mesh's BLAS and triangle records built on the device first
    std::vector<std::unique_ptr<hdr::DeviceBlasBuild>> dev_blas;
    std::vector<hdr::ExternalBlas> ext;
    bool dev_empty_box = false;
    if (device_build) {
        if (desc->num_meshes < 0) return fail(HDR_EINVAL, "negative count in hdr_scene_desc");
        for (int mi = 0; mi < desc->num_meshes; ++mi) {
            const hdr_mesh_desc &m = desc->meshes[mi];
            if ((m.num_points > 0 && !m.points) || (m.num_triangles > 0 && !m.indices) || (m.num_uvs > 0 && !m.uvs) ||
                (m.num_normals > 0 && !m.normals) || (m.num_colors > 0 && !m.colors))
                return fail(HDR_EINVAL, "mesh %d: NULL array with non-zero count", mi);
        }
        ext.resize((size_t)desc->num_meshes);
        for (int mi = 0; mi < desc->num_meshes; ++mi) {
            dev_blas.emplace_back(new hdr::DeviceBlasBuild);
            const cudaError_t e = dev_blas.back()->run(desc->meshes[mi], c->stream);
            if (e != cudaSuccess) return fail(HDR_ECUDA, "device BLAS build of mesh %d: %s", mi, cudaGetErrorString(e));
            const hdr::DeviceBlasResult &r = dev_blas.back()->result;
            ext[mi].num_nodes = r.num_nodes;
            ext[mi].num_tris = r.num_tris;
            ext[mi].max_depth = r.max_depth;
            dev_empty_box = dev_empty_box || r.empty_box;
        }
    }
    hdr::FlatScene f;
    std::string err;
    if (!hdr::build_flat_scene(*desc, f, err, device_build ? ext.data() : nullptr))
        return fail(HDR_EINVAL, "%s", err.c_str());
    // binary walk: one pending sibling per level of each tree, plus the two instance slots of a TLAS leaf
    if (f.max_blas_depth + f.max_tlas_depth + 4 > hdr::kTraceStack)
        return fail(HDR_EINVAL, "BVH depth %d + TLAS depth %d exceeds the device traversal stack (%d)",
                    f.max_blas_depth, f.max_tlas_depth, hdr::kTraceStack);
    // wide walk: at most three pending siblings per wide level, the root entry and a TLAS leaf's second instance
    if (3 * (f.max_blas4_depth + f.max_tlas4_depth) + 6 > hdr::kWideStack)
        return fail(HDR_EINVAL, "wide BVH depth %d + wide TLAS depth %d exceeds the device traversal stack (%d)",
                    f.max_blas4_depth, f.max_tlas4_depth, hdr::kWideStack);
    HDR_CUDA(cudaStreamSynchronize(c->stream));
    // this ctx lets go of its scene (another ctx sharing it keeps the memory alive)
    c->scene_store.reset();
    c->allocated -= c->scene_bytes_accounted;
    c->scene_bytes_accounted = 0;
    c->has_scene = false;
    c->have_wave = false;

    auto store = std::make_shared<SceneStore>();
    store->device = c->device;
    auto upload = [&](const void *src, size_t bytes, const void **dst) -> hdr_status {
        DevBuf b;
        hdr_status st = dev_alloc(c, b, std::max<size_t>(bytes, 16));
        if (st != HDR_OK) return st;
        store->ptrs.push_back(b.ptr);
        store->bytes += b.bytes;
        if (bytes && src) HDR_CUDA(cudaMemcpyAsync(b.ptr, src, bytes, cudaMemcpyHostToDevice, c->stream));
        *dst = b.ptr;
        return HDR_OK;
    };
    hdr::DeviceScene s{};
    hdr_status st;
#define UP(vec, field)                                                                              \
    st = upload(vec.data(), vec.size() * sizeof(vec[0]), (const void **)&s.field);                   \
    if (st != HDR_OK) {                                                                             \
        cudaStreamSynchronize(c->stream);                                                           \
        c->allocated -= store->bytes;                                                               \
        return st;                                                                                  \
    }                                                                                               \
    store->arrays[#field] = {s.field, vec.size() * sizeof(vec[0])};
    if (device_build) {
        const size_t node_bytes = f.num_blas_nodes * 2 * sizeof(float4);
        const size_t geo_bytes = f.num_triangles * (hdr::kTriGeoFloats * sizeof(float));
        const size_t attr_bytes = f.num_triangles * (hdr::kTriAttrFloats * sizeof(float));
        if ((st = upload(nullptr, node_bytes, (const void **)&s.blas_nodes)) != HDR_OK ||
            (st = upload(nullptr, geo_bytes, (const void **)&s.tri_geo)) != HDR_OK ||
            (st = upload(nullptr, attr_bytes, (const void **)&s.tri_attr)) != HDR_OK) {
            cudaStreamSynchronize(c->stream);
            c->allocated -= store->bytes;
            return st;
        }
        size_t node_base = 0, tri_base = 0;
        for (size_t mi = 0; mi < dev_blas.size(); ++mi) {
            const cudaError_t e = dev_blas[mi]->write(const_cast<float4 *>(s.blas_nodes) + 2 * node_base,
                                                      const_cast<float4 *>(s.tri_geo) + 3 * tri_base,
                                                      const_cast<float4 *>(s.tri_attr) + 9 * tri_base);
            if (e != cudaSuccess) {
                cudaStreamSynchronize(c->stream);
                c->allocated -= store->bytes;
                return fail(HDR_ECUDA, "device BLAS build of mesh %zu: %s", mi, cudaGetErrorString(e));
            }
            node_base += (size_t)ext[mi].num_nodes;
            tri_base += (size_t)ext[mi].num_tris;
        }
        store->arrays["blas_nodes"] = {s.blas_nodes, node_bytes};
        store->arrays["tri_geo"] = {s.tri_geo, geo_bytes};
        store->arrays["tri_attr"] = {s.tri_attr, attr_bytes};
    } else {
        UP(f.blas_nodes, blas_nodes);
        UP(f.tri_geo, tri_geo);
        UP(f.tri_attr, tri_attr);
    }
    UP(f.instances, instances);
    // room for the TLAS of any transforms of the same instances (hdr_scene_set_instance_transforms):
    // each visited node allocates two, and at most 2n - 1 nodes are visited
    const int tlas_capacity = 4 * f.num_instances;
    if (f.tlas_nodes.size() < 8 * (size_t)tlas_capacity) f.tlas_nodes.resize(8 * (size_t)tlas_capacity, 0.0f);
    UP(f.tlas_nodes, tlas_nodes);
    UP(f.tlas_inst, tlas_inst);
    UP(f.materials, materials);
    UP(f.textures, textures);
    UP(f.lights, lights);
    UP(f.dome_pixels, dome_pixels);
    UP(f.dome_row_cdf, dome_row_cdf);
    UP(f.dome_col_cdf, dome_col_cdf);
    UP(f.blas4, blas4);
    UP(f.blas_roots, blas_roots);
    UP(f.tlas4, tlas4);
    // shadow-ray BVH: built unless this ctx walks the reference trees for shadow rays
    hdr::ShadowBvh sb;
    if (!(c->flags & HDR_CTX_REFERENCE_SHADOWS)) {
        if (!hdr::build_shadow_bvh(*desc, f, sb, err)) {
            cudaStreamSynchronize(c->stream);
            c->allocated -= store->bytes;
            return fail(HDR_EINVAL, "%s", err.c_str());
        }
    }
    if (sb.ok) {
        UP(sb.nodes, sh4_nodes);
        UP(sb.tris, sh4_tris);
        UP(sb.inst_root, sh4_inst_root);
        UP(sb.inst_rank, sh4_inst_rank);
        store->sh4 = true;
        store->sh4_inst_root = sb.inst_root;
        store->sh4_tlas_capacity = sb.tlas_capacity;
        store->sh4_blas_depth = sb.blas_depth;
        RefLinks links;  // exact closest hits on the SAH trees (closest_mode 2)
        std::vector<float> dev_nodes;  // a device build's BLAS nodes, copied back for the links
        if (device_build && f.num_blas_nodes > 0) {
            dev_nodes.resize((size_t)f.num_blas_nodes * 8);
            HDR_CUDA(cudaMemcpyAsync(dev_nodes.data(), s.blas_nodes, dev_nodes.size() * sizeof(float),
                                     cudaMemcpyDeviceToHost, c->stream));
            HDR_CUDA(cudaStreamSynchronize(c->stream));
        }
        if (build_ref_links(f, device_build ? dev_nodes : f.blas_nodes,
                            device_build ? (size_t)f.num_triangles : f.tri_geo.size() / 12, links)) {
            UP(links.tlas_path, ref_tlas_path);
            UP(links.inst_leaf, ref_inst_leaf);
            UP(links.blas_path, ref_blas_path);
            UP(links.tri_leaf, ref_tri_leaf);
            store->ref_links = true;
        }
    }
#undef UP
    {  // the device TLAS rebuild's inputs and scratch
        const size_t n = (size_t)f.num_instances;
        const void *ranges = nullptr, *bounds = nullptr, *xf = nullptr, *stk = nullptr, *info = nullptr;
        if ((st = upload(f.mesh_ranges.data(), f.mesh_ranges.size() * sizeof(float), &ranges)) != HDR_OK ||
            (st = upload(nullptr, n * 9 * sizeof(float), &bounds)) != HDR_OK ||
            (st = upload(nullptr, n * 16 * sizeof(float), &xf)) != HDR_OK ||
            (st = upload(nullptr, (n + 2) * sizeof(int4), &stk)) != HDR_OK ||
            (st = upload(nullptr, 4 * sizeof(int), &info)) != HDR_OK) {
            cudaStreamSynchronize(c->stream);
            c->allocated -= store->bytes;
            return st;
        }
        store->mesh_ranges = (float *)ranges;
        store->inst_bounds = (float *)bounds;
        store->xf_staging = (float *)xf;
        store->tlas_stack = (int4 *)stk;
        store->tlas_info = (int *)info;
        store->num_instances = f.num_instances;
        store->max_blas_depth = f.max_blas_depth;
        store->tlas_capacity = tlas_capacity;
        store->blas_proper = blas_boxes_proper(f) && !dev_empty_box;
        store->wide_stale = device_build;  // the device build makes no wide trees
    }
    std::memcpy(&s.tlas_root_lo, f.tlas_root, sizeof(float4));
    std::memcpy(&s.tlas_root_hi, f.tlas_root + 4, sizeof(float4));
    s.wide = (c->flags & HDR_CTX_WIDE_BVH) ? 1 : 0;
    s.num_instances = f.num_instances;
    s.num_materials = f.num_materials;
    s.num_lights = f.num_lights;
    s.env_light = f.env_light;
    s.sky = desc->enable_physical_sky ? 1 : 0;
    s.blackbody = 0;
    for (int i = 0; i < desc->num_lights; ++i) s.blackbody |= desc->lights[i].temperature > 0.0f ? 1 : 0;
    if (s.sky) {  // PhysicalSky's sun (scene.cpp:249-254, physical_sky.cpp:161-169), with the host's libm
        const hdr::V3 sun = hdr::sky_sun_direction(desc->physical_sky_time);
        const hdr::V3 sun_n = hdr::normalized(sun);
        hdr::V3 color{0.0f, 0.0f, 0.0f};
        const bool lit = hdr::sky_sun_color(sun, color);
        s.sky_sun = make_float4(sun.x, sun.y, sun.z, lit ? 1.0f : 0.0f);
        s.sky_sun_n = make_float4(sun_n.x, sun_n.y, sun_n.z, 0.0f);
        s.sky_sun_color = make_float4(color.x, color.y, color.z, 0.0f);
    }
    s.dome_width = f.dome_width;
    s.dome_height = f.dome_height;
    s.dome_total_lum = f.dome_total_lum;
    s.has_tlas = f.num_instances > 0 ? 1 : 0;
    s.proper_boxes = (store->blas_proper && tlas_boxes_proper(f)) ? 1 : 0;
    s.shallow = (f.max_blas_depth + f.max_tlas_depth + 4 <= hdr::kShallowStack) ? 1 : 0;
    s.has_textures = f.textures.empty() ? 0 : 1;
    s.sh4 = store->sh4 ? 1 : 0;
    s.sh4_closest = closest_mode(c->flags, store->sh4, store->ref_links);
    // the descriptor itself, for callees that are not inlined into a kernel
    hdr::DeviceScene copies[kDescCopies];
    {
        DevBuf b;
        st = dev_alloc(c, b, sizeof(copies));
        if (st != HDR_OK) {
            cudaStreamSynchronize(c->stream);
            c->allocated -= store->bytes;
            return st;
        }
        store->ptrs.push_back(b.ptr);
        store->bytes += b.bytes;
        store->desc_dev = (const hdr::DeviceScene *)b.ptr;
        fill_desc_copies(s, store->desc_dev, copies, store->sh4);
        HDR_CUDA(cudaMemcpyAsync(b.ptr, copies, sizeof(copies), cudaMemcpyHostToDevice, c->stream));
    }
    s.dev = store->desc_dev + desc_index(s);
    const cudaError_t sync_err = cudaStreamSynchronize(c->stream);
    c->scene_store = store;  // owns the buffers from here on, also on the error path below
    c->scene_bytes_accounted = store->bytes;
    if (sync_err != cudaSuccess) return fail(HDR_ECUDA, "scene upload: %s", cudaGetErrorString(sync_err));
    c->scene = s;
    c->has_scene = true;
    c->have_wave = false;
    c->scene_opaque = true;
    for (int i = 0; i < desc->num_materials; ++i)
        if (!(desc->materials[i].opacity >= 0.999f)) c->scene_opaque = false;
    c->scene_light_geometry = false;
    for (int i = 0; i < desc->num_instances; ++i)
        if (desc->instances[i].light >= 0) c->scene_light_geometry = true;
    c->scene_emissive = false;
    for (int i = 0; i < desc->num_materials; ++i)  // the closure's emission, as the scene builder computes it
        for (int k = 0; k < 3; ++k)
            if (!(desc->materials[i].emission_color[k] * desc->materials[i].emission == 0.0f)) c->scene_emissive = true;
    return HDR_OK;
}

static hdr_status raycast_pass(hdr_ctx *c, const hdr_camera *cam, int32_t frame_index, uint32_t aov_mask) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    hdr_status st = check_camera(cam);
    if (st != HDR_OK) return st;
    if (!c->has_scene) return fail(HDR_ENOSCENE, "hdr_raycast before hdr_scene_upload");
    if ((st = check_cancel(c)) != HDR_OK) return st;
    HDR_CUDA(cudaSetDevice(c->device));
    const size_t count = (size_t)cam->width * cam->height;
    hdr::GBufferView gb;
    if ((st = gbuffer_view(c, count, true, gb)) != HDR_OK) return st;
    hdr::AovView aov{nullptr, nullptr, nullptr};
    void *p;
    if (aov_mask & HDR_AOV_DEPTH) {
        if ((st = ensure_buffer(c, "Depth", count * 4, &p)) != HDR_OK) return st;
        aov.depth = (float *)p;
    }
    if (aov_mask & HDR_AOV_ALBEDO) {
        if ((st = ensure_buffer(c, "Albedo", count * 12, &p)) != HDR_OK) return st;
        aov.albedo = (float *)p;
    }
    if (aov_mask & HDR_AOV_NORMAL) {
        if ((st = ensure_buffer(c, "Normal", count * 12, &p)) != HDR_OK) return st;
        aov.normal = (float *)p;
    }
    hdr::CameraD d = make_camera(cam);
    if ((st = record_frame_index(c, frame_index, &d)) != HDR_OK) return st;
    c->width = cam->width;
    c->height = cam->height;
    if ((st = begin_pass(c, 0)) != HDR_OK) return st;
    hdr::launch_raycast(c->scene, d, frame_index, gb, aov, c->d_err, c->stream);
    c->launches += 1;
    return end_pass(c, 0);
}

}  // extern "C"

namespace {

// Device time of `launch` (ms, best of two runs) on the ctx stream; `prepare`
// runs before each run, outside the timed part. -1 on a launch failure.
template <class Prepare, class Launch>
hdr_status time_best_of_two(hdr_ctx *c, Prepare prepare, Launch launch, float &ms_out) {
    cudaEvent_t ev[2] = {c->region_ev[3][0], c->region_ev[3][1]};
    float best = 3.4e38f;
    for (int rep = 0; rep < 2; ++rep) {
        hdr_status st = prepare();
        if (st != HDR_OK) return st;
        HDR_CUDA(cudaEventRecord(ev[0], c->stream));
        const int n = launch();
        if (n < 0) return fail(HDR_ECUDA, "launch failed while tuning: %s", cudaGetErrorString(cudaGetLastError()));
        c->launches += (uint64_t)n;
        HDR_CUDA(cudaEventRecord(ev[1], c->stream));
        HDR_CUDA(cudaEventSynchronize(ev[1]));
        float ms = 0.0f;
        HDR_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        best = std::min(best, ms);
    }
    ms_out = best;
    return HDR_OK;
}

// The trace-schedule search over queues the generate kernel filled: node quorum x
// persistent blocks per SM (x the shadow walk's register budget on the 4-wide SAH
// trees). The trace kernels only read the queues and rewrite the same hit and
// occlusion slots, so each rerun needs nothing but its fetch counters at zero.
hdr_status search_trace_schedule(hdr_ctx *c, const hdr::WaveBuffers &wb, hdr::TraceTuning &pick, float &pick_ms) {
    static const int kQuorum[] = {8, 12, 16, 20, 24, 28};
    static const int kBlocks[] = {4, 6, 8, 16};
    hdr::TraceTuning t = c->tune;
    pick = c->tune;
    pick_ms = 3.4e38f;
    const int n_shapes = c->scene.sh4 ? hdr::kShadowShapes : 1;
    for (int si = 0; si < n_shapes; ++si)
        for (int quorum : kQuorum)
            for (int blocks : kBlocks) {
                t.node_quorum = quorum;
                t.blocks_per_sm = blocks;
                if (c->scene.sh4) t.shadow_shape = si;
                float ms = 0.0f;
                hdr_status st = time_best_of_two(
                    c,
                    [&]() -> hdr_status {
                        HDR_CUDA(cudaMemsetAsync(wb.counts + 2, 0, 2 * sizeof(int), c->stream));
                        return HDR_OK;
                    },
                    [&]() { return hdr::launch_wave_trace(c->scene, wb, t, c->d_err, c->stream); }, ms);
                if (st != HDR_OK) return st;
                if (ms < pick_ms) pick_ms = ms, pick = t;
            }
    return HDR_OK;
}

// hdr_autotune_frame's wavefront frame: generate once, then the trace kernels once per
// trace schedule and the resampling kernel once per launch shape, each shade run from a
// copy of the reservoirs it reads (it merges into them in place) and with the winner
// queue emptied; every run writes the same bytes. The fastest schedule and shape stay in
// the ctx. Returns the kernel launches of one plain frame in *frame_launches.
hdr_status tune_wave_frame(hdr_ctx *c, const hdr::CameraD &cd, int frame_index, const hdr::RisParamsD &d,
                           const hdr::GBufferView &gb, const hdr::ReservoirView &rv, const hdr::WaveBuffers &wb,
                           float4 *color, int trace_level, hdr_trace_tuning *best, int *frame_launches) {
    const bool tex = c->scene.has_textures;
    cudaStream_t s = c->stream;
    HDR_CUDA(cudaMemsetAsync(wb.counts, 0, (wb.q_winner ? 6 : 4) * sizeof(int), s));
    if ((tex ? hdr::textured::launch_ris_generate : hdr::launch_ris_generate)(c->scene, cd, frame_index, d, gb, wb,
                                                                             color, trace_level, c->d_err, s) < 0)
        return fail(HDR_ECUDA, "generate launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    hdr::TraceTuning pick;
    float trace_ms = 0.0f;
    hdr_status st = search_trace_schedule(c, wb, pick, trace_ms);
    if (st != HDR_OK) return st;
    c->tune.node_quorum = pick.node_quorum;
    c->tune.blocks_per_sm = pick.blocks_per_sm;
    c->tune.shadow_shape = pick.shadow_shape;
    void *snap = nullptr;
    const size_t res_bytes = wb.pixels * kResPlanes * sizeof(float4);
    if (rv.dir_dist) {
        if ((st = ensure_scratch(c, "__tune_reservoir", res_bytes, &snap)) != HDR_OK) return st;
        HDR_CUDA(cudaMemcpyAsync(snap, rv.dir_dist, res_bytes, cudaMemcpyDeviceToDevice, s));
    }
    hdr::TraceTuning t = c->tune;
    int shade_pick = t.shade_shape;
    float shade_ms = 3.4e38f;
    for (int shape = 0; shape < hdr::kShadeShapes; ++shape) {
        t.shade_shape = shape;
        float ms = 0.0f;
        st = time_best_of_two(
            c,
            [&]() -> hdr_status {
                if (snap) HDR_CUDA(cudaMemcpyAsync(rv.dir_dist, snap, res_bytes, cudaMemcpyDeviceToDevice, s));
                if (wb.q_winner) HDR_CUDA(cudaMemsetAsync(wb.counts + 4, 0, 2 * sizeof(int), s));
                return HDR_OK;
            },
            [&]() {
                return (tex ? hdr::textured::launch_ris_shade : hdr::launch_ris_shade)(
                    c->scene, cd, frame_index, d, gb, rv, wb, color, trace_level, c->d_err, s, t);
            },
            ms);
        if (st != HDR_OK) return st;
        if (ms < shade_ms) shade_ms = ms, shade_pick = shape;
    }
    c->tune.shade_shape = shade_pick;
    int n = 4;
    if (wb.q_winner) {
        if ((tex ? hdr::textured::launch_winner_visibility : hdr::launch_winner_visibility)(
                c->scene, cd, frame_index, d, gb, rv, wb, color, c->d_err, s, c->tune) < 0)
            return fail(HDR_ECUDA, "winner visibility launch failed: %s", cudaGetErrorString(cudaGetLastError()));
        n += 2;
    }
    if (best) {
        best->node_quorum = c->tune.node_quorum;
        best->blocks_per_sm = c->tune.blocks_per_sm;
        best->trace_ms = trace_ms;
        best->shade_shape = c->tune.shade_shape;
        best->shadow_shape = c->tune.shadow_shape;
        best->shade_ms = shade_ms;
    }
    *frame_launches = n;
    return HDR_OK;
}

}  // namespace

extern "C" {

static hdr_status ris_path_trace_pass(hdr_ctx *c, const hdr_camera *cam, int32_t frame_index,
                                      const hdr_ris_params *p, hdr_trace_tuning *tune = nullptr) {
    if (!c || !p) return fail(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(c->mu);
    struct TuneScope {  // hdr_autotune_frame: this call only
        hdr_ctx *c;
        ~TuneScope() { c->tune_frame = false, c->tune_out = nullptr; }
    } tune_scope{c};
    c->tune_frame = tune != nullptr;
    c->tune_out = tune;
    if (tune) HDR_NOT_RECORDING(c, "hdr_autotune_frame");
    hdr_status st = check_camera(cam);
    if (st != HDR_OK) return st;
    if (!c->has_scene) return fail(HDR_ENOSCENE, "hdr_ris_path_trace before hdr_scene_upload");
    if (p->candidate_count < 1 || p->candidate_count > 4096)
        return fail(HDR_EINVAL, "candidate_count %d out of range [1, 4096]", p->candidate_count);
    if (p->path.max_depth < 1) return fail(HDR_EINVAL, "max_depth must be >= 1");
    if (p->spatial_neighbors < 0 || p->spatial_neighbors > 64 || !(p->spatial_radius >= 0.0f))
        return fail(HDR_EINVAL, "spatial_neighbors %d / spatial_radius out of range ([0, 64], >= 0)",
                    p->spatial_neighbors);
    // wavefront form: direct light only (no later bounces), no stochastic opacity, no physical
    // sky (its sun technique is served by the one-kernel form only) and no blackbody lights
    // (an extension the wavefront kernels are built without, to keep their registers)
    const bool wave = p->path.max_depth == 1 && c->scene_opaque && !c->scene.sky && !c->scene.blackbody &&
                      !(p->flags & HDR_RIS_ONE_KERNEL);
    const bool spatial = p->spatial_neighbors > 0 && p->use_reservoir;
    if (spatial && !wave)
        return fail(HDR_EINVAL, "spatial reuse runs in the wavefront form only (max_depth 1, opaque scene)");
    if (tune && !wave)
        return fail(HDR_EINVAL, "hdr_autotune_frame tunes the wavefront form (max_depth 1, opaque scene, "
                    "no HDR_RIS_ONE_KERNEL)");
    if ((st = check_cancel(c)) != HDR_OK) return st;
    HDR_CUDA(cudaSetDevice(c->device));
    const size_t count = (size_t)cam->width * cam->height;
    hdr::GBufferView gb;
    if ((st = gbuffer_view(c, count, false, gb)) != HDR_OK) return st;
    void *color = nullptr, *res = nullptr;
    if ((st = ensure_buffer(c, "Color", count * 16, &color)) != HDR_OK) return st;
    hdr::ReservoirView rv{};
    if (p->use_reservoir) {
        // GetOrCreatePersistent("__ris_reservoir") (ris_direct_light_integrator.cpp:56-67)
        if ((st = ensure_buffer(c, "__ris_reservoir", count * kResPlanes * sizeof(float4), &res)) != HDR_OK) return st;
        float4 *r = (float4 *)res;
        rv = hdr::ReservoirView{r, r + count, r + 2 * count, r + 3 * count, r + 4 * count};
    }
    hdr::RisParamsD d{};
    d.candidate_count = p->candidate_count;
    d.use_reservoir = p->use_reservoir;
    d.skip_visibility = p->skip_visibility;
    d.max_depth = p->path.max_depth;
    d.enable_subsurface = p->path.enable_subsurface;
    d.max_refl = p->path.max_reflection_bounces;
    d.max_refr = p->path.max_refraction_bounces;
    d.render_ibl_background = p->path.render_ibl_background;
    d.roulette = p->path.roulette_aggressiveness;
    d.m_cap = p->m_cap;
    d.spatial_neighbors = p->spatial_neighbors;
    d.spatial_radius = p->spatial_radius;
    hdr::CameraD cd = make_camera(cam);
    if ((st = record_frame_index(c, frame_index, &cd)) != HDR_OK) return st;
    const bool reproject = (p->flags & HDR_RIS_REPROJECT) && p->use_reservoir;
    hdr::GBufferView gb_prev{};
    if (reproject) {  // this frame's temporal history comes from where its hit points were last frame
        void *q, *pos;
        if ((st = ensure_buffer(c, "__ris_reservoir_prev", count * kResPlanes * sizeof(float4), &q)) != HDR_OK)
            return st;
        if ((st = ensure_buffer(c, "__prev_pos_depth", count * sizeof(float4), &pos)) != HDR_OK) return st;
        gb_prev.pos_depth = (float4 *)pos;
        hdr::ReprojD &rj = d.reproj;
        rj.mode = 2;
        if (c->reproj_valid && c->reproj_w == cam->width && c->reproj_h == cam->height) {
            HDR_CUDA(cudaMemcpyAsync(q, rv.dir_dist, count * kResPlanes * sizeof(float4), cudaMemcpyDeviceToDevice,
                                     c->stream));
            float4 *r = (float4 *)q;
            rj.mode = 1;
            rj.width = c->reproj_w;
            rj.height = c->reproj_h;
            std::memcpy(rj.view, c->reproj_view, sizeof(rj.view));
            std::memcpy(rj.proj, c->reproj_proj, sizeof(rj.proj));
            rj.prev_pos = gb_prev.pos_depth;
            rj.prev = hdr::ReservoirView{r, r + count, r + 2 * count, r + 3 * count, r + 4 * count};
        }
    }
    // after the pass: this frame's hit points and camera become the next frame's history
    auto keep_history = [&]() -> hdr_status {
        if (!reproject) return HDR_OK;
        HDR_CUDA(cudaMemcpyAsync(gb_prev.pos_depth, gb.pos_depth, count * sizeof(float4), cudaMemcpyDeviceToDevice,
                                 c->stream));
        c->reproj_valid = true;
        c->reproj_w = cam->width;
        c->reproj_h = cam->height;
        std::memcpy(c->reproj_view, cam->view, sizeof(c->reproj_view));
        std::memcpy(c->reproj_proj, cam->proj, sizeof(c->reproj_proj));
        return HDR_OK;
    };
    hdr::ReservoirView rv_spatial{};
    if (spatial) {  // neighbours read this frame's reservoirs while the merged ones are written here
        void *q;
        if ((st = ensure_buffer(c, "__ris_reservoir_spatial", count * kResPlanes * sizeof(float4), &q)) != HDR_OK)
            return st;
        float4 *r = (float4 *)q;
        rv_spatial = hdr::ReservoirView{r, r + count, r + 2 * count, r + 3 * count, r + 4 * count};
    }
    if (wave) {
        const int n_nee = std::max(1, p->candidate_count / 2);
        const int n_bsdf = std::max(0, p->candidate_count - n_nee);
        const int trace_level = ris_trace_level(c, p);
        hdr::WaveBuffers wb{};
        wb.pixels = count;
        wb.n_closest = closest_slots(trace_level, n_bsdf);
        wb.n_shadow = n_nee;
        void *q;
        if ((st = ensure_buffer(c, "__wave_q_closest", count * wb.n_closest * 32, &q)) != HDR_OK) return st;
        wb.q_closest = (float4 *)q;
        if ((st = ensure_buffer(c, "__wave_q_shadow", count * wb.n_shadow * 32, &q)) != HDR_OK) return st;
        wb.q_shadow = (float4 *)q;
        if ((st = ensure_buffer(c, "__wave_counts", 32, &q)) != HDR_OK) return st;
        wb.counts = (int *)q;
        if ((st = ensure_buffer(c, "__wave_fix", count * wb.n_closest * 4, &q)) != HDR_OK) return st;
        wb.fix = (int *)q;
        if ((st = ensure_buffer(c, "__wave_hits", count * wb.n_closest * 16, &q)) != HDR_OK) return st;
        wb.hits = (float4 *)q;
        if ((st = ensure_buffer(c, "__wave_hit_v", count * wb.n_closest * 4, &q)) != HDR_OK) return st;
        wb.hit_v = (float *)q;
        if ((st = ensure_buffer(c, "__wave_occ", count * wb.n_shadow, &q)) != HDR_OK) return st;
        wb.occ = (unsigned char *)q;
        if ((st = ensure_buffer(c, "__wave_rng", count * 48, &q)) != HDR_OK) return st;
        wb.rng_state = (uint4 *)q;
        if ((st = ensure_buffer(c, "__wave_done", count, &q)) != HDR_OK) return st;
        wb.done = (unsigned char *)q;
        if (c->flags & HDR_CTX_RECORD_LIGHTS) {
            if ((st = ensure_buffer(c, "__ris_nee_lights", count * wb.n_shadow * 4, &q)) != HDR_OK) return st;
            wb.nee_light = (int *)q;
        }
        if (p->skip_visibility || reproject || spatial) {  // winners whose visibility is still untested: one per pixel
            if ((st = ensure_buffer(c, "__wave_q_winner", count * 32, &q)) != HDR_OK) return st;
            wb.q_winner = (float4 *)q;
            if ((st = ensure_buffer(c, "__wave_occ_winner", count, &q)) != HDR_OK) return st;
            wb.occ_winner = (unsigned char *)q;
        }
        if ((st = begin_pass(c, 1)) != HDR_OK) return st;
        const bool timed = timing_on(c);
        if (timed)
            for (int k = kSlotWaveFirst; k < kSlotWaveFirst + 4; ++k)
                if ((st = fold_pass_time(c, k)) != HDR_OK) return st;
        int n = 0;
        if (c->tune_frame) {  // hdr_autotune_frame: the same frame, its kernels run once per schedule and shape
            if ((st = tune_wave_frame(c, cd, frame_index, d, gb, rv, wb, (float4 *)color, trace_level, c->tune_out,
                                      &n)) != HDR_OK)
                return st;
        } else {
            n = (c->scene.has_textures ? hdr::textured::launch_ris_wavefront : hdr::launch_ris_wavefront)(
                c->scene, cd, frame_index, d, gb, rv, wb, (float4 *)color, trace_level, c->d_err, c->stream, c->tune,
                timed ? c->ev_start + kSlotWaveFirst : nullptr, timed ? c->ev_stop + kSlotWaveFirst : nullptr);
            if (n < 0) return fail(HDR_ECUDA, "wavefront launch failed: %s", cudaGetErrorString(cudaGetLastError()));
        }
        if (timed)
            for (int k = kSlotWaveFirst; k < kSlotWaveFirst + 4; ++k) c->ev_pending[k] = true;
        c->launches += (uint64_t)n;
        if (spatial) {  // merged reservoirs, copied back, then the moved samples' shadow rays
            HDR_CUDA(cudaMemsetAsync(wb.counts + 4, 0, 2 * sizeof(int), c->stream));
            if (hdr::launch_ris_spatial(c->scene, cd, frame_index, d, gb, rv, rv_spatial, (float4 *)color,
                                        wb.q_winner, wb.counts + 4, c->d_err, c->stream) < 0)
                return fail(HDR_ECUDA, "spatial reuse launch failed: %s", cudaGetErrorString(cudaGetLastError()));
            HDR_CUDA(cudaMemcpyAsync(rv.dir_dist, rv_spatial.dir_dist, count * kResPlanes * sizeof(float4),
                                     cudaMemcpyDeviceToDevice, c->stream));
            if ((c->scene.has_textures ? hdr::textured::launch_winner_visibility : hdr::launch_winner_visibility)(c->scene, cd, frame_index, d, gb, rv, wb, (float4 *)color, c->d_err,
                                              c->stream, c->tune) < 0)
                return fail(HDR_ECUDA, "winner visibility launch failed: %s", cudaGetErrorString(cudaGetLastError()));
            c->launches += 3;
        }
        c->last_wave = wb;
        c->have_wave = true;
        if ((st = keep_history()) != HDR_OK) return st;
        return end_pass(c, 1);
    }
    if ((st = begin_pass(c, 1)) != HDR_OK) return st;
    hdr::launch_ris_path_trace(c->scene, cd, frame_index, d, gb, rv, (float4 *)color, c->d_err, c->stream);
    c->launches += 1;
    if ((st = keep_history()) != HDR_OK) return st;
    return end_pass(c, 1);
}

}  // extern "C"

namespace {
// The per-path planes, queues and hit slots of the wavefront PathTracePass for
// `count` paths; alloc(name, bytes, &ptr) provides each (per-frame scratch of a
// ctx, or a scene store's batch buffers).
template <class Alloc>
hdr_status pt_buffers_from(Alloc alloc, size_t count, hdr::PtBuffers &B) {
    B = hdr::PtBuffers{};
    B.pixels = count;
    struct Plane {
        const char *name;
        size_t bytes;
        void **dst;
    };
    void *rng, *tp, *total, *outer, *ro, *rd, *bo, *bd, *bt, *nee, *state, *a0, *a1, *cnt, *qc, *qs, *hits, *hv, *occ,
        *fix;
    const Plane planes[] = {
        {"__pt_rng", count * 48, &rng},     {"__pt_tp", count * 16, &tp},       {"__pt_total", count * 16, &total},
        {"__pt_outer", count * 16, &outer}, {"__pt_ray_o", count * 16, &ro},    {"__pt_ray_d", count * 16, &rd},
        {"__pt_b_origin", count * 16, &bo}, {"__pt_b_dir", count * 16, &bd},    {"__pt_b_tmul", count * 16, &bt},
        {"__pt_nee", count * 16, &nee},     {"__pt_state", count * 16, &state}, {"__pt_active0", count * 4, &a0},
        {"__pt_active1", count * 4, &a1},   {"__pt_counts", 32, &cnt},          {"__pt_q_closest", count * 32, &qc},
        {"__pt_q_shadow", count * 32, &qs}, {"__pt_hits", count * 16, &hits},   {"__pt_hit_v", count * 4, &hv},
        {"__pt_occ", count, &occ},          {"__pt_fix", count * 4, &fix}};
    hdr_status st;
    for (const Plane &pl : planes)
        if ((st = alloc(pl.name, pl.bytes, pl.dst)) != HDR_OK) return st;
    B.rng = (uint4 *)rng;
    B.tp = (float4 *)tp;
    B.total = (float4 *)total;
    B.outer = (float4 *)outer;
    B.ray_o = (float4 *)ro;
    B.ray_d = (float4 *)rd;
    B.b_origin_pdf = (float4 *)bo;
    B.b_dir = (float4 *)bd;
    B.b_tmul = (float4 *)bt;
    B.nee_add = (float4 *)nee;
    B.state = (int4 *)state;
    B.active[0] = (int *)a0;
    B.active[1] = (int *)a1;
    B.counts = (int *)cnt;
    B.fix = (int *)fix;
    B.q_closest = (float4 *)qc;
    B.q_shadow = (float4 *)qs;
    B.hits = (float4 *)hits;
    B.hit_v = (float *)hv;
    B.occ = (unsigned char *)occ;
    return HDR_OK;
}
hdr_status pt_buffers(hdr_ctx *c, size_t count, hdr::PtBuffers &B) {
    return pt_buffers_from([c](const char *name, size_t bytes, void **p) { return ensure_scratch(c, name, bytes, p); },
                           count, B);
}
}  // namespace

extern "C" {

hdr_status hdr_scene_share(hdr_ctx *dst, hdr_ctx *src) {
    if (!dst || !src || dst == src) return fail(HDR_EINVAL, "need two distinct contexts");
    if (dst->device != src->device) return fail(HDR_EINVAL, "contexts are on different devices");
    std::lock(dst->mu, src->mu);
    std::lock_guard<std::mutex> l1(dst->mu, std::adopt_lock), l2(src->mu, std::adopt_lock);
    HDR_NOT_RECORDING(dst, "hdr_scene_share");
    if (!src->has_scene) return fail(HDR_ENOSCENE, "the source context has no scene");
    if ((dst->flags & HDR_CTX_WIDE_BVH) && src->scene_store->wide_stale)
        return fail(HDR_EINVAL, "the scene's instances moved on the device: its wide TLAS is not rebuilt");
    HDR_CUDA(cudaSetDevice(dst->device));
    HDR_CUDA(cudaStreamSynchronize(dst->stream));  // dst's old scene may still be in use on its stream
    dst->scene_store = src->scene_store;
    dst->allocated -= dst->scene_bytes_accounted;
    dst->scene_bytes_accounted = 0;
    dst->scene = src->scene;
    dst->scene.wide = (dst->flags & HDR_CTX_WIDE_BVH) ? 1 : 0;
    dst->scene.sh4 = (dst->scene_store->sh4 && !(dst->flags & HDR_CTX_REFERENCE_SHADOWS)) ? 1 : 0;
    dst->scene.sh4_closest = closest_mode(dst->flags, dst->scene.sh4, dst->scene_store->ref_links);
    dst->scene.dev = dst->scene_store->desc_dev + desc_index(dst->scene);
    dst->scene_opaque = src->scene_opaque;
    dst->scene_light_geometry = src->scene_light_geometry;
    dst->scene_emissive = src->scene_emissive;
    dst->has_scene = true;
    dst->have_wave = false;
    return HDR_OK;
}

// Scene::BuildRenderState after HdRestirMesh::Sync took new transforms
// (hd_restir_mesh.cpp:160-162, scene.cpp:118-244, 333-407): the instance records
// and the binary TLAS rebuilt in place on the ctx stream, the same bits a fresh
// hdr_scene_upload of the scene with these transforms would give.
hdr_status hdr_scene_set_instance_transforms(hdr_ctx *c, const float *transforms, int32_t num_instances,
                                             int32_t transforms_on_device) {
    if (!c || !transforms) return fail(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_scene_set_instance_transforms");
    if (!c->has_scene) return fail(HDR_ENOSCENE, "hdr_scene_set_instance_transforms before hdr_scene_upload");
    SceneStore *store = c->scene_store.get();
    if (num_instances != store->num_instances)
        return fail(HDR_EINVAL, "%d transforms for a scene of %d instances", num_instances, store->num_instances);
    if (c->scene.wide) return fail(HDR_EINVAL, "no device TLAS rebuild for the wide BVH walk (HDR_CTX_WIDE_BVH)");
    if (c->scene_store.use_count() > 1)
        return fail(HDR_EINVAL, "the scene is shared with another context (hdr_scene_share)");
    if (num_instances == 0) return HDR_OK;
    HDR_CUDA(cudaSetDevice(c->device));
    const float *xf = transforms;
    if (!transforms_on_device) {
        HDR_CUDA(cudaMemcpyAsync(store->xf_staging, transforms, (size_t)num_instances * 16 * sizeof(float),
                                 cudaMemcpyHostToDevice, c->stream));
        xf = store->xf_staging;
    }
    hdr::DeviceScene &s = c->scene;
    const int launched = hdr::launch_tlas_rebuild(
        xf, const_cast<float4 *>(s.instances), store->mesh_ranges, store->inst_bounds, num_instances,
        const_cast<float4 *>(s.tlas_nodes), store->tlas_capacity, const_cast<int *>(s.tlas_inst), store->tlas_stack,
        num_instances + 2, store->tlas_info, c->stream);
    if (launched < 0) {
        c->has_scene = false;
        return fail(HDR_ECUDA, "TLAS rebuild launch: %s", cudaGetErrorString(cudaGetLastError()));
    }
    c->launches += (uint64_t)launched;
    int info[4] = {};
    HDR_CUDA(cudaMemcpyAsync(info, store->tlas_info, sizeof(info), cudaMemcpyDeviceToHost, c->stream));
    HDR_CUDA(cudaStreamSynchronize(c->stream));
    store->wide_stale = true;
    if (info[2] || store->max_blas_depth + info[1] + 4 > hdr::kTraceStack) {
        c->has_scene = false;  // the records are rewritten but the TLAS cannot be walked: upload again
        return fail(HDR_EINVAL, "TLAS depth %d + BVH depth %d exceeds the device traversal stack (%d)", info[1],
                    store->max_blas_depth, hdr::kTraceStack);
    }
    s.proper_boxes = (store->blas_proper && !info[3]) ? 1 : 0;
    s.shallow = (store->max_blas_depth + info[1] + 4 <= hdr::kShallowStack) ? 1 : 0;
    if (store->sh4) {  // the shadow BVH's TLAS over the moved instances' world boxes
        std::vector<float> b9((size_t)num_instances * 9), b6((size_t)num_instances * 6);
        HDR_CUDA(cudaMemcpyAsync(b9.data(), store->inst_bounds, b9.size() * sizeof(float), cudaMemcpyDeviceToHost,
                                 c->stream));
        HDR_CUDA(cudaStreamSynchronize(c->stream));
        for (int i = 0; i < num_instances; ++i)
            for (int k = 0; k < 6; ++k) b6[6 * (size_t)i + k] = b9[9 * (size_t)i + k];
        std::vector<float> tlas;
        int depth = 0;
        // closest-hit tie-breaks follow the rebuilt reference TLAS's instance order
        std::vector<int> tlas_inst((size_t)num_instances), rank;
        HDR_CUDA(cudaMemcpyAsync(tlas_inst.data(), s.tlas_inst, tlas_inst.size() * sizeof(int),
                                 cudaMemcpyDeviceToHost, c->stream));
        HDR_CUDA(cudaStreamSynchronize(c->stream));
        hdr::shadow_ranks(tlas_inst, num_instances, rank);
        if (hdr::rebuild_shadow_tlas(b6, store->sh4_inst_root, store->sh4_blas_depth, tlas, store->sh4_tlas_capacity,
                                     depth)) {
            HDR_CUDA(cudaMemcpyAsync(const_cast<float4 *>(s.sh4_nodes), tlas.data(), tlas.size() * sizeof(float),
                                     cudaMemcpyHostToDevice, c->stream));
            HDR_CUDA(cudaMemcpyAsync(const_cast<int *>(s.sh4_inst_rank), rank.data(), rank.size() * sizeof(int),
                                     cudaMemcpyHostToDevice, c->stream));
            HDR_CUDA(cudaStreamSynchronize(c->stream));  // `tlas` and `rank` are host buffers
        } else {
            store->sh4 = false;  // too deep for the shadow walk's stack: the reference trees serve shadow rays
        }
    }
    // the reference TLAS changed on the device: its path records are rebuilt from it (the BLAS
    // ones still hold); if the new tree does not fit them, closest hits go back to the reference
    // walk for this scene
    if (store->ref_links && store->sh4) {
        const size_t n_rec = store->arrays["ref_tlas_path"].second / 32;
        const size_t n_nodes = std::min(n_rec, (size_t)store->tlas_capacity);
        std::vector<float> nodes(8 * n_nodes);
        std::vector<int> tlas_inst((size_t)num_instances), inst_leaf;
        std::vector<float> path;
        HDR_CUDA(cudaMemcpyAsync(nodes.data(), s.tlas_nodes, nodes.size() * sizeof(float), cudaMemcpyDeviceToHost,
                                 c->stream));
        HDR_CUDA(cudaMemcpyAsync(tlas_inst.data(), s.tlas_inst, tlas_inst.size() * sizeof(int),
                                 cudaMemcpyDeviceToHost, c->stream));
        HDR_CUDA(cudaStreamSynchronize(c->stream));
        store->ref_links =
            tlas_links(nodes.data(), n_nodes, tlas_inst.data(), tlas_inst.size(), num_instances, path, inst_leaf);
        if (store->ref_links) {
            HDR_CUDA(cudaMemcpyAsync(const_cast<float4 *>(s.ref_tlas_path), path.data(), path.size() * sizeof(float),
                                     cudaMemcpyHostToDevice, c->stream));
            HDR_CUDA(cudaMemcpyAsync(const_cast<int *>(s.ref_inst_leaf), inst_leaf.data(),
                                     inst_leaf.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream));
            HDR_CUDA(cudaStreamSynchronize(c->stream));  // host buffers
        }
    } else {
        store->ref_links = false;
    }
    s.sh4 = (store->sh4 && !(c->flags & HDR_CTX_REFERENCE_SHADOWS)) ? 1 : 0;
    s.sh4_closest = closest_mode(c->flags, s.sh4, store->ref_links);
    s.dev = store->desc_dev + desc_index(s);
    hdr::DeviceScene copies[kDescCopies];
    fill_desc_copies(s, store->desc_dev, copies, store->sh4);
    HDR_CUDA(cudaMemcpyAsync(const_cast<hdr::DeviceScene *>(store->desc_dev), copies, sizeof(copies),
                             cudaMemcpyHostToDevice, c->stream));
    HDR_CUDA(cudaStreamSynchronize(c->stream));  // `copies` is a host stack buffer
    return HDR_OK;
}

hdr_status hdr_scene_array(hdr_ctx *c, const char *name, void *dst, size_t bytes, size_t *size) {
    if (!c || !name) return fail(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_scene_array");
    if (!c->has_scene) return fail(HDR_ENOSCENE, "hdr_scene_array before hdr_scene_upload");
    const auto it = c->scene_store->arrays.find(name);
    if (it == c->scene_store->arrays.end()) return fail(HDR_EINVAL, "no scene array named '%s'", name);
    if (size) *size = it->second.second;
    if (!dst) return HDR_OK;
    if (bytes != it->second.second)
        return fail(HDR_EINVAL, "scene array '%s' holds %zu bytes, not %zu", name, it->second.second, bytes);
    HDR_CUDA(cudaSetDevice(c->device));
    if (bytes) HDR_CUDA(cudaMemcpyAsync(dst, it->second.first, bytes, cudaMemcpyDeviceToHost, c->stream));
    HDR_CUDA(cudaStreamSynchronize(c->stream));
    return HDR_OK;
}

namespace {

// Everything one image of a wavefront RIS frame needs, prepared on its own ctx.
struct RisJob {
    hdr_ctx *c;
    hdr::CameraD cd;
    hdr::RisParamsD d;
    hdr::GBufferView gb;
    hdr::ReservoirView rv;
    float4 *color;
    int frame;
    int trace_level;
    size_t count;
    int n_closest, n_shadow;
    uint4 *rng_state;
    unsigned char *done;
};

hdr_status prepare_ris_job(hdr_ctx *c, const hdr_camera *cam, int32_t frame_index, const hdr_ris_params *p,
                           RisJob &j) {
    hdr_status st = check_camera(cam);
    if (st != HDR_OK) return st;
    if (!c->has_scene) return fail(HDR_ENOSCENE, "hdr_ris_path_trace_batch before hdr_scene_upload");
    if (p->candidate_count < 1 || p->candidate_count > 4096)
        return fail(HDR_EINVAL, "candidate_count %d out of range [1, 4096]", p->candidate_count);
    if ((st = check_cancel(c)) != HDR_OK) return st;
    j.c = c;
    j.frame = frame_index;
    j.count = (size_t)cam->width * cam->height;
    if ((st = gbuffer_view(c, j.count, false, j.gb)) != HDR_OK) return st;
    void *q = nullptr;
    if ((st = ensure_buffer(c, "Color", j.count * 16, &q)) != HDR_OK) return st;
    j.color = (float4 *)q;
    j.rv = hdr::ReservoirView{};
    if (p->use_reservoir) {
        if ((st = ensure_buffer(c, "__ris_reservoir", j.count * kResPlanes * sizeof(float4), &q)) != HDR_OK) return st;
        float4 *r = (float4 *)q;
        j.rv = hdr::ReservoirView{r, r + j.count, r + 2 * j.count, r + 3 * j.count, r + 4 * j.count};
    }
    hdr::RisParamsD &d = j.d;
    d = hdr::RisParamsD{};
    d.candidate_count = p->candidate_count;
    d.use_reservoir = p->use_reservoir;
    d.skip_visibility = p->skip_visibility;
    d.max_depth = p->path.max_depth;
    d.enable_subsurface = p->path.enable_subsurface;
    d.max_refl = p->path.max_reflection_bounces;
    d.max_refr = p->path.max_refraction_bounces;
    d.render_ibl_background = p->path.render_ibl_background;
    d.roulette = p->path.roulette_aggressiveness;
    d.m_cap = p->m_cap;
    d.spatial_neighbors = p->spatial_neighbors;
    d.spatial_radius = p->spatial_radius;
    j.cd = make_camera(cam);
    const int n_nee = std::max(1, p->candidate_count / 2);
    j.trace_level = ris_trace_level(c, p);
    j.n_closest = closest_slots(j.trace_level, std::max(0, p->candidate_count - n_nee));
    j.n_shadow = n_nee;
    if ((st = ensure_buffer(c, "__wave_rng", j.count * 48, &q)) != HDR_OK) return st;
    j.rng_state = (uint4 *)q;
    if ((st = ensure_buffer(c, "__wave_done", j.count, &q)) != HDR_OK) return st;
    j.done = (unsigned char *)q;
    return HDR_OK;
}

}  // namespace

hdr_status hdr_ris_path_trace_batch(hdr_ctx *const *ctxs, int32_t n, const hdr_camera *cams,
                                    const int32_t *frame_indices, const hdr_ris_params *params) {
    if (!ctxs || !cams || !frame_indices || !params || n < 1 || n > 1024) return fail(HDR_EINVAL, "bad argument");
    for (int32_t i = 0; i < n; ++i)
        if (!ctxs[i]) return fail(HDR_EINVAL, "ctx %d is NULL", i);
    // one shared trace needs one resident scene, one device and the wavefront form for every image;
    // otherwise the images are rendered one after another
    bool together = n > 1;
    for (int32_t i = 0; i < n && together; ++i) {
        hdr_ctx *c = ctxs[i];
        const hdr_ris_params *p = &params[i];
        together = p->spatial_neighbors == 0 && !(p->flags & HDR_RIS_REPROJECT) && c->device == ctxs[0]->device && c->has_scene && c->scene_store &&
                   c->scene_store == ctxs[0]->scene_store && c->scene.wide == ctxs[0]->scene.wide &&
                   p->path.max_depth == 1 && c->scene_opaque && !c->scene.sky && !c->scene.blackbody &&
                   !(p->flags & HDR_RIS_ONE_KERNEL);
    }
    std::vector<hdr_ctx *> order(ctxs, ctxs + n);
    std::sort(order.begin(), order.end());
    if (std::adjacent_find(order.begin(), order.end()) != order.end())
        return fail(HDR_EINVAL, "a context appears twice in the batch");
    if (!together) {
        for (int32_t i = 0; i < n; ++i) {
            const hdr_status st = hdr_ris_path_trace(ctxs[i], &cams[i], frame_indices[i], &params[i]);
            if (st != HDR_OK) return st;
        }
        return HDR_OK;
    }
    for (hdr_ctx *c : order) c->mu.lock();  // address order: no deadlock between batches
    struct Unlock {
        std::vector<hdr_ctx *> &v;
        ~Unlock() {
            for (hdr_ctx *c : v) c->mu.unlock();
        }
    } unlock{order};
    for (hdr_ctx *c : order) HDR_NOT_RECORDING(c, "hdr_ris_path_trace_batch");
    hdr_ctx *lead = ctxs[0];
    HDR_CUDA(cudaSetDevice(lead->device));
    std::vector<RisJob> jobs((size_t)n);
    std::vector<long long> base_c((size_t)n), base_s((size_t)n);
    long long total_c = 0, total_s = 0;
    hdr_status st;
    for (int32_t i = 0; i < n; ++i) {
        if ((st = prepare_ris_job(ctxs[i], &cams[i], frame_indices[i], &params[i], jobs[(size_t)i])) != HDR_OK)
            return st;
        base_c[(size_t)i] = total_c;
        base_s[(size_t)i] = total_s;
        total_c += (long long)jobs[(size_t)i].count * jobs[(size_t)i].n_closest;
        total_s += (long long)jobs[(size_t)i].count * jobs[(size_t)i].n_shadow;
    }
    if (total_c >= (1ll << 31) || total_s >= (1ll << 31))
        return fail(HDR_EINVAL, "batch of %lld closest / %lld shadow ray slots exceeds 2^31", total_c, total_s);
    // the shared queues and result slots belong to the resident scene, whichever ctx leads
    SceneStore *store = lead->scene_store.get();
    std::lock_guard<std::mutex> batch_lock(store->batch_mu);
    hdr::WaveBuffers all{};
    void *q;
    cudaEvent_t done = store->batch_done;
    if ((st = ensure_batch_scratch(store, "q_closest", (size_t)total_c * 32, &q, done, lead->stream)) != HDR_OK) return st;
    all.q_closest = (float4 *)q;
    if ((st = ensure_batch_scratch(store, "q_shadow", (size_t)total_s * 32, &q, done, lead->stream)) != HDR_OK) return st;
    all.q_shadow = (float4 *)q;
    if ((st = ensure_batch_scratch(store, "counts", 32, &q, done, lead->stream)) != HDR_OK) return st;
    all.counts = (int *)q;
    if ((st = ensure_batch_scratch(store, "fix", (size_t)total_c * 4, &q, done, lead->stream)) != HDR_OK) return st;
    all.fix = (int *)q;
    if ((st = ensure_batch_scratch(store, "hits", (size_t)total_c * 16, &q, done, lead->stream)) != HDR_OK) return st;
    all.hits = (float4 *)q;
    if ((st = ensure_batch_scratch(store, "hit_v", (size_t)total_c * 4, &q, done, lead->stream)) != HDR_OK) return st;
    all.hit_v = (float *)q;
    if ((st = ensure_batch_scratch(store, "occ", (size_t)total_s, &q, done, lead->stream)) != HDR_OK) return st;
    all.occ = (unsigned char *)q;
    if (!store->batch_done) HDR_CUDA(cudaEventCreateWithFlags(&store->batch_done, cudaEventDisableTiming));
    // the previous batch on this scene (another lead's stream) has finished with the queues
    HDR_CUDA(cudaStreamWaitEvent(lead->stream, store->batch_done, 0));
    // every image's earlier work (its raycast) runs on its own stream: the lead stream waits for it
    for (int32_t i = 1; i < n; ++i) {
        HDR_CUDA(cudaEventRecord(ctxs[i]->sync_ev, ctxs[i]->stream));
        HDR_CUDA(cudaStreamWaitEvent(lead->stream, ctxs[i]->sync_ev, 0));
    }
    if ((st = begin_pass(lead, 1)) != HDR_OK) return st;
    cudaStream_t s = lead->stream;
    HDR_CUDA(cudaMemsetAsync(all.counts, 0, 16, s));
    std::vector<hdr::WaveBuffers> wbs((size_t)n);
    for (int32_t i = 0; i < n; ++i) {
        const RisJob &j = jobs[(size_t)i];
        hdr::WaveBuffers &wb = wbs[(size_t)i];
        wb = all;
        wb.hits = all.hits + base_c[(size_t)i];
        wb.hit_v = all.hit_v + base_c[(size_t)i];
        wb.occ = all.occ + base_s[(size_t)i];
        wb.rng_state = j.rng_state;
        wb.done = j.done;
        wb.pixels = j.count;
        wb.n_closest = j.n_closest;
        wb.n_shadow = j.n_shadow;
        wb.slot_base_closest = (int)base_c[(size_t)i];
        wb.slot_base_shadow = (int)base_s[(size_t)i];
        if ((lead->scene.has_textures ? hdr::textured::launch_ris_generate : hdr::launch_ris_generate)(lead->scene, j.cd, j.frame, j.d, j.gb, wb, j.color, j.trace_level, j.c->d_err,
                                     s) < 0)
            return fail(HDR_ECUDA, "generate launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    const int traced = hdr::launch_wave_trace(lead->scene, all, lead->tune, lead->d_err, s);
    if (traced < 0) return fail(HDR_ECUDA, "trace launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    for (int32_t i = 0; i < n; ++i) {
        const RisJob &j = jobs[(size_t)i];
        if ((lead->scene.has_textures ? hdr::textured::launch_ris_shade : hdr::launch_ris_shade)(lead->scene, j.cd, j.frame, j.d, j.gb, j.rv, wbs[(size_t)i], j.color, j.trace_level,
                                  j.c->d_err, s, lead->tune) < 0)
            return fail(HDR_ECUDA, "shade launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    // later work on each image's own stream (accumulate, download) waits for the batch
    HDR_CUDA(cudaEventRecord(lead->sync_ev, s));
    HDR_CUDA(cudaEventRecord(store->batch_done, s));
    for (int32_t i = 1; i < n; ++i) HDR_CUDA(cudaStreamWaitEvent(ctxs[i]->stream, lead->sync_ev, 0));
    lead->launches += (uint64_t)(2 * n + traced);
    // the queues belong to the scene and the next batch reuses them: no autotuning rerun of this one
    lead->have_wave = false;
    return end_pass(lead, 1);
}

static hdr_status path_trace_pass(hdr_ctx *c, const hdr_camera *cam, int32_t frame_index,
                                  const hdr_path_settings *p) {
    if (!c || !p) return fail(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(c->mu);
    hdr_status st = check_camera(cam);
    if (st != HDR_OK) return st;
    if (!c->has_scene) return fail(HDR_ENOSCENE, "hdr_path_trace before hdr_scene_upload");
    if (p->max_depth < 1) return fail(HDR_EINVAL, "max_depth must be >= 1");
    if ((st = check_cancel(c)) != HDR_OK) return st;
    HDR_CUDA(cudaSetDevice(c->device));
    const size_t count = (size_t)cam->width * cam->height;
    hdr::GBufferView gb;
    if ((st = gbuffer_view(c, count, false, gb)) != HDR_OK) return st;
    void *color = nullptr;
    if ((st = ensure_buffer(c, "Color", count * 16, &color)) != HDR_OK) return st;
    hdr::PathParamsD d{};
    d.max_depth = p->max_depth;
    d.enable_subsurface = p->enable_subsurface;
    d.max_refl = p->max_reflection_bounces;
    d.max_refr = p->max_refraction_bounces;
    d.render_ibl_background = p->render_ibl_background;
    d.roulette = p->roulette_aggressiveness;
    hdr::CameraD cd = make_camera(cam);
    if ((st = record_frame_index(c, frame_index, &cd)) != HDR_OK) return st;
    // wavefront form: opaque scenes without the physical sky (whose sun needs a second
    // shadow ray per vertex, cast by the one-thread form)
    if (c->scene_opaque && !c->scene.sky && !(c->flags & HDR_CTX_PT_ONE_KERNEL)) {
        hdr::PtBuffers B{};
        if ((st = pt_buffers(c, count, B)) != HDR_OK) return st;
        if ((st = begin_pass(c, 1)) != HDR_OK) return st;
        hdr::PtJobD job{};
        job.cam = cd;
        job.gb = gb;
        job.color = (float4 *)color;
        job.err = c->d_err;
        job.pr = hdr::path_run_of(d);
        job.frame_index = frame_index;
        const int n = hdr::launch_path_trace_wavefront(c->scene, &job, 1, nullptr,
                                                       hdr::tile_blocks(cam->width, cam->height), B, c->tune,
                                                       c->d_err, c->stream);
        if (n < 0) return fail(HDR_ECUDA, "path trace launch failed: %s", cudaGetErrorString(cudaGetLastError()));
        c->launches += (uint64_t)n;
        return end_pass(c, 1);
    }
    if ((st = begin_pass(c, 1)) != HDR_OK) return st;
    hdr::launch_path_trace(c->scene, cd, frame_index, d, gb, (float4 *)color, c->d_err, c->stream);
    c->launches += 1;
    return end_pass(c, 1);
}

hdr_status hdr_path_trace_batch(hdr_ctx *const *ctxs, int32_t n, const hdr_camera *cams,
                                const int32_t *frame_indices, const hdr_path_settings *settings) {
    if (!ctxs || !cams || !frame_indices || !settings || n < 1 || n > 4096) return fail(HDR_EINVAL, "bad argument");
    for (int32_t i = 0; i < n; ++i)
        if (!ctxs[i]) return fail(HDR_EINVAL, "ctx %d is NULL", i);
    bool together = n > 1;
    for (int32_t i = 0; i < n && together; ++i)
        together = ctxs[i]->device == ctxs[0]->device && ctxs[i]->has_scene && ctxs[i]->scene_store &&
                   ctxs[i]->scene_store == ctxs[0]->scene_store && ctxs[i]->scene.wide == ctxs[0]->scene.wide;
    std::vector<hdr_ctx *> order(ctxs, ctxs + n);
    std::sort(order.begin(), order.end());
    if (std::adjacent_find(order.begin(), order.end()) != order.end())
        return fail(HDR_EINVAL, "a context appears twice in the batch");
    if (!together) {
        for (int32_t i = 0; i < n; ++i) {
            const hdr_status st = hdr_path_trace(ctxs[i], &cams[i], frame_indices[i], &settings[i]);
            if (st != HDR_OK) return st;
        }
        return HDR_OK;
    }
    for (hdr_ctx *c : order) c->mu.lock();
    struct Unlock {
        std::vector<hdr_ctx *> &v;
        ~Unlock() {
            for (hdr_ctx *c : v) c->mu.unlock();
        }
    } unlock{order};
    for (hdr_ctx *c : order) HDR_NOT_RECORDING(c, "hdr_path_trace_batch");
    hdr_ctx *lead = ctxs[0];
    HDR_CUDA(cudaSetDevice(lead->device));
    std::vector<hdr::PtJobD> jobs((size_t)n);
    long long tiles = 0;
    hdr_status st;
    for (int32_t i = 0; i < n; ++i) {
        hdr_ctx *c = ctxs[i];
        const hdr_camera *cam = &cams[i];
        const hdr_path_settings *p = &settings[i];
        if ((st = check_camera(cam)) != HDR_OK) return st;
        if (p->max_depth < 1) return fail(HDR_EINVAL, "max_depth must be >= 1");
        if ((st = check_cancel(c)) != HDR_OK) return st;
        const size_t count = (size_t)cam->width * cam->height;
        hdr::PtJobD &j = jobs[(size_t)i];
        if ((st = gbuffer_view(c, count, false, j.gb)) != HDR_OK) return st;
        void *color = nullptr;
        if ((st = ensure_buffer(c, "Color", count * 16, &color)) != HDR_OK) return st;
        hdr::PathParamsD d{};
        d.max_depth = p->max_depth;
        d.enable_subsurface = p->enable_subsurface;
        d.max_refl = p->max_reflection_bounces;
        d.max_refr = p->max_refraction_bounces;
        d.render_ibl_background = p->render_ibl_background;
        d.roulette = p->roulette_aggressiveness;
        j.cam = make_camera(cam);
        j.color = (float4 *)color;
        j.err = c->d_err;
        j.pr = hdr::path_run_of(d);
        j.frame_index = frame_indices[i];
        j.tile_begin = (int)tiles;
        tiles += (long long)hdr::tile_blocks(cam->width, cam->height);
    }
    if (tiles >= (1ll << 31)) return fail(HDR_EINVAL, "batch of %lld tiles is too large", tiles);
    // the wavefront form needs an opaque scene and one set of path settings for all images
    bool wave = lead->scene_opaque && !lead->scene.sky && !(lead->flags & HDR_CTX_PT_ONE_KERNEL);
    long long paths = 0;
    for (int32_t i = 0; i < n; ++i) {
        hdr::PtJobD &j = jobs[(size_t)i];
        j.pixel_begin = (int)paths;
        paths += (long long)j.cam.width * j.cam.height;
        wave = wave && std::memcmp(&settings[i], &settings[0], sizeof(hdr_path_settings)) == 0;
    }
    if (paths >= (1ll << 31)) return fail(HDR_EINVAL, "batch of %lld paths is too large", paths);
    // the path planes, queues and job table belong to the resident scene, as the RIS batch's queues
    // do: batches of changing images and leads (a server's steps) allocate nothing once large enough
    SceneStore *store = lead->scene_store.get();
    std::lock_guard<std::mutex> batch_lock(store->batch_mu);
    if (!store->pt_done) HDR_CUDA(cudaEventCreateWithFlags(&store->pt_done, cudaEventDisableTiming));
    for (cudaEvent_t &ev : store->pt_copied)
        if (!ev) HDR_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    auto alloc = [store, lead](const char *name, size_t bytes, void **p) {
        return ensure_batch_scratch(store, (std::string("pt") + name).c_str(), bytes, p, store->pt_done,
                                    lead->stream);
    };
    hdr::PtBuffers B{};
    if (wave && (st = pt_buffers_from(alloc, (size_t)paths, B)) != HDR_OK) return st;
    const size_t table_bytes = jobs.size() * sizeof(hdr::PtJobD);
    void *table = nullptr;
    if ((st = alloc("__jobs", table_bytes, &table)) != HDR_OK) return st;
    // the table goes up from pinned memory: one of two staging buffers, reused once the copy that
    // last read it has run, so the host never waits for the batch itself
    const int slot = store->pt_slot;
    store->pt_slot ^= 1;
    HDR_CUDA(cudaEventSynchronize(store->pt_copied[slot]));
    if (store->pt_table_cap[slot] < table_bytes) {
        if (store->pt_table_host[slot]) HDR_CUDA(cudaFreeHost(store->pt_table_host[slot]));
        store->pt_table_host[slot] = nullptr;
        store->pt_table_cap[slot] = 0;
        HDR_CUDA(cudaHostAlloc(&store->pt_table_host[slot], table_bytes, cudaHostAllocDefault));
        store->pt_table_cap[slot] = table_bytes;
    }
    std::memcpy(store->pt_table_host[slot], jobs.data(), table_bytes);
    // the previous batch on this scene (another lead's stream) has finished with the buffers, and
    // every image's earlier work (its raycast, on its own stream) is done
    HDR_CUDA(cudaStreamWaitEvent(lead->stream, store->pt_done, 0));
    for (int32_t i = 1; i < n; ++i) {
        HDR_CUDA(cudaEventRecord(ctxs[i]->sync_ev, ctxs[i]->stream));
        HDR_CUDA(cudaStreamWaitEvent(lead->stream, ctxs[i]->sync_ev, 0));
    }
    if ((st = begin_pass(lead, 1)) != HDR_OK) return st;
    HDR_CUDA(cudaMemcpyAsync(table, store->pt_table_host[slot], table_bytes, cudaMemcpyHostToDevice, lead->stream));
    HDR_CUDA(cudaEventRecord(store->pt_copied[slot], lead->stream));
    if (wave) {
        const int nl = hdr::launch_path_trace_wavefront(lead->scene, jobs.data(), n, (const hdr::PtJobD *)table,
                                                        (int)tiles, B, lead->tune, lead->d_err, lead->stream);
        if (nl < 0) return fail(HDR_ECUDA, "path trace launch failed: %s", cudaGetErrorString(cudaGetLastError()));
        lead->launches += (uint64_t)nl - 1;
    } else {
        hdr::launch_path_trace_batch(lead->scene, (const hdr::PtJobD *)table, n, (int)tiles, lead->stream);
    }
    HDR_CUDA(cudaGetLastError());
    HDR_CUDA(cudaEventRecord(lead->sync_ev, lead->stream));
    HDR_CUDA(cudaEventRecord(store->pt_done, lead->stream));
    for (int32_t i = 1; i < n; ++i) HDR_CUDA(cudaStreamWaitEvent(ctxs[i]->stream, lead->sync_ev, 0));
    lead->launches += 1;
    return end_pass(lead, 1);
}

static hdr_status accumulate_pass(hdr_ctx *c, int32_t frame_index, int32_t firefly, int32_t mode) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    if (mode != HDR_ACCUM_PARITY && mode != HDR_ACCUM_SHADER) return fail(HDR_EINVAL, "unknown accumulation mode");
    if (frame_index < 0) return fail(HDR_EINVAL, "frame_index must be >= 0");
    hdr_status st;
    if ((st = check_cancel(c)) != HDR_OK) return st;
    HDR_CUDA(cudaSetDevice(c->device));
    size_t bytes = 0;
    void *color = find_buffer(c, "Color", &bytes);
    if (!color || c->width <= 0 || bytes != (size_t)c->width * c->height * 16)
        return fail(HDR_EINVAL, "Color must be present (produced by PathTracePass) at the current frame size");
    const size_t count = (size_t)c->width * c->height;
    void *accum = nullptr, *scratch = nullptr;
    if ((st = ensure_buffer(c, "__accum_color", count * 16, &accum)) != HDR_OK) return st;
    if (firefly)
        if ((st = ensure_buffer(c, "__firefly_scratch", count * 16, &scratch)) != HDR_OK) return st;
    if ((st = record_frame_index(c, frame_index, nullptr)) != HDR_OK) return st;
    if ((st = begin_pass(c, 2)) != HDR_OK) return st;
    cudaError_t err = cudaSuccess;
    const int n = hdr::launch_accumulate((float4 *)color, (float4 *)accum, (float4 *)scratch, c->d_flag, c->width,
                                         c->height, frame_index, firefly, mode, c->stream, &err,
                                         c->recording ? c->d_frame_slot : nullptr);
    if (n < 0) return fail(HDR_ECUDA, "accumulation launch failed: %s", cudaGetErrorString(err));
    c->launches += (uint64_t)n;
    return end_pass(c, 2);
}

hdr_status hdr_clear_persistent(hdr_ctx *c) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_clear_persistent");
    HDR_CUDA(cudaSetDevice(c->device));
    for (const char *name : {"__accum_color", "__ris_reservoir", "__ris_reservoir_prev", "__prev_pos_depth"}) {
        auto it = c->buffers.find(name);
        if (it != c->buffers.end()) frame_free(c, it->second), c->buffers.erase(it);
    }
    c->reproj_valid = false;
    return HDR_OK;
}

hdr_status hdr_zero_persistent(hdr_ctx *c) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_CUDA(cudaSetDevice(c->device));
    for (const char *name : {"__accum_color", "__ris_reservoir", "__ris_reservoir_prev", "__prev_pos_depth"}) {
        auto it = c->buffers.find(name);
        if (it != c->buffers.end() && it->second.bytes)
            HDR_CUDA(cudaMemsetAsync(it->second.ptr, 0, it->second.bytes, c->stream));
    }
    c->reproj_valid = false;
    return HDR_OK;
}

hdr_status hdr_buffer_size(hdr_ctx *c, const char *name, size_t *bytes) {
    if (!c || !name || !bytes) return fail(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(c->mu);
    if (!find_buffer(c, name, bytes)) return fail(HDR_EINVAL, "no buffer named '%s'", name);
    return HDR_OK;
}

static hdr_status resolve_pass(hdr_ctx *c, const char *name, int32_t src_components, int32_t component_format,
                               int32_t dst_components, void *dst, size_t dst_bytes, int32_t dst_on_device) {
    if (!c || !name || (!dst && dst_bytes)) return fail(HDR_EINVAL, "NULL argument");
    if (src_components < 1 || src_components > 4 || dst_components < 1 || dst_components > 4)
        return fail(HDR_EINVAL, "components must be 1..4 (source %d, destination %d)", src_components,
                    dst_components);
    static const size_t kSize[] = {4, 2, 1, 1, 4};
    if (component_format < HDR_FMT_FLOAT32 || component_format > HDR_FMT_INT32)
        return fail(HDR_EINVAL, "unknown component format %d", component_format);
    std::lock_guard<std::mutex> lock(c->mu);
    if (!dst_on_device) HDR_NOT_RECORDING(c, "hdr_resolve into host memory");
    HDR_CUDA(cudaSetDevice(c->device));
    size_t have = 0;
    void *src = find_buffer(c, name, &have);
    if (!src) return fail(HDR_EINVAL, "no buffer named '%s'", name);
    if (std::strcmp(name, "GBuffer") == 0 || std::strncmp(name, "__", 2) == 0)
        return fail(HDR_EINVAL, "'%s' is not a float frame buffer", name);
    const size_t src_px = (size_t)src_components * sizeof(float);
    if (have % src_px != 0) return fail(HDR_EINVAL, "buffer '%s' (%zu bytes) is not %d floats per pixel", name, have,
                                        src_components);
    const size_t pixels = have / src_px;
    const size_t want = pixels * (size_t)dst_components * kSize[component_format];
    if (dst_bytes != want)
        return fail(HDR_EINVAL, "resolve of '%s' writes %zu bytes, %zu given", name, want, dst_bytes);
    // CopyFromFrameBuffer (hd_restir_render_buffer.cpp:117-127): a pixel of the frame buffer the size of a
    // render-buffer pixel is copied as bytes, whatever the formats
    if (src_px == (size_t)dst_components * kSize[component_format]) {
        if (want)
            HDR_CUDA(cudaMemcpyAsync(dst, src, want, dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                     c->stream));
        if (!dst_on_device) HDR_CUDA(cudaStreamSynchronize(c->stream));
        return HDR_OK;
    }
    void *out = dst;
    if (!dst_on_device && want) {  // converted on the device, then copied out
        hdr_status st = ensure_buffer(c, "__resolve_staging", want, &out);
        if (st != HDR_OK) return st;
    }
    const int n = hdr::launch_resolve((const float *)src, src_components, component_format, dst_components, out, pixels,
                                      c->tune.sm_count, c->stream);
    hdr_status st = HDR_OK;
    if (n < 0) st = fail(HDR_ECUDA, "resolve launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    c->launches += n > 0 ? (uint64_t)n : 0;
    if (!dst_on_device && want) {
        cudaError_t e = cudaSuccess;
        if (st == HDR_OK) e = cudaMemcpyAsync(dst, out, want, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (st == HDR_OK && e != cudaSuccess) st = fail(HDR_ECUDA, "resolve read-back: %s", cudaGetErrorString(e));
    }
    return st;
}

hdr_status hdr_upscale(hdr_ctx *c, const char *name, int32_t components, int32_t src_w, int32_t src_h,
                       int32_t dst_w, int32_t dst_h) {
    if (!c || !name) return fail(HDR_EINVAL, "NULL argument");
    if (components < 1 || components > 4 || src_w < 1 || src_h < 1 || dst_w < 1 || dst_h < 1 ||
        (size_t)dst_w * dst_h > ((size_t)1 << 31))
        return fail(HDR_EINVAL, "bad upscale sizes");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_upscale");
    HDR_CUDA(cudaSetDevice(c->device));
    auto it = c->buffers.find(name);
    if (it == c->buffers.end()) return fail(HDR_EINVAL, "no buffer named '%s'", name);
    const size_t want = (size_t)src_w * src_h * components * sizeof(float);
    if (it->second.bytes != want)
        return fail(HDR_EINVAL, "buffer '%s' holds %zu bytes, %d x %d x %d floats expected", name, it->second.bytes,
                    src_w, src_h, components);
    DevBuf nb;
    hdr_status st = frame_alloc(c, nb, (size_t)dst_w * dst_h * components * sizeof(float));
    if (st != HDR_OK) return st;
    if (hdr::launch_upscale((const float *)it->second.ptr, (float *)nb.ptr, components, src_w, src_h, dst_w, dst_h,
                            c->tune.sm_count, c->stream) < 0) {
        frame_free(c, nb);
        return fail(HDR_ECUDA, "upscale launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    c->launches += 1;
    frame_free(c, it->second);  // in stream order, after the upscale that reads it
    it->second = nb;
    return HDR_OK;
}

static hdr_status denoise_pass(hdr_ctx *c, const char *name, int32_t width, int32_t height,
                               int32_t chromaticity_blur) {
    if (!c || !name) return fail(HDR_EINVAL, "NULL argument");
    if (width < 0 || height < 0) return fail(HDR_EINVAL, "bad size");
    std::lock_guard<std::mutex> lock(c->mu);
    if (width == 0 || height == 0 || !chromaticity_blur) return HDR_OK;  // Denoiser::Run: nothing to do
    HDR_CUDA(cudaSetDevice(c->device));
    size_t have = 0;
    void *buf = find_buffer(c, name, &have);
    if (!buf) return fail(HDR_EINVAL, "no buffer named '%s'", name);
    const size_t bytes = (size_t)width * height * sizeof(float4);
    if (have != bytes) return fail(HDR_EINVAL, "buffer '%s' holds %zu bytes, %zu for RGBA %d x %d", name, have, bytes,
                                   width, height);
    void *tmp = nullptr;
    hdr_status st = ensure_buffer(c, "__denoise_scratch", bytes, &tmp);
    if (st != HDR_OK) return st;
    if (hdr::launch_chroma_blur((const float4 *)buf, (float4 *)tmp, width, height, c->tune.sm_count, c->stream) < 0)
        return fail(HDR_ECUDA, "denoise launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    HDR_CUDA(cudaMemcpyAsync(buf, tmp, bytes, cudaMemcpyDeviceToDevice, c->stream));
    c->launches += 1;
    return HDR_OK;
}

hdr_status hdr_download_async(hdr_ctx *c, const char *name, void *dst, size_t bytes) {
    if (!c || !name || (!dst && bytes)) return fail(HDR_EINVAL, "NULL argument");
    if (std::strcmp(name, "GBuffer") == 0) return fail(HDR_EINVAL, "GBuffer is read with hdr_download");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_download_async");
    HDR_CUDA(cudaSetDevice(c->device));
    size_t have = 0;
    void *src = find_buffer(c, name, &have);
    if (!src) return fail(HDR_EINVAL, "no buffer named '%s'", name);
    if (have != bytes) return fail(HDR_EINVAL, "buffer '%s' holds %zu bytes, %zu requested", name, have, bytes);
    if (!c->copy_stream) {
        HDR_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        HDR_CUDA(cudaEventCreateWithFlags(&c->copy_ready, cudaEventDisableTiming));
        HDR_CUDA(cudaEventCreateWithFlags(&c->copy_done, cudaEventDisableTiming));
        HDR_CUDA(cudaEventRecord(c->copy_done, c->copy_stream));
    }
    if (!bytes) return HDR_OK;
    size_t staged = 0;
    if (find_buffer(c, "__download_staging", &staged) && staged != bytes)
        HDR_CUDA(cudaEventSynchronize(c->copy_done));  // the staging buffer is about to be replaced
    void *snap = nullptr;
    hdr_status st = ensure_buffer(c, "__download_staging", bytes, &snap);
    if (st != HDR_OK) return st;
    // the previous read-back of the staging buffer ends before the next snapshot overwrites it
    HDR_CUDA(cudaStreamWaitEvent(c->stream, c->copy_done, 0));
    HDR_CUDA(cudaMemcpyAsync(snap, src, bytes, cudaMemcpyDeviceToDevice, c->stream));
    HDR_CUDA(cudaEventRecord(c->copy_ready, c->stream));
    HDR_CUDA(cudaStreamWaitEvent(c->copy_stream, c->copy_ready, 0));
    HDR_CUDA(cudaMemcpyAsync(dst, snap, bytes, cudaMemcpyDeviceToHost, c->copy_stream));
    HDR_CUDA(cudaEventRecord(c->copy_done, c->copy_stream));
    return HDR_OK;
}

hdr_status hdr_download_wait(hdr_ctx *c) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_download_wait");
    if (!c->copy_stream) return HDR_OK;
    HDR_CUDA(cudaSetDevice(c->device));
    HDR_CUDA(cudaStreamWaitEvent(c->stream, c->copy_done, 0));  // later work on the ctx stream follows the copy
    HDR_CUDA(cudaEventSynchronize(c->copy_done));
    return HDR_OK;
}

hdr_status hdr_download(hdr_ctx *c, const char *name, void *dst, size_t bytes) {
    if (!c || !name || (!dst && bytes)) return fail(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_download");
    HDR_CUDA(cudaSetDevice(c->device));
    size_t have = 0;
    void *src = find_buffer(c, name, &have);
    if (!src) return fail(HDR_EINVAL, "no buffer named '%s'", name);
    if (have != bytes) return fail(HDR_EINVAL, "buffer '%s' holds %zu bytes, %zu requested", name, have, bytes);
    if (std::strcmp(name, "GBuffer") == 0) {
        // planar float4 planes -> hdr_gbuffer_texel records
        const size_t count = have / (kGbPlanes * sizeof(float4));
        std::vector<float4> planes(count * kGbPlanes);
        HDR_CUDA(cudaMemcpyAsync(planes.data(), src, have, cudaMemcpyDeviceToHost, c->stream));
        HDR_CUDA(cudaStreamSynchronize(c->stream));
        hdr_gbuffer_texel *t = (hdr_gbuffer_texel *)dst;
        if (have != count * sizeof(hdr_gbuffer_texel))
            return fail(HDR_EINVAL, "GBuffer texel size mismatch");
        for (size_t i = 0; i < count; ++i) {
            const float4 a = planes[i], b = planes[count + i], s = planes[2 * count + i], al = planes[3 * count + i];
            const float4 x0 = planes[4 * count + i], x1 = planes[5 * count + i];
            hdr_gbuffer_texel &o = t[i];
            int prim, tri;
            std::memcpy(&prim, &b.w, 4);
            std::memcpy(&tri, &s.w, 4);
            o.position[0] = a.x, o.position[1] = a.y, o.position[2] = a.z, o.depth = a.w;
            o.normal[0] = b.x, o.normal[1] = b.y, o.normal[2] = b.z, o.prim_id = prim;
            o.smooth_normal[0] = s.x, o.smooth_normal[1] = s.y, o.smooth_normal[2] = s.z, o.tri_id = tri;
            o.albedo[0] = al.x, o.albedo[1] = al.y, o.albedo[2] = al.z, o.hit = prim >= 0 ? 1 : 0;
            o.uv[0] = al.w, o.uv[1] = x0.x;
            o.dpdu[0] = x0.y, o.dpdu[1] = x0.z, o.dpdu[2] = x0.w;
            o.dpdv[0] = x1.x, o.dpdv[1] = x1.y, o.dpdv[2] = x1.z;
        }
        return read_device_error(c);
    }
    HDR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
    HDR_CUDA(cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

hdr_status hdr_upload(hdr_ctx *c, const char *name, const void *src, size_t bytes) {
    if (!c || !name || (!src && bytes)) return fail(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_upload");
    HDR_CUDA(cudaSetDevice(c->device));
    if (std::strcmp(name, "GBuffer") == 0) return fail(HDR_EINVAL, "GBuffer is produced on the device only");
    void *dst = nullptr;
    hdr_status st = ensure_buffer(c, name, bytes, &dst);
    if (st != HDR_OK) return st;
    if (bytes) HDR_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
    return HDR_OK;
}

hdr_status hdr_synchronize(hdr_ctx *c) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_synchronize");
    HDR_CUDA(cudaSetDevice(c->device));
    HDR_CUDA(cudaStreamSynchronize(c->stream));
    return read_device_error(c);
}

hdr_status hdr_set_cancel(hdr_ctx *c, const volatile int32_t *flag) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    c->cancel = flag;
    return HDR_OK;
}

hdr_status hdr_trace_rays(hdr_ctx *c, const float *rays, const float *tmax, int32_t n, int32_t any_hit,
                          hdr_gbuffer_texel *out) {
    if (!c || (n > 0 && (!rays || !out)) || n < 0) return fail(HDR_EINVAL, "bad argument");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_trace_rays");
    if (!c->has_scene) return fail(HDR_ENOSCENE, "hdr_trace_rays before hdr_scene_upload");
    if (n == 0) return HDR_OK;
    HDR_CUDA(cudaSetDevice(c->device));
    static_assert(sizeof(hdr_gbuffer_texel) == 96, "texel layout");
    DevBuf dr, dt, dout;
    hdr_status st;
    if ((st = dev_alloc(c, dr, (size_t)n * 24)) != HDR_OK) return st;
    if ((st = dev_alloc(c, dt, tmax ? (size_t)n * 4 : 0)) != HDR_OK) return dev_free(c, dr), st;
    if ((st = dev_alloc(c, dout, (size_t)n * 96)) != HDR_OK) return dev_free(c, dr), dev_free(c, dt), st;
    cudaError_t e = cudaMemcpyAsync(dr.ptr, rays, (size_t)n * 24, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && tmax) e = cudaMemcpyAsync(dt.ptr, tmax, (size_t)n * 4, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        hdr::launch_trace_rays(c->scene, (const float *)dr.ptr, tmax ? (const float *)dt.ptr : nullptr, n, any_hit,
                               (float4 *)dout.ptr, c->d_err, c->stream);
        c->launches += 1;
        e = cudaGetLastError();
    }
    std::vector<float4> raw;
    if (e == cudaSuccess) {
        raw.resize((size_t)n * 6);
        e = cudaMemcpyAsync(raw.data(), dout.ptr, (size_t)n * 96, cudaMemcpyDeviceToHost, c->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dev_free(c, dr);
    dev_free(c, dt);
    dev_free(c, dout);
    if (e != cudaSuccess) return fail(HDR_ECUDA, "hdr_trace_rays: %s", cudaGetErrorString(e));
    for (int32_t k = 0; k < n; ++k) {
        const float4 *r = &raw[(size_t)k * 6];
        hdr_gbuffer_texel &o = out[k];
        int prim, tri, hit;
        std::memcpy(&prim, &r[1].w, 4);
        std::memcpy(&tri, &r[2].w, 4);
        std::memcpy(&hit, &r[3].w, 4);
        o.position[0] = r[0].x, o.position[1] = r[0].y, o.position[2] = r[0].z, o.depth = r[0].w;
        o.normal[0] = r[1].x, o.normal[1] = r[1].y, o.normal[2] = r[1].z, o.prim_id = prim;
        o.smooth_normal[0] = r[2].x, o.smooth_normal[1] = r[2].y, o.smooth_normal[2] = r[2].z, o.tri_id = tri;
        o.albedo[0] = r[3].x, o.albedo[1] = r[3].y, o.albedo[2] = r[3].z, o.hit = hit;
        o.uv[0] = r[4].x, o.uv[1] = r[4].y;
        o.dpdu[0] = r[4].z, o.dpdu[1] = r[4].w, o.dpdu[2] = r[5].x;
        o.dpdv[0] = r[5].y, o.dpdv[1] = r[5].z, o.dpdv[2] = r[5].w;
    }
    return read_device_error(c);
}

hdr_status hdr_trace_stats(hdr_ctx *c, const float *rays, const float *tmax, int32_t n, int32_t walk,
                           int32_t *out) {
    if (!c || (n > 0 && (!rays || !out)) || n < 0 || walk < 0 || walk > 5) return fail(HDR_EINVAL, "bad argument");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_trace_stats");
    if (!c->has_scene) return fail(HDR_ENOSCENE, "hdr_trace_stats before hdr_scene_upload");
    if (walk >= 4 && !c->scene.sh4) return fail(HDR_EINVAL, "walk %d: the scene has no 4-wide SAH trees on this ctx", walk);
    if (n == 0) return HDR_OK;
    HDR_CUDA(cudaSetDevice(c->device));
    DevBuf dr, dt, dout;
    hdr_status st;
    if ((st = dev_alloc(c, dr, (size_t)n * 24)) != HDR_OK) return st;
    if ((st = dev_alloc(c, dt, tmax ? (size_t)n * 4 : 0)) != HDR_OK) return dev_free(c, dr), st;
    if ((st = dev_alloc(c, dout, (size_t)n * 16)) != HDR_OK) return dev_free(c, dr), dev_free(c, dt), st;
    cudaError_t e = cudaMemcpyAsync(dr.ptr, rays, (size_t)n * 24, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && tmax) e = cudaMemcpyAsync(dt.ptr, tmax, (size_t)n * 4, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        hdr::launch_trace_stats(c->scene, (const float *)dr.ptr, tmax ? (const float *)dt.ptr : nullptr, n, walk,
                                (int4 *)dout.ptr, c->d_err, c->stream);
        c->launches += 1;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout.ptr, (size_t)n * 16, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dev_free(c, dr);
    dev_free(c, dt);
    dev_free(c, dout);
    if (e != cudaSuccess) return fail(HDR_ECUDA, "hdr_trace_stats: %s", cudaGetErrorString(e));
    return read_device_error(c);
}

hdr_status hdr_get_trace_tuning(hdr_ctx *c, hdr_trace_tuning *out) {
    if (!c || !out) return fail(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(c->mu);
    out->node_quorum = c->tune.node_quorum;
    out->blocks_per_sm = c->tune.blocks_per_sm;
    out->trace_ms = 0.0f;
    out->shade_shape = c->tune.shade_shape;
    out->shadow_shape = c->tune.shadow_shape;
    out->shade_ms = 0.0f;
    return HDR_OK;
}

hdr_status hdr_set_trace_tuning(hdr_ctx *c, const hdr_trace_tuning *t) {
    if (!c || !t) return fail(HDR_EINVAL, "NULL argument");
    if (t->node_quorum < 1 || t->node_quorum > 32 || t->blocks_per_sm < 1 || t->blocks_per_sm > 64 ||
        t->shade_shape < 0 || t->shade_shape >= hdr::kShadeShapes || t->shadow_shape < 0 ||
        t->shadow_shape >= hdr::kShadowShapes)
        return fail(HDR_EINVAL, "node_quorum must be 1..32, blocks_per_sm 1..64, shade_shape 0..%d, shadow_shape 0..%d",
                    hdr::kShadeShapes - 1, hdr::kShadowShapes - 1);
    std::lock_guard<std::mutex> lock(c->mu);
    c->tune.node_quorum = t->node_quorum;
    c->tune.blocks_per_sm = t->blocks_per_sm;
    c->tune.shade_shape = t->shade_shape;
    c->tune.shadow_shape = t->shadow_shape;
    return HDR_OK;
}

hdr_status hdr_autotune_trace(hdr_ctx *c, hdr_trace_tuning *best) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_autotune_trace");
    if (!c->have_wave || !c->has_scene)
        return fail(HDR_EINVAL, "hdr_autotune_trace needs a previous wavefront hdr_ris_path_trace on this ctx");
    HDR_CUDA(cudaSetDevice(c->device));
    hdr::TraceTuning pick;
    float pick_ms = 0.0f;
    hdr_status st = search_trace_schedule(c, c->last_wave, pick, pick_ms);
    if (st != HDR_OK) return st;
    c->tune.node_quorum = pick.node_quorum;
    c->tune.blocks_per_sm = pick.blocks_per_sm;
    c->tune.shadow_shape = pick.shadow_shape;
    if (best) {
        best->node_quorum = pick.node_quorum;
        best->blocks_per_sm = pick.blocks_per_sm;
        best->trace_ms = pick_ms;
        best->shade_shape = c->tune.shade_shape;
        best->shadow_shape = c->tune.shadow_shape;
        best->shade_ms = 0.0f;  // not measured here (hdr_autotune_frame measures it)
    }
    return read_device_error(c);
}

hdr_status hdr_autotune_frame(hdr_ctx *c, const hdr_camera *cam, int32_t frame_index, const hdr_ris_params *p,
                              hdr_trace_tuning *best) {
    hdr_trace_tuning local{};
    hdr_status st = ris_path_trace_pass(c, cam, frame_index, p, best ? best : &local);
    if (st != HDR_OK) return st;
    std::lock_guard<std::mutex> lock(c->mu);
    return read_device_error(c);
}

hdr_status hdr_rng_floats(hdr_ctx *c, const uint32_t *seeds, int32_t n_seeds, int32_t count, float *out) {
    if (!c || n_seeds < 0 || count < 0 || (n_seeds > 0 && (!seeds || !out))) return fail(HDR_EINVAL, "bad argument");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_rng_floats");
    if (n_seeds == 0 || count == 0) return HDR_OK;
    HDR_CUDA(cudaSetDevice(c->device));
    DevBuf ds, dout;
    hdr_status st;
    if ((st = dev_alloc(c, ds, (size_t)n_seeds * 4)) != HDR_OK) return st;
    if ((st = dev_alloc(c, dout, (size_t)n_seeds * count * 4)) != HDR_OK) return dev_free(c, ds), st;
    cudaError_t e = cudaMemcpyAsync(ds.ptr, seeds, (size_t)n_seeds * 4, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        hdr::launch_rng_floats((const uint32_t *)ds.ptr, n_seeds, count, (float *)dout.ptr, c->stream);
        c->launches += 1;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, dout.ptr, (size_t)n_seeds * count * 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    dev_free(c, ds);
    dev_free(c, dout);
    if (e != cudaSuccess) return fail(HDR_ECUDA, "hdr_rng_floats: %s", cudaGetErrorString(e));
    return HDR_OK;
}

hdr_status hdr_pass_times(hdr_ctx *c, float *avg_ms, int32_t *counts, int32_t n, int32_t reset) {
    if (!c || (n > 0 && (!avg_ms || !counts))) return fail(HDR_EINVAL, "bad argument");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_pass_times");
    for (int k = 0; k < kTimeSlots; ++k) {
        hdr_status st = fold_pass_time(c, k);
        if (st != HDR_OK) return st;
    }
    for (int i = 0; i < n && i < kTimeSlots; ++i) {
        avg_ms[i] = c->pass_count[i] ? (float)(c->pass_sum_ms[i] / c->pass_count[i]) : 0.0f;
        counts[i] = c->pass_count[i];
    }
    if (reset)
        for (int k = 0; k < kTimeSlots; ++k) c->pass_sum_ms[k] = 0.0, c->pass_count[k] = 0;
    return HDR_OK;
}

hdr_status hdr_region_begin(hdr_ctx *c, int32_t slot) {
    if (!c || slot < 0 || slot >= 4) return fail(HDR_EINVAL, "bad region slot");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_region_begin");
    HDR_CUDA(cudaEventRecord(c->region_ev[slot][0], c->stream));
    return HDR_OK;
}

hdr_status hdr_region_end(hdr_ctx *c, int32_t slot) {
    if (!c || slot < 0 || slot >= 4) return fail(HDR_EINVAL, "bad region slot");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_region_end");
    HDR_CUDA(cudaEventRecord(c->region_ev[slot][1], c->stream));
    return HDR_OK;
}

hdr_status hdr_region_elapsed(hdr_ctx *c, int32_t slot, float *ms) {
    if (!c || !ms || slot < 0 || slot >= 4) return fail(HDR_EINVAL, "bad argument");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_region_elapsed");
    HDR_CUDA(cudaEventSynchronize(c->region_ev[slot][1]));
    HDR_CUDA(cudaEventElapsedTime(ms, c->region_ev[slot][0], c->region_ev[slot][1]));
    return HDR_OK;
}

hdr_status hdr_trim_frame_memory(int32_t device, size_t keep_bytes) {
    int ndev = 0;
    HDR_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(HDR_EINVAL, "device %d not present (%d devices)", device, ndev);
    int prev = 0;
    HDR_CUDA(cudaGetDevice(&prev));
    HDR_CUDA(cudaSetDevice(device));
    cudaMemPool_t pool = frame_pool(device);
    const cudaError_t e = pool ? cudaMemPoolTrimTo(pool, keep_bytes) : cudaErrorMemoryAllocation;
    cudaSetDevice(prev);
    if (e != cudaSuccess) return fail(HDR_ECUDA, "trimming the frame-buffer pool: %s", cudaGetErrorString(e));
    return HDR_OK;
}

hdr_status hdr_launch_count(hdr_ctx *c, uint64_t *count) {
    if (!c || !count) return fail(HDR_EINVAL, "bad argument");
    std::lock_guard<std::mutex> lock(c->mu);
    *count = c->recording ? c->rec_launches0 : c->launches;  // recorded kernels count when the graph runs
    return HDR_OK;
}

// A frame's pass chain as one CUDA graph. The passes' kernels take the frame
// index and the camera by value, so a new frame is recorded again (stream
// capture records launches without submitting them) and the executable graph
// is updated in place (cudaGraphExecUpdate) rather than instantiated anew.
hdr_status hdr_graph_begin(hdr_ctx *c) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    if (c->recording) return fail(HDR_EINVAL, "the ctx is already recording");
    HDR_CUDA(cudaSetDevice(c->device));
    HDR_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    c->recording = true;
    c->rec_failed = false;
    c->rec_has_frame = false;
    c->rec_launches0 = c->launches;
    return HDR_OK;
}

hdr_status hdr_graph_end(hdr_ctx *c) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    if (!c->recording) return fail(HDR_EINVAL, "hdr_graph_end without hdr_graph_begin");
    HDR_CUDA(cudaSetDevice(c->device));
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->recording = false;
    const uint64_t kernels = c->launches - c->rec_launches0;
    c->launches = c->rec_launches0;  // the recorded kernels run at hdr_graph_launch
    if (e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
        return fail(HDR_ECUDA, "recording failed (a recorded call was not capturable): %s", cudaGetErrorString(e));
    }
    if (c->rec_failed) {  // the record lacks a failed pass's work: discarded, the previous graph is kept
        cudaGraphDestroy(g);
        return fail(HDR_EINVAL, "a pass failed while recording; the recording is discarded");
    }
    if (c->graph_exec) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(c->graph_exec, g, &info) == cudaSuccess) {
            c->graph_updates += 1;
        } else {  // another chain (other passes, sizes or launch shapes): instantiate it
            (void)cudaGetLastError();
            cudaGraphExecDestroy(c->graph_exec);
            c->graph_exec = nullptr;
        }
    }
    if (!c->graph_exec) {
        e = cudaGraphInstantiate(&c->graph_exec, g, 0);
        if (e != cudaSuccess) {
            c->graph_exec = nullptr;
            cudaGraphDestroy(g);
            return fail(HDR_ECUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
        }
        c->graph_instantiations += 1;
    }
    cudaGraphDestroy(g);
    c->graph_kernels = kernels;
    c->graph_has_frame = c->rec_has_frame;
    c->graph_frame = c->rec_frame;
    return HDR_OK;
}

hdr_status hdr_graph_launch(hdr_ctx *c, int32_t frame_index) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    HDR_NOT_RECORDING(c, "hdr_graph_launch");
    if (!c->graph_exec) return fail(HDR_EINVAL, "no recorded graph (hdr_graph_begin / hdr_graph_end)");
    hdr_status st;
    if ((st = check_cancel(c)) != HDR_OK) return st;
    HDR_CUDA(cudaSetDevice(c->device));
    if (c->graph_has_frame) {  // the frame the recorded passes render, read by their kernels
        set_frame_slot_kernel<<<1, 1, 0, c->stream>>>(c->d_frame_slot, frame_index >= 0 ? frame_index
                                                                                       : c->graph_frame);
        HDR_CUDA(cudaGetLastError());
        c->launches += 1;
    }
    HDR_CUDA(cudaGraphLaunch(c->graph_exec, c->stream));
    c->launches += c->graph_kernels;
    return HDR_OK;
}

// The passes a graph may record. One that fails while its ctx records leaves
// the record without its work, so the recording is marked and hdr_graph_end
// discards it.
static hdr_status noted(hdr_ctx *c, hdr_status st) {
    if (st != HDR_OK && c) {
        std::lock_guard<std::mutex> lock(c->mu);
        if (c->recording) c->rec_failed = true;
    }
    return st;
}
hdr_status hdr_raycast(hdr_ctx *c, const hdr_camera *cam, int32_t frame_index, uint32_t aov_mask) {
    return noted(c, raycast_pass(c, cam, frame_index, aov_mask));
}
hdr_status hdr_ris_path_trace(hdr_ctx *c, const hdr_camera *cam, int32_t frame_index, const hdr_ris_params *p) {
    return noted(c, ris_path_trace_pass(c, cam, frame_index, p));
}
hdr_status hdr_path_trace(hdr_ctx *c, const hdr_camera *cam, int32_t frame_index, const hdr_path_settings *p) {
    return noted(c, path_trace_pass(c, cam, frame_index, p));
}
hdr_status hdr_accumulate(hdr_ctx *c, int32_t frame_index, int32_t firefly, int32_t mode) {
    return noted(c, accumulate_pass(c, frame_index, firefly, mode));
}
hdr_status hdr_resolve(hdr_ctx *c, const char *name, int32_t src_components, int32_t component_format,
                       int32_t dst_components, void *dst, size_t dst_bytes, int32_t dst_on_device) {
    return noted(c, resolve_pass(c, name, src_components, component_format, dst_components, dst, dst_bytes,
                                 dst_on_device));
}
hdr_status hdr_denoise(hdr_ctx *c, const char *name, int32_t width, int32_t height, int32_t chromaticity_blur) {
    return noted(c, denoise_pass(c, name, width, height, chromaticity_blur));
}

hdr_status hdr_graph_info(hdr_ctx *c, int32_t *kernels, int32_t *instantiations, int32_t *updates) {
    if (!c) return fail(HDR_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lock(c->mu);
    if (kernels) *kernels = (int32_t)c->graph_kernels;
    if (instantiations) *instantiations = c->graph_instantiations;
    if (updates) *updates = c->graph_updates;
    return HDR_OK;
}

}  // extern "C"
