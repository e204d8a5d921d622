// hdr_accumulate_noalloc: the accumulation pass (firefly clamp + running mean,
// the same kernels and launch sequence as hdr_accumulate) on caller-owned
// device planes, with no device allocation on any call.
//
// Who needs it: callers that may not allocate device memory at the moment they
// accumulate. Examples are a host renderer that runs the pass inside its own
// memory-pool budget, where a cudaMalloc would fail, and one that cannot pay
// the device-wide synchronisation a cudaMalloc/cudaFree may cause between
// frames. hdr_accumulate keeps its scratch in context-owned buffers that it
// grows on demand. This entry point instead takes the firefly scratch (one RGBA
// f32 plane) and the in-place-order flag from a file-scope __device__ array of
// fixed size.
//
// Limits and set-up:
//  * at most kNoAllocMaxPixels = 2,097,152 pixels (2^21, covers 1920x1080)
//    when the firefly clamp is on; larger frames are rejected with HDR_EINVAL.
//    Without the clamp any size is accepted (the scratch is not used).
//  * the scratch is 32 MiB of static device memory, held until the process
//    exits on every GPU that loads this module. With CUDA's lazy module loading
//    (the default; CUDA_MODULE_LOADING=LAZY) that happens at the first call on a
//    device; with eager loading (CUDA_MODULE_LOADING=EAGER) when the process
//    creates its context on that device, whether or not this entry point is
//    ever called. Either way the memory is outside every hdr_ctx's
//    hbm_budget_bytes and the server's admission budget.
//  * the first call on a device (made with that device current) resolves the
//    scratch address with cudaGetSymbolAddress, which loads this module. Make
//    one call per device (any size, e.g. 1x1 with firefly on) before any stream
//    capture or allocation-restricted region if the module load must not happen
//    there. The address is cached per device together with the CUDA context it
//    was resolved in; a call in a new context (after cudaDeviceReset, say)
//    resolves it again.
//  * neither mode reads anything back to the host or waits for the stream: the
//    in-place-order check and its fallback run on the device.
//  * nothing in the scratch has to start at zero: the clamp pass writes the
//    plane in full before anything reads it, and the flag is zeroed on the
//    stream before every use. The caller's accum plane must be zero before
//    frame 0, as "__accum_color" is after hdr_clear_persistent.
//  * one scratch per device, shared by all callers: calls that overlap on the
//    same device (different streams or host threads) race on it. Serialise
//    them.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/hdrestir.h"

namespace hdr {
int launch_accumulate(float4 *color, float4 *accum, float4 *scratch, int *flag_dev, int width, int height,
                      int frame_index, int firefly, int mode, cudaStream_t st, cudaError_t *err,
                      const int *frame_slot);
hdr_status set_last_error(hdr_status st, const char *fmt, ...);
}  // namespace hdr

namespace {

constexpr size_t kNoAllocMaxPixels = size_t(1) << 21;

// one plane of kNoAllocMaxPixels RGBA f32 (the clamped frame)
static __device__ __align__(256) float4 g_accum_scratch[kNoAllocMaxPixels];
static __device__ __align__(256) int g_accum_flag[64];

constexpr int kMaxDevices = 64;

struct ScratchAddr {
    float4 *planes = nullptr;
    int *flag = nullptr;
    CUcontext ctx = nullptr;  // the context the addresses belong to
};

std::mutex g_addr_mu;
ScratchAddr g_addr[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext *);

// cuCtxGetCurrent through the runtime's driver entry point (no link to libcuda).
CUcontext current_context() {
    static CtxGetCurrentFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    CUcontext c = nullptr;
    if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
    return c;
}

// Resolves this device's scratch address once per context (the current device
// must be `dev`, with its context current).
hdr_status scratch_for(int dev, ScratchAddr &out) {
    std::lock_guard<std::mutex> lock(g_addr_mu);
    ScratchAddr &a = g_addr[dev];
    const CUcontext now = current_context();
    if (!a.planes || a.ctx != now) {
        void *planes = nullptr, *flag = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&planes, g_accum_scratch);
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&flag, g_accum_flag);
        if (e != cudaSuccess)
            return hdr::set_last_error(HDR_ECUDA, "cudaGetSymbolAddress(accumulation scratch) on device %d: %s", dev,
                                       cudaGetErrorString(e));
        a.planes = static_cast<float4 *>(planes);
        a.flag = static_cast<int *>(flag);
        a.ctx = current_context();  // the symbol lookup may have created the primary context
    }
    out = a;
    return HDR_OK;
}

}  // namespace

extern "C" hdr_status hdr_accumulate_noalloc(float *color, float *accum, int32_t width, int32_t height,
                                             int32_t frame_index, int32_t firefly, int32_t mode, void *stream) {
    if (!color || !accum) return hdr::set_last_error(HDR_EINVAL, "color and accum must be device pointers");
    if (width <= 0 || height <= 0) return hdr::set_last_error(HDR_EINVAL, "bad frame size %dx%d", width, height);
    if (mode != HDR_ACCUM_PARITY && mode != HDR_ACCUM_SHADER)
        return hdr::set_last_error(HDR_EINVAL, "unknown accumulation mode");
    if (frame_index < 0) return hdr::set_last_error(HDR_EINVAL, "frame_index must be >= 0");
    const size_t count = (size_t)width * (size_t)height;
    if (firefly && count > kNoAllocMaxPixels)
        return hdr::set_last_error(HDR_EINVAL,
                                   "frame of %zu pixels exceeds the no-alloc firefly scratch (%zu pixels); "
                                   "use hdr_accumulate",
                                   count, kNoAllocMaxPixels);
    if ((reinterpret_cast<uintptr_t>(color) | reinterpret_cast<uintptr_t>(accum)) & 15)
        return hdr::set_last_error(HDR_EINVAL, "color and accum must be 16-byte aligned");
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return hdr::set_last_error(HDR_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return hdr::set_last_error(HDR_EINVAL, "device %d out of range", dev);
    ScratchAddr s;
    const hdr_status st = scratch_for(dev, s);
    if (st != HDR_OK) return st;
    const int n = hdr::launch_accumulate(reinterpret_cast<float4 *>(color), reinterpret_cast<float4 *>(accum),
                                         s.planes, s.flag, width, height, frame_index, firefly, mode,
                                         static_cast<cudaStream_t>(stream), &e, nullptr);
    if (n < 0) return hdr::set_last_error(HDR_ECUDA, "accumulation launch failed: %s", cudaGetErrorString(e));
    return HDR_OK;
}
