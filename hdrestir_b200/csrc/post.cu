// Post passes on the device.
//   UpscalePass (passes/upscale_pass.cpp:13-95): nearest-pixel upscale of a
//     frame rendered at a reduced resolution level to the window size,
//     srcX = min(srcW - 1, dstX * srcW / dstW) in integers, same for y.
//   Denoiser without OIDN (passes/denoiser.cpp:54-96,164-201): the
//     chromaticity blur, which keeps each pixel's luma Y = r/4 + g/2 + b/4 and
//     replaces its chroma (Co, Cg) by the mean over the 3x3 neighbourhood
//     (clamped at the borders), accumulated in the reference's order; alpha is
//     kept. OIDN itself is not part of this library.
// Both are one thread per output pixel and HBM-bound.
#include "device/frame.cuh"

namespace hdr {
namespace {

__global__ void upscale_kernel(const float *__restrict__ src, float *__restrict__ dst, int comps, int src_w,
                               int src_h, int dst_w, int dst_h) {
    const size_t n = (size_t)dst_w * (size_t)dst_h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % (size_t)dst_w), y = (int)(i / (size_t)dst_w);
        const int sx = min(src_w - 1, (int)((long long)x * src_w / dst_w));
        const int sy = min(src_h - 1, (int)((long long)y * src_h / dst_h));
        const size_t s = ((size_t)sy * (size_t)src_w + (size_t)sx) * (size_t)comps;
        for (int c = 0; c < comps; ++c) dst[i * (size_t)comps + c] = src[s + c];
    }
}

__device__ __forceinline__ float ref_max0(float v) { return (0.0f < v) ? v : 0.0f; }  // std::max(0.0f, v)

__global__ void chroma_blur_kernel(const float4 *__restrict__ src, float4 *__restrict__ dst, int w, int h) {
    const size_t n = (size_t)w * (size_t)h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % (size_t)w), y = (int)(i / (size_t)w);
        const float4 p = src[i];
        const float Y = 0.25f * p.x + 0.5f * p.y + 0.25f * p.z;
        float sum_co = 0.0f, sum_cg = 0.0f, weight = 0.0f;
        for (int dy = -1; dy <= 1; ++dy) {
            for (int dx = -1; dx <= 1; ++dx) {
                const int nx = min(max(x + dx, 0), w - 1), ny = min(max(y + dy, 0), h - 1);
                const float4 q = src[(size_t)ny * (size_t)w + (size_t)nx];
                sum_co += 0.50f * q.x - 0.5f * q.z;
                sum_cg += -0.25f * q.x + 0.5f * q.y - 0.25f * q.z;
                weight += 1.0f;
            }
        }
        const float co = sum_co / weight, cg = sum_cg / weight;
        dst[i] = make_float4(ref_max0(Y + co - cg), ref_max0(Y + cg), ref_max0(Y - co - cg), p.w);
    }
}

int grid_for(size_t n, int sm_count) {
    return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)sm_count * 8));
}

}  // namespace

int launch_upscale(const float *src, float *dst, int comps, int src_w, int src_h, int dst_w, int dst_h, int sm_count,
                   cudaStream_t st) {
    upscale_kernel<<<grid_for((size_t)dst_w * dst_h, sm_count), 256, 0, st>>>(src, dst, comps, src_w, src_h, dst_w,
                                                                              dst_h);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

int launch_chroma_blur(const float4 *src, float4 *dst, int w, int h, int sm_count, cudaStream_t st) {
    chroma_blur_kernel<<<grid_for((size_t)w * h, sm_count), 256, 0, st>>>(src, dst, w, h);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

}  // namespace hdr
