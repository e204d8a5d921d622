// AccumulationPass::_execute (passes/accumulation_pass.cpp:64-139) and
// GpuAccumulationPass (gpu_functions/shaders/accumulation.slang:39-97):
// optional 3x3 firefly clamp (luminance > 4 x neighbourhood max + 0.5), then
// accum += Color, Color = accum * (1 / (frameIndex + 1)).
//
// The CPU pass clamps in place in row-major order, so a pixel sees its four
// earlier neighbours already clamped; the shader clamps against the unclamped
// input. For colours with non-negative luminance the two agree: if an earlier
// neighbour q was clamped then lum(q) > 4 lum(p) + 0.5 (p is q's neighbour),
// and its clamped luminance stays >= 4 lum(p) + 0.5, so p is not clamped in
// either order. Parity mode therefore runs the parallel clamp, verifies that
// no pixel's decision changes under the in-place order, and only if one does
// (possible for negative or non-finite inputs) iterates the in-place rule to
// its fixed point, which is the sequential result because the dependencies
// only point backwards in row-major order.
#include <cuda_runtime.h>

#include <algorithm>

#include "device/gf.cuh"

namespace hdr {

__device__ __forceinline__ float lum4(float4 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

__device__ __forceinline__ bool same_bits(float4 a, float4 b) {
    return __float_as_int(a.x) == __float_as_int(b.x) && __float_as_int(a.y) == __float_as_int(b.y) &&
           __float_as_int(a.z) == __float_as_int(b.z) && __float_as_int(a.w) == __float_as_int(b.w);
}

// One firefly pass. Neighbours earlier in row-major order come from `prev`
// (when given), later ones (and the pixel itself) from `orig`.
__global__ void __launch_bounds__(256) firefly_kernel(const float4 *__restrict__ orig, const float4 *prev,
                                                      float4 *dst, int width, int height, int *changed) {
    const int x = blockIdx.x * 16 + (threadIdx.x & 15);
    const int y = blockIdx.y * 16 + (threadIdx.x >> 4);
    if (x >= width || y >= height) return;
    const size_t p = (size_t)y * width + x;
    float4 c = orig[p];
    const float lum = lum4(c);
    float max_n = 0.0f;
    for (int dy = -1; dy <= 1; ++dy) {
        for (int dx = -1; dx <= 1; ++dx) {
            if (dx == 0 && dy == 0) continue;
            const int nx = sclampi(x + dx, 0, width - 1);
            const int ny = sclampi(y + dy, 0, height - 1);
            const size_t q = (size_t)ny * width + nx;
            const float4 v = (prev && q < p) ? prev[q] : orig[q];
            max_n = smaxf(max_n, lum4(v));
        }
    }
    const float thr = max_n * 4.0f + 0.5f;
    if (lum > thr && lum > 0.0f) {
        const float scale = thr / lum;
        c.x *= scale;
        c.y *= scale;
        c.z *= scale;
    }
    if (dst) dst[p] = c;
    if (changed && prev && !same_bits(c, prev[p])) atomicOr(changed, 1);
}

__global__ void __launch_bounds__(256) accumulate_kernel(const float4 *__restrict__ in, float4 *__restrict__ accum,
                                                         float4 *__restrict__ out, size_t count, float inv_n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        const float4 c = in[i];
        float4 a = accum[i];
        a.x += c.x;
        a.y += c.y;
        a.z += c.z;
        a.w += c.w;
        accum[i] = a;
        out[i] = make_float4(a.x * inv_n, a.y * inv_n, a.z * inv_n, a.w * inv_n);
    }
}

// Returns the number of kernels launched, or -1 on a CUDA error.
// scratch holds two float4 planes of width*height (only used with firefly).
int launch_accumulate(float4 *color, float4 *accum, float4 *scratch, int *flag_dev, int width, int height,
                      int frame_index, int firefly, int mode, cudaStream_t st) {
    const size_t count = (size_t)width * height;
    const float inv_n = 1.0f / (float)(frame_index + 1);
    int launches = 0;
    const float4 *src = color;
    if (firefly) {
        const dim3 grid((width + 15) / 16, (height + 15) / 16);
        float4 *a = scratch, *b = scratch + count;
        firefly_kernel<<<grid, 256, 0, st>>>(color, nullptr, a, width, height, nullptr);
        ++launches;
        src = a;
        if (mode == 0) {
            // in-place-order check; the fallback loop runs only when it fails
            if (cudaMemsetAsync(flag_dev, 0, sizeof(int), st) != cudaSuccess) return -1;
            firefly_kernel<<<grid, 256, 0, st>>>(color, a, nullptr, width, height, flag_dev);
            ++launches;
            int changed = 0;
            if (cudaMemcpyAsync(&changed, flag_dev, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return -1;
            if (cudaStreamSynchronize(st) != cudaSuccess) return -1;
            for (size_t iter = 0; changed && iter < count; ++iter) {
                if (cudaMemsetAsync(flag_dev, 0, sizeof(int), st) != cudaSuccess) return -1;
                firefly_kernel<<<grid, 256, 0, st>>>(color, a, b, width, height, flag_dev);
                ++launches;
                if (cudaMemcpyAsync(&changed, flag_dev, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess)
                    return -1;
                if (cudaStreamSynchronize(st) != cudaSuccess) return -1;
                float4 *t = a;
                a = b;
                b = t;
            }
            src = a;
        }
    }
    const int blocks = (int)std::min<size_t>((count + 255) / 256, (size_t)148 * 8);
    accumulate_kernel<<<blocks > 0 ? blocks : 1, 256, 0, st>>>(src, accum, color, count, inv_n);
    ++launches;
    if (cudaGetLastError() != cudaSuccess) return -1;
    return launches;
}

}  // namespace hdr
