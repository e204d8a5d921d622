// AccumulationPass::_execute (passes/accumulation_pass.cpp:64-139) and
// GpuAccumulationPass (gpu_functions/shaders/accumulation.slang:39-97):
// optional 3x3 firefly clamp (luminance > 4 x neighbourhood max + 0.5), then
// accum += Color, Color = accum * (1 / (frameIndex + 1)).
//
// The CPU pass clamps in place in row-major order, so a pixel sees its four
// earlier neighbours already clamped; the shader clamps against the unclamped
// input. For finite colours the two agree: the neighbourhood maximum starts at
// 0, so every threshold is >= 0.5 and a clamped pixel q keeps a luminance of
// about its threshold 4 max_n(q) + 0.5 >= 4 lum(p) + 0.5 for every later
// neighbour p. Such a p would need lum(p) > 4 lum(q') + 0.5 for its clamped
// neighbour q' as well, which no positive luminance satisfies, so a clamped
// pixel never changes a neighbour's decision or threshold. An infinite
// luminance breaks this (its clamp scale is 0 and inf * 0 is NaN, which the
// neighbour maximum then skips).
//
// Parity mode therefore runs the parallel clamp, lets a second pass check on
// the device whether any pixel's result changes under the in-place order, and
// hands the frame to `firefly_sequential_kernel` only when one does. That
// kernel reads the check's flag itself and returns at once when it is clear,
// so no mode reads anything back to the host or waits for the stream.
#include <cuda_runtime.h>

#include <algorithm>

#include "device/gf.cuh"

namespace hdr {

__device__ __forceinline__ float lum4(float4 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

__device__ __forceinline__ bool same_bits(float4 a, float4 b) {
    return __float_as_int(a.x) == __float_as_int(b.x) && __float_as_int(a.y) == __float_as_int(b.y) &&
           __float_as_int(a.z) == __float_as_int(b.z) && __float_as_int(a.w) == __float_as_int(b.w);
}

// ApplyFireflySuppression's body for pixel (x, y): neighbours earlier in
// row-major order come from `prev` (when given), later ones (and the pixel
// itself, which a clamped coordinate at the border can name) from `orig`.
__device__ __forceinline__ float4 firefly_pixel(const float4 *__restrict__ orig, const float4 *prev, int x, int y,
                                                int width, int height) {
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
    return c;
}

// One firefly pass over the frame: the shader's clamp (prev == nullptr), or
// the in-place-order check of a clamped plane `prev`, which sets *changed when
// some pixel's result differs from prev's.
__global__ void __launch_bounds__(256) firefly_kernel(const float4 *__restrict__ orig, const float4 *prev,
                                                      float4 *dst, int width, int height, int *changed) {
    const int x = blockIdx.x * 16 + (threadIdx.x & 15);
    const int y = blockIdx.y * 16 + (threadIdx.x >> 4);
    if (x >= width || y >= height) return;
    const size_t p = (size_t)y * width + x;
    const float4 c = firefly_pixel(orig, prev, x, y, width, height);
    if (dst) dst[p] = c;
    if (changed && prev && !same_bits(c, prev[p])) atomicOr(changed, 1);
}

// The row-major in-place clamp, exactly, in one block, run only when the check
// set *changed (else it returns at once). Pixel (x, y) depends on its earlier
// neighbours (x-1, y), (x-1, y-1), (x, y-1), (x+1, y-1) (or on itself, at the
// border), and all of them lie on earlier anti-diagonals t = x + 2y. So the
// block walks t = 0 .. (w-1) + 2(h-1), computes every pixel of one diagonal in
// parallel from the final values of earlier ones (in `plane`) and the
// unclamped values of later ones (in `orig`), and meets at a barrier before the
// next diagonal. Bounded: w + 2h - 2 steps, each at most min(h, w/2 + 1) pixels.
__global__ void __launch_bounds__(1024) firefly_sequential_kernel(const float4 *__restrict__ orig, float4 *plane,
                                                                  int width, int height, int *changed) {
    __shared__ int run;
    if (threadIdx.x == 0) run = *(volatile int *)changed;
    __syncthreads();
    if (!run) return;
    const int t_end = (width - 1) + 2 * (height - 1);
    for (int t = 0; t <= t_end; ++t) {
        // y with 0 <= t - 2y <= width - 1 and 0 <= y <= height - 1
        const int y_lo = smaxi(0, (t - (width - 1) + 1) / 2);
        const int y_hi = smini(height - 1, t / 2);
        for (int y = y_lo + (int)threadIdx.x; y <= y_hi; y += (int)blockDim.x) {
            const int x = t - 2 * y;
            plane[(size_t)y * width + x] = firefly_pixel(orig, plane, x, y, width, height);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) accumulate_kernel(const float4 *__restrict__ in, float4 *__restrict__ accum,
                                                         float4 *__restrict__ out, size_t count, float inv_n,
                                                         const int *frame_slot) {
    // a recorded pass reads its frame index from the slot (the same float division the host does)
    if (frame_slot) inv_n = 1.0f / (float)(*frame_slot + 1);
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

// Enqueues the pass on `st`; nothing waits for the device. Returns the number
// of kernels launched, or -1 with the CUDA error in *err.
// scratch holds one float4 plane of width*height (only used with firefly);
// flag_dev one int, zeroed on the stream before each parity-mode check.
int launch_accumulate(float4 *color, float4 *accum, float4 *scratch, int *flag_dev, int width, int height,
                      int frame_index, int firefly, int mode, cudaStream_t st, cudaError_t *err,
                      const int *frame_slot) {
    const size_t count = (size_t)width * height;
    const float inv_n = 1.0f / (float)(frame_index + 1);
    int launches = 0;
    const float4 *src = color;
    cudaError_t e = cudaSuccess;
    if (firefly) {
        const dim3 grid((width + 15) / 16, (height + 15) / 16);
        firefly_kernel<<<grid, 256, 0, st>>>(color, nullptr, scratch, width, height, nullptr);
        ++launches;
        src = scratch;
        if (mode == 0) {
            // in-place-order check, then the exact in-place clamp when it failed
            if ((e = cudaMemsetAsync(flag_dev, 0, sizeof(int), st)) != cudaSuccess) {
                if (err) *err = e;
                return -1;
            }
            firefly_kernel<<<grid, 256, 0, st>>>(color, scratch, nullptr, width, height, flag_dev);
            firefly_sequential_kernel<<<1, 1024, 0, st>>>(color, scratch, width, height, flag_dev);
            launches += 2;
        }
    }
    const int blocks = (int)std::min<size_t>((count + 255) / 256, (size_t)148 * 8);
    accumulate_kernel<<<blocks > 0 ? blocks : 1, 256, 0, st>>>(src, accum, color, count, inv_n, frame_slot);
    ++launches;
    if ((e = cudaGetLastError()) != cudaSuccess) {
        if (err) *err = e;
        return -1;
    }
    return launches;
}

}  // namespace hdr
