// HdRestirRenderBuffer::CopyFromFrameBuffer / _WriteOutput on the device
// (hydra/hd_restir_render_buffer.cpp:46-73,113-148): a float frame buffer
// ("Color", "Depth", "Albedo", "Normal") converted to the render buffer's
// component format, so the renderer's resolve can take the image from HBM
// instead of a host frame buffer. (A source pixel of the destination pixel's
// size is copied as bytes by the caller, as CopyFromFrameBuffer does.) Per
// component c of a pixel:
//   c >= the source's components : 0
//   Float32 : the value
//   Float16 : GfHalf(value) (round to nearest even)
//   UNorm8  : (uint8_t)clamp(value * 255, 0, 255)   (truncating)
//   SNorm8  : (int8_t)clamp(value * 127, -128, 127)  (truncating)
//   Int32   : (int32_t)value                          (truncating)
// std::clamp(v, lo, hi) is (v < lo) ? lo : (hi < v) ? hi : v. Values the
// reference converts with undefined behaviour (NaN, Int32 out of range) are
// not part of the contract.
#include <cuda_fp16.h>

#include "device/frame.cuh"

namespace hdr {
namespace {

__device__ __forceinline__ float ref_clamp(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }

template <int kFormat>
__global__ void resolve_kernel(const float *__restrict__ src, int src_comps, void *__restrict__ dst, int dst_comps,
                               size_t pixels) {
    const size_t n = pixels * (size_t)dst_comps;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const size_t px = k / (size_t)dst_comps;
        const int c = (int)(k - px * (size_t)dst_comps);
        const bool have = c < src_comps;
        const float v = have ? src[px * (size_t)src_comps + c] : 0.0f;
        if (kFormat == kResolveFloat32) {
            ((float *)dst)[k] = v;
        } else if (kFormat == kResolveFloat16) {
            ((unsigned short *)dst)[k] = have ? __half_as_ushort(__float2half_rn(v)) : (unsigned short)0;
        } else if (kFormat == kResolveUNorm8) {
            ((unsigned char *)dst)[k] = have ? (unsigned char)ref_clamp(v * 255.0f, 0.0f, 255.0f) : (unsigned char)0;
        } else if (kFormat == kResolveSNorm8) {
            ((signed char *)dst)[k] = have ? (signed char)ref_clamp(v * 127.0f, -128.0f, 127.0f) : (signed char)0;
        } else {
            ((int *)dst)[k] = have ? (int)v : 0;
        }
    }
}

}  // namespace

int launch_resolve(const float *src, int src_comps, int format, int dst_comps, void *dst, size_t pixels,
                   int sm_count, cudaStream_t st) {
    const size_t n = pixels * (size_t)dst_comps;
    if (n == 0) return 0;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)sm_count * 8);
    switch (format) {
        case kResolveFloat32: resolve_kernel<kResolveFloat32><<<blocks, 256, 0, st>>>(src, src_comps, dst, dst_comps, pixels); break;
        case kResolveFloat16: resolve_kernel<kResolveFloat16><<<blocks, 256, 0, st>>>(src, src_comps, dst, dst_comps, pixels); break;
        case kResolveUNorm8: resolve_kernel<kResolveUNorm8><<<blocks, 256, 0, st>>>(src, src_comps, dst, dst_comps, pixels); break;
        case kResolveSNorm8: resolve_kernel<kResolveSNorm8><<<blocks, 256, 0, st>>>(src, src_comps, dst, dst_comps, pixels); break;
        case kResolveInt32: resolve_kernel<kResolveInt32><<<blocks, 256, 0, st>>>(src, src_comps, dst, dst_comps, pixels); break;
        default: return -1;
    }
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

}  // namespace hdr
