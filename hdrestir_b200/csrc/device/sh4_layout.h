// Layout constants of the shadow-ray BVH shared by the host builder
// (host/shadow_bvh.cpp) and the device walk (device/shadow4.cuh).
#pragma once

namespace hdr {

constexpr int kSh4NodeFloats = 28;  // 7 float4 per node: child min.x, max.x, min.y, max.y, min.z, max.z, codes
constexpr int kSh4Stack = 64;       // traversal stack entries of the device walk

}  // namespace hdr
