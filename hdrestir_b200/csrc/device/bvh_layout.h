// Layout of the 4-wide BVH records shared by the host builder
// (host/scene_build.cpp) and the device traversal (device/traverse.cuh).
//
// Wide node: 32 floats = min.x[4] min.y[4] min.z[4] max.x[4] max.y[4] max.z[4]
// code[4] pad[4]. A slot code is (payload << kWideTagBits) | tag, or -1 for an
// empty slot; the code is pushed on the traversal stack as it is.
//   inner slots: payload = wide-node index (TLAS: global; BLAS: relative to the
//                mesh's first wide node)
//   BLAS leaf:   payload = (first triangle << 2) | (triangle count - 1), count 1..4
//   TLAS leaf:   payload = (first instance slot << 1) | (instance count - 1), count 1..2
//   instance:    payload = instance slot in the TLAS instance-index array
#pragma once

namespace hdr {

constexpr int kWideNodeFloats = 32;
constexpr int kWideTagBits = 3;
constexpr int kWTagTlasNode = 0, kWTagTlasLeaf = 1, kWTagInst = 2, kWTagBlasNode = 3, kWTagBlasLeaf = 4;
constexpr int kBlasLeafCountBits = 2, kTlasLeafCountBits = 1;

}  // namespace hdr
