// Device BLAS build (blas_build.cu): the host builder's tree for one mesh,
// built on the GPU. run() uploads the mesh's arrays, builds, and keeps the
// tree in scratch memory; write() stores the nodes (2 float4 each, child
// indices relative to the mesh's first node) and the triangle records (3 + 9
// float4 each) into the scene's arrays. Scratch is freed with the object.
#pragma once

#include <cuda_runtime.h>

#include "../../../include/hdrestir.h"

namespace hdr {

struct DeviceBlasResult {
    int num_nodes = 0, num_tris = 0, max_depth = 0;
    bool empty_box = false;  // some node box is empty (min > max on an axis)
};

class DeviceBlasBuild {
public:
    DeviceBlasBuild();
    ~DeviceBlasBuild();
    DeviceBlasBuild(const DeviceBlasBuild &) = delete;
    DeviceBlasBuild &operator=(const DeviceBlasBuild &) = delete;
    cudaError_t run(const hdr_mesh_desc &host_mesh, cudaStream_t st);
    cudaError_t write(float4 *nodes, float4 *tri_geo, float4 *tri_attr);
    DeviceBlasResult result;

private:
    struct Impl;
    Impl *impl_;
};

}  // namespace hdr
