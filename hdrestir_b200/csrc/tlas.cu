// TLAS rebuild on the device for moved instances (hdr_scene_set_instance_transforms).
// The reference rebuilds its TLAS whenever Scene::BuildRenderState runs
// (renderer.cpp:410-415, scene.cpp:187-222 and 333-407); here the instances'
// records and the TLAS are rebuilt in HBM from new transforms, with the same
// arithmetic as the host scene builder, so the tree, its node order and every
// box are the ones a fresh upload of the same scene would build:
//   1. per instance (one thread each): inverse (cofactor expansion in double),
//      forward rows, world box of the mesh's bounds (Scene::_TransformBounds)
//      and its centre;
//   2. the TLAS (one thread): Scene::_SubdivideTLAS replayed depth-first with
//      an explicit stack, which allocates nodes in the recursion's order (two
//      children per visited node, leaves of at most two instances, midpoint
//      split of the longest axis with the two-pointer partition).
#include "device/frame.cuh"

namespace hdr {
namespace {

struct Box3 {  // GfRange3f semantics (default = empty)
    V3 mn{3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f};
    V3 mx{-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f};
    __device__ __forceinline__ void extend(V3 p) {
        if (p.x < mn.x) mn.x = p.x;
        if (p.y < mn.y) mn.y = p.y;
        if (p.z < mn.z) mn.z = p.z;
        if (p.x > mx.x) mx.x = p.x;
        if (p.y > mx.y) mx.y = p.y;
        if (p.z > mx.z) mx.z = p.z;
    }
    __device__ __forceinline__ bool empty() const { return mn.x > mx.x || mn.y > mx.y || mn.z > mx.z; }
};

// instance record: 32 floats = inverse (16) | T row 0, node base | T row 1, triangle base |
// T row 2, material | light, BLAS present, wide base, mesh
__global__ void instance_update_kernel(const float *__restrict__ xf, float4 *instances,
                                       const float *__restrict__ mesh_ranges, float *bounds, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float *T = xf + 16 * (size_t)k;
    float inv[16];
    gf_inverse4f(T, inv);
    float4 *rec = instances + 8 * (size_t)k;
    for (int r = 0; r < 4; ++r) rec[r] = make_float4(inv[4 * r], inv[4 * r + 1], inv[4 * r + 2], inv[4 * r + 3]);
    const float4 r4 = rec[4], r5 = rec[5], r6 = rec[6], r7 = rec[7];
    rec[4] = make_float4(T[0], T[1], T[2], r4.w);
    rec[5] = make_float4(T[4], T[5], T[6], r5.w);
    rec[6] = make_float4(T[8], T[9], T[10], r6.w);
    const int mesh = __float_as_int(r7.w);
    const float *mr = mesh_ranges + 6 * (size_t)mesh;
    Box3 src, world;
    src.mn = V3{mr[0], mr[1], mr[2]};
    src.mx = V3{mr[3], mr[4], mr[5]};
    if (src.empty()) {
        world = src;
    } else {
        const V3 a = src.mn, b = src.mx;
        const V3 corners[8] = {{a.x, a.y, a.z}, {b.x, a.y, a.z}, {a.x, b.y, a.z}, {b.x, b.y, a.z},
                               {a.x, a.y, b.z}, {b.x, a.y, b.z}, {a.x, b.y, b.z}, {b.x, b.y, b.z}};
        for (int c = 0; c < 8; ++c) world.extend(m4f_transform(T, corners[c]));
    }
    const V3 ctr = (world.mn + world.mx) * 0.5f;
    float *o = bounds + 9 * (size_t)k;
    o[0] = world.mn.x, o[1] = world.mn.y, o[2] = world.mn.z;
    o[3] = world.mx.x, o[4] = world.mx.y, o[5] = world.mx.z;
    o[6] = ctr.x, o[7] = ctr.y, o[8] = ctr.z;
}

// Instances whose boxes and indices fit in shared memory (the build is one
// thread's dependent loads; shared memory keeps each near 30 cycles).
constexpr int kTlasSmemBytes = 200 * 1024;
constexpr int kInstSmemBytes = 10 * 4;  // box (6) + centre (3) + index (1)

// info[0] = nodes written, info[1] = maximum depth, info[2] = 1 when the node or stack capacity was
// too small, info[3] = 1 when a visited node's box is empty
__global__ void __launch_bounds__(256) tlas_build_kernel(const float *__restrict__ bounds_g, int n, float4 *nodes,
                                                         int cap_nodes, int *tlas_inst, int4 *stack, int cap_stack,
                                                         int *info, int staged) {
    extern __shared__ float smem[];
    float *bounds = staged ? smem : const_cast<float *>(bounds_g);
    int *idx = staged ? (int *)(smem + 9 * (size_t)n) : tlas_inst;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        if (staged)
            for (int k = 0; k < 9; ++k) bounds[9 * (size_t)i + k] = bounds_g[9 * (size_t)i + k];
        idx[i] = i;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int count_nodes = 1, max_depth = 0, sp = 0, overflow = 0, any_empty = 0;
        const float4 lo_empty = make_float4(3.402823466e+38f, 3.402823466e+38f, 3.402823466e+38f, 0.0f);
        const float4 hi_empty = make_float4(-3.402823466e+38f, -3.402823466e+38f, -3.402823466e+38f, 0.0f);
        stack[sp++] = make_int4(0, 0, n, 1);  // node, start, end, depth
        while (sp > 0) {
            const int4 t = stack[--sp];
            const int node = t.x, start = t.y, end = t.z, depth = t.w;
            if (depth > max_depth) max_depth = depth;
            if (count_nodes + 2 > cap_nodes || sp + 2 > cap_stack) {
                overflow = 1;
                break;
            }
            const int left_idx = count_nodes;  // both children are allocated when the node is visited
            count_nodes += 2;
            nodes[2 * (size_t)left_idx] = lo_empty;  // a leaf's two children stay default (empty) nodes
            nodes[2 * (size_t)left_idx + 1] = hi_empty;
            nodes[2 * (size_t)left_idx + 2] = lo_empty;
            nodes[2 * (size_t)left_idx + 3] = hi_empty;
            Box3 b;
            for (int i = start; i < end; ++i) {
                const float *bb = bounds + 9 * (size_t)idx[i];
                b.extend(V3{bb[0], bb[1], bb[2]});
                b.extend(V3{bb[3], bb[4], bb[5]});
            }
            if (b.empty()) any_empty = 1;
            const int count = end - start;
            if (count <= 2) {
                nodes[2 * (size_t)node] = make_float4(b.mn.x, b.mn.y, b.mn.z, __int_as_float(-start - 1));
                nodes[2 * (size_t)node + 1] = make_float4(b.mx.x, b.mx.y, b.mx.z, __int_as_float(count));
                continue;
            }
            nodes[2 * (size_t)node] = make_float4(b.mn.x, b.mn.y, b.mn.z, __int_as_float(left_idx));
            nodes[2 * (size_t)node + 1] = make_float4(b.mx.x, b.mx.y, b.mx.z, __int_as_float(0));
            const V3 size = b.mx - b.mn;
            int axis = 0;
            if (size.y > size.x) axis = 1;
            if (comp(size, 2) > comp(size, axis)) axis = 2;
            const float split = comp(b.mn, axis) + comp(size, axis) * 0.5f;
            int i = start, j = end - 1;
            while (i <= j) {
                if (bounds[9 * (size_t)idx[i] + 6 + axis] < split) {
                    ++i;
                } else {
                    const int tmp = idx[i];
                    idx[i] = idx[j];
                    idx[j] = tmp;
                    --j;
                }
            }
            if (i == start || i == end) i = start + count / 2;
            // right pushed first: the left subtree is visited (and allocates) first, as in the recursion
            stack[sp++] = make_int4(left_idx + 1, i, end, depth + 1);
            stack[sp++] = make_int4(left_idx, start, i, depth + 1);
        }
        info[0] = count_nodes;
        info[1] = max_depth;
        info[2] = overflow;
        info[3] = any_empty;
    }
    if (staged) {
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) tlas_inst[i] = idx[i];
    }
}

}  // namespace

int launch_tlas_rebuild(const float *xf, float4 *instances, const float *mesh_ranges, float *bounds, int n,
                        float4 *tlas_nodes, int cap_nodes, int *tlas_inst, int4 *stack, int cap_stack, int *info,
                        cudaStream_t st) {
    if (n <= 0) return 0;
    instance_update_kernel<<<(n + 127) / 128, 128, 0, st>>>(xf, instances, mesh_ranges, bounds, n);
    const size_t smem = (size_t)n * kInstSmemBytes;
    const int staged = smem <= (size_t)kTlasSmemBytes ? 1 : 0;
    if (staged) cudaFuncSetAttribute(tlas_build_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    tlas_build_kernel<<<1, 256, staged ? smem : 0, st>>>(bounds, n, tlas_nodes, cap_nodes, tlas_inst, stack,
                                                         cap_stack, info, staged);
    return cudaPeekAtLastError() == cudaSuccess ? 2 : -1;
}

}  // namespace hdr
