// BLAS build on the device: BVH::Build / _Subdivide (renderContext/bvh.cpp:66-208)
// producing the tree, node order and triangle order the host builder (and the
// reference) produce, bit for bit. The recursion is replayed breadth-first,
// one kernel sequence per tree level over every triangle of the mesh:
//
//  * node boxes: GfRange3f::UnionWith over the node's triangles in order keeps,
//    per axis, the FIRST vertex holding the extreme value (strict < / >; +0 and
//    -0 compare equal, NaN never enters). Each vertex offers a 64-bit key
//    (order-preserving value bits, then its position in the node's vertex
//    sequence) and the node keeps the smallest key: the same vertex, so the
//    same bits, whatever the order of the atomics.
//  * the split: longest axis, midpoint, as the host builder computes them.
//  * the two-pointer partition (i from the left, j from the right, a failing
//    element swapped with a[j]) has a closed form. Read the node's elements as
//    a left stream (positions start, start+1, ...) and a right stream
//    (end-1, end-2, ...); the loop takes from the left stream after a pass and
//    from the right stream after a fail. With f_k the left index of the k-th
//    failing left element and g_k the right index of the k-th passing right
//    element (g_0 = -1), the left stream reaches index p iff
//    p + (g_{nf(p)} + 1) < count, nf(p) being the fails before p; past that
//    point the right stream holds the rest. Then: a left pass stays at p, the
//    k-th left fail goes to count-2-g_{k-1}, the k-th right pass to f_k, and a
//    right fail at right index q to count-2-q. Prefix counts of one pass-flag
//    scan give every term.
//  * node numbering: the recursion allocates a node's two children when it
//    visits the node, so the children of the r-th inner node in depth-first
//    pre-order sit at 1 + 2r and 2 + 2r. Inner-node counts of the subtrees
//    (bottom-up) give each node's pre-order rank (top-down).
#include <cub/device/device_scan.cuh>

#include <vector>

#include "device/blas_build.h"
#include "device/tri_setup.cuh"

namespace hdr {
namespace {

constexpr unsigned long long kNoKey = ~0ull;
constexpr int kThreads = 256;

inline int blocks_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

// order-preserving bits of a float with +0 and -0 equal
__device__ __forceinline__ unsigned order_bits(float v) {
    unsigned b = __float_as_uint(v);
    if ((b & 0x7fffffffu) == 0u) b = 0u;
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ unsigned long long umin64(unsigned long long a, unsigned long long b) {
    return b < a ? b : a;
}

__global__ void tri_valid_kernel(hdr_mesh_desc m, int *valid) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m.num_triangles) return;
    if (i == m.num_triangles) {  // the scan's total
        valid[i] = 0;
        return;
    }
    const int np = m.num_points;
    const int i0 = m.indices[3 * i], i1 = m.indices[3 * i + 1], i2 = m.indices[3 * i + 2];
    valid[i] = (i0 >= 0 && i0 < np && i1 >= 0 && i1 < np && i2 >= 0 && i2 < np) ? 1 : 0;
}

__global__ void tri_setup_kernel(hdr_mesh_desc m, const int *valid, const int *slot, float *geo, float *attr,
                                 float *vtx, float *cen) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.num_triangles || !valid[i]) return;
    BlasTriangle t;
    make_triangle(m, i, t);
    const size_t s = (size_t)slot[i];
    pack_triangle(t, geo + kTriGeoFloats * s, attr + kTriAttrFloats * s);
    const float v[9] = {t.v0.x, t.v0.y, t.v0.z, t.v1.x, t.v1.y, t.v1.z, t.v2.x, t.v2.y, t.v2.z};
    for (int k = 0; k < 9; ++k) vtx[9 * s + k] = v[k];
    cen[3 * s] = t.centroid.x, cen[3 * s + 1] = t.centroid.y, cen[3 * s + 2] = t.centroid.z;
}

__global__ void iota_kernel(int *perm, int *seg, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    perm[p] = p;
    seg[p] = 0;
}

struct Nodes {  // breadth-first build records
    int *start, *end, *child, *axis, *pfinal, *inner_flag, *inner_rank, *subtree, *rank, *index;
    float *split, *box;  // box: 6 per node
    unsigned long long *keys;  // 6 per node: min x/y/z, max x/y/z
};

// per position: the first extreme vertex of each axis, reduced over runs of one node in the warp
__global__ void box_keys_kernel(const int *perm, const int *seg, const float *vtx, int M, unsigned long long *keys) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    int s = -1;
    unsigned long long k[6] = {kNoKey, kNoKey, kNoKey, kNoKey, kNoKey, kNoKey};
    if (p < M) {
        s = seg[p];
        if (s >= 0) {
            const float *v = vtx + 9 * (size_t)perm[p];
            for (int c = 0; c < 3; ++c)
                for (int a = 0; a < 3; ++a) {
                    const float x = v[3 * c + a];
                    const unsigned long long seq = 3ull * (unsigned)p + (unsigned)c;
                    if (x < 3.402823466e+38f) k[a] = umin64(k[a], ((unsigned long long)order_bits(x) << 32) | seq);
                    if (x > -3.402823466e+38f)
                        k[3 + a] = umin64(k[3 + a], ((unsigned long long)(~order_bits(x)) << 32) | seq);
                }
        }
    }
    // positions of one node are contiguous: a segmented inclusive scan over the warp
    const int lane = threadIdx.x & 31;
    for (int off = 1; off < 32; off <<= 1) {
        const int so = __shfl_up_sync(0xffffffffu, s, off);
        for (int j = 0; j < 6; ++j) {
            const unsigned long long o = __shfl_up_sync(0xffffffffu, k[j], off);
            if (lane >= off && so == s) k[j] = umin64(k[j], o);
        }
    }
    const int sn = __shfl_down_sync(0xffffffffu, s, 1);
    if (s >= 0 && (lane == 31 || sn != s))
        for (int j = 0; j < 6; ++j)
            if (k[j] != kNoKey) atomicMin(&keys[6 * (size_t)s + j], k[j]);
}

// per node of the level: its box from the keys; leaf or split axis and position
__global__ void node_kernel(Nodes n, int lb, int le, const int *perm, const float *vtx, int *info) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = lb + t;
    if (b > le) return;
    if (b == le) {  // the scan's total
        n.inner_flag[t] = 0;
        return;
    }
    float bx[6];
    for (int j = 0; j < 6; ++j) {
        const unsigned long long key = n.keys[6 * (size_t)b + j];
        if (key == kNoKey) {
            bx[j] = j < 3 ? 3.402823466e+38f : -3.402823466e+38f;
        } else {
            const unsigned seq = (unsigned)(key & 0xffffffffu);
            bx[j] = vtx[9 * (size_t)perm[seq / 3] + 3 * (seq % 3) + j % 3];
        }
        n.box[6 * (size_t)b + j] = bx[j];
    }
    const V3 mn{bx[0], bx[1], bx[2]}, mx{bx[3], bx[4], bx[5]};
    if (mn.x > mx.x || mn.y > mx.y || mn.z > mx.z) atomicOr(info, 1);
    const int count = n.end[b] - n.start[b];
    const bool leaf = count <= 4;
    n.inner_flag[t] = leaf ? 0 : 1;
    int axis = -1;
    float split = 0.0f;
    if (!leaf) {
        const V3 size = mx - mn;
        axis = 0;
        if (size.y > size.x) axis = 1;
        if (comp(size, 2) > comp(size, axis)) axis = 2;
        split = comp(mn, axis) + comp(size, axis) * 0.5f;
    }
    n.axis[b] = axis;
    n.split[b] = split;
}

// children of the level's inner nodes: the next level, in the order of their parents
__global__ void child_kernel(Nodes n, int lb, int le) {
    const int b = lb + blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= le) return;
    n.child[b] = n.inner_flag[b - lb] ? le + 2 * n.inner_rank[b - lb] : -1;
}

__global__ void pass_flag_kernel(Nodes n, const int *perm, const int *seg, const float *cen, int M, int *pf) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > M) return;
    int pass = 0;
    if (p < M) {
        const int s = seg[p];
        if (s >= 0) {
            const int axis = n.axis[s];
            if (axis >= 0) pass = cen[3 * (size_t)perm[p] + axis] < n.split[s] ? 1 : 0;
        }
    }
    pf[p] = pass;
}

struct PosTerms {
    int start, end, c, pl, pb, pass, T;
};

__device__ __forceinline__ bool pos_terms(const Nodes &n, const int *seg, const int *pf, const int *pex, int p,
                                          PosTerms &t, int &s) {
    s = seg[p];
    if (s < 0 || n.axis[s] < 0) return false;
    t.start = n.start[s];
    t.end = n.end[s];
    t.c = t.end - t.start;
    t.pl = p - t.start;
    t.pb = pex[p] - pex[t.start];  // passes before p in the node
    t.pass = pf[p];
    t.T = pex[t.end] - pex[t.start];
    return true;
}

// fail_list[start + k - 1] = left index of the k-th fail; pass_list[start + k - 1] = right index of the k-th
// pass counted from the right
__global__ void lists_kernel(Nodes n, const int *seg, const int *pf, const int *pex, int M, int *fail_list,
                             int *pass_list) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= M) return;
    PosTerms t;
    int s;
    if (!pos_terms(n, seg, pf, pex, p, t, s)) return;
    if (!t.pass)
        fail_list[t.start + (t.pl - t.pb)] = t.pl;
    else
        pass_list[t.start + (t.T - t.pb - 1)] = t.end - 1 - p;
}

__device__ __forceinline__ int right_consumed(const int *pass_list, const PosTerms &t, int nf) {
    if (nf == 0) return 0;
    return nf <= t.T ? pass_list[t.start + nf - 1] + 1 : t.c;
}

// the left stream's length (the one position where the reach condition flips) and the children's ranges
__global__ void pfinal_kernel(Nodes n, const int *seg, const int *pf, const int *pex, int M, const int *pass_list) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= M) return;
    PosTerms t;
    int s;
    if (!pos_terms(n, seg, pf, pex, p, t, s)) return;
    const int nf = t.pl - t.pb;
    if (t.pl + right_consumed(pass_list, t, nf) < t.c) {
        if (t.pl == t.c - 1)
            n.pfinal[s] = t.c;
        else if (!(t.pl + 1 + right_consumed(pass_list, t, nf + 1 - t.pass) < t.c))
            n.pfinal[s] = t.pl + 1;
    }
    if (t.pl == 0) {
        const int i = (t.T == 0 || t.T == t.c) ? t.start + t.c / 2 : t.start + t.T;
        const int l = n.child[s];
        n.start[l] = t.start;
        n.end[l] = i;
        n.start[l + 1] = i;
        n.end[l + 1] = t.end;
    }
}

// info[1] is set (and the element left out) if an index leaves its node: the closed form rules that out
__global__ void dest_kernel(Nodes n, const int *perm, const int *seg, const int *pf, const int *pex, int M,
                            const int *fail_list, const int *pass_list, int *perm_next, int *seg_next, int *info) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= M) return;
    PosTerms t;
    int s;
    if (!pos_terms(n, seg, pf, pex, p, t, s)) {  // a leaf, or finished earlier: stays
        perm_next[p] = perm[p];
        seg_next[p] = -1;
        return;
    }
    const int nf = t.pl - t.pb;
    int d = -1;
    if (t.pl < n.pfinal[s]) {
        if (t.pass) {
            d = t.pl;
        } else if (nf <= t.T) {
            const int g = nf == 0 ? -1 : pass_list[t.start + nf - 1];
            d = t.c - 2 - g;
        }
    } else if (!t.pass) {
        d = t.pl - 1;
    } else if (t.T - t.pb <= t.c - t.T) {  // the k-th right pass takes the k-th left fail's slot
        d = fail_list[t.start + (t.T - t.pb) - 1];
    }
    if (d < 0 || d >= t.c) {
        atomicOr(info + 1, 1);
        return;
    }
    const int dst = t.start + d;
    const int i = (t.T == 0 || t.T == t.c) ? t.start + t.c / 2 : t.start + t.T;
    perm_next[dst] = perm[p];
    seg_next[dst] = dst < i ? n.child[s] : n.child[s] + 1;
}

__global__ void subtree_kernel(Nodes n, int lb, int le) {
    const int b = lb + blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= le) return;
    const int c = n.child[b];
    n.subtree[b] = c < 0 ? 0 : 1 + n.subtree[c] + n.subtree[c + 1];
}

__global__ void rank_kernel(Nodes n, int lb, int le) {
    const int b = lb + blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= le) return;
    const int c = n.child[b];
    if (c < 0) return;
    const int r = n.rank[b];
    n.rank[c] = r + 1;
    n.rank[c + 1] = r + 1 + n.subtree[c];
    n.index[c] = 1 + 2 * r;
    n.index[c + 1] = 2 + 2 * r;
}

__global__ void emit_kernel(Nodes n, int B, float4 *out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B || n.index[b] < 0 || n.index[b] >= B) return;
    const int c = n.child[b];
    const int left = c < 0 ? -n.start[b] - 1 : 1 + 2 * n.rank[b];
    const int count = c < 0 ? n.end[b] - n.start[b] : 0;
    const float *bx = n.box + 6 * (size_t)b;
    const size_t o = 2 * (size_t)n.index[b];
    out[o] = make_float4(bx[0], bx[1], bx[2], __int_as_float(left));
    out[o + 1] = make_float4(bx[3], bx[4], bx[5], __int_as_float(count));
}

__global__ void gather_tris_kernel(const int *perm, int M, const float4 *geo, const float4 *attr, float4 *geo_out,
                                   float4 *attr_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= M) return;
    const size_t src = (size_t)perm[p];
    for (int k = 0; k < kTriGeoFloats / 4; ++k) geo_out[3 * (size_t)p + k] = geo[3 * src + k];
    for (int k = 0; k < kTriAttrFloats / 4; ++k) attr_out[9 * (size_t)p + k] = attr[9 * src + k];
}

}  // namespace

struct DeviceBlasBuild::Impl {
    std::vector<void *> bufs;
    cudaStream_t st = nullptr;
    int M = 0, B = 0;
    int *perm = nullptr;
    float4 *geo = nullptr, *attr = nullptr;
    Nodes n{};

    template <class T>
    cudaError_t alloc(T **p, size_t count) {
        void *q = nullptr;
        const cudaError_t e = cudaMalloc(&q, count * sizeof(T) > 0 ? count * sizeof(T) : 16);
        if (e == cudaSuccess) bufs.push_back(q);
        *p = (T *)q;
        return e;
    }
    template <class T>
    cudaError_t upload(T **p, const T *src, size_t count) {
        cudaError_t e = alloc(p, count);
        if (e == cudaSuccess && count) e = cudaMemcpyAsync(*p, src, count * sizeof(T), cudaMemcpyHostToDevice, st);
        return e;
    }
    cudaError_t scan(const int *in, int *out, int count) {
        size_t bytes = 0;
        cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, count, st);
        if (e != cudaSuccess) return e;
        void *tmp = nullptr;
        if ((e = cudaMallocAsync(&tmp, bytes > 0 ? bytes : 16, st)) != cudaSuccess) return e;
        e = cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, count, st);
        cudaFreeAsync(tmp, st);
        return e;
    }
    int read_int(const int *p) {
        int v = 0;
        cudaMemcpyAsync(&v, p, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        return v;
    }
    ~Impl() {
        if (st) cudaStreamSynchronize(st);  // kernels of an unfinished build may still read the scratch
        for (void *p : bufs) cudaFree(p);
    }
};

DeviceBlasBuild::DeviceBlasBuild() : impl_(new Impl) {}
DeviceBlasBuild::~DeviceBlasBuild() { delete impl_; }

#define HDR_BB_CHECK(call)                   \
    do {                                     \
        const cudaError_t e_ = (call);       \
        if (e_ != cudaSuccess) return e_;    \
    } while (0)

cudaError_t DeviceBlasBuild::run(const hdr_mesh_desc &host_mesh, cudaStream_t st) {
    Impl &I = *impl_;
    I.st = st;
    result = DeviceBlasResult{};
    const int N = host_mesh.num_triangles;
    if (N <= 0 || host_mesh.num_points <= 0) return cudaSuccess;
    // the mesh's arrays in device memory
    hdr_mesh_desc m = host_mesh;
    float *fp;
    int *ip;
    HDR_BB_CHECK(I.upload(&fp, host_mesh.points, 3 * (size_t)host_mesh.num_points));
    m.points = fp;
    HDR_BB_CHECK(I.upload(&ip, host_mesh.indices, 3 * (size_t)N));
    m.indices = ip;
    if (host_mesh.num_uvs > 0) {
        HDR_BB_CHECK(I.upload(&fp, host_mesh.uvs, 2 * (size_t)host_mesh.num_uvs));
        m.uvs = fp;
    }
    if (host_mesh.num_normals > 0) {
        HDR_BB_CHECK(I.upload(&fp, host_mesh.normals, 3 * (size_t)host_mesh.num_normals));
        m.normals = fp;
    }
    if (host_mesh.num_colors > 0) {
        HDR_BB_CHECK(I.upload(&fp, host_mesh.colors, 3 * (size_t)host_mesh.num_colors));
        m.colors = fp;
    }
    if (host_mesh.material_indices && host_mesh.num_material_indices > 0) {
        const size_t n_mat = (size_t)(host_mesh.num_material_indices < N ? host_mesh.num_material_indices : N);
        HDR_BB_CHECK(I.upload(&ip, host_mesh.material_indices, n_mat));
        m.material_indices = ip;
        m.num_material_indices = (int32_t)n_mat;
    } else {
        m.material_indices = nullptr;
    }
    // triangle records of the valid triangles, in mesh order
    int *valid, *slot;
    HDR_BB_CHECK(I.alloc(&valid, (size_t)N + 1));
    HDR_BB_CHECK(I.alloc(&slot, (size_t)N + 1));
    tri_valid_kernel<<<blocks_for(N + 1), kThreads, 0, st>>>(m, valid);
    HDR_BB_CHECK(I.scan(valid, slot, N + 1));
    const int M = I.read_int(slot + N);
    I.M = M;
    if (M == 0) return cudaGetLastError();
    float *geo, *attr, *vtx, *cen;
    HDR_BB_CHECK(I.alloc(&geo, (size_t)M * kTriGeoFloats));
    HDR_BB_CHECK(I.alloc(&attr, (size_t)M * kTriAttrFloats));
    HDR_BB_CHECK(I.alloc(&vtx, (size_t)M * 9));
    HDR_BB_CHECK(I.alloc(&cen, (size_t)M * 3));
    tri_setup_kernel<<<blocks_for(N), kThreads, 0, st>>>(m, valid, slot, geo, attr, vtx, cen);
    I.geo = (float4 *)geo;
    I.attr = (float4 *)attr;

    // build state
    const size_t cap = 2 * (size_t)M + 1;  // breadth-first nodes: at most 2M - 1
    Nodes &n = I.n;
    HDR_BB_CHECK(I.alloc(&n.start, cap));
    HDR_BB_CHECK(I.alloc(&n.end, cap));
    HDR_BB_CHECK(I.alloc(&n.child, cap));
    HDR_BB_CHECK(I.alloc(&n.axis, cap));
    HDR_BB_CHECK(I.alloc(&n.pfinal, cap));
    HDR_BB_CHECK(I.alloc(&n.inner_flag, cap + 1));
    HDR_BB_CHECK(I.alloc(&n.inner_rank, cap + 1));
    HDR_BB_CHECK(I.alloc(&n.subtree, cap));
    HDR_BB_CHECK(I.alloc(&n.rank, cap));
    HDR_BB_CHECK(I.alloc(&n.index, cap));
    HDR_BB_CHECK(I.alloc(&n.split, cap));
    HDR_BB_CHECK(I.alloc(&n.box, 6 * cap));
    HDR_BB_CHECK(I.alloc(&n.keys, 6 * cap));
    int *perm, *perm_next, *seg, *seg_next, *pf, *pex, *fail_list, *pass_list, *info;
    HDR_BB_CHECK(I.alloc(&perm, (size_t)M));
    HDR_BB_CHECK(I.alloc(&perm_next, (size_t)M));
    HDR_BB_CHECK(I.alloc(&seg, (size_t)M));
    HDR_BB_CHECK(I.alloc(&seg_next, (size_t)M));
    HDR_BB_CHECK(I.alloc(&pf, (size_t)M + 1));
    HDR_BB_CHECK(I.alloc(&pex, (size_t)M + 1));
    HDR_BB_CHECK(I.alloc(&fail_list, (size_t)M));
    HDR_BB_CHECK(I.alloc(&pass_list, (size_t)M));
    HDR_BB_CHECK(I.alloc(&info, 4));
    HDR_BB_CHECK(cudaMemsetAsync(info, 0, 4 * sizeof(int), st));
    iota_kernel<<<blocks_for(M), kThreads, 0, st>>>(perm, seg, M);
    // defined contents for every slot (indices in range even if a level left one unwritten)
    HDR_BB_CHECK(cudaMemsetAsync(perm_next, 0, (size_t)M * sizeof(int), st));
    HDR_BB_CHECK(cudaMemsetAsync(seg_next, 0xff, (size_t)M * sizeof(int), st));
    const int root[2] = {0, M};
    HDR_BB_CHECK(cudaMemcpyAsync(n.start, &root[0], sizeof(int), cudaMemcpyHostToDevice, st));
    HDR_BB_CHECK(cudaMemcpyAsync(n.end, &root[1], sizeof(int), cudaMemcpyHostToDevice, st));
    HDR_BB_CHECK(cudaMemsetAsync(n.pfinal, 0, cap * sizeof(int), st));
    HDR_BB_CHECK(cudaMemsetAsync(n.rank, 0, sizeof(int), st));
    HDR_BB_CHECK(cudaMemsetAsync(n.index, 0, sizeof(int), st));

    std::vector<std::pair<int, int>> levels;
    int lb = 0, le = 1;
    while (lb < le) {
        levels.emplace_back(lb, le);
        const int nl = le - lb;
        HDR_BB_CHECK(cudaMemsetAsync(n.keys + 6 * (size_t)lb, 0xff, 6 * (size_t)nl * sizeof(unsigned long long), st));
        box_keys_kernel<<<blocks_for(M), kThreads, 0, st>>>(perm, seg, vtx, M, n.keys);
        node_kernel<<<blocks_for(nl + 1), kThreads, 0, st>>>(n, lb, le, perm, vtx, info);
        HDR_BB_CHECK(I.scan(n.inner_flag, n.inner_rank, nl + 1));
        child_kernel<<<blocks_for(nl), kThreads, 0, st>>>(n, lb, le);
        const int inner = I.read_int(n.inner_rank + nl);
        if ((size_t)le + 2 * (size_t)inner > cap) return cudaErrorInvalidValue;  // cannot happen: 2M - 1 nodes at most
        if (inner == 0) break;
        pass_flag_kernel<<<blocks_for(M + 1), kThreads, 0, st>>>(n, perm, seg, cen, M, pf);
        HDR_BB_CHECK(I.scan(pf, pex, M + 1));
        lists_kernel<<<blocks_for(M), kThreads, 0, st>>>(n, seg, pf, pex, M, fail_list, pass_list);
        pfinal_kernel<<<blocks_for(M), kThreads, 0, st>>>(n, seg, pf, pex, M, pass_list);
        dest_kernel<<<blocks_for(M), kThreads, 0, st>>>(n, perm, seg, pf, pex, M, fail_list, pass_list, perm_next,
                                                         seg_next, info);
        std::swap(perm, perm_next);
        std::swap(seg, seg_next);
        lb = le;
        le += 2 * inner;
    }
    I.B = le;
    for (size_t k = levels.size(); k-- > 0;)
        subtree_kernel<<<blocks_for(levels[k].second - levels[k].first), kThreads, 0, st>>>(n, levels[k].first,
                                                                                            levels[k].second);
    for (const auto &lv : levels)
        rank_kernel<<<blocks_for(lv.second - lv.first), kThreads, 0, st>>>(n, lv.first, lv.second);
    HDR_BB_CHECK(cudaGetLastError());
    I.perm = perm;
    result.num_tris = M;
    result.num_nodes = 1 + 2 * I.read_int(n.subtree);
    result.max_depth = (int)levels.size();
    result.empty_box = I.read_int(info) != 0;
    if (I.read_int(info + 1) != 0) return cudaErrorUnknown;  // a partition index left its node
    return cudaGetLastError();
}

cudaError_t DeviceBlasBuild::write(float4 *nodes, float4 *tri_geo, float4 *tri_attr) {
    Impl &I = *impl_;
    if (I.M == 0) return cudaSuccess;
    emit_kernel<<<blocks_for(I.B), kThreads, 0, I.st>>>(I.n, I.B, nodes);
    gather_tris_kernel<<<blocks_for(I.M), kThreads, 0, I.st>>>(I.perm, I.M, I.geo, I.attr, tri_geo, tri_attr);
    return cudaGetLastError();
}

}  // namespace hdr
