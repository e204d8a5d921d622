// Scene query on the device: Scene::IntersectScene (scene/scene.cpp:409-535)
// over the reference's own two-level tree (TLAS of instances, one midpoint-split
// BLAS per mesh subset), replayed in the reference's visiting order so the
// closest hit and its tie-breaks are bit-identical:
//  * TLAS: explicit stack, right child pushed before left, nodes rejected when
//    the slab entry distance exceeds the current closest t (scene.cpp:414-510);
//  * BLAS: depth-first, left before right, leaf triangles in array order,
//    closest hit replaced only on strictly smaller t (bvh.cpp:243-305);
//  * slab and Moller-Trumbore tests with the reference's thresholds: the BLAS
//    slab compares |d| < 1e-8 in double (bvh.cpp:43), the TLAS slab in float
//    (scene.cpp:25), the triangle determinant in double (bvh.cpp:16).
// Shadow rays only need "is the closest hit nearer than L": running the same
// traversal and stopping as soon as the running closest t drops below L gives
// exactly that answer, because the running t only decreases.
#pragma once

#include "bvh_layout.h"
#include "gf.cuh"

namespace hdr {

// error bits reported back to the host
constexpr unsigned kErrBlasStack = 1u;
constexpr unsigned kErrTlasStack = 2u;

struct DeviceScene {
    const float4 *blas_nodes;  // 2 per node
    const float4 *tri_geo;     // 3 per triangle
    const float4 *tri_attr;    // 9 per triangle
    const float4 *instances;   // 8 per instance
    const float4 *tlas_nodes;  // 2 per node
    const int *tlas_inst;
    const float4 *materials;   // 12 per material
    const float *textures;     // material texels (RGB f32), located by the material records
    const float4 *lights;      // 12 per light
    const float *dome_pixels;
    const float *dome_row_cdf;
    const float *dome_col_cdf;
    int num_instances;
    int num_materials;
    int num_lights;
    int env_light;             // the first dome light (the environment unless `sky`), -1 = none
    // PhysicalSky (sky.cuh): the environment when `sky` is 1. Its sun is light index
    // num_lights for reservoirs and the delta-light test, outside the light sampler.
    int sky;
    int blackbody;             // extension: some light has a temperature (blackbody emission)
    float4 sky_sun;            // the sun direction; w = 1 when SampleDirect gives a sample
    float4 sky_sun_n;          // the direction normalised again, as Sample() uses it
    float4 sky_sun_color;      // SampleDirect's colour
    int dome_width, dome_height;
    float dome_total_lum;
    int has_tlas;
    // 4-wide collapse of the same trees (bvh_layout.h)
    const float4 *blas4;       // 8 per wide node
    const float4 *blas_roots;  // 2 per mesh: root min.xyz + root code, root max.xyz
    const float4 *tlas4;       // 8 per wide node
    float4 tlas_root_lo, tlas_root_hi;
    int wide;                  // 1: walk the wide trees, 0: the binary ones (same results)
    int proper_boxes;          // 1: no node box of any tree is empty (min > max on some axis)
    int shallow;               // 1: the binary walk's stack never exceeds kShallowStack entries
    int has_textures;          // 1: some material has a texture (closures read uv and tangents)
    // shadow-ray BVH (host/shadow_bvh.h): 4-wide SAH trees over the same triangles,
    // walked for "hit nearer than the limit" queries when sh4 is 1
    const float4 *sh4_nodes;   // 7 per node
    const float4 *sh4_tris;    // 3 per triangle (tri_geo records in leaf order)
    const int *sh4_inst_root;  // per instance: its mesh's root node, -1 = no triangles
    const int *sh4_inst_rank;  // per instance: its position in the reference TLAS's leaf order
    int sh4;                   // 1: shadow queries walk the 4-wide SAH trees
    // closest hits: 0 walk the reference trees; 1 walk the SAH trees (HDR_CTX_SAH_CLOSEST);
    // 2 walk the SAH trees and check each hit against the reference walk (ref_reaches),
    // which then walks the reference trees for the rare ray whose answer it cannot vouch for
    int sh4_closest;
    // parent links of the reference trees for that check
    // path records, 2 float4 per node: (box min, parent index bits, -1 at a root), (box max, 0)
    const float4 *ref_tlas_path;  // per TLAS node
    const int *ref_inst_leaf;     // per instance: its TLAS leaf
    const float4 *ref_blas_path;  // per BLAS node of all meshes, mesh-local parents
    const int *ref_tri_leaf;      // per triangle record: its mesh-local leaf
    // This struct's own copy in device memory. Kernels take the scene by value
    // (parameter space); a non-inlined callee gets this pointer instead of the
    // parameter's address, which would make every thread copy the parameter
    // block to local memory.
    const DeviceScene *dev;
};

__device__ __forceinline__ int fbits(float f) { return __float_as_int(f); }

struct SlabRay {
    V3 o;
    V3 inv;
    bool small[3];
    bool any_small;
};

// IntersectAABB of scene.cpp:16-47 (float thresholds) or bvh.cpp:32-64 (double ones).
template <bool kDoubleThresholds>
__device__ __forceinline__ SlabRay make_slab_ray(V3 o, V3 d) {
    SlabRay r;
    r.o = o;
    const float dd[3] = {d.x, d.y, d.z};
    float inv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float a = fabsf(dd[i]);
        // |d| < 1e-8 in double  <=>  |d| <= 9.99999993922529e-09f (the float nearest below 1e-8)
        r.small[i] = kDoubleThresholds ? (a <= 9.99999993922529e-09f) : (a < 1e-8f);
        inv[i] = 1.0f / dd[i];
    }
    r.inv = V3{inv[0], inv[1], inv[2]};
    r.any_small = r.small[0] | r.small[1] | r.small[2];
    return r;
}

// IntersectAABB without branches. The reference returns false as soon as the
// running entry distance passes the running exit distance; the entry only
// grows and the exit only shrinks, so testing once after all three axes gives
// the same answer. Each axis' (t1, t2) pair is ordered with min/max instead of
// a swap (no NaN can occur on an axis with |d| above the threshold, where
// 1/d is finite); an axis below the threshold only checks the origin. The
// entry distance is the reference's value (up to the sign of a zero, which no
// comparison sees).
__device__ __forceinline__ bool slab_test(const SlabRay &r, float4 lo, float4 hi, float &t_entry) {
    const float o[3] = {r.o.x, r.o.y, r.o.z};
    const float iv[3] = {r.inv.x, r.inv.y, r.inv.z};
    const float mn[3] = {lo.x, lo.y, lo.z};
    const float mx[3] = {hi.x, hi.y, hi.z};
    bool fail = (lo.x > hi.x) | (lo.y > hi.y) | (lo.z > hi.z);  // GfRange3f::IsEmpty
    float tmin = -1e30f, tmax = 1e30f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float t1 = (mn[i] - o[i]) * iv[i];
        const float t2 = (mx[i] - o[i]) * iv[i];
        fail |= r.small[i] & ((o[i] < mn[i]) | (o[i] > mx[i]));
        tmin = r.small[i] ? tmin : fmaxf(tmin, fminf(t1, t2));
        tmax = r.small[i] ? tmax : fminf(tmax, fmaxf(t1, t2));
    }
    t_entry = tmin;
    return !fail & !(tmin > tmax) & (tmax > 1e-4f);
}

// slab_test for a ray without small axes against a box that is not empty
// (DeviceScene::proper_boxes): the two checks that cannot fire are left out,
// the rest is the same arithmetic, so answer and entry distance are equal.
__device__ __forceinline__ bool slab_test_regular(const SlabRay &r, float4 lo, float4 hi, float &t_entry) {
    const float t1x = (lo.x - r.o.x) * r.inv.x, t2x = (hi.x - r.o.x) * r.inv.x;
    const float t1y = (lo.y - r.o.y) * r.inv.y, t2y = (hi.y - r.o.y) * r.inv.y;
    const float t1z = (lo.z - r.o.z) * r.inv.z, t2z = (hi.z - r.o.z) * r.inv.z;
    const float tmin = fmaxf(fmaxf(fmaxf(-1e30f, fminf(t1x, t2x)), fminf(t1y, t2y)), fminf(t1z, t2z));
    const float tmax = fminf(fminf(fminf(1e30f, fmaxf(t1x, t2x)), fmaxf(t1y, t2y)), fmaxf(t1z, t2z));
    t_entry = tmin;
    return !(tmin > tmax) & (tmax > 1e-4f);
}

// slab_test, or slab_test_regular where kRegular says the ray and the scene allow it
template <bool kRegular>
__device__ __forceinline__ bool box_test(const SlabRay &r, float4 lo, float4 hi, float &t_entry) {
    return kRegular ? slab_test_regular(r, lo, hi, t_entry) : slab_test(r, lo, hi, t_entry);
}

// IntersectTriangle (bvh.cpp:8-30)
__device__ __forceinline__ bool tri_test(V3 o, V3 d, const float4 *g, float &t, float &u, float &v) {
    const float4 g0 = __ldg(g), g1 = __ldg(g + 1), g2 = __ldg(g + 2);
    const V3 v0{g0.x, g0.y, g0.z};
    const V3 e1{g0.w, g1.x, g1.y};
    const V3 e2{g1.z, g1.w, g2.x};
    const V3 pvec = cross(d, e2);
    const float det = dot(e1, pvec);
    if (fabsf(det) <= 9.99999993922529e-09f) return false;  // std::abs(det) < 1e-8 (double)
    const float inv_det = 1.0f / det;
    const V3 tvec = o - v0;
    u = dot(tvec, pvec) * inv_det;
    if (u < 0.0f || u > 1.0f) return false;
    const V3 qvec = cross(tvec, e1);
    v = dot(d, qvec) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot(e2, qvec) * inv_det;
    return t > 1e-4f;
}

// Traversal counters for the statistics entry point; NoStats compiles away.
struct NoStats {
    __device__ __forceinline__ void pop() {}
    __device__ __forceinline__ void leaf() {}
    __device__ __forceinline__ void tri() {}
};
struct CountStats {
    int pops = 0, leaves = 0, tris = 0;
    __device__ __forceinline__ void pop() { ++pops; }
    __device__ __forceinline__ void leaf() { ++leaves; }
    __device__ __forceinline__ void tri() { ++tris; }
};

struct HitId {
    float t;
    int inst;  // -1: miss
    int tri;   // triangle index local to the instance's mesh
    float u, v;
};

// Closest hit (kAnyHit = false), or "closest t < t_limit" test (kAnyHit = true).
//
// One loop over one stack holds TLAS nodes, instance slots and BLAS nodes
// (tag in the low 2 bits), so the threads of a warp step through the two
// levels together instead of diverging in nested loops. The visiting order is
// the reference's: a TLAS leaf pushes its instances so they pop in leaf order;
// an instance pushes its BLAS root, whose nodes all pop before the next
// instance; BLAS children pop left first. A single running closest t replaces
// the reference's per-instance copy (instT starts at hit.t and hit.t is only
// written from it), which gives the same comparisons.
// err receives kErr* bits if the stack would overflow (the host rejects scenes
// deeper than the stack, so this is a guard, not a path).
constexpr int kTraceStack = 96;
constexpr int kTagTlas = 0, kTagInst = 1, kTagBlas = 2;

// Traversal stacks. A walk holds only scalars and a stack object, so its
// state stays in registers; the entries live where the stack object says.
template <class T>
struct LocalStack {  // all entries in per-thread local memory
    static constexpr int kCapacity = kTraceStack;
    T *e;
    __device__ __forceinline__ T get(int k) const { return e[k]; }
    __device__ __forceinline__ void set(int k, T v) { e[k] = v; }
};
// Entries below kDepth in this thread's column of a shared-memory array
// (entry k at col[k * kThreads]), deeper ones in a per-thread local array:
// depth-first walks rarely go deep, so the hot entries stay on chip.
template <class T, int kDepth, int kThreads>
struct SplitStack {
    static constexpr int kCapacity = kTraceStack;
    T *col;
    T *deep;
    __device__ __forceinline__ T get(int k) const { return k < kDepth ? col[k * kThreads] : deep[k - kDepth]; }
    __device__ __forceinline__ void set(int k, T v) {
        if (k < kDepth)
            col[k * kThreads] = v;
        else
            deep[k - kDepth] = v;
    }
};

// All entries in this thread's shared-memory column, for trees shallow enough
// that kDepth entries always suffice (checked at upload; a deeper walk stops
// with a stack error instead of writing past the column).
constexpr int kShallowStack = 40;
template <class T, int kDepth, int kThreads>
struct ColumnStack {
    static constexpr int kCapacity = kDepth;
    T *col;
    __device__ __forceinline__ T get(int k) const { return col[k * kThreads]; }
    __device__ __forceinline__ void set(int k, T v) { col[k * kThreads] = v; }
};

// The binary walk as a resumable state machine: start() takes a ray, each
// step() pops one stack entry. A persistent kernel can then give a lane whose
// ray is finished the next queued ray while the other lanes keep walking.
template <bool kAnyHit, class Stk = LocalStack<int>>
struct BinaryWalk {
    V3 o, d, oo, od;
    SlabRay wr, br;
    int cur_inst, node_base, tri_base, sp;
    float t_limit;
    HitId hit;
    Stk stack;

    __device__ __forceinline__ void start(const DeviceScene &s, V3 ro, V3 rd, float limit) {
        o = ro;
        d = rd;
        t_limit = limit;
        hit.t = 1e30f;
        hit.inst = -1;
        hit.tri = -1;
        hit.u = hit.v = 0.0f;
        wr = make_slab_ray<false>(o, d);
        br = wr;
        oo = o;
        od = d;
        cur_inst = -1;
        node_base = tri_base = 0;
        sp = 0;
        if (s.has_tlas) stack.set(sp++, (0 << 2) | kTagTlas);
    }
    // "closest hit nearer than t_limit" (kAnyHit) once the walk is over
    __device__ __forceinline__ bool shadow_answer() const { return hit.inst >= 0 && hit.t < t_limit; }

    // Pops one entry; false once the walk is over (stack empty, an any-hit
    // answer found, or a stack limit reached, which sets err).
    template <class St>
    __device__ __forceinline__ bool step(const DeviceScene &s, unsigned &err, St &st) {
        if (sp <= 0) return false;
        const int e = stack.get(--sp);
        st.pop();
        const int tag = e & 3, idx = e >> 2;
        if (tag != kTagInst) {  // a TLAS or BLAS node: one code path for both levels
            const bool blas = tag == kTagBlas;
            const float4 *np = blas ? s.blas_nodes + 2 * (size_t)(node_base + idx) : s.tlas_nodes + 2 * (size_t)idx;
            const float4 lo = __ldg(np), hi = __ldg(np + 1);
            float ta;
            if (!slab_test(blas ? br : wr, lo, hi, ta) || ta > hit.t) return sp > 0;
            const int left = fbits(lo.w);
            if (left >= 0) {
                if (sp + 2 > Stk::kCapacity) {
                    err |= blas ? kErrBlasStack : kErrTlasStack;
                    sp = 0;
                    return false;
                }
                stack.set(sp++, ((left + 1) << 2) | tag);
                stack.set(sp++, (left << 2) | tag);
            } else if (blas) {
                const int first = -left - 1;
                const int cnt = fbits(hi.w);
                st.leaf();
                for (int q = 0; q < cnt; ++q) {
                    float tt, uu, vv;
                    st.tri();
                    if (tri_test(oo, od, s.tri_geo + 3 * (size_t)(tri_base + first + q), tt, uu, vv) &&
                        tt < hit.t) {
                        hit.t = tt;
                        hit.inst = cur_inst;
                        hit.tri = first + q;
                        hit.u = uu;
                        hit.v = vv;
                    }
                }
                if (kAnyHit && hit.inst >= 0 && hit.t < t_limit) {
                    sp = 0;
                    return false;
                }
            } else {
                if (sp + 2 > Stk::kCapacity) {
                    err |= kErrTlasStack;
                    sp = 0;
                    return false;
                }
                const int first = -left - 1;
                const int count = fbits(hi.w);
                for (int k = count - 1; k >= 0; --k) stack.set(sp++, ((first + k) << 2) | kTagInst);
            }
        } else {  // instance slot of a TLAS leaf: enter its BLAS in object space
            const int ii = __ldg(&s.tlas_inst[idx]);
            const float4 *ip = s.instances + 8 * ii;
            const float4 r7 = __ldg(ip + 7);
            if (fbits(r7.y) == 0) return sp > 0;  // mesh without triangles: empty BVH
            const float4 m0 = __ldg(ip), m1 = __ldg(ip + 1), m2 = __ldg(ip + 2), m3 = __ldg(ip + 3);
            const float inv[16] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w,
                                   m2.x, m2.y, m2.z, m2.w, m3.x, m3.y, m3.z, m3.w};
            oo = m4f_transform(inv, o);
            od = m4f_transform_dir(inv, d);
            br = make_slab_ray<true>(oo, od);
            node_base = fbits(__ldg(&ip[4].w));
            tri_base = fbits(__ldg(&ip[5].w));
            cur_inst = ii;
            stack.set(sp++, (0 << 2) | kTagBlas);
        }
        return sp > 0;
    }
};

// The binary walk split into phases for warps that trace many rays. A lane's
// node steps are cheap and frequent; its leaves (triangle tests), instance
// entries (ray transform) and ray starts are costly and rare, and when every
// step may take any of them the warp pays for all of them on most steps. So a
// lane that pops a leaf or an instance entry, or finishes its walk, parks it
// (mode) and stops stepping; the warp keeps stepping the other lanes' nodes
// and serves the parked work of all lanes together afterwards. Each lane
// still handles its own entries in its own order, with the same running t at
// every test, so the results are BinaryWalk's.
enum : int { kModeNode = 0, kModeLeaf = 1, kModeInst = 2, kModeDone = 3, kModeIdle = 4 };

template <bool kAnyHit, class Stk>
struct PhasedWalk {
    V3 o, d, oo, od;
    SlabRay wr, br;
    int cur_inst, node_base, tri_base, sp;
    float t_limit;
    HitId hit;
    int mode;
    int pend;  // kModeLeaf: (first triangle << 3) | count; kModeInst: TLAS instance slot
    Stk stack;

    __device__ __forceinline__ void start(const DeviceScene &s, V3 ro, V3 rd, float limit) {
        o = ro;
        d = rd;
        t_limit = limit;
        hit.t = 1e30f;
        hit.inst = -1;
        hit.tri = -1;
        hit.u = hit.v = 0.0f;
        wr = make_slab_ray<false>(o, d);
        br = wr;
        oo = o;
        od = d;
        cur_inst = -1;
        node_base = tri_base = 0;
        sp = 0;
        if (s.has_tlas) stack.set(sp++, (0 << 2) | kTagTlas);
        mode = sp > 0 ? kModeNode : kModeDone;
    }
    __device__ __forceinline__ bool shadow_answer() const { return hit.inst >= 0 && hit.t < t_limit; }
    // both rays of the walk may use slab_test_regular
    __device__ __forceinline__ bool regular(const DeviceScene &s) const {
        return s.proper_boxes && !wr.any_small && !br.any_small;
    }

    // one stack entry of a lane in kModeNode
    template <bool kRegular, class St>
    __device__ __forceinline__ void node_step(const DeviceScene &s, unsigned &err, St &st) {
        if (sp <= 0) {
            mode = kModeDone;
            return;
        }
        const int e = stack.get(--sp);
        st.pop();
        const int tag = e & 3, idx = e >> 2;
        if (tag == kTagInst) {
            pend = idx;
            mode = kModeInst;
            return;
        }
        const bool blas = tag == kTagBlas;
        const float4 *np = blas ? s.blas_nodes + 2 * (size_t)(node_base + idx) : s.tlas_nodes + 2 * (size_t)idx;
        const float4 lo = __ldg(np), hi = __ldg(np + 1);
        float ta;
        if (!box_test<kRegular>(blas ? br : wr, lo, hi, ta) || ta > hit.t) return;
        const int left = fbits(lo.w);
        if (left >= 0 || !blas) {
            if (sp + 2 > Stk::kCapacity) {
                err |= blas ? kErrBlasStack : kErrTlasStack;
                sp = 0;
                mode = kModeDone;
                return;
            }
            if (left >= 0) {
                stack.set(sp++, ((left + 1) << 2) | tag);
                stack.set(sp++, (left << 2) | tag);
            } else {  // TLAS leaf: its instances pop in leaf order
                const int first = -left - 1;
                const int count = fbits(hi.w);
                for (int k = count - 1; k >= 0; --k) stack.set(sp++, ((first + k) << 2) | kTagInst);
            }
        } else {
            pend = ((-left - 1) << 3) | fbits(hi.w);
            mode = kModeLeaf;
        }
    }
    template <class St>
    __device__ __forceinline__ void leaf(const DeviceScene &s, St &st) {
        const int first = pend >> 3, cnt = pend & 7;
        st.leaf();
        for (int q = 0; q < cnt; ++q) {
            float tt, uu, vv;
            st.tri();
            if (tri_test(oo, od, s.tri_geo + 3 * (size_t)(tri_base + first + q), tt, uu, vv) && tt < hit.t) {
                hit.t = tt;
                hit.inst = cur_inst;
                hit.tri = first + q;
                hit.u = uu;
                hit.v = vv;
            }
        }
        if (kAnyHit && hit.inst >= 0 && hit.t < t_limit) sp = 0;
        mode = sp > 0 ? kModeNode : kModeDone;
    }
    __device__ __forceinline__ void inst(const DeviceScene &s) {
        const int ii = __ldg(&s.tlas_inst[pend]);
        const float4 *ip = s.instances + 8 * ii;
        const float4 r7 = __ldg(ip + 7);
        if (fbits(r7.y) != 0) {  // a mesh without triangles has an empty BVH
            const float4 m0 = __ldg(ip), m1 = __ldg(ip + 1), m2 = __ldg(ip + 2), m3 = __ldg(ip + 3);
            const float inv[16] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w,
                                   m2.x, m2.y, m2.z, m2.w, m3.x, m3.y, m3.z, m3.w};
            oo = m4f_transform(inv, o);
            od = m4f_transform_dir(inv, d);
            br = make_slab_ray<true>(oo, od);
            node_base = fbits(__ldg(&ip[4].w));
            tri_base = fbits(__ldg(&ip[5].w));
            cur_inst = ii;
            stack.set(sp++, (0 << 2) | kTagBlas);
        }
        mode = sp > 0 ? kModeNode : kModeDone;
    }
};

template <bool kAnyHit, class St = NoStats>
__device__ bool trace_ray_binary(const DeviceScene &s, V3 o, V3 d, float t_limit, HitId &hit, unsigned &err,
                                 St &&st = St()) {
    int mem[kTraceStack];
    BinaryWalk<kAnyHit> w;
    w.stack.e = mem;
    w.start(s, o, d, t_limit);
    while (w.step(s, err, st)) {
    }
    hit = w.hit;
    return hit.inst >= 0;
}

// The same query over the 4-wide collapse of the same trees. A wide node holds
// the boxes of a binary node's grandchildren (or of a child that is a leaf);
// the skipped middle boxes contain their children's, and the slab test is
// monotone under inclusion, so dropping them changes neither which leaves are
// reached nor the order or running t with which their triangles are tested:
// the result, ties included, is the binary walk's. Slab tests run when the
// parent is visited; the entry distance travels on the stack and the
// reference's "tAabb > closest t" cull is applied when the entry pops, with
// the closest t of that moment, as in the binary walk.
constexpr int kWideStack = 96;

template <bool kRegular = false>
__device__ __forceinline__ int wide_children(const SlabRay &r, const float4 *n, int codes_out[4], float ta_out[4]) {
    const float4 lx = __ldg(n), ly = __ldg(n + 1), lz = __ldg(n + 2);
    const float4 hx = __ldg(n + 3), hy = __ldg(n + 4), hz = __ldg(n + 5);
    const float4 cd = __ldg(n + 6);
    const float lxs[4] = {lx.x, lx.y, lx.z, lx.w}, lys[4] = {ly.x, ly.y, ly.z, ly.w}, lzs[4] = {lz.x, lz.y, lz.z, lz.w};
    const float hxs[4] = {hx.x, hx.y, hx.z, hx.w}, hys[4] = {hy.x, hy.y, hy.z, hy.w}, hzs[4] = {hz.x, hz.y, hz.z, hz.w};
    const int cs[4] = {fbits(cd.x), fbits(cd.y), fbits(cd.z), fbits(cd.w)};
    int m = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        float ta = 0.0f;
        const bool pass = cs[k] >= 0 && box_test<kRegular>(r, make_float4(lxs[k], lys[k], lzs[k], 0.0f),
                                                           make_float4(hxs[k], hys[k], hzs[k], 0.0f), ta);
        codes_out[k] = pass ? cs[k] : -1;
        ta_out[k] = ta;
        m += pass ? 1 : 0;
    }
    return m;
}

template <bool kAnyHit, class Stk = LocalStack<int2>>
struct WideWalk {
    V3 o, d, oo, od;
    SlabRay wr, br;
    int cur_inst, wide_base, tri_base, sp;
    float t_limit;
    HitId hit;
    Stk stack;

    __device__ __forceinline__ void start(const DeviceScene &s, V3 ro, V3 rd, float limit) {
        o = ro;
        d = rd;
        t_limit = limit;
        hit.t = 1e30f;
        hit.inst = -1;
        hit.tri = -1;
        hit.u = hit.v = 0.0f;
        wr = make_slab_ray<false>(o, d);
        br = wr;
        oo = o;
        od = d;
        cur_inst = -1;
        wide_base = tri_base = 0;
        sp = 0;
        if (!s.has_tlas) return;
        float ta = 0.0f;
        const int code = fbits(s.tlas_root_lo.w);
        if (code >= 0 && slab_test(wr, s.tlas_root_lo, s.tlas_root_hi, ta)) stack.set(sp++, make_int2(code, fbits(ta)));
    }
    __device__ __forceinline__ bool shadow_answer() const { return hit.inst >= 0 && hit.t < t_limit; }

    template <class St>
    __device__ __forceinline__ bool step(const DeviceScene &s, unsigned &err, St &st) {
        if (sp <= 0) return false;
        const int2 e = stack.get(--sp);
        st.pop();
        if (__int_as_float(e.y) > hit.t) return sp > 0;  // entry beyond the closest hit so far
        const int tag = e.x & ((1 << kWideTagBits) - 1), pay = e.x >> kWideTagBits;
        if (tag == kWTagBlasNode || tag == kWTagTlasNode) {
            if (sp + 4 > kWideStack) {
                err |= (tag == kWTagBlasNode) ? kErrBlasStack : kErrTlasStack;
                sp = 0;
                return false;
            }
            const bool blas = tag == kWTagBlasNode;
            const float4 *n = blas ? s.blas4 + 8 * (size_t)(wide_base + pay) : s.tlas4 + 8 * (size_t)pay;
            int cs[4];
            float ts[4];
            wide_children(blas ? br : wr, n, cs, ts);
#pragma unroll
            for (int k = 3; k >= 0; --k)
                if (cs[k] >= 0) stack.set(sp++, make_int2(cs[k], fbits(ts[k])));
        } else if (tag == kWTagBlasLeaf) {
            const int first = pay >> kBlasLeafCountBits;
            const int cnt = (pay & ((1 << kBlasLeafCountBits) - 1)) + 1;
            st.leaf();
            for (int q = 0; q < cnt; ++q) {
                float tt, uu, vv;
                st.tri();
                if (tri_test(oo, od, s.tri_geo + 3 * (size_t)(tri_base + first + q), tt, uu, vv) && tt < hit.t) {
                    hit.t = tt;
                    hit.inst = cur_inst;
                    hit.tri = first + q;
                    hit.u = uu;
                    hit.v = vv;
                }
            }
            if (kAnyHit && hit.inst >= 0 && hit.t < t_limit) {
                sp = 0;
                return false;
            }
        } else if (tag == kWTagTlasLeaf) {
            if (sp + 2 > kWideStack) {
                err |= kErrTlasStack;
                sp = 0;
                return false;
            }
            const int first = pay >> kTlasLeafCountBits;
            const int cnt = (pay & ((1 << kTlasLeafCountBits) - 1)) + 1;
            // instances pop in leaf order; no entry-distance cull at this level
            for (int k = cnt - 1; k >= 0; --k)
                stack.set(sp++, make_int2(((first + k) << kWideTagBits) | kWTagInst, fbits(-3.402823466e+38f)));
        } else {  // instance of a TLAS leaf: enter its BLAS in object space
            const int ii = __ldg(&s.tlas_inst[pay]);
            const float4 *ip = s.instances + 8 * ii;
            const float4 r7 = __ldg(ip + 7);
            if (fbits(r7.y) == 0) return sp > 0;  // mesh without triangles: empty BVH
            const float4 m0 = __ldg(ip), m1 = __ldg(ip + 1), m2 = __ldg(ip + 2), m3 = __ldg(ip + 3);
            const float inv[16] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w,
                                   m2.x, m2.y, m2.z, m2.w, m3.x, m3.y, m3.z, m3.w};
            oo = m4f_transform(inv, o);
            od = m4f_transform_dir(inv, d);
            br = make_slab_ray<true>(oo, od);
            wide_base = fbits(r7.z);
            tri_base = fbits(__ldg(&ip[5].w));
            cur_inst = ii;
            const int mesh = fbits(r7.w);
            const float4 rlo = __ldg(&s.blas_roots[2 * mesh]), rhi = __ldg(&s.blas_roots[2 * mesh + 1]);
            float ta = 0.0f;
            const int code = fbits(rlo.w);
            if (code >= 0 && slab_test(br, rlo, rhi, ta)) stack.set(sp++, make_int2(code, fbits(ta)));
        }
        return sp > 0;
    }
};

// WideWalk split into phases like PhasedWalk: node steps (a wide node's four
// slab tests and pushes, or a TLAS leaf's instance pushes) run for the lanes
// that have them; a lane that pops a BLAS leaf or an instance entry parks it.
// Each lane handles its own entries in its own order with the same running t,
// so the results are WideWalk's, which are BinaryWalk's.
template <bool kAnyHit, class Stk>
struct PhasedWideWalk {
    V3 o, d, oo, od;
    SlabRay wr, br;
    int cur_inst, wide_base, tri_base, sp;
    float t_limit;
    HitId hit;
    int mode;
    int pend;  // kModeLeaf: BLAS leaf payload; kModeInst: TLAS instance slot
    Stk stack;

    __device__ __forceinline__ void start(const DeviceScene &s, V3 ro, V3 rd, float limit) {
        o = ro;
        d = rd;
        t_limit = limit;
        hit.t = 1e30f;
        hit.inst = -1;
        hit.tri = -1;
        hit.u = hit.v = 0.0f;
        wr = make_slab_ray<false>(o, d);
        br = wr;
        oo = o;
        od = d;
        cur_inst = -1;
        wide_base = tri_base = 0;
        sp = 0;
        if (s.has_tlas) {
            float ta = 0.0f;
            const int code = fbits(s.tlas_root_lo.w);
            if (code >= 0 && slab_test(wr, s.tlas_root_lo, s.tlas_root_hi, ta))
                stack.set(sp++, make_int2(code, fbits(ta)));
        }
        mode = sp > 0 ? kModeNode : kModeDone;
    }
    __device__ __forceinline__ bool shadow_answer() const { return hit.inst >= 0 && hit.t < t_limit; }
    __device__ __forceinline__ bool regular(const DeviceScene &s) const {
        return s.proper_boxes && !wr.any_small && !br.any_small;
    }

    template <bool kRegular, class St>
    __device__ __forceinline__ void node_step(const DeviceScene &s, unsigned &err, St &st) {
        if (sp <= 0) {
            mode = kModeDone;
            return;
        }
        const int2 e = stack.get(--sp);
        st.pop();
        if (__int_as_float(e.y) > hit.t) return;  // entry beyond the closest hit so far
        const int tag = e.x & ((1 << kWideTagBits) - 1), pay = e.x >> kWideTagBits;
        if (tag == kWTagBlasNode || tag == kWTagTlasNode) {
            if (sp + 4 > Stk::kCapacity) {
                err |= (tag == kWTagBlasNode) ? kErrBlasStack : kErrTlasStack;
                sp = 0;
                mode = kModeDone;
                return;
            }
            const bool blas = tag == kWTagBlasNode;
            const float4 *n = blas ? s.blas4 + 8 * (size_t)(wide_base + pay) : s.tlas4 + 8 * (size_t)pay;
            int cs[4];
            float ts[4];
            wide_children<kRegular>(blas ? br : wr, n, cs, ts);
#pragma unroll
            for (int k = 3; k >= 0; --k)
                if (cs[k] >= 0) stack.set(sp++, make_int2(cs[k], fbits(ts[k])));
        } else if (tag == kWTagTlasLeaf) {
            if (sp + 2 > Stk::kCapacity) {
                err |= kErrTlasStack;
                sp = 0;
                mode = kModeDone;
                return;
            }
            const int first = pay >> kTlasLeafCountBits;
            const int cnt = (pay & ((1 << kTlasLeafCountBits) - 1)) + 1;
            // instances pop in leaf order; no entry-distance cull at this level
            for (int k = cnt - 1; k >= 0; --k)
                stack.set(sp++, make_int2(((first + k) << kWideTagBits) | kWTagInst, fbits(-3.402823466e+38f)));
        } else {
            pend = pay;
            mode = tag == kWTagBlasLeaf ? kModeLeaf : kModeInst;
        }
    }
    template <class St>
    __device__ __forceinline__ void leaf(const DeviceScene &s, St &st) {
        const int first = pend >> kBlasLeafCountBits;
        const int cnt = (pend & ((1 << kBlasLeafCountBits) - 1)) + 1;
        st.leaf();
        for (int q = 0; q < cnt; ++q) {
            float tt, uu, vv;
            st.tri();
            if (tri_test(oo, od, s.tri_geo + 3 * (size_t)(tri_base + first + q), tt, uu, vv) && tt < hit.t) {
                hit.t = tt;
                hit.inst = cur_inst;
                hit.tri = first + q;
                hit.u = uu;
                hit.v = vv;
            }
        }
        if (kAnyHit && hit.inst >= 0 && hit.t < t_limit) sp = 0;
        mode = sp > 0 ? kModeNode : kModeDone;
    }
    __device__ __forceinline__ void inst(const DeviceScene &s) {
        const int ii = __ldg(&s.tlas_inst[pend]);
        const float4 *ip = s.instances + 8 * ii;
        const float4 r7 = __ldg(ip + 7);
        if (fbits(r7.y) != 0) {  // a mesh without triangles has an empty BVH
            const float4 m0 = __ldg(ip), m1 = __ldg(ip + 1), m2 = __ldg(ip + 2), m3 = __ldg(ip + 3);
            const float inv[16] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w,
                                   m2.x, m2.y, m2.z, m2.w, m3.x, m3.y, m3.z, m3.w};
            oo = m4f_transform(inv, o);
            od = m4f_transform_dir(inv, d);
            br = make_slab_ray<true>(oo, od);
            wide_base = fbits(r7.z);
            tri_base = fbits(__ldg(&ip[5].w));
            cur_inst = ii;
            const int mesh = fbits(r7.w);
            const float4 rlo = __ldg(&s.blas_roots[2 * mesh]), rhi = __ldg(&s.blas_roots[2 * mesh + 1]);
            float ta = 0.0f;
            const int code = fbits(rlo.w);
            if (code >= 0 && slab_test(br, rlo, rhi, ta)) stack.set(sp++, make_int2(code, fbits(ta)));
        }
        mode = sp > 0 ? kModeNode : kModeDone;
    }
};

template <bool kAnyHit, class St = NoStats>
__device__ bool trace_ray_wide(const DeviceScene &s, V3 o, V3 d, float t_limit, HitId &hit, unsigned &err,
                               St &&st = St()) {
    int2 mem[kWideStack];
    WideWalk<kAnyHit> w;
    w.stack.e = mem;
    w.start(s, o, d, t_limit);
    while (w.step(s, err, st)) {
    }
    hit = w.hit;
    return hit.inst >= 0;
}

}  // namespace hdr
#include "shadow4.cuh"
namespace hdr {

// The check of a closest hit found on the 4-wide SAH trees (DeviceScene::sh4_closest
// == 2). The reference's walk (scene.cpp:414-510, bvh.cpp:243-305) skips a node only
// when its slab test fails or its entry distance exceeds the running closest t. No
// triangle lies nearer than the SAH walk's nearest hit t, so that running t never
// drops below t before the hit's triangle is tested. Hence, if every box on the way
// from the TLAS root down to the instance's leaf, and from the instance's BLAS root
// down to the triangle's leaf (object-space ray, BLAS thresholds), passes the
// reference's slab test with an entry distance no farther than t, the reference walk
// tests the triangle and takes it: the same IntersectTriangle arithmetic gives the
// same t, and the SAH walk breaks ties in the reference's walk order. A hit that
// grazes a box the reference's rounding rejects fails the check.
__device__ __noinline__ static bool ref_reaches(const DeviceScene *s, V3 o, V3 d, int inst, int tri, float t) {
    const SlabRay wr = make_slab_ray<false>(o, d);
    const float4 *ip = s->instances + 8 * (size_t)inst;
    const float4 m0 = __ldg(ip), m1 = __ldg(ip + 1), m2 = __ldg(ip + 2), m3 = __ldg(ip + 3);
    const float inv[16] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w,
                           m2.x, m2.y, m2.z, m2.w, m3.x, m3.y, m3.z, m3.w};
    const SlabRay br = make_slab_ray<true>(m4f_transform(inv, o), m4f_transform_dir(inv, d));
    const int node_base = fbits(__ldg(&ip[4].w)), tri_base = fbits(__ldg(&ip[5].w));
    // The boxes on these paths are reachable ones, so DeviceScene::proper_boxes lets
    // the walks' regular slab test stand in for the full one, as in the walks.
    const bool wreg = s->proper_boxes && !wr.any_small, breg = s->proper_boxes && !br.any_small;
    // Both paths are climbed together, one level of each per iteration: every level
    // reads one 32-byte record (the box and the link up), and the two records'
    // loads are issued together so that their latencies overlap. A finished path
    // re-reads its last record (in bounds) and tests nothing.
    int nt = __ldg(&s->ref_inst_leaf[inst]), nb = __ldg(&s->ref_tri_leaf[tri_base + tri]);
    if (nt < 0 || nb < 0) return false;  // in no leaf of the reference's trees: its walk decides
    int lt = nt, lb = nb;
    while (nt >= 0 || nb >= 0) {
        const float4 *tp = s->ref_tlas_path + 2 * (size_t)(nt >= 0 ? nt : lt);
        const float4 *bp = s->ref_blas_path + 2 * (size_t)(node_base + (nb >= 0 ? nb : lb));
        const float4 tlo = __ldg(tp), thi = __ldg(tp + 1), blo = __ldg(bp), bhi = __ldg(bp + 1);
        float ta;
        if (nt >= 0) {
            if (!(wreg ? slab_test_regular(wr, tlo, thi, ta) : slab_test(wr, tlo, thi, ta)) || ta > t) return false;
            lt = nt;
            nt = __float_as_int(tlo.w);
        }
        if (nb >= 0) {
            if (!(breg ? slab_test_regular(br, blo, bhi, ta) : slab_test(br, blo, bhi, ta)) || ta > t) return false;
            lb = nb;
            nb = __float_as_int(blo.w);
        }
    }
    return true;
}

// The reference walk for a ray whose SAH hit the check could not vouch for.
struct RefClosest {
    HitId hit;
    unsigned err;
};
__device__ __noinline__ static RefClosest reference_closest(const DeviceScene *s, V3 o, V3 d) {
    RefClosest r;
    r.err = 0;
    trace_ray_binary<false>(*s, o, d, 0.0f, r.hit, r.err);
    return r;
}

// A ray's walk: the reference's own trees (binary, or their 4-wide collapse),
// or, for closest hits with s.sh4_closest, the Closest4Walk over the 4-wide SAH
// trees: checked against the reference walk (mode 2, the reference's answer bit
// for bit), or alone (mode 1, the reference's answer except where the reference's
// own rounded box tests cull a hit, e.g. on coplanar surfaces).
template <bool kAnyHit>
__device__ __forceinline__ bool trace_ray(const DeviceScene &s, V3 o, V3 d, float t_limit, HitId &hit,
                                          unsigned &err) {
    if (!kAnyHit && s.sh4_closest) {
        NoStats ns;
        const bool found = closest4_ray(s, o, d, hit, err, ns);
        if (s.sh4_closest == 2 && found && !ref_reaches(s.dev, o, d, hit.inst, hit.tri, hit.t)) {
            const RefClosest r = reference_closest(s.dev, o, d);
            hit = r.hit;
            err |= r.err;
            return hit.inst >= 0;
        }
        return found;
    }
    return s.wide ? trace_ray_wide<kAnyHit>(s, o, d, t_limit, hit, err)
                  : trace_ray_binary<kAnyHit>(s, o, d, t_limit, hit, err);
}


// Shadow query of the reference, "IntersectScene(o, d) && Depth < limit"
// (ris_direct_light_integrator.cpp:513-515). With the shadow BVH (s.sh4) its
// 4-wide walk answers it; otherwise the closest-hit walk of the reference's
// trees, stopped as soon as its running closest t drops below limit (the running
// t only decreases, so the answer is the full walk's).
__device__ __forceinline__ bool shadow_ray(const DeviceScene &s, V3 o, V3 d, float limit, unsigned &err) {
    if (s.sh4) {
        NoStats ns;
        return shadow4_ray(s, o, d, limit, err, ns);
    }
    HitId h;
    return trace_ray<true>(s, o, d, limit, h, err) && h.t < limit;
}

// HitRecord (core/hit_record.h:15-27) of IntersectScene (scene.cpp:437-535)
struct Hit {
    V3 position;
    V3 normal;
    V3 smooth_normal;
    V3 dpdu, dpdv;
    V2 uv;
    V3 albedo;
    float depth;
    int prim;      // PrimId == MatId == instance index
    int tri;
    int material;  // PreviewSurface params index, -1 = DefaultMaterial
    int light;     // GetLightAtHit result, -1 = none
};

__device__ __forceinline__ V3 ld3(float4 a) { return V3{a.x, a.y, a.z}; }

__device__ inline Hit make_hit(const DeviceScene &s, V3 o, V3 d, const HitId &h) {
    Hit r;
    const float4 *ip = s.instances + 8 * h.inst;
    const float4 t0 = __ldg(ip + 4), t1 = __ldg(ip + 5), t2 = __ldg(ip + 6), r7 = __ldg(ip + 7);
    const float T[16] = {t0.x, t0.y, t0.z, 0.0f, t1.x, t1.y, t1.z, 0.0f, t2.x, t2.y, t2.z, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f};
    const int tri_base = fbits(t1.w);
    const float4 *a = s.tri_attr + 9 * (size_t)(tri_base + h.tri);
    const float4 a0 = __ldg(a), a1 = __ldg(a + 1), a2 = __ldg(a + 2), a3 = __ldg(a + 3), a4 = __ldg(a + 4);
    const float4 a5 = __ldg(a + 5), a6 = __ldg(a + 6), a7 = __ldg(a + 7), a8 = __ldg(a + 8);
    const float w = 1.0f - h.u - h.v;
    const V3 ng = ld3(a0);
    // bvh.cpp:276-292
    const V2 uv = (V2{a1.w, a2.w} * w + V2{a3.w, a4.w} * h.u) + V2{a5.w, a6.w} * h.v;
    V3 sn = ng;
    if (a0.w != 0.0f) sn = normalized((ld3(a1) * w + ld3(a2) * h.u) + ld3(a3) * h.v);
    const V3 color = (ld3(a4) * w + ld3(a5) * h.u) + ld3(a6) * h.v;
    // scene.cpp:467-474
    r.normal = normalized(m4f_transform_dir(T, ng));
    r.smooth_normal = normalized(m4f_transform_dir(T, sn));
    r.dpdu = normalized(m4f_transform_dir(T, ld3(a7)));
    r.dpdv = normalized(m4f_transform_dir(T, ld3(a8)));
    r.uv = uv;
    r.material = fbits(t2.w);
    r.light = fbits(r7.x);
    if (r.material >= 0) {
        const float4 m0 = __ldg(&s.materials[12 * r.material]);
        r.albedo = ld3(m0);  // PreviewSurfaceParams::DiffuseColor (scene.cpp:476-478)
    } else {
        r.albedo = color;
    }
    r.position = o + h.t * d;
    r.depth = h.t;
    r.prim = h.inst;
    r.tri = h.tri;
    return r;
}

}  // namespace hdr
