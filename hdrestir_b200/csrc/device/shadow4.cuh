// Shadow-ray walk over the shadow BVH (host/shadow_bvh.h): "is there a hit
// nearer than the limit", the visibility query of _evaluateLightSample
// (ris_direct_light_integrator.cpp:628-658) and of the MIS integrator's NEE.
//
// The answer is the reference's: a triangle blocks the ray exactly when
// IntersectTriangle (bvh.cpp:8-30, restated in tri_test) returns t < limit for
// it in its instance's space, which is the same arithmetic on the same records
// whatever tree finds it. The trees only cull, so their box tests are made
// conservative: the near and far slab distances are computed with the
// reciprocal direction shrunk and grown by 2^-20 and offset by 2^-20 of the
// origin term, which covers the rounding of the fused form
// t = bound * (1/d) - o * (1/d), so a box is never skipped when a ray hits a
// triangle inside it. (The reference culls with its own rounded slab tests on
// its own boxes; it can miss a hit that grazes a box face by an ulp, which no
// tree change reproduces. Such rays are counted by the tests.)
#pragma once

#include "gf.cuh"
#include "sh4_layout.h"

namespace hdr {

constexpr int kSh4Tlas = 0, kSh4Blas = 1, kSh4Inst = 2, kSh4Leaf = 3;
constexpr unsigned kErrShadowStack = 16u;

// A ray prepared for the 4-child box tests.
struct Sh4Ray {
    float inx, iny, inz;  // near bounds: 1/d shrunk by 2^-20
    float ifx, ify, ifz;  // far bounds: 1/d grown by 2^-20
    float onx, ony, onz;  // near offsets: -o/d, conservatively lowered
    float ofx, ofy, ofz;  // far offsets: -o/d, conservatively raised
    int sgn;              // bit k: direction component k is negative (its near bound is the box max)
};

__device__ __forceinline__ void sh4_axis(float o, float d, float &in, float &iff, float &on, float &of, int &neg) {
    const float dd = fabsf(d) > 1e-20f ? d : copysignf(1e-20f, d);
    const float inv = __frcp_rn(dd);  // IEEE reciprocal, rounded to nearest
    in = inv * (1.0f - 9.5367431640625e-07f);
    iff = inv * (1.0f + 9.5367431640625e-07f);
    const float oi = -o * inv;
    const float e = fabsf(oi) * 9.5367431640625e-07f;
    on = -o * in - e;
    of = -o * iff + e;
    neg = dd < 0.0f ? 1 : 0;
}

__device__ __forceinline__ Sh4Ray sh4_ray(V3 o, V3 d) {
    Sh4Ray r;
    int nx, ny, nz;
    sh4_axis(o.x, d.x, r.inx, r.ifx, r.onx, r.ofx, nx);
    sh4_axis(o.y, d.y, r.iny, r.ify, r.ony, r.ofy, ny);
    sh4_axis(o.z, d.z, r.inz, r.ifz, r.onz, r.ofz, nz);
    r.sgn = nx | (ny << 1) | (nz << 2);
    return r;
}

// The four child boxes of node `np` against the ray: bit k of the result is set
// when child k's box overlaps [0, limit] along the ray; tn[k] its entry distance.
__device__ __forceinline__ unsigned sh4_children(const float4 *np, const Sh4Ray &r, float limit, float tn[4],
                                                 int4 &code) {
    const int sx = r.sgn & 1, sy = (r.sgn >> 1) & 1, sz = (r.sgn >> 2) & 1;
    const float4 nx = __ldg(np + sx), fx = __ldg(np + 1 - sx);
    const float4 ny = __ldg(np + 2 + sy), fy = __ldg(np + 3 - sy);
    const float4 nz = __ldg(np + 4 + sz), fz = __ldg(np + 5 - sz);
    const float4 c = __ldg(np + 6);
    code = make_int4(__float_as_int(c.x), __float_as_int(c.y), __float_as_int(c.z), __float_as_int(c.w));
    const float n_x[4] = {nx.x, nx.y, nx.z, nx.w}, f_x[4] = {fx.x, fx.y, fx.z, fx.w};
    const float n_y[4] = {ny.x, ny.y, ny.z, ny.w}, f_y[4] = {fy.x, fy.y, fy.z, fy.w};
    const float n_z[4] = {nz.x, nz.y, nz.z, nz.w}, f_z[4] = {fz.x, fz.y, fz.z, fz.w};
    unsigned mask = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float t0 = fmaxf(fmaxf(__fmaf_rn(n_x[k], r.inx, r.onx), __fmaf_rn(n_y[k], r.iny, r.ony)),
                               fmaxf(__fmaf_rn(n_z[k], r.inz, r.onz), 0.0f));
        const float t1 = fminf(fminf(__fmaf_rn(f_x[k], r.ifx, r.ofx), __fmaf_rn(f_y[k], r.ify, r.ofy)),
                               fminf(__fmaf_rn(f_z[k], r.ifz, r.ofz), limit));
        tn[k] = t0;
        mask |= (t0 <= t1 ? 1u : 0u) << k;
    }
    return mask;
}

// IntersectTriangle (bvh.cpp:8-30) on a tri_geo record, as tri_test.
__device__ __forceinline__ bool sh4_tri_blocks(V3 o, V3 d, const float4 *g, float limit) {
    const float4 g0 = __ldg(g), g1 = __ldg(g + 1), g2 = __ldg(g + 2);
    const V3 v0{g0.x, g0.y, g0.z};
    const V3 e1{g0.w, g1.x, g1.y};
    const V3 e2{g1.z, g1.w, g2.x};
    const V3 pvec = cross(d, e2);
    const float det = dot(e1, pvec);
    if (fabsf(det) <= 9.99999993922529e-09f) return false;  // std::abs(det) < 1e-8 (double)
    const float inv_det = 1.0f / det;
    const V3 tvec = o - v0;
    const float u = dot(tvec, pvec) * inv_det;
    if (u < 0.0f || u > 1.0f) return false;
    const V3 qvec = cross(tvec, e1);
    const float v = dot(d, qvec) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return false;
    const float t = dot(e2, qvec) * inv_det;
    return t > 1e-4f && t < limit;
}


// Phases of a shadow walk: the entry in hand is a TLAS or BLAS node, a BLAS
// leaf's triangles, or an instance to enter; or the walk is over.
enum : int { kSh4ModeNode = 0, kSh4ModeLeaf = 1, kSh4ModeInst = 2, kSh4ModeDone = 3, kSh4ModeIdle = 4 };

// The walk as a resumable state machine. Entries are (payload << 2) | tag:
// nodes (TLAS / BLAS node index), instances (instance index) and BLAS leaves
// ((first triangle << 2) | (count - 1)). The entry in hand is `cur`; its tag
// sets the mode. A node step tests the node's four child boxes, takes a hit
// leaf (or else the nearest hit child) into hand and pushes the other hits,
// the nearest last. Leaf and instance entries are served in their own phases,
// so the node steps of a warp stay in step.
template <class Stk>
struct Shadow4Walk {
    V3 o, d, oo, od;
    Sh4Ray wr, br;
    float limit;
    int sp, cur, mode;
    bool blocked;
    Stk stack;

    __device__ __forceinline__ void take(int e) {
        cur = e;
        const int tag = e & 3;
        mode = e < 0 ? kSh4ModeDone : (tag == kSh4Leaf ? kSh4ModeLeaf : (tag == kSh4Inst ? kSh4ModeInst : kSh4ModeNode));
    }
    __device__ __forceinline__ void next() { take(sp > 0 ? stack.get(--sp) : -1); }

    __device__ __forceinline__ void start(const DeviceScene &s, V3 ro, V3 rd, float lim) {
        o = ro;
        d = rd;
        oo = ro;
        od = rd;
        limit = lim;
        wr = sh4_ray(ro, rd);
        br = wr;
        sp = 0;
        blocked = false;
        take(s.has_tlas ? ((0 << 2) | kSh4Tlas) : -1);
    }
    __device__ __forceinline__ void finish(bool hit) {
        blocked = hit;
        sp = 0;
        cur = -1;
        mode = kSh4ModeDone;
    }

    // one node entry (mode kSh4ModeNode)
    template <class St>
    __device__ __forceinline__ void node_step(const DeviceScene &s, unsigned &err, St &st) {
        st.pop();
        const int tag = cur & 3, idx = cur >> 2;
        const bool blas = tag == kSh4Blas;
        float tn[4];
        int4 code;
        const unsigned hits = sh4_children(s.sh4_nodes + 7 * (size_t)idx, blas ? br : wr, limit, tn, code);
        if (!hits) {
            next();
            return;
        }
        if (sp + 4 > Stk::kCapacity) {
            err |= kErrShadowStack;
            finish(false);
            return;
        }
        const int codes[4] = {code.x, code.y, code.z, code.w};
        int ent[4];
        int pick = -1;
        float t_pick = 3.402823466e+38f;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int c = codes[k];
            ent[k] = c >= 0 ? ((c << 2) | tag) : (blas ? (((~c) << 2) | kSh4Leaf) : ((((~c) >> 2) << 2) | kSh4Inst));
            if (!((hits >> k) & 1u)) continue;
            // a leaf first (its triangles may end the walk), else the nearest child
            const float key = (c < 0 && blas) ? -1.0f : tn[k];
            if (key < t_pick) {
                t_pick = key;
                pick = k;
            }
        }
        // the other hits, the nearest of them pushed last
        int second = -1;
        float t_second = 3.402823466e+38f;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k != pick && ((hits >> k) & 1u) && tn[k] < t_second) {
                t_second = tn[k];
                second = k;
            }
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k != pick && k != second && ((hits >> k) & 1u)) stack.set(sp++, ent[k]);
        if (second >= 0) stack.set(sp++, ent[second]);
        take(ent[pick]);
    }

    // a BLAS leaf's triangles (mode kSh4ModeLeaf)
    template <class St>
    __device__ __forceinline__ void leaf(const DeviceScene &s, St &st) {
        const int p = cur >> 2, first = p >> 2, cnt = (p & 3) + 1;
        st.leaf();
        for (int q = 0; q < cnt; ++q) {
            st.tri();
            if (sh4_tri_blocks(oo, od, s.sh4_tris + 3 * (size_t)(first + q), limit)) {
                finish(true);
                return;
            }
        }
        next();
    }

    // enter an instance (mode kSh4ModeInst): its ray, then its BLAS root
    template <class St>
    __device__ __forceinline__ void inst(const DeviceScene &s, St &st) {
        const int ii = cur >> 2;
        st.leaf();
        const float4 *ip = s.instances + 8 * (size_t)ii;
        const float4 m0 = __ldg(ip), m1 = __ldg(ip + 1), m2 = __ldg(ip + 2), m3 = __ldg(ip + 3);
        const float inv[16] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w,
                               m2.x, m2.y, m2.z, m2.w, m3.x, m3.y, m3.z, m3.w};
        oo = m4f_transform(inv, o);
        od = m4f_transform_dir(inv, d);
        br = sh4_ray(oo, od);
        take((__ldg(&s.sh4_inst_root[ii]) << 2) | kSh4Blas);
    }

    template <class St>
    __device__ __forceinline__ void step(const DeviceScene &s, unsigned &err, St &st) {
        if (mode == kSh4ModeNode)
            node_step(s, err, st);
        else if (mode == kSh4ModeLeaf)
            leaf(s, st);
        else if (mode == kSh4ModeInst)
            inst(s, st);
    }
};

// Entries below kShared in this thread's column of a shared-memory array, the
// rest (up to kSh4Stack) in a per-thread local array.
template <int kShared, int kThreads>
struct Sh4SplitStack {
    static constexpr int kCapacity = kSh4Stack;
    int *col;
    int *deep;
    __device__ __forceinline__ int get(int k) const { return k < kShared ? col[k * kThreads] : deep[k - kShared]; }
    __device__ __forceinline__ void set(int k, int v) {
        if (k < kShared)
            col[k * kThreads] = v;
        else
            deep[k - kShared] = v;
    }
};

template <class T, int kCap>
struct Sh4LocalStack {
    static constexpr int kCapacity = kCap;
    T e[kCap];
    __device__ __forceinline__ T get(int k) const { return e[k]; }
    __device__ __forceinline__ void set(int k, T v) { e[k] = v; }
};

// Closest-hit walk over the same trees (IntersectScene, scene.cpp:409-535), with
// the reference's answer: boxes are culled only beyond the running closest t
// (conservatively, as above), every triangle test is IntersectTriangle in its
// instance's space, and among hits at equal t the smallest (instance position in
// the reference TLAS's leaf order, triangle index in the reference BLAS order)
// wins, the hit the reference's left-first walks meet first with their strict
// `<`. Same phases as the shadow walk.
template <class Stk>
struct Closest4Walk {
    V3 o, d, oo, od;
    Sh4Ray wr, br;
    float best_t, best_u, best_v;
    int best_inst, best_tri, best_rank;
    int cur_inst, cur_rank;
    int sp, cur, mode;
    Stk stack;

    __device__ __forceinline__ void take(int e) {
        cur = e;
        const int tag = e & 3;
        mode = e < 0 ? kSh4ModeDone : (tag == kSh4Leaf ? kSh4ModeLeaf : (tag == kSh4Inst ? kSh4ModeInst : kSh4ModeNode));
    }
    __device__ __forceinline__ void next() { take(sp > 0 ? stack.get(--sp) : -1); }

    __device__ __forceinline__ void start(const DeviceScene &s, V3 ro, V3 rd) {
        o = ro;
        d = rd;
        oo = ro;
        od = rd;
        wr = sh4_ray(ro, rd);
        br = wr;
        best_t = 1e30f;  // IntersectScene's initial closest distance
        best_u = best_v = 0.0f;
        best_inst = best_tri = -1;
        best_rank = 0x7fffffff;
        cur_inst = -1;
        cur_rank = 0x7fffffff;
        sp = 0;
        take(s.has_tlas ? ((0 << 2) | kSh4Tlas) : -1);
    }

    template <class St>
    __device__ __forceinline__ void node_step(const DeviceScene &s, unsigned &err, St &st) {
        st.pop();
        const int tag = cur & 3, idx = cur >> 2;
        const bool blas = tag == kSh4Blas;
        float tn[4];
        int4 code;
        const unsigned hits = sh4_children(s.sh4_nodes + 7 * (size_t)idx, blas ? br : wr, best_t, tn, code);
        if (!hits) {
            next();
            return;
        }
        if (sp + 4 > Stk::kCapacity) {
            err |= kErrShadowStack;
            sp = 0;
            take(-1);
            return;
        }
        const int codes[4] = {code.x, code.y, code.z, code.w};
        int ent[4];
        int pick = -1, second = -1;
        float t_pick = 3.402823466e+38f, t_second = 3.402823466e+38f;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int c = codes[k];
            ent[k] = c >= 0 ? ((c << 2) | tag) : (blas ? (((~c) << 2) | kSh4Leaf) : ((((~c) >> 2) << 2) | kSh4Inst));
            if (!((hits >> k) & 1u)) continue;
            if (tn[k] < t_pick) {
                t_second = t_pick;
                second = pick;
                t_pick = tn[k];
                pick = k;
            } else if (tn[k] < t_second) {
                t_second = tn[k];
                second = k;
            }
        }
        // the nearest in hand, the next nearest pushed last (taken next), the others below it
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k != pick && k != second && ((hits >> k) & 1u)) stack.set(sp++, ent[k]);
        if (second >= 0) stack.set(sp++, ent[second]);
        take(ent[pick]);
    }

    template <class St>
    __device__ __forceinline__ void leaf(const DeviceScene &s, St &st) {
        const int p = cur >> 2, first = p >> 2, cnt = (p & 3) + 1;
        st.leaf();
        for (int q = 0; q < cnt; ++q) {
            st.tri();
            const float4 *g = s.sh4_tris + 3 * (size_t)(first + q);
            float t, u, v;
            if (!tri_test(oo, od, g, t, u, v)) continue;
            const int tri = __float_as_int(__ldg(&g[2].y));
            if (t < best_t || (t == best_t && (cur_rank < best_rank || (cur_rank == best_rank && tri < best_tri)))) {
                best_t = t;
                best_u = u;
                best_v = v;
                best_inst = cur_inst;
                best_rank = cur_rank;
                best_tri = tri;
            }
        }
        next();
    }

    template <class St>
    __device__ __forceinline__ void inst(const DeviceScene &s, St &st) {
        const int ii = cur >> 2;
        st.leaf();
        const float4 *ip = s.instances + 8 * (size_t)ii;
        const float4 m0 = __ldg(ip), m1 = __ldg(ip + 1), m2 = __ldg(ip + 2), m3 = __ldg(ip + 3);
        const float inv[16] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w,
                               m2.x, m2.y, m2.z, m2.w, m3.x, m3.y, m3.z, m3.w};
        oo = m4f_transform(inv, o);
        od = m4f_transform_dir(inv, d);
        br = sh4_ray(oo, od);
        cur_inst = ii;
        cur_rank = __ldg(&s.sh4_inst_rank[ii]);
        take((__ldg(&s.sh4_inst_root[ii]) << 2) | kSh4Blas);
    }

    template <class St>
    __device__ __forceinline__ void step(const DeviceScene &s, unsigned &err, St &st) {
        if (mode == kSh4ModeNode)
            node_step(s, err, st);
        else if (mode == kSh4ModeLeaf)
            leaf(s, st);
        else if (mode == kSh4ModeInst)
            inst(s, st);
    }
    __device__ __forceinline__ bool found() const { return best_inst >= 0; }
};

// One ray's answer (callers outside the wavefront trace kernels).
template <class St>
__device__ inline bool shadow4_ray(const DeviceScene &s, V3 o, V3 d, float limit, unsigned &err, St &st) {
    Shadow4Walk<Sh4LocalStack<int, kSh4Stack>> w;
    w.start(s, o, d, limit);
    while (w.mode != kSh4ModeDone) w.step(s, err, st);
    return w.blocked;
}

}  // namespace hdr

namespace hdr {
// Closest hit of one ray (callers outside the wavefront trace kernels).
template <class St>
__device__ inline bool closest4_ray(const DeviceScene &s, V3 o, V3 d, HitId &hit, unsigned &err, St &st) {
    Closest4Walk<Sh4LocalStack<int, kSh4Stack>> w;
    w.start(s, o, d);
    while (w.mode != kSh4ModeDone) w.step(s, err, st);
    hit.t = w.best_t;
    hit.inst = w.best_inst;
    hit.tri = w.best_tri;
    hit.u = w.best_u;
    hit.v = w.best_v;
    return w.found();
}
}  // namespace hdr
