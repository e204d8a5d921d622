// RISPathTracePass as a wavefront (maxDepth 1, opaque materials): the same
// per-pixel integrator as the one-thread-per-pixel kernel, with its rays cast
// by dedicated traversal kernels instead of inside the shading code.
//
//   generate : per pixel, draws exactly the numbers IntegrationPass::_execute
//              and RisDirectLightIntegrator draw while building the candidate
//              list (integration_pass.cpp:210-226, ris_direct_light_integrator.cpp:
//              230-262), and appends the rays those draws define to two
//              compacted queues: closest-hit (the bounce ray, BSDF candidates)
//              and shadow (one per NEE candidate that passes the early-outs of
//              _evaluateLightSample, :628-658). It saves the stream state at the
//              end of generation: the reservoir-update numbers start there.
//   trace    : one thread per queued ray; closest hit or "occluded before the
//              light" for the ray's slot.
//   shade    : per pixel, repeats the same draws, reads the slot results instead
//              of tracing, and runs the reference's resampling, temporal merge and
//              colour write-back with the saved stream state supplying the
//              update numbers.
// The shade kernel checks that its own stream ends where generate's did
// whenever it replays every candidate.
//
// Rays whose result cannot reach the image are not queued unless the caller
// asks for them: a generated BSDF candidate contributes only when its ray hits
// light geometry or escapes to an environment, so a scene with neither makes
// every such candidate an empty one whatever the ray hits; without emissive
// materials either, the path's bounce ray cannot change the connection
// candidate's weight. Generate then only advances the stream past those
// candidates, and shade counts them as misses and continues from the stream
// state generate saved.
// Compiled twice: here (namespace hdr) with closures that leave the texture code
// out, for scenes without textures, and in wavefront_tex.cu (namespace
// hdr::textured) with it. Untextured frames keep the registers they had.
#ifndef HDR_WAVE_TEXTURED
#define HDR_TEXTURES 0
#endif
#define HDR_SKY 0        // the launchers never take a scene under the physical sky
#define HDR_BLACKBODY 0  // nor one with blackbody lights (extension)
#define HDR_CANDIDATE_INLINE __forceinline__
#define HDR_BOUNCE_INLINE __forceinline__

#include "device/integrator.cuh"
#include "device/pixel.cuh"

namespace hdr {
#ifdef HDR_WAVE_TEXTURED
namespace textured {
#endif

__device__ __forceinline__ int queue_append(int *counter, bool want) {
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, want);
    if (!want) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

// Kernel parameters of struct type are __grid_constant__: code that takes their
// address (a reference kept in a struct, a call) reads the parameter space
// instead of a per-thread copy in local memory (a few hundred bytes written per
// thread).
__global__ void __launch_bounds__(256)
    ris_generate_kernel(const __grid_constant__ DeviceScene s, const __grid_constant__ CameraD cam, int frame_arg,
                        const __grid_constant__ PathRun pr, const __grid_constant__ RisRun ris,
                        const __grid_constant__ GBufferView gb, const __grid_constant__ WaveBuffers wb, float4 *color,
                        int trace_level, unsigned *err) {
    uint64_t spill[312];
    MtStream rng;
    PixelStart ps;
    if (!pixel_start(s, cam, live_frame(cam, frame_arg), gb, rng, spill, ps)) return;
    const size_t i = ps.i;
    if (!ps.has_hit) {  // PathIntegrator::Li without a hit: background only, no reservoir access
        V3 rgb = v3s(0.0f);
        if (env_present(s) && pr.render_ibl_background)
            rgb = spectrum_to_rgb(rgb_to_spectrum(env_radiance(s, ps.ray.d), ps.sc.up), ps.sc.cie);
        if (cam.p.has_params && cam.p.enable_exposure) rgb = rgb * cam.p.exposure_mult;
        color[i] = make_float4(rgb.x, rgb.y, rgb.z, 1.0f);
        wb.done[i] = 1;
        if (wb.nee_light)
            for (int j = 0; j < wb.n_shadow; ++j) wb.nee_light[i * (size_t)wb.n_shadow + j] = -1;
        return;
    }
    wb.done[i] = 0;
    Closure c = get_closure(s, ps.hit);
    if (!pr.enable_subsurface) c.subsurface = 0.0f;
    const bool inside = dot(c.normal, ps.ray.d) > 0.0f;
    const Surface sf = make_surface(s, ps.ray.o, ps.ray.d, ps.hit, c, inside);
    const size_t cbase = i * (size_t)wb.n_closest, sbase = i * (size_t)wb.n_shadow;
    // the path's bounce ray (_li, path_integrator.cpp:104-111)
    BounceState st{0, 0};
    const Bounce fb = sample_bounce(c, sf.sn, inside, ps.hit.position, ps.ray.d, pr.max_refl, pr.max_refr, st, ps.sc,
                                    rng);
    {
        const int q = queue_append(&wb.counts[0], fb.ok && trace_level >= kTraceBounceRay);
        if (q >= 0) {
            wb.q_closest[2 * (size_t)q] =
                make_float4(fb.origin.x, fb.origin.y, fb.origin.z, __int_as_float(wb.slot_base_closest + (int)cbase));
            wb.q_closest[2 * (size_t)q + 1] = make_float4(fb.dir.x, fb.dir.y, fb.dir.z, 0.0f);
        }
    }
    // technique split and NEE candidates (:239-246, :553-589)
    const int N = ris.candidate_count;
    const int n_nee = smaxi(1, N / 2), n_bsdf = smaxi(0, N - n_nee);
    for (int j = 0; j < n_nee; ++j) {
        int li;
        LightSampleD ls;
        V3 o, d;
        float lim = 0.0f;
        const bool proposed = propose_candidate(s, ps.hit.position, rng, li, ls);
        if (wb.nee_light) wb.nee_light[sbase + j] = proposed ? li : -1;
        const bool want = proposed && ris_nee_shadow_ray(s, sf, li, ls, ris.skip_vis, o, d, lim);
        const int q = queue_append(&wb.counts[1], want);
        if (q >= 0) {
            wb.q_shadow[2 * (size_t)q] =
                make_float4(o.x, o.y, o.z, __int_as_float(wb.slot_base_shadow + (int)(sbase + j)));
            wb.q_shadow[2 * (size_t)q + 1] = make_float4(d.x, d.y, d.z, lim);
        }
    }
    // generated BSDF candidates (:442-450)
    const int n_fresh = n_bsdf - ((fb.ok && fb.pdf > 0.0f) ? 1 : 0);
    if (trace_level < kTraceAllBsdfRays) {  // their rays are not cast: only the stream has to advance
        const BounceDraws bd = bounce_draws_of(c, sf.sn, inside, ps.ray.d, ps.sc);
        for (int k = 0; k < n_fresh; ++k) {
            BounceState st2{0, 0};
            bounce_draws(bd, 1, 1, st2, rng);
        }
        store_stream(wb.rng_state, i, wb.pixels, rng);
        return;
    }
    for (int k = 0; k < n_fresh; ++k) {
        BounceState st2{0, 0};
        const Bounce b = sample_bounce(c, sf.sn, inside, ps.hit.position, ps.ray.d, 1, 1, st2, ps.sc, rng);
        const int q = queue_append(&wb.counts[0], b.ok);
        if (q >= 0) {
            wb.q_closest[2 * (size_t)q] = make_float4(b.origin.x, b.origin.y, b.origin.z,
                                                      __int_as_float(wb.slot_base_closest + (int)(cbase + 1 + k)));
            wb.q_closest[2 * (size_t)q + 1] = make_float4(b.dir.x, b.dir.y, b.dir.z, 0.0f);
        }
    }
    store_stream(wb.rng_state, i, wb.pixels, rng);
}


// Trace kernels. Rays of a warp take very different numbers of steps (shadow
// rays towards random lights: 43 % of lane-steps did work when each lane
// traced a fixed ray), so the default form is persistent: a lane whose ray is
// finished takes the next queued ray (one atomic per warp for all its idle
// lanes) and every lane steps its own walk, one stack entry per iteration,
// until the queue is drained. fetch_at counts the rays handed out.
constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ int fetch_ray(int *fetch_at, int n, bool need, bool &drained) {
    const unsigned want = __ballot_sync(kFullMask, need);
    if (!want || drained) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(want) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(fetch_at, __popc(want));
    base = __shfl_sync(kFullMask, base, leader);
    if (base + __popc(want) >= n) drained = true;  // warp-uniform
    const int k = base + __popc(want & ((1u << lane) - 1));
    return (need && k < n) ? k : -1;
}

// Stack entries below kSharedDepth live in the block's shared memory (one
// column per thread), deeper ones in local memory.
constexpr int kTraceThreads = 128;
constexpr int kSharedDepth = 24;
static_assert(kTraceStack == kWideStack, "one spill size for both walks");

template <bool kWide, bool kAnyHit>
struct TraceWalk {
    using Entry = typename std::conditional<kWide, int2, int>::type;
    using Stack = SplitStack<Entry, kSharedDepth, kTraceThreads>;
    using type = typename std::conditional<kWide, WideWalk<kAnyHit, Stack>, BinaryWalk<kAnyHit, Stack>>::type;
};

// Phased schedule (PhasedWalk): node steps run while at least `quorum` lanes
// of the warp are stepping nodes; then the parked leaves, instance entries and
// finished rays of all lanes are served, and finished lanes take the next
// queued rays.
// Shared-memory stack entries per thread of the phased wide walk (8-byte
// entries: the same 12 KB per block as the binary walk's 24 four-byte ones).
constexpr int kSharedDepthWide = 12;

// kShallow (binary walk only): the scene's trees fit a kShallowStack-entry
// stack, which then lives wholly in shared memory (20 KB per block).
template <bool kWide, bool kAnyHit, bool kShallow>
struct PhasedTraceWalk {
    static_assert(!(kWide && kShallow), "the shallow stack serves the binary walk");
    using Entry = typename std::conditional<kWide, int2, int>::type;
    static constexpr int kShared = kShallow ? kShallowStack : (kWide ? kSharedDepthWide : kSharedDepth);
    using Stack = typename std::conditional<kShallow, ColumnStack<Entry, kShared, kTraceThreads>,
                                            SplitStack<Entry, kShared, kTraceThreads>>::type;
    using type = typename std::conditional<kWide, PhasedWideWalk<kAnyHit, Stack>, PhasedWalk<kAnyHit, Stack>>::type;
};

template <class Stk, class Entry>
__device__ __forceinline__ void bind_deep(Stk &, Entry *) {}
template <class Entry, int kDepth, int kThreads>
__device__ __forceinline__ void bind_deep(SplitStack<Entry, kDepth, kThreads> &st, Entry *deep) {
    st.deep = deep;
}

template <bool kWide, bool kShallow, bool kAnyHit, class Put>
__device__ __forceinline__ void phased_trace(const DeviceScene &s, const float4 *__restrict__ q,
                                             const int *__restrict__ order, int n, int *fetch_at, int quorum,
                                             Put put, unsigned &e) {
    using PW = PhasedTraceWalk<kWide, kAnyHit, kShallow>;
    __shared__ typename PW::Entry col[PW::kShared * kTraceThreads];
    typename PW::Entry deep[kShallow ? 1 : kTraceStack - PW::kShared];
    typename PW::type w;
    w.stack.col = col + threadIdx.x;
    bind_deep(w.stack, deep);
    w.mode = kModeDone;
    NoStats ns;
    int slot = -1;
    bool drained = false;
    for (;;) {
        const bool done = w.mode == kModeDone;
        if (done && slot >= 0) {
            put(slot, w);
            slot = -1;
        }
        const int k = fetch_ray(fetch_at, n, done, drained);
        if (done) {
            if (k >= 0) {
                const size_t r = order ? (size_t)order[k] : (size_t)k;
                const float4 a = q[2 * r], b = q[2 * r + 1];
                w.start(s, V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, kAnyHit ? b.w : 0.0f);
                slot = __float_as_int(a.w);
            } else {
                w.mode = kModeIdle;
            }
        }
        if (!__any_sync(kFullMask, w.mode != kModeIdle)) break;
        do {
            if (w.mode == kModeNode) {
                if (w.regular(s))
                    w.template node_step<true>(s, e, ns);
                else
                    w.template node_step<false>(s, e, ns);
            }
        } while (__popc(__ballot_sync(kFullMask, w.mode == kModeNode)) >= quorum);
        if (w.mode == kModeLeaf) w.leaf(s, ns);
        if (w.mode == kModeInst) w.inst(s);
    }
}

// Resident blocks per SM the phased kernels are compiled for (64 registers for
// the binary walk, 80 for the wide one).
template <bool kWide>
constexpr int phased_min_blocks() {
    return kWide ? 6 : 8;
}

// Closest hits on the reference's trees for the queue entries order[0..*count)
// (order nullptr: entries 0..*count), fetch counting the entries handed out.
template <bool kWide, bool kShallow>
__global__ void __launch_bounds__(kTraceThreads, phased_min_blocks<kWide>()) trace_closest_phased_kernel(DeviceScene s, const float4 *__restrict__ q,
                                                                             const int *order, const int *count,
                                                                             int *fetch, float4 *hits, float *hit_v,
                                                                             int quorum, unsigned *err) {
    unsigned e = 0;
    phased_trace<kWide, kShallow, false>(
        s, q, order, *count, fetch, quorum,
        [&](int slot, const auto &w) {
            hits[slot] = make_float4(w.hit.t, __int_as_float(w.hit.inst), __int_as_float(w.hit.tri), w.hit.u);
            hit_v[slot] = w.hit.v;
        },
        e);
    if (e) atomicOr(err, e);
}

template <bool kWide, bool kShallow>
__global__ void __launch_bounds__(kTraceThreads, phased_min_blocks<kWide>()) trace_shadow_phased_kernel(DeviceScene s, const float4 *__restrict__ q,
                                                                            const int *count, int *fetch,
                                                                            unsigned char *occ, int quorum,
                                                                            unsigned *err) {
    unsigned e = 0;
    phased_trace<kWide, kShallow, true>(
        s, q, nullptr, *count, fetch, quorum,
        [&](int slot, const auto &w) { occ[slot] = w.shadow_answer() ? 1 : 0; }, e);
    if (e) atomicOr(err, e);
}

// Shadow queue over the shadow BVH (DeviceScene::sh4): persistent lanes, each on
// its own ray's 4-wide walk. Node steps run while at least `quorum` lanes of
// the warp are on node entries; then the parked leaves (triangle tests) and
// instance entries of all lanes are served, and finished lanes take new rays.
constexpr int kSh4Shared = 32;

template <int kMinBlocks>
__global__ void __launch_bounds__(kTraceThreads, kMinBlocks) trace_shadow4_kernel(DeviceScene s, const float4 *__restrict__ q,
                                                                       const int *count, int *fetch,
                                                                       unsigned char *occ, int quorum,
                                                                       unsigned *err) {
    __shared__ int col[kSh4Shared * kTraceThreads];
    int deep[kSh4Stack - kSh4Shared];
    Shadow4Walk<Sh4SplitStack<kSh4Shared, kTraceThreads>> w;
    w.stack.col = col + threadIdx.x;
    w.stack.deep = deep;
    w.mode = kSh4ModeDone;
    w.blocked = false;
    const int n = *count;
    unsigned e = 0;
    NoStats ns;
    int slot = -1;
    bool drained = false;
    for (;;) {
        const bool done = w.mode == kSh4ModeDone;
        if (done && slot >= 0) {
            occ[slot] = w.blocked ? 1 : 0;
            slot = -1;
        }
        const int k = fetch_ray(fetch, n, done, drained);
        if (done) {
            if (k >= 0) {
                const float4 a = q[2 * (size_t)k], b = q[2 * (size_t)k + 1];
                w.start(s, V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, b.w);
                slot = __float_as_int(a.w);
            } else {
                w.mode = kSh4ModeIdle;
            }
        }
        if (!__any_sync(kFullMask, w.mode != kSh4ModeIdle)) break;
        do {
            if (w.mode == kSh4ModeNode) w.node_step(s, e, ns);
        } while (__popc(__ballot_sync(kFullMask, w.mode == kSh4ModeNode)) >= quorum);
        if (w.mode == kSh4ModeLeaf) w.leaf(s, ns);
        if (w.mode == kSh4ModeInst) w.inst(s, ns);
    }
    if (e) atomicOr(err, e);
}

// Closest-hit queue over the 4-wide SAH trees (DeviceScene::sh4_closest),
// scheduled like trace_shadow4_kernel (Closest4Walk). With sh4_closest == 2 the
// hits are then checked by check_closest_kernel.
template <int kMinBlocks>
__global__ void __launch_bounds__(kTraceThreads, kMinBlocks) trace_closest4_kernel(DeviceScene s, const float4 *__restrict__ q,
                                                                                 int *counts, float4 *hits,
                                                                                 float *hit_v, int quorum,
                                                                                 unsigned *err) {
    __shared__ int col[kSh4Shared * kTraceThreads];
    int deep[kSh4Stack - kSh4Shared];
    Closest4Walk<Sh4SplitStack<kSh4Shared, kTraceThreads>> w;
    w.stack.col = col + threadIdx.x;
    w.stack.deep = deep;
    w.mode = kSh4ModeDone;
    w.best_inst = -1;
    const int n = counts[0];
    unsigned e = 0;
    NoStats ns;
    int slot = -1;
    bool drained = false;
    for (;;) {
        const bool done = w.mode == kSh4ModeDone;
        if (done && slot >= 0) {
            hits[slot] = make_float4(w.best_t, __int_as_float(w.best_inst), __int_as_float(w.best_tri), w.best_u);
            hit_v[slot] = w.best_v;
            slot = -1;
        }
        const int k = fetch_ray(&counts[3], n, done, drained);
        if (done) {
            if (k >= 0) {
                const float4 a = q[2 * (size_t)k], b = q[2 * (size_t)k + 1];
                w.start(s, V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z});
                slot = __float_as_int(a.w);
            } else {
                w.mode = kSh4ModeIdle;
            }
        }
        if (!__any_sync(kFullMask, w.mode != kSh4ModeIdle)) break;
        do {
            if (w.mode == kSh4ModeNode) w.node_step(s, e, ns);
        } while (__popc(__ballot_sync(kFullMask, w.mode == kSh4ModeNode)) >= quorum);
        if (w.mode == kSh4ModeLeaf) w.leaf(s, ns);
        if (w.mode == kSh4ModeInst) w.inst(s, ns);
    }
    if (e) atomicOr(err, e);
}

// The check of the SAH walk's closest hits (sh4_closest == 2), one thread per
// queue entry: an entry whose hit ref_reaches cannot vouch for is listed in
// fix[0..*n_fix) for the reference walk. A miss needs no check: the SAH trees'
// boxes hold every triangle, so the reference walk finds no hit either.
__global__ void __launch_bounds__(256) check_closest_kernel(DeviceScene s, const float4 *__restrict__ q,
                                                            const int *count, const float4 *__restrict__ hits,
                                                            int *fix, int *n_fix) {
    const int n = *count;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float4 a = q[2 * (size_t)k];
        const float4 h = hits[__float_as_int(a.w)];
        const int inst = __float_as_int(h.y);
        if (inst < 0) continue;
        const float4 b = q[2 * (size_t)k + 1];
        if (!ref_reaches(s.dev, V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, inst, __float_as_int(h.z), h.x))
            fix[atomicAdd(n_fix, 1)] = k;
    }
}

// The shadow-ray queue q (count / fetch counters on the device, answers into occ).
int launch_shadow_queue(const DeviceScene &s, const float4 *q, const int *count, int *fetch, unsigned char *occ,
                        const TraceTuning &tune, unsigned *err, cudaStream_t st) {
    const int tgrid = tune.sm_count * tune.blocks_per_sm;
    if (s.sh4) {
        // register budget: 64 (8 resident blocks), 80 (6) or 90 (5) per thread
        auto k = tune.shadow_shape == 0 ? trace_shadow4_kernel<8>
                                        : (tune.shadow_shape == 1 ? trace_shadow4_kernel<6> : trace_shadow4_kernel<5>);
        k<<<tgrid, kTraceThreads, 0, st>>>(s, q, count, fetch, occ, tune.node_quorum, err);
    } else {
        const bool shallow = s.shallow && (tune.mode & kTraceSplitStack) == 0;
        auto shadow = s.wide ? trace_shadow_phased_kernel<true, false>
                             : (shallow ? trace_shadow_phased_kernel<false, true>
                                        : trace_shadow_phased_kernel<false, false>);
        shadow<<<tgrid, kTraceThreads, 0, st>>>(s, q, count, fetch, occ, tune.node_quorum, err);
    }
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

template <bool kWide, bool kRefill>
__global__ void __launch_bounds__(kTraceThreads) trace_closest_kernel(DeviceScene s, const float4 *__restrict__ q,
                                                                      int *counts, float4 *hits, float *hit_v,
                                                                      unsigned *err) {
    using TW = TraceWalk<kWide, false>;
    __shared__ typename TW::Entry col[kSharedDepth * kTraceThreads];
    typename TW::Entry deep[kTraceStack - kSharedDepth];
    typename TW::type w;
    w.stack.col = col + threadIdx.x;
    w.stack.deep = deep;
    const int n = counts[0];
    unsigned e = 0;
    NoStats ns;
    if (!kRefill) {
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
            const float4 a = q[2 * (size_t)k], b = q[2 * (size_t)k + 1];
            w.start(s, V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, 0.0f);
            while (w.step(s, e, ns)) {
            }
            const int slot = __float_as_int(a.w);
            hits[slot] = make_float4(w.hit.t, __int_as_float(w.hit.inst), __int_as_float(w.hit.tri), w.hit.u);
            hit_v[slot] = w.hit.v;
        }
    } else {
        int slot = -1;
        bool drained = false;
        for (;;) {
            const int k = fetch_ray(&counts[3], n, slot < 0, drained);
            if (k >= 0) {
                const float4 a = q[2 * (size_t)k], b = q[2 * (size_t)k + 1];
                w.start(s, V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, 0.0f);
                slot = __float_as_int(a.w);
            }
            if (!__any_sync(kFullMask, slot >= 0)) break;
            if (slot >= 0 && !w.step(s, e, ns)) {
                hits[slot] = make_float4(w.hit.t, __int_as_float(w.hit.inst), __int_as_float(w.hit.tri), w.hit.u);
                hit_v[slot] = w.hit.v;
                slot = -1;
            }
        }
    }
    if (e) atomicOr(err, e);
}

template <bool kWide, bool kRefill>
__global__ void __launch_bounds__(kTraceThreads) trace_shadow_kernel(DeviceScene s, const float4 *__restrict__ q,
                                                                     int *counts, unsigned char *occ, unsigned *err) {
    using TW = TraceWalk<kWide, true>;
    __shared__ typename TW::Entry col[kSharedDepth * kTraceThreads];
    typename TW::Entry deep[kTraceStack - kSharedDepth];
    typename TW::type w;
    w.stack.col = col + threadIdx.x;
    w.stack.deep = deep;
    const int n = counts[1];
    unsigned e = 0;
    NoStats ns;
    if (!kRefill) {
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
            const float4 a = q[2 * (size_t)k], b = q[2 * (size_t)k + 1];
            w.start(s, V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, b.w);
            while (w.step(s, e, ns)) {
            }
            occ[__float_as_int(a.w)] = w.shadow_answer() ? 1 : 0;
        }
    } else {
        int slot = -1;
        bool drained = false;
        for (;;) {
            const int k = fetch_ray(&counts[2], n, slot < 0, drained);
            if (k >= 0) {
                const float4 a = q[2 * (size_t)k], b = q[2 * (size_t)k + 1];
                w.start(s, V3{a.x, a.y, a.z}, V3{b.x, b.y, b.z}, b.w);
                slot = __float_as_int(a.w);
            }
            if (!__any_sync(kFullMask, slot >= 0)) break;
            if (slot >= 0 && !w.step(s, e, ns)) {
                occ[slot] = w.shadow_answer() ? 1 : 0;
                slot = -1;
            }
        }
    }
    if (e) atomicOr(err, e);
}

template <int kThreads, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks)
    ris_shade_kernel(const __grid_constant__ DeviceScene s, const __grid_constant__ CameraD cam, int frame_arg,
                     const __grid_constant__ PathRun pr, const __grid_constant__ RisRun ris,
                     const __grid_constant__ GBufferView gb, const __grid_constant__ ReservoirView rv,
                     const __grid_constant__ WaveBuffers wb, float4 *color, int trace_level, unsigned *err) {
    uint64_t spill[312];
    MtStream rng;
    PixelStart ps;
    if (!pixel_start<kThreads>(s, cam, live_frame(cam, frame_arg), gb, rng, spill, ps)) return;
    const size_t i = ps.i;
    if (wb.done[i]) return;
    unsigned e = 0;
    const TracedResults tr{&s, wb.hits + i * (size_t)wb.n_closest, wb.hit_v + i * (size_t)wb.n_closest,
                           wb.occ + i * (size_t)wb.n_shadow, trace_level, wb.q_winner, wb.counts + 4, (int)i};
    const MtStream gen_end = load_stream(wb.rng_state, i, wb.pixels);
    // past 311 draws the state lives in local memory only: replay instead
    const MtStream *gen_end_ptr = gen_end.k < 312 ? &gen_end : nullptr;
    // the wavefront form runs only for maxDepth 1 and opaque scenes
    const Spec L =
        path_li<true, TracedResults, true>(s, tr, ps.ray.o, ps.ray.d, true, ps.hit, ps.sc, rng, pr, ris, rv, i, gen_end_ptr, e);
    V3 rgb = spectrum_to_rgb(L, ps.sc.cie);
    if (cam.p.has_params && cam.p.enable_exposure) rgb = rgb * cam.p.exposure_mult;
    color[i] = make_float4(rgb.x, rgb.y, rgb.z, 1.0f);
    if (e) atomicOr(err, e);
}

int launch_wave_trace(const DeviceScene &s, WaveBuffers wb, const TraceTuning &tune, unsigned *err, cudaStream_t st,
                      cudaEvent_t *ev_begin, cudaEvent_t *ev_end) {
    auto mark = [&](cudaEvent_t *ev, int k) { return !ev || cudaEventRecord(ev[k], st) == cudaSuccess; };
    const int tgrid = tune.sm_count * tune.blocks_per_sm;
    const bool refill = (tune.mode & kTraceLanePerRay) == 0;
    const bool phased = refill && (tune.mode & kTraceUnphased) == 0;
    const bool shallow = s.shallow && (tune.mode & kTraceSplitStack) == 0;
    if (!mark(ev_begin, 0)) return -1;
    int launches = 2;
    auto reference_phased = s.wide    ? trace_closest_phased_kernel<true, false>
                            : shallow ? trace_closest_phased_kernel<false, true>
                                      : trace_closest_phased_kernel<false, false>;
    if (s.sh4_closest) {
        auto closest = tune.shadow_shape == 0 ? trace_closest4_kernel<8>
                                              : (tune.shadow_shape == 1 ? trace_closest4_kernel<6>
                                                                        : trace_closest4_kernel<5>);
        closest<<<tgrid, kTraceThreads, 0, st>>>(s, wb.q_closest, wb.counts, wb.hits, wb.hit_v, tune.node_quorum, err);
        if (s.sh4_closest == 2 && wb.fix) {  // (no fix list: the queue has no entries)
            // counts[6] entries the check rejected, counts[7] of them handed out
            if (cudaMemsetAsync(wb.counts + 6, 0, 2 * sizeof(int), st) != cudaSuccess) return -1;
            check_closest_kernel<<<tune.sm_count * 8, 256, 0, st>>>(s, wb.q_closest, wb.counts, wb.hits, wb.fix,
                                                                      wb.counts + 6);
            reference_phased<<<tgrid, kTraceThreads, 0, st>>>(s, wb.q_closest, wb.fix, wb.counts + 6, wb.counts + 7,
                                                              wb.hits, wb.hit_v, tune.node_quorum, err);
            launches += 2;
        }
    } else if (phased) {
        reference_phased<<<tgrid, kTraceThreads, 0, st>>>(s, wb.q_closest, nullptr, wb.counts, wb.counts + 3, wb.hits,
                                                          wb.hit_v, tune.node_quorum, err);
    } else {
        auto closest = s.wide ? (refill ? trace_closest_kernel<true, true> : trace_closest_kernel<true, false>)
                              : (refill ? trace_closest_kernel<false, true> : trace_closest_kernel<false, false>);
        closest<<<tgrid, kTraceThreads, 0, st>>>(s, wb.q_closest, wb.counts, wb.hits, wb.hit_v, err);
    }
    if (!mark(ev_end, 0) || !mark(ev_begin, 1)) return -1;
    if (phased || s.sh4) {
        if ((launch_shadow_queue)(s, wb.q_shadow, wb.counts + 1, wb.counts + 2, wb.occ, tune, err, st) < 0) return -1;
    } else {
        auto shadow = s.wide ? (refill ? trace_shadow_kernel<true, true> : trace_shadow_kernel<true, false>)
                             : (refill ? trace_shadow_kernel<false, true> : trace_shadow_kernel<false, false>);
        shadow<<<tgrid, kTraceThreads, 0, st>>>(s, wb.q_shadow, wb.counts, wb.occ, err);
    }
    if (!mark(ev_end, 1)) return -1;
    return cudaPeekAtLastError() == cudaSuccess ? launches : -1;
}

namespace {
PathRun path_run(const RisParamsD &p) {
    PathRun pr;
    pr.max_depth = p.max_depth;
    pr.enable_subsurface = p.enable_subsurface != 0;
    pr.max_refl = p.max_refl;
    pr.max_refr = p.max_refr;
    pr.render_ibl_background = p.render_ibl_background != 0;
    pr.roulette = p.roulette;
    return pr;
}
RisRun ris_run(const RisParamsD &p) {
    RisRun ris;
    ris.candidate_count = p.candidate_count;
    ris.use_reservoir = p.use_reservoir != 0;
    ris.skip_vis = p.skip_visibility != 0;
    ris.m_cap = p.m_cap;
    ris.reproj = p.reproj;
    return ris;
}
}  // namespace

int launch_ris_generate(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                        GBufferView gb, WaveBuffers wb, float4 *color, int trace_level, unsigned *err,
                        cudaStream_t st) {
    ris_generate_kernel<<<tile_blocks(cam.width, cam.height), 256, 0, st>>>(s, cam, frame_index, path_run(p),
                                                                             ris_run(p), gb, wb, color, trace_level,
                                                                             err);
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

int launch_ris_shade(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                     GBufferView gb, ReservoirView rv, WaveBuffers wb, float4 *color, int trace_level, unsigned *err,
                     cudaStream_t st, const TraceTuning &tune) {
    const PathRun pr = path_run(p);
    const RisRun ris = ris_run(p);
    const int blocks = tile_blocks(cam.width, cam.height);
    switch (tune.shade_shape) {
        case 1:
            ris_shade_kernel<256, 2><<<blocks, 256, 0, st>>>(s, cam, frame_index, pr, ris, gb, rv, wb, color,
                                                             trace_level, err);
            break;
        case 2:
            ris_shade_kernel<128, 3><<<tile_blocks<128>(cam.width, cam.height), 128, 0, st>>>(
                s, cam, frame_index, pr, ris, gb, rv, wb, color, trace_level, err);
            break;
        case 3:
            ris_shade_kernel<128, 4><<<tile_blocks<128>(cam.width, cam.height), 128, 0, st>>>(
                s, cam, frame_index, pr, ris, gb, rv, wb, color, trace_level, err);
            break;
        default:
            ris_shade_kernel<256, 1><<<blocks, 256, 0, st>>>(s, cam, frame_index, pr, ris, gb, rv, wb, color,
                                                             trace_level, err);
    }
    return cudaPeekAtLastError() == cudaSuccess ? 1 : -1;
}

// After the queued winner shadow rays: a pixel whose winner turned out occluded
// gets what the test on the spot would have given it, throughput 0 (so the
// direct term is 0) and Color = Beer * emission of its surface.
__global__ void __launch_bounds__(256) ris_winner_fixup_kernel(DeviceScene s, CameraD cam, int frame_arg, PathRun pr,
                                                              GBufferView gb, ReservoirView rv, const float4 *q,
                                                              const int *count, const unsigned char *occ,
                                                              float4 *color) {
    const int frame_index = live_frame(cam, frame_arg);
    const int n = *count;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int px = __float_as_int(q[2 * (size_t)k].w);
        if (!occ[px]) continue;
        const int x = px % cam.width, y = px / cam.width;
        MtStream rng;
        rng.init((uint32_t)px ^ (uint32_t)((unsigned long long)frame_index * 12345ULL), nullptr);
        const float fx = (float)x + rng.next_float();
        const float fy = (float)y + rng.next_float();
        const RayF ray = camera_ray(cam, fx, fy, rng);
        const SpectralCtx sc = make_spectral_ctx(rng.next_float());
        Hit h;
        if (!load_gbuffer_hit(s, gb, (size_t)px, h)) continue;
        Closure c = get_closure(s, h);
        if (!pr.enable_subsurface) c.subsurface = 0.0f;
        const bool inside = dot(c.normal, ray.d) > 0.0f;
        Spec tp = spec(1.0f);
        beer_absorption(tp, c, h.depth, inside, sc);
        if (rv.throughput) rv.throughput[px] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        const Spec L = tp * (rgb_to_spectrum(c.emission, sc.up) + spec(0.0f));
        V3 rgb = spectrum_to_rgb(L, sc.cie);
        if (cam.p.has_params && cam.p.enable_exposure) rgb = rgb * cam.p.exposure_mult;
        color[px] = make_float4(rgb.x, rgb.y, rgb.z, 1.0f);
    }
}

int launch_winner_visibility(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                             GBufferView gb, ReservoirView rv, WaveBuffers wb, float4 *color, unsigned *err,
                             cudaStream_t st, const TraceTuning &tune) {
    if ((launch_shadow_queue)(s, wb.q_winner, wb.counts + 4, wb.counts + 5, wb.occ_winner, tune, err, st) < 0)
        return -1;
    ris_winner_fixup_kernel<<<tune.sm_count * 4, 256, 0, st>>>(s, cam, frame_index, path_run(p), gb, rv, wb.q_winner,
                                                               wb.counts + 4, wb.occ_winner, color);
    return cudaPeekAtLastError() == cudaSuccess ? 2 : -1;
}

int launch_ris_wavefront(const DeviceScene &s, const CameraD &cam, int frame_index, const RisParamsD &p,
                         GBufferView gb, ReservoirView rv, WaveBuffers wb, float4 *color, int trace_level,
                         unsigned *err, cudaStream_t st, const TraceTuning &tune, cudaEvent_t *ev_begin,
                         cudaEvent_t *ev_end) {
    // [0] closest rays queued, [1] shadow rays queued, [2] / [3] shadow / closest rays handed out,
    // [4] / [5] winner shadow rays queued / handed out
    if (cudaMemsetAsync(wb.counts, 0, (wb.q_winner ? 6 : 4) * sizeof(int), st) != cudaSuccess) return -1;
    auto mark = [&](cudaEvent_t *ev, int k) { return !ev || cudaEventRecord(ev[k], st) == cudaSuccess; };
    if (!mark(ev_begin, 0)) return -1;
    // callee names in parentheses: no argument-dependent lookup, so the hdr::textured build
    // calls its own launchers, not hdr::'s
    if ((launch_ris_generate)(s, cam, frame_index, p, gb, wb, color, trace_level, err, st) < 0) return -1;
    if (!mark(ev_end, 0)) return -1;
    const int traced =
        (launch_wave_trace)(s, wb, tune, err, st, ev_begin ? ev_begin + 1 : nullptr, ev_end ? ev_end + 1 : nullptr);
    if (traced < 0) return -1;
    if (!mark(ev_begin, 3)) return -1;
    if ((launch_ris_shade)(s, cam, frame_index, p, gb, rv, wb, color, trace_level, err, st, tune) < 0) return -1;
    int launches = 2 + traced;
    if (wb.q_winner) {  // the winners' shadow rays, then the pixels they found occluded
        if ((launch_winner_visibility)(s, cam, frame_index, p, gb, rv, wb, color, err, st, tune) < 0) return -1;
        launches += 2;
    }
    if (!mark(ev_end, 3)) return -1;
    return launches;
}

#ifdef HDR_WAVE_TEXTURED
}  // namespace textured
#endif
}  // namespace hdr
