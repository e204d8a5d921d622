// PathTracePass (passes/path_trace_pass.h:12-39) in wavefront form, for
// opaque scenes: PathIntegrator::Li / _li (integrators/path_integrator.cpp:
// 48-209) with MisDirectLightIntegrator (mis_direct_light_integrator.cpp:
// 122-269), one vertex of every live path per round:
//   start   (vertex 0)  the pixel prologue of IntegrationPass (seed, jitter,
//                       wavelengths, GBuffer hit), then `sample`
//   sample  (vertex v)  BSDF sample of the vertex (its draws), queued as the
//                       extension ray; the light sample of _integrateNEE (its
//                       draws, after the BSDF's), queued as a shadow ray with
//                       what it adds if unoccluded
//   trace               the phased closest-hit and shadow kernels over the queues
//   connect (vertex v)  NEE term if unoccluded, _integrateBSDFConnection with
//                       the extension hit, throughput, roulette (its draw);
//                       surviving paths are appended to the next active list
// The draws of a pixel keep the order of the one-thread form (BSDF sample,
// light sample, roulette per vertex) and every value is computed by the same
// functions, so the image is that form's. The stream state, throughput and
// running radiance of a path live in SoA planes between kernels. A stream that
// reaches draw 250 would soon need its full 312-word state, which does not
// travel between kernels: such a path is finished in the connect kernel's
// thread, by the one-thread loop (path_li_continue).
// bounce sampling and the NEE estimate inlined: as calls they keep the surface,
// closure, spectral context and random stream they are given in local memory
#define HDR_BOUNCE_INLINE __forceinline__
#include "device/integrator.cuh"

namespace hdr {

namespace {

constexpr unsigned kFlagNee = 1, kFlagOk = 2, kFlagImpossibleNee = 4, kFlagSkipRoulette = 8;
constexpr uint32_t kStreamHandOffLimit = 250;

__device__ __forceinline__ int active_append(int *count, int *list, bool want, int path) {
    const unsigned m = __ballot_sync(__activemask(), want);
    if (!want) return -1;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(count, __popc(m));
    base = __shfl_sync(m, base, leader);
    const int k = base + __popc(m & ((1u << lane) - 1));
    list[k] = path;
    return k;
}

__device__ __forceinline__ int queue_slot(int *count, bool want) {
    const unsigned m = __ballot_sync(__activemask(), want);
    if (!want) return -1;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(count, __popc(m));
    base = __shfl_sync(m, base, leader);
    return base + __popc(m & ((1u << lane) - 1));
}

__device__ __forceinline__ float4 f4(V3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
__device__ __forceinline__ float4 f4(const Spec &s) { return make_float4(s.v[0], s.v[1], s.v[2], s.v[3]); }
__device__ __forceinline__ Spec spec4(float4 a) { return Spec{{a.x, a.y, a.z, a.w}}; }
__device__ __forceinline__ V3 v3(float4 a) { return V3{a.x, a.y, a.z}; }

// BSDF sample and light sample of vertex `v` of path i (surface sf), queued.
__device__ __forceinline__ void sample_vertex(const DeviceScene &s, const PtBuffers &B, size_t i, const Surface &sf,
                                              BounceState &st, const SpectralCtx &sc, MtStream &rng,
                                              const PathRun &pr) {
    const Bounce b = sample_bounce(sf.c, sf.sn, sf.inside, sf.hit.position, sf.ray_d, pr.max_refl, pr.max_refr, st,
                                   sc, rng);
    const int qc = queue_slot(&B.counts[0], b.ok);
    if (qc >= 0) {
        B.q_closest[2 * (size_t)qc] = f4(b.origin, __int_as_float((int)i));
        B.q_closest[2 * (size_t)qc + 1] = f4(b.dir, 0.0f);
    }
    const MisNeePart nee = mis_nee_part(s, sf, b.ok, sc, rng);
    const int qs = queue_slot(&B.counts[1], nee.cast);
    if (qs >= 0) {
        B.q_shadow[2 * (size_t)qs] = f4(nee.o, __int_as_float((int)i));
        B.q_shadow[2 * (size_t)qs + 1] = f4(nee.d, nee.limit);
    }
    const unsigned flags = (nee.cast ? kFlagNee : 0) | (b.ok ? kFlagOk : 0) |
                           (b.impossible_nee ? kFlagImpossibleNee : 0) | (b.skip_roulette ? kFlagSkipRoulette : 0);
    B.b_origin_pdf[i] = f4(b.origin, b.pdf);
    B.b_dir[i] = f4(b.dir, 0.0f);
    B.b_tmul[i] = f4(b.tmul);
    B.nee_add[i] = f4(nee.add);
    B.state[i] = make_int4(st.refl, st.refr, (int)flags, B.state[i].w);
    store_stream(B.rng, i, B.pixels, rng);
}

__device__ __forceinline__ void finish_path(const PtJobD &job, const PtBuffers &B, size_t i, const Spec &total,
                                            const SpectralCtx &sc) {
    const Spec L = spec4(B.outer[i]) * total;
    V3 rgb = spectrum_to_rgb(L, sc.cie);
    if (job.cam.p.has_params && job.cam.p.enable_exposure) rgb = rgb * job.cam.p.exposure_mult;
    job.color[i - (size_t)job.pixel_begin] = make_float4(rgb.x, rgb.y, rgb.z, 1.0f);
}

// the image a batch grid block works on: the last whose first tile is <= blockIdx.x
__device__ __forceinline__ int job_of_block(const PtJobD *table, int n_jobs) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&table[mid].tile_begin) <= (int)blockIdx.x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

}  // namespace

// The rest of a path in one thread (its stream may now pass draw 311). Its
// arguments are values and a device-memory scene, so that no variable of the
// caller has its address taken (which would keep it in local memory).
__device__ __noinline__ Spec pt_finish_in_thread(const DeviceScene *s, Spec total, Spec tp, V3 ro, V3 rd, Hit next,
                                                 BounceState st, SpectralCtx sc, MtStream rng, PathRun pr,
                                                 int first_bounce, unsigned *err) {
    uint64_t spill[312];
    rng.spill = spill;
    const RisRun ris{};
    const ReservoirView rv{};
    unsigned e = 0;
    const Spec r = path_li_continue<false>(*s, total, tp, ro, rd, true, next, st, sc, rng, pr, ris, rv, 0, first_bounce,
                                           e);
    if (e) atomicOr(err, e);
    return r;
}

template <bool kBatch>
__global__ void __launch_bounds__(256) pt_start_kernel(const __grid_constant__ DeviceScene s, const __grid_constant__ PtJobD one, const PtJobD *table,
                                                       int n_jobs, const __grid_constant__ PtBuffers B) {
    const int jk = kBatch ? job_of_block(table, n_jobs) : 0;
    const PtJobD &job = kBatch ? table[jk] : one;
    const CameraD &cam = job.cam;
    const PathRun &pr = job.pr;
    int x, y;
    if (!tile_pixel(cam.width, cam.height, x, y, (int)blockIdx.x - job.tile_begin)) return;
    const size_t li = (size_t)y * (size_t)cam.width + (size_t)x;  // pixel of the image
    const size_t i = (size_t)job.pixel_begin + li;                // path of the batch
    uint64_t spill[312];
    MtStream rng;
    // IntegrationPass prologue (integration_pass.cpp:210-233), as integrate_kernel
    rng.init((uint32_t)li ^ (uint32_t)((unsigned long long)live_frame(cam, job.frame_index) * 12345ULL), spill);
    const float px = (float)x + rng.next_float();
    const float py = (float)y + rng.next_float();
    const RayF ray = camera_ray(cam, px, py, rng);
    const float u = rng.next_float();
    const SpectralCtx sc = make_spectral_ctx(u);
    Hit h;
    const bool has = load_gbuffer_hit(s, job.gb, li, h);
    B.outer[i] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
    if (!has) {  // PathIntegrator::Li without a hit: the background
        const Spec L = (env_present(s) && pr.render_ibl_background) ? rgb_to_spectrum(env_radiance(s, ray.d), sc.up)
                                                                    : spec(0.0f);
        finish_path(job, B, i, L, sc);
        return;
    }
    // PathIntegrator::Li on an opaque hit: Beer on the primary segment, then _li's vertex 0
    Closure c = get_closure(s, h);
    if (!pr.enable_subsurface) c.subsurface = 0.0f;
    const bool inside = dot(c.normal, ray.d) > 0.0f;
    Spec outer = spec(1.0f);
    beer_absorption(outer, c, h.depth, inside, sc);
    const Surface sf = make_surface(s, ray.o, ray.d, h, c, inside);
    B.outer[i] = f4(outer);
    B.total[i] = f4(rgb_to_spectrum(sf.c.emission, sc.up));
    B.tp[i] = f4(spec(1.0f));
    B.ray_o[i] = f4(ray.o, u);
    B.ray_d[i] = f4(ray.d, 0.0f);
    B.state[i] = make_int4(0, 0, 0, jk);  // .w: the path's image
    BounceState st{0, 0};
    sample_vertex(s, B, i, sf, st, sc, rng, pr);
    active_append(&B.counts[4], B.active[0], true, (int)i);
}

// vertex v >= 1 of the paths in `list` (their extension hit is in the hit slots)
__global__ void __launch_bounds__(256) pt_sample_kernel(const __grid_constant__ DeviceScene s, const __grid_constant__ PathRun pr, const __grid_constant__ PtBuffers B, const int *list,
                                                        const int *count, unsigned *err) {
    const int n = *count;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const size_t i = (size_t)list[k];
        MtStream rng = load_stream(B.rng, i, B.pixels);
        const float4 ro4 = B.ray_o[i], rd4 = B.ray_d[i];
        const SpectralCtx sc = make_spectral_ctx(ro4.w);
        const float4 hr = B.hits[i];
        const HitId id{hr.x, __float_as_int(hr.y), __float_as_int(hr.z), hr.w, B.hit_v[i]};
        const V3 ro = v3(ro4), rd = v3(rd4);
        const Hit bh = make_hit(s, ro, rd, id);
        Closure c = get_closure(s, bh);
        if (!pr.enable_subsurface) c.subsurface = 0.0f;
        const bool inside = dot(c.normal, rd) > 0.0f;
        Spec tp = spec4(B.tp[i]);
        beer_absorption(tp, c, bh.depth, inside, sc);
        B.tp[i] = f4(tp);
        const Surface sf = make_surface(s, ro, rd, bh, c, inside);
        const int4 stt = B.state[i];
        BounceState st{stt.x, stt.y};
        sample_vertex(s, B, i, sf, st, sc, rng, pr);
    }
}

// vertex v of the paths in `list`: the vertex's direct light, then the path goes
// on (appended to `next`) or ends (its colour written)
template <bool kBatch>
__global__ void __launch_bounds__(256) pt_connect_kernel(const __grid_constant__ DeviceScene s, const __grid_constant__ PtJobD one, const PtJobD *table,
                                                         const __grid_constant__ PathRun pr, const __grid_constant__ PtBuffers B, const int *list, const int *count, int *next,
                                                         int *next_count, int vertex, unsigned *err) {
    const int n = *count;
    unsigned e = 0;
    // every lane of a warp runs the loop the same number of times (active_append is warp-wide)
    const int stride = gridDim.x * blockDim.x;
    const int rounds = (n + stride - 1) / stride;
    for (int r = 0; r < rounds; ++r) {
        const int k = r * stride + blockIdx.x * blockDim.x + threadIdx.x;
        bool go_on = false;
        size_t i = 0;
        if (k < n) {
            i = (size_t)list[k];
            const int4 stt = B.state[i];
            const unsigned flags = (unsigned)stt.z;
            const float4 ro4 = B.ray_o[i];
            const SpectralCtx sc = make_spectral_ctx(ro4.w);
            MtStream rng = load_stream(B.rng, i, B.pixels);
            // _integrateNEE's term if its shadow ray was unoccluded
            Spec direct = spec(0.0f);
            if ((flags & kFlagNee) && B.occ[i] == 0) direct = direct + spec4(B.nee_add[i]);
            // _integrateBSDFConnection with the extension ray's hit
            const float4 bo = B.b_origin_pdf[i], bd = B.b_dir[i];
            Connection cn;
            cn.b.ok = (flags & kFlagOk) != 0;
            cn.b.origin = v3(bo);
            cn.b.dir = v3(bd);
            cn.b.tmul = spec4(B.b_tmul[i]);
            cn.b.integrand = spec(0.0f);
            cn.b.pdf = bo.w;
            cn.b.impossible_nee = (flags & kFlagImpossibleNee) != 0;
            cn.b.skip_roulette = (flags & kFlagSkipRoulette) != 0;
            cn.has_hit = false;
            if (cn.b.ok) {
                const float4 hr = B.hits[i];
                const HitId id{hr.x, __float_as_int(hr.y), __float_as_int(hr.z), hr.w, B.hit_v[i]};
                if (id.inst >= 0) {
                    cn.hit = make_hit(s, cn.b.origin, cn.b.dir, id);
                    cn.has_hit = true;
                }
            }
            direct = mis_conn_part(s, direct, cn.b.ok, cn, sc);
            Spec tp = spec4(B.tp[i]);
            Spec total = spec4(B.total[i]) + tp * direct;
            bool alive = cn.b.ok;
            if (alive) {
                tp = tp * cn.b.tmul;
                if (vertex >= 1 && !cn.b.skip_roulette && vertex > 3) {
                    const float p = sclampf(spec_max(tp) * pr.roulette, 0.0f, 1.0f);
                    if (rng.next_float() > p)
                        alive = false;
                    else
                        tp = tp * (1.0f / p);
                }
            }
            // _li's loop test for the next vertex: bounce < maxDepth and a hit to shade
            alive = alive && vertex + 1 < pr.max_depth && cn.has_hit;
            if (alive && rng.k >= kStreamHandOffLimit) {
                const BounceState st{stt.x, stt.y};
                total = pt_finish_in_thread(s.dev, total, tp, cn.b.origin, cn.b.dir, cn.hit, st, sc, rng, pr,
                                            vertex + 1, err);
                alive = false;
            }
            if (alive) {
                B.tp[i] = f4(tp);
                B.total[i] = f4(total);
                B.ray_o[i] = f4(cn.b.origin, ro4.w);
                B.ray_d[i] = f4(cn.b.dir, 0.0f);
                store_stream(B.rng, i, B.pixels, rng);
                go_on = true;
            } else {
                finish_path(kBatch ? table[stt.w] : one, B, i, total, sc);
            }
        }
        active_append(next_count, next, go_on, (int)i);
    }
    if (e) atomicOr(err, e);
}

int launch_path_trace_wavefront(const DeviceScene &s, const PtJobD *jobs, int n_jobs, const PtJobD *table,
                                int total_tiles, PtBuffers B, const TraceTuning &tune, unsigned *err,
                                cudaStream_t st) {
    const bool batch = n_jobs > 1;
    const PathRun pr = jobs[0].pr;
    int launches = 0;
    // [0] / [1] closest / shadow queue, [2] / [3] their fetch counters, [4] / [5] active-list lengths
    if (cudaMemsetAsync(B.counts, 0, 8 * sizeof(int), st) != cudaSuccess) return -1;
    (batch ? pt_start_kernel<true> : pt_start_kernel<false>)<<<total_tiles, 256, 0, st>>>(s, jobs[0], table, n_jobs, B);
    ++launches;
    WaveBuffers wb{};
    wb.q_closest = B.q_closest;
    wb.q_shadow = B.q_shadow;
    wb.counts = B.counts;
    wb.fix = B.fix;
    wb.hits = B.hits;
    wb.hit_v = B.hit_v;
    wb.occ = B.occ;
    const int grid = tune.sm_count * 8;
    for (int v = 0; v < pr.max_depth; ++v) {
        const int cur = v & 1, nxt = cur ^ 1;
        if (v > 0) {
            // the queues of this vertex start empty; `cur` was filled by the last connect
            if (cudaMemsetAsync(B.counts, 0, 4 * sizeof(int), st) != cudaSuccess) return -1;
            pt_sample_kernel<<<grid, 256, 0, st>>>(s, pr, B, B.active[cur], &B.counts[4 + cur], err);
            ++launches;
        }
        const int t = launch_wave_trace(s, wb, tune, err, st);
        if (t < 0) return -1;
        launches += t;
        if (cudaMemsetAsync(&B.counts[4 + nxt], 0, sizeof(int), st) != cudaSuccess) return -1;
        (batch ? pt_connect_kernel<true> : pt_connect_kernel<false>)<<<grid, 256, 0, st>>>(
            s, jobs[0], table, pr, B, B.active[cur], &B.counts[4 + cur], B.active[nxt], &B.counts[4 + nxt], v, err);
        ++launches;
    }
    return cudaPeekAtLastError() == cudaSuccess ? launches : -1;
}

}  // namespace hdr
