// Render-job server over the C ABI (declared in include/hdrestir.h). No
// reference counterpart: the reference renders one job per Hydra delegate and
// frame. This is the serving form of the same passes:
//  * scenes are uploaded once and shared by every job that renders them
//    (hdr_scene_share), so a job costs only its frame buffers;
//  * jobs are admitted first-in first-out while the estimate of their frame
//    buffers fits the HBM budget;
//  * each hdr_server_step advances every admitted job by one frame:
//    raycasts on the jobs' own streams, one batched RIS launch per scene
//    (hdr_ris_path_trace_batch: all images' rays traced together), one
//    batched wavefront PathTracePass per scene and path settings
//    (hdr_path_trace_batch: every image's live paths in each launch), then
//    accumulation.
//    Jobs that arrive while others are running join at the next step
//    (continuous batching).
// The context of a job whose result was taken is kept (persistent buffers
// zeroed in stream order) and given to the next job of the same size, so
// steady serving allocates and frees nothing: a cudaFree synchronises the whole
// device and would stall every job in flight.
// HDR_SERVER_SERIAL runs one job at a time, each frame alone: the plain
// per-frame pipeline, kept as the baseline the batched form is measured
// against. A job's images are the same in both modes.
#include <algorithm>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/hdrestir.h"

namespace hdr {
hdr_status set_last_error(hdr_status st, const char *fmt, ...);
}

namespace {

struct Job {
    int64_t id = 0;
    hdr_job_desc d{};
    hdr_ctx *ctx = nullptr;
    int32_t frames_done = 0;
    int32_t state = HDR_JOB_QUEUED;
    size_t bytes = 0;  // admission estimate of its device buffers
    int64_t rendered_at_submit = 0;  // hdr_server::rendered when the job was submitted
};

size_t pixels_of(const hdr_job_desc &d) { return (size_t)d.camera.width * (size_t)d.camera.height; }

// Device bytes a job's context allocates, per pixel: GBuffer 96, Color 16,
// accumulator 16, firefly scratch 16; RIS adds the reservoir (80), the
// stream state and done flag (49) and its share of the batch's ray queues and
// result slots (52 per closest-hit slot, 33 per shadow slot).
size_t job_bytes(const hdr_job_desc &d) {
    const size_t px = pixels_of(d);
    size_t per = 96 + 16 + 16 + (d.firefly ? 16 : 0);
    if (d.pipeline == HDR_JOB_RIS) {
        const int n_nee = std::max(1, d.ris.candidate_count / 2);
        const int n_closest = 1 + std::max(0, d.ris.candidate_count - n_nee);
        per += (d.ris.use_reservoir ? 80 : 0) + 49 + (size_t)n_closest * 52 + (size_t)n_nee * 33;
    }
    return px * per + (1u << 20);
}

}  // namespace

struct hdr_server {
    int device = 0;
    uint32_t flags = 0;
    size_t budget = 0;
    size_t in_use = 0;
    int max_batch = 64;
    int64_t step_pixels = 0;
    double age_weight = 0.5;
    int64_t rendered = 0;  // pixels of every frame the server has rendered (its work clock)
    std::vector<hdr_ctx *> scenes;  // one owner ctx per uploaded scene
    std::deque<std::unique_ptr<Job>> queued;
    std::vector<std::unique_ptr<Job>> active;
    std::map<int64_t, std::unique_ptr<Job>> finished;
    std::vector<int64_t> unreported;  // finished jobs not yet returned by hdr_server_drain_finished
    // Contexts of released jobs, kept for the next jobs: a released context keeps its stream and
    // frame buffers, so a job of the same size allocates nothing (a cudaFree would synchronise
    // the whole device and stall every job in flight). Their bytes count against the budget.
    struct Pooled {
        hdr_ctx *ctx;
        hdr_job_desc d;
        size_t bytes;
    };
    std::vector<Pooled> pool;
    size_t pooled_bytes = 0;
    int64_t next_id = 1;
    std::mutex mu;
};

namespace {

// Frame buffers of two jobs have the same sizes when these agree.
bool same_buffers(const hdr_job_desc &a, const hdr_job_desc &b) {
    return a.camera.width == b.camera.width && a.camera.height == b.camera.height && a.pipeline == b.pipeline &&
           (a.pipeline != HDR_JOB_RIS || a.ris.candidate_count == b.ris.candidate_count);
}

// hands an admitted job's context to the pool (or frees it: pool full, or the job failed)
void release(hdr_server *sv, Job &j, bool keep = true) {
    if (!j.ctx) return;
    sv->in_use -= std::min(sv->in_use, j.bytes);
    if (keep && j.state == HDR_JOB_DONE && sv->pool.size() < (size_t)sv->max_batch &&
        hdr_zero_persistent(j.ctx) == HDR_OK) {
        sv->pool.push_back(hdr_server::Pooled{j.ctx, j.d, j.bytes});
        sv->pooled_bytes += j.bytes;
    } else {
        hdr_ctx_destroy(j.ctx);
    }
    j.ctx = nullptr;
}

// a pooled context whose buffers have job j's sizes (nullptr if none)
hdr_ctx *take_pooled(hdr_server *sv, const Job &j) {
    for (size_t k = 0; k < sv->pool.size(); ++k)
        if (same_buffers(sv->pool[k].d, j.d)) {
            hdr_ctx *c = sv->pool[k].ctx;
            sv->pooled_bytes -= std::min(sv->pooled_bytes, sv->pool[k].bytes);
            sv->pool.erase(sv->pool.begin() + (long)k);
            return c;
        }
    return nullptr;
}

// frees pooled contexts until `need` more bytes fit the budget (or the pool is empty)
void shrink_pool(hdr_server *sv, size_t need) {
    while (!sv->pool.empty() && sv->budget && sv->in_use + sv->pooled_bytes + need > sv->budget) {
        sv->pooled_bytes -= std::min(sv->pooled_bytes, sv->pool.front().bytes);
        hdr_ctx_destroy(sv->pool.front().ctx);
        sv->pool.erase(sv->pool.begin());
    }
}

hdr_status admit(hdr_server *sv) {
    const bool serial = (sv->flags & HDR_SERVER_SERIAL) != 0;
    while (!sv->queued.empty()) {
        Job &j = *sv->queued.front();
        if (serial && !sv->active.empty()) break;
        if (sv->budget && !sv->active.empty() && sv->in_use + j.bytes > sv->budget) break;
        hdr_ctx *c = take_pooled(sv, j);
        hdr_status st = HDR_OK;
        if (!c) {  // a new context: pooled ones of other sizes give way when the budget needs it
            shrink_pool(sv, j.bytes);
            hdr_ctx_desc cd{};
            cd.device = sv->device;
            st = hdr_ctx_create(&c, &cd);
        }
        if (st == HDR_OK) st = hdr_scene_share(c, sv->scenes[(size_t)j.d.scene]);
        std::unique_ptr<Job> job = std::move(sv->queued.front());
        sv->queued.pop_front();
        if (st != HDR_OK) {  // the job fails; its error stays in hdr_last_error
            hdr_ctx_destroy(c);
            job->state = HDR_JOB_FAILED;
            const int64_t id = job->id;
            sv->finished[id] = std::move(job);
            sv->unreported.push_back(id);
            continue;
        }
        job->ctx = c;
        sv->in_use += job->bytes;
        job->state = HDR_JOB_RUNNING;
        sv->active.push_back(std::move(job));
    }
    return HDR_OK;
}

void fail_job(hdr_server *sv, Job &j) {
    j.state = HDR_JOB_FAILED;
    release(sv, j, false);
}

}  // namespace

extern "C" {

hdr_status hdr_server_create(hdr_server **out, const hdr_server_desc *desc) {
    if (!out || !desc) return hdr::set_last_error(HDR_EINVAL, "NULL argument");
    *out = nullptr;
    if (desc->max_batch < 0) return hdr::set_last_error(HDR_EINVAL, "max_batch must be >= 0");
    auto *sv = new hdr_server();
    sv->device = desc->device;
    sv->flags = desc->flags;
    sv->budget = desc->hbm_budget_bytes;
    sv->max_batch = desc->max_batch > 0 ? desc->max_batch : 64;
    sv->step_pixels = desc->step_pixels > 0 ? desc->step_pixels : 0;
    sv->age_weight = desc->age_weight > 0.0f ? desc->age_weight : (desc->age_weight < 0.0f ? 0.0 : 0.5);
    *out = sv;
    return HDR_OK;
}

void hdr_server_destroy(hdr_server *sv) {
    if (!sv) return;
    for (auto &j : sv->active) release(sv, *j, false);
    for (auto &kv : sv->finished) release(sv, *kv.second, false);
    for (auto &p : sv->pool) hdr_ctx_destroy(p.ctx);
    sv->pool.clear();
    for (hdr_ctx *c : sv->scenes) hdr_ctx_destroy(c);
    hdr_trim_frame_memory(sv->device, 0);  // the jobs' frame buffers go back to the device
    delete sv;
}

hdr_status hdr_server_add_scene(hdr_server *sv, const hdr_scene_desc *scene, int32_t *scene_id) {
    if (!sv || !scene || !scene_id) return hdr::set_last_error(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    hdr_ctx_desc cd{};
    cd.device = sv->device;
    hdr_ctx *c = nullptr;
    hdr_status st = hdr_ctx_create(&c, &cd);
    if (st == HDR_OK) st = hdr_scene_upload(c, scene);
    if (st != HDR_OK) {
        hdr_ctx_destroy(c);
        return st;
    }
    *scene_id = (int32_t)sv->scenes.size();
    sv->scenes.push_back(c);
    return HDR_OK;
}

hdr_status hdr_server_submit(hdr_server *sv, const hdr_job_desc *job, int64_t *job_id) {
    if (!sv || !job || !job_id) return hdr::set_last_error(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    if (job->scene < 0 || job->scene >= (int32_t)sv->scenes.size())
        return hdr::set_last_error(HDR_EINVAL, "unknown scene %d", job->scene);
    if (job->pipeline != HDR_JOB_PATH_TRACER && job->pipeline != HDR_JOB_RIS)
        return hdr::set_last_error(HDR_EINVAL, "unknown pipeline %d", job->pipeline);
    if (job->frames < 1) return hdr::set_last_error(HDR_EINVAL, "frames must be >= 1");
    if (job->camera.width <= 0 || job->camera.height <= 0)
        return hdr::set_last_error(HDR_EINVAL, "bad frame size %dx%d", job->camera.width, job->camera.height);
    auto j = std::make_unique<Job>();
    j->id = sv->next_id++;
    j->rendered_at_submit = sv->rendered;
    j->d = *job;
    j->bytes = job_bytes(*job);
    if (sv->budget && j->bytes > sv->budget)
        return hdr::set_last_error(HDR_ENOMEM, "job needs about %zu bytes, above the %zu-byte budget", j->bytes,
                                   sv->budget);
    *job_id = j->id;
    sv->queued.push_back(std::move(j));
    return HDR_OK;
}

hdr_status hdr_server_step(hdr_server *sv, int32_t *jobs_finished) {
    if (!sv) return hdr::set_last_error(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    if (jobs_finished) *jobs_finished = 0;
    hdr_status st = admit(sv);
    if (st != HDR_OK) return st;
    if (sv->active.empty()) return HDR_OK;
    const bool serial = (sv->flags & HDR_SERVER_SERIAL) != 0;
    // this step's jobs: all admitted ones, or by priority up to step_pixels. Key: remaining work
    // less a credit for the work served since the job arrived. Least remaining work alone gives
    // the best median latency, but a large job that arrives early waits behind every later small
    // one and finishes last, so the tail is worse than one job at a time; the credit, measured on
    // the server's own work clock (pixels rendered, so an idle server ages nothing), bounds that.
    std::vector<Job *> run;
    for (auto &j : sv->active) run.push_back(j.get());
    if (sv->step_pixels > 0) {
        auto key = [sv](const Job *j) {
            return (double)(j->d.frames - j->frames_done) * (double)pixels_of(j->d) -
                   sv->age_weight * (double)(sv->rendered - j->rendered_at_submit);
        };
        std::stable_sort(run.begin(), run.end(), [&](const Job *a, const Job *b) { return key(a) < key(b); });
        int64_t px = 0;
        size_t k = 0;
        while (k < run.size() && (k == 0 || px + (int64_t)pixels_of(run[k]->d) <= sv->step_pixels))
            px += (int64_t)pixels_of(run[k++]->d);
        run.resize(k);
    }
    for (const Job *j : run) sv->rendered += (int64_t)pixels_of(j->d);
    // 1. primary rays, each job on its own stream
    for (Job *j : run)
        if (hdr_raycast(j->ctx, &j->d.camera, j->frames_done, 0) != HDR_OK) fail_job(sv, *j);
    // 2. integration: RIS jobs of one scene in batched launches; path-traced jobs of one scene
    //    and one set of path settings in batched wavefront launches
    std::map<int32_t, std::vector<Job *>> ris_by_scene;
    std::vector<std::vector<Job *>> pt_groups;
    for (Job *j : run) {
        if (j->state != HDR_JOB_RUNNING) continue;
        if (j->d.pipeline == HDR_JOB_RIS && !serial) {
            ris_by_scene[j->d.scene].push_back(j);
        } else if (j->d.pipeline == HDR_JOB_RIS) {
            if (hdr_ris_path_trace(j->ctx, &j->d.camera, j->frames_done, &j->d.ris) != HDR_OK) fail_job(sv, *j);
        } else if (!serial) {
            auto same = [j](const std::vector<Job *> &g) {
                return g[0]->d.scene == j->d.scene &&
                       std::memcmp(&g[0]->d.ris.path, &j->d.ris.path, sizeof(hdr_path_settings)) == 0;
            };
            auto g = std::find_if(pt_groups.begin(), pt_groups.end(), same);
            if (g == pt_groups.end()) pt_groups.push_back({j});
            else g->push_back(j);
        } else if (hdr_path_trace(j->ctx, &j->d.camera, j->frames_done, &j->d.ris.path) != HDR_OK) {
            fail_job(sv, *j);
        }
    }
    for (const std::vector<Job *> &js : pt_groups) {
        for (size_t k0 = 0; k0 < js.size(); k0 += (size_t)sv->max_batch) {
            const size_t n = std::min(js.size() - k0, (size_t)sv->max_batch);
            std::vector<hdr_ctx *> ctxs(n);
            std::vector<hdr_camera> cams(n);
            std::vector<int32_t> frames(n);
            std::vector<hdr_path_settings> settings(n);
            for (size_t k = 0; k < n; ++k) {
                const Job &j = *js[k0 + k];
                ctxs[k] = j.ctx;
                cams[k] = j.d.camera;
                frames[k] = j.frames_done;
                settings[k] = j.d.ris.path;
            }
            if (hdr_path_trace_batch(ctxs.data(), (int32_t)n, cams.data(), frames.data(), settings.data()) != HDR_OK)
                for (size_t k = 0; k < n; ++k) fail_job(sv, *js[k0 + k]);
        }
    }
    for (auto &kv : ris_by_scene) {
        const std::vector<Job *> &js = kv.second;
        for (size_t k0 = 0; k0 < js.size(); k0 += (size_t)sv->max_batch) {
            const size_t n = std::min(js.size() - k0, (size_t)sv->max_batch);
            std::vector<hdr_ctx *> ctxs(n);
            std::vector<hdr_camera> cams(n);
            std::vector<int32_t> frames(n);
            std::vector<hdr_ris_params> params(n);
            for (size_t k = 0; k < n; ++k) {
                const Job &j = *js[k0 + k];
                ctxs[k] = j.ctx;
                cams[k] = j.d.camera;
                frames[k] = j.frames_done;
                params[k] = j.d.ris;
            }
            if (hdr_ris_path_trace_batch(ctxs.data(), (int32_t)n, cams.data(), frames.data(), params.data()) !=
                HDR_OK)
                for (size_t k = 0; k < n; ++k) fail_job(sv, *js[k0 + k]);
        }
    }
    // 3. accumulation, then the jobs that have all their frames leave the active set
    for (Job *j : run) {
        if (j->state != HDR_JOB_RUNNING) continue;
        // GpuAccumulationPass semantics (the reference's accumulation when its GPU is enabled): no
        // host round trip per frame, so the step's work stays queued on the streams
        if (hdr_accumulate(j->ctx, j->frames_done, j->d.firefly, HDR_ACCUM_SHADER) != HDR_OK) {
            fail_job(sv, *j);
            continue;
        }
        ++j->frames_done;
    }
    int32_t done = 0;
    std::vector<std::unique_ptr<Job>> keep;
    for (auto &j : sv->active) {
        if (j->state == HDR_JOB_RUNNING && j->frames_done >= j->d.frames) {
            if (hdr_synchronize(j->ctx) != HDR_OK) fail_job(sv, *j);
            if (j->state == HDR_JOB_RUNNING) j->state = HDR_JOB_DONE;
        }
        if (j->state == HDR_JOB_RUNNING) {
            keep.push_back(std::move(j));
        } else {
            ++done;
            const int64_t id = j->id;
            sv->finished[id] = std::move(j);
            sv->unreported.push_back(id);
        }
    }
    sv->active = std::move(keep);
    if (jobs_finished) *jobs_finished = done;
    return HDR_OK;
}

hdr_status hdr_server_job_state(hdr_server *sv, int64_t job_id, int32_t *state, int32_t *frames_done) {
    if (!sv || !state) return hdr::set_last_error(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    const Job *found = nullptr;
    for (auto &j : sv->queued)
        if (j->id == job_id) found = j.get();
    for (auto &j : sv->active)
        if (j->id == job_id) found = j.get();
    auto it = sv->finished.find(job_id);
    if (it != sv->finished.end()) found = it->second.get();
    if (!found) return hdr::set_last_error(HDR_EINVAL, "unknown job %lld", (long long)job_id);
    *state = found->state;
    if (frames_done) *frames_done = found->frames_done;
    return HDR_OK;
}

hdr_status hdr_server_take_result(hdr_server *sv, int64_t job_id, float *rgba, size_t bytes) {
    if (!sv) return hdr::set_last_error(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    auto it = sv->finished.find(job_id);
    if (it == sv->finished.end()) return hdr::set_last_error(HDR_EINVAL, "job %lld has not finished", (long long)job_id);
    Job &j = *it->second;
    hdr_status st = HDR_OK;
    if (j.state != HDR_JOB_DONE) {
        st = hdr::set_last_error(HDR_EDEVICE, "job %lld failed", (long long)job_id);
    } else if (rgba) {
        if (bytes != pixels_of(j.d) * 16)
            return hdr::set_last_error(HDR_EINVAL, "result of job %lld is %zu bytes", (long long)job_id,
                                       pixels_of(j.d) * 16);
        st = hdr_download(j.ctx, "Color", rgba, bytes);
    }
    release(sv, j);
    sv->finished.erase(it);
    return st;
}

hdr_status hdr_server_drain_finished(hdr_server *sv, int64_t *ids, int32_t cap, int32_t *n) {
    if (!sv || !n || (cap > 0 && !ids) || cap < 0) return hdr::set_last_error(HDR_EINVAL, "bad argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    const size_t k = std::min(sv->unreported.size(), (size_t)cap);
    for (size_t q = 0; q < k; ++q) ids[q] = sv->unreported[q];
    sv->unreported.erase(sv->unreported.begin(), sv->unreported.begin() + (long)k);
    *n = (int32_t)k;
    return HDR_OK;
}

hdr_status hdr_server_load(hdr_server *sv, int32_t *queued, int32_t *running, size_t *bytes_in_use) {
    if (!sv) return hdr::set_last_error(HDR_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    if (queued) *queued = (int32_t)sv->queued.size();
    if (running) *running = (int32_t)sv->active.size();
    if (bytes_in_use) *bytes_in_use = sv->in_use;
    return HDR_OK;
}

}  // extern "C"
