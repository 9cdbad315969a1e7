// The serving loop: render sessions and probe queries that arrive at any time, on one
// GPU. No counterpart in the reference (its Renderer serves one viewport).
//
// - A render thread owns a batch (a wave of path-tracing members, integrator.cu). Queued
//   sessions are admitted, in arrival order, while a live slot is free and the device
//   memory budget holds their scene (uploaded on first use) and their film; idle scenes
//   are evicted least recently used first to make room. Every live session advances in
//   the same passes; the thread keeps two passes in flight, and while the newer one runs
//   admits, retires and notes progress (first image, completion). A
//   finished session's image leaves through a pinned buffer, its copy queued beside the
//   passes that follow and its session retired once it has landed; nothing the thread
//   does between passes waits for the device.
// - A probe thread runs probe queries on its own high-priority stream, so a probe's
//   kernel starts ahead of the next render kernel instead of behind the queued passes.
//   Probes go through lr_probe_static, which allocates nothing, up to its pixel limit.
// - Scenes stay resident in HBM between requests until evicted; a session's film and
//   sampling state (a cursor into its stateless sampler) stay resident while it lives.
// Times are host steady-clock seconds since the server started.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.hpp"
#include "device.hpp"

namespace {

using Clock = std::chrono::steady_clock;

struct SceneSlot {
    const lr_scene *scene = nullptr;
    lr_gpu_scene *gs = nullptr;  // the resident upload, or null
    uint64_t bytes = 0;          // its device bytes while resident
    uint64_t last_use = 0;       // a tick of the server's clock of uses (LRU)
    int users = 0;               // live sessions and running probes
    bool loading = false;
    uint64_t image_bytes = 0;    // what each session's light records add for a dome's image
};

struct Request {
    int kind = LR_REQUEST_RENDER;
    int state = LR_REQUEST_QUEUED;
    int status = LR_OK;
    std::string message;
    uint32_t scene = 0;
    lr_settings settings{};
    lr_frame frame{};
    bool framed = false;
    float *rgba = nullptr;
    uint32_t *faces = nullptr;
    float *distances = nullptr;
    uint32_t flags = 0;
    uint32_t member = 0;
    uint64_t pixels = 0;
    uint32_t samples = 0, samples_done = 0;
    uint64_t bytes = 0;  // device bytes a live session holds (film, image, lights)
    double submitted = -1, admitted = -1, first = -1, finished = -1;
    // A finished session's image on its way out: the pinned buffer it lands in and the
    // batch's ticket for the copy.
    float *staging = nullptr;
    uint64_t staging_bytes = 0, ticket = 0;
};

// Pinned host buffers that finished images land in before they are copied to the
// caller's memory, so that a copy runs beside the passes after it rather than draining
// them; reused by size (powers of two from 1 MiB), at most kStagingLimit bytes in all.
constexpr uint64_t kStagingLimit = 1ull << 30;

uint64_t staging_size(uint64_t bytes) {
    uint64_t size = 1ull << 20;
    while (size < bytes) size <<= 1;
    return size;
}

double seconds_since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

}  // namespace

struct lr_server {
    lr_server_settings cfg{};
    lr_context *ctx = nullptr, *probe_ctx = nullptr, *load_ctx = nullptr;
    lr_batch *batch = nullptr;
    uint64_t wave_bytes = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_loaded;
    std::deque<SceneSlot> scenes;  // by id (deques keep references stable as they grow)
    std::deque<Request> requests;
    std::deque<uint64_t> render_queue, probe_queue;
    std::vector<uint64_t> live;
    uint64_t bytes_in_use = 0;  // resident scenes and live sessions
    uint64_t tick = 0;
    bool stopping = false;
    std::thread render_thread, probe_thread;
    Clock::time_point t0;
    lr_server_stats stats{};
    // The batch's autotuner runs (lr_batch_tune) once enough sessions are live to stand for
    // the mix, and again when the mix may have changed (every kRetune seconds).
    double tuned_at = -1.0;
    uint64_t tunings = 0;
    std::vector<std::pair<uint64_t, float *>> staging_free;  // (bytes, buffer)
    uint64_t staging_total = 0;
};

namespace {

using lr::fail;

void check(int status) {
    if (status != LR_OK) fail(status, lr_last_error());
}

// A session's film and image, its records, and a dome's image in its light records
// (per texel a float4 and a cumulative weight).
uint64_t session_bytes(const Request &r, uint64_t image_bytes) { return r.pixels * 32 + (1u << 20) + image_bytes; }

uint64_t dome_image_bytes(const lr_scene *scene) {
    for (size_t i = 0; i < scene->lights.size(); i++)
        if (scene->lights[i].shape == LR_LIGHT_DOME && !scene->light_images[i].empty()) {
            const uint64_t pixels = scene->light_images[i].size() / 3;
            return pixels * 20 + (uint64_t)scene->lights[i].image_height * 4 + 64;
        }
    return 0;
}

// Live sessions that make the mix worth tuning for, and the seconds between tunings.
constexpr size_t kTuneSessions = 32;
constexpr double kRetune = 20.0;

// The budget left for scenes and sessions once the pool is paid for.
uint64_t available(const lr_server *s) {
    return s->cfg.budget_bytes > s->wave_bytes ? s->cfg.budget_bytes - s->wave_bytes : 0;
}

// Upload size before the upload: about 230 bytes a triangle (BVH2 entries for both box
// tests, triangles, wide collapses, shading) and 12 a point, rounded up.
uint64_t upload_estimate(const lr_scene *scene) {
    lr_scene_info info{};
    check(lr_scene_info_get(scene, &info));
    return info.triangle_count * 256 + info.point_count * 16 + (1u << 20);
}

// Frees idle resident scenes, least recently used first, until `need` more bytes fit
// the budget; false when they cannot now. Called with the lock held.
bool make_room(lr_server *s, uint64_t need) {
    const uint64_t budget = available(s);
    while (s->bytes_in_use + need > budget) {
        SceneSlot *victim = nullptr;
        for (auto &slot : s->scenes)
            if (slot.gs && slot.users == 0 && !slot.loading && (!victim || slot.last_use < victim->last_use))
                victim = &slot;
        if (!victim) return false;
        lr_gpu_scene_destroy(victim->gs);
        victim->gs = nullptr;
        s->bytes_in_use -= victim->bytes;
        victim->bytes = 0;
        s->stats.evictions++;
    }
    return true;
}

// Makes scene `index` resident through `ctx` (waiting for another thread's upload of
// it), taking room from idle scenes. False when it does not fit the budget now (room
// held by live sessions or other uploads); fails when it never could. Called with the
// lock held; uploads without it.
bool ensure_resident(lr_server *s, std::unique_lock<std::mutex> &lk, uint32_t index, lr_context *ctx) {
    SceneSlot &slot = s->scenes[index];
    s->cv_loaded.wait(lk, [&] { return !slot.loading; });
    if (slot.gs) return true;
    const uint64_t estimate = upload_estimate(slot.scene);
    if (estimate > available(s)) fail(LR_LIMIT, "the scene does not fit the server's memory budget");
    if (!make_room(s, estimate)) return false;
    slot.loading = true;
    s->bytes_in_use += estimate;
    lk.unlock();
    lr_gpu_scene *gs = nullptr;
    const int status = lr_gpu_scene_upload(ctx, slot.scene, &gs);
    std::string message = status == LR_OK ? "" : lr_last_error();
    lr_gpu_scene_info gi{};
    if (status == LR_OK) lr_gpu_scene_info_get(gs, &gi);
    lk.lock();
    slot.loading = false;
    s->bytes_in_use -= estimate;
    if (status != LR_OK) {
        s->cv_loaded.notify_all();
        fail(status, message);
    }
    slot.gs = gs;
    slot.bytes = gi.bytes;
    s->bytes_in_use += gi.bytes;
    s->stats.uploads++;
    s->cv_loaded.notify_all();
    return true;
}

void finish_request(lr_server *s, Request &r, int status, const std::string &message) {
    r.status = status;
    r.message = message;
    r.state = status == LR_OK ? LR_REQUEST_DONE : LR_REQUEST_FAILED;
    r.finished = seconds_since(s->t0);
    if (status != LR_OK) s->stats.failed++;
    s->cv_done.notify_all();
}

// Host seconds of admitting between two passes: one pass runs meanwhile (about a
// millisecond or two), so a burst of admissions spreads over the gaps that follow.
constexpr double kAdmitSeconds = 5e-4;

// Admits queued sessions while slots and memory allow, for about kAdmitSeconds while
// sessions are live (an idle server admits all it can). Lock held.
void admit(lr_server *s, std::unique_lock<std::mutex> &lk) {
    const Clock::time_point start = Clock::now();
    while (!s->render_queue.empty() && s->live.size() < s->cfg.capacity && !s->stopping) {
        if (!s->live.empty() && std::chrono::duration<double>(Clock::now() - start).count() > kAdmitSeconds) return;
        const uint64_t id = s->render_queue.front();
        Request &r = s->requests[id];
        try {
            SceneSlot &slot = s->scenes[r.scene];
            const uint64_t scene_bytes = slot.gs ? slot.bytes : upload_estimate(slot.scene);
            if (scene_bytes + r.bytes > available(s))
                fail(LR_LIMIT, "the session and its scene do not fit the server's memory budget");
            if (!ensure_resident(s, lk, r.scene, s->load_ctx)) return;  // waits for memory
            slot.users++;  // held while room is made, so it is not the scene evicted
            if (!make_room(s, r.bytes)) {
                slot.users--;
                return;  // waits for memory
            }
            s->bytes_in_use += r.bytes;
            uint32_t member = 0;
            lk.unlock();
            const int status = lr_batch_add(s->batch, slot.gs, slot.scene, &r.settings, r.framed ? &r.frame : nullptr,
                                            &member);
            const std::string message = status == LR_OK ? "" : lr_last_error();
            lk.lock();
            if (status != LR_OK) {
                slot.users--;
                s->bytes_in_use -= r.bytes;
                fail(status, message);
            }
            r.member = member;
            r.state = LR_REQUEST_RUNNING;
            r.admitted = seconds_since(s->t0);
            slot.last_use = ++s->tick;
            s->live.push_back(id);
        } catch (const lr::Error &e) {
            finish_request(s, r, e.code, e.what());
        }
        s->render_queue.pop_front();
    }
}

// A pinned buffer of at least `bytes` for a finished image, or null when the staging
// limit is reached. Lock held (released while a buffer is allocated).
float *take_staging(lr_server *s, std::unique_lock<std::mutex> &lk, uint64_t bytes, uint64_t &size) {
    size = staging_size(bytes);
    for (size_t i = 0; i < s->staging_free.size(); i++)
        if (s->staging_free[i].first == size) {
            float *buffer = s->staging_free[i].second;
            s->staging_free.erase(s->staging_free.begin() + (long)i);
            return buffer;
        }
    if (s->staging_total + size > kStagingLimit) return nullptr;
    s->staging_total += size;
    lk.unlock();
    void *buffer = nullptr;
    const cudaError_t e = cudaHostAlloc(&buffer, size, cudaHostAllocDefault);
    lk.lock();
    if (e != cudaSuccess) {
        cudaGetLastError();
        s->staging_total -= size;
        return nullptr;
    }
    return (float *)buffer;
}

// Copies a finished session's image out: a ticketed read into a pinned buffer, landed
// on a later call; or, with no buffer to spare, a read that waits. True once the image
// is in the caller's memory (or failed: `status`). Lock held (released around copies).
bool image_out(lr_server *s, std::unique_lock<std::mutex> &lk, Request &r, int &status, std::string &message) {
    const uint64_t bytes = r.pixels * 16;
    if (!r.staging) {
        uint64_t size = 0;
        float *buffer = take_staging(s, lk, bytes, size);
        if (!buffer) {
            lk.unlock();
            if (lr_batch_read(s->batch, r.member, r.rgba, r.pixels * 4) != LR_OK) {
                status = LR_DEVICE;
                message = lr_last_error();
            }
            lk.lock();
            return true;
        }
        r.staging = buffer;
        r.staging_bytes = size;
        lk.unlock();
        const int e = lr_batch_read_ticket(s->batch, r.member, buffer, r.pixels * 4, &r.ticket);
        const std::string why = e == LR_OK ? "" : lr_last_error();
        lk.lock();
        if (e != LR_OK) {
            status = LR_DEVICE;
            message = why;
        } else {
            return false;  // lands on a later call
        }
    } else {
        int32_t landed = 0;
        if (lr_batch_read_landed(s->batch, r.ticket, &landed) != LR_OK) {
            status = LR_DEVICE;
            message = lr_last_error();
        } else if (!landed) {
            return false;
        } else {
            lk.unlock();
            std::memcpy(r.rgba, r.staging, bytes);
            lk.lock();
        }
    }
    s->staging_free.push_back({r.staging_bytes, r.staging});
    r.staging = nullptr;
    return true;
}

// Notes each live session's progress after a pass retired; retires finished ones. Lock
// held (released while a finished image is copied out).
void progress(lr_server *s, std::unique_lock<std::mutex> &lk) {
    const double now = seconds_since(s->t0);
    for (size_t i = 0; i < s->live.size();) {
        Request &r = s->requests[s->live[i]];
        uint32_t done = 0;
        lr_batch_member_info(s->batch, r.member, &done, nullptr, nullptr);
        if (done > r.samples_done) {
            s->stats.pixel_samples += (uint64_t)(done - r.samples_done) * r.pixels;
            r.samples_done = done;
            if (r.first < 0) r.first = now;
        }
        if (done >= r.samples) {
            int status = LR_OK;
            std::string message;
            if (r.rgba && !image_out(s, lk, r, status, message)) {
                i++;  // its image is on its way
                continue;
            }
            lr_batch_remove(s->batch, r.member);
            SceneSlot &slot = s->scenes[r.scene];
            slot.users--;
            slot.last_use = ++s->tick;
            s->bytes_in_use -= r.bytes;
            s->stats.sessions_done++;
            finish_request(s, r, status, message);
            s->live.erase(s->live.begin() + (long)i);
        } else {
            i++;
        }
    }
}

void render_loop(lr_server *s) {
    std::unique_lock<std::mutex> lk(s->mu);
    auto since = [](Clock::time_point t) { return std::chrono::duration<double>(Clock::now() - t).count(); };
    for (;;) {
        if (s->stopping) break;
        Clock::time_point t = Clock::now();
        admit(s, lk);
        s->stats.seconds_admit += since(t);
        if (s->live.empty()) {
            if (s->render_queue.empty())
                s->cv_work.wait(lk, [&] { return s->stopping || !s->render_queue.empty(); });
            else  // the head of the queue waits for memory that probes hold
                s->cv_done.wait_for(lk, std::chrono::milliseconds(20));
            continue;
        }
        const double now = seconds_since(s->t0);
        const bool retune = s->live.size() >= std::min<size_t>(kTuneSessions, s->cfg.capacity) &&
                            (s->tuned_at < 0.0 || now - s->tuned_at > kRetune);
        lk.unlock();
        if (retune) {
            // Dry passes on the live sessions (films untouched): the BVH width, stack and
            // block size per scene-size class, the pass fill, the ray sort interval and
            // the traversal warps' refill.
            t = Clock::now();
            const bool tuned = lr_batch_tune(s->batch, nullptr) == LR_OK;
            std::lock_guard<std::mutex> note(s->mu);
            if (tuned) s->tunings++;
            s->tuned_at = seconds_since(s->t0);
            s->stats.seconds_tune += since(t);
        }
        // Two passes in flight (a pass queues only while fewer run), then the oldest
        // retires: one pass always runs while this thread admits and retires sessions,
        // and the two lanes overlap one pass's thin last rounds with the next one's first.
        int32_t more = 0, in_flight = 0;
        t = Clock::now();
        int status = lr_batch_advance(s->batch, &more);
        if (status == LR_OK) status = lr_batch_advance(s->batch, &more);
        const double advancing = since(t);
        t = Clock::now();
        if (status == LR_OK) status = lr_batch_wait(s->batch, &in_flight);
        const double waiting = since(t);
        std::string message = status == LR_OK ? "" : lr_last_error();
        lk.lock();
        s->stats.seconds_advance += advancing;
        s->stats.seconds_wait += waiting;
        s->stats.passes++;
        if (status != LR_OK) {
            // A device failure ends every live session with its status.
            for (uint64_t id : s->live) {
                Request &r = s->requests[id];
                if (r.staging) {
                    s->staging_free.push_back({r.staging_bytes, r.staging});
                    r.staging = nullptr;
                }
                finish_request(s, r, status, message);
            }
            s->live.clear();
            continue;
        }
        t = Clock::now();
        progress(s, lk);
        s->stats.seconds_progress += since(t);
    }
}

void probe_loop(lr_server *s) {
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_work.wait(lk, [&] { return s->stopping || !s->probe_queue.empty(); });
        if (s->stopping) break;
        const uint64_t id = s->probe_queue.front();
        s->probe_queue.pop_front();
        Request &r = s->requests[id];
        SceneSlot &slot = s->scenes[r.scene];
        bool failed = false;
        try {
            // Wait for room while sessions and uploads hold the memory.
            while (!ensure_resident(s, lk, r.scene, s->probe_ctx)) {
                if (s->stopping) fail(LR_STOPPED, "the server stopped");
                s->cv_done.wait_for(lk, std::chrono::milliseconds(20));
            }
        } catch (const lr::Error &e) {
            finish_request(s, r, e.code, e.what());
            failed = true;
        }
        if (failed) continue;
        slot.users++;
        slot.last_use = ++s->tick;
        r.state = LR_REQUEST_RUNNING;
        r.admitted = seconds_since(s->t0);
        lr_gpu_scene *gs = slot.gs;
        lk.unlock();
        const int status = r.pixels <= LR_PROBE_STATIC_PIXELS
                               ? lr_probe_static(s->probe_ctx, gs, &r.frame, r.flags, r.faces, r.distances)
                               : lr_probe(s->probe_ctx, gs, &r.frame, r.flags, r.faces, r.distances);
        std::string message = status == LR_OK ? "" : lr_last_error();
        lk.lock();
        slot.users--;
        slot.last_use = ++s->tick;
        s->stats.probes_done++;
        s->stats.probe_rays += r.pixels;
        finish_request(s, r, status, message);
    }
}

uint64_t submit(lr_server *s, Request &&r, bool probe) {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) fail(LR_STOPPED, "the server is stopping");
    if (r.scene >= s->scenes.size()) fail(LR_INVALID, "no such scene");
    if (!probe) r.bytes = session_bytes(r, s->scenes[r.scene].image_bytes);
    r.submitted = seconds_since(s->t0);
    const uint64_t id = s->requests.size();
    s->requests.push_back(std::move(r));
    (probe ? s->probe_queue : s->render_queue).push_back(id);
    s->cv_work.notify_all();
    return id;
}

void stop(lr_server *s) {
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->cv_work.notify_all();
        s->cv_loaded.notify_all();
    }
    if (s->render_thread.joinable()) s->render_thread.join();
    if (s->probe_thread.joinable()) s->probe_thread.join();
}

}  // namespace

extern "C" {

void lr_server_settings_default(lr_server_settings *out) {
    if (!out) return;
    *out = lr_server_settings{};
    out->device = 0;
    out->budget_bytes = 150ull * 1000 * 1000 * 1000;
    out->capacity = 128;
    out->pool = 1u << 22;
    out->max_bounces = 12;
    out->probe_priority = 1;
}

int lr_server_create(const lr_server_settings *settings, lr_server **out) {
    return lr::guarded([&] {
        if (!settings || !out) fail(LR_INVALID, "a server needs settings");
        *out = nullptr;
        if (settings->capacity == 0 || settings->capacity > 512) fail(LR_INVALID, "a server runs 1 to 512 sessions at once");
        auto s = std::make_unique<lr_server>();
        s->cfg = *settings;
        s->t0 = Clock::now();
        try {
            check(lr_context_create(settings->device, &s->ctx));
            check(lr_context_create_ex(settings->device, settings->probe_priority ? 1 : 0, &s->probe_ctx));
            check(lr_context_create(settings->device, &s->load_ctx));
            lr_batch_settings bs;
            lr_batch_settings_default(&bs);
            bs.pool = settings->pool;
            bs.max_bounces = settings->max_bounces;
            // Room beyond the live sessions: a session that finished keeps its member's
            // slot until the passes in flight retire, and a new session admitted
            // meanwhile must not wait for them.
            bs.capacity = settings->capacity * 2 + 16;
            check(lr_batch_create(s->ctx, &bs, &s->batch));
            // The wave's own memory: 15 float4 arrays of pool entries, and small parts; and
            // the static probe array (lr_probe_static), which the device holds from the
            // module's load on. Its set-up runs here, before the threads start, so a first
            // probe does not load the module after the scenes have filled the budget.
            lr::probe_static_setup(settings->device);
            s->wave_bytes = (uint64_t)std::min<uint32_t>(settings->pool, 1u << 23) * 16 * 15 + (1u << 20) +
                            (uint64_t)LR_PROBE_STATIC_PIXELS * 8;
            if (s->wave_bytes >= settings->budget_bytes) fail(LR_LIMIT, "the pool alone exceeds the memory budget");
        } catch (...) {
            if (s->batch) lr_batch_destroy(s->batch);
            if (s->load_ctx) lr_context_destroy(s->load_ctx);
            if (s->probe_ctx) lr_context_destroy(s->probe_ctx);
            if (s->ctx) lr_context_destroy(s->ctx);
            throw;
        }
        lr_server *raw = s.get();
        raw->render_thread = std::thread(render_loop, raw);
        raw->probe_thread = std::thread(probe_loop, raw);
        *out = s.release();
    });
}

int lr_server_add_scene(lr_server *s, const lr_scene *scene, uint32_t *scene_id) {
    return lr::guarded([&] {
        if (!s || !scene || !scene_id) fail(LR_INVALID, "a scene to serve");
        std::lock_guard<std::mutex> lk(s->mu);
        SceneSlot slot;
        slot.scene = scene;
        slot.image_bytes = dome_image_bytes(scene);
        s->scenes.push_back(slot);
        *scene_id = (uint32_t)(s->scenes.size() - 1);
    });
}

int lr_server_preload(lr_server *s, uint32_t scene_id) {
    return lr::guarded([&] {
        if (!s) fail(LR_INVALID, "no server");
        std::unique_lock<std::mutex> lk(s->mu);
        if (scene_id >= s->scenes.size()) fail(LR_INVALID, "no such scene");
        if (!ensure_resident(s, lk, scene_id, s->load_ctx)) fail(LR_LIMIT, "the scene does not fit the budget now");
        s->scenes[scene_id].last_use = ++s->tick;
    });
}

int lr_server_submit_render(lr_server *s, uint32_t scene_id, const lr_settings *settings, const lr_frame *frame,
                            float *rgba, uint64_t *request) {
    return lr::guarded([&] {
        if (!s || !settings || !request) fail(LR_INVALID, "a render request needs settings");
        Request r;
        r.kind = LR_REQUEST_RENDER;
        r.scene = scene_id;
        r.settings = *settings;
        if (frame) {
            r.frame = *frame;
            r.framed = true;
        }
        const uint64_t w = frame ? frame->width : settings->width, h = frame ? frame->height : settings->height;
        if (w == 0 || h == 0) fail(LR_INVALID, "an image needs pixels");
        if (settings->samples == 0) fail(LR_INVALID, "a render needs samples");
        r.pixels = w * h;
        r.samples = settings->samples;
        r.rgba = rgba;
        *request = submit(s, std::move(r), false);
    });
}

int lr_server_submit_probe(lr_server *s, uint32_t scene_id, const lr_frame *frame, uint32_t flags, uint32_t *faces,
                           float *distances, uint64_t *request) {
    return lr::guarded([&] {
        if (!s || !frame || !faces || !distances || !request) fail(LR_INVALID, "a probe needs one result per pixel");
        if (frame->width == 0 || frame->height == 0) fail(LR_INVALID, "an image needs pixels");
        Request r;
        r.kind = LR_REQUEST_PROBE;
        r.scene = scene_id;
        r.frame = *frame;
        r.framed = true;
        r.flags = flags;
        r.faces = faces;
        r.distances = distances;
        r.pixels = (uint64_t)frame->width * frame->height;
        *request = submit(s, std::move(r), true);
    });
}

int lr_server_request_info(lr_server *s, uint64_t request, lr_request_info *out) {
    return lr::guarded([&] {
        if (!s || !out) fail(LR_INVALID, "no server");
        std::lock_guard<std::mutex> lk(s->mu);
        if (request >= s->requests.size()) fail(LR_INVALID, "no such request");
        const Request &r = s->requests[request];
        out->kind = r.kind;
        out->state = r.state;
        out->status = r.status;
        out->scene = r.scene;
        out->pixels = r.pixels;
        out->samples = r.samples;
        out->samples_done = r.samples_done;
        out->submitted = r.submitted;
        out->admitted = r.admitted;
        out->first = r.first;
        out->finished = r.finished;
    });
}

int lr_server_wait(lr_server *s, uint64_t request, double timeout_seconds) {
    return lr::guarded([&] {
        if (!s) fail(LR_INVALID, "no server");
        std::unique_lock<std::mutex> lk(s->mu);
        if (request >= s->requests.size()) fail(LR_INVALID, "no such request");
        auto finished = [&] {
            const int st = s->requests[request].state;
            return st == LR_REQUEST_DONE || st == LR_REQUEST_FAILED;
        };
        if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_seconds), finished))
            fail(LR_TIMEOUT, "the request has not finished");
        const Request &r = s->requests[request];
        if (r.state == LR_REQUEST_FAILED) fail(r.status, r.message);
    });
}

int lr_server_stats_get(lr_server *s, lr_server_stats *out) {
    return lr::guarded([&] {
        if (!s || !out) fail(LR_INVALID, "no server");
        std::lock_guard<std::mutex> lk(s->mu);
        *out = s->stats;
        out->queued = s->render_queue.size() + s->probe_queue.size();
        out->live = s->live.size();
        out->bytes_in_use = s->bytes_in_use + s->wave_bytes;
        out->scenes_resident = (uint64_t)std::count_if(s->scenes.begin(), s->scenes.end(),
                                                       [](const SceneSlot &x) { return x.gs != nullptr; });
        out->seconds = seconds_since(s->t0);
        out->tunings = s->tunings;
    });
}

void lr_server_destroy(lr_server *s) {
    if (!s) return;
    stop(s);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (auto &r : s->requests)
            if (r.state == LR_REQUEST_QUEUED || r.state == LR_REQUEST_RUNNING) {
                r.state = LR_REQUEST_FAILED;
                r.status = LR_STOPPED;
                r.message = "the server stopped";
            }
        s->cv_done.notify_all();
    }
    if (s->batch) lr_batch_destroy(s->batch);  // waits for its copies
    for (auto &r : s->requests)
        if (r.staging) s->staging_free.push_back({r.staging_bytes, r.staging});
    for (auto &b : s->staging_free) cudaFreeHost(b.second);
    for (auto &slot : s->scenes)
        if (slot.gs) lr_gpu_scene_destroy(slot.gs);
    if (s->load_ctx) lr_context_destroy(s->load_ctx);
    if (s->probe_ctx) lr_context_destroy(s->probe_ctx);
    if (s->ctx) lr_context_destroy(s->ctx);
    delete s;
}

}  // extern "C"
