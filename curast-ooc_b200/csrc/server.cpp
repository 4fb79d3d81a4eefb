// server.cpp -- serving with continuous batching (cr_server_*).
//
// No counterpart in the reference, which renders one interactive view.  Two
// threads own the context while a server exists:
//   dispatcher  admits requests in arrival order as their framebuffers fit in
//               the memory budget (a first-fit arena over one device
//               allocation), and whenever one of the slots (a stream plus the
//               queues, records and tables of one batched frame) is free,
//               issues the admitted requests of the scene of the oldest one as
//               one batched frame (scratch_issue: the kernels of
//               cr_render_batch).  A host function enqueued after the frame
//               stamps its completion time on the device timeline and wakes
//               the dispatcher, which checks the frame's counters (re-issuing
//               it with larger queues after an overflow) and publishes the
//               results.  Batches of several slots overlap on the device.
//   ooc lane    renders requests of out-of-core scenes one at a time with
//               cr_ooc_render on its own stream, beside the batches.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "context.h"

using namespace cr;

namespace {

double now_us() {
    return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// First-fit allocator over [0, size) in 256-byte granules, coalescing frees.
class Arena {
public:
    void init(uint64_t bytes) {
        free_.clear();
        if (bytes) free_[0] = bytes;
    }
    bool alloc(uint64_t size, uint64_t& off) {
        size = (size + 255) & ~255ull;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < size) continue;
            off = it->first;
            const uint64_t rest = it->second - size;
            free_.erase(it);
            if (rest) free_[off + size] = rest;
            return true;
        }
        return false;
    }
    void release(uint64_t off, uint64_t size) {
        size = (size + 255) & ~255ull;
        auto it = free_.emplace(off, size).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }

private:
    std::map<uint64_t, uint64_t> free_;
};

enum class State { Pending, Admitted, Running, Done, Polled };

struct Req {
    uint64_t ticket = 0;
    uint32_t scene = 0;
    cr_camera cam{};
    State state = State::Pending;
    uint64_t off = 0, bytes = 0, visBytes = 0;
    int32_t status = CR_OK;
    double tSubmit = 0, tStart = 0, tDone = 0;
    uint32_t batchViews = 0;
};

struct Scene {
    bool ooc = false;
    std::vector<cr_instance> instances;
    cr_ooc* handle = nullptr;
    // largest queue demand per pixel seen in this scene's frames: sizes the
    // queues of its next batches so that they rarely overflow
    double ntPerPixel = 0.0, tilesPerPixel = 0.0;
};

struct Slot {
    cr_server* server = nullptr;
    cudaStream_t stream = nullptr;
    BatchScratch S;
    bool busy = false;
    std::vector<uint64_t> tickets;
    std::vector<cr_view> views;
    uint32_t scene = 0;
    double tStart = 0;
    uint64_t pixels = 0;
    int attempts = 0;
    std::atomic<bool> done{false};
    std::atomic<double> tDone{0.0};
};

uint64_t fb_bytes(const cr_camera& c, uint64_t* visBytes) {
    const uint64_t P = (uint64_t)c.width * (uint64_t)c.height;
    *visBytes = (8 * P + 255) & ~255ull;
    return *visBytes + ((4 * P + 255) & ~255ull);
}

}  // namespace

struct cr_server {
    cr_context* ctx = nullptr;
    cr_server_config cfg{};
    char* fbBase = nullptr;
    uint64_t fbCap = 0;
    Arena arena;
    uint64_t fbUsed = 0, peak = 0;
    std::vector<Scene> scenes;
    std::vector<std::unique_ptr<Slot>> slots;
    cudaStream_t oocStream = nullptr;
    std::mutex mu;
    std::condition_variable wake;      // dispatcher
    std::condition_variable wakeOoc;   // ooc lane
    std::condition_variable doneCv;    // waiters
    std::unordered_map<uint64_t, Req> reqs;
    std::deque<uint64_t> pending, admitted, oocQueue, completed;
    uint64_t nextTicket = 1;
    uint64_t running = 0;
    bool stop = false;
    std::thread dispatcher, oocLane;
    // statistics
    uint64_t nSubmitted = 0, nCompleted = 0, nBatches = 0, nBatchedViews = 0;
    std::vector<double> latencies;  // ms
    double firstSubmit = 0, lastDone = 0;
};

namespace {

void CUDART_CB on_slot_done(void* p) {  // CUDA host-function thread: no CUDA calls
    Slot* s = static_cast<Slot*>(p);
    s->tDone.store(now_us());
    s->done.store(true);
    std::lock_guard<std::mutex> lk(s->server->mu);
    s->server->wake.notify_one();
}

void publish(cr_server* sv, Req& r, int32_t status, double tDone) {
    r.status = status;
    r.tDone = tDone;
    r.state = State::Done;
    sv->completed.push_back(r.ticket);
    sv->nCompleted++;
    sv->latencies.push_back((tDone - r.tSubmit) / 1000.0);
    sv->lastDone = std::max(sv->lastDone, tDone);
}

// Runs with sv->mu held.  Admits pending requests in arrival order.
void admit(cr_server* sv) {
    while (!sv->pending.empty()) {
        Req& r = sv->reqs[sv->pending.front()];
        uint64_t off = 0;
        if (!sv->arena.alloc(r.bytes, off)) break;  // wait for releases
        r.off = off;
        r.state = State::Admitted;
        sv->fbUsed += (r.bytes + 255) & ~255ull;
        sv->pending.pop_front();
        if (sv->scenes[r.scene].ooc) {
            sv->oocQueue.push_back(r.ticket);
            sv->wakeOoc.notify_one();
        } else {
            sv->admitted.push_back(r.ticket);
        }
    }
    uint64_t scratch = 0;
    for (auto& s : sv->slots) scratch += scratch_bytes(s->S);
    sv->peak = std::max(sv->peak, sv->fbUsed + scratch);
}

// Queue capacities for a batch of `pixels` pixels of a scene: its demand
// per pixel so far with 50 % headroom (at least 1M entries each).
void size_queues(cr_server* sv, Slot& s, const Scene& sc, cr_status* st) {
    const uint64_t nt = std::max<uint64_t>(1ull << 20, (uint64_t)(sc.ntPerPixel * 1.5 * (double)s.pixels) + 65536);
    const uint64_t hu = std::max<uint64_t>(1ull << 20, (uint64_t)(sc.tilesPerPixel * 1.5 * (double)s.pixels) + 65536);
    *st = scratch_grow_queues(sv->ctx, s.S, nt, hu);
}

cr_status issue(cr_server* sv, Slot& s) {
    const Scene& sc = sv->scenes[s.scene];
    cr_status st = scratch_issue(sv->ctx, s.S, sc.instances.data(), (uint32_t)sc.instances.size(), s.views.data(),
                                 (uint32_t)s.views.size(), sv->cfg.display, 0, s.stream);
    if (!st && cudaLaunchHostFunc(s.stream, on_slot_done, &s) != cudaSuccess) st = CR_ERR_CUDA;
    return st;
}

// The frame of a slot finished: check its counters, publish its requests --
// or, after a queue overflow, issue the batch again with queues grown to the
// measured demand (the counters hold the exact demand of every queue fed in
// full), leaving the slot busy.  Called with sv->mu held.
void finish(cr_server* sv, Slot& s, std::unique_lock<std::mutex>& lk) {
    int32_t status = CR_OK;
    const unsigned long long* c = s.S.hCounters;
    Scene& sc = sv->scenes[s.scene];
    if (s.pixels) {
        sc.ntPerPixel = std::max(sc.ntPerPixel, (double)c[CR_CTR_NONTRIVIAL] / (double)s.pixels);
        sc.tilesPerPixel = std::max(sc.tilesPerPixel, (double)c[CR_CTR_HUGE] / (double)s.pixels);
    }
    if (c[CR_CTR_TIMEOUT]) {
        status = CR_ERR_TIMEOUT;
    } else if (c[CR_CTR_OVERFLOW]) {
        if (s.attempts < 3) {
            s.attempts++;
            const uint64_t nt = std::max<uint64_t>(s.S.ntCap, c[CR_CTR_NONTRIVIAL] + c[CR_CTR_NONTRIVIAL] / 4 + 4096);
            const uint64_t hu = (c[CR_CTR_OVERFLOW] & 1) ? std::max<uint64_t>(s.S.hugeCap, 2 * s.S.hugeCap)
                                                         : std::max<uint64_t>(s.S.hugeCap, c[CR_CTR_HUGE] + c[CR_CTR_HUGE] / 4 + 4096);
            s.done.store(false);
            lk.unlock();
            cr_status st = scratch_grow_queues(sv->ctx, s.S, nt, hu);
            if (!st) st = issue(sv, s);
            lk.lock();
            if (!st) return;  // the slot stays busy with the same batch
            status = st;
        } else {
            status = CR_ERR_QUEUE_OVERFLOW;
        }
    }
    const double tDone = s.tDone.load();
    for (uint64_t t : s.tickets) publish(sv, sv->reqs[t], status, tDone);
    sv->running -= s.tickets.size();
    s.tickets.clear();
    s.busy = false;
    s.done.store(false);
    sv->doneCv.notify_all();
}

// Issues a batch on a free slot.  Called with sv->mu held; unlocks around the
// CUDA calls.
void launch(cr_server* sv, Slot& s, std::unique_lock<std::mutex>& lk) {
    const uint32_t scene = sv->reqs[sv->admitted.front()].scene;
    s.tickets.clear();
    s.views.clear();
    const uint32_t maxViews = std::min<uint32_t>(sv->cfg.max_batch_views, CR_MAX_BATCH_VIEWS);
    for (auto it = sv->admitted.begin(); it != sv->admitted.end() && s.tickets.size() < maxViews;) {
        Req& r = sv->reqs[*it];
        if (r.scene != scene) {
            ++it;
            continue;
        }
        s.tickets.push_back(r.ticket);
        cr_view v{};
        v.camera = r.cam;
        v.d_visbuffer = (uint64_t)(uintptr_t)(sv->fbBase + r.off);
        v.d_rgba = v.d_visbuffer + r.visBytes;
        s.views.push_back(v);
        it = sv->admitted.erase(it);
    }
    const double t0 = now_us();
    s.pixels = 0;
    for (uint64_t t : s.tickets) {
        Req& r = sv->reqs[t];
        r.state = State::Running;
        r.tStart = t0;
        r.batchViews = (uint32_t)s.tickets.size();
        s.pixels += (uint64_t)r.cam.width * (uint64_t)r.cam.height;
    }
    s.busy = true;
    s.scene = scene;
    s.attempts = 0;
    s.done.store(false);
    sv->running += s.tickets.size();
    sv->nBatches++;
    sv->nBatchedViews += s.tickets.size();
    lk.unlock();
    cr_status st = CR_OK;
    size_queues(sv, s, sv->scenes[scene], &st);
    if (!st) st = issue(sv, s);
    lk.lock();
    if (st) {  // nothing will complete: publish the error now
        for (uint64_t t : s.tickets) publish(sv, sv->reqs[t], st, now_us());
        sv->running -= s.tickets.size();
        s.tickets.clear();
        s.busy = false;
        sv->doneCv.notify_all();
    }
}

void dispatcher_main(cr_server* sv) {
    cudaSetDevice(sv->ctx->device);
    std::unique_lock<std::mutex> lk(sv->mu);
    while (true) {
        for (auto& s : sv->slots)
            if (s->busy && s->done.load()) finish(sv, *s, lk);
        admit(sv);
        for (auto& s : sv->slots)
            if (!s->busy && !sv->admitted.empty()) launch(sv, *s, lk);
        const bool quiet = sv->admitted.empty() && sv->oocQueue.empty() && sv->running == 0;
        if (sv->stop && quiet && !sv->pending.empty()) {
            // stopping with requests that can never be admitted (results were
            // never released): fail them
            for (uint64_t t : sv->pending) publish(sv, sv->reqs[t], CR_ERR_BUSY, now_us());
            sv->pending.clear();
            sv->doneCv.notify_all();
        }
        if (sv->stop && quiet && sv->pending.empty()) break;
        bool anyDone = false;
        for (auto& s : sv->slots) anyDone |= s->busy && s->done.load();
        if (!anyDone) sv->wake.wait_for(lk, std::chrono::milliseconds(2));
    }
    sv->wakeOoc.notify_all();
}

void ooc_main(cr_server* sv) {
    cudaSetDevice(sv->ctx->device);
    std::unique_lock<std::mutex> lk(sv->mu);
    while (true) {
        sv->wakeOoc.wait(lk, [&] { return !sv->oocQueue.empty() || (sv->stop && sv->pending.empty()); });
        if (sv->oocQueue.empty()) {
            if (sv->stop && sv->pending.empty()) break;
            continue;
        }
        const uint64_t t = sv->oocQueue.front();
        sv->oocQueue.pop_front();
        Req& r = sv->reqs[t];
        r.state = State::Running;
        r.tStart = now_us();
        r.batchViews = 1;
        sv->running++;
        const cr_camera cam = r.cam;
        const uint64_t vis = (uint64_t)(uintptr_t)(sv->fbBase + r.off);
        const uint64_t rgba = vis + r.visBytes;
        cr_ooc* o = sv->scenes[r.scene].handle;
        lk.unlock();
        const cr_status st = cr_ooc_render(o, &cam, vis, rgba, sv->cfg.display, CR_RENDER_SYNC, sv->oocStream, nullptr);
        const double tDone = now_us();
        lk.lock();
        sv->running--;
        publish(sv, sv->reqs[t], st, tDone);
        sv->doneCv.notify_all();
        sv->wake.notify_one();
    }
}

void fill_result(const cr_server* sv, const Req& r, cr_server_result* out) {
    memset(out, 0, sizeof(*out));
    out->ticket = r.ticket;
    out->status = r.status;
    out->scene = r.scene;
    out->width = r.cam.width;
    out->height = r.cam.height;
    out->d_visbuffer = (uint64_t)(uintptr_t)(sv->fbBase + r.off);
    out->d_rgba = out->d_visbuffer + r.visBytes;
    out->submit_us = r.tSubmit;
    out->start_us = r.tStart;
    out->done_us = r.tDone;
    out->batch_views = r.batchViews;
}

}  // namespace

extern "C" {

cr_status cr_server_create(cr_context* ctx, const cr_server_config* cfg, cr_server** out) {
    if (!ctx || !out) return fail(CR_ERR_INVALID, "cr_server_create: NULL argument");
    *out = nullptr;
    cr_server_config c{};
    if (cfg) c = *cfg;
    if (!c.memory_budget) c.memory_budget = 64ull << 30;
    if (!c.slots) c.slots = 3;
    if (!c.max_batch_views || c.max_batch_views > CR_MAX_BATCH_VIEWS) c.max_batch_views = CR_MAX_BATCH_VIEWS;
    CR_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cr_server* sv = new cr_server();
    sv->ctx = ctx;
    sv->cfg = c;
    for (uint32_t k = 0; k < c.slots; k++) {
        auto s = std::make_unique<Slot>();
        s->server = sv;
        if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            cr_server_destroy(sv);
            return fail(CR_ERR_CUDA, "server stream");
        }
        sv->slots.push_back(std::move(s));
    }
    if (cudaStreamCreateWithFlags(&sv->oocStream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        cr_server_destroy(sv);
        return fail(CR_ERR_CUDA, "server stream");
    }
    sv->dispatcher = std::thread(dispatcher_main, sv);
    sv->oocLane = std::thread(ooc_main, sv);
    *out = sv;
    return CR_OK;
}

cr_status cr_server_add_scene(cr_server* sv, const cr_instance* instances, uint32_t count, uint32_t* scene_out) {
    if (!sv || !scene_out || (!instances && count)) return fail(CR_ERR_INVALID, "cr_server_add_scene: NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->fbBase) return fail(CR_ERR_INVALID, "scenes are added before the first request");
    for (uint32_t i = 0; i < count; i++)
        if (instances[i].mesh >= sv->ctx->meshes.size() || !sv->ctx->meshes[instances[i].mesh].live)
            return fail(CR_ERR_NOT_FOUND, "instance %u: unknown mesh %u", i, instances[i].mesh);
    Scene s;
    s.instances.assign(instances, instances + count);
    sv->scenes.push_back(std::move(s));
    *scene_out = (uint32_t)(sv->scenes.size() - 1);
    return CR_OK;
}

cr_status cr_server_add_ooc_scene(cr_server* sv, cr_ooc* ooc, uint32_t* scene_out) {
    if (!sv || !ooc || !scene_out) return fail(CR_ERR_INVALID, "cr_server_add_ooc_scene: NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->fbBase) return fail(CR_ERR_INVALID, "scenes are added before the first request");
    Scene s;
    s.ooc = true;
    s.handle = ooc;
    sv->scenes.push_back(std::move(s));
    *scene_out = (uint32_t)(sv->scenes.size() - 1);
    return CR_OK;
}

cr_status cr_server_submit(cr_server* sv, const cr_server_request* req, uint64_t* ticket) {
    if (!sv || !req || !ticket) return fail(CR_ERR_INVALID, "cr_server_submit: NULL argument");
    const cr_camera& c = req->camera;
    if (c.width <= 0 || c.height <= 0 || (uint64_t)c.width * c.height >= (1ull << 31))
        return fail(CR_ERR_INVALID, "bad resolution %dx%d", c.width, c.height);
    std::lock_guard<std::mutex> lk(sv->mu);
    if (req->scene >= sv->scenes.size()) return fail(CR_ERR_INVALID, "unknown scene %u", req->scene);
    if (!sv->fbBase) {
        // the framebuffer arena takes what the slots' largest batches leave:
        // per slot the view-mask records of the largest scene and 2 x 1M
        // queue entries
        uint64_t maxV = 0;
        for (const Scene& s : sv->scenes) {
            uint64_t v = 0;
            for (const cr_instance& i : s.instances) v += align_up(sv->ctx->meshes[i.mesh].numVertices, 16);
            maxV = std::max(maxV, v);
        }
        const uint64_t perSlot = maxV * sizeof(CrViewMasks) + (2ull << 20) * 24 + (4ull << 20);
        const uint64_t reserve = perSlot * sv->slots.size();
        if (reserve >= sv->cfg.memory_budget) return fail(CR_ERR_OOM, "memory budget below the slots' scratch");
        sv->fbCap = (sv->cfg.memory_budget - reserve) & ~255ull;
        cr_status s = sv->ctx->dev_alloc((void**)&sv->fbBase, sv->fbCap, "server framebuffers");
        if (s) return s;
        sv->arena.init(sv->fbCap);
        for (auto& sl : sv->slots) {
            s = scratch_grow_queues(sv->ctx, sl->S, 1ull << 20, 1ull << 20);
            if (s) return s;
        }
    }
    Req r;
    r.ticket = sv->nextTicket++;
    r.scene = req->scene;
    r.cam = c;
    r.bytes = fb_bytes(c, &r.visBytes);
    if (r.bytes > sv->fbCap) return fail(CR_ERR_INVALID, "request needs %llu bytes, the budget holds %llu",
                                         (unsigned long long)r.bytes, (unsigned long long)sv->fbCap);
    r.tSubmit = now_us();
    if (!sv->nSubmitted) sv->firstSubmit = r.tSubmit;
    sv->nSubmitted++;
    sv->reqs[r.ticket] = r;
    sv->pending.push_back(r.ticket);
    *ticket = r.ticket;
    sv->wake.notify_one();
    return CR_OK;
}

cr_status cr_server_poll(cr_server* sv, cr_server_result* results, uint32_t max, uint32_t* count) {
    if (!sv || !count || (!results && max)) return fail(CR_ERR_INVALID, "cr_server_poll: NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    uint32_t n = 0;
    while (n < max && !sv->completed.empty()) {
        Req& r = sv->reqs[sv->completed.front()];
        sv->completed.pop_front();
        if (r.state != State::Done) continue;  // returned by cr_server_wait already
        r.state = State::Polled;
        fill_result(sv, r, &results[n++]);
    }
    *count = n;
    return CR_OK;
}

cr_status cr_server_wait(cr_server* sv, uint64_t ticket, uint32_t timeout_ms, cr_server_result* result) {
    if (!sv || !result) return fail(CR_ERR_INVALID, "cr_server_wait: NULL argument");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return fail(CR_ERR_NOT_FOUND, "unknown ticket %llu", (unsigned long long)ticket);
    const bool ok = sv->doneCv.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] {
        const State s = sv->reqs[ticket].state;
        return s == State::Done || s == State::Polled;
    });
    if (!ok) return fail(CR_ERR_TIMEOUT, "request %llu not done after %u ms", (unsigned long long)ticket, timeout_ms);
    Req& r = sv->reqs[ticket];
    r.state = State::Polled;
    fill_result(sv, r, result);
    return CR_OK;
}

cr_status cr_server_release(cr_server* sv, uint64_t ticket) {
    if (!sv) return fail(CR_ERR_INVALID, "cr_server_release: NULL server");
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(ticket);
    if (it == sv->reqs.end()) return fail(CR_ERR_NOT_FOUND, "unknown ticket %llu", (unsigned long long)ticket);
    if (it->second.state != State::Done && it->second.state != State::Polled)
        return fail(CR_ERR_INVALID, "request %llu is not done", (unsigned long long)ticket);
    sv->arena.release(it->second.off, it->second.bytes);
    sv->fbUsed -= (it->second.bytes + 255) & ~255ull;
    sv->reqs.erase(it);
    sv->wake.notify_one();
    return CR_OK;
}

cr_status cr_server_get_stats(cr_server* sv, cr_server_stats* st) {
    if (!sv || !st) return fail(CR_ERR_INVALID, "cr_server_get_stats: NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    memset(st, 0, sizeof(*st));
    st->submitted = sv->nSubmitted;
    st->completed = sv->nCompleted;
    st->batches = sv->nBatches;
    st->batched_views = sv->nBatchedViews;
    st->budget_bytes = sv->cfg.memory_budget;
    st->peak_bytes = sv->peak;
    if (!sv->latencies.empty()) {
        std::vector<double> l = sv->latencies;
        auto q = [&](double f) {
            const size_t k = std::min(l.size() - 1, (size_t)(f * (double)(l.size() - 1) + 0.5));
            std::nth_element(l.begin(), l.begin() + k, l.end());
            return l[k];
        };
        st->p50_ms = q(0.50);
        st->p99_ms = q(0.99);
        double sum = 0;
        for (double x : sv->latencies) sum += x;
        st->mean_ms = sum / (double)sv->latencies.size();
        const double span = (sv->lastDone - sv->firstSubmit) * 1e-6;
        st->views_per_s = span > 0 ? (double)sv->nCompleted / span : 0.0;
    }
    return CR_OK;
}

cr_status cr_server_reset_stats(cr_server* sv) {
    if (!sv) return fail(CR_ERR_INVALID, "cr_server_reset_stats: NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->nSubmitted = sv->nCompleted = sv->nBatches = sv->nBatchedViews = 0;
    sv->latencies.clear();
    sv->firstSubmit = 0;
    sv->lastDone = 0;
    sv->peak = 0;
    return CR_OK;
}

cr_status cr_server_destroy(cr_server* sv) {
    if (!sv) return CR_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->wake.notify_all();
    sv->wakeOoc.notify_all();
    if (sv->dispatcher.joinable()) sv->dispatcher.join();
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->wakeOoc.notify_all();
    }
    if (sv->oocLane.joinable()) sv->oocLane.join();
    cudaSetDevice(sv->ctx->device);
    cudaDeviceSynchronize();
    for (auto& s : sv->slots) {
        scratch_free(sv->ctx, s->S);
        if (s->stream) cudaStreamDestroy(s->stream);
    }
    if (sv->oocStream) cudaStreamDestroy(sv->oocStream);
    sv->ctx->dev_free(sv->fbBase, sv->fbCap);
    delete sv;
    return CR_OK;
}

}  // extern "C"
