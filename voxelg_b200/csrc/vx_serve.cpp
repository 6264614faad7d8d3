// vx_serve.cpp -- device-resident ray-query serving loop with continuous
// batching (vx_server_* / vx_serve_bench in include/voxrt.h).
//
// Threads: callers submit requests into a FIFO; one worker thread
//   1. retires finished slots (event query), scatters each request's records
//      into its caller buffer and marks it done;
//   2. at the FIFO head: an edit is launched on the edit stream after every
//      in-flight batch (stream waits on their events) and later batches wait
//      on it; requests are packed into a free slot until the slot is full or
//      the FIFO is empty, copied to the device, traced and copied back on the
//      slot's own stream.
// Several slots are in flight at once, so a batch formed while others run
// overlaps them on the device.  The slots' device buffers are the admission
// budget: a request that does not fit in the free slot waits for the next.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <random>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "vx_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    const VxRay *rays = nullptr;
    size_t n = 0;
    VxHitRecord *out = nullptr;
    uint64_t ticket = 0;
    Clock::time_point t_submit;
    std::atomic<int> done{0};
    bool external = false;  // registered for vx_server_poll / vx_server_wait
    bool pinned_in = false;  // caller buffers in page-locked memory: copied
    bool pinned_out = false; // straight to / from the slot's device buffers
};

struct Edit {
    std::vector<uint32_t> idx;
    std::vector<VxBrick> bricks;
};

struct Cmd {
    Request *req = nullptr;
    Edit *edit = nullptr;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    VxRay *h_rays = nullptr;       // pinned staging
    VxHitRecord *h_out = nullptr;  // pinned staging
    VxRay *d_rays = nullptr;
    VxHitRecord *d_out = nullptr;
    std::vector<Request *> reqs;
    std::vector<size_t> offs;
    size_t n = 0;
    bool busy = false;
};

bool is_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

double ms_since(Clock::time_point t) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
}

}  // namespace

struct VxServer {
    VxWorld *world = nullptr;
    int device = 0;
    vx::TraceArgs ta{};
    size_t cap = 0;
    size_t max_reqs = 0;               // requests per batch, 0 = no limit
    std::vector<Slot> slots;

    std::mutex mu;  // fifo + tickets
    std::deque<Cmd> fifo;
    std::unordered_map<uint64_t, Request *> tickets;
    std::atomic<uint64_t> next_ticket{1};

    std::mutex done_mu;
    std::condition_variable done_cv;

    std::thread worker;
    std::atomic<bool> stop{false};
    std::string worker_error;

    cudaStream_t edit_stream = nullptr;
    cudaEvent_t edit_done = nullptr;  // last edit: later batches wait on it
    bool edited = false;
    // two staging buffers, alternated, so that an edit never waits on the host
    // for the copy of the previous one
    struct EditBuf {
        uint32_t *h_idx = nullptr, *d_idx = nullptr;
        VxBrick *h_bricks = nullptr, *d_bricks = nullptr;
        size_t cap = 0;
        cudaEvent_t used = nullptr;  // the copies out of this buffer are done
        bool pending = false;
    } ebuf[2];
    int ecur = 0;

    std::mutex stat_mu;
    std::vector<double> lat_ms;
    uint64_t rays = 0, batches = 0, rejected = 0, edits = 0, edited_bricks = 0;
    uint64_t inflight = 0, peak_inflight = 0;
    Clock::time_point t0 = Clock::now();
};

namespace {

void complete(VxServer *s, Request *r) {
    const double l = ms_since(r->t_submit);
    {
        std::lock_guard<std::mutex> lk(s->stat_mu);
        s->lat_ms.push_back(l);
        s->rays += r->n;
    }
    {
        std::lock_guard<std::mutex> lk(s->done_mu);
        r->done.store(1, std::memory_order_release);
    }
    s->done_cv.notify_all();
}

// returns false on a CUDA error (recorded in worker_error)
bool retire(VxServer *s, bool *progress) {
    for (Slot &sl : s->slots) {
        if (!sl.busy) continue;
        const cudaError_t q = cudaEventQuery(sl.done);
        if (q == cudaErrorNotReady) continue;
        if (q != cudaSuccess) {
            s->worker_error = cudaGetErrorString(q);
            return false;
        }
        for (size_t i = 0; i < sl.reqs.size(); ++i) {
            Request *r = sl.reqs[i];
            if (!r->pinned_out)
                std::memcpy(r->out, sl.h_out + sl.offs[i], r->n * sizeof(VxHitRecord));
            complete(s, r);
        }
        {
            std::lock_guard<std::mutex> lk(s->stat_mu);
            s->inflight -= sl.n;
        }
        sl.reqs.clear();
        sl.offs.clear();
        sl.n = 0;
        sl.busy = false;
        *progress = true;
    }
    return true;
}

bool run_edit(VxServer *s, Edit *e) {
    const size_t n = e->idx.size();
    VxServer::EditBuf &b = s->ebuf[s->ecur];
    s->ecur ^= 1;
    cudaError_t err = cudaSuccess;
    if (b.pending) err = cudaEventSynchronize(b.used);  // two edits back: long done
    if (err == cudaSuccess && n > b.cap) {
        cudaFreeHost(b.h_idx);
        cudaFreeHost(b.h_bricks);
        cudaFree(b.d_idx);
        cudaFree(b.d_bricks);
        b.h_idx = b.d_idx = nullptr;
        b.h_bricks = b.d_bricks = nullptr;
        b.cap = 0;
        err = cudaMallocHost(&b.h_idx, n * sizeof(uint32_t));
        if (err == cudaSuccess) err = cudaMallocHost(&b.h_bricks, n * sizeof(VxBrick));
        if (err == cudaSuccess) err = cudaMalloc(&b.d_idx, n * sizeof(uint32_t));
        if (err == cudaSuccess) err = cudaMalloc(&b.d_bricks, n * sizeof(VxBrick));
        if (err == cudaSuccess) b.cap = n;
    }
    if (err == cudaSuccess && !b.used) err = cudaEventCreateWithFlags(&b.used, cudaEventDisableTiming);
    if (err == cudaSuccess && n > 0) {
        std::memcpy(b.h_idx, e->idx.data(), n * sizeof(uint32_t));
        std::memcpy(b.h_bricks, e->bricks.data(), n * sizeof(VxBrick));
        // after every batch already on the device
        for (Slot &sl : s->slots)
            if (sl.busy && err == cudaSuccess) err = cudaStreamWaitEvent(s->edit_stream, sl.done, 0);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(b.d_idx, b.h_idx, n * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                  s->edit_stream);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(b.d_bricks, b.h_bricks, n * sizeof(VxBrick),
                                  cudaMemcpyHostToDevice, s->edit_stream);
        if (err == cudaSuccess) {
            vx::world_masks_changed(s->world);
            err = vx::launch_apply_dirty(s->ta.w, b.d_idx, b.d_bricks, n, s->edit_stream);
        }
        if (err == cudaSuccess) err = cudaEventRecord(b.used, s->edit_stream);
        if (err == cudaSuccess) err = cudaEventRecord(s->edit_done, s->edit_stream);
        if (err == cudaSuccess) {
            s->edited = true;
            b.pending = true;
        }
    }
    {
        std::lock_guard<std::mutex> lk(s->stat_mu);
        s->edits += 1;
        s->edited_bricks += n;
    }
    delete e;
    if (err != cudaSuccess) {
        s->worker_error = cudaGetErrorString(err);
        return false;
    }
    return true;
}

bool launch_batch(VxServer *s, Slot &sl) {
    size_t off = 0;
    for (Request *r : sl.reqs) {
        sl.offs.push_back(off);
        if (!r->pinned_in) std::memcpy(sl.h_rays + off, r->rays, r->n * sizeof(VxRay));
        off += r->n;
    }
    sl.n = off;
    sl.busy = true;
    {
        std::lock_guard<std::mutex> lk(s->stat_mu);
        s->batches += 1;
        s->inflight += off;
        s->peak_inflight = std::max(s->peak_inflight, s->inflight);
    }
    cudaError_t err = cudaSuccess;
    if (s->edited) err = cudaStreamWaitEvent(sl.stream, s->edit_done, 0);
    for (size_t i = 0; i < sl.reqs.size() && err == cudaSuccess; ++i) {
        const Request *r = sl.reqs[i];
        const void *src = r->pinned_in ? (const void *)r->rays : (const void *)(sl.h_rays + sl.offs[i]);
        err = cudaMemcpyAsync(sl.d_rays + sl.offs[i], src, r->n * sizeof(VxRay),
                              cudaMemcpyHostToDevice, sl.stream);
    }
    if (err == cudaSuccess) err = vx::launch_trace_rays(s->ta, sl.d_rays, off, sl.d_out, sl.stream);
    for (size_t i = 0; i < sl.reqs.size() && err == cudaSuccess; ++i) {
        Request *r = sl.reqs[i];
        void *dst = r->pinned_out ? (void *)r->out : (void *)(sl.h_out + sl.offs[i]);
        err = cudaMemcpyAsync(dst, sl.d_out + sl.offs[i], r->n * sizeof(VxHitRecord),
                              cudaMemcpyDeviceToHost, sl.stream);
    }
    if (err == cudaSuccess) err = cudaEventRecord(sl.done, sl.stream);
    if (err != cudaSuccess) {
        s->worker_error = cudaGetErrorString(err);
        return false;
    }
    return true;
}

void worker_loop(VxServer *s) {
    cudaSetDevice(s->device);
    while (!s->stop.load(std::memory_order_acquire)) {
        bool progress = false;
        if (!retire(s, &progress)) break;
        Slot *free_slot = nullptr;
        for (Slot &sl : s->slots)
            if (!sl.busy) {
                free_slot = &sl;
                break;
            }
        Edit *edit = nullptr;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (!s->fifo.empty() && s->fifo.front().edit) {
                edit = s->fifo.front().edit;
                s->fifo.pop_front();
            } else if (free_slot) {
                size_t n = 0;
                while (!s->fifo.empty() && s->fifo.front().req &&
                       n + s->fifo.front().req->n <= s->cap &&
                       (s->max_reqs == 0 || free_slot->reqs.size() < s->max_reqs)) {
                    Request *r = s->fifo.front().req;
                    s->fifo.pop_front();
                    free_slot->reqs.push_back(r);
                    n += r->n;
                }
            }
        }
        if (edit) {
            if (!run_edit(s, edit)) break;
            progress = true;
        } else if (free_slot && !free_slot->reqs.empty()) {
            if (!launch_batch(s, *free_slot)) break;
            progress = true;
        }
        if (!progress) std::this_thread::yield();
    }
}

void free_server(VxServer *s) {
    for (Slot &sl : s->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        cudaFreeHost(sl.h_rays);
        cudaFreeHost(sl.h_out);
        cudaFree(sl.d_rays);
        cudaFree(sl.d_out);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    if (s->edit_stream) cudaStreamSynchronize(s->edit_stream);
    for (auto &b : s->ebuf) {
        cudaFreeHost(b.h_idx);
        cudaFreeHost(b.h_bricks);
        cudaFree(b.d_idx);
        cudaFree(b.d_bricks);
        if (b.used) cudaEventDestroy(b.used);
    }
    if (s->edit_done) cudaEventDestroy(s->edit_done);
    if (s->edit_stream) cudaStreamDestroy(s->edit_stream);
    for (auto &kv : s->tickets) delete kv.second;
    for (Cmd &c : s->fifo) {
        delete c.edit;
        if (c.req && !c.req->external) delete c.req;
    }
}

Request *submit_internal(VxServer *s, const VxRay *rays, size_t n, VxHitRecord *out,
                         bool external) {
    Request *r = new Request();
    r->rays = rays;
    r->n = n;
    r->out = out;
    r->ticket = s->next_ticket.fetch_add(1);
    r->external = external;
    r->pinned_in = n > 0 && is_pinned(rays);
    r->pinned_out = n > 0 && is_pinned(out);
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (external) s->tickets[r->ticket] = r;
    s->fifo.push_back(Cmd{r, nullptr});
    return r;
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const size_t i = std::min(v.size() - 1, (size_t)std::ceil(q * (double)v.size()) - (q > 0 ? 1 : 0));
    return v[i];
}

}  // namespace

extern "C" {

int vx_server_create(VxWorld *w, const int32_t origin[3], const VxTraceParams *p,
                     const VxServeConfig *cfg, VxServer **out) {
    if (!w || !origin || !p || !cfg || !out || cfg->slots < 1 || cfg->slots > 16 ||
        cfg->max_batch_rays < 0 || cfg->max_batch_requests < 0 ||
        cfg->mem_budget_bytes < 56ull * (uint64_t)cfg->slots) {
        vx::set_error("vx_server_create: need 1..16 slots and a budget of at least 56 B per slot");
        return VX_ERR_INVALID;
    }
    if (p->max_iters < 0 || p->any_max_iters < 0 || p->max_iters > (1 << 20) ||
        p->any_max_iters > (1 << 20)) {
        vx::set_error("vx_server_create: iteration caps outside [0, 2^20]");
        return VX_ERR_INVALID;
    }
    if (!vx::origin_ok(origin, "vx_server_create")) return VX_ERR_INVALID;
    size_t cap = (size_t)(cfg->mem_budget_bytes / (uint64_t)cfg->slots / 56ull);
    if (cfg->max_batch_rays > 0) cap = std::min(cap, (size_t)cfg->max_batch_rays);
    if (cap < 1) {
        vx::set_error("vx_server_create: budget too small for one ray per slot");
        return VX_ERR_INVALID;
    }
    VxServer *s = new (std::nothrow) VxServer();
    if (!s) return VX_ERR_OOM;
    s->world = w;
    s->device = vx::world_device(w);
    s->ta.w = vx::world_dev(w);
    s->ta.p = *p;
    s->ta.ro[0] = origin[0];
    s->ta.ro[1] = origin[1];
    s->ta.ro[2] = origin[2];
    s->cap = cap;
    s->max_reqs = (size_t)cfg->max_batch_requests;
    cudaError_t e = cudaSetDevice(s->device);
    s->slots.resize((size_t)cfg->slots);
    for (Slot &sl : s->slots) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMallocHost(&sl.h_rays, cap * sizeof(VxRay));
        if (e == cudaSuccess) e = cudaMallocHost(&sl.h_out, cap * sizeof(VxHitRecord));
        if (e == cudaSuccess) e = cudaMalloc(&sl.d_rays, cap * sizeof(VxRay));
        if (e == cudaSuccess) e = cudaMalloc(&sl.d_out, cap * sizeof(VxHitRecord));
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->edit_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->edit_done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        vx::set_error(std::string("vx_server_create: ") + cudaGetErrorString(e));
        free_server(s);
        delete s;
        return e == cudaErrorMemoryAllocation ? VX_ERR_OOM : VX_ERR_CUDA;
    }
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return VX_OK;
}

int vx_server_submit(VxServer *s, const VxRay *rays, size_t n, VxHitRecord *out,
                     uint64_t *ticket) {
    if (!s || !ticket || (n > 0 && (!rays || !out))) {
        vx::set_error("vx_server_submit: null argument");
        return VX_ERR_INVALID;
    }
    if (n > s->cap) {
        std::lock_guard<std::mutex> lk(s->stat_mu);
        s->rejected += 1;
        vx::set_error("vx_server_submit: request larger than a batch slot");
        return VX_ERR_BUSY;
    }
    if (!s->worker_error.empty()) {
        vx::set_error("vx_server_submit: server stopped: " + s->worker_error);
        return VX_ERR_CUDA;
    }
    *ticket = submit_internal(s, rays, n, out, true)->ticket;
    return VX_OK;
}

int vx_server_poll(VxServer *s, uint64_t ticket) {
    if (!s) return VX_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) {
        vx::set_error("vx_server_poll: unknown ticket");
        return VX_ERR_INVALID;
    }
    if (!it->second->done.load(std::memory_order_acquire)) return 0;
    delete it->second;
    s->tickets.erase(it);
    return 1;
}

int vx_server_wait(VxServer *s, uint64_t ticket, double timeout_s) {
    if (!s) return VX_ERR_INVALID;
    Request *r = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) {
            vx::set_error("vx_server_wait: unknown ticket");
            return VX_ERR_INVALID;
        }
        r = it->second;
    }
    {
        std::unique_lock<std::mutex> lk(s->done_mu);
        const Clock::time_point deadline =
            Clock::now() + std::chrono::duration_cast<Clock::duration>(
                               std::chrono::duration<double>(timeout_s));
        while (!r->done.load(std::memory_order_acquire)) {
            if (!s->worker_error.empty()) {
                vx::set_error("vx_server_wait: server stopped: " + s->worker_error);
                return VX_ERR_CUDA;
            }
            if (Clock::now() >= deadline) break;
            const Clock::time_point tick = Clock::now() + std::chrono::milliseconds(50);
            s->done_cv.wait_until(lk, tick < deadline ? tick : deadline);
        }
        if (!r->done.load(std::memory_order_acquire)) return 0;
    }
    return vx_server_poll(s, ticket);
}

int vx_server_edit(VxServer *s, const uint32_t *brick_idx, const VxBrick *bricks, size_t n) {
    if (!s || (n > 0 && (!brick_idx || !bricks))) {
        vx::set_error("vx_server_edit: null argument");
        return VX_ERR_INVALID;
    }
    Edit *e = new Edit();
    std::unordered_map<uint32_t, size_t> last;
    last.reserve(n * 2);
    for (size_t i = 0; i < n; ++i) {
        if ((int64_t)brick_idx[i] >= s->ta.w.d.n_bricks) {
            delete e;
            vx::set_error("vx_server_edit: brick index out of range");
            return VX_ERR_INVALID;
        }
        last[brick_idx[i]] = i;
    }
    for (size_t i = 0; i < n; ++i)
        if (last[brick_idx[i]] == i) {
            e->idx.push_back(brick_idx[i]);
            e->bricks.push_back(bricks[i]);
        }
    std::lock_guard<std::mutex> lk(s->mu);
    s->fifo.push_back(Cmd{nullptr, e});
    return VX_OK;
}

int vx_server_stats(VxServer *s, VxServeStats *st, int32_t reset) {
    if (!s || !st) return VX_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->stat_mu);
    std::memset(st, 0, sizeof(*st));
    st->requests = s->lat_ms.size();
    st->rays = s->rays;
    st->batches = s->batches;
    st->rejected = s->rejected;
    st->edits = s->edits;
    st->edited_bricks = s->edited_bricks;
    st->p50_ms = percentile(s->lat_ms, 0.50);
    st->p99_ms = percentile(s->lat_ms, 0.99);
    double sum = 0.0, mx = 0.0;
    for (double v : s->lat_ms) {
        sum += v;
        mx = std::max(mx, v);
    }
    st->mean_ms = s->lat_ms.empty() ? 0.0 : sum / (double)s->lat_ms.size();
    st->max_ms = mx;
    st->seconds = std::chrono::duration<double>(Clock::now() - s->t0).count();
    st->mrays_per_s = st->seconds > 0 ? (double)s->rays / st->seconds / 1e6 : 0.0;
    st->peak_inflight_rays = s->peak_inflight;
    if (reset) {
        s->lat_ms.clear();
        s->rays = s->batches = s->rejected = s->edits = s->edited_bricks = 0;
        s->peak_inflight = s->inflight;
        s->t0 = Clock::now();
    }
    return s->worker_error.empty() ? VX_OK : VX_ERR_CUDA;
}

int vx_server_destroy(VxServer *s) {
    if (!s) return VX_OK;
    s->stop.store(true, std::memory_order_release);
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->device);
    free_server(s);
    delete s;
    return VX_OK;
}

int vx_serve_bench(VxServer *s, const VxServeLoad *L, VxServeStats *st) {
    if (!s || !L || !st || L->clients < 1 || L->clients > 1024 || !(L->rate_per_client > 0) ||
        !(L->seconds > 0) || L->min_rays < 1 || L->max_rays < L->min_rays ||
        (size_t)L->max_rays > s->cap || !(L->min_len > 0) || L->max_len < L->min_len ||
        L->edit_fraction_per_s < 0) {
        vx::set_error("vx_serve_bench: invalid load (max_rays must fit a batch slot)");
        return VX_ERR_INVALID;
    }
    const vx::Dims &d = s->ta.w.d;
    // a pool of seeded query rays in the window; requests copy a slice
    const size_t pool_n = (size_t)1 << 20;
    std::vector<VxRay> pool(pool_n);
    {
        std::mt19937_64 rng(L->seed);
        std::uniform_real_distribution<float> ux(0.f, (float)d.vx), uy(0.f, (float)d.vy),
            uz(0.f, (float)d.vz);
        std::normal_distribution<float> nd(0.f, 1.f);
        for (VxRay &r : pool) {
            r.org[0] = (float)s->ta.ro[0] + ux(rng);
            r.org[1] = (float)s->ta.ro[1] + uy(rng);
            r.org[2] = (float)s->ta.ro[2] + uz(rng);
            float x = nd(rng), y = nd(rng), z = nd(rng);
            const float l = std::sqrt((x * x + y * y) + z * z);
            r.dir[0] = x / l;
            r.dir[1] = y / l;
            r.dir[2] = z / l;
            r.tmax = 0.f;
            r.kind = (rng() & 3u) == 0u ? 1u : 0u;  // a quarter line-of-sight, the rest first hit
        }
    }
    std::atomic<bool> failed{false};
    // Each client owns a few page-locked request buffers (the receive buffers
    // of a network front end would be allocated so); a request waits for a
    // free one only if all of them are still in flight.
    constexpr int kBufs = 4;
    const size_t max_n = (size_t)L->max_rays;
    std::vector<VxRay *> pin_rays((size_t)L->clients * kBufs, nullptr);
    std::vector<VxHitRecord *> pin_out((size_t)L->clients * kBufs, nullptr);
    for (size_t i = 0; i < pin_rays.size(); ++i) {
        if (cudaMallocHost(&pin_rays[i], max_n * sizeof(VxRay)) != cudaSuccess ||
            cudaMallocHost(&pin_out[i], max_n * sizeof(VxHitRecord)) != cudaSuccess) {
            for (auto p : pin_rays) cudaFreeHost(p);
            for (auto p : pin_out) cudaFreeHost(p);
            vx::set_error("vx_serve_bench: cannot allocate page-locked request buffers");
            return VX_ERR_OOM;
        }
    }
    VxServeStats dummy;
    vx_server_stats(s, &dummy, 1);
    const auto t_start = Clock::now();
    const auto t_end = t_start + std::chrono::duration<double>(L->seconds);
    auto client = [&](int ci) {
        std::mt19937_64 rng(L->seed * 1000003ull + (uint64_t)ci);
        std::exponential_distribution<double> gap(L->rate_per_client);
        std::uniform_real_distribution<double> u01(0.0, 1.0);
        std::uniform_int_distribution<size_t> off_d(0, pool_n - max_n);
        Request *inflight[kBufs] = {};
        auto reap = [&](bool all) {
            for (int b = 0; b < kBufs; ++b) {
                while (inflight[b] && !inflight[b]->done.load(std::memory_order_acquire)) {
                    if (!all) break;
                    if (!s->worker_error.empty()) {
                        failed = true;
                        return;
                    }
                    std::this_thread::yield();
                }
                if (inflight[b] && inflight[b]->done.load(std::memory_order_acquire)) {
                    delete inflight[b];
                    inflight[b] = nullptr;
                }
            }
        };
        auto next = t_start + std::chrono::duration_cast<Clock::duration>(
                                  std::chrono::duration<double>(gap(rng)));
        while (next < t_end && !failed) {
            std::this_thread::sleep_until(next);
            const double lr = std::log((double)L->min_rays) +
                              u01(rng) * (std::log((double)L->max_rays) - std::log((double)L->min_rays));
            const size_t n = std::min(max_n, std::max((size_t)L->min_rays,
                                                      (size_t)std::llround(std::exp(lr))));
            const float len = (float)std::exp(std::log((double)L->min_len) +
                                              u01(rng) * (std::log((double)L->max_len) -
                                                          std::log((double)L->min_len)));
            int b = -1;
            while (b < 0 && !failed) {
                reap(false);
                for (int k = 0; k < kBufs; ++k)
                    if (!inflight[k]) {
                        b = k;
                        break;
                    }
                if (b < 0) std::this_thread::yield();
            }
            if (b < 0) break;
            VxRay *rays = pin_rays[(size_t)ci * kBufs + b];
            VxHitRecord *out = pin_out[(size_t)ci * kBufs + b];
            std::memcpy(rays, pool.data() + off_d(rng), n * sizeof(VxRay));
            for (size_t i = 0; i < n; ++i) rays[i].tmax = len;
            inflight[b] = submit_internal(s, rays, n, out, false);
            next += std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(gap(rng)));
        }
        reap(true);
    };
    std::atomic<bool> editing{true};
    std::thread editor([&]() {
        if (!(L->edit_fraction_per_s > 0)) return;
        std::mt19937_64 rng(L->seed ^ 0xED17ull);
        const double per_tick = L->edit_fraction_per_s * (double)d.n_bricks * 0.01;  // 10 ms ticks
        double carry = 0.0;
        auto next = Clock::now();
        std::uniform_int_distribution<uint64_t> bd(0, (uint64_t)d.n_bricks - 1);
        const uint8_t mats[4] = {2, 3, 4, 12};
        while (editing.load()) {
            next += std::chrono::milliseconds(10);
            std::this_thread::sleep_until(next);
            carry += per_tick;
            const size_t k = (size_t)carry;
            carry -= (double)k;
            if (k == 0) continue;
            std::vector<uint32_t> idx(k);
            std::vector<VxBrick> b(k);
            for (size_t i = 0; i < k; ++i) {
                idx[i] = (uint32_t)bd(rng);
                const uint64_t occ = rng() & rng();  // about a quarter of the voxels solid
                b[i].occupancy = occ;
                for (int v = 0; v < 64; ++v)
                    b[i].materials[v] = ((occ >> v) & 1ull) ? mats[rng() & 3u] : 0;
            }
            vx_server_edit(s, idx.data(), b.data(), k);
        }
    });
    std::vector<std::thread> clients;
    for (int i = 0; i < L->clients; ++i) clients.emplace_back(client, i);
    for (auto &t : clients) t.join();
    editing = false;
    editor.join();
    for (auto p : pin_rays) cudaFreeHost(p);
    for (auto p : pin_out) cudaFreeHost(p);
    const int rc = vx_server_stats(s, st, 0);
    st->seconds = std::chrono::duration<double>(Clock::now() - t_start).count();
    st->mrays_per_s = (double)st->rays / st->seconds / 1e6;
    if (failed) {
        vx::set_error("vx_serve_bench: server stopped: " + s->worker_error);
        return VX_ERR_CUDA;
    }
    return rc;
}

}  // extern "C"
