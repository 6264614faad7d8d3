// vx_serve.cpp -- device-resident ray-query serving loop with continuous
// batching (vx_server_* / vx_serve_bench in include/voxrt.h).
//
// Threads: callers submit requests into a FIFO; one worker thread drives
// the device in one of two modes.
//
// VX_SERVE_SLOTS, each round:
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
//
// VX_SERVE_RESIDENT (the loop itself is vx_resident.cu), each round:
//   1. retires requests whose completion word the loop has written (copying
//      staged records to the caller) and notes an instance that has ended;
//   2. at the FIFO head: a request is admitted while the rays in flight fit
//      the budget and its descriptor slot is free, staged if the caller's
//      buffers are not page-locked, and published (descriptor, then head);
//      an edit publishes a fence, waits until an instance has taken it and
//      ended, then runs on the loop's stream, so it lands after every
//      request before it and before every request after it;
//   3. starts an instance when none runs and published descriptors wait.
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
    // device addresses of the caller's buffers when page-locked, mapped and
    // 16-byte aligned: the resident loop reads and writes them in place;
    // 0 = staged
    uint64_t rays_dev = 0, out_dev = 0;
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

// the device address of page-locked host memory p, if mapped and aligned
uint64_t mapped_address(const void *p, uintptr_t align) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (a.type != cudaMemoryTypeHost || a.devicePointer == nullptr) return 0;
    const uintptr_t d = reinterpret_cast<uintptr_t>(a.devicePointer);
    // the loop packs addresses into 48 bits beside a tag
    return d % align == 0 && ((uint64_t)d >> 48) == 0 ? (uint64_t)d : 0;
}

// A published request of the resident loop (position order).
struct ResFlight {
    Request *r = nullptr;
    uint64_t pos = 0;
    size_t n = 0;
    size_t off = SIZE_MAX;   // staging range [off, off + n), SIZE_MAX = none
    bool stage_out = false;  // records land in staging and are copied out
    bool done = false;
};

// Page-locked staging for callers whose buffers are not page-locked (or not
// 16-byte aligned): one ring of rays and one of records, ranges taken in
// position order and given back in position order.
struct StageRing {
    size_t cap = 0, head = 0;
    std::deque<std::pair<size_t, size_t>> live;  // (offset, length), oldest first
    size_t take(size_t n) {
        if (n > cap) return SIZE_MAX;
        if (live.empty()) {
            head = n;
            live.emplace_back(0, n);
            return 0;
        }
        const size_t tail = live.front().first;
        size_t off = SIZE_MAX;
        if (head > tail) {
            if (head + n <= cap) off = head;
            else if (n <= tail) off = 0;
        } else if (head < tail && head + n <= tail) {
            off = head;
        }
        if (off != SIZE_MAX) {
            head = off + n;
            live.emplace_back(off, n);
        }
        return off;
    }
    void give_back() {
        live.pop_front();
        if (live.empty()) head = 0;
    }
};

struct ResState {
    vx::ResHostBox *hbox = nullptr, *hbox_d = nullptr;    // host / device addresses
    vx::ResReplyBox *rbox = nullptr, *rbox_d = nullptr;
    vx::ResCounters *ctr = nullptr;
    unsigned long long *req = nullptr, *unit = nullptr;  // tagged words (vx_internal.h)
    uint32_t *cnt = nullptr;
    uint32_t unit_ring = 0;
    VxRay *st_rays = nullptr;
    VxHitRecord *st_out = nullptr;
    uint64_t st_rays_d = 0, st_out_d = 0;
    StageRing stage;
    cudaStream_t stream = nullptr;
    cudaEvent_t inst_done = nullptr;
    unsigned grid = 0;
    bool live = false;              // an instance may still run
    uint64_t published = 0;         // descriptors written (requests and fences)
    uint64_t edits_enqueued = 0;    // edits on the stream so far
    bool fence_pending = false;
    uint64_t fence_pos = 0;
    std::deque<ResFlight> flight;
    size_t flight_rays = 0;
    std::deque<Cmd> local;          // commands taken from the FIFO, in order
    uint64_t idle_ns = 0, life_ns = 0, wait_ns = 0;
};

double ms_since(Clock::time_point t) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
}

}  // namespace

struct VxServer {
    VxWorld *world = nullptr;
    int device = 0;
    vx::TraceArgs ta{};
    size_t cap = 0;                    // rays of one request at most
    size_t max_reqs = 0;               // requests per batch, 0 = no limit
    std::vector<Slot> slots;
    bool resident = false;             // VX_SERVE_RESIDENT
    size_t budget_rays = 0;            // RESIDENT: rays in flight at most
    ResState res;

    std::mutex mu;  // fifo + tickets
    std::deque<Cmd> fifo;
    // commands in fifo: the polling worker takes the lock only when there are some
    std::atomic<size_t> queued{0};
    std::unordered_map<uint64_t, Request *> tickets;
    std::atomic<uint64_t> next_ticket{1};

    std::mutex done_mu;
    std::condition_variable done_cv;

    std::thread worker;
    std::atomic<bool> stop{false};
    // Written by the worker thread only, before it sets `failed` and stops;
    // other threads read it only after seeing `failed`.
    std::string worker_error;
    std::atomic<bool> failed{false};
    bool device_error = false;  // worker_error came from a kernel's error word

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

// Enqueues the edit's copies and brick update on the edit stream (SLOTS:
// after every batch on the device) or on the loop's stream (RESIDENT: after
// the instance that took the edit's fence).
bool run_edit(VxServer *s, Edit *e) {
    const size_t n = e->idx.size();
    cudaStream_t es = s->resident ? s->res.stream : s->edit_stream;
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
            if (sl.busy && err == cudaSuccess) err = cudaStreamWaitEvent(es, sl.done, 0);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(b.d_idx, b.h_idx, n * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                  es);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(b.d_bricks, b.h_bricks, n * sizeof(VxBrick),
                                  cudaMemcpyHostToDevice, es);
        if (err == cudaSuccess) {
            vx::world_masks_changed(s->world);
            err = vx::launch_apply_dirty(s->ta.w, b.d_idx, b.d_bricks, n, es);
        }
        if (err == cudaSuccess) err = cudaEventRecord(b.used, es);
        if (err == cudaSuccess) err = cudaEventRecord(s->edit_done, es);
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

// ---------------------------------------------------------------- RESIDENT
uint64_t res_consumed(const ResState &R) {
    return __atomic_load_n(&R.rbox->consumed, __ATOMIC_ACQUIRE);
}

// a descriptor may go to position pos: its slot was taken by the loop and the
// request that last used the slot is done
bool res_slot_free(const ResState &R, uint64_t pos) {
    if (pos - res_consumed(R) >= vx::kResRing) return false;
    return R.flight.empty() || pos - R.flight.front().pos < vx::kResRing;
}

void res_write(ResState &R, const vx::ResDesc &d) {
    R.hbox->desc[R.published % vx::kResRing] = d;
    __atomic_store_n(&R.hbox->head, R.published + 1, __ATOMIC_RELEASE);
    R.published += 1;
}

// completion words -> caller buffers; returns false on a loop error
bool res_retire(VxServer *s, bool *progress) {
    ResState &R = s->res;
    for (ResFlight &f : R.flight) {
        if (f.done) continue;
        const uint64_t w = __atomic_load_n(&R.rbox->done[f.pos % vx::kResRing], __ATOMIC_ACQUIRE);
        if (w != vx::res_done_word(f.pos)) continue;
        if (f.stage_out)
            std::memcpy(f.r->out, R.st_out + f.off, f.n * sizeof(VxHitRecord));
        f.done = true;
        R.flight_rays -= f.n;
        {
            std::lock_guard<std::mutex> lk(s->stat_mu);
            s->inflight -= f.n;
        }
        complete(s, f.r);  // the caller may free f.r from here on
        f.r = nullptr;
        *progress = true;
    }
    while (!R.flight.empty() && R.flight.front().done) {
        if (R.flight.front().off != SIZE_MAX) R.stage.give_back();
        R.flight.pop_front();
    }
    // a wait in the loop that ran out, whether or not the launch is still up
    const uint32_t err = __atomic_load_n(&R.rbox->error, __ATOMIC_ACQUIRE);
    if (err != vx::RES_ERR_NONE) {
        s->device_error = true;
        s->worker_error = err == vx::RES_ERR_UNIT_WAIT
                              ? "resident loop: a worker's wait for its unit ran out"
                              : "resident loop: the wait for room in the unit table ran out";
        return false;
    }
    if (R.live) {
        const cudaError_t q = cudaEventQuery(R.inst_done);
        if (q == cudaErrorNotReady) return true;
        if (q != cudaSuccess) {
            s->worker_error = cudaGetErrorString(q);
            return false;
        }
        R.live = false;
        *progress = true;
    }
    return true;
}

bool res_launch(VxServer *s) {
    ResState &R = s->res;
    vx::ResArgs a{};
    a.ta = s->ta;
    a.host = R.hbox_d;
    a.reply = R.rbox_d;
    a.ctr = R.ctr;
    a.req = R.req;
    a.unit = R.unit;
    a.cnt = R.cnt;
    a.unit_ring = R.unit_ring;
    // the previous instance has ended: its last words are final
    a.consumed = res_consumed(R);
    a.unit_base = __atomic_load_n(&R.rbox->unit_end, __ATOMIC_ACQUIRE);
    a.edits_before = R.edits_enqueued;
    a.idle_ns = R.idle_ns;
    a.life_ns = R.life_ns;
    a.wait_ns = R.wait_ns;
    cudaError_t err = cudaMemsetAsync(R.ctr, 0, sizeof(vx::ResCounters), R.stream);
    if (err == cudaSuccess) err = vx::launch_serve_loop(a, R.grid, R.stream);
    if (err == cudaSuccess) err = cudaEventRecord(R.inst_done, R.stream);
    if (err != cudaSuccess) {
        s->worker_error = cudaGetErrorString(err);
        return false;
    }
    R.live = true;
    std::lock_guard<std::mutex> lk(s->stat_mu);
    s->batches += 1;
    return true;
}

// publish one request; false when it must wait for admission
bool res_publish(VxServer *s, Request *r) {
    ResState &R = s->res;
    if (R.flight_rays + r->n > s->budget_rays || !res_slot_free(R, R.published)) return false;
    ResFlight f;
    f.r = r;
    f.pos = R.published;
    f.n = r->n;
    uint64_t rays = r->rays_dev, out = r->out_dev;
    if (!rays || !out) {
        // whole units, so that every unit's records start 16-byte aligned
        f.off = R.stage.take((r->n + 31) / 32 * 32);
        if (f.off == SIZE_MAX) return false;
        if (!rays) {
            std::memcpy(R.st_rays + f.off, r->rays, r->n * sizeof(VxRay));
            rays = R.st_rays_d + f.off * sizeof(VxRay);
        }
        if (!out) {
            out = R.st_out_d + f.off * sizeof(VxHitRecord);
            f.stage_out = true;
        }
    }
    vx::ResDesc d;
    d.rays = rays;
    d.out = out;
    d.n = (uint32_t)r->n;
    d.kind = vx::RES_REQ;
    d.seq = R.published;
    res_write(R, d);
    R.flight.push_back(f);
    R.flight_rays += r->n;
    std::lock_guard<std::mutex> lk(s->stat_mu);
    s->inflight += r->n;
    s->peak_inflight = std::max(s->peak_inflight, s->inflight);
    return true;
}

// the edit at the FIFO head; *taken once it is on the stream
bool res_edit(VxServer *s, Edit *e, bool *taken) {
    ResState &R = s->res;
    if (!R.fence_pending) {
        if (!R.live && res_consumed(R) == R.published) {
            R.edits_enqueued += 1;
            *taken = true;
            return run_edit(s, e);
        }
        if (!res_slot_free(R, R.published)) return true;
        vx::ResDesc d{};
        d.kind = vx::RES_FENCE;
        d.seq = R.edits_enqueued + 1;
        R.fence_pos = R.published;
        res_write(R, d);
        R.fence_pending = true;
        return true;
    }
    if (!R.live && res_consumed(R) > R.fence_pos) {
        R.fence_pending = false;
        R.edits_enqueued += 1;
        *taken = true;
        return run_edit(s, e);
    }
    return true;
}

void resident_loop(VxServer *s) {
    ResState &R = s->res;
    while (!s->stop.load(std::memory_order_acquire)) {
        bool progress = false;
        if (!res_retire(s, &progress)) break;
        bool ok = true;
        if (s->queued.load(std::memory_order_acquire) != 0) {
            // everything queued, in order, under one hold of the lock
            std::lock_guard<std::mutex> lk(s->mu);
            s->queued.fetch_sub(s->fifo.size(), std::memory_order_relaxed);
            for (Cmd &c : s->fifo) R.local.push_back(c);
            s->fifo.clear();
        }
        while (!R.local.empty()) {
            const Cmd head = R.local.front();
            if (head.edit) {
                bool taken = false;
                ok = res_edit(s, head.edit, &taken);
                if (taken) {  // run_edit has consumed the Edit
                    R.local.pop_front();
                    progress = true;
                }
                if (!ok || !taken) break;
                continue;
            }
            Request *r = head.req;
            if (r->n == 0) {
                R.local.pop_front();
                complete(s, r);
                progress = true;
                continue;
            }
            if (!res_publish(s, r)) break;
            R.local.pop_front();
            progress = true;
        }
        if (!ok) break;
        if (!R.live && res_consumed(R) < R.published) {
            if (!res_launch(s)) break;
            progress = true;
        }
        if (!progress) std::this_thread::yield();
    }
    // the instance ends at its next poll
    __atomic_store_n(&R.hbox->stop, 1u, __ATOMIC_RELEASE);
}

void worker_loop_body(VxServer *s);

void worker_loop(VxServer *s) {
    cudaSetDevice(s->device);
    if (s->resident)
        resident_loop(s);
    else
        worker_loop_body(s);
    // every path out of the loops other than stop has set worker_error
    if (!s->worker_error.empty()) s->failed.store(true, std::memory_order_release);
    s->done_cv.notify_all();
}

void worker_loop_body(VxServer *s) {
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
        if (s->queued.load(std::memory_order_acquire) != 0) {
            std::lock_guard<std::mutex> lk(s->mu);
            if (!s->fifo.empty() && s->fifo.front().edit) {
                edit = s->fifo.front().edit;
                s->fifo.pop_front();
                s->queued.fetch_sub(1, std::memory_order_relaxed);
            } else if (free_slot) {
                size_t n = 0;
                while (!s->fifo.empty() && s->fifo.front().req &&
                       n + s->fifo.front().req->n <= s->cap &&
                       (s->max_reqs == 0 || free_slot->reqs.size() < s->max_reqs)) {
                    Request *r = s->fifo.front().req;
                    s->fifo.pop_front();
                    s->queued.fetch_sub(1, std::memory_order_relaxed);
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

void free_resident(ResState &R) {
    if (R.hbox) __atomic_store_n(&R.hbox->stop, 1u, __ATOMIC_RELEASE);
    if (R.stream) cudaStreamSynchronize(R.stream);
    cudaFreeHost(R.hbox);
    cudaFreeHost(R.rbox);
    cudaFreeHost(R.st_rays);
    cudaFreeHost(R.st_out);
    cudaFree(R.ctr);
    cudaFree(R.req);
    cudaFree(R.unit);
    cudaFree(R.cnt);
    if (R.inst_done) cudaEventDestroy(R.inst_done);
    if (R.stream) cudaStreamDestroy(R.stream);
}

cudaError_t host_mapped(size_t bytes, void **host, uint64_t *dev) {
    cudaError_t e = cudaHostAlloc(host, bytes, cudaHostAllocMapped | cudaHostAllocPortable);
    if (e != cudaSuccess) {
        *host = nullptr;
        return e;
    }
    std::memset(*host, 0, bytes);
    void *d = nullptr;
    e = cudaHostGetDevicePointer(&d, *host, 0);
    *dev = reinterpret_cast<uint64_t>(d);
    return e;
}

cudaError_t create_resident(VxServer *s, int32_t idle_us, int32_t wait_us) {
    ResState &R = s->res;
    R.idle_ns = (uint64_t)(idle_us > 0 ? idle_us : 2000) * 1000ull;
    R.life_ns = 250ull * 1000 * 1000;  // a quarter second per instance
    // every other wait: by default longer than any instance lives
    R.wait_ns = wait_us > 0 ? (uint64_t)wait_us * 1000ull : R.life_ns + R.idle_ns + 1000000000ull;
    R.unit_ring = (uint32_t)(s->budget_rays / 32 + vx::kResRing + 64);
    void *h = nullptr;
    uint64_t d = 0;
    cudaError_t e = host_mapped(sizeof(vx::ResHostBox), &h, &d);
    R.hbox = static_cast<vx::ResHostBox *>(h);
    R.hbox_d = reinterpret_cast<vx::ResHostBox *>(d);
    if (e == cudaSuccess) {
        e = host_mapped(sizeof(vx::ResReplyBox), &h, &d);
        R.rbox = static_cast<vx::ResReplyBox *>(h);
        R.rbox_d = reinterpret_cast<vx::ResReplyBox *>(d);
    }
    // staging in whole units: room for any admissible request, rounded up
    const size_t stage_rays = (s->budget_rays + 31) / 32 * 32;
    if (e == cudaSuccess) {
        e = host_mapped(stage_rays * sizeof(VxRay), &h, &R.st_rays_d);
        R.st_rays = static_cast<VxRay *>(h);
    }
    if (e == cudaSuccess) {
        e = host_mapped(stage_rays * sizeof(VxHitRecord), &h, &R.st_out_d);
        R.st_out = static_cast<VxHitRecord *>(h);
    }
    R.stage.cap = stage_rays;
    // the loop packs addresses into 48 bits beside a tag
    if (e == cudaSuccess && ((uint64_t)(R.st_rays_d | R.st_out_d) >> 48) != 0)
        e = cudaErrorInvalidValue;
    if (e == cudaSuccess) e = cudaMalloc(&R.ctr, sizeof(vx::ResCounters));
    // the tagged words start all ones: a tag that no position or unit of the
    // rings' first turn carries
    if (e == cudaSuccess) e = cudaMalloc(&R.req, vx::kResRing * 4 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(R.req, 0xFF, vx::kResRing * 4 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&R.unit, (size_t)R.unit_ring * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(R.unit, 0xFF, (size_t)R.unit_ring * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&R.cnt, vx::kResRing * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(R.cnt, 0, vx::kResRing * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&R.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&R.inst_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = vx::serve_loop_grid(s->ta, &R.grid);
    return e;
}

void free_server(VxServer *s) {
    if (s->resident) free_resident(s->res);
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
    for (std::deque<Cmd> *q : {&s->fifo, &s->res.local})
        for (Cmd &c : *q) {
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
    if (s->resident) {
        r->rays_dev = n > 0 ? mapped_address(rays, 16) : 0;
        r->out_dev = n > 0 ? mapped_address(out, 16) : 0;
    } else {
        r->pinned_in = n > 0 && is_pinned(rays);
        r->pinned_out = n > 0 && is_pinned(out);
    }
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (external) s->tickets[r->ticket] = r;
    s->fifo.push_back(Cmd{r, nullptr});
    s->queued.fetch_add(1, std::memory_order_release);
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
    if (!w || !origin || !p || !cfg || !out ||
        (cfg->mode != VX_SERVE_SLOTS && cfg->mode != VX_SERVE_RESIDENT) || cfg->idle_us < 0 ||
        cfg->wait_us < 0) {
        vx::set_error("vx_server_create: null argument, unknown mode or negative idle / wait time");
        return VX_ERR_INVALID;
    }
    const bool resident = cfg->mode == VX_SERVE_RESIDENT;
    if (!resident && (cfg->slots < 1 || cfg->slots > 16 || cfg->max_batch_rays < 0 ||
                      cfg->max_batch_requests < 0 ||
                      cfg->mem_budget_bytes < 56ull * (uint64_t)cfg->slots)) {
        vx::set_error("vx_server_create: need 1..16 slots and a budget of at least 56 B per slot");
        return VX_ERR_INVALID;
    }
    if (resident && (cfg->max_batch_rays < 0 || cfg->mem_budget_bytes < 56ull * 32 ||
                     cfg->mem_budget_bytes / 56ull > (1ull << 31))) {
        vx::set_error("vx_server_create: the resident loop needs a budget of 32 to 2^31 rays");
        return VX_ERR_INVALID;
    }
    if (p->max_iters < 0 || p->any_max_iters < 0 || p->max_iters > (1 << 20) ||
        p->any_max_iters > (1 << 20)) {
        vx::set_error("vx_server_create: iteration caps outside [0, 2^20]");
        return VX_ERR_INVALID;
    }
    if (!vx::origin_ok(origin, "vx_server_create")) return VX_ERR_INVALID;
    size_t cap = (size_t)(cfg->mem_budget_bytes / (uint64_t)(resident ? 1 : cfg->slots) / 56ull);
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
    s->resident = resident;
    s->budget_rays = (size_t)(cfg->mem_budget_bytes / 56ull);
    if (resident && e == cudaSuccess) e = create_resident(s, cfg->idle_us, cfg->wait_us);
    s->slots.resize(resident ? 0 : (size_t)cfg->slots);
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
    if (s->failed.load(std::memory_order_acquire)) {
        vx::set_error("vx_server_submit: server stopped: " + s->worker_error);
        return s->device_error ? VX_ERR_DEVICE : VX_ERR_CUDA;
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
            if (s->failed.load(std::memory_order_acquire)) {
                vx::set_error("vx_server_wait: server stopped: " + s->worker_error);
                return s->device_error ? VX_ERR_DEVICE : VX_ERR_CUDA;
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
    s->queued.fetch_add(1, std::memory_order_release);
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
    if (!s->failed.load(std::memory_order_acquire)) return VX_OK;
    return s->device_error ? VX_ERR_DEVICE : VX_ERR_CUDA;
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
                    if (s->failed.load(std::memory_order_acquire)) {
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
    // every client has reaped its last request: the load is served
    const double seconds = std::chrono::duration<double>(Clock::now() - t_start).count();
    editing = false;
    editor.join();
    for (auto p : pin_rays) cudaFreeHost(p);
    for (auto p : pin_out) cudaFreeHost(p);
    const int rc = vx_server_stats(s, st, 0);
    st->seconds = seconds;
    st->mrays_per_s = (double)st->rays / st->seconds / 1e6;
    if (failed) {
        vx::set_error("vx_serve_bench: server stopped: " + s->worker_error);
        return s->device_error ? VX_ERR_DEVICE : VX_ERR_CUDA;
    }
    return rc;
}

}  // extern "C"
