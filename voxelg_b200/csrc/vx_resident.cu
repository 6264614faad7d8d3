// vx_resident.cu -- the device-resident request loop of the ray-query server
// (VX_SERVE_RESIDENT in include/voxrt.h; host side in vx_serve.cpp).
//
// One launch ("instance") stays on the device while requests arrive.  Its
// first warp is the leader: it polls the host's descriptor ring (page-locked
// host memory mapped into the device's address space), takes descriptors in
// order, splits each request into 32-ray units and publishes them.  Every
// other warp is a worker: it takes a unit ticket, waits until the leader has
// published that unit, reads the unit's rays from host memory, traces them
// with the same walk as vx_trace (so records are identical), writes the
// records into host memory and, when it finishes the request's last unit,
// stores res_done_word(position) into the request's completion word.
//
// Ordering.  The host writes a descriptor, then releases `head`; the leader
// sees `head` move, takes one system-scope acquire fence and reads the
// descriptors.  What the leader publishes to the workers (the request's
// words, one word per unit, the published-unit count) carries tags and is
// read by the workers with plain device-coherent loads that wait for the
// right tag: no acquire load or fence in a worker's path.  (Polling with
// acquire loads measured slower under load: a query-sized load's p99 2.6 ms
// against 0.72.)  A warp
// counts its unit with a release atomic at system scope (its record stores
// to host memory come first); the warp that counts the request's last unit
// takes an acquire-release fence before it stores the completion word, so
// the host sees every record of a request once it sees the word.
//
// Ending.  An instance ends when the host sets `stop`, when it meets a fence
// descriptor (an edit follows on the same stream, after this launch), after
// idle_ns without a descriptor, or once it has run life_ns (the host starts
// the next instance).  The leader then sets the closing bit beside the
// final published count; workers finish every published unit and return.
// Every wait is bounded (wait_ns, and an iteration cap): a warp whose wait
// runs out records RES_ERR_* in the reply box and returns; the host reports
// it and stops the loop.
#include <cuda_runtime.h>

#include "vx_internal.h"
#include "vx_walk.cuh"

namespace vx {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint64_t kMaxPolls = 1ull << 26;  // iteration cap of every wait
constexpr uint32_t kClosing = 1u << 31;
constexpr uint64_t kPtrMask = (1ull << 48) - 1ull;

__device__ __forceinline__ uint64_t now_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// device-coherent loads and stores that neither read nor fill the SM's L1
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint64_t ld_relaxed(const unsigned long long *p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t *p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(unsigned long long *p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// host memory: system-scope accesses
__device__ __forceinline__ uint32_t ld_sys(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.relaxed.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint64_t ld_sys(const uint64_t *p) {
    uint64_t v;
    asm volatile("ld.relaxed.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_sys(uint64_t *p, uint64_t v) {
    asm volatile("st.relaxed.sys.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_sys(uint32_t *p, uint32_t v) {
    asm volatile("st.relaxed.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_sys() { asm volatile("fence.acq_rel.sys;" ::: "memory"); }
// *p += 1 with release order at system scope; returns the old value
__device__ __forceinline__ uint32_t count_release_sys(uint32_t *p) {
    uint32_t old;
    asm volatile("atom.release.sys.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(p) : "memory");
    return old;
}
// 16 bytes of host memory, fetched again rather than from a cached line (the
// caller's buffers are rewritten between requests)
__device__ __forceinline__ uint4 ld_fresh_u4(const void *p) {
    return __ldcv(reinterpret_cast<const uint4 *>(p));
}
__device__ __forceinline__ void st_u4(void *p, uint4 v) {
    asm volatile("st.global.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(v.x), "r"(v.y),
                 "r"(v.z), "r"(v.w)
                 : "memory");
}
__device__ __forceinline__ void st_u2(void *p, uint2 v) {
    asm volatile("st.global.v2.u32 [%0], {%1, %2};" ::"l"(p), "r"(v.x), "r"(v.y) : "memory");
}
__device__ __forceinline__ float4 u4_as_f4(uint4 v) {
    return make_float4(__uint_as_float(v.x), __uint_as_float(v.y), __uint_as_float(v.z),
                       __uint_as_float(v.w));
}

__device__ __forceinline__ void record_error(const ResArgs &a, uint32_t code) {
    st_sys(&a.reply->error, code);
    __threadfence_system();
}

// The leader warp: descriptors -> units.
__device__ void leader(const ResArgs &a) {
    const uint32_t lane = threadIdx.x & 31u;
    uint64_t c = a.consumed;
    uint64_t t0 = lane == 0 ? now_ns() : 0;
    t0 = __shfl_sync(kFull, t0, 0);
    uint64_t t_idle = t0;
    uint32_t pub = 0, reason = RES_RUNNING, backoff = 64;
    for (uint64_t it = 0; reason == RES_RUNNING; ++it) {
        uint64_t h = 0, t = 0;
        uint32_t stop = 0;
        if (lane == 0) {
            h = ld_sys(&a.host->head);
            stop = ld_sys(&a.host->stop);
            t = now_ns();
        }
        h = __shfl_sync(kFull, h, 0);
        stop = __shfl_sync(kFull, stop, 0);
        t = __shfl_sync(kFull, t, 0);
        if (stop) {
            reason = RES_STOPPED;
            break;
        }
        if (t - t0 > a.life_ns || it > kMaxPolls) {
            reason = RES_ROTATE;
            break;
        }
        if (c >= h) {
            if (t - t_idle > a.idle_ns) {
                reason = RES_IDLE;
                break;
            }
            __nanosleep(backoff);
            backoff = min(backoff * 2u, 1024u);
            continue;
        }
        backoff = 64;
        // the host's descriptors up to h, and the rays they point to, are visible
        fence_acq_rel_sys();
        // up to 32 descriptors at once, one per lane
        const uint32_t navail = (uint32_t)min(h - c, (uint64_t)32);
        ResDesc d{};
        if (lane < navail) {
            const ResDesc *src = &a.host->desc[(c + lane) % kResRing];
            d.rays = ld_sys(&src->rays);
            d.out = ld_sys(&src->out);
            d.n = ld_sys(&src->n);
            d.kind = ld_sys(&src->kind);
            d.seq = ld_sys(&src->seq);
        }
        for (uint32_t k = 0; k < navail; ++k) {
            const uint32_t kind = __shfl_sync(kFull, d.kind, k);
            const uint64_t seq = __shfl_sync(kFull, d.seq, k);
            const uint32_t n = kind == RES_FENCE ? 0u : __shfl_sync(kFull, d.n, k);
            const uint64_t rays = __shfl_sync(kFull, d.rays, k);
            const uint64_t out = __shfl_sync(kFull, d.out, k);
            const uint32_t nu = (n + 31u) / 32u;
            // room in the unit table (the host's admission keeps it; the
            // wait is a bound, not a schedule)
            uint32_t room = 0;
            if (lane == 0) {
                const uint64_t tw = now_ns();
                for (uint64_t w = 0;; ++w) {
                    if (pub + nu - ld_relaxed(&a.ctr->done_units) <= a.unit_ring) {
                        room = 1;
                        break;
                    }
                    if (w > kMaxPolls || now_ns() - tw > a.wait_ns) break;
                    __nanosleep(256);
                }
            }
            room = __shfl_sync(kFull, room, 0);
            if (!room) {
                if (lane == 0) record_error(a, RES_ERR_RING_WAIT);
                reason = RES_ROTATE;
                break;
            }
            // the request's words, tagged with its position (fences too, so
            // that a slot never holds words older than one ring turn)
            const uint32_t p32 = (uint32_t)c;
            const uint64_t tag16 = (uint64_t)(p32 & 0xFFFFu) << 48;
            const uint32_t g0 = a.unit_base + pub;
            if (lane < 4u) {
                const uint64_t w = lane == 0 ? ((rays & kPtrMask) | tag16)
                                 : lane == 1 ? ((out & kPtrMask) | tag16)
                                 : lane == 2 ? (((uint64_t)p32 << 32) | n)
                                             : (((uint64_t)p32 << 32) | g0);
                st_relaxed(a.req + (size_t)(c % kResRing) * 4u + lane, w);
            }
            ++c;
            if (kind == RES_FENCE) {
                // an edit enqueued before this instance is already applied
                if (seq > a.edits_before) {
                    reason = RES_FENCED;
                    break;
                }
                continue;
            }
            for (uint32_t j = lane; j < nu; j += 32u) {
                const uint32_t g = g0 + j;
                st_relaxed(a.unit + g % a.unit_ring, ((uint64_t)g << 32) | p32);
            }
            pub += nu;
            __syncwarp();
            if (lane == 0) st_relaxed(&a.ctr->pubw, pub);
        }
        if (lane == 0) st_sys(&a.reply->consumed, c);
        t_idle = t;
    }
    if (lane == 0) {
        st_sys(&a.reply->consumed, c);
        st_sys(&a.reply->unit_end, a.unit_base + pub);
        st_sys(&a.reply->status, reason);
        __threadfence_system();
        st_relaxed(&a.ctr->pubw, pub | kClosing);
    }
}

// A worker warp: unit tickets -> records.
template <uint32_t FL>
__device__ void worker(const ResArgs &a, uint4 *stage) {
    const uint32_t lane = threadIdx.x & 31u;
    const Ro ro{a.ta.ro[0], a.ta.ro[1], a.ta.ro[2]};
    for (;;) {
        // lane 0: a ticket, then the unit's words once their tags match
        uint32_t ok = 0, g = 0, n = 0, u0 = 0, p32 = 0;
        uint64_t rays = 0, out = 0;
        if (lane == 0) {
            const uint32_t rel = atomicAdd(&a.ctr->claim, 1u);
            g = a.unit_base + rel;
            const uint64_t tw = now_ns();
            uint32_t backoff = 32, stage = 0;
            for (uint64_t w = 0;; ++w) {
                if (stage == 0) {
                    const uint32_t pw = ld_relaxed(&a.ctr->pubw);
                    if (rel < (pw & ~kClosing)) {
                        stage = 1;
                        continue;
                    }
                    if (pw & kClosing) break;  // never published: done
                    // tickets near the published edge poll often, the rest rarely
                    __nanosleep(rel - (pw & ~kClosing) < 64u ? backoff : 8192u);
                    backoff = min(backoff * 2u, 1024u);
                } else {
                    const uint64_t uw = ld_relaxed(a.unit + g % a.unit_ring);
                    if ((uint32_t)(uw >> 32) == g) {
                        p32 = (uint32_t)uw;
                        const unsigned long long *rq = a.req + (size_t)(p32 % kResRing) * 4u;
                        const uint64_t w0 = ld_relaxed(rq), w1 = ld_relaxed(rq + 1);
                        const uint64_t w2 = ld_relaxed(rq + 2), w3 = ld_relaxed(rq + 3);
                        const uint64_t t16 = p32 & 0xFFFFu;
                        if ((w0 >> 48) == t16 && (w1 >> 48) == t16 &&
                            (uint32_t)(w2 >> 32) == p32 && (uint32_t)(w3 >> 32) == p32) {
                            rays = w0 & kPtrMask;
                            out = w1 & kPtrMask;
                            n = (uint32_t)w2;
                            u0 = (uint32_t)w3;
                            ok = 1;
                            break;
                        }
                    }
                    __nanosleep(32);
                }
                if (w > kMaxPolls || now_ns() - tw > a.wait_ns) {
                    record_error(a, RES_ERR_UNIT_WAIT);
                    break;
                }
            }
        }
        ok = __shfl_sync(kFull, ok, 0);
        if (!ok) return;
        g = __shfl_sync(kFull, g, 0);
        n = __shfl_sync(kFull, n, 0);
        u0 = __shfl_sync(kFull, u0, 0);
        p32 = __shfl_sync(kFull, p32, 0);
        rays = __shfl_sync(kFull, rays, 0);
        out = __shfl_sync(kFull, out, 0);
        // The unit's rays and records cross PCIe as contiguous 16-byte
        // pieces, one per lane (the warp's share of the request is one
        // contiguous range each way), staged in shared memory: a lane-per-ray
        // access would split each transfer into many small transactions.
        const uint32_t first = (g - u0) * 32u;
        const uint32_t cnt = min(32u, n - first);
        const char *src = reinterpret_cast<const char *>(rays) + (size_t)first * sizeof(VxRay);
        {
            // both reads in flight before either lands in the stage
            const bool h0 = lane < 2u * cnt, h1 = lane + 32u < 2u * cnt;
            uint4 c0 = make_uint4(0u, 0u, 0u, 0u), c1 = c0;
            if (h0) c0 = ld_fresh_u4(src + 16u * lane);
            if (h1) c1 = ld_fresh_u4(src + 16u * (lane + 32u));
            if (h0) stage[lane] = c0;
            if (h1) stage[lane + 32u] = c1;
        }
        __syncwarp();
        Hit h;
        if (lane < cnt) {
            const float4 r0 = u4_as_f4(stage[2u * lane]), r1 = u4_as_f4(stage[2u * lane + 1u]);
            // kind in the low two bits, as vx_trace reads it
            const uint32_t kind = __float_as_uint(r1.w) & 3u;
            uint64_t bytes = 0;
            if (kind == 1u) {
                uint32_t steps;
                const bool occ = trace_any_ray<FL, false>(a.ta.w, a.ta.p, ro, r0.x, r0.y, r0.z,
                                                          r0.w, r1.x, r1.y, r1.z, steps, bytes);
                set_miss(h);
                h.flags = occ ? 1u : 0u;
                h.steps = steps;
            } else if (kind == 2u) {
                trace_no_water_ray<FL, false>(a.ta.w, a.ta.p, ro, r0.x, r0.y, r0.z, r0.w, r1.x,
                                              r1.y, r1.z, h, bytes);
            } else {
                trace_ray<FL, false>(a.ta.w, a.ta.p, ro, r0.x, r0.y, r0.z, r0.w, r1.x, r1.y,
                                     r1.z, h, bytes);
            }
        }
        __syncwarp();  // every lane has its ray out of the stage
        if (lane < cnt)
            store_record(reinterpret_cast<VxHitRecord *>(reinterpret_cast<char *>(stage) + 24u * lane), h);
        __syncwarp();
        {
            // 24 * cnt bytes from a 16-byte aligned start (first is a
            // multiple of 32, the buffer 16-byte aligned)
            char *dst = reinterpret_cast<char *>(out) + (size_t)first * sizeof(VxHitRecord);
            const uint32_t bytes = 24u * cnt, full = bytes / 16u;
            for (uint32_t j = lane; j < full; j += 32u) st_u4(dst + 16u * j, stage[j]);
            if ((bytes & 15u) != 0u && lane == 0)
                st_u2(dst + 16u * full, reinterpret_cast<const uint2 *>(stage)[2u * full]);
        }
        __syncwarp();
        if (lane == 0) {
            // the unit counts with release order at system scope: the warp's
            // records reach host memory first; the warp that counts the last
            // unit acquires every other unit's records before it resets the
            // count and stores the completion word
            const uint32_t slot = p32 % kResRing;
            const uint32_t nu = (n + 31u) / 32u;
            if (count_release_sys(a.cnt + slot) == nu - 1u) {
                atomicExch(a.cnt + slot, 0u);
                fence_acq_rel_sys();
                st_sys(&a.reply->done[slot], res_done_word(p32));
            }
            atomicAdd(&a.ctr->done_units, 1u);
        }
    }
}

template <uint32_t FL>
__global__ void __launch_bounds__(128) k_serve_loop(ResArgs a) {
    // per warp: 32 rays in, then 32 records out
    __shared__ uint4 stage[4][64];
    if (blockIdx.x == 0 && threadIdx.x < 32u)
        leader(a);
    else
        worker<FL>(a, stage[threadIdx.x >> 5]);
}

template <uint32_t FL>
struct LoopK {
    static void *fn() { return reinterpret_cast<void *>(&k_serve_loop<FL>); }
};

void *loop_fn(const TraceArgs &ta) { return pick_fl<LoopK>((ta.p.flags & 7u) | pow2_bit(ta.w.d)); }

}  // namespace

cudaError_t serve_loop_grid(const TraceArgs &ta, unsigned *grid) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, loop_fn(ta), 128, 0);
    if (e != cudaSuccess) return e;
    per_sm = per_sm < 1 ? 1 : (per_sm > 4 ? 4 : per_sm);
    *grid = (unsigned)(sms * per_sm);
    return cudaSuccess;
}

cudaError_t launch_serve_loop(const ResArgs &a, unsigned grid, cudaStream_t s) {
    ResArgs args = a;
    void *p[] = {&args};
    return cudaLaunchKernel(loop_fn(a.ta), dim3(grid), dim3(128), p, 0, s);
}

}  // namespace vx
