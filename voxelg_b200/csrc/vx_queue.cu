// vx_queue.cu -- the mixed ray queue: rays of different kinds and very
// uneven lengths (primary with spawned shadow, GI-probe, picking, any-hit
// line-of-sight, no-water) traced by ONE persistent launch.
//
// Every lane walks one ray at a time with the shared cascade step
// (vx_walk.cuh) and takes the next queue item when its ray ends; a primary
// that hits and carries VX_RAY_SPAWN_SHADOW continues in the same lane with
// its shadow ray (raymarch.wgsl:3953-3994).  Lanes of a warp refill together
// once `refill_min` of them are idle (a lone refill would stall 31 lanes
// through a ray set-up).  Optionally the queue is first reordered by a
// coherence key (kind, window half in x and z, direction on a 64x64 octahedral
// grid) with a counting sort, so that a warp's rays start near each other
// and head the same way.  Results do not depend on
// any of these choices; the autotuner checks that and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "vx_internal.h"
#include "vx_walk.cuh"

namespace vx {
namespace {

constexpr uint32_t kSortBins = 1u << 16;

struct QueueArgs {
    TraceArgs ta;
    const VxRay *rays;
    const uint32_t *order;    // coherence permutation or nullptr (identity)
    uint32_t n;
    VxHitRecord *out;
    VxShadowRecord *shadow;   // shadow records of spawning rays, or nullptr
    uint32_t *work;           // {next item, warps done}, self-resetting
    uint32_t refill_min;
};

__device__ __forceinline__ void load_ray(const VxRay *rays, uint32_t i, float &ox, float &oy,
                                         float &oz, float &dx, float &dy, float &dz, float &tmax,
                                         uint32_t &kind) {
    const float4 a = __ldg(reinterpret_cast<const float4 *>(rays + i));
    const float4 b = __ldg(reinterpret_cast<const float4 *>(rays + i) + 1);
    ox = a.x; oy = a.y; oz = a.z; dx = a.w; dy = b.x; dz = b.y; tmax = b.z;
    kind = __float_as_uint(b.w);
}

template <uint32_t FL>
__global__ void __launch_bounds__(256) k_queue(QueueArgs q) {
    constexpr uint32_t FULL = 0xFFFFFFFFu, IDLE = 0xFFFFFFFFu, DONE = 0xFFFFFFFEu;
    const uint32_t lane = threadIdx.x & 31u;
    const DevWorld &w = q.ta.w;
    const Ro ro{q.ta.ro[0], q.ta.ro[1], q.ta.ro[2]};
    const Geo g = geo_of<FL>(w.d, ro);
    const VxTraceParams &p = q.ta.p;
    uint64_t bytes = 0;
    Walk k;
    Hit h;
    uint32_t item = IDLE;     // queue slot being walked (IDLE / DONE otherwise)
    uint32_t ray = 0;         // index of the ray in q.rays
    uint32_t rkind = 0;       // kind word of that ray
    bool shadow_phase = false;
    float ox = 0.f, oy = 0.f, oz = 0.f;
    for (;;) {
        const bool need = item == IDLE;
        const unsigned ask = __ballot_sync(FULL, need);
        const unsigned busy = __ballot_sync(FULL, item < DONE);
        if (ask && ((uint32_t)__popc(ask) >= q.refill_min || busy == 0u)) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(q.work, (uint32_t)__popc(ask));
            base = __shfl_sync(FULL, base, 0);
            if (need) {
                const uint32_t slot = base + (uint32_t)__popc(ask & ((1u << lane) - 1u));
                if (slot >= q.n) {
                    item = DONE;
                } else {
                    item = slot;
                    ray = q.order ? __ldg(q.order + slot) : slot;
                    float dx, dy, dz, tmax;
                    load_ray(q.rays, ray, ox, oy, oz, dx, dy, dz, tmax, rkind);
                    shadow_phase = false;
                    set_miss(h);
                    if (q.shadow) reinterpret_cast<uint2 *>(q.shadow)[ray] = make_uint2(0u, 0u);
                    const uint32_t kind = rkind & 3u;
                    if (!walk_init(w.d, ro, kind > 2u ? KIND_TRACE : kind, p, ox, oy, oz, dx, dy,
                                   dz, tmax, k)) {
                        if (kind == KIND_ANY) h.flags = 0u;
                        h.steps = 0;
                        store_record(q.out + ray, h);
                        item = IDLE;
                    }
                }
            }
        }
        if (__all_sync(FULL, item == DONE)) break;
        if (item < DONE) {
            const int r = walk_step<FL, false, -1>(w, g, p, ro, k, h, bytes);
            if (r != WALK_CONT) {
                item = IDLE;
                if (shadow_phase) {
                    reinterpret_cast<uint2 *>(q.shadow)[ray] =
                        make_uint2(k.iters, (r == WALK_HIT ? 1u : 0u) | (1u << 8));
                } else if (k.kind == KIND_ANY) {
                    set_miss(h);
                    h.flags = r == WALK_HIT ? 1u : 0u;
                    h.steps = k.iters;
                    store_record(q.out + ray, h);
                } else {
                    h.steps = k.iters;
                    store_record(q.out + ray, h);
                    if (q.shadow && (rkind & VX_RAY_SPAWN_SHADOW) && r == WALK_HIT) {
                        {
                            // raymarch.wgsl:3953-3994 from this ray's hit; the
                            // jitter is seeded by the ray index
                            const int ax = (int)(h.face >> 1);
                            const float nv = (h.face & 1u) ? -1.0f : 1.0f;
                            const float sox = (ox + k.s.dx * h.t) + (ax == 0 ? nv : 0.0f) * 0.001f;
                            const float soy = (oy + k.s.dy * h.t) + (ax == 1 ? nv : 0.0f) * 0.001f;
                            const float soz = (oz + k.s.dz * h.t) + (ax == 2 ? nv : 0.0f) * 0.001f;
                            const float jit = ign((float)(ray & 0xFFFFu), (float)(ray >> 16), p.frame);
                            const float theta = jit * 2.39996323f;
                            const float radius = p.cone_tan * sqrtf(jit);
                            float sn, cs;
                            sincos_series(theta, sn, cs);
                            float sdx = p.sun[0] + (p.sun_tangent[0] * cs + p.sun_bitangent[0] * sn) * radius;
                            float sdy = p.sun[1] + (p.sun_tangent[1] * cs + p.sun_bitangent[1] * sn) * radius;
                            float sdz = p.sun[2] + (p.sun_tangent[2] * cs + p.sun_bitangent[2] * sn) * radius;
                            normalize3(sdx, sdy, sdz);
                            if (walk_init(w.d, ro, KIND_ANY, p, sox, soy, soz, sdx, sdy, sdz,
                                          p.shadow_max_dist, k)) {
                                shadow_phase = true;
                                item = 0u;
                            } else {
                                reinterpret_cast<uint2 *>(q.shadow)[ray] = make_uint2(0u, 1u << 8);
                            }
                        }
                    }
                }
            }
        }
    }
    if (lane == 0) {
        const uint32_t warps = gridDim.x * (blockDim.x >> 5);
        if (atomicAdd(q.work + 1, 1u) == warps - 1u) {
            q.work[0] = 0u;
            q.work[1] = 0u;
        }
    }
}

// ---- coherence reorder: 16-bit key = kind(2) | origin cell(6) | direction(8)

// atomicAdd(base + key, 1) for every active lane, one atomic per distinct
// key in the warp; returns this lane's slot among the lanes sharing its key
__device__ __forceinline__ uint32_t warp_count(uint32_t *base, uint32_t key) {
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, key);
    const int leader = __ffs(peers) - 1;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t off = 0;
    if ((int)lane == leader) off = atomicAdd(base + key, (uint32_t)__popc(peers));
    off = __shfl_sync(peers, off, leader);
    return off + (uint32_t)__popc(peers & ((1u << lane) - 1u));
}

__global__ void k_sort_keys(const VxRay *rays, uint32_t n, int32_t rox, int32_t roy, int32_t roz,
                            uint32_t shift, uint32_t *keys, uint32_t *hist) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float ox, oy, oz, dx, dy, dz, tmax;
    uint32_t kind;
    load_ray(rays, i, ox, oy, oz, dx, dy, dz, tmax, kind);
    // direction on a 64x64 octahedral grid (rays sharing an origin -- the
    // primaries -- then group by screen region)
    const float l1 = fabsf(dx) + fabsf(dy) + fabsf(dz);
    float u = l1 > 0.f ? dx / l1 : 0.f, v = l1 > 0.f ? dz / l1 : 0.f;
    if (dy < 0.f) {
        const float uu = (1.f - fabsf(v)) * (u < 0.f ? -1.f : 1.f);
        v = (1.f - fabsf(u)) * (v < 0.f ? -1.f : 1.f);
        u = uu;
    }
    const uint32_t qu = (uint32_t)min(63, max(0, (int32_t)((u + 1.f) * 32.f)));
    const uint32_t qv = (uint32_t)min(63, max(0, (int32_t)((v + 1.f) * 32.f)));
    // origin: which half of the window in x and in z (the window split in
    // quarters by `shift`, then halved)
    const int32_t cx = max(0, (int32_t)floorf(ox) - rox) >> shift;
    const int32_t cz = max(0, (int32_t)floorf(oz) - roz) >> shift;
    (void)roy;
    const uint32_t cell = ((uint32_t)(cx >> 1) & 1u) | (((uint32_t)(cz >> 1) & 1u) << 1);
    const uint32_t key = ((kind & 3u) << 14) | (cell << 12) | (qv << 6) | qu;
    keys[i] = key;
    warp_count(hist, key);
}

// exclusive scan of the 65536-bin histogram in one 1024-thread CTA
__global__ void __launch_bounds__(1024) k_scan_bins(uint32_t *hist) {
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x;
    const uint32_t per = kSortBins / 1024u;
    uint32_t sum = 0;
    for (uint32_t j = 0; j < per; ++j) sum += hist[t * per + j];
    part[t] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < 1024u; off <<= 1) {
        const uint32_t v = t >= off ? part[t - off] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = part[t] - sum;
    for (uint32_t j = 0; j < per; ++j) {
        const uint32_t c = hist[t * per + j];
        hist[t * per + j] = run;
        run += c;
    }
}

__global__ void k_scatter(const uint32_t *keys, uint32_t n, uint32_t *cursor, uint32_t *order) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    order[warp_count(cursor, keys[i])] = i;
}

// order-independent fingerprint of the outputs (autotuner consistency check)
__global__ void k_fingerprint(const uint32_t *a, size_t na, const uint32_t *b, size_t nb,
                              unsigned long long *out) {
    unsigned long long acc = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < na + nb;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t v = i < na ? a[i] : b[i - na];
        unsigned long long x = ((unsigned long long)v << 32) ^ (unsigned long long)(i * 0x9E3779B97F4A7C15ull);
        x ^= x >> 29;
        x *= 0xBF58476D1CE4E5B9ull;
        x ^= x >> 32;
        acc += x;
    }
    atomicAdd(out, acc);
}

template <uint32_t FL>
struct QueueK {
    static void *fn() { return reinterpret_cast<void *>(&k_queue<FL>); }
};

void *queue_kernel(uint32_t fl) { return pick_fl<QueueK>(fl); }

}  // namespace

cudaError_t QueueScratch::reserve(size_t n) {
    if (!work) {
        cudaError_t e = cudaMalloc(&work, 2 * sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMemset(work, 0, 2 * sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMalloc(&hist, kSortBins * sizeof(uint32_t));
        if (e == cudaSuccess) e = cudaMalloc(&fp, sizeof(unsigned long long));
        if (e != cudaSuccess) return e;
    }
    if (cap >= n && keys) return cudaSuccess;
    cudaFree(keys);
    cudaFree(order);
    keys = order = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&keys, std::max<size_t>(n, 1) * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&order, std::max<size_t>(n, 1) * sizeof(uint32_t));
    if (e == cudaSuccess) cap = n;
    return e;
}

void QueueScratch::release() {
    cudaFree(work);
    cudaFree(keys);
    cudaFree(order);
    cudaFree(hist);
    cudaFree(fp);
    *this = QueueScratch();
}

cudaError_t launch_queue(const TraceArgs &ta, const VxRay *rays, size_t n, VxHitRecord *out,
                         VxShadowRecord *shadow, const VxQueueTuning &t, QueueScratch &sc,
                         cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint32_t nn = (uint32_t)n;
    const uint32_t *order = nullptr;
    if (t.sort) {
        // origin cells: 4 per horizontal axis across the window
        uint32_t shift = 6;
        while (((uint32_t)std::max(ta.w.d.vx, ta.w.d.vz) >> shift) > 4u) ++shift;
        cudaError_t e = cudaMemsetAsync(sc.hist, 0, kSortBins * sizeof(uint32_t), s);
        if (e != cudaSuccess) return e;
        k_sort_keys<<<(nn + 255) / 256, 256, 0, s>>>(rays, nn, ta.ro[0], ta.ro[1], ta.ro[2], shift,
                                                     sc.keys, sc.hist);
        k_scan_bins<<<1, 1024, 0, s>>>(sc.hist);
        k_scatter<<<(nn + 255) / 256, 256, 0, s>>>(sc.keys, nn, sc.hist, sc.order);
        order = sc.order;
    }
    QueueArgs q;
    q.ta = ta;
    q.rays = rays;
    q.order = order;
    q.n = nn;
    q.out = out;
    q.shadow = shadow;
    q.work = sc.work;
    q.refill_min = (uint32_t)std::min(32, std::max(1, t.refill_min));
    void *fn = queue_kernel((ta.p.flags & 7u) | pow2_bit(ta.w.d));
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, t.block_threads, 0);
    if (e != cudaSuccess) return e;
    if (t.ctas_per_sm > 0) per_sm = std::min(per_sm, t.ctas_per_sm);
    per_sm = std::max(per_sm, 1);
    void *args[] = {&q};
    return cudaLaunchKernel(fn, dim3((unsigned)(sms * per_sm)), dim3((unsigned)t.block_threads),
                            args, 0, s);
}

cudaError_t queue_fingerprint(const VxHitRecord *out, size_t n, const VxShadowRecord *shadow,
                              QueueScratch &sc, cudaStream_t s, unsigned long long *host) {
    cudaError_t e = cudaMemsetAsync(sc.fp, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    k_fingerprint<<<296, 256, 0, s>>>(reinterpret_cast<const uint32_t *>(out), n * 6,
                                      reinterpret_cast<const uint32_t *>(shadow),
                                      shadow ? n * 2 : 0, sc.fp);
    e = cudaMemcpyAsync(host, sc.fp, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
}

}  // namespace vx
