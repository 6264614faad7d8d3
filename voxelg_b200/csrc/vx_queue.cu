// vx_queue.cu -- the mixed ray queue: rays of different kinds and very
// uneven lengths (primary with spawned shadow, GI-probe, picking, any-hit
// line-of-sight, no-water) traced by ONE persistent launch.
//
// Every lane walks one ray at a time with the shared cascade step
// (vx_walk.cuh) and takes the next queue item when its ray ends; a primary
// that hits and carries VX_RAY_SPAWN_SHADOW continues in the same lane with
// its shadow ray (raymarch.wgsl:3953-3994).  Lanes of a warp refill together
// once `refill_min` of them are idle (a lone refill would stall 31 lanes
// through a ray set-up).  Optionally the queue is first reordered by a 32-bit
// coherence key -- kind, then the direction on a 1024x1024 octahedral grid in
// Morton order, then the 64-voxel origin cell -- with a stable LSD radix sort
// (four 8-bit passes), so that a warp's rays head the same way from nearby
// origins: rays of one camera fall into pixel-sized direction cells, the
// rays of one probe site stay together.  Results do not depend on any of
// these choices; the autotuner checks that and keeps the fastest.
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

constexpr uint32_t kTileItems = 2048;   // radix sort: items per warp-tile

struct QueueArgs {
    TraceArgs ta;
    const VxRay *rays;
    const uint2 *order;       // sorted (key, ray) pairs or nullptr (identity order)
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
                    ray = q.order ? __ldg(q.order + slot).y : slot;
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

// ---- coherence reorder: stable LSD radix sort of a 32-bit key
// key = kind(2) | Morton(octahedral direction, 10+10 bits) | origin cell(10:
// 64-voxel cells, 4 bits each in x and z, 2 in y)

__device__ __forceinline__ uint32_t spread_bits(uint32_t x) {   // 10 bits -> even bits
    x &= 0x3FFu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}

__global__ void k_radix_keys(const VxRay *rays, uint32_t n, int32_t rox, int32_t roz,
                             uint2 *kv) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float ox, oy, oz, dx, dy, dz, tmax;
    uint32_t kind;
    load_ray(rays, i, ox, oy, oz, dx, dy, dz, tmax, kind);
    // direction on the octahedral map, lower hemisphere folded out
    const float l1 = fabsf(dx) + fabsf(dy) + fabsf(dz);
    float u = l1 > 0.f ? dx / l1 : 0.f, v = l1 > 0.f ? dz / l1 : 0.f;
    if (dy < 0.f) {
        const float uu = (1.f - fabsf(v)) * (u < 0.f ? -1.f : 1.f);
        v = (1.f - fabsf(u)) * (v < 0.f ? -1.f : 1.f);
        u = uu;
    }
    const uint32_t qu = (uint32_t)min(1023, max(0, (int32_t)((u + 1.f) * 512.f)));
    const uint32_t qv = (uint32_t)min(1023, max(0, (int32_t)((v + 1.f) * 512.f)));
    const uint32_t morton = spread_bits(qu) | (spread_bits(qv) << 1);
    // origin cell of 64 voxels relative to the window corner (x, z) and in y
    auto cell = [](float o, int32_t corner) -> uint32_t {
        const float f = floorf(o);
        const int32_t c = f != f ? 0 : (int32_t)fminf(fmaxf(f - (float)corner, 0.f), 1e9f);
        return ((uint32_t)c >> 6) & 15u;
    };
    const uint32_t oc = cell(ox, rox) | (cell(oz, roz) << 4) | ((cell(oy, 0) & 3u) << 8);
    kv[i] = make_uint2(((kind & 3u) << 30) | (morton << 10) | oc, i);
}

// Per warp-tile histogram of one 8-bit digit: counts[digit * tiles + tile].
__global__ void __launch_bounds__(128) k_radix_hist(const uint2 *kv, uint32_t n,
                                                    uint32_t shift, uint32_t tiles,
                                                    uint32_t *counts) {
    __shared__ uint32_t h[4][256];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    for (uint32_t d = lane; d < 256u; d += 32u) h[warp][d] = 0u;
    __syncwarp();
    const uint32_t tile = blockIdx.x * 4u + warp;
    if (tile < tiles) {
        const uint32_t end = min(n, (tile + 1u) * kTileItems);
        for (uint32_t i = tile * kTileItems + lane; i < end; i += 32u)
            atomicAdd(&h[warp][(kv[i].x >> shift) & 255u], 1u);
        __syncwarp();
        for (uint32_t d = lane; d < 256u; d += 32u) counts[d * tiles + tile] = h[warp][d];
    }
}

// Exclusive scan of the digit-major counts: first the row totals, then each
// row scanned by one 256-thread CTA from its digit's base (the totals of the
// smaller digits), 1024 entries a round, four per thread.
__device__ __forceinline__ uint32_t block_sum256(uint32_t v, uint32_t *wsum) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    __syncthreads();                       // wsum may still be read by a previous call
    if (lane == 0) wsum[warp] = v;
    __syncthreads();
    uint32_t t = 0;
#pragma unroll
    for (uint32_t w = 0; w < 8u; ++w) t += wsum[w];
    return t;
}

// row totals: one warp per digit row (its loads are independent, so one warp
// keeps many in flight; a CTA per row measured slower)
__global__ void __launch_bounds__(256) k_radix_rowsum(const uint32_t *counts, uint32_t tiles,
                                                      uint32_t *rowsum) {
    const uint32_t d = blockIdx.x * 8u + (threadIdx.x >> 5), lane = threadIdx.x & 31u;
    const uint32_t *row = counts + (size_t)d * tiles;
    uint32_t sum = 0;
    for (uint32_t t = lane; t < tiles; t += 32u) sum += row[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
    if (lane == 0) rowsum[d] = sum;
}

__global__ void __launch_bounds__(256) k_radix_rowscan(uint32_t *counts, uint32_t tiles,
                                                       const uint32_t *rowsum) {
    __shared__ uint32_t wsum[8];
    const uint32_t d = blockIdx.x, tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    uint32_t base = 0;
    for (uint32_t k = tid; k < d; k += blockDim.x) base += rowsum[k];
    base = block_sum256(base, wsum);
    uint32_t *row = counts + (size_t)d * tiles;
    for (uint32_t c0 = 0; c0 < tiles; c0 += 1024u) {
        const uint32_t t0 = c0 + tid * 4u;
        uint32_t x[4], run = 0;
#pragma unroll
        for (uint32_t i = 0; i < 4u; ++i) {
            x[i] = t0 + i < tiles ? row[t0 + i] : 0u;
            const uint32_t c = x[i];
            x[i] = run;                    // exclusive within the thread
            run += c;
        }
        uint32_t inc = run;                // inclusive scan of thread totals in the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += v;
        }
        __syncthreads();                   // wsum of the previous round is consumed
        if (lane == 31u) wsum[warp] = inc;
        __syncthreads();
        uint32_t before = 0, total = 0;
#pragma unroll
        for (uint32_t w = 0; w < 8u; ++w) {
            const uint32_t s = wsum[w];
            before += w < warp ? s : 0u;
            total += s;
        }
        const uint32_t first = base + before + inc - run;
#pragma unroll
        for (uint32_t i = 0; i < 4u; ++i)
            if (t0 + i < tiles) row[t0 + i] = first + x[i];
        base += total;
    }
}

// Stable scatter, one 2048-item tile per CTA of eight warps; warp w owns
// items [256 w, 256 w + 256) of the tile.
//   1. each warp reads its slice (8 items a lane, kept in registers) and
//      ranks every item among the slice's items of the same digit (lanes
//      sharing a digit in a round rank in lane order);
//   2. per digit, the counts of the warps give each warp's first rank and the
//      digit's total; a scan over the 256 digits gives each digit's first
//      slot in the tile;
//   3. every item moves to its slot of the tile sorted by (digit, index), in
//      shared memory;
//   4. the sorted tile is written out in slot order: slot j of digit d goes
//      to the digit's first position for this tile (the scanned counts) plus
//      j minus the digit's first slot.  Items of one digit leave as one run,
//      so stores coalesce instead of touching one sector per item.
// The order is the stable one: by tile, then by index within the tile.
constexpr uint32_t kScatterWarps = 8;
constexpr uint32_t kSliceItems = kTileItems / kScatterWarps;   // 256 = 8 rounds of 32
__global__ void __launch_bounds__(32 * kScatterWarps) k_radix_scatter(
    const uint2 *in, uint32_t n, uint32_t shift, uint32_t tiles, const uint32_t *counts,
    uint2 *out) {
    __shared__ __align__(16) uint2 st[kTileItems];
    __shared__ uint32_t wrank[kScatterWarps][256];   // per warp and digit: count, then first rank
    __shared__ uint32_t dfirst[256];                 // first slot of each digit in the tile
    __shared__ uint32_t gbase[256];                  // first output position of each digit
    __shared__ uint32_t wtot[kScatterWarps];
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t tile = blockIdx.x;
    const uint32_t begin = tile * kTileItems, end = min(n, begin + kTileItems);
    const uint32_t cnt = end - begin;
    for (uint32_t i = tid; i < kScatterWarps * 256u; i += blockDim.x) (&wrank[0][0])[i] = 0u;
    __syncthreads();
    // 1. rank within the warp's slice
    const uint32_t s0 = warp * kSliceItems;
    uint2 v[8];
    uint32_t rk[8];
#pragma unroll
    for (uint32_t k = 0; k < 8u; ++k) {
        const uint32_t i = s0 + k * 32u + lane;
        const unsigned valid = __ballot_sync(0xFFFFFFFFu, i < cnt);
        v[k] = make_uint2(0u, 0u);
        rk[k] = 0u;
        if (i < cnt) {
            v[k] = in[begin + i];
            const uint32_t dg = (v[k].x >> shift) & 255u;
            const unsigned peers = __match_any_sync(valid, dg);
            rk[k] = wrank[warp][dg] + (uint32_t)__popc(peers & ((1u << lane) - 1u));
            __syncwarp(valid);
            if ((uint32_t)(__ffs(peers) - 1) == lane) wrank[warp][dg] += (uint32_t)__popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    // 2. per digit (one thread each): warps' first ranks, the digit's total,
    //    then an exclusive scan of the totals over the digits
    const uint32_t d = tid;                          // blockDim.x == 256
    uint32_t tot = 0;
#pragma unroll
    for (uint32_t w = 0; w < kScatterWarps; ++w) {
        const uint32_t c = wrank[w][d];
        wrank[w][d] = tot;
        tot += c;
    }
    gbase[d] = counts[d * tiles + tile];
    uint32_t inc = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if ((int)lane >= o) inc += t;
    }
    if (lane == 31u) wtot[warp] = inc;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t w = 0; w < warp; ++w) before += wtot[w];
    dfirst[d] = before + inc - tot;
    __syncthreads();
    // 3. each item to its slot of the sorted tile
#pragma unroll
    for (uint32_t k = 0; k < 8u; ++k) {
        const uint32_t i = s0 + k * 32u + lane;
        if (i < cnt) {
            const uint32_t dg = (v[k].x >> shift) & 255u;
            st[dfirst[dg] + wrank[warp][dg] + rk[k]] = v[k];
        }
    }
    __syncthreads();
    // 4. slot order out: runs of one digit go to consecutive positions
    for (uint32_t j = tid; j < cnt; j += blockDim.x) {
        const uint2 item = st[j];
        const uint32_t dg = (item.x >> shift) & 255u;
        out[gbase[dg] + (j - dfirst[dg])] = item;
    }
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
        if (e == cudaSuccess) e = cudaMalloc(&fp, sizeof(unsigned long long));
        if (e != cudaSuccess) return e;
    }
    if (cap >= n && kv) return cudaSuccess;
    cudaFree(kv);
    cudaFree(kv2);
    cudaFree(hist);
    kv = kv2 = nullptr;
    hist = nullptr;
    cap = 0;
    const size_t m = std::max<size_t>(n, 1);
    const size_t tiles = (m + kTileItems - 1) / kTileItems;
    cudaError_t e = cudaMalloc(&kv, m * sizeof(uint2));
    if (e == cudaSuccess) e = cudaMalloc(&kv2, m * sizeof(uint2));
    if (e == cudaSuccess) e = cudaMalloc(&hist, (tiles + 1) * 256 * sizeof(uint32_t));
    if (e == cudaSuccess) cap = n;
    return e;
}

void QueueScratch::release() {
    cudaFree(work);
    cudaFree(kv);
    cudaFree(kv2);
    cudaFree(hist);
    cudaFree(fp);
    *this = QueueScratch();
}

cudaError_t launch_queue(const TraceArgs &ta, const VxRay *rays, size_t n, VxHitRecord *out,
                         VxShadowRecord *shadow, const VxQueueTuning &t, QueueScratch &sc,
                         cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint32_t nn = (uint32_t)n;
    const uint2 *order = nullptr;
    if (t.sort) {
        const uint32_t tiles = (nn + kTileItems - 1) / kTileItems;
        const unsigned tb = (tiles + 3) / 4;
        k_radix_keys<<<(nn + 255) / 256, 256, 0, s>>>(rays, nn, ta.ro[0], ta.ro[2], sc.kv);
        uint2 *in = sc.kv, *out = sc.kv2;
        for (uint32_t shift = 0; shift < 32u; shift += 8u) {
            k_radix_hist<<<tb, 128, 0, s>>>(in, nn, shift, tiles, sc.hist);
            k_radix_rowsum<<<32, 256, 0, s>>>(sc.hist, tiles, sc.hist + (size_t)tiles * 256u);
            k_radix_rowscan<<<256, 256, 0, s>>>(sc.hist, tiles, sc.hist + (size_t)tiles * 256u);
            k_radix_scatter<<<tiles, 32 * kScatterWarps, 0, s>>>(in, nn, shift, tiles, sc.hist,
                                                                 out);
            std::swap(in, out);
        }
        order = in;
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
