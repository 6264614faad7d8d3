// vx_trace.cu -- sm_100a traversal kernels: beam pre-pass, primary trace
// (+ shadow any-hit), batched generic rays and the flat picking DDA.
//
// The method is the reference's, restated for the GPU:
//   dda_init            shaders/raymarch.wgsl:3369-3411
//   dda_step            shaders/raymarch.wgsl:3416-3448
//   skip_to_cell        shaders/raymarch.wgsl:4807-4864
//   trace               shaders/raymarch.wgsl:4600-4777
//   trace_any           shaders/raymarch.wgsl:4345-4409
//   trace_no_water      shaders/raymarch.wgsl:3450-3532
//   trace_first_tile    shaders/beam.wgsl:51-113
//   cs_main traversal   shaders/raymarch.wgsl:576-631
//   raycast (picking)   src/raycast.rs:21-133
//
// Bit-exactness: this file is compiled with --fmad=false -prec-div=true
// -prec-sqrt=true -ftz=false, so every float operation is one IEEE binary32
// operation in the reference's order.  min/max/normalize/f32->i32 follow the
// conventions listed in the library's design notes (the WGSL leaves them
// implementation-defined); the CPU oracle uses the same ones.
//
// GPU structure: one thread per ray; every ray state component lives in a
// named register (no dynamic array indexing, so nothing spills to local
// memory); the pyramid loads of one iteration are issued together -- the L4,
// chunk and tile words and the tile LUT byte are all addressed by the slot
// coordinate, so they leave as one batch and the level cascade then runs on
// registers.  Brick occupancy + brick LUT form the second batch, the material
// byte the third (only on a solid voxel).
#include <cuda_runtime.h>

#include <climits>

#include "vx_internal.h"
#include "vx_walk.cuh"

namespace vx {
namespace {

// ------------------------------------------------------------------ beam
// Chunk masks staged in shared memory for the beam walk when they fit.
// 40 KB keeps dynamic plus static shared memory under the default 48 KB.
constexpr uint32_t kBeamSmemBytes = 40u * 1024u;
constexpr uint32_t kWaitLimit = 1u << 20;   // mbarrier polls before giving up

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0u;
}

// chunk word ci of the shared-memory copy of the chunk masks (checked like
// ld_chunk in the checked library)
__device__ __forceinline__ uint64_t s_chunk_at(const DevWorld &w, const uint64_t *s, uint32_t ci) {
    return index_ok(w, ci, w.d.n_chunks, ARR_CHUNK) ? s[ci] : 0ull;
}

// cs_beam + trace_first_tile, beam.wgsl:30-113 (world, non-rebased coords).
// SMEM: the whole chunk-mask array is brought into shared memory by one bulk
// TMA copy (cp.async.bulk completing on an mbarrier) before the walk, so each
// of the up to 80 dependent steps reads shared memory.  The wait is bounded:
// on a timeout the CTA reads global memory instead (same values, same
// records) and waits, again bounded, for the copy to land before it exits.
template <bool STATS, bool SMEM>
__global__ void __launch_bounds__(128) k_beam(FrameArgs fa, float *beam_out) {
    extern __shared__ __align__(16) uint64_t s_chunk[];
    __shared__ __align__(8) uint64_t s_bar;
    const Dims &d = fa.ta.w.d;
    bool staged = false;
    uint32_t bar = 0;
    if (SMEM) {
        bar = (uint32_t)__cvta_generic_to_shared(&s_bar);
        const uint32_t bytes = (uint32_t)d.n_chunks * 8u;  // launcher: 16-byte multiple
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                         "r"(bytes)
                         : "memory");
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], "
                "%2, [%3];" ::"r"((uint32_t)__cvta_generic_to_shared(s_chunk)),
                "l"(fa.ta.w.chunk_mask), "r"(bytes), "r"(bar)
                : "memory");
        }
        for (uint32_t it = 0; it < kWaitLimit && !staged; ++it) staged = mbar_try_wait(bar, 0u);
    }
    const uint32_t gx = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gy = blockIdx.y;
    if (gx < fa.bw && gy < fa.bh) {
        const VxCamera &c = fa.cam;
        uint64_t bytes = 0, iters = 0;
        float dx, dy, dz;
        ray_dir_uv(c, ((float)gx * 8.0f + 4.0f) / c.res_x, ((float)gy * 8.0f + 4.0f) / c.res_y,
                   dx, dy, dz);
        float result = 1e9f;
        const float ix = safe_inv(dx), iy = safe_inv(dy), iz = safe_inv(dz);
        const float wminx = (float)c.world_origin[0], wminy = (float)c.world_origin[1],
                    wminz = (float)c.world_origin[2];
        const float wmaxx = wminx + (float)d.vx, wmaxy = wminy + (float)d.vy,
                    wmaxz = wminz + (float)d.vz;
        const float t0x = (wminx - c.origin[0]) * ix, t1x = (wmaxx - c.origin[0]) * ix;
        const float t0y = (wminy - c.origin[1]) * iy, t1y = (wmaxy - c.origin[1]) * iy;
        const float t0z = (wminz - c.origin[2]) * iz, t1z = (wmaxz - c.origin[2]) * iz;
        const float t_enter =
            vmax(vmax(vmin(t0x, t1x), vmin(t0y, t1y)), vmax(vmin(t0z, t1z), 0.0f));
        const float t_exit = vmin(vmin(vmax(t0x, t1x), vmax(t0y, t1y)), vmax(t0z, t1z));
        if (!(t_enter >= t_exit || t_exit < 0.0f)) {
            const float tb = t_enter + 0.05f;
            const float px = clampf(c.origin[0] + dx * tb, wminx + 0.01f, wmaxx - 0.01f);
            const float py = clampf(c.origin[1] + dy * tb, wminy + 0.01f, wmaxy - 0.01f);
            const float pz = clampf(c.origin[2] + dz * tb, wminz + 0.01f, wmaxz - 0.01f);
            int32_t tx = f2i(floorf(px / 16.0f)), ty = f2i(floorf(py / 16.0f)),
                    tz = f2i(floorf(pz / 16.0f));
            const int32_t sx = sgn(dx), sy = sgn(dy), sz = sgn(dz);
            const float tdx = fabsf(ix) * 16.0f, tdy = fabsf(iy) * 16.0f, tdz = fabsf(iz) * 16.0f;
            float mx = sx > 0 ? ((float)((tx + 1) * 16) - c.origin[0]) * ix
                              : ((float)(tx * 16) - c.origin[0]) * ix;
            float my = sy > 0 ? ((float)((ty + 1) * 16) - c.origin[1]) * iy
                              : ((float)(ty * 16) - c.origin[1]) * iy;
            float mz = sz > 0 ? ((float)((tz + 1) * 16) - c.origin[2]) * iz
                              : ((float)(tz * 16) - c.origin[2]) * iz;
            const int32_t otx = c.world_origin[0] / 16, oty = c.world_origin[1] / 16,
                          otz = c.world_origin[2] / 16;
            // slot of window tile 0; inside the window the slot of tile t is
            // (t - ot) + slot0, folded once (== pos_mod(t, tiles))
            const uint32_t sox = (uint32_t)pos_mod(otx, d.tx), soz = (uint32_t)pos_mod(otz, d.tz);
            float t_cur = t_enter;
            for (int s = 0; s < 80; ++s) {
                ++iters;
                const uint32_t rx = (uint32_t)(tx - otx), rz = (uint32_t)(tz - otz);
                if (rx >= (uint32_t)d.tx || (uint32_t)(ty - oty) >= (uint32_t)d.ty ||
                    rz >= (uint32_t)d.tz)
                    break;
                uint32_t stx = rx + sox, stz = rz + soz;
                if (stx >= (uint32_t)d.tx) stx -= (uint32_t)d.tx;
                if (stz >= (uint32_t)d.tz) stz -= (uint32_t)d.tz;
                const uint32_t sty = (uint32_t)ty;
                const uint32_t ci = (stx >> 2) + (sty >> 2) * (uint32_t)d.cx +
                                    (stz >> 2) * (uint32_t)(d.cx * d.cy);
                const int lin = (int)((stx & 3u) + (stz & 3u) * 4u + (sty & 3u) * 16u);
                if (STATS) bytes += 8;
                const uint64_t cw = (SMEM && staged) ? s_chunk_at(fa.ta.w, s_chunk, ci)
                                                     : ld_chunk(fa.ta.w, ci);
                if (bit64(cw, lin)) {
                    result = t_cur;
                    break;
                }
                if (mx < my && mx < mz) {
                    tx += sx; t_cur = mx; mx = mx + tdx;
                } else if (my < mz) {
                    ty += sy; t_cur = my; my = my + tdy;
                } else {
                    tz += sz; t_cur = mz; mz = mz + tdz;
                }
            }
        }
        beam_out[(size_t)gy * fa.bw + gx] = result;
        if (STATS) flush_stats(fa.stats, bytes, iters);
    }
    if (SMEM && !staged) {
        // the copy still targets this CTA's shared memory: let it land (bounded)
        bool done = false;
        for (uint32_t it = 0; it < kWaitLimit && !done; ++it) done = mbar_try_wait(bar, 0u);
        // still in flight: the CTA exits anyway (no unbounded wait), and the
        // host learns of it through the world's fault word (VX_ERR_DEVICE at
        // the next synchronising call); SMEM launches always have one
        if (!done) *reinterpret_cast<volatile uint32_t *>(fa.ta.w.fault) = kFaultBeamCopyLost;
    }
}

// cs_main's temporal-differential gate (raymarch.wgsl:580-587): is the 8x8
// screen tile of this pixel marked dirty?
__device__ __forceinline__ bool tile_dirty(const FrameArgs &fa, uint32_t px, uint32_t py) {
    const uint32_t ti = (py >> 3) * ((fa.W + 7u) >> 3) + (px >> 3);
    return (__ldg(fa.tile_gate + (ti >> 5)) >> (ti & 31u)) & 1u;
}

// ------------------------------------------------------------- primary
// Per-pixel work of cs_main's traversal part (raymarch.wgsl:576-631): ray
// through the pixel centre, beam fast-forward, trace, t re-based to the
// camera, then one shadow any-hit ray from the hit (raymarch.wgsl:3953-3994).
template <uint32_t FL, bool STATS>
__device__ __forceinline__ void primary_pixel(const FrameArgs &fa, uint32_t px, uint32_t py,
                                              uint64_t &bytes, uint64_t &iters) {
    const VxCamera &c = fa.cam;
    const VxTraceParams &p = fa.ta.p;
    const Ro ro{fa.ta.ro[0], fa.ta.ro[1], fa.ta.ro[2]};
    float dx, dy, dz;
    const float u = (((float)px + 0.5f) + c.jitter_x) / c.res_x;
    const float v = (((float)py + 0.5f) + c.jitter_y) / c.res_y;
    ray_dir_uv(c, u, v, dx, dy, dz);
    float ox = c.origin[0], oy = c.origin[1], oz = c.origin[2];
    float skip = 0.0f;
    const bool beam_on = (p.flags & VX_F_BEAM) != 0u;
    if (beam_on) {
        const float bt = fa.beam[(size_t)(py >> 3) * fa.bw + (px >> 3)];
        skip = vmax(0.0f, bt - p.beam_margin);
        ox = c.origin[0] + dx * skip;
        oy = c.origin[1] + dy * skip;
        oz = c.origin[2] + dz * skip;
    }
    Hit h;
    trace_ray<FL, STATS>(fa.ta.w, p, ro, ox, oy, oz, dx, dy, dz, p.max_dist, h, bytes);
    if (beam_on && (h.flags & 1u)) h.t = h.t + skip;
    const size_t idx = (size_t)py * fa.W + px;
    store_record(fa.rec + idx, h);
    iters += h.steps;
    if (fa.shadow) {
        uint32_t ssteps = 0, occ = 0, traced = 0;
        if ((p.flags & VX_F_SHADOW) && (h.flags & 1u)) {
            // p_off = p_hit + n*0.001; golden-angle jitter in the sun cone
            const int ax = (int)(h.face >> 1);
            const float nv = (h.face & 1u) ? -1.0f : 1.0f;
            const float sox = (c.origin[0] + dx * h.t) + (ax == 0 ? nv : 0.0f) * 0.001f;
            const float soy = (c.origin[1] + dy * h.t) + (ax == 1 ? nv : 0.0f) * 0.001f;
            const float soz = (c.origin[2] + dz * h.t) + (ax == 2 ? nv : 0.0f) * 0.001f;
            const float jit = ign((float)px, (float)py, p.frame);
            const float theta = jit * 2.39996323f;
            const float radius = p.cone_tan * sqrtf(jit);
            float sn, cs;
            sincos_series(theta, sn, cs);
            float sdx = p.sun[0] + (p.sun_tangent[0] * cs + p.sun_bitangent[0] * sn) * radius;
            float sdy = p.sun[1] + (p.sun_tangent[1] * cs + p.sun_bitangent[1] * sn) * radius;
            float sdz = p.sun[2] + (p.sun_tangent[2] * cs + p.sun_bitangent[2] * sn) * radius;
            normalize3(sdx, sdy, sdz);
            occ = trace_any_ray<FL, STATS>(fa.ta.w, p, ro, sox, soy, soz, sdx, sdy, sdz,
                                       p.shadow_max_dist, ssteps, bytes) ? 1u : 0u;
            traced = 1u;
            iters += ssteps;
        }
        reinterpret_cast<uint2 *>(fa.shadow)[idx] = make_uint2(ssteps, occ | (traced << 8));
    }
}

// Grid form: one thread per pixel; a warp covers an 8x4 pixel tile, a
// 128-thread CTA a 16x8 region, so a warp's rays share one beam cell.
template <uint32_t FL, bool STATS>
__global__ void VX_FRAME_BOUNDS k_primary(FrameArgs fa) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t px = blockIdx.x * 16u + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t py = fa.y0 + blockIdx.y * 8u + (warp >> 1) * 4u + (lane >> 3);
    if (px >= fa.W || py >= fa.y1) return;
    if (fa.tile_gate && !tile_dirty(fa, px, py)) return;  // raymarch.wgsl:580-587
    uint64_t bytes = 0, iters = 0;
    primary_pixel<FL, STATS>(fa, px, py, bytes, iters);
    if (STATS) flush_stats(fa.stats, bytes, iters);
}

// Persistent form with per-lane refill: one wave of CTAs; every lane walks
// one ray at a time and, the moment its ray ends, takes the next one -- its
// own shadow ray after a primary hit, else the next pixel -- so no lane of a
// warp idles while the others finish long rays.  Pixels are handed out in
// 8x4 tiles (32 consecutive work items) so that lanes start coherent; a
// warp-aggregated atomic on work[0] hands out items.  The last warp out
// resets both counters (next item, warps done) for the next launch.
template <uint32_t FL, bool STATS>
__global__ void VX_FRAME_BOUNDS k_primary_refill(FrameArgs fa) {
    constexpr uint32_t FULL = 0xFFFFFFFFu, IDLE = 0xFFFFFFFFu, DONE = 0xFFFFFFFEu;
    const uint32_t lane = threadIdx.x & 31u;
    const DevWorld &w = fa.ta.w;
    const Ro ro{fa.ta.ro[0], fa.ta.ro[1], fa.ta.ro[2]};
    const Geo g = geo_of<FL>(w.d, ro);
    const VxTraceParams &p = fa.ta.p;
    const VxCamera &c = fa.cam;
    const bool beam_on = (p.flags & VX_F_BEAM) != 0u;
    const bool shadows_on = fa.shadow != nullptr && (p.flags & VX_F_SHADOW) != 0u;
    const uint32_t tiles_x = (fa.W + 7u) / 8u;
    const uint32_t total = tiles_x * ((fa.H + 3u) / 4u) * 32u;
    uint64_t bytes = 0, iters_acc = 0;
    Walk k;
    Hit h;
    uint32_t item = IDLE, px = 0, py = 0;
    float skip = 0.0f;
    for (;;) {
        const bool need = item == IDLE;
        const unsigned ask = __ballot_sync(FULL, need);
        // refill in batches: a lane's set-up runs while the rest of the warp
        // waits, so wait until enough lanes are idle (or no lane is walking)
        const unsigned busy = __ballot_sync(FULL, item < DONE);
        if (ask && ((uint32_t)__popc(ask) >= VX_REFILL_MIN || busy == 0u)) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(fa.work, (uint32_t)__popc(ask));
            base = __shfl_sync(FULL, base, 0);
            if (need) {
                const uint32_t idx = base + (uint32_t)__popc(ask & ((1u << lane) - 1u));
                if (idx >= total) {
                    item = DONE;
                } else {
                    const uint32_t tile = idx >> 5, in = idx & 31u;
                    px = (tile % tiles_x) * 8u + (in & 7u);
                    py = (tile / tiles_x) * 4u + (in >> 3);
                    if (px < fa.W && py < fa.H && (!fa.tile_gate || tile_dirty(fa, px, py))) {
                        item = idx;
                        float dx, dy, dz;
                        const float u = (((float)px + 0.5f) + c.jitter_x) / c.res_x;
                        const float v = (((float)py + 0.5f) + c.jitter_y) / c.res_y;
                        ray_dir_uv(c, u, v, dx, dy, dz);
                        float ox = c.origin[0], oy = c.origin[1], oz = c.origin[2];
                        skip = 0.0f;
                        if (beam_on) {
                            const float bt = fa.beam[(size_t)(py >> 3) * fa.bw + (px >> 3)];
                            skip = vmax(0.0f, bt - p.beam_margin);
                            ox = c.origin[0] + dx * skip;
                            oy = c.origin[1] + dy * skip;
                            oz = c.origin[2] + dz * skip;
                        }
                        set_miss(h);
                        if (!walk_init(w.d, ro, KIND_TRACE, p, ox, oy, oz, dx, dy, dz,
                                       p.max_dist, k)) {
                            // misses the window: empty record, no shadow ray
                            h.steps = 0;
                            const size_t pi = (size_t)py * fa.W + px;
                            store_record(fa.rec + pi, h);
                            if (fa.shadow) reinterpret_cast<uint2 *>(fa.shadow)[pi] = make_uint2(0u, 0u);
                            item = IDLE;
                        }
                    }
                    // else: a pad item beyond the frame edge; stays IDLE
                }
            }
        }
        if (__all_sync(FULL, item == DONE)) break;
        if (item < DONE) {
            const int r = walk_step<FL, STATS, -1>(w, g, p, ro, k, h, bytes);
            if (r != WALK_CONT) {
                const size_t pi = (size_t)py * fa.W + px;
                iters_acc += k.iters;
                if (k.kind == KIND_TRACE) {
                    h.steps = k.iters;
                    if (r == WALK_HIT && beam_on) h.t = h.t + skip;
                    store_record(fa.rec + pi, h);
                    item = IDLE;
                    if (r == WALK_HIT && shadows_on) {
                        // raymarch.wgsl:3953-3994: p_off = p_hit + n*0.001, cone jitter
                        const int ax = (int)(h.face >> 1);
                        const float nv = (h.face & 1u) ? -1.0f : 1.0f;
                        const float sox = (c.origin[0] + k.s.dx * h.t) + (ax == 0 ? nv : 0.0f) * 0.001f;
                        const float soy = (c.origin[1] + k.s.dy * h.t) + (ax == 1 ? nv : 0.0f) * 0.001f;
                        const float soz = (c.origin[2] + k.s.dz * h.t) + (ax == 2 ? nv : 0.0f) * 0.001f;
                        const float jit = ign((float)px, (float)py, p.frame);
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
                            item = 0u;  // keep walking: the shadow ray of this pixel
                        } else {
                            reinterpret_cast<uint2 *>(fa.shadow)[pi] = make_uint2(0u, 1u << 8);
                        }
                    } else if (fa.shadow) {
                        reinterpret_cast<uint2 *>(fa.shadow)[pi] = make_uint2(0u, 0u);
                    }
                } else {
                    reinterpret_cast<uint2 *>(fa.shadow)[pi] =
                        make_uint2(k.iters, (r == WALK_HIT ? 1u : 0u) | (1u << 8));
                    item = IDLE;
                }
            }
        }
    }
    if (lane == 0) {
        const uint32_t warps = gridDim.x * (blockDim.x >> 5);
        if (atomicAdd(fa.work + 1, 1u) == warps - 1u) {
            fa.work[0] = 0u;
            fa.work[1] = 0u;
        }
    }
    if (STATS) flush_stats(fa.stats, bytes, iters_acc);
}

// --------------------------------------------------------- generic rays
template <uint32_t FL>
__global__ void __launch_bounds__(128) k_trace_rays(TraceArgs ta, const VxRay *__restrict__ rays,
                                                    size_t n, VxHitRecord *out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(reinterpret_cast<const float4 *>(rays + i));
    const float4 b = __ldg(reinterpret_cast<const float4 *>(rays + i) + 1);
    // kind in the low two bits (1 any hit, 2 no water, else trace); the
    // queue's spawn bit and other high bits are ignored here, as in the queue
    const uint32_t kind = __float_as_uint(b.w) & 3u;
    const Ro ro{ta.ro[0], ta.ro[1], ta.ro[2]};
    uint64_t bytes = 0;
    Hit h;
    if (kind == 1u) {
        uint32_t steps;
        const bool occ = trace_any_ray<FL, false>(ta.w, ta.p, ro, a.x, a.y, a.z, a.w, b.x, b.y, b.z,
                                              steps, bytes);
        set_miss(h);
        h.flags = occ ? 1u : 0u;
        h.steps = steps;
    } else if (kind == 2u) {
        trace_no_water_ray<FL, false>(ta.w, ta.p, ro, a.x, a.y, a.z, a.w, b.x, b.y, b.z, h, bytes);
    } else {
        trace_ray<FL, false>(ta.w, ta.p, ro, a.x, a.y, a.z, a.w, b.x, b.y, b.z, h, bytes);
    }
    store_record(out + i, h);
}

// ------------------------------------------------------------- picking
// raycast(), src/raycast.rs:21-133: flat per-voxel DDA in world coords with
// toroidal folding, phase 1 leaves solids the origin is inside, phase 2
// returns the first solid non-fringe voxel and its entry normal.
struct PickArgs {
    DevWorld w;
    int32_t origin[3];
    float ray[6];   // single calls: camera and direction, when cams is null
};

__device__ __forceinline__ bool o1_in_window(const Dims &d, const int32_t v[3],
                                             const int32_t o[3]) {
    return (uint32_t)(v[0] - o[0]) < (uint32_t)d.vx && (uint32_t)(v[1] - o[1]) < (uint32_t)d.vy &&
           (uint32_t)(v[2] - o[2]) < (uint32_t)d.vz;
}

__device__ __forceinline__ bool o1_in_solid(const DevWorld &w, const int32_t v[3],
                                            const int32_t o[3]) {
    const Dims &d = w.d;
    if (!o1_in_window(d, v, o)) return false;
    const int32_t sx = pos_mod(v[0], d.vx), sy = v[1], sz = pos_mod(v[2], d.vz);
    const int64_t bi = (int64_t)(sx >> 2) + (int64_t)(sy >> 2) * d.bx +
                       (int64_t)(sz >> 2) * d.bx * d.by;
    const uint64_t occ = ld_occ(w, (uint64_t)bi);
    if (occ == 0ull) return false;
    const int vi = child_bit(sx & 3, sy & 3, sz & 3);
    if (!bit64(occ, vi)) return false;
    return ld_mat(w, (uint64_t)bi, (uint32_t)vi) != 33u;
}

// The walk of raycast(): direction normalised as glam 0.29.3's
// normalize_or_zero (self * (1 / sqrt(dot))), window clip, start voxel
// (raycast.rs:21-90).  False when the ray has no walk (zero direction,
// misses the window).
struct O1State {
    int32_t voxel[3], step[3];
    float tdel[3], tm[3];
};

__device__ __forceinline__ bool o1_start(const Dims &d, const int32_t o[3], const float cam[3],
                                         const float din[3], O1State &s) {
    const float len = sqrtf((din[0] * din[0] + din[1] * din[1]) + din[2] * din[2]);
    const float rcp = 1.0f / len;
    if (!(isfinite(rcp) && rcp > 0.0f)) return false;
    const float dir[3] = {din[0] * rcp, din[1] * rcp, din[2] * rcp};
    if (dir[0] == 0.0f && dir[1] == 0.0f && dir[2] == 0.0f) return false;
    const float dims[3] = {(float)d.vx, (float)d.vy, (float)d.vz};
    float wmin[3], wmax[3], inv[3], tmn[3], tmx[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        wmin[k] = (float)o[k];
        wmax[k] = wmin[k] + dims[k];
        inv[k] = safe_inv(dir[k]);
        const float t0 = (wmin[k] - cam[k]) * inv[k];
        const float t1 = (wmax[k] - cam[k]) * inv[k];
        tmn[k] = vmin(t0, t1);
        tmx[k] = vmax(t0, t1);
    }
    const float t_enter = vmax(vmax(tmn[0], vmax(tmn[1], tmn[2])), 0.0f);
    const float t_exit = vmin(tmx[0], vmin(tmx[1], tmx[2]));
    if (t_enter >= t_exit || t_exit < 0.0f) return false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float pk = cam[k] + dir[k] * (t_enter + 1e-3f);
        pk = vmin(vmax(pk, wmin[k] + 1e-3f), wmax[k] - 1e-3f);
        s.voxel[k] = f2i(floorf(pk));
        s.step[k] = sgn(dir[k]);
        s.tdel[k] = fabsf(inv[k]);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float nxt = s.step[k] > 0 ? (float)(s.voxel[k] + 1) : (float)s.voxel[k];
        s.tm[k] = (nxt - cam[k]) * inv[k];
    }
    return true;
}

// argmin_step, raycast.rs:92-103 (ties go to the lowest axis); -1: no axis
__device__ __forceinline__ int o1_argmin_step(O1State &s) {
    int a = -1;
    float m = __int_as_float(0x7f800000);
    if (s.step[0] != 0 && s.tm[0] < m) { a = 0; m = s.tm[0]; }
    if (s.step[1] != 0 && s.tm[1] < m) { a = 1; m = s.tm[1]; }
    if (s.step[2] != 0 && s.tm[2] < m) { a = 2; m = s.tm[2]; }
    if (a == 0) { s.voxel[0] += s.step[0]; s.tm[0] += s.tdel[0]; }
    else if (a == 1) { s.voxel[1] += s.step[1]; s.tm[1] += s.tdel[1]; }
    else if (a == 2) { s.voxel[2] += s.step[2]; s.tm[2] += s.tdel[2]; }
    return a;
}

__device__ __forceinline__ void o1_normal(const O1State &s, int last_axis, VxPickHit &res) {
    const int sa = last_axis == 0 ? s.step[0] : (last_axis == 1 ? s.step[1] : s.step[2]);
    if (last_axis == 0) res.normal[0] = -sa;
    else if (last_axis == 1) res.normal[1] = -sa;
    else if (last_axis == 2) res.normal[2] = -sa;
}

__global__ void __launch_bounds__(128) k_raycast(PickArgs pa, const float *__restrict__ cams,
                                                 const float *__restrict__ dirs, size_t n,
                                                 VxPickHit *out, int32_t *hit) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Dims &d = pa.w.d;
    const int32_t *o = pa.origin;
    VxPickHit res;
    res.voxel[0] = res.voxel[1] = res.voxel[2] = 0;
    res.normal[0] = res.normal[1] = res.normal[2] = 0;
    int32_t found = 0;
    const float cam[3] = {cams[3 * i], cams[3 * i + 1], cams[3 * i + 2]};
    const float din[3] = {dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]};
    O1State s;
    do {
        if (!o1_start(d, o, cam, din, s)) break;
        int last_axis = -1;
        int steps_left = 4096;
        bool dead = false;
        // phase 1: leave the solids the start voxel is in
        while (steps_left > 0 && o1_in_solid(pa.w, s.voxel, o)) {
            const int ax = o1_argmin_step(s);
            if (ax < 0) { dead = true; break; }
            last_axis = ax;
            steps_left--;
            if (!o1_in_window(d, s.voxel, o)) { dead = true; break; }
        }
        if (dead) break;
        // phase 2: the first solid non-fringe voxel
        while (steps_left > 0) {
            if (!o1_in_window(d, s.voxel, o)) break;
            if (o1_in_solid(pa.w, s.voxel, o)) {
                res.voxel[0] = s.voxel[0]; res.voxel[1] = s.voxel[1]; res.voxel[2] = s.voxel[2];
                o1_normal(s, last_axis, res);
                found = 1;
                break;
            }
            const int ax = o1_argmin_step(s);
            if (ax < 0) break;
            last_axis = ax;
            steps_left--;
        }
    } while (0);
    out[i] = res;
    hit[i] = found;
}

// One ray with a whole warp (the single-call pick, where one thread's chain
// of dependent voxel loads is the latency).  The voxel sequence of the walk
// depends on arithmetic only, so lane 0 emits the next 32 voxels with the
// same argmin steps, every lane tests its voxel (window, solid) at once, and
// lane 0 runs raycast.rs's two phases over the resulting bits: element k of
// the walk is examined with 4096 - k steps left, a phase-1 step is followed
// by the window test of the voxel it reaches.  At most 129 rounds.
__global__ void __launch_bounds__(32) k_raycast_warp(PickArgs pa, const float *__restrict__ cams,
                                                     const float *__restrict__ dirs, VxPickHit *out,
                                                     int32_t *hit) {
    constexpr unsigned FULL = 0xFFFFFFFFu;
    __shared__ int32_t sv[32][4];   // voxel, axis of the step into it
    const uint32_t lane = threadIdx.x;
    const Dims &d = pa.w.d;
    const int32_t *o = pa.origin;
    // a single call passes its ray in the launch parameters: no read of
    // host-mapped memory before the walk can start
    const float *rc = cams ? cams : pa.ray, *rd = cams ? dirs : pa.ray + 3;
    const float cam[3] = {rc[0], rc[1], rc[2]};
    const float din[3] = {rd[0], rd[1], rd[2]};
    VxPickHit res;
    res.voxel[0] = res.voxel[1] = res.voxel[2] = 0;
    res.normal[0] = res.normal[1] = res.normal[2] = 0;
    int32_t found = 0;
    O1State s;
    if (o1_start(d, o, cam, din, s)) {   // same on every lane
        bool alive = true;               // lane 0: the walk can still step
        int la_next = -1;                // lane 0: axis of the step into the next voxel
        int phase = 1;
        bool post_check = false, done = false;
        for (int32_t base = 0; base <= 4096 && !done; base += 32) {
            uint32_t exist = 0;
            if (lane == 0) {
                for (int j = 0; j < 32 && alive; ++j) {
                    sv[j][0] = s.voxel[0]; sv[j][1] = s.voxel[1]; sv[j][2] = s.voxel[2];
                    sv[j][3] = la_next;
                    exist |= 1u << j;
                    const int ax = o1_argmin_step(s);
                    if (ax < 0) alive = false;
                    else la_next = ax;
                }
            }
            exist = __shfl_sync(FULL, exist, 0);
            __syncwarp();
            bool inwin = false, solid = false;
            if ((exist >> lane) & 1u) {
                const int32_t v[3] = {sv[lane][0], sv[lane][1], sv[lane][2]};
                inwin = o1_in_window(d, v, o);
                solid = o1_in_solid(pa.w, v, o);
            }
            const unsigned win = __ballot_sync(FULL, inwin), sol = __ballot_sync(FULL, solid);
            if (lane == 0) {
                int j = 0;
                while (j < 32 && !done) {
                    const int32_t left = 4096 - (base + j);
                    const bool next = j + 1 < 32 ? ((exist >> (j + 1)) & 1u) != 0u : alive;
                    if (post_check) {
                        post_check = false;
                        if (!((win >> j) & 1u)) { done = true; break; }   // phase-1 step left the window
                    }
                    const bool is_solid = (sol >> j) & 1u;
                    if (phase == 1) {
                        if (left > 0 && is_solid) {
                            if (!next) { done = true; break; }
                            post_check = true;
                            ++j;
                            continue;
                        }
                        phase = 2;
                    }
                    if (left <= 0 || !((win >> j) & 1u)) { done = true; break; }
                    if (is_solid) {
                        res.voxel[0] = sv[j][0]; res.voxel[1] = sv[j][1]; res.voxel[2] = sv[j][2];
                        o1_normal(s, sv[j][3], res);
                        found = 1;
                        done = true;
                        break;
                    }
                    if (!next) { done = true; break; }
                    ++j;
                }
            }
            done = __shfl_sync(FULL, done ? 1 : 0, 0) != 0;
            __syncwarp();
        }
    }
    if (lane == 0) {
        *out = res;
        *hit = found;
    }
}

// ------------------------------------------------------- temporal gating
// project_brick_to_tiles, src/temporal.rs:16-111: one thread per dirty
// brick projects the world AABB of the brick and ORs the covered 8x8 tiles
// into the mask.  The slot -> world fold follows the toroidal window at
// camera.world_origin.
__global__ void k_project_dirty(DevWorld w, VxCamera c, const uint32_t *__restrict__ idx,
                                size_t n, uint32_t *mask) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Dims &d = w.d;
    const uint32_t bi = idx[i];
    const int32_t bx = (int32_t)(bi % (uint32_t)d.bx);
    const int32_t by = (int32_t)((bi / (uint32_t)d.bx) % (uint32_t)d.by);
    const int32_t bz = (int32_t)(bi / ((uint32_t)d.bx * (uint32_t)d.by));
    const float b0 = (float)(c.world_origin[0] + pos_mod(bx * 4 - c.world_origin[0], d.vx));
    const float b1 = (float)(by * 4);
    const float b2 = (float)(c.world_origin[2] + pos_mod(bz * 4 - c.world_origin[2], d.vz));
    const uint32_t W = (uint32_t)c.res_x, H = (uint32_t)c.res_y;
    const uint32_t tiles_w = (W + 7u) / 8u, tiles_h = (H + 7u) / 8u;
    const float aspect = (float)W / (float)H;
    const float wf = (float)W, hf = (float)H;
    int32_t min_x = INT_MAX, min_y = INT_MAX, max_x = INT_MIN, max_y = INT_MIN;
    bool any_visible = false, any_behind = false;
#pragma unroll
    for (int ci = 0; ci < 8; ++ci) {
        const float dx = (b0 + (float)(ci & 1) * 4.0f) - c.origin[0];
        const float dy = (b1 + (float)((ci >> 1) & 1) * 4.0f) - c.origin[1];
        const float dz = (b2 + (float)((ci >> 2) & 1) * 4.0f) - c.origin[2];
        const float z_cam = (dx * c.forward[0] + dy * c.forward[1]) + dz * c.forward[2];
        if (z_cam <= 0.1f) {
            any_behind = true;
            continue;
        }
        const float x_cam = (dx * c.right[0] + dy * c.right[1]) + dz * c.right[2];
        const float y_cam = (dx * c.up[0] + dy * c.up[1]) + dz * c.up[2];
        const float inv_z = 1.0f / (z_cam * c.tan_half_fov);
        const float ndc_x = (x_cam * inv_z) / aspect;
        const float ndc_y = y_cam * inv_z;
        const int32_t px = f2i((ndc_x + 1.0f) * 0.5f * wf);
        const int32_t py = f2i((1.0f - ndc_y) * 0.5f * hf);
        min_x = min(min_x, px);
        min_y = min(min_y, py);
        max_x = max(max_x, px);
        max_y = max(max_y, py);
        any_visible = true;
    }
    if (!any_visible) return;
    if (any_behind) {
        min_x = 0; min_y = 0;
        max_x = (int32_t)W - 1; max_y = (int32_t)H - 1;
    }
    if (max_x < 0 || max_y < 0 || min_x >= (int32_t)W || min_y >= (int32_t)H) return;
    const uint32_t tx0 = (uint32_t)max(min_x, 0) / 8u, ty0 = (uint32_t)max(min_y, 0) / 8u;
    const uint32_t tx1 = min((uint32_t)min(max_x, (int32_t)W - 1) / 8u, tiles_w - 1u);
    const uint32_t ty1 = min((uint32_t)min(max_y, (int32_t)H - 1) / 8u, tiles_h - 1u);
    for (uint32_t ty = ty0; ty <= ty1; ++ty)
        for (uint32_t tx = tx0; tx <= tx1; ++tx) {
            const uint32_t t = ty * tiles_w + tx;
            atomicOr(mask + (t >> 5), 1u << (t & 31u));
        }
}

// Rotating hash-scattered refresh of src/app.rs:706-725 (64-bit wrapping
// hash, as the reference's usize arithmetic on 64-bit targets).
__global__ void k_refresh_tiles(uint32_t tiles_w, uint32_t tiles_h, uint32_t spread,
                                uint32_t phase, uint32_t *mask) {
    const uint32_t ti = blockIdx.x * blockDim.x + threadIdx.x;
    if (ti >= tiles_w * tiles_h) return;
    const uint64_t tx = ti % tiles_w, ty = ti / tiles_w;
    const uint64_t h = ((tx * 73856093ull) ^ (ty * 19349663ull)) * 2654435761ull;
    if ((h >> 8) % spread == phase) atomicOr(mask + (ti >> 5), 1u << (ti & 31u));
}

// ------------------------------------------------------------------ AO
// Contact AO of primary hits: compute_ao / ao_corner / ao_occluder /
// is_voxel_solid (raymarch.wgsl:4417-4475, :297-322, skip rule :3862-3863,
// AO_DIST :4522).  1.0 for misses and skipped hits.
constexpr float kAoDist = 64.0f;

__device__ __forceinline__ bool is_leaf_block(uint32_t m) {
    return m == 14u || m == 25u || m == 26u || m == 27u;
}

// is_voxel_solid + !is_decoration_mat(voxel_material_at) at world voxel (x, y, z)
__device__ __forceinline__ bool ao_occluder(const DevWorld &w, const Geo &g, Ro ro, int32_t x,
                                            int32_t y, int32_t z) {
    const Dims &d = w.d;
    if ((uint32_t)(x - ro.x) >= (uint32_t)d.vx || (uint32_t)(y - ro.y) >= (uint32_t)d.vy ||
        (uint32_t)(z - ro.z) >= (uint32_t)d.vz)
        return false;
    const uint32_t sx = (uint32_t)pos_mod(x, d.vx), sy = (uint32_t)y,
                   sz = (uint32_t)pos_mod(z, d.vz);
    if (!bit64(ld_chunk(w, chunk_index(g, sx, sy, sz)), child_of(sx, sy, sz, 4)))
        return false;
    if (!bit64(ld_tile(w, tile_index(g, sx, sy, sz)), child_of(sx, sy, sz, 2)))
        return false;
    const uint32_t bi = brick_index(g, sx >> 2, sy >> 2, sz >> 2);
    const int vi = child_of(sx, sy, sz, 0);
    if (!bit64(ld_occ(w, bi), vi)) return false;
    return !is_decoration(ld_mat(w, bi, (uint32_t)vi));
}

// ao_corner: the two side voxels and the diagonal of one face corner
__device__ __forceinline__ float ao_corner(const DevWorld &w, const Geo &g, Ro ro, int32_t bx,
                                           int32_t by, int32_t bz, int32_t ax, int32_t ay,
                                           int32_t az, int32_t cx, int32_t cy, int32_t cz) {
    const bool s1 = ao_occluder(w, g, ro, bx + ax, by + ay, bz + az);
    const bool s2 = ao_occluder(w, g, ro, bx + cx, by + cy, bz + cz);
    const bool cd = ao_occluder(w, g, ro, bx + ax + cx, by + ay + cy, bz + az + cz);
    if (s1 && s2) return 0.35f;
    const int cnt = (int)s1 + (int)s2 + (int)cd;
    return 1.0f - (float)cnt * 0.22f;
}

// WGSL mix(a, b, t) = a * (1 - t) + b * t
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }

// one thread per pixel; origin = camera origin, dir = the pixel's ray_dir_uv
__global__ void __launch_bounds__(128) k_ao(DevWorld w, VxCamera c,
                                            const VxHitRecord *__restrict__ rec, uint32_t W,
                                            uint32_t H, float *__restrict__ ao) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t px = blockIdx.x * 16u + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t py = blockIdx.y * 8u + (warp >> 1) * 4u + (lane >> 3);
    if (px >= W || py >= H) return;
    const size_t idx = (size_t)py * W + px;
    const uint2 *q = reinterpret_cast<const uint2 *>(rec + idx);
    const uint2 q0 = q[0], q1 = q[1], q2 = q[2];
    const uint32_t face = q1.y & 0xFFu, m = (q1.y >> 8) & 0xFFu, flags = (q1.y >> 16) & 0xFFu;
    const float t = __uint_as_float(q2.x);
    float r = 1.0f;
    if ((flags & 1u) && !(t > kAoDist) && !is_leaf_block(m) && m != 33u) {
        const Ro ro{c.world_origin[0], c.world_origin[1], c.world_origin[2]};
        const Geo g = geo_of<kFlPow2>(w.d, ro);  // strides only
        float dx, dy, dz;
        const float u = (((float)px + 0.5f) + c.jitter_x) / c.res_x;
        const float v = (((float)py + 0.5f) + c.jitter_y) / c.res_y;
        ray_dir_uv(c, u, v, dx, dy, dz);
        const int32_t vx = (int32_t)q0.x, vy = (int32_t)q0.y, vz = (int32_t)q1.x;
        const float lx = (c.origin[0] + dx * t) - (float)vx;
        const float ly = (c.origin[1] + dy * t) - (float)vy;
        const float lz = (c.origin[2] + dz * t) - (float)vz;
        const int na = (int)(face >> 1);
        const int32_t nd = (face & 1u) ? -1 : 1;  // outward normal = -step
        // face axes (da, db): (y, z) on an x face, (x, z) on y, (x, y) on z
        const int32_t ax = na == 0 ? 0 : 1, ay = na == 0 ? 1 : 0, az = 0;
        const int32_t cx = 0, cy = na == 2 ? 1 : 0, cz = na == 2 ? 0 : 1;
        const float fa = na == 0 ? ly : lx, fb = na == 2 ? ly : lz;
        const int32_t bx = vx + (na == 0 ? nd : 0), by = vy + (na == 1 ? nd : 0),
                      bz = vz + (na == 2 ? nd : 0);
        const float ao00 = ao_corner(w, g, ro, bx, by, bz, -ax, -ay, -az, -cx, -cy, -cz);
        const float ao10 = ao_corner(w, g, ro, bx, by, bz, ax, ay, az, -cx, -cy, -cz);
        const float ao01 = ao_corner(w, g, ro, bx, by, bz, -ax, -ay, -az, cx, cy, cz);
        const float ao11 = ao_corner(w, g, ro, bx, by, bz, ax, ay, az, cx, cy, cz);
        const float fa_c = clampf(fa, 0.0f, 1.0f), fb_c = clampf(fb, 0.0f, 1.0f);
        r = mixf(mixf(ao00, ao10, fa_c), mixf(ao01, ao11, fa_c), fb_c);
    }
    ao[idx] = r;
}

// DevWorld::tile_meta of tile ti (layout at kMetaChunkOnly): the L4 and
// chunk tests (raymarch.wgsl:4648-4668) as trace evaluates them at any voxel
// of the tile, beside the tile LUT byte.
__global__ void k_tile_meta(DevWorld w) {
    const int64_t ti = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const Dims &d = w.d;
    if (ti >= d.n_tiles) return;
    const int32_t tx = (int32_t)(ti % d.tx);
    const int32_t ty = (int32_t)((ti / d.tx) % d.ty);
    const int32_t tz = (int32_t)(ti / ((int64_t)d.tx * d.ty));
    const int32_t cx = tx >> 2, cy = ty >> 2, cz = tz >> 2;
    const uint64_t lw =
        w.l4_mask[(cx >> 2) + (int64_t)(cy >> 2) * d.lx + (int64_t)(cz >> 2) * d.lx * d.ly];
    const uint64_t cw = w.chunk_mask[cx + (int64_t)cy * d.cx + (int64_t)cz * d.cx * d.cy];
    const bool tile_clear = !bit64(cw, child_bit(tx & 3, ty & 3, tz & 3));
    uint32_t code = 0u;
    if (lw == 0ull) code = 3u;
    else if (!bit64(lw, child_bit(cx & 3, cy & 3, cz & 3))) code = 2u;
    else if (tile_clear) code = 1u;
    // the LUT byte only where the tile LUT test ends a walk (a uniform,
    // optimisable material), so the walk tests it against 0 alone
    const uint32_t lut = w.tile_uniform[ti];
    w.tile_meta[ti] = (uint16_t)((is_uniform_optimisable(lut) ? lut : 0u) | (code << 8) |
                                 (tile_clear ? kMetaChunkOnly : 0u));
}

}  // namespace

// ------------------------------------------------------------- launchers
cudaError_t launch_tile_meta(const DevWorld &w, cudaStream_t s) {
    if (!w.tile_meta) return cudaGetLastError();
    k_tile_meta<<<(unsigned)((w.d.n_tiles + 255) / 256), 256, 0, s>>>(w);
    return cudaGetLastError();
}

cudaError_t launch_ao(const DevWorld &w, const VxCamera &cam, const VxHitRecord *rec, float *ao,
                      cudaStream_t s) {
    const uint32_t W = (uint32_t)cam.res_x, H = (uint32_t)cam.res_y;
    const dim3 grid((W + 15u) / 16u, (H + 7u) / 8u);
    k_ao<<<grid, 128, 0, s>>>(w, cam, rec, W, H, ao);
    return cudaGetLastError();
}

cudaError_t launch_project_dirty(const DevWorld &w, const VxCamera &cam, const uint32_t *idx,
                                 size_t n, uint32_t *mask, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_project_dirty<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(w, cam, idx, n, mask);
    return cudaGetLastError();
}

cudaError_t launch_refresh_tiles(uint32_t tiles_w, uint32_t tiles_h, uint32_t spread,
                                 uint32_t phase, uint32_t *mask, cudaStream_t s) {
    const uint32_t n = tiles_w * tiles_h;
    if (n == 0 || spread == 0) return cudaSuccess;
    k_refresh_tiles<<<(n + 127) / 128, 128, 0, s>>>(tiles_w, tiles_h, spread, phase, mask);
    return cudaGetLastError();
}
cudaError_t launch_beam(const FrameArgs &fa, float *beam_out, cudaStream_t s) {
    dim3 block(128), grid((fa.bw + 127) / 128, fa.bh);
    const uint64_t bytes = (uint64_t)fa.ta.w.d.n_chunks * 8u;
    // staging needs a place to report a copy that never lands (w.fault)
    const bool smem = fa.ta.w.fault != nullptr && bytes <= kBeamSmemBytes &&
                      (bytes % 16u) == 0u &&
                      (reinterpret_cast<uintptr_t>(fa.ta.w.chunk_mask) & 15u) == 0u;
    if (smem) {
        if (fa.stats) k_beam<true, true><<<grid, block, (size_t)bytes, s>>>(fa, beam_out);
        else k_beam<false, true><<<grid, block, (size_t)bytes, s>>>(fa, beam_out);
    } else {
        if (fa.stats) k_beam<true, false><<<grid, block, 0, s>>>(fa, beam_out);
        else k_beam<false, false><<<grid, block, 0, s>>>(fa, beam_out);
    }
    return cudaGetLastError();
}

// Method flags (L4 | LUT | LOD) -> the matching kernel instantiation.
template <uint32_t FL>
struct GridK {
    static void *fn() { return reinterpret_cast<void *>(&k_primary<FL, false>); }
};
template <uint32_t FL>
struct GridKStats {
    static void *fn() { return reinterpret_cast<void *>(&k_primary<FL, true>); }
};
template <uint32_t FL>
struct PersistK {
    static void *fn() { return reinterpret_cast<void *>(&k_primary_refill<FL, false>); }
};
template <uint32_t FL>
struct PersistKStats {
    static void *fn() { return reinterpret_cast<void *>(&k_primary_refill<FL, true>); }
};

cudaError_t launch_primary(const FrameArgs &fa, cudaStream_t s) {
    const uint32_t fl = (fa.ta.p.flags & 7u) | pow2_bit(fa.ta.w.d);
    FrameArgs a = fa;
    void *args[] = {&a};
    if (fa.work) {
        void *fn = fa.stats ? pick_fl<PersistKStats>(fl) : pick_fl<PersistK>(fl);
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 128, 0);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        return cudaLaunchKernel(fn, dim3((unsigned)(sms * per_sm)), dim3(128), args, 0, s);
    }
    void *fn = fa.stats ? pick_fl<GridKStats>(fl) : pick_fl<GridK>(fl);
    if (fa.y1 <= fa.y0) return cudaSuccess;
    return cudaLaunchKernel(fn, dim3((fa.W + 15) / 16, (fa.y1 - fa.y0 + 7) / 8), dim3(128), args,
                            0, s);
}

template <uint32_t FL>
struct TraceK {
    static void *fn() { return reinterpret_cast<void *>(&k_trace_rays<FL>); }
};

cudaError_t launch_trace_rays(const TraceArgs &ta, const VxRay *rays, size_t n, VxHitRecord *out,
                              cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((n + 127) / 128);
    void *fn = pick_fl<TraceK>((ta.p.flags & 7u) | pow2_bit(ta.w.d));
    TraceArgs a = ta;
    const VxRay *r = rays;
    size_t nn = n;
    VxHitRecord *o = out;
    void *args[] = {&a, &r, &nn, &o};
    return cudaLaunchKernel(fn, dim3(blocks), dim3(128), args, 0, s);
}

cudaError_t launch_raycast_one(const DevWorld &w, const int32_t origin[3], const float cam[3],
                               const float dir[3], VxPickHit *out, int32_t *hit, cudaStream_t s) {
    PickArgs pa;
    pa.w = w;
    for (int k = 0; k < 3; ++k) {
        pa.origin[k] = origin[k];
        pa.ray[k] = cam[k];
        pa.ray[3 + k] = dir[k];
    }
    k_raycast_warp<<<1, 32, 0, s>>>(pa, nullptr, nullptr, out, hit);
    return cudaGetLastError();
}

cudaError_t launch_raycast(const DevWorld &w, const int32_t origin[3], const float *cams,
                           const float *dirs, size_t n, VxPickHit *out, int32_t *hit,
                           cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    PickArgs pa;
    pa.w = w;
    pa.origin[0] = origin[0]; pa.origin[1] = origin[1]; pa.origin[2] = origin[2];
    if (n == 1) {
        k_raycast_warp<<<1, 32, 0, s>>>(pa, cams, dirs, out, hit);
        return cudaGetLastError();
    }
    const unsigned blocks = (unsigned)((n + 127) / 128);
    k_raycast<<<blocks, 128, 0, s>>>(pa, cams, dirs, n, out, hit);
    return cudaGetLastError();
}

}  // namespace vx
