// vx_walk.cuh -- device-side traversal shared by the frame, queue and
// proposal kernels: the DDA state, the reference's dda_init / dda_step /
// skip_to_cell, the level cascade of trace / trace_any / trace_no_water as
// one iteration step, ray generation and record stores.
//
// Reference lines: dda_init raymarch.wgsl:3369-3411, dda_step :3416-3448,
// skip_to_cell :4807-4864, trace :4600-4777, trace_any :4345-4409,
// trace_no_water :3450-3532, ray_dir_uv :430-438, ign :394-396,
// brick_topmost_material :253-295, common.wgsl:49-58.
//
// Include from .cu files compiled with --fmad=false -prec-div=true
// -prec-sqrt=true -ftz=false: every float operation is one IEEE binary32
// operation in the reference's order (records are bit-exact against the CPU
// restatement).
#pragma once

#include <cuda_runtime.h>

#include <climits>

#include "vx_internal.h"

namespace vx {
namespace {

// Internal template bit beside the method flags: the world's x and z voxel
// dims are powers of two, so the toroidal slot is a mask.  Launchers set it
// from the world's dims; callers never see it.
constexpr uint32_t kFlPow2 = 1u << 8;
inline uint32_t pow2_bit(const Dims &d) {
    return ((d.vx & (d.vx - 1)) == 0 && (d.vz & (d.vz - 1)) == 0) ? kFlPow2 : 0u;
}
// kernel pointer K<fl>::fn() for method flags (low 3 bits) + kFlPow2
template <template <uint32_t> class K>
void *pick_fl(uint32_t fl) {
    switch (fl & (7u | kFlPow2)) {
#define VX_FL_CASE(v) \
    case v: return K<v>::fn(); \
    case v | kFlPow2: return K<v | kFlPow2>::fn();
        VX_FL_CASE(0) VX_FL_CASE(1) VX_FL_CASE(2) VX_FL_CASE(3)
        VX_FL_CASE(4) VX_FL_CASE(5) VX_FL_CASE(6) VX_FL_CASE(7)
#undef VX_FL_CASE
        default: return nullptr;
    }
}

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ float vmin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float vmax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) {
    return vmin(vmax(x, lo), hi);
}
// f32 -> i32 toward zero, saturating (NaN -> 0), clamped to +-2^30.  The PTX
// conversion (cvt.rzi.s32.f32) already saturates and maps NaN to 0; the clamp
// narrows the range so later integer cell arithmetic cannot overflow.
__device__ __forceinline__ int32_t f2i(float x) {
    return min(max(__float2int_rz(x), -1073741824), 1073741824);
}
// common.wgsl:49-52
__device__ __forceinline__ int32_t pos_mod(int32_t a, int32_t b) {
    if (a >= 0) return a % b;
    return (b - 1) - ((-1 - a) % b);
}
// common.wgsl:55-58
__device__ __forceinline__ float safe_inv(float x) {
    return (fabsf(x) < 1e-8f) ? 1e30f : 1.0f / x;
}
__device__ __forceinline__ int32_t sgn(float x) { return x > 0.0f ? 1 : (x < 0.0f ? -1 : 0); }
__device__ __forceinline__ float fractf(float x) { return x - floorf(x); }
__device__ __forceinline__ int child_bit(int lx, int ly, int lz) { return lx + lz * 4 + ly * 16; }
__device__ __forceinline__ bool bit64(uint64_t w, int b) { return (w >> b) & 1ull; }

template <typename T>
__device__ __forceinline__ T ldg(const T *p) { return __ldg(p); }

// ------------------------------------------------------------ world loads
// Every load of a world array by the traversal goes through these.  The
// checked library (libvoxrt_checked.so, built with VX_CHECKED) first compares
// the index with the array's length.  A bad index is recorded in w.oob (array
// id << 56 | index, the first one wins) and the load returns 0 without
// reading; nothing traps, and the host reads the word (vx_world_oob).
enum : uint32_t {
    ARR_L4 = 1, ARR_CHUNK = 2, ARR_TILE = 3, ARR_TILE_META = 4, ARR_TILE_UNIFORM = 5,
    ARR_OCC = 6, ARR_BRICK_UNIFORM = 7, ARR_MAT = 8
};
// checked library: is i inside an array of n entries?  If not, record it.
__device__ __forceinline__ bool index_ok(const DevWorld &w, uint64_t i, int64_t n, uint32_t arr) {
#ifdef VX_CHECKED
    if (i < (uint64_t)n) return true;
    if (w.oob)
        atomicCAS(w.oob, 0ull, ((unsigned long long)arr << 56) | (i & ((1ull << 56) - 1ull)));
    return false;
#else
    (void)w; (void)i; (void)n; (void)arr;
    return true;
#endif
}
template <typename T>
__device__ __forceinline__ T wload(const DevWorld &w, const T *base, uint64_t i, int64_t n,
                                   uint32_t arr) {
    if (!index_ok(w, i, n, arr)) return T(0);
    return __ldg(base + i);
}
__device__ __forceinline__ uint64_t ld_l4(const DevWorld &w, uint64_t i) {
    return wload(w, w.l4_mask, i, w.d.n_l4, ARR_L4);
}
__device__ __forceinline__ uint64_t ld_chunk(const DevWorld &w, uint64_t i) {
    return wload(w, w.chunk_mask, i, w.d.n_chunks, ARR_CHUNK);
}
__device__ __forceinline__ uint64_t ld_tile(const DevWorld &w, uint64_t i) {
    return wload(w, w.tile_mask, i, w.d.n_tiles, ARR_TILE);
}
__device__ __forceinline__ uint32_t ld_tile_meta(const DevWorld &w, uint64_t i) {
    return wload(w, w.tile_meta, i, w.d.n_tiles, ARR_TILE_META);
}
__device__ __forceinline__ uint32_t ld_tile_uniform(const DevWorld &w, uint64_t i) {
    return wload(w, w.tile_uniform, i, w.d.n_tiles, ARR_TILE_UNIFORM);
}
__device__ __forceinline__ uint64_t ld_occ(const DevWorld &w, uint64_t bi) {
    return wload(w, w.occ, bi, w.d.n_bricks, ARR_OCC);
}
__device__ __forceinline__ uint32_t ld_brick_uniform(const DevWorld &w, uint64_t bi) {
    return wload(w, w.brick_uniform, bi, w.d.n_bricks, ARR_BRICK_UNIFORM);
}
// material byte vi (0..63) of brick bi
__device__ __forceinline__ uint32_t ld_mat(const DevWorld &w, uint64_t bi, uint32_t vi) {
    return wload(w, w.mat, bi * 64u + vi, w.d.n_bricks * 64, ARR_MAT);
}

// Frame kernels: 128 threads, at least VX_MIN_BLOCKS CTAs per SM.  The walk
// is issue-bound, and the register budget this floor allows (76 registers at
// 5 CTAs) lets the compiler keep more of the walk's state live: on the c2
// frame 5 measured 0.408 ms against 0.414 (6), 0.418 (4), 0.427 (7) and
// 0.424 ms with no floor (56 registers, 9 CTAs), records identical.
#ifndef VX_MIN_BLOCKS
#define VX_MIN_BLOCKS 5
#endif
// Idle lanes a warp of the refill kernel waits for before it hands out new
// pixels (32 = refill only when the whole warp is idle).
#ifndef VX_REFILL_MIN
#define VX_REFILL_MIN 16
#endif
#if VX_MIN_BLOCKS > 0
#define VX_FRAME_BOUNDS __launch_bounds__(128, VX_MIN_BLOCKS)
#else
#define VX_FRAME_BOUNDS __launch_bounds__(128)
#endif

// Materials (src/voxel.rs:100-157, raymarch.wgsl:875-920)
__device__ __forceinline__ bool is_water(uint32_t m) { return m >= 5u && m <= 12u; }
__device__ __forceinline__ bool is_transparent(uint32_t m) { return is_water(m) || m == 18u; }
__device__ __forceinline__ bool is_decoration(uint32_t m) {
    return m == 30u || m == 31u || m == 33u || m == 34u || m == 35u || m == 36u || m == 37u;
}
__device__ __forceinline__ bool is_foliage(uint32_t m) {
    return m == 14u || m == 25u || m == 26u || m == 27u || is_decoration(m);
}
__device__ __forceinline__ bool is_uniform_optimisable(uint32_t m) {
    return !is_foliage(m) && !is_transparent(m);
}
// resolves_as_opaque_cube beyond both sub-voxel radii (raymarch.wgsl:4541)
__device__ __forceinline__ bool resolves_cube(uint32_t m) { return !is_decoration(m); }
// shadow_voxel_occludes far branch (raymarch.wgsl:4314-4343)
__device__ __forceinline__ bool shadow_occludes(uint32_t m) {
    return !(m == 33u || m == 35u || is_decoration(m));
}

// ------------------------------------------------------------- DDA state
// The voxel is kept relative to the window corner ro (the reference keeps
// it absolute and subtracts ro wherever it forms a float or a window test;
// every float the walk computes takes the relative value, so results are
// unchanged).  pm* = -1 where the step is positive, else 0.
struct Dda {
    float ox, oy, oz;      // origin rebased to the window corner
    float dx, dy, dz;
    float ix, iy, iz;      // safe_inv(dir)
    float mx, my, mz;      // t_max
    int32_t vx, vy, vz;    // voxel - ro
    int32_t stx, sty, stz; // step
    int32_t pmx, pmy, pmz; // -(step > 0)
};

struct Ro {
    int32_t x, y, z;
};

// dda_init, raymarch.wgsl:3369-3411.  Returns t_enter via *te.
__device__ __forceinline__ bool dda_init(const Dims &d, Ro ro, float o0, float o1, float o2,
                                         float d0, float d1, float d2, Dda &s, float *te) {
    const float fx = (float)d.vx, fy = (float)d.vy, fz = (float)d.vz;
    s.ox = o0 - (float)ro.x;
    s.oy = o1 - (float)ro.y;
    s.oz = o2 - (float)ro.z;
    s.dx = d0; s.dy = d1; s.dz = d2;
    s.ix = safe_inv(d0);
    s.iy = safe_inv(d1);
    s.iz = safe_inv(d2);
    float t0x = (0.0f - s.ox) * s.ix, t1x = (fx - s.ox) * s.ix;
    float t0y = (0.0f - s.oy) * s.iy, t1y = (fy - s.oy) * s.iy;
    float t0z = (0.0f - s.oz) * s.iz, t1z = (fz - s.oz) * s.iz;
    float tmnx = vmin(t0x, t1x), tmxx = vmax(t0x, t1x);
    float tmny = vmin(t0y, t1y), tmxy = vmax(t0y, t1y);
    float tmnz = vmin(t0z, t1z), tmxz = vmax(t0z, t1z);
    float t_enter = vmax(vmax(tmnx, tmny), vmax(tmnz, 0.0f));
    float t_exit = vmin(vmin(tmxx, tmxy), tmxz);
    *te = t_enter;
    if (t_enter >= t_exit || t_exit < 0.0f) return false;
    const float tb = t_enter + 1e-3f;
    float px = clampf(s.ox + d0 * tb, 0.01f, fx - 0.01f);
    float py = clampf(s.oy + d1 * tb, 0.01f, fy - 0.01f);
    float pz = clampf(s.oz + d2 * tb, 0.01f, fz - 0.01f);
    s.stx = sgn(d0); s.sty = sgn(d1); s.stz = sgn(d2);
    s.pmx = s.stx > 0 ? -1 : 0; s.pmy = s.sty > 0 ? -1 : 0; s.pmz = s.stz > 0 ? -1 : 0;
    // p is clamped into the window, so the floor converts without saturating
    const int32_t lx = __float2int_rd(px), ly = __float2int_rd(py), lz = __float2int_rd(pz);
    s.vx = lx; s.vy = ly; s.vz = lz;
    s.mx = ((float)(lx - s.pmx) - s.ox) * s.ix;
    s.my = ((float)(ly - s.pmy) - s.oy) * s.iy;
    s.mz = ((float)(lz - s.pmz) - s.oz) * s.iz;
    return true;
}

// Entry axis + t when a ray hits in its very first cell (last_axis == -1):
// recomputes tmin3/t_enter exactly as dda_init did (raymarch.wgsl:3335-3340).
__device__ __forceinline__ void first_cell_entry(const Dims &d, const Dda &s, int *ax,
                                                 float *t) {
    float t0x = (0.0f - s.ox) * s.ix, t1x = ((float)d.vx - s.ox) * s.ix;
    float t0y = (0.0f - s.oy) * s.iy, t1y = ((float)d.vy - s.oy) * s.iy;
    float t0z = (0.0f - s.oz) * s.iz, t1z = ((float)d.vz - s.oz) * s.iz;
    float a = vmin(t0x, t1x), b = vmin(t0y, t1y), c = vmin(t0z, t1z);
    *t = vmax(vmax(a, b), vmax(c, 0.0f));
    if (a >= b && a >= c) *ax = 0;
    else if (b >= c) *ax = 1;
    else *ax = 2;
}

// dda_step, raymarch.wgsl:3416-3448: the axis of the smallest t_max (x
// before y before z on ties, as the reference's strict compares order them),
// written with selects so that lanes stepping different axes do not diverge
__device__ __forceinline__ void dda_step(Dda &s, float &t_cur, int &la) {
    const bool ax = s.mx < s.my && s.mx < s.mz;
    const bool ay = !ax && s.my < s.mz;
    const bool az = !ax && !ay;
    t_cur = ax ? s.mx : (ay ? s.my : s.mz);
    s.vx += ax ? s.stx : 0;
    s.vy += ay ? s.sty : 0;
    s.vz += az ? s.stz : 0;
    s.mx = ax ? s.mx + fabsf(s.ix) : s.mx;
    s.my = ay ? s.my + fabsf(s.iy) : s.my;
    s.mz = az ? s.mz + fabsf(s.iz) : s.mz;
    la = ax ? 0 : (ay ? 1 : 2);
}

// skip_to_cell, raymarch.wgsl:4807-4864, for the cell of edge `cell` (a
// power of two dividing the window's dims) that holds the slot voxel
// (sx, sy, sz).  The reference aligns the cell in absolute coordinates,
// v - pos_mod(v, cell); the slot has the same residue mod cell, so the cell
// corner relative to the window is v_rel - (slot & (cell - 1)), and the
// exit-face boundary b - ro is that plus cell on positive-step axes: the same
// integers the reference converts, so the same floats follow.
// The landing floor(o + d * (t_min + 1e-3)) converts with saturation and no
// further clamp: a landing outside the int range is outside the window, so
// the next iteration ends the walk exactly as the reference's does, and the
// snapped axis and t of the crossed face are exact either way.
__device__ __forceinline__ void skip_to_cell(Dda &s, uint32_t sx, uint32_t sy, uint32_t sz,
                                             int32_t cell, int &la) {
    const uint32_t m = (uint32_t)cell - 1u;
    // boundary of the exit face, relative to the window corner
    const int32_t bx = s.vx - (int32_t)(sx & m) + (cell & s.pmx);
    const int32_t by = s.vy - (int32_t)(sy & m) + (cell & s.pmy);
    const int32_t bz = s.vz - (int32_t)(sz & m) + (cell & s.pmz);
    const float tfx = ((float)bx - s.ox) * s.ix;
    const float tfy = ((float)by - s.oy) * s.iy;
    const float tfz = ((float)bz - s.oz) * s.iz;
    const float eps = 1e-6f;
    float t_min = 1e30f;
    int ax = 0;
    if (s.stx != 0 && tfx > eps && tfx < t_min) { t_min = tfx; ax = 0; }
    if (s.sty != 0 && tfy > eps && tfy < t_min) { t_min = tfy; ax = 1; }
    if (s.stz != 0 && tfz > eps && tfz < t_min) { t_min = tfz; ax = 2; }
    const float tb = t_min + 1e-3f;
    // the voxel across the crossed face: b on positive steps, b - 1 on
    // negative ones (b is then the cell corner)
    const int32_t nx = ax == 0 ? bx + ~s.pmx : __float2int_rd(s.ox + s.dx * tb);
    const int32_t ny = ax == 1 ? by + ~s.pmy : __float2int_rd(s.oy + s.dy * tb);
    const int32_t nz = ax == 2 ? bz + ~s.pmz : __float2int_rd(s.oz + s.dz * tb);
    s.vx = nx; s.vy = ny; s.vz = nz;
    // t_max of the new voxel (a saturated landing wraps here; that walk ends
    // at its next window test)
    s.mx = ((float)(int32_t)((uint32_t)nx - (uint32_t)s.pmx) - s.ox) * s.ix;
    s.my = ((float)(int32_t)((uint32_t)ny - (uint32_t)s.pmy) - s.oy) * s.iy;
    s.mz = ((float)(int32_t)((uint32_t)nz - (uint32_t)s.pmz) - s.oz) * s.iz;
    la = ax;
}

// t of the face just crossed: t_max[la] - t_delta[la]
__device__ __forceinline__ float crossed_t(const Dda &s, int la) {
    return la == 0 ? s.mx - fabsf(s.ix) : (la == 1 ? s.my - fabsf(s.iy) : s.mz - fabsf(s.iz));
}

struct Hit {
    int32_t vx, vy, vz;
    float t;
    uint32_t steps;
    uint32_t mat;
    uint32_t face;    // 0xFF = miss
    uint32_t flags;
};

__device__ __forceinline__ void set_miss(Hit &h) {
    h.vx = h.vy = h.vz = 0;
    h.t = 0.0f;
    h.mat = 0;
    h.face = 0xFFu;
    h.flags = 0;
}

// entry_normal_and_t + last_axis_after_entry (raymarch.wgsl:3321-3342, :4800)
__device__ __forceinline__ void set_hit(const Dims &d, const Dda &s, Ro ro, int la, uint32_t m,
                                        bool early, Hit &h) {
    int ax;
    float t;
    if (la >= 0) {
        ax = la;
        t = crossed_t(s, la);
    } else {
        first_cell_entry(d, s, &ax, &t);
    }
    const int32_t st = ax == 0 ? s.stx : (ax == 1 ? s.sty : s.stz);
    h.vx = s.vx + ro.x; h.vy = s.vy + ro.y; h.vz = s.vz + ro.z;
    h.t = t;
    h.mat = m;
    h.face = (uint32_t)(2 * ax + (st > 0 ? 1 : 0));
    h.flags = 1u | (early ? 2u : 0u);
}

// brick_topmost_material, raymarch.wgsl:253-295
template <bool STATS>
__device__ __forceinline__ uint32_t brick_topmost(const DevWorld &w, uint64_t bi, uint64_t occ,
                                                  uint64_t &bytes) {
    const uint32_t lo = (uint32_t)occ, hi = (uint32_t)(occ >> 32);
    const uint32_t layer[4] = {(hi >> 16) & 0xFFFFu, hi & 0xFFFFu, (lo >> 16) & 0xFFFFu,
                               lo & 0xFFFFu};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (layer[i] != 0u) {
            const int bit = __ffs(layer[i]) - 1;
            const uint32_t m = ld_mat(w, bi, (uint32_t)((48 - 16 * i) + bit));
            if (STATS) bytes += 1;
            if (m != 35u) return m;
        }
    }
    return (lo | hi) != 0u ? 35u : 0u;
}

// 32-bit strides of every level (all cell indices of a world that fits in
// device memory are below 2^32; only the material row offset is widened).
struct Geo {
    uint32_t bx, bxy, tx, txy, cx, cxy, lx, lxy;
    uint32_t rox, roz;  // pos_mod(window corner x / z, dims): slot of window voxel 0
};
template <uint32_t FL>
__device__ __forceinline__ Geo geo_of(const Dims &d, Ro ro) {
    Geo g;
    g.rox = (uint32_t)pos_mod(ro.x, d.vx);
    g.roz = (uint32_t)pos_mod(ro.z, d.vz);
    g.bx = (uint32_t)d.bx;
    g.bxy = (uint32_t)(d.bx * d.by);
    g.tx = (uint32_t)d.tx;
    g.txy = (uint32_t)(d.tx * d.ty);
    g.cx = (uint32_t)d.cx;
    g.cxy = (uint32_t)(d.cx * d.cy);
    g.lx = (uint32_t)d.lx;
    g.lxy = (uint32_t)(d.lx * d.ly);
    return g;
}
__device__ __forceinline__ uint32_t l4_index(const Geo &g, uint32_t sx, uint32_t sy, uint32_t sz) {
    return (sx >> 8) + (sy >> 8) * g.lx + (sz >> 8) * g.lxy;
}
__device__ __forceinline__ uint32_t chunk_index(const Geo &g, uint32_t sx, uint32_t sy, uint32_t sz) {
    return (sx >> 6) + (sy >> 6) * g.cx + (sz >> 6) * g.cxy;
}
__device__ __forceinline__ uint32_t tile_index(const Geo &g, uint32_t sx, uint32_t sy, uint32_t sz) {
    return (sx >> 4) + (sy >> 4) * g.tx + (sz >> 4) * g.txy;
}
__device__ __forceinline__ uint32_t brick_index(const Geo &g, uint32_t bx, uint32_t by, uint32_t bz) {
    return bx + by * g.bx + bz * g.bxy;
}
// child bit x + z*4 + y*16 of the level whose cell size is 1 << sh
__device__ __forceinline__ int child_of(uint32_t sx, uint32_t sy, uint32_t sz, int sh) {
    return (int)(((sx >> sh) & 3u) + ((sz >> sh) & 3u) * 4u + ((sy >> sh) & 3u) * 16u);
}

// ------------------------------------------------------------ tile meta
// DevWorld::tile_meta word.  Every voxel of a tile shares the tile's chunk
// and L4 cell, so trace's L4 and chunk tests (raymarch.wgsl:4648-4668) have
// one outcome per tile:
//   bits 0-7   the tile LUT byte where the tile LUT test ends a walk (the
//              byte is a uniform_optimisable material), else 0
//   bits 8-9   the cell the L4 and chunk tests skip: 0 none, 1 the 16-voxel
//              tile, 2 the 64-voxel chunk, 3 the 256-voxel L4 cell
//   bit 10     the chunk test alone skips the tile (walks without L4)
constexpr uint32_t kMetaChunkOnly = 1u << 10;

// ------------------------------------------------------------------ walk
// One traversal = dda_init + repeated cascade iterations.  The three kinds
// share the level cascade and differ only where the reference differs:
//   KIND_TRACE    trace()           raymarch.wgsl:4600-4777 (L4 optional,
//                                   LUT + LOD per method flags, cube rule)
//   KIND_ANY      trace_any()       raymarch.wgsl:4345-4409 (occluder rule)
//   KIND_NO_WATER trace_no_water()  raymarch.wgsl:3450-3532 (first
//                                   non-transparent voxel; t_cur not
//                                   refreshed after a skip)
enum : uint32_t { KIND_TRACE = 0, KIND_ANY = 1, KIND_NO_WATER = 2 };

struct Walk {
    Dda s;
    float t_cur;
    float tmax;       // MAX_RAY_DIST / max_dist / t_cap of this ray
    int la;           // last_axis
    uint32_t iters;   // loop iterations begun
    uint32_t cap;     // iteration cap (1024 / 768 / 1024)
    uint32_t kind;
};

enum : int { WALK_CONT = 0, WALK_END = 1, WALK_HIT = 2 };

__device__ __forceinline__ bool walk_init(const Dims &d, Ro ro, uint32_t kind,
                                          const VxTraceParams &p, float o0, float o1, float o2,
                                          float d0, float d1, float d2, float tmax, Walk &k) {
    k.kind = kind;
    k.tmax = tmax;
    k.la = -1;
    k.iters = 0;
    k.cap = (uint32_t)(kind == KIND_ANY ? p.any_max_iters : p.max_iters);
    return dda_init(d, ro, o0, o1, o2, d0, d1, d2, k.s, &k.t_cur);
}

// One cascade iteration.  On WALK_HIT the record fields of h are set (for
// KIND_ANY only "occluded" matters).  FL holds VX_F_L4|VX_F_LUT|VX_F_LOD as
// compile-time bits; KNOWN >= 0 fixes the kind at compile time.
template <uint32_t FL, bool STATS, int KNOWN>
__device__ __forceinline__ int walk_step(const DevWorld &w, const Geo &g, const VxTraceParams &p,
                                         Ro ro, Walk &k, Hit &h, uint64_t &bytes) {
    const uint32_t kind = KNOWN >= 0 ? (uint32_t)KNOWN : k.kind;
    const bool is_trace = kind == KIND_TRACE;
    const bool use_l4 = !is_trace || (FL & VX_F_L4) != 0u;
    const bool f_lut = is_trace && (FL & VX_F_LUT) != 0u;
    const bool f_lod = is_trace && (FL & VX_F_LOD) != 0u;
    const Dims &d = w.d;
    Dda &s = k.s;
    if (k.iters >= k.cap) return WALK_END;
    ++k.iters;
    if (k.t_cur > k.tmax) return WALK_END;
    // window test, then the toroidal slot (world_to_slot_voxel,
    // raymarch.wgsl:17-23) from the window-relative voxel: rel < dims and
    // rox < dims, so a mask (power-of-two dims) or one conditional
    // subtraction folds it
    const uint32_t lx = (uint32_t)s.vx, lz = (uint32_t)s.vz;
    if (lx >= (uint32_t)d.vx || (uint32_t)s.vy >= (uint32_t)d.vy || lz >= (uint32_t)d.vz)
        return WALK_END;
    uint32_t sx = lx + g.rox, sz = lz + g.roz;
    if ((FL & kFlPow2) != 0u) {
        sx &= (uint32_t)(d.vx - 1);
        sz &= (uint32_t)(d.vz - 1);
    } else {
        if (sx >= (uint32_t)d.vx) sx -= (uint32_t)d.vx;
        if (sz >= (uint32_t)d.vz) sz -= (uint32_t)d.vz;
    }
    const uint32_t sy = (uint32_t)s.vy;
    const uint32_t ti = tile_index(g, sx, sy, sz);
    // batch 1: every coarse word addressed by the slot coordinate
    const uint64_t tw = ld_tile(w, ti);
    uint32_t tum;
    bool tum_exit = false;  // the tile LUT test ends the walk (with material tum)
    int32_t cell = 0;
    if (w.tile_meta != nullptr) {
        const uint32_t meta = ld_tile_meta(w, ti);
        tum = f_lut ? (meta & 0xFFu) : 0u;
        tum_exit = tum != 0u;  // pre-filtered by k_tile_meta
        if (use_l4) {
            const uint32_t code = (meta >> 8) & 3u;
            if (STATS) bytes += code >= 2u ? 8 : 16;
            if (code != 0u) cell = 4 << (2 * code);
        } else {
            if (STATS) bytes += 8;
            if ((meta & kMetaChunkOnly) != 0u) cell = 16;
        }
    } else {
        uint64_t lw = ~0ull;
        if (use_l4) lw = ld_l4(w, l4_index(g, sx, sy, sz));
        const uint64_t cw = ld_chunk(w, chunk_index(g, sx, sy, sz));
        tum = f_lut ? ld_tile_uniform(w, ti) : 0u;
        tum_exit = tum != 0u && is_uniform_optimisable(tum);
        if (use_l4) {
            if (STATS) bytes += 8;
            if (lw == 0ull) cell = 256;
            else if (!bit64(lw, child_of(sx, sy, sz, 6))) cell = 64;
        }
        if (cell == 0) {
            if (STATS) bytes += 8;
            if (!bit64(cw, child_of(sx, sy, sz, 4))) cell = 16;
        }
    }
    if (cell == 0) {
        // tile-level LOD (raymarch.wgsl:4672-4689)
        if (f_lod && k.t_cur > p.tile_lod_t) {
            if (STATS) bytes += 8;
            uint32_t lm = 0u;
            if (tw != 0ull) {
                const int lin = __ffsll((long long)tw) - 1;
                const uint32_t rbi = brick_index(g, (sx >> 4) * 4u + (uint32_t)(lin & 3),
                                                 (sy >> 4) * 4u + (uint32_t)((lin >> 4) & 3),
                                                 (sz >> 4) * 4u + (uint32_t)((lin >> 2) & 3));
                if (STATS) bytes += 8;
                lm = brick_topmost<STATS>(w, rbi, ld_occ(w, rbi), bytes);
            }
            if (lm != 0u && is_uniform_optimisable(lm)) {
                set_hit(d, s, ro, k.la, lm, true, h);
                return WALK_HIT;
            }
        }
        // tile LUT (raymarch.wgsl:4692-4706)
        if (f_lut) {
            if (STATS) bytes += 1;
            if (tum_exit) {
                set_hit(d, s, ro, k.la, tum, true, h);
                return WALK_HIT;
            }
        }
        if (STATS) bytes += 8;
        const int tb = child_of(sx, sy, sz, 2);
        if (!bit64(tw, tb)) {
            cell = 4;
        } else {
            const uint32_t bi = brick_index(g, sx >> 2, sy >> 2, sz >> 2);
            // batch 2: brick occupancy + brick LUT byte
            const uint64_t occ = ld_occ(w, bi);
            const uint32_t bum = f_lut ? ld_brick_uniform(w, bi) : 0u;
            if (f_lut) {
                // brick LUT (raymarch.wgsl:4716-4731)
                if (STATS) bytes += 1;
                if (bum != 0u && is_uniform_optimisable(bum)) {
                    set_hit(d, s, ro, k.la, bum, true, h);
                    return WALK_HIT;
                }
            }
            bool lod_done = false;
            if (f_lod && k.t_cur > p.lod_brick_t) {
                if (STATS) bytes += 8;
                if (occ == 0ull) {
                    cell = 4;
                    lod_done = true;
                } else {
                    const uint32_t m = brick_topmost<STATS>(w, bi, occ, bytes);
                    if (!is_foliage(m)) {
                        set_hit(d, s, ro, k.la, m, true, h);
                        return WALK_HIT;
                    }
                }
            }
            if (!lod_done) {
                const int vi = child_of(sx, sy, sz, 0);
                if (STATS) bytes += 8;
                if (bit64(occ, vi)) {
                    // the material byte of a solid voxel
                    const uint32_t m = ld_mat(w, bi, (uint32_t)vi);
                    if (STATS) bytes += 1;
                    const bool stop = kind == KIND_TRACE ? resolves_cube(m)
                                      : (kind == KIND_ANY ? shadow_occludes(m) : !is_transparent(m));
                    if (stop) {
                        if (kind != KIND_ANY) set_hit(d, s, ro, k.la, m, false, h);
                        return WALK_HIT;
                    }
                }
            }
        }
    }
    if (cell != 0) {
        skip_to_cell(s, sx, sy, sz, cell, k.la);
        if (kind != KIND_NO_WATER) k.t_cur = crossed_t(s, k.la);
    } else {
        dda_step(s, k.t_cur, k.la);
    }
    return WALK_CONT;
}

// trace() over one ray
template <uint32_t FL, bool STATS>
__device__ __forceinline__ void trace_ray(const DevWorld &w, const VxTraceParams &p, Ro ro,
                                          float o0, float o1, float o2, float d0, float d1,
                                          float d2, float max_dist, Hit &h, uint64_t &bytes) {
    const Geo g = geo_of<FL>(w.d, ro);
    set_miss(h);
    Walk k;
    if (!walk_init(w.d, ro, KIND_TRACE, p, o0, o1, o2, d0, d1, d2, max_dist, k)) {
        h.steps = 0;
        return;
    }
    while (walk_step<FL, STATS, KIND_TRACE>(w, g, p, ro, k, h, bytes) == WALK_CONT) {
    }
    h.steps = k.iters;
}

// trace_any() over one ray: returns occluded (FLP carries kFlPow2 only)
template <uint32_t FLP, bool STATS>
__device__ __forceinline__ bool trace_any_ray(const DevWorld &w, const VxTraceParams &p, Ro ro,
                                              float o0, float o1, float o2, float d0, float d1,
                                              float d2, float max_dist, uint32_t &steps,
                                              uint64_t &bytes) {
    const Geo g = geo_of<FLP>(w.d, ro);
    Walk k;
    Hit h;
    steps = 0;
    if (!walk_init(w.d, ro, KIND_ANY, p, o0, o1, o2, d0, d1, d2, max_dist, k)) return false;
    int r;
    while ((r = walk_step<FLP & kFlPow2, STATS, KIND_ANY>(w, g, p, ro, k, h, bytes)) == WALK_CONT) {
    }
    steps = k.iters;
    return r == WALK_HIT;
}

// trace_no_water() over one ray (FLP carries kFlPow2 only)
template <uint32_t FLP, bool STATS>
__device__ __forceinline__ void trace_no_water_ray(const DevWorld &w, const VxTraceParams &p,
                                                   Ro ro, float o0, float o1, float o2,
                                                   float d0, float d1, float d2, float t_cap,
                                                   Hit &h, uint64_t &bytes) {
    const Geo g = geo_of<FLP>(w.d, ro);
    set_miss(h);
    Walk k;
    if (!walk_init(w.d, ro, KIND_NO_WATER, p, o0, o1, o2, d0, d1, d2, t_cap, k)) {
        h.steps = 0;
        return;
    }
    while (walk_step<FLP & kFlPow2, STATS, KIND_NO_WATER>(w, g, p, ro, k, h, bytes) == WALK_CONT) {
    }
    h.steps = k.iters;
}

// normalize with IEEE sqrt + divide
__device__ __forceinline__ void normalize3(float &x, float &y, float &z) {
    const float len = sqrtf((x * x + y * y) + z * z);
    x = x / len;
    y = y / len;
    z = z / len;
}

// ray_dir_uv, raymarch.wgsl:430-438
__device__ __forceinline__ void ray_dir_uv(const VxCamera &c, float u, float v, float &x,
                                           float &y, float &z) {
    const float ndc_x = u * 2.0f - 1.0f;
    const float ndc_y = 1.0f - v * 2.0f;
    const float aspect = c.res_x / c.res_y;
    const float a = ndc_x * c.tan_half_fov * aspect;
    const float b = ndc_y * c.tan_half_fov;
    x = (c.forward[0] + c.right[0] * a) + c.up[0] * b;
    y = (c.forward[1] + c.right[1] * a) + c.up[1] * b;
    z = (c.forward[2] + c.right[2] * a) + c.up[2] * b;
    normalize3(x, y, z);
}

// ign, raymarch.wgsl:394-396
__device__ __forceinline__ float ign(float x, float y, float frame) {
    const float a = x + frame * 5.588238f;
    const float b = y + frame * 4.182857f;
    return fractf(52.9829189f * fractf(0.06711056f * a + 0.00583715f * b));
}

// sin/cos by the Maclaurin series nested in x^2 (terms through x^17 / x^18),
// evaluated in a fixed order so host and device agree bit for bit.
__device__ __forceinline__ void sincos_series(float x, float &sn, float &cs) {
    const float x2 = x * x;
    float ps = 1.0f - x2 * 0.0036764706f;
    ps = 1.0f - x2 * 0.0047619049f * ps;
    ps = 1.0f - x2 * 0.0064102565f * ps;
    ps = 1.0f - x2 * 0.0090909088f * ps;
    ps = 1.0f - x2 * 0.013888889f * ps;
    ps = 1.0f - x2 * 0.023809524f * ps;
    ps = 1.0f - x2 * 0.050000001f * ps;
    ps = 1.0f - x2 * 0.16666667f * ps;
    sn = x * ps;
    float pc = 1.0f - x2 * 0.0032679739f;
    pc = 1.0f - x2 * 0.0041666669f * pc;
    pc = 1.0f - x2 * 0.0054945056f * pc;
    pc = 1.0f - x2 * 0.0075757578f * pc;
    pc = 1.0f - x2 * 0.011111111f * pc;
    pc = 1.0f - x2 * 0.017857144f * pc;
    pc = 1.0f - x2 * 0.033333335f * pc;
    pc = 1.0f - x2 * 0.083333336f * pc;
    pc = 1.0f - x2 * 0.5f * pc;
    cs = pc;
}

__device__ __forceinline__ void store_record(VxHitRecord *r, const Hit &h) {
    // 24-byte record written as three 8-byte words (records are 8-aligned)
    uint2 *q = reinterpret_cast<uint2 *>(r);
    q[0] = make_uint2((uint32_t)h.vx, (uint32_t)h.vy);
    q[1] = make_uint2((uint32_t)h.vz, h.face | (h.mat << 8) | (h.flags << 16));
    q[2] = make_uint2(__float_as_uint(h.t), h.steps);
}

__device__ __forceinline__ void flush_stats(unsigned long long *stats, uint64_t bytes,
                                            uint64_t iters) {
    atomicAdd(stats + 0, (unsigned long long)bytes);
    atomicAdd(stats + 1, (unsigned long long)iters);
}


}  // namespace
}  // namespace vx
