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

#include "vx_internal.h"

namespace vx {
namespace {

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ float vmin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float vmax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) {
    return vmin(vmax(x, lo), hi);
}
__device__ __forceinline__ int32_t f2i(float x) {
    if (x != x) return 0;
    if (x >= 1073741824.0f) return 1073741824;
    if (x <= -1073741824.0f) return -1073741824;
    return (int32_t)x;
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
struct Dda {
    float ox, oy, oz;      // origin rebased to the window corner
    float dx, dy, dz;
    float ix, iy, iz;      // safe_inv(dir)
    float mx, my, mz;      // t_max
    int32_t vx, vy, vz;    // voxel, absolute world coords
    int32_t sx, sz;        // toroidal slot x/z (slot y == vy)
    int32_t stx, sty, stz; // step
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
    int32_t lx = f2i(floorf(px)), ly = f2i(floorf(py)), lz = f2i(floorf(pz));
    s.vx = lx + ro.x; s.vy = ly + ro.y; s.vz = lz + ro.z;
    s.mx = s.stx > 0 ? ((float)(lx + 1) - s.ox) * s.ix : ((float)lx - s.ox) * s.ix;
    s.my = s.sty > 0 ? ((float)(ly + 1) - s.oy) * s.iy : ((float)ly - s.oy) * s.iy;
    s.mz = s.stz > 0 ? ((float)(lz + 1) - s.oz) * s.iz : ((float)lz - s.oz) * s.iz;
    s.sx = pos_mod(s.vx, d.vx);
    s.sz = pos_mod(s.vz, d.vz);
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

// dda_step, raymarch.wgsl:3416-3448
__device__ __forceinline__ void dda_step(const Dims &d, Dda &s, float &t_cur, int &la) {
    if (s.mx < s.my && s.mx < s.mz) {
        t_cur = s.mx;
        s.vx += s.stx;
        s.sx += s.stx;
        if (s.sx >= d.vx) s.sx -= d.vx;
        else if (s.sx < 0) s.sx += d.vx;
        s.mx = s.mx + fabsf(s.ix);
        la = 0;
    } else if (s.my < s.mz) {
        t_cur = s.my;
        s.vy += s.sty;
        s.my = s.my + fabsf(s.iy);
        la = 1;
    } else {
        t_cur = s.mz;
        s.vz += s.stz;
        s.sz += s.stz;
        if (s.sz >= d.vz) s.sz -= d.vz;
        else if (s.sz < 0) s.sz += d.vz;
        s.mz = s.mz + fabsf(s.iz);
        la = 2;
    }
}

// skip_to_cell, raymarch.wgsl:4807-4864.  cell is a power of two, so
// v - pos_mod(v, cell) == v & ~(cell - 1) for every int v.
__device__ __forceinline__ void skip_to_cell(const Dims &d, Ro ro, int32_t cell, Dda &s,
                                             int &la) {
    const int32_t hi = ~(cell - 1);
    const int32_t cox = s.vx & hi, coy = s.vy & hi, coz = s.vz & hi;
    const float tfx = ((float)((s.stx > 0 ? cox + cell : cox) - ro.x) - s.ox) * s.ix;
    const float tfy = ((float)((s.sty > 0 ? coy + cell : coy) - ro.y) - s.oy) * s.iy;
    const float tfz = ((float)((s.stz > 0 ? coz + cell : coz) - ro.z) - s.oz) * s.iz;
    const float eps = 1e-6f;
    float t_min = 1e30f;
    int ax = 0;
    if (s.stx != 0 && tfx > eps && tfx < t_min) { t_min = tfx; ax = 0; }
    if (s.sty != 0 && tfy > eps && tfy < t_min) { t_min = tfy; ax = 1; }
    if (s.stz != 0 && tfz > eps && tfz < t_min) { t_min = tfz; ax = 2; }
    const float tb = t_min + 1e-3f;
    int32_t nx = f2i(floorf(s.ox + s.dx * tb)) + ro.x;
    int32_t ny = f2i(floorf(s.oy + s.dy * tb)) + ro.y;
    int32_t nz = f2i(floorf(s.oz + s.dz * tb)) + ro.z;
    if (ax == 0) nx = s.stx > 0 ? cox + cell : cox - 1;
    else if (ax == 1) ny = s.sty > 0 ? coy + cell : coy - 1;
    else nz = s.stz > 0 ? coz + cell : coz - 1;
    s.vx = nx; s.vy = ny; s.vz = nz;
    const int32_t lx = nx - ro.x, ly = ny - ro.y, lz = nz - ro.z;
    s.mx = s.stx > 0 ? ((float)(lx + 1) - s.ox) * s.ix : ((float)lx - s.ox) * s.ix;
    s.my = s.sty > 0 ? ((float)(ly + 1) - s.oy) * s.iy : ((float)ly - s.oy) * s.iy;
    s.mz = s.stz > 0 ? ((float)(lz + 1) - s.oz) * s.iz : ((float)lz - s.oz) * s.iz;
    la = ax;
    s.sx = pos_mod(nx, d.vx);
    s.sz = pos_mod(nz, d.vz);
}

// t of the face just crossed: t_max[la] - t_delta[la]
__device__ __forceinline__ float crossed_t(const Dda &s, int la) {
    return la == 0 ? s.mx - fabsf(s.ix) : (la == 1 ? s.my - fabsf(s.iy) : s.mz - fabsf(s.iz));
}

__device__ __forceinline__ bool out_of_window(const Dims &d, const Dda &s, Ro ro) {
    return (uint32_t)(s.vx - ro.x) >= (uint32_t)d.vx || (uint32_t)(s.vy - ro.y) >= (uint32_t)d.vy ||
           (uint32_t)(s.vz - ro.z) >= (uint32_t)d.vz;
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
__device__ __forceinline__ void set_hit(const Dims &d, const Dda &s, int la, uint32_t m,
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
    h.vx = s.vx; h.vy = s.vy; h.vz = s.vz;
    h.t = t;
    h.mat = m;
    h.face = (uint32_t)(2 * ax + (st > 0 ? 1 : 0));
    h.flags = 1u | (early ? 2u : 0u);
}

// brick_topmost_material, raymarch.wgsl:253-295
template <bool STATS>
__device__ __forceinline__ uint32_t brick_topmost(const uint8_t *__restrict__ mrow, uint64_t occ,
                                                  uint64_t &bytes) {
    const uint32_t lo = (uint32_t)occ, hi = (uint32_t)(occ >> 32);
    const uint32_t layer[4] = {(hi >> 16) & 0xFFFFu, hi & 0xFFFFu, (lo >> 16) & 0xFFFFu,
                               lo & 0xFFFFu};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        if (layer[i] != 0u) {
            const int bit = __ffs(layer[i]) - 1;
            const uint32_t m = ldg(mrow + (48 - 16 * i) + bit);
            if (STATS) bytes += 1;
            if (m != 35u) return m;
        }
    }
    return (lo | hi) != 0u ? 35u : 0u;
}

// ------------------------------------------------------------------ trace
// trace(), raymarch.wgsl:4600-4777, far-distance cube resolution.
template <bool STATS>
__device__ __forceinline__ void trace_ray(const DevWorld &w, const VxTraceParams &p, Ro ro,
                                          float o0, float o1, float o2, float d0, float d1,
                                          float d2, float max_dist, Hit &h, uint64_t &bytes) {
    const Dims &d = w.d;
    set_miss(h);
    Dda s;
    float t_cur;
    uint32_t iters = 0;
    if (!dda_init(d, ro, o0, o1, o2, d0, d1, d2, s, &t_cur)) {
        h.steps = 0;
        return;
    }
    const bool f_l4 = (p.flags & VX_F_L4) != 0u;
    const bool f_lut = (p.flags & VX_F_LUT) != 0u;
    const bool f_lod = (p.flags & VX_F_LOD) != 0u;
    int la = -1;
    for (int it = 0; it < p.max_iters; ++it) {
        ++iters;
        if (t_cur > max_dist) break;
        if (out_of_window(d, s, ro)) break;
        const int32_t sx = s.sx, sy = s.vy, sz = s.sz;
        const int64_t ci = (int64_t)(sx >> 6) + (int64_t)(sy >> 6) * d.cx +
                           (int64_t)(sz >> 6) * d.cx * d.cy;
        const int64_t ti = (int64_t)(sx >> 4) + (int64_t)(sy >> 4) * d.tx +
                           (int64_t)(sz >> 4) * d.tx * d.ty;
        // batch 1: every coarse word addressed by the slot coordinate
        uint64_t lw = ~0ull;
        if (f_l4) {
            const int64_t li = (int64_t)(sx >> 8) + (int64_t)(sy >> 8) * d.lx +
                               (int64_t)(sz >> 8) * d.lx * d.ly;
            lw = ldg(w.l4_mask + li);
        }
        const uint64_t cw = ldg(w.chunk_mask + ci);
        const uint64_t tw = ldg(w.tile_mask + ti);
        const uint32_t tum = f_lut ? (uint32_t)ldg(w.tile_uniform + ti) : 0u;
        int32_t cell = 0;
        if (f_l4) {
            if (STATS) bytes += 8;
            if (lw == 0ull) cell = 256;
            else if (!bit64(lw, child_bit((sx >> 6) & 3, (sy >> 6) & 3, (sz >> 6) & 3))) cell = 64;
        }
        if (cell == 0) {
            if (STATS) bytes += 8;
            if (!bit64(cw, child_bit((sx >> 4) & 3, (sy >> 4) & 3, (sz >> 4) & 3))) cell = 16;
        }
        if (cell == 0) {
            // tile-level LOD (raymarch.wgsl:4672-4689)
            if (f_lod && t_cur > p.tile_lod_t) {
                if (STATS) bytes += 8;
                uint32_t lm = 0u;
                const uint32_t tlo = (uint32_t)tw, thi = (uint32_t)(tw >> 32);
                int lin = -1;
                if (tlo != 0u) lin = __ffs(tlo) - 1;
                else if (thi != 0u) lin = 32 + __ffs(thi) - 1;
                if (lin >= 0) {
                    const int64_t rbi = (int64_t)((sx >> 4) * 4 + (lin & 3)) +
                                        (int64_t)((sy >> 4) * 4 + ((lin >> 4) & 3)) * d.bx +
                                        (int64_t)((sz >> 4) * 4 + ((lin >> 2) & 3)) * d.bx * d.by;
                    if (STATS) bytes += 8;
                    lm = brick_topmost<STATS>(w.mat + rbi * 64, ldg(w.occ + rbi), bytes);
                }
                if (lm != 0u && is_uniform_optimisable(lm)) {
                    set_hit(d, s, la, lm, true, h);
                    break;
                }
            }
            if (f_lut) {
                if (STATS) bytes += 1;
                if (tum != 0u && is_uniform_optimisable(tum)) {
                    set_hit(d, s, la, tum, true, h);
                    break;
                }
            }
            if (STATS) bytes += 8;
            const int bx = sx >> 2, by = sy >> 2, bz = sz >> 2;
            if (!bit64(tw, child_bit(bx & 3, by & 3, bz & 3))) {
                cell = 4;
            } else {
                const int64_t bi = (int64_t)bx + (int64_t)by * d.bx + (int64_t)bz * d.bx * d.by;
                // batch 2: brick occupancy + brick LUT byte
                const uint64_t occ = ldg(w.occ + bi);
                const uint32_t bum = f_lut ? (uint32_t)ldg(w.brick_uniform + bi) : 0u;
                if (f_lut) {
                    if (STATS) bytes += 1;
                    if (bum != 0u && is_uniform_optimisable(bum)) {
                        set_hit(d, s, la, bum, true, h);
                        break;
                    }
                }
                const uint8_t *mrow = w.mat + bi * 64;
                bool lod_done = false;
                if (f_lod && t_cur > p.lod_brick_t) {
                    if (STATS) bytes += 8;
                    if (occ == 0ull) {
                        cell = 4;
                        lod_done = true;
                    } else {
                        const uint32_t m = brick_topmost<STATS>(mrow, occ, bytes);
                        if (!is_foliage(m)) {
                            set_hit(d, s, la, m, true, h);
                            break;
                        }
                    }
                }
                if (!lod_done) {
                    const int vi = child_bit(sx - bx * 4, sy - by * 4, sz - bz * 4);
                    if (STATS) bytes += 8;
                    if (bit64(occ, vi)) {
                        // batch 3: the material byte of a solid voxel
                        const uint32_t m = ldg(mrow + vi);
                        if (STATS) bytes += 1;
                        if (resolves_cube(m)) {
                            set_hit(d, s, la, m, false, h);
                            break;
                        }
                    }
                }
            }
        }
        if (cell != 0) {
            skip_to_cell(d, ro, cell, s, la);
            t_cur = crossed_t(s, la);
        } else {
            dda_step(d, s, t_cur, la);
        }
    }
    h.steps = iters;
    if (STATS) bytes += 0;
}

// trace_any(), raymarch.wgsl:4345-4409 -- returns occluded.
template <bool STATS>
__device__ __forceinline__ bool trace_any_ray(const DevWorld &w, const VxTraceParams &p, Ro ro,
                                              float o0, float o1, float o2, float d0, float d1,
                                              float d2, float max_dist, uint32_t &steps,
                                              uint64_t &bytes) {
    const Dims &d = w.d;
    Dda s;
    float t_cur;
    uint32_t iters = 0;
    steps = 0;
    if (!dda_init(d, ro, o0, o1, o2, d0, d1, d2, s, &t_cur)) return false;
    int la = -1;
    bool occluded = false;
    for (int it = 0; it < p.any_max_iters; ++it) {
        ++iters;
        if (t_cur > max_dist) break;
        if (out_of_window(d, s, ro)) break;
        const int32_t sx = s.sx, sy = s.vy, sz = s.sz;
        const int64_t li = (int64_t)(sx >> 8) + (int64_t)(sy >> 8) * d.lx +
                           (int64_t)(sz >> 8) * d.lx * d.ly;
        const int64_t ci = (int64_t)(sx >> 6) + (int64_t)(sy >> 6) * d.cx +
                           (int64_t)(sz >> 6) * d.cx * d.cy;
        const int64_t ti = (int64_t)(sx >> 4) + (int64_t)(sy >> 4) * d.tx +
                           (int64_t)(sz >> 4) * d.tx * d.ty;
        const uint64_t lw = ldg(w.l4_mask + li);
        const uint64_t cw = ldg(w.chunk_mask + ci);
        const uint64_t tw = ldg(w.tile_mask + ti);
        int32_t cell = 0;
        if (STATS) bytes += 8;
        if (lw == 0ull) cell = 256;
        else if (!bit64(lw, child_bit((sx >> 6) & 3, (sy >> 6) & 3, (sz >> 6) & 3))) cell = 64;
        if (cell == 0) {
            if (STATS) bytes += 8;
            if (!bit64(cw, child_bit((sx >> 4) & 3, (sy >> 4) & 3, (sz >> 4) & 3))) cell = 16;
        }
        if (cell == 0) {
            if (STATS) bytes += 8;
            const int bx = sx >> 2, by = sy >> 2, bz = sz >> 2;
            if (!bit64(tw, child_bit(bx & 3, by & 3, bz & 3))) {
                cell = 4;
            } else {
                const int64_t bi = (int64_t)bx + (int64_t)by * d.bx + (int64_t)bz * d.bx * d.by;
                const uint64_t occ = ldg(w.occ + bi);
                const int vi = child_bit(sx - bx * 4, sy - by * 4, sz - bz * 4);
                if (STATS) bytes += 8;
                if (bit64(occ, vi)) {
                    const uint32_t m = ldg(w.mat + bi * 64 + vi);
                    if (STATS) bytes += 1;
                    if (shadow_occludes(m)) {
                        occluded = true;
                        break;
                    }
                }
            }
        }
        if (cell != 0) {
            skip_to_cell(d, ro, cell, s, la);
            t_cur = crossed_t(s, la);
        } else {
            dda_step(d, s, t_cur, la);
        }
    }
    steps = iters;
    return occluded;
}

// trace_no_water(), raymarch.wgsl:3450-3532 (t_cur is not refreshed after
// a skip there; reproduced).
template <bool STATS>
__device__ __forceinline__ void trace_no_water_ray(const DevWorld &w, const VxTraceParams &p,
                                                   Ro ro, float o0, float o1, float o2,
                                                   float d0, float d1, float d2, float t_cap,
                                                   Hit &h, uint64_t &bytes) {
    const Dims &d = w.d;
    set_miss(h);
    Dda s;
    float t_cur;
    uint32_t iters = 0;
    if (!dda_init(d, ro, o0, o1, o2, d0, d1, d2, s, &t_cur)) {
        h.steps = 0;
        return;
    }
    int la = -1;
    for (int it = 0; it < p.max_iters; ++it) {
        ++iters;
        if (t_cur > t_cap) break;
        if (out_of_window(d, s, ro)) break;
        const int32_t sx = s.sx, sy = s.vy, sz = s.sz;
        const int64_t li = (int64_t)(sx >> 8) + (int64_t)(sy >> 8) * d.lx +
                           (int64_t)(sz >> 8) * d.lx * d.ly;
        const int64_t ci = (int64_t)(sx >> 6) + (int64_t)(sy >> 6) * d.cx +
                           (int64_t)(sz >> 6) * d.cx * d.cy;
        const int64_t ti = (int64_t)(sx >> 4) + (int64_t)(sy >> 4) * d.tx +
                           (int64_t)(sz >> 4) * d.tx * d.ty;
        const uint64_t lw = ldg(w.l4_mask + li);
        const uint64_t cw = ldg(w.chunk_mask + ci);
        const uint64_t tw = ldg(w.tile_mask + ti);
        int32_t cell = 0;
        if (STATS) bytes += 8;
        if (lw == 0ull) cell = 256;
        else if (!bit64(lw, child_bit((sx >> 6) & 3, (sy >> 6) & 3, (sz >> 6) & 3))) cell = 64;
        if (cell == 0) {
            if (STATS) bytes += 8;
            if (!bit64(cw, child_bit((sx >> 4) & 3, (sy >> 4) & 3, (sz >> 4) & 3))) cell = 16;
        }
        if (cell == 0) {
            if (STATS) bytes += 8;
            const int bx = sx >> 2, by = sy >> 2, bz = sz >> 2;
            if (!bit64(tw, child_bit(bx & 3, by & 3, bz & 3))) {
                cell = 4;
            } else {
                const int64_t bi = (int64_t)bx + (int64_t)by * d.bx + (int64_t)bz * d.bx * d.by;
                const uint64_t occ = ldg(w.occ + bi);
                const int vi = child_bit(sx - bx * 4, sy - by * 4, sz - bz * 4);
                if (STATS) bytes += 8;
                if (bit64(occ, vi)) {
                    const uint32_t m = ldg(w.mat + bi * 64 + vi);
                    if (STATS) bytes += 1;
                    if (!is_transparent(m)) {
                        set_hit(d, s, la, m, false, h);
                        break;
                    }
                }
            }
        }
        if (cell != 0) skip_to_cell(d, ro, cell, s, la);
        else dda_step(d, s, t_cur, la);
    }
    h.steps = iters;
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

// ------------------------------------------------------------------ beam
// cs_beam + trace_first_tile, beam.wgsl:30-113 (world, non-rebased coords)
template <bool STATS>
__global__ void __launch_bounds__(128) k_beam(FrameArgs fa, float *beam_out) {
    const uint32_t gx = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gy = blockIdx.y;
    if (gx >= fa.bw || gy >= fa.bh) return;
    const VxCamera &c = fa.cam;
    const Dims &d = fa.ta.w.d;
    uint64_t bytes = 0, iters = 0;
    float dx, dy, dz;
    ray_dir_uv(c, ((float)gx * 8.0f + 4.0f) / c.res_x, ((float)gy * 8.0f + 4.0f) / c.res_y, dx,
               dy, dz);
    float result = 1e9f;
    const float ix = safe_inv(dx), iy = safe_inv(dy), iz = safe_inv(dz);
    const float wminx = (float)c.world_origin[0], wminy = (float)c.world_origin[1],
                wminz = (float)c.world_origin[2];
    const float wmaxx = wminx + (float)d.vx, wmaxy = wminy + (float)d.vy,
                wmaxz = wminz + (float)d.vz;
    const float t0x = (wminx - c.origin[0]) * ix, t1x = (wmaxx - c.origin[0]) * ix;
    const float t0y = (wminy - c.origin[1]) * iy, t1y = (wmaxy - c.origin[1]) * iy;
    const float t0z = (wminz - c.origin[2]) * iz, t1z = (wmaxz - c.origin[2]) * iz;
    const float t_enter = vmax(vmax(vmin(t0x, t1x), vmin(t0y, t1y)), vmax(vmin(t0z, t1z), 0.0f));
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
        float t_cur = t_enter;
        for (int s = 0; s < 80; ++s) {
            ++iters;
            if ((uint32_t)(tx - otx) >= (uint32_t)d.tx || (uint32_t)(ty - oty) >= (uint32_t)d.ty ||
                (uint32_t)(tz - otz) >= (uint32_t)d.tz)
                break;
            const int32_t stx = pos_mod(tx, d.tx), sty = ty, stz = pos_mod(tz, d.tz);
            const int64_t ci = (int64_t)(stx / 4) + (int64_t)(sty / 4) * d.cx +
                               (int64_t)(stz / 4) * d.cx * d.cy;
            const int lin = (stx & 3) + (stz & 3) * 4 + (sty & 3) * 16;
            if (STATS) bytes += 8;
            if (bit64(ldg(fa.ta.w.chunk_mask + ci), lin)) {
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

// ------------------------------------------------------------- primary
// One thread per pixel; a warp covers an 8x4 pixel tile, a 128-thread CTA a
// 16x8 region, so the 32 rays of a warp share one beam cell and start
// coherent.
template <bool STATS>
__global__ void __launch_bounds__(128) k_primary(FrameArgs fa) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t px = blockIdx.x * 16u + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t py = blockIdx.y * 8u + (warp >> 1) * 4u + (lane >> 3);
    if (px >= fa.W || py >= fa.H) return;
    const VxCamera &c = fa.cam;
    const VxTraceParams &p = fa.ta.p;
    const Ro ro{fa.ta.ro[0], fa.ta.ro[1], fa.ta.ro[2]};
    uint64_t bytes = 0;
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
    trace_ray<STATS>(fa.ta.w, p, ro, ox, oy, oz, dx, dy, dz, p.max_dist, h, bytes);
    if (beam_on && (h.flags & 1u)) h.t = h.t + skip;
    const size_t idx = (size_t)py * fa.W + px;
    store_record(fa.rec + idx, h);
    uint64_t iters = h.steps;
    if (fa.shadow) {
        VxShadowRecord sr;
        sr.steps = 0; sr.occluded = 0; sr.traced = 0; sr.pad = 0;
        if ((p.flags & VX_F_SHADOW) && (h.flags & 1u)) {
            // raymarch.wgsl:3953-3994: p_off = p_hit + n*0.001, cone jitter
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
            uint32_t ssteps;
            const bool occ = trace_any_ray<STATS>(fa.ta.w, p, ro, sox, soy, soz, sdx, sdy, sdz,
                                                  p.shadow_max_dist, ssteps, bytes);
            sr.steps = ssteps;
            sr.occluded = occ ? 1 : 0;
            sr.traced = 1;
            iters += ssteps;
        }
        fa.shadow[idx] = sr;
    }
    if (STATS) flush_stats(fa.stats, bytes, iters);
}

// --------------------------------------------------------- generic rays
__global__ void __launch_bounds__(128) k_trace_rays(TraceArgs ta, const VxRay *__restrict__ rays,
                                                    size_t n, VxHitRecord *out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = __ldg(reinterpret_cast<const float4 *>(rays + i));
    const float4 b = __ldg(reinterpret_cast<const float4 *>(rays + i) + 1);
    const uint32_t kind = __float_as_uint(b.w);
    const Ro ro{ta.ro[0], ta.ro[1], ta.ro[2]};
    uint64_t bytes = 0;
    Hit h;
    if (kind == 1u) {
        uint32_t steps;
        const bool occ = trace_any_ray<false>(ta.w, ta.p, ro, a.x, a.y, a.z, a.w, b.x, b.y, b.z,
                                              steps, bytes);
        set_miss(h);
        h.flags = occ ? 1u : 0u;
        h.steps = steps;
    } else if (kind == 2u) {
        trace_no_water_ray<false>(ta.w, ta.p, ro, a.x, a.y, a.z, a.w, b.x, b.y, b.z, h, bytes);
    } else {
        trace_ray<false>(ta.w, ta.p, ro, a.x, a.y, a.z, a.w, b.x, b.y, b.z, h, bytes);
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
    const uint64_t occ = ldg(w.occ + bi);
    if (occ == 0ull) return false;
    const int vi = child_bit(sx & 3, sy & 3, sz & 3);
    if (!bit64(occ, vi)) return false;
    return ldg(w.mat + bi * 64 + vi) != 33u;
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
    // glam 0.29.3 normalize_or_zero: self * (1 / sqrt(dot(self, self)))
    const float len = sqrtf((din[0] * din[0] + din[1] * din[1]) + din[2] * din[2]);
    const float rcp = 1.0f / len;
    do {
        if (!(isfinite(rcp) && rcp > 0.0f)) break;
        float dir[3] = {din[0] * rcp, din[1] * rcp, din[2] * rcp};
        if (dir[0] == 0.0f && dir[1] == 0.0f && dir[2] == 0.0f) break;
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
        if (t_enter >= t_exit || t_exit < 0.0f) break;
        int32_t voxel[3], step[3];
        float tdel[3], tm[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float pk = cam[k] + dir[k] * (t_enter + 1e-3f);
            pk = vmin(vmax(pk, wmin[k] + 1e-3f), wmax[k] - 1e-3f);
            voxel[k] = f2i(floorf(pk));
            step[k] = sgn(dir[k]);
            tdel[k] = fabsf(inv[k]);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float nxt = step[k] > 0 ? (float)(voxel[k] + 1) : (float)voxel[k];
            tm[k] = (nxt - cam[k]) * inv[k];
        }
        int last_axis = -1;
        int steps_left = 4096;
        bool dead = false;
        // argmin_step, raycast.rs:92-103 (ties go to the lowest axis)
        auto argmin_step = [&]() -> int {
            int a = -1;
            float m = __int_as_float(0x7f800000);
            if (step[0] != 0 && tm[0] < m) { a = 0; m = tm[0]; }
            if (step[1] != 0 && tm[1] < m) { a = 1; m = tm[1]; }
            if (step[2] != 0 && tm[2] < m) { a = 2; m = tm[2]; }
            if (a == 0) { voxel[0] += step[0]; tm[0] += tdel[0]; }
            else if (a == 1) { voxel[1] += step[1]; tm[1] += tdel[1]; }
            else if (a == 2) { voxel[2] += step[2]; tm[2] += tdel[2]; }
            return a;
        };
        while (steps_left > 0 && o1_in_solid(pa.w, voxel, o)) {
            const int ax = argmin_step();
            if (ax < 0) { dead = true; break; }
            last_axis = ax;
            steps_left--;
            if (!o1_in_window(d, voxel, o)) { dead = true; break; }
        }
        if (dead) break;
        while (steps_left > 0) {
            if (!o1_in_window(d, voxel, o)) break;
            if (o1_in_solid(pa.w, voxel, o)) {
                res.voxel[0] = voxel[0]; res.voxel[1] = voxel[1]; res.voxel[2] = voxel[2];
                const int sa = last_axis == 0 ? step[0] : (last_axis == 1 ? step[1] : step[2]);
                if (last_axis == 0) res.normal[0] = -sa;
                else if (last_axis == 1) res.normal[1] = -sa;
                else if (last_axis == 2) res.normal[2] = -sa;
                found = 1;
                break;
            }
            const int ax = argmin_step();
            if (ax < 0) break;
            last_axis = ax;
            steps_left--;
        }
    } while (0);
    out[i] = res;
    hit[i] = found;
}

}  // namespace

// ------------------------------------------------------------- launchers
cudaError_t launch_beam(const FrameArgs &fa, float *beam_out, cudaStream_t s) {
    dim3 block(128), grid((fa.bw + 127) / 128, fa.bh);
    if (fa.stats) k_beam<true><<<grid, block, 0, s>>>(fa, beam_out);
    else k_beam<false><<<grid, block, 0, s>>>(fa, beam_out);
    return cudaGetLastError();
}

cudaError_t launch_primary(const FrameArgs &fa, cudaStream_t s) {
    dim3 block(128), grid((fa.W + 15) / 16, (fa.H + 7) / 8);
    if (fa.stats) k_primary<true><<<grid, block, 0, s>>>(fa);
    else k_primary<false><<<grid, block, 0, s>>>(fa);
    return cudaGetLastError();
}

cudaError_t launch_trace_rays(const TraceArgs &ta, const VxRay *rays, size_t n, VxHitRecord *out,
                              cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((n + 127) / 128);
    k_trace_rays<<<blocks, 128, 0, s>>>(ta, rays, n, out);
    return cudaGetLastError();
}

cudaError_t launch_raycast(const DevWorld &w, const int32_t origin[3], const float *cams,
                           const float *dirs, size_t n, VxPickHit *out, int32_t *hit,
                           cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    PickArgs pa;
    pa.w = w;
    pa.origin[0] = origin[0]; pa.origin[1] = origin[1]; pa.origin[2] = origin[2];
    const unsigned blocks = (unsigned)((n + 127) / 128);
    k_raycast<<<blocks, 128, 0, s>>>(pa, cams, dirs, n, out, hit);
    return cudaGetLastError();
}

}  // namespace vx
