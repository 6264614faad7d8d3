// vx_learned.cu -- the learned-proposal form of the primary frame: per pixel
// the plain hierarchical DDA (trace(), method flags without the beam), but
// after its first iteration a cheap verification walk checks the ray segment
// up to the proposed start distance and, where it verifies, the DDA restarts
// from a point inside the last verified cell.  Records equal the plain DDA's
// bit for bit except `steps` (iterations actually executed).
//
// Why a restart is exact.  skip_to_cell (raymarch.wgsl:4807-4864) derives the
// whole DDA state (voxel, t_max, last axis, t_cur) from the cell it leaves
// and the ray alone, and the level decision of an iteration depends only on
// the current voxel's ancestors.  The verification walk steps along the ray
// through aligned cells -- a 64^3 chunk whose tile bits are all clear (L4
// method only), a 16^3 tile whose chunk bit is clear, or a 4^3 brick whose
// tile bit is clear inside a non-empty tile -- which are each contained in
// the cell the plain DDA skips from at that point.  Every face crossing is
// required to be "clean": the two other coordinates of the crossing point lie
// at least kClean from the faces of the finer of the two cells meeting there.
// Then each skip of the plain DDA lands in the cell the ray actually enters
// (its 1e-3 nudge and float rounding stay far below kClean), so the plain DDA
// visits a cell containing every verified cell, and a restart from a voxel of
// verified cell C performs the same skip as the plain DDA's iteration there.
// A verified empty brick or tile cannot stop the plain DDA: hits need a set
// voxel bit, and the tile LOD / uniform-tile early-outs need a non-empty tile
// entered beyond tile_lod_t (excluded: brick cells must end before
// tile_lod_t - kTEps) or a fully solid tile (whose bricks are not empty).
// The iteration cap is kept exact by starting the restarted walk's counter at
// the number of verified cells (an upper bound on the plain DDA's iterations
// across them); a restarted walk that still reaches the cap is replaced by the
// plain DDA from the origin.  A segment verified past the window or past
// max_dist + kTEps is a miss for the plain DDA too.
//
// The verification is restricted to windows whose corner is chunk-aligned in
// x/z with y = 0 (every verification cell then lies wholly inside or outside
// the window); other windows run the plain DDA.
#include <cuda_runtime.h>

#include "vx_walk.cuh"

namespace vx {
namespace {

constexpr float kClean = 0.01f;   // voxels from cell faces
constexpr float kTEps = 0.01f;    // t margin against max_dist / tile_lod_t
constexpr uint32_t kMaxCells = 4096u;

enum : uint32_t { OUT_NONE = 0, OUT_PARTIAL = 1, OUT_ACCEPTED = 2, OUT_MISS = 3 };

// x at least kClean from every multiple of g (g a power of two, ig = 1/g
// exactly, so x * ig is exact)
__device__ __forceinline__ bool clean_at(float x, float g, float ig) {
    const float r = x - g * floorf(x * ig);
    return r >= kClean && r <= g - kClean;
}
__device__ __forceinline__ float inv_level(int g) {
    return g == 4 ? 0.25f : (g == 16 ? 0.0625f : 0.015625f);
}

struct Slots {
    int32_t rox, roz;  // pos_mod(window corner x/z, dims)
};

// Level of the cell holding rebased voxel (lx, ly, lz) inside the window:
// 64 = empty chunk (L4 method only), 16 = empty tile, 4 = empty brick of a
// non-empty tile, 0 = non-empty brick.
template <bool L4>
__device__ __forceinline__ int cell_level(const DevWorld &w, const Geo &g, const Slots &sl,
                                          int32_t lx, int32_t ly, int32_t lz) {
    int32_t sx = lx + sl.rox, sz = lz + sl.roz;
    if (sx >= w.d.vx) sx -= w.d.vx;
    if (sz >= w.d.vz) sz -= w.d.vz;
    const uint32_t ux = (uint32_t)sx, uy = (uint32_t)ly, uz = (uint32_t)sz;
    const uint64_t cw = ld_chunk(w, chunk_index(g, ux, uy, uz));
    if (L4 && cw == 0ull) return 64;
    if (!bit64(cw, child_of(ux, uy, uz, 4))) return 16;
    const uint64_t tw = ld_tile(w, tile_index(g, ux, uy, uz));
    if (!bit64(tw, child_of(ux, uy, uz, 2))) return 4;
    return 0;
}

struct Verdict {
    uint32_t outcome;
    uint32_t cells;       // verification cells stepped
    uint32_t good_cells;  // cells up to and including the restart cell
    float t_r;            // restart t (midpoint of the restart cell's segment)
    int32_t r[3];         // restart voxel (rebased)
};

template <typename T>
__device__ __forceinline__ T sel3(int a, T x, T y, T z) { return a == 0 ? x : (a == 1 ? y : z); }

// Restart point of a verified cell whose ray segment is [a, b]: its midpoint,
// usable when it lies at least kClean inside the cell on every axis.
__device__ __forceinline__ bool restart_in(const Dda &s, float a, float b, int gs, Verdict &v) {
    const float gf = (float)gs, ig = inv_level(gs);
    const float tm = 0.5f * (a + b);
    const float mx = s.ox + s.dx * tm, my = s.oy + s.dy * tm, mz = s.oz + s.dz * tm;
    if (!(clean_at(mx, gf, ig) && clean_at(my, gf, ig) && clean_at(mz, gf, ig))) return false;
    v.t_r = tm;
    v.r[0] = f2i(floorf(mx));
    v.r[1] = f2i(floorf(my));
    v.r[2] = f2i(floorf(mz));
    return true;
}

// Mask words of rebased tile (tx, ty, tz): the chunk word (its tile bits)
// and the tile word (its brick bits).  The window corner is chunk-aligned,
// so rebased and slot coordinates agree modulo 4 at every level.
__device__ __forceinline__ uint64_t chunk_word_of(const DevWorld &w, const Geo &g,
                                                  const Slots &sl, int32_t tx, int32_t ty,
                                                  int32_t tz) {
    int32_t sx = (tx << 4) + sl.rox, sz = (tz << 4) + sl.roz;
    if (sx >= w.d.vx) sx -= w.d.vx;
    if (sz >= w.d.vz) sz -= w.d.vz;
    return ld_chunk(w, chunk_index(g, (uint32_t)sx, (uint32_t)(ty << 4), (uint32_t)sz));
}
__device__ __forceinline__ uint64_t tile_word_of(const DevWorld &w, const Geo &g, const Slots &sl,
                                                 int32_t tx, int32_t ty, int32_t tz) {
    int32_t sx = (tx << 4) + sl.rox, sz = (tz << 4) + sl.roz;
    if (sx >= w.d.vx) sx -= w.d.vx;
    if (sz >= w.d.vz) sz -= w.d.vz;
    return ld_tile(w, tile_index(g, (uint32_t)sx, (uint32_t)(ty << 4), (uint32_t)sz));
}
// child bit x + z*4 + y*16 of cell coordinates (any level)
__device__ __forceinline__ int cbit(int32_t x, int32_t y, int32_t z) {
    return (x & 3) + (z & 3) * 4 + (y & 3) * 16;
}
// t at which the ray leaves cell c (size gs) along an axis
__device__ __forceinline__ float exit_t(int32_t c, int gs, int32_t st, float o, float iv) {
    return st == 0 ? 1e30f : ((float)((c + (st > 0 ? 1 : 0)) * gs) - o) * iv;
}

// Verification walk from the plain DDA's state after one iteration (voxel in
// s, last crossing on axis la) up to t_target: an incremental DDA over tiles,
// descending to bricks inside non-empty tiles.  Each step recomputes only the
// exit time of the axis it crossed and tests one cached mask word; the
// restart point is chosen once, in the last verified cell (or the one before).
template <uint32_t FL>
__device__ __forceinline__ void verify(const DevWorld &w, const Geo &g, const VxTraceParams &p,
                                       Ro ro, const Slots &sl, const Dda &s, int la,
                                       float t_target, float tmax, Verdict &v) {
    constexpr bool L4 = (FL & VX_F_L4) != 0u;
    constexpr bool LOD = (FL & VX_F_LOD) != 0u;
    const Dims &d = w.d;
    const int32_t lx = s.vx - ro.x, ly = s.vy - ro.y, lz = s.vz - ro.z;
    v.outcome = OUT_NONE;
    v.cells = 0;
    v.good_cells = 0;
    if (la < 0) return;
    if ((uint32_t)lx >= (uint32_t)d.vx || (uint32_t)ly >= (uint32_t)d.vy ||
        (uint32_t)lz >= (uint32_t)d.vz)
        return;
    const int lvl = cell_level<L4>(w, g, sl, lx, ly, lz);
    if (lvl == 0) return;
    bool bricks = lvl == 4;  // walking bricks of a non-empty tile
    // the crossing that led into the current voxel, clean at the cell's level
    float tin;
    {
        const int gs = bricks ? 4 : 16;
        const int32_t lv = sel3(la, lx, ly, lz);
        const int32_t st = sel3(la, s.stx, s.sty, s.stz);
        const float pl = (float)(st > 0 ? lv : lv + 1);
        tin = (pl - sel3(la, s.ox, s.oy, s.oz)) * sel3(la, s.ix, s.iy, s.iz);
        const float x = s.ox + s.dx * tin, y = s.oy + s.dy * tin, z = s.oz + s.dz * tin;
        const float gf = (float)gs, ig = inv_level(gs);
        const int32_t hi = ~(gs - 1);
        if (la != 0 && (!clean_at(x, gf, ig) || (f2i(floorf(x)) & hi) != (lx & hi))) return;
        if (la != 1 && (!clean_at(y, gf, ig) || (f2i(floorf(y)) & hi) != (ly & hi))) return;
        if (la != 2 && (!clean_at(z, gf, ig) || (f2i(floorf(z)) & hi) != (lz & hi))) return;
    }
    const int32_t ntx = d.vx >> 4, nty = d.vy >> 4, ntz = d.vz >> 4;
    int32_t tx = lx >> 4, ty = ly >> 4, tz = lz >> 4;
    float ttx = exit_t(tx, 16, s.stx, s.ox, s.ix);
    float tty = exit_t(ty, 16, s.sty, s.oy, s.iy);
    float ttz = exit_t(tz, 16, s.stz, s.oz, s.iz);
    uint64_t cw = chunk_word_of(w, g, sl, tx, ty, tz);
    int32_t bx = lx >> 2, by = ly >> 2, bz = lz >> 2;
    uint64_t tw = 0;
    float tbx = 0.f, tby = 0.f, tbz = 0.f;
    if (bricks) {
        tw = tile_word_of(w, g, sl, tx, ty, tz);
        tbx = exit_t(bx, 4, s.stx, s.ox, s.ix);
        tby = exit_t(by, 4, s.sty, s.oy, s.iy);
        tbz = exit_t(bz, 4, s.stz, s.oz, s.iz);
    }
    // Clean crossings from exit times: at a crossing at time t, axis b lies
    // at least kClean inside its current slab of size gs iff
    // lo_b <= e_b - t <= gs |1/d_b| - lo_b with lo_b = kClean |1/d_b| (e_b the
    // slab's exit time).  An axis the ray does not move along is tested once
    // on its constant coordinate (lo = -inf: always clean, +inf: never).
    const float aix = fabsf(s.ix), aiy = fabsf(s.iy), aiz = fabsf(s.iz);
    const float kInf = __int_as_float(0x7f800000);
    auto lo_of = [&](int32_t st, float ai, float o) {
        if (st != 0 && ai < 1e29f) return kClean * ai;
        return clean_at(o, 16.0f, 0.0625f) && clean_at(o, 4.0f, 0.25f) ? -kInf : kInf;
    };
    const float lox = lo_of(s.stx, aix, s.ox), loy = lo_of(s.sty, aiy, s.oy),
                loz = lo_of(s.stz, aiz, s.oz);
    float l_a = 0.f, l_b = 0.f, p_a = 0.f, p_b = 0.f;
    int l_g = 0, p_g = 0;
    bool reached = false;
    uint32_t cells = 0;
    const float t_near = tmax - kTEps;
    for (uint32_t it = 0; it < kMaxCells; ++it) {
        if (tin > t_near) {
            if (tin > tmax + kTEps) {
                v.outcome = OUT_MISS;
                v.cells = cells;
                return;
            }
            break;
        }
        const int gs = bricks ? 4 : 16;
        const float ex = bricks ? tbx : ttx, ey = bricks ? tby : tty, ez = bricks ? tbz : ttz;
        int ax = 0;
        float tout = ex;
        if (ey < tout) { ax = 1; tout = ey; }
        if (ez < tout) { ax = 2; tout = ez; }
        if (!(tout > tin)) break;
        if (LOD && bricks && tout > p.tile_lod_t - kTEps) break;
        ++cells;
        p_a = l_a; p_b = l_b; p_g = l_g;
        l_a = tin; l_b = tout; l_g = gs;
        if (t_target < tout) {
            reached = true;
            break;
        }
        // the crossing point must sit clear of the faces of this level
        {
            const float gf = (float)gs;
            const float qx = ex - tout, qy = ey - tout, qz = ez - tout;
            const bool cx_ = ax == 0 || (qx >= lox && qx <= gf * aix - lox);
            const bool cy_ = ax == 1 || (qy >= loy && qy <= gf * aiy - loy);
            const bool cz_ = ax == 2 || (qz >= loz && qz <= gf * aiz - loz);
            if (!(cx_ && cy_ && cz_)) break;
        }
        tin = tout;
        // step along ax; stay in the tile (brick walk) or move to the next tile
        bool new_tile = true;
        if (bricks) {
            const int32_t nb = sel3(ax, bx, by, bz) + sel3(ax, s.stx, s.sty, s.stz);
            if ((nb >> 2) == sel3(ax, tx, ty, tz)) {
                new_tile = false;
                if (ax == 0) { bx = nb; tbx = exit_t(bx, 4, s.stx, s.ox, s.ix); }
                else if (ax == 1) { by = nb; tby = exit_t(by, 4, s.sty, s.oy, s.iy); }
                else { bz = nb; tbz = exit_t(bz, 4, s.stz, s.oz, s.iz); }
                if (bit64(tw, cbit(bx, by, bz))) break;  // non-empty brick
            }
        }
        if (!new_tile) continue;
        {
            const int32_t nt = sel3(ax, tx, ty, tz) + sel3(ax, s.stx, s.sty, s.stz);
            if ((uint32_t)nt >= (uint32_t)sel3(ax, ntx, nty, ntz)) {
                v.outcome = OUT_MISS;  // leaves the window through a clean crossing
                v.cells = cells;
                return;
            }
            const int32_t oc = sel3(ax, tx, ty, tz) >> 2;
            if (ax == 0) { tx = nt; ttx = exit_t(tx, 16, s.stx, s.ox, s.ix); }
            else if (ax == 1) { ty = nt; tty = exit_t(ty, 16, s.sty, s.oy, s.iy); }
            else { tz = nt; ttz = exit_t(tz, 16, s.stz, s.oz, s.iz); }
            if ((nt >> 2) != oc) cw = chunk_word_of(w, g, sl, tx, ty, tz);
        }
        if (!bit64(cw, cbit(tx, ty, tz))) {
            bricks = false;  // an empty tile (the crossing was checked at 4 or 16)
            continue;
        }
        // a non-empty tile: plain's tile LOD / uniform test happen at its entry
        if (LOD && tout > p.tile_lod_t - kTEps) break;
        if (!bricks) {
            // entering bricks from the tile walk: the crossing must also clear
            // the brick faces (crossing coordinates, tested directly)
            const float ig = 0.25f;
            const float xx = s.ox + s.dx * tout, xy = s.oy + s.dy * tout, xz = s.oz + s.dz * tout;
            if (!((ax == 0 || clean_at(xx, 4.0f, ig)) && (ax == 1 || clean_at(xy, 4.0f, ig)) &&
                  (ax == 2 || clean_at(xz, 4.0f, ig))))
                break;
            bx = ax == 0 ? (s.stx > 0 ? tx * 4 : tx * 4 + 3) : (f2i(floorf(xx)) >> 2);
            by = ax == 1 ? (s.sty > 0 ? ty * 4 : ty * 4 + 3) : (f2i(floorf(xy)) >> 2);
            bz = ax == 2 ? (s.stz > 0 ? tz * 4 : tz * 4 + 3) : (f2i(floorf(xz)) >> 2);
            tbx = exit_t(bx, 4, s.stx, s.ox, s.ix);
            tby = exit_t(by, 4, s.sty, s.oy, s.iy);
            tbz = exit_t(bz, 4, s.stz, s.oz, s.iz);
            bricks = true;
        } else {
            // brick walk continuing into the next tile along ax
            if (ax == 0) { bx += s.stx; tbx = exit_t(bx, 4, s.stx, s.ox, s.ix); }
            else if (ax == 1) { by += s.sty; tby = exit_t(by, 4, s.sty, s.oy, s.iy); }
            else { bz += s.stz; tbz = exit_t(bz, 4, s.stz, s.oz, s.iz); }
        }
        tw = tile_word_of(w, g, sl, tx, ty, tz);
        if (bit64(tw, cbit(bx, by, bz))) break;  // non-empty brick at the entry
    }
    v.cells = cells;
    if (l_g && restart_in(s, l_a, l_b, l_g, v)) {
        v.good_cells = cells;
        v.outcome = reached ? OUT_ACCEPTED : OUT_PARTIAL;
    } else if (p_g && restart_in(s, p_a, p_b, p_g, v)) {
        v.good_cells = cells - 1;
        v.outcome = OUT_PARTIAL;
    }
}

struct LearnedArgs {
    TraceArgs ta;
    VxCamera cam;
    uint32_t W, H;
    const float *proposal;     // log t per pixel, or nullptr = verify until a failure
    float scale;               // t_target = exp(proposal) * scale
    VxHitRecord *rec;
    unsigned long long *stats; // [none, partial, accepted, miss, cells, iters, fallback, rays]
    bool verify_on;            // window suits the verification
    Slots sl;
};

template <uint32_t FL>
__global__ void __launch_bounds__(128, 8) k_learned(LearnedArgs la) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t px = blockIdx.x * 16u + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t py = blockIdx.y * 8u + (warp >> 1) * 4u + (lane >> 3);
    const bool live = px < la.W && py < la.H;
    uint32_t outcome = OUT_NONE, cells = 0, iters = 0, fallback = 0;
    if (live) {
        const DevWorld &w = la.ta.w;
        const Ro ro{la.ta.ro[0], la.ta.ro[1], la.ta.ro[2]};
        const Geo g = geo_of<FL>(w.d, ro);
        const VxTraceParams &p = la.ta.p;
        const VxCamera &c = la.cam;
        float dx, dy, dz;
        const float u = (((float)px + 0.5f) + c.jitter_x) / c.res_x;
        const float vv = (((float)py + 0.5f) + c.jitter_y) / c.res_y;
        ray_dir_uv(c, u, vv, dx, dy, dz);
        const float ox = c.origin[0], oy = c.origin[1], oz = c.origin[2];
        const size_t idx = (size_t)py * la.W + px;
        Hit h;
        set_miss(h);
        uint64_t bytes = 0;
        Walk k;
        if (!walk_init(w.d, ro, KIND_TRACE, p, ox, oy, oz, dx, dy, dz, p.max_dist, k)) {
            h.steps = 0;
        } else {
            int r = walk_step<FL, false, KIND_TRACE>(w, g, p, ro, k, h, bytes);
            uint32_t executed = 1;
            if (r == WALK_CONT && la.verify_on) {
                float t_target = 3.0e38f;
                if (la.proposal) t_target = expf(la.proposal[idx]) * la.scale;
                Verdict vd;
                if (t_target > k.t_cur) {
                    verify<FL>(w, g, p, ro, la.sl, k.s, k.la, t_target, p.max_dist, vd);
                    outcome = vd.outcome;
                    cells = vd.cells;
                    if (outcome == OUT_MISS) {
                        r = WALK_END;
                    } else if (outcome != OUT_NONE) {
                        // restart inside the last verified cell
                        Dda &s = k.s;
                        s.vx = vd.r[0] + ro.x;
                        s.vy = vd.r[1] + ro.y;
                        s.vz = vd.r[2] + ro.z;
                        k.t_cur = vd.t_r;
                        k.la = -1;
                        k.iters = vd.good_cells;
                    }
                }
            }
            const uint32_t base = k.iters;
            while (r == WALK_CONT) r = walk_step<FL, false, KIND_TRACE>(w, g, p, ro, k, h, bytes);
            executed += k.iters - base;
            if (r == WALK_END && k.iters >= k.cap && outcome != OUT_NONE && outcome != OUT_MISS) {
                // the inflated counter reached the cap: the plain DDA decides
                fallback = 1;
                set_miss(h);
                walk_init(w.d, ro, KIND_TRACE, p, ox, oy, oz, dx, dy, dz, p.max_dist, k);
                while (walk_step<FL, false, KIND_TRACE>(w, g, p, ro, k, h, bytes) == WALK_CONT) {
                }
                executed += k.iters;
            }
            h.steps = executed;
            iters = executed;
        }
        store_record(la.rec + idx, h);
    }
    if (la.stats) {
        const unsigned FULL = 0xFFFFFFFFu;
        const uint32_t n_none = __reduce_add_sync(FULL, live && outcome == OUT_NONE ? 1u : 0u);
        const uint32_t n_part = __reduce_add_sync(FULL, live && outcome == OUT_PARTIAL ? 1u : 0u);
        const uint32_t n_acc = __reduce_add_sync(FULL, live && outcome == OUT_ACCEPTED ? 1u : 0u);
        const uint32_t n_miss = __reduce_add_sync(FULL, live && outcome == OUT_MISS ? 1u : 0u);
        const uint32_t n_cells = __reduce_add_sync(FULL, cells);
        const uint32_t n_iters = __reduce_add_sync(FULL, iters);
        const uint32_t n_fb = __reduce_add_sync(FULL, fallback);
        const uint32_t n_live = __reduce_add_sync(FULL, live ? 1u : 0u);
        if (lane == 0) {
            atomicAdd(la.stats + 0, (unsigned long long)n_none);
            atomicAdd(la.stats + 1, (unsigned long long)n_part);
            atomicAdd(la.stats + 2, (unsigned long long)n_acc);
            atomicAdd(la.stats + 3, (unsigned long long)n_miss);
            atomicAdd(la.stats + 4, (unsigned long long)n_cells);
            atomicAdd(la.stats + 5, (unsigned long long)n_iters);
            atomicAdd(la.stats + 6, (unsigned long long)n_fb);
            atomicAdd(la.stats + 7, (unsigned long long)n_live);
        }
    }
}

template <uint32_t FL>
struct LearnedK {
    static void *fn() { return reinterpret_cast<void *>(&k_learned<FL>); }
};

}  // namespace

cudaError_t launch_learned(const TraceArgs &ta, const VxCamera &cam, const float *proposal,
                           float scale, VxHitRecord *rec, unsigned long long *stats,
                           cudaStream_t stream) {
    LearnedArgs la{};
    la.ta = ta;
    la.cam = cam;
    la.W = (uint32_t)cam.res_x;
    la.H = (uint32_t)cam.res_y;
    la.proposal = proposal;
    la.scale = scale;
    la.rec = rec;
    la.stats = stats;
    const Dims &d = ta.w.d;
    la.verify_on = (ta.ro[0] & 63) == 0 && (ta.ro[2] & 63) == 0 && ta.ro[1] == 0;
    la.sl.rox = ((ta.ro[0] % d.vx) + d.vx) % d.vx;
    la.sl.roz = ((ta.ro[2] % d.vz) + d.vz) % d.vz;
    const dim3 grid((la.W + 15u) / 16u, (la.H + 7u) / 8u);
    const uint32_t fl = (ta.p.flags & (VX_F_L4 | VX_F_LUT | VX_F_LOD)) | pow2_bit(d);
    void *args[] = {&la};
    const void *fn = pick_fl<LearnedK>(fl);
    return cudaLaunchKernel(fn, grid, dim3(128), args, 0, stream);
}

}  // namespace vx
