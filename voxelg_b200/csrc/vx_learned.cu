// vx_learned.cu -- the learned-proposal form of the primary frame: per pixel
// the plain hierarchical DDA (trace(), method flags without the beam), but
// first a verification walk proves the ray's segment from the camera up to
// the proposed start distance empty, and the DDA restarts from a point inside
// that segment.  Records equal the plain DDA's bit for bit except `steps`
// (iterations actually executed).
//
// Verification.  Two empty-space distance fields (vx_distfield.cu) give, per
// tile and per brick, the Chebyshev distance to the nearest non-empty cell of
// that level.  From the current point the walk takes one of three steps:
//   tile box   tile field D >= 2: every tile within D-1 of the current tile
//              is empty; jump to where the ray leaves that cube of tiles,
//              ending kMu inside its face;
//   brick box  else brick field D >= 2: the same with the cube of bricks;
//   brick walk else brick field D == 1 (this brick empty, a neighbour not):
//              cross into the next brick along the ray, requiring the
//              crossing to be clean (the other coordinates at least kClean
//              from brick planes) and stopping at the first non-empty brick.
// It stops at the proposal, at a non-empty brick, at a failed check, or when
// the proven segment passes max_dist or the window exit (a verified miss).
//
// Why a restart is exact (window corner a multiple of 16 in x and z, camera
// inside the window; all coordinates below are window-relative, so brick,
// tile, chunk and L4 planes are multiples of 4 and the plain DDA's cells are
// bounded by such planes):
//  1. A plain iteration at voxel V skips the coarsest empty cell holding V
//     (L4 / chunk / tile / brick), and skip_to_cell (raymarch.wgsl:4807-4864)
//     derives the next state from that cell and the ray alone: it lands at
//     floor(o + d (t_min + 1e-3)) with the crossed axis snapped, t_min the
//     cell's first forward face.  So every voxel the plain DDA visits
//     contains a point within eps (rounding of o + d t, a few 1e-4 at most)
//     of the ray at time t_min + 1e-3.
//  2. Every such voxel up to the restart lies in proven-empty space: box
//     steps end kMu (> 1e-3 + eps) inside their cubes, and walk crossings are
//     clean, so the plain DDA lands exactly in the walk's bricks.  Empty
//     cells only ever skip: no hit, and no LUT early-out (a uniform tile or
//     brick is full).  The tile LOD test runs only in non-empty tiles, so
//     brick steps end before tile_lod_t (tile boxes hold no non-empty tile).
//  3. The plain DDA makes progress: its t_min strictly increases.  On the
//     crossed axis the next face is 4 voxels on; on another axis a with
//     |d_a| >= delta the rounding of the landing moves the next face's time
//     back by at most eps/|d_a| < 1e-3 - (time rounding), the nudge.  Axes
//     with |d_a| < delta are checked explicitly in box steps: at each of
//     their brick-plane crossings no other plane crossing lies within the
//     window in which a landing could round to the wrong side (walk
//     crossings are clean, which covers them).  Axes with |d_a| < 1e-6
//     never carry a forward face and are required to sit clear of planes.
//  4. Let P = ray(t_P) be the restart point, at least kClean from every
//     brick plane, and C* the plain DDA's cell for floor(P).  The first
//     plain iteration whose t_min exceeds t_P starts at a voxel within eps
//     of the ray at a time <= t_P + 1e-3, inside a cell whose forward faces
//     all lie beyond t_P; that cell therefore meets C*, and aligned cells
//     that meet are nested, and both are the coarsest empty cell of their
//     voxels -- it is C*.  A DDA restarted at floor(P) skips from C* too and
//     is bit-identical from there on: same voxel, face, material and t.
//  5. Iteration cap: each plain iteration before C*'s crosses a distinct
//     brick-aligned plane (t_min increases), so their number is at most
//     the brick planes between camera and P.  The restarted counter starts
//     at that bound; a restarted walk that still reaches the cap is replaced
//     by the plain DDA from the camera.
//  6. A segment proven empty past max_dist + kTEps or past the window exit
//     is a miss for the plain DDA too.
// The proposal (a per-block network output) only decides how far to verify.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "vx_mlp_infer.cuh"
#include "vx_walk.cuh"

namespace vx {
namespace {

constexpr float kMu = 0.02f;      // box steps end this far inside the cube (voxels)
constexpr float kClean = 0.01f;   // walk crossings and restart points: distance from brick planes
constexpr float kTEps = 0.05f;    // t margin past max_dist / window exit, before tile_lod_t
constexpr float kFixed = 1e-6f;   // |d| below this: the axis never carries a forward face

enum : uint32_t { OUT_NONE = 0, OUT_PARTIAL = 1, OUT_ACCEPTED = 2, OUT_MISS = 3 };

// distance of x from the nearest multiple of 4 (exact in binary32)
__device__ __forceinline__ float plane_dist4(float x) {
    const float r = x - 4.0f * floorf(x * 0.25f);
    return fminf(r, 4.0f - r);
}

struct VerifyArgs {
    int32_t sbx, sbz;     // slot of window-relative brick 0 / tile 0 in x and z
    int32_t stx, stz;
    int32_t ob[3];        // brick of the camera (window-relative, per frame)
    float delta;          // axes with |d| below: small (explicit crossing checks)
    float coord_eps;      // bound on the plain DDA's landing rounding (voxels)
    float t_eps;          // bound on its time rounding
};

// Frustum tiles: one 8 x 4 pixel tile per warp of the frame kernel; one
// proposal per 16 x 8 pixels (four tiles).
constexpr uint32_t kTileW = kLearnedTileW, kTileH = kLearnedTileH;
constexpr uint32_t kPropW = kLearnedPropW, kPropH = kLearnedPropH;
// A bundle's proof takes at most this many box steps: the pass lasts as long
// as its longest proof, and on the 512x256x512 benchmark frame 99.9% of the
// tiles need fewer (capping at 24 leaves 0.2% more DDA iterations than no cap)
constexpr uint32_t kFrustumSteps = 24u;

struct FrustumArgs {
    DevWorld w;
    VxTraceParams p;
    VxCamera cam;
    int32_t ro[3];
    uint32_t W, H, tiles_x, tiles_y;
    VerifyArgs va;
    float *depth;              // per tile: proven depth
    unsigned long long *stats; // stats[4] += box steps, or nullptr
};

// The frustum pre-pass: one thread per 8 x 4 pixel tile.  The rays of the
// tile share the camera; with dmin / dmax the per-axis extremes of their
// directions (widened by 1e-6 over the rounding of the approximate
// normalisation used here), every ray's point at time t >= 0 lies in the box
// [o + t dmin, o + t dmax].  Box steps then prove the whole bundle's segment
// [0, depth] empty: from the box around the bundle's centre brick (tile
// field D >= 2: the cube of tiles within D-1; else brick field D >= 2: the
// cube of bricks), require the bundle's cross-section at t inside the cube
// shrunk by kMu and advance to the first time a side of the bundle's box
// reaches the shrunk cube's face.  Brick cubes stop before tile_lod_t (they
// may hold non-empty tiles); tile cubes hold none.
template <uint32_t FL>
__device__ __forceinline__ void frustum_body(const FrustumArgs &fa, uint32_t cta) {
    constexpr bool LOD = (FL & VX_F_LOD) != 0u;
    const uint32_t i0 = cta * blockDim.x + threadIdx.x;
    const bool live = i0 < fa.tiles_x * fa.tiles_y;
    const uint32_t i = live ? i0 : 0u;  // dead lanes redo tile 0 and store nothing
    const uint32_t tx = i % fa.tiles_x, ty = i / fa.tiles_x;
    const VxCamera &c = fa.cam;
    const Dims &D = fa.w.d;
    float dmin[3] = {3.0e38f, 3.0e38f, 3.0e38f}, dmax[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
    // the tile's screen offsets, in ray_dir_uv's operation order (so each
    // unnormalised direction below equals the frame kernel's bit for bit)
    const float aspect = c.res_x / c.res_y;
    float ax[kTileW], by[kTileH];
#pragma unroll
    for (uint32_t lx = 0; lx < kTileW; ++lx) {
        const uint32_t px = min(tx * kTileW + lx, fa.W - 1u);
        const float u = (((float)px + 0.5f) + c.jitter_x) / c.res_x;
        ax[lx] = (u * 2.0f - 1.0f) * c.tan_half_fov * aspect;
    }
#pragma unroll
    for (uint32_t ly = 0; ly < kTileH; ++ly) {
        const uint32_t py = min(ty * kTileH + ly, fa.H - 1u);
        const float v = (((float)py + 0.5f) + c.jitter_y) / c.res_y;
        by[ly] = (1.0f - v * 2.0f) * c.tan_half_fov;
    }
#pragma unroll
    for (uint32_t ly = 0; ly < kTileH; ++ly) {
        float fu[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) fu[k] = c.up[k] * by[ly];
#pragma unroll
        for (uint32_t lx = 0; lx < kTileW; ++lx) {
            float q[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) q[k] = (c.forward[k] + c.right[k] * ax[lx]) + fu[k];
            const float inv = rsqrtf((q[0] * q[0] + q[1] * q[1]) + q[2] * q[2]);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                dmin[k] = fminf(dmin[k], q[k] * inv);
                dmax[k] = fmaxf(dmax[k], q[k] * inv);
            }
        }
    }
    float o[3], dm[3], rmin[3], rmax[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dmin[k] -= 1e-6f;
        dmax[k] += 1e-6f;
        dm[k] = 0.5f * (dmin[k] + dmax[k]);
        o[k] = c.origin[k] - (float)fa.ro[k];
        // exit times use reciprocals, rounded toward zero so that each exit
        // time is never later than the exact quotient's
        rmin[k] = dmin[k] < 0.0f ? __frcp_rz(dmin[k]) : 0.0f;
        rmax[k] = dmax[k] > 0.0f ? __frcp_rz(dmax[k]) : 0.0f;
    }
    float t = 0.0f;
    uint32_t steps = 0;
    const uint32_t txy = (uint32_t)(D.tx * D.ty), bxy = (uint32_t)(D.bx * D.by);
    while (steps < kFrustumSteps) {
        int32_t bl[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) bl[k] = (int32_t)floorf((o[k] + dm[k] * t) * 0.25f);
        if ((uint32_t)bl[0] >= (uint32_t)D.bx || (uint32_t)bl[1] >= (uint32_t)D.by ||
            (uint32_t)bl[2] >= (uint32_t)D.bz)
            break;
        // both fields' bytes are loaded together (one round of latency)
        int32_t sx = (bl[0] >> 2) + fa.va.stx, sz = (bl[2] >> 2) + fa.va.stz;
        if (sx >= D.tx) sx -= D.tx;
        if (sz >= D.tz) sz -= D.tz;
        int32_t bx = bl[0] + fa.va.sbx, bz = bl[2] + fa.va.sbz;
        if (bx >= D.bx) bx -= D.bx;
        if (bz >= D.bz) bz -= D.bz;
        const int32_t dt = (int32_t)__ldg(fa.w.tdf + (uint32_t)sx + (uint32_t)(bl[1] >> 2) * (uint32_t)D.tx +
                                         (uint32_t)sz * txy);
        const int32_t db = (int32_t)__ldg(fa.w.bdf + (uint32_t)bx + (uint32_t)bl[1] * (uint32_t)D.bx +
                                         (uint32_t)bz * bxy);
        float lo[3], hi[3];
        // the larger of the two cubes (radii beyond the centre cell, voxels);
        // only a tile cube holds no non-empty tile (the tile LOD test)
        const bool tile_box = dt >= 2 && 16 * (dt - 1) >= 4 * (db - 1);
        if (!tile_box && db < 2) break;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            lo[k] = tile_box ? 16.0f * (float)((bl[k] >> 2) - (dt - 1)) + kMu
                             : 4.0f * (float)(bl[k] - (db - 1)) + kMu;
            hi[k] = tile_box ? 16.0f * (float)((bl[k] >> 2) + dt) - kMu
                             : 4.0f * (float)(bl[k] + db) - kMu;
        }
        bool inside = true;
        float t_out = 3.0e38f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (!(o[k] + t * dmin[k] >= lo[k] && o[k] + t * dmax[k] <= hi[k])) inside = false;
            if (dmax[k] > 0.0f) t_out = fminf(t_out, (hi[k] - o[k]) * rmax[k]);
            if (dmin[k] < 0.0f) t_out = fminf(t_out, (lo[k] - o[k]) * rmin[k]);
        }
        if (!inside || !(t_out > t)) break;
        ++steps;
        bool stop = false;
        if (LOD && !tile_box && t_out > fa.p.tile_lod_t - kTEps) {
            t_out = fa.p.tile_lod_t - kTEps;
            stop = true;
        }
        if (t_out > t) t = t_out;
        if (stop || t > fa.p.max_dist + kTEps) break;
    }
    if (live) fa.depth[i] = t;
    if (fa.stats) {
        const uint32_t n = __reduce_add_sync(0xFFFFFFFFu, live ? steps : 0u);
        if ((threadIdx.x & 31u) == 0u) atomicAdd(fa.stats + 4, (unsigned long long)n);
    }
}

// The learned frame's pre-pass, one launch: CTAs [0, frustum_ctas) prove the
// tiles' bundles, the rest infer the proposals (the network's 16-ray passes),
// so the inference runs inside the time the latency-bound proofs take.  It
// lets the frame kernel launch at once (programmatic dependent launch): the
// frame kernel's per-pixel set-up runs meanwhile, and it waits for this grid
// before it reads what this grid writes.
template <uint32_t FL>
__global__ void __launch_bounds__(128) k_prepass(FrustumArgs fa, InferArgs ia,
                                                 uint32_t frustum_ctas, uint32_t infer_ctas) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (blockIdx.x < frustum_ctas) frustum_body<FL>(fa, blockIdx.x);
    else mlp_infer_body<true>(ia, blockIdx.x - frustum_ctas, infer_ctas);
}

struct Restart {
    float t;              // restart time
    uint32_t bound;       // plain iterations before the restart cell, at most
};

// Small axes (0 < |d_k| < delta): every brick-plane crossing of axis k ahead
// of the camera with time in (t_from - 2e-3, t_to + 2e-3] must keep the
// plane crossings of the other axes (ahead of the camera) out of the window
// where the plain DDA's landing after one of them could round to the wrong
// side of axis k's plane.  Returns the time of the first crossing that
// fails, or 3e38; counts the crossings checked.
__device__ __forceinline__ float small_axis_fail(const VerifyArgs &va, const float o[3],
                                                 const float d[3], const float iv[3],
                                                 const int32_t st[3], const bool fixed[3],
                                                 const bool small[3], float t_from, float t_to,
                                                 uint32_t &checks) {
    float fail = 3.0e38f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (!small[k]) continue;
        const float win = va.coord_eps / fabsf(d[k]) + va.t_eps + 1e-4f;
        const float xk = o[k] + d[k] * fmaxf(t_from - 2e-3f, 0.0f);
        float plane = 4.0f * (floorf(xk * 0.25f) + (st[k] > 0 ? 1.0f : 0.0f));
        if ((plane - o[k]) * (float)st[k] <= 0.0f) plane += 4.0f * (float)st[k];
        bool done = false;
        for (uint32_t n = 0; n < 96u; ++n) {
            const float tf = (plane - o[k]) * iv[k];
            if (!(tf <= t_to + 2e-3f)) {
                done = true;
                break;
            }
            ++checks;
            bool ok = true;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                if (j == k || fixed[j]) continue;
                const float xj = o[j] + d[j] * (tf - 1e-3f);
                const float q0 = 4.0f * floorf(xj * 0.25f);
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const float q = q0 + 4.0f * (float)e;
                    if ((q - o[j]) * (float)st[j] <= 0.0f) continue;
                    if (fabsf((q - o[j]) * iv[j] + 1e-3f - tf) < win) ok = false;
                }
            }
            if (!ok) {
                fail = fminf(fail, tf);
                done = true;
                break;
            }
            plane += 4.0f * (float)st[k];
        }
        if (!done) fail = fminf(fail, (plane - o[k]) * iv[k]);  // unchecked crossings left
    }
    return fail;
}

// A ray's part of the proof.  Its segment [0, depth] lies in its tile's
// bundle boxes; the ray checks what is particular to it (small axes) and
// picks its restart point.  Returns the outcome; on PARTIAL / ACCEPTED, r
// holds the restart.  o, d, iv, st are the plain DDA's rebased ray.
__device__ __forceinline__ uint32_t lane_restart(const Dims &D, const VxTraceParams &p,
                                                 const VerifyArgs &va, const float o[3],
                                                 const float d[3], const float iv[3],
                                                 const int32_t st[3], float depth, bool reached,
                                                 Restart &r, uint32_t &checks) {
    const float dims[3] = {(float)D.vx, (float)D.vy, (float)D.vz};
    bool fixed[3], small[3];
    float t_win = 3.0e38f;
    checks = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (!(o[k] >= 0.02f && o[k] <= dims[k] - 0.02f)) return OUT_NONE;
        const float ad = fabsf(d[k]);
        fixed[k] = ad < kFixed;
        small[k] = !fixed[k] && ad < va.delta;
        if (fixed[k] && plane_dist4(o[k]) < 2.0f * kClean) return OUT_NONE;
        if (!fixed[k]) t_win = fminf(t_win, ((st[k] > 0 ? dims[k] : 0.0f) - o[k]) * iv[k]);
    }
    if (!(depth > 0.0f)) return OUT_NONE;
    const float t_limit = fminf(p.max_dist, t_win) + kTEps;
    float t = fminf(depth, t_limit);
    bool cut = false;
    if (small[0] || small[1] || small[2]) {
        const float f = small_axis_fail(va, o, d, iv, st, fixed, small, 0.0f, t, checks);
        if (f < 3.0e38f) {
            t = fminf(t, f - 2.0f * kClean);
            cut = true;
        }
    }
    if (!cut && depth >= t_limit) return OUT_MISS;
    // the restart point: the end of the proof (for the bundle's outermost
    // rays kMu inside the last box), or a little before it, with every
    // moving coordinate clear of brick planes; the iteration bound counts
    // the brick planes between the camera's brick (ob) and the point's
    float tc = t;
    for (int attempt = 0; attempt < 4; ++attempt, tc -= 0.0625f) {
        if (!(tc > 0.0f)) break;
        bool ok = true;
        uint32_t bnd = 2u;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (fixed[k]) continue;
            const float x = o[k] + d[k] * tc;
            const float fb = floorf(x * 0.25f);
            const float rr = x - 4.0f * fb;
            if (!(rr >= kClean && rr <= 4.0f - kClean)) ok = false;
            bnd += (uint32_t)abs((int32_t)fb - va.ob[k]);
        }
        if (!ok) continue;
        r.t = tc;
        r.bound = bnd;
        return reached && !cut && attempt == 0 ? OUT_ACCEPTED : OUT_PARTIAL;
    }
    return OUT_NONE;
}

struct LearnedArgs {
    TraceArgs ta;
    VxCamera cam;
    uint32_t W, H, tiles_x;
    const float *depth;        // per tile: the frustum pre-pass's proven depth, or nullptr
    const float *proposal;     // log t per proposal block, or nullptr (restart at the proof's end)
    uint32_t prop_bw;          // proposal blocks per row
    float scale;               // proposed start distance = exp(proposal) * scale
    VxHitRecord *rec;
    unsigned long long *stats; // [none, partial, accepted, miss, steps, iters, fallback, rays]
    bool verify_on;            // window and fields suit the verification
    VerifyArgs va;
};

template <uint32_t FL>
// At least 6 CTAs per SM (up to 85 registers; 71 used): the learned frame
// measured 0.203 ms against 0.211 ms at 7 and 0.212 ms at 8 (the register
// budget of 8 forces the walk's state into fewer registers), 0.228 ms at 5.
__global__ void __launch_bounds__(128, 6) k_learned(LearnedArgs la) {
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
            // the pre-pass's depths and proposals are read only after its grid
            // has finished (programmatic dependent launch)
            asm volatile("griddepcontrol.wait;" ::: "memory");
            if (la.verify_on) {
                // the proposal is accepted where the bundle's proof covers it;
                // otherwise the ray restarts at the proof's end
                float dep = __ldg(la.depth + (py / kTileH) * la.tiles_x + px / kTileW);
                bool accepted = false;
                if (la.proposal) {
                    const float t_prop =
                        expf(__ldg(la.proposal + (py / kPropH) * la.prop_bw + px / kPropW)) *
                        la.scale;
                    if (t_prop <= dep) {
                        dep = t_prop;
                        accepted = true;
                    }
                }
                const float o[3] = {k.s.ox, k.s.oy, k.s.oz}, d[3] = {k.s.dx, k.s.dy, k.s.dz};
                const float iv[3] = {k.s.ix, k.s.iy, k.s.iz};
                const int32_t st[3] = {k.s.stx, k.s.sty, k.s.stz};
                Restart rs{0.0f, 0u};
                outcome = lane_restart(w.d, p, la.va, o, d, iv, st, dep, accepted, rs, cells);
                if (outcome == OUT_PARTIAL || outcome == OUT_ACCEPTED) {
                    // restart at floor(P): its first iteration skips the same
                    // cell the plain DDA skips there
                    Dda &s = k.s;  // (voxel relative to the window corner)
                    s.vx = (int32_t)floorf(s.ox + s.dx * rs.t);
                    s.vy = (int32_t)floorf(s.oy + s.dy * rs.t);
                    s.vz = (int32_t)floorf(s.oz + s.dz * rs.t);
                    k.t_cur = rs.t;
                    k.la = -1;
                    k.iters = rs.bound;
                }
            }
            uint32_t executed = 0;
            if (outcome != OUT_MISS) {
                const uint32_t base = k.iters;
                int r = WALK_CONT;
                while (r == WALK_CONT) r = walk_step<FL, false, KIND_TRACE>(w, g, p, ro, k, h, bytes);
                executed = k.iters - base;
                if (r == WALK_END && k.iters >= k.cap && outcome != OUT_NONE) {
                    // the inflated counter reached the cap: the plain DDA decides
                    fallback = 1;
                    set_miss(h);
                    walk_init(w.d, ro, KIND_TRACE, p, ox, oy, oz, dx, dy, dz, p.max_dist, k);
                    while (walk_step<FL, false, KIND_TRACE>(w, g, p, ro, k, h, bytes) == WALK_CONT) {
                    }
                    executed += k.iters;
                }
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


namespace {
// The verification constants of a window (see the rounding bounds below)
VerifyArgs verify_args(const TraceArgs &ta, bool *ok) {
    VerifyArgs va{};
    const Dims &d = ta.w.d;
    // Rounding bounds of the plain DDA (window-relative coordinates below
    // cmax, times up to tmax):
    //   coord_eps = 2 h: a landing coordinate fl(o + fl(d tb)) and a face
    //     distance fl(F - o) are each off by at most h, half an ulp of the
    //     largest float below cmax;
    //   t_eps = 4 tmax 2^-24 + h(tmax) + 1e-5: the landing product, the face
    //     time's two relative roundings and the nudged time fl(t + 1e-3).
    // t_min strictly increases wherever coord_eps / |d_a| + t_eps < 1e-3 (the
    // nudge) on every moving axis; axes below delta get explicit checks.
    const float cmax = (float)std::max(d.vx, std::max(d.vy, d.vz));
    const float tmax = std::max(ta.p.max_dist, 0.0f) + 16.0f;
    auto half_ulp_below = [](float x) { return ldexpf(1.0f, ilogbf(nextafterf(x, 0.0f)) - 24); };
    auto half_ulp_at = [](float x) { return ldexpf(1.0f, ilogbf(x) - 24); };
    va.coord_eps = 2.0f * half_ulp_below(std::max(cmax, 2.0f));
    va.t_eps = 4.0f * tmax * 5.9604645e-8f + half_ulp_at(tmax) + 1e-5f;
    const float room = 1e-3f - va.t_eps;
    va.delta = room > 1e-4f ? va.coord_eps / room : 2.0f;
    auto pmod = [](int32_t a, int32_t b) { return ((a % b) + b) % b; };
    va.sbx = pmod(ta.ro[0] / 4, d.bx);
    va.sbz = pmod(ta.ro[2] / 4, d.bz);
    va.stx = pmod(ta.ro[0] / 16, d.tx);
    va.stz = pmod(ta.ro[2] / 16, d.tz);
    va.ob[0] = va.ob[1] = va.ob[2] = 0;
    *ok = ta.w.bdf != nullptr && ta.w.tdf != nullptr && (ta.ro[0] & 15) == 0 &&
          (ta.ro[2] & 15) == 0 && ta.ro[1] == 0 && room > 1e-4f;
    return va;
}

uint32_t flags_of(const TraceArgs &ta) {
    return (ta.p.flags & (VX_F_L4 | VX_F_LUT | VX_F_LOD)) | pow2_bit(ta.w.d);
}

template <uint32_t FL>
struct PrepassK {
    static void *fn() { return reinterpret_cast<void *>(&k_prepass<FL>); }
};
}  // namespace

bool learned_proof_ok(const TraceArgs &ta) {
    bool ok = false;
    verify_args(ta, &ok);
    return ok;
}

cudaError_t launch_learned_prepass(const TraceArgs &ta, const VxCamera &cam, float *depth,
                                   const Mlp *mlp, float *pred, unsigned long long *stats,
                                   cudaStream_t stream) {
    bool ok = false;
    FrustumArgs fa{};
    fa.va = verify_args(ta, &ok);
    if (!ok || !depth) return cudaErrorInvalidValue;
    fa.w = ta.w;
    fa.p = ta.p;
    fa.cam = cam;
    for (int k = 0; k < 3; ++k) fa.ro[k] = ta.ro[k];
    fa.W = (uint32_t)cam.res_x;
    fa.H = (uint32_t)cam.res_y;
    fa.tiles_x = (fa.W + kTileW - 1u) / kTileW;
    fa.tiles_y = (fa.H + kTileH - 1u) / kTileH;
    fa.depth = depth;
    fa.stats = stats;
    const uint32_t frustum_ctas = (fa.tiles_x * fa.tiles_y + 127u) / 128u;
    InferArgs ia{};
    uint32_t infer_ctas = 0;
    if (mlp && pred) {
        ia.w = reinterpret_cast<const __nv_bfloat16 *>(mlp->w16);
        ia.f32 = mlp->p;
        ia.cam = cam;
        ia.W = fa.W;
        ia.blk_w = kPropW;
        ia.blk_h = kPropH;
        ia.bw = (fa.W + kPropW - 1u) / kPropW;
        ia.n = ia.bw * ((fa.H + kPropH - 1u) / kPropH);
        ia.world = ta.w;
        for (int k = 0; k < 3; ++k) ia.ro[k] = ta.ro[k];
        ia.out = pred;
        // one 16-ray pass per warp, four warps per CTA
        infer_ctas = (((ia.n + 15u) / 16u) + 3u) / 4u;
    }
    void *args[] = {&fa, &ia, (void *)&frustum_ctas, (void *)&infer_ctas};
    return cudaLaunchKernel(pick_fl<PrepassK>(flags_of(ta)), dim3(frustum_ctas + infer_ctas),
                            dim3(128), args, 0, stream);
}

cudaError_t launch_learned(const TraceArgs &ta, const VxCamera &cam, const float *depth,
                           const float *proposal, float scale, VxHitRecord *rec,
                           unsigned long long *stats, cudaStream_t stream) {
    LearnedArgs la{};
    la.ta = ta;
    la.cam = cam;
    la.W = (uint32_t)cam.res_x;
    la.H = (uint32_t)cam.res_y;
    la.tiles_x = (la.W + kTileW - 1u) / kTileW;
    la.rec = rec;
    la.stats = stats;
    la.depth = depth;
    la.proposal = proposal;
    la.prop_bw = (la.W + kPropW - 1u) / kPropW;
    la.scale = scale;
    bool ok = false;
    la.va = verify_args(ta, &ok);
    // the camera's brick, from the rebased origin exactly as dda_init forms it
    for (int k = 0; k < 3; ++k)
        la.va.ob[k] = (int32_t)floorf((cam.origin[k] - (float)ta.ro[k]) * 0.25f);
    la.verify_on = ok && depth != nullptr;
    const dim3 grid((la.W + 15u) / 16u, (la.H + 7u) / 8u);
    void *args[] = {&la};
    // after the pre-pass: programmatic dependent launch (the kernel waits
    // for the pre-pass's grid before it reads its outputs)
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(128);
    cfg.stream = stream;
    cudaLaunchAttribute attr{};
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = la.verify_on ? 1u : 0u;
    return cudaLaunchKernelExC(&cfg, pick_fl<LearnedK>(flags_of(ta)), args);
}

}  // namespace vx
