// vx_internal.h -- definitions shared by the CUDA kernels and the C++ host
// side of libvoxrt.  Not part of the public ABI (include/voxrt.h is).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "voxrt.h"

#include <nvtx3/nvToolsExt.h>

namespace vx {

// Names one library call on a profiler's timeline (an NVTX range); it costs
// nothing when no tool is attached.
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};

// World dimensions; the derived counts follow src/world_dims.rs:12-37.
struct Dims {
    int32_t bx, by, bz;  // bricks
    int32_t vx, vy, vz;  // voxels
    int32_t tx, ty, tz;  // tiles (16^3 voxels)
    int32_t cx, cy, cz;  // chunks (64^3)
    int32_t lx, ly, lz;  // L4 cells (256^3)
    int64_t n_bricks, n_tiles, n_chunks, n_l4;
};

inline Dims make_dims(int32_t bx, int32_t by, int32_t bz) {
    Dims d;
    d.bx = bx; d.by = by; d.bz = bz;
    d.vx = bx * 4; d.vy = by * 4; d.vz = bz * 4;
    d.tx = bx / 4; d.ty = by / 4; d.tz = bz / 4;
    d.cx = (d.tx + 3) / 4; d.cy = (d.ty + 3) / 4; d.cz = (d.tz + 3) / 4;
    d.lx = (d.cx + 3) / 4; d.ly = (d.cy + 3) / 4; d.lz = (d.cz + 3) / 4;
    d.n_bricks = (int64_t)bx * by * bz;
    d.n_tiles = (int64_t)d.tx * d.ty * d.tz;
    d.n_chunks = (int64_t)d.cx * d.cy * d.cz;
    d.n_l4 = (int64_t)d.lx * d.ly * d.lz;
    return d;
}

// Device-resident pyramid.  Bricks are split structure-of-arrays: the 8-byte
// occupancy words (read on every voxel-level iteration) are packed densely,
// the 64 material bytes of a brick sit in their own 64-byte-aligned row and
// are only touched on a solid voxel.
struct DevWorld {
    Dims d;
    uint64_t *occ;            // n_bricks
    uint8_t *mat;             // n_bricks * 64
    uint64_t *tile_mask;      // n_tiles
    uint64_t *chunk_mask;     // n_chunks
    uint64_t *l4_mask;        // n_l4
    uint8_t *brick_uniform;   // n_bricks
    uint8_t *tile_uniform;    // n_tiles
    // n_tiles, derived from the masks above by launch_tile_meta: what the
    // walk's L4 and chunk tests decide for every voxel of a tile, beside the
    // tile LUT byte (layout in vx_walk.cuh at kMetaChunkOnly).  nullptr for caller-owned worlds: the
    // walk then evaluates the tests from the masks.
    uint16_t *tile_meta;
    // First out-of-range world index met by a load of the checked library
    // (array id << 56 | index; 0 = none).  nullptr: not recorded.
    unsigned long long *oob;
    // Device-visible word (host-mapped) for faults the kernels survive but
    // must report: bit 0 = a beam CTA exited before its bulk copy of the
    // chunk masks into shared memory had completed (both bounded waits ran
    // out).  nullptr: the world has no place to report one, and the beam
    // pre-pass then reads the masks with plain loads instead of staging them.
    uint32_t *fault;
    // Empty-space distance fields (vx_distfield.cu), built on demand for the
    // learned form: per brick / per tile the Chebyshev distance, in cells of
    // that level, to the nearest non-empty cell (0 = non-empty, cap + 1 =
    // nothing within the cap).  nullptr when not built.
    const uint8_t *bdf;
    const uint8_t *tdf;
};
constexpr uint32_t kFaultBeamCopyLost = 1u;
// bit 1: a compact frame held a record VxCompactRecord cannot hold
constexpr uint32_t kFaultCompactLossy = 2u;
constexpr int32_t kBrickFieldCap = 16;  // bricks (64 voxels)
constexpr int32_t kTileFieldCap = 12;   // tiles (192 voxels)

// Per-frame constants of the traversal kernels (passed by value).
struct TraceArgs {
    DevWorld w;
    VxTraceParams p;
    int32_t ro[3];            // loaded-window corner (camera.world_origin)
};

struct FrameArgs {
    TraceArgs ta;
    VxCamera cam;
    const float *beam;        // beam depth (bw*bh) or nullptr
    uint32_t W, H, bw, bh;
    uint32_t y0, y1;            // rows [y0, y1) of this launch (grid form)
    VxHitRecord *rec;
    VxShadowRecord *shadow;
    unsigned long long *stats;  // [bytes, iters] or nullptr
    uint32_t *work;             // persistent schedule: {next tile, warps done}, or nullptr
    const uint32_t *tile_gate;  // dirty 8x8-tile bits (cs_main gate) or nullptr = all
};

// ---- kernel launchers (vx_trace.cu / vx_world.cu) ----
cudaError_t launch_beam(const FrameArgs &fa, float *beam_out, cudaStream_t s);
cudaError_t launch_primary(const FrameArgs &fa, cudaStream_t s);
cudaError_t launch_trace_rays(const TraceArgs &ta, const VxRay *rays, size_t n, VxHitRecord *out,
                              cudaStream_t s);
// one pick ray whose camera and direction travel in the launch parameters
cudaError_t launch_raycast_one(const DevWorld &w, const int32_t origin[3], const float cam[3],
                               const float dir[3], VxPickHit *out, int32_t *hit, cudaStream_t s);
cudaError_t launch_raycast(const DevWorld &w, const int32_t origin[3], const float *cams,
                           const float *dirs, size_t n, VxPickHit *out, int32_t *hit,
                           cudaStream_t s);

// contact AO of a frame's primary records (f32 per pixel)
cudaError_t launch_ao(const DevWorld &w, const VxCamera &cam, const VxHitRecord *rec, float *ao,
                      cudaStream_t s);
cudaError_t launch_project_dirty(const DevWorld &w, const VxCamera &cam, const uint32_t *idx,
                                 size_t n, uint32_t *mask, cudaStream_t s);
cudaError_t launch_refresh_tiles(uint32_t tiles_w, uint32_t tiles_h, uint32_t spread,
                                 uint32_t phase, uint32_t *mask, cudaStream_t s);

cudaError_t launch_bricks_from_aos(const DevWorld &w, const VxBrick *aos, int64_t first,
                                   int64_t count, cudaStream_t s);
cudaError_t launch_bricks_to_aos(const DevWorld &w, VxBrick *aos, int64_t first, int64_t count,
                                 cudaStream_t s);
// gen_slot_bricks on the device.  Explicit plans (window == false) list
// their jobs: kGenJobInts ints each -- world chunk x, y, z; slot x, y, z;
// the index of its xz chunk in `cols`; the indices in `srcs` of its 3x3
// source chunks in (z, x) order; cols / srcs hold (x, z) pairs.  A window
// plan (window == true) generates every slot of the window whose lower
// corner is world chunk (ox, 0, oz) and derives all of that on the device:
// job b is slot (b % SX, b / SX % SY, b / (SX SY)), column k the slot column
// (k % SX, k / SX), source k world chunk (ox - 1 + k % (SX + 2),
// oz - 1 + k / (SX + 2)).  colw has 1024 words per column chunk, prims
// gen_prim_bytes_per_src() bytes and hdr 12 ints per source chunk.  The
// pyramid is rebuilt afterwards.
constexpr int kGenJobInts = 16;
struct GenPlan {
    bool window;
    int32_t ox, oz;            // window plans
    const int32_t *jobs;       // explicit plans
    uint32_t n_jobs;
    const int32_t *cols;       // explicit plans
    uint32_t n_cols;
    const int32_t *srcs;       // explicit plans
    uint32_t n_srcs;
    uint32_t *colw;
    void *prims;
    int32_t *hdr;
    const uint32_t *lmx;       // vx_gmath.h exception table on the device
};
size_t gen_prim_bytes_per_src();
// the generator's powf / cosf / sinf (vx_gmath.h function fn) on n inputs
cudaError_t launch_gen_math(const uint32_t *lmx, uint32_t fn, const float *in, size_t n, float *out,
                            cudaStream_t s);
cudaError_t launch_gen_slots(const DevWorld &w, uint64_t seed, const GenPlan &p, cudaStream_t s);
cudaError_t launch_generate(const DevWorld &w, const VxTerrainParams &t, int16_t *heights,
                            cudaStream_t s);
cudaError_t launch_rebuild_pyramid(const DevWorld &w, cudaStream_t s);
// the brick and tile distance fields of w (tmp: n_bricks bytes of scratch)
// a frame's records (and shadow records, or nullptr) [first, first + n) in
// the 16-byte packed form (vx_pack.cu)
// records [first, first + n) as VxCompactRecord; a record the form cannot
// hold sets kFaultCompactLossy in *fault
cudaError_t launch_pack_compact(const VxHitRecord *rec, const VxShadowRecord *sh, size_t first,
                                size_t n, const int32_t ro[3], uint32_t wx, uint32_t wy,
                                VxCompactRecord *out, uint32_t *fault, cudaStream_t s);
cudaError_t launch_pack(const VxHitRecord *rec, const VxShadowRecord *sh, size_t first, size_t n,
                        const int32_t ro[3], uint32_t wx, uint32_t wy, VxPackedRecord *out,
                        cudaStream_t s);
cudaError_t launch_dist_fields(const DevWorld &w, uint8_t *bdf, uint8_t *tdf, uint8_t *tmp,
                               cudaStream_t s);
// tile_meta of every tile from the masks and the tile LUT
cudaError_t launch_tile_meta(const DevWorld &w, cudaStream_t s);
// Persistent edits: ed[i] = {brick, voxel | material << 8}, distinct voxels;
// idx the distinct bricks they touch (uniform bytes and masks refreshed).
cudaError_t launch_edits(const DevWorld &w, const uint2 *ed, size_t n_edits, const uint32_t *idx,
                         size_t n_bricks, cudaStream_t s);
// launch_apply_dirty for n entries that may repeat a brick (the last entry
// wins); win is a zeroed word per brick, zeroed again when the update ends
cudaError_t launch_apply_dirty_last_wins(const DevWorld &w, uint32_t *win, const uint32_t *idx,
                                         const VxBrick *bricks, size_t n, cudaStream_t s);
cudaError_t launch_apply_dirty(const DevWorld &w, const uint32_t *idx, const VxBrick *bricks,
                               size_t n, cudaStream_t s);

// Scratch of one ray-queue configuration (owned by a world or a graph):
// work counters, coherence-sort keys / permutation / histogram, fingerprint.
struct QueueScratch {
    uint32_t *work = nullptr;
    uint2 *kv = nullptr;          // coherence sort: (key, ray) pairs
    uint2 *kv2 = nullptr;         // and their ping-pong partner
    uint32_t *hist = nullptr;     // per-tile digit counts
    unsigned long long *fp = nullptr;
    size_t cap = 0;
    cudaError_t reserve(size_t n);
    void release();
};

cudaError_t launch_queue(const TraceArgs &ta, const VxRay *rays, size_t n, VxHitRecord *out,
                         VxShadowRecord *shadow, const VxQueueTuning &t, QueueScratch &sc,
                         cudaStream_t s);
// order-independent fingerprint of a queue's outputs (synchronizes s)
cudaError_t queue_fingerprint(const VxHitRecord *out, size_t n, const VxShadowRecord *shadow,
                              QueueScratch &sc, cudaStream_t s, unsigned long long *host);

// ---- learned start-distance proposal (vx_mlp.cu, vx_learned.cu) ----
// MLP 70 -> 64 -> 64 -> 64 -> 1 with GELU; flat f32 parameters in the order
// W1[64][80] (columns 70..79 zero), b1, W2[64][64], b2, W3[64][64], b3, wo, bo.
constexpr int kMlpIn = 80, kMlpHidden = 64;
constexpr int kMlpFloats = kMlpHidden * kMlpIn + kMlpHidden + 2 * (kMlpHidden * kMlpHidden + kMlpHidden) +
                           kMlpHidden + 1;

struct Mlp {
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // params, grads, Adam moments
    uint16_t *w16 = nullptr;   // bf16 W1 | W2 | W3 with padded rows (inference)
    int adam_t = 0;
    size_t cap = 0;            // training batch capacity of the activations below
    float *z1 = nullptr, *a1 = nullptr, *z2 = nullptr, *a2 = nullptr, *z3 = nullptr, *a3 = nullptr;
    float *y = nullptr, *dy = nullptr, *da = nullptr, *dz = nullptr, *loss = nullptr;
};

cudaError_t mlp_alloc(Mlp &m);
void mlp_free(Mlp &m);
cudaError_t mlp_sync_bf16(Mlp &m, cudaStream_t s);
// forward + backward of one batch (X [B][80] f32 device, targets [B]):
// gradients in m.g (zeroed first), mean squared error in *m.loss
cudaError_t mlp_grad(Mlp &m, const float *X, const float *target, int B, cudaStream_t s);
cudaError_t mlp_adam(Mlp &m, float lr, cudaStream_t s);
cudaError_t mlp_infer_features(const Mlp &m, const float *feats, size_t n, float *out,
                               cudaStream_t s);
// proposals of a camera frame, one per bw x bh pixel block (the ray through
// the block's centre), row-major with ceil(W / bw) blocks per row
cudaError_t mlp_infer_frame(const Mlp &m, const DevWorld &w, const VxCamera &cam,
                            const int32_t ro[3], uint32_t bw, uint32_t bh, float *out,
                            cudaStream_t s);
// features of rays idx(j) = ((base + j) % n) * mult % n, j < count (mult = 1: in order)
cudaError_t mlp_features(const DevWorld &w, const int32_t ro[3], const VxRay *rays, size_t n,
                         uint64_t base, uint64_t mult, size_t count, float *feats,
                         const float *targets_src, float *targets_dst, cudaStream_t s);
cudaError_t mlp_targets(const VxHitRecord *rec, size_t n, float max_dist, float *target,
                        cudaStream_t s);
cudaError_t mlp_pose_rays(const VxCamera &c, uint64_t seed, size_t n, VxRay *rays,
                          float max_dist, cudaStream_t s);
// learned frame: a frustum pre-pass proves, per 8 x 4 pixel tile, the rays'
// common segment from the camera empty as far as it can into depth (one
// float per tile, ceil(W / 8) per row); every pixel then restarts the plain
// DDA inside its proven segment, at exp(proposal) * scale where the proof
// covers that (proposal: log t per 16 x 8 pixel block, ceil(W / 16) per row,
// or nullptr)
constexpr uint32_t kLearnedTileW = 8, kLearnedTileH = 4;
constexpr uint32_t kLearnedPropW = 16, kLearnedPropH = 8;
// does the window suit the proof (fields built, corner a multiple of 16 in
// x and z)?
bool learned_proof_ok(const TraceArgs &ta);
// the pre-pass: the proofs into depth and, when mlp and pred are given, the
// proposals into pred, in one launch
cudaError_t launch_learned_prepass(const TraceArgs &ta, const VxCamera &cam, float *depth,
                                   const Mlp *mlp, float *pred, unsigned long long *stats,
                                   cudaStream_t s);
// depth: the proof's output, or nullptr = the plain DDA for every ray
cudaError_t launch_learned(const TraceArgs &ta, const VxCamera &cam, const float *depth,
                           const float *proposal, float scale, VxHitRecord *rec,
                           unsigned long long *stats, cudaStream_t s);

// ---- device-resident request loop (vx_resident.cu, driven by vx_serve.cpp) ----
// The host publishes request descriptors into a ring in page-locked host
// memory mapped into the device's address space; one persistent launch (an
// "instance") takes them in order, splits each into 32-ray units and traces
// the units on every warp it holds, writes the records straight into host
// memory and, for each finished request, a completion word the host polls.
// Every wait in the loop is bounded.
constexpr uint32_t kResRing = 1024;  // descriptor and completion slots
enum : uint32_t { RES_REQ = 0, RES_FENCE = 1 };
// how an instance ended (ResReplyBox::status)
enum : uint32_t {
    RES_RUNNING = 0, RES_IDLE = 1, RES_ROTATE = 2, RES_FENCED = 3, RES_STOPPED = 4
};
// ResReplyBox::error: a wait of the loop ran out (the loop then ends)
enum : uint32_t { RES_ERR_NONE = 0, RES_ERR_UNIT_WAIT = 1, RES_ERR_RING_WAIT = 2 };
struct ResDesc {    // 32 bytes, written by the host
    uint64_t rays;  // device address of the request's VxRay array (mapped host memory, < 2^48)
    uint64_t out;   // device address of its VxHitRecord array (< 2^48)
    uint32_t n;     // rays, >= 1
    uint32_t kind;  // RES_REQ, or RES_FENCE: an edit follows, the instance ends here
    uint64_t seq;   // RES_FENCE: the edit's number (from 1)
};
struct ResHostBox {  // mapped host memory, written by the host
    uint64_t head;   // descriptors published (release order after the descriptor)
    uint32_t stop;   // 1: the instance ends at its next poll
    uint32_t pad[13];
    ResDesc desc[kResRing];  // position p in desc[p % kResRing]
};
// completion word of the request at position p: res_done_word(p), in slot p % kResRing
__host__ __device__ inline uint64_t res_done_word(uint64_t pos) {
    return ((pos & 0xFFFFFFFFull) << 1) | 1ull;
}
struct ResReplyBox {              // mapped host memory, written by the device
    uint64_t done[kResRing];      // res_done_word of the request finished in that slot
    uint64_t consumed;            // descriptors taken by the loop
    uint32_t unit_end;            // global unit number after the last one published
    uint32_t status;              // how the last instance ended (RES_IDLE ...)
    uint32_t error;               // RES_ERR_*, sticky
    uint32_t pad;
};
// Device memory.  Workers read what the leader publishes with plain
// device-coherent (relaxed) loads, never acquire loads (polling with acquire
// loads measured slower under load): every word carries a tag of the
// publication it belongs to, and a reader waits until the tag matches.
//   unit word  (global unit g) << 32 | (position p, low 32 bits)
//   request    slot p % kResRing, four words:
//                rays | (p & 0xFFFF) << 48,  out | (p & 0xFFFF) << 48,
//                (p32) << 32 | n,           (p32) << 32 | first global unit
struct ResCounters {              // zeroed before every instance
    uint32_t pubw;                // bit 31: closing; bits 0-30: units published
    uint32_t pad0[31];
    uint32_t claim;               // next unit ticket (relative to the instance)
    uint32_t pad1[31];
    uint32_t done_units;          // units finished
    uint32_t pad2[31];
};
struct ResArgs {
    TraceArgs ta;
    ResHostBox *host;             // device addresses of the two mailboxes
    ResReplyBox *reply;
    ResCounters *ctr;
    unsigned long long *req;      // [kResRing][4] tagged request words
    unsigned long long *unit;     // [unit_ring] tagged unit words
    uint32_t *cnt;                // [kResRing] units finished of the slot's request (reset to 0 at its end)
    uint32_t unit_ring;
    uint32_t unit_base;           // global number of this instance's first unit
    uint64_t consumed;            // descriptors taken before this instance
    uint64_t edits_before;        // edits ordered before this instance (fences up to it are past)
    uint64_t idle_ns;             // the instance ends after this long without a descriptor
    uint64_t life_ns;             // ... and takes no descriptor after this long in all
    uint64_t wait_ns;             // bound on every other wait of the loop
};
// CTAs of one instance for the method flags of ta (SMs x resident CTAs, at most 4 per SM)
cudaError_t serve_loop_grid(const TraceArgs &ta, unsigned *grid);
cudaError_t launch_serve_loop(const ResArgs &a, unsigned grid, cudaStream_t s);

// accessors for library parts outside vx_api.cpp
DevWorld world_dev(const VxWorld *w);
int world_device(const VxWorld *w);
// The world's masks changed (every path that rewrites them calls this): the
// distance fields are stale until the next world_dist_fields.
void world_masks_changed(VxWorld *w);
// DevWorld of w with its distance fields, (re)built on `s` first when the
// masks changed since they were last built; VX_OK or an error code.
int world_dist_fields(VxWorld *w, cudaStream_t s, DevWorld *out);
// n floats of per-tile depth scratch owned by w, for learned frames without
// a proposal (grown on demand; learned frames on one world must not overlap)
int world_learned_depth(VxWorld *w, size_t n, float **out);

// thread-local error text
void set_error(const std::string &msg);

// The loaded window moves in x/z only (src/voxel.rs:439-445 keeps its y at
// 0): storage y is world y, so a window corner with y != 0 would index past
// the y extent of every level.  Entry points reject it.
inline bool origin_ok(const int32_t o[3], const char *fn) {
    if (o[1] != 0) {
        set_error(std::string(fn) + ": window origin y must be 0 (windows move in x/z only)");
        return false;
    }
    return true;
}

}  // namespace vx
