/*
 * voxrt.h -- C ABI of the B200-native voxel ray-traversal engine for voxelG.
 *
 * A drop-in for voxelG's traversal boundary: the CPU picking call
 * `raycast()` (src/raycast.rs:21) and the GPU hierarchical DDA that
 * shaders/raymarch.wgsl + shaders/beam.wgsl run over the world pyramid that
 * src/voxel.rs maintains.  All kernels are hand-written CUDA for sm_100a; the
 * library has no CPU fallback -- every traversal entry point fails with
 * VX_ERR_CUDA when no usable GPU is present.
 *
 * Conventions
 *   - Every entry point returns an int status (VX_OK = 0, negative = error)
 *     except where stated; vx_last_error() returns a thread-local message.
 *     No exceptions cross the ABI, nothing aborts.
 *   - Ownership: the caller owns every pointer it passes; the library owns
 *     the device copy of a world.  No pointer is retained after a call.
 *   - "_dev" pointers are device memory on the world's device; other pointers
 *     are host memory.  Calls taking a `stream` (a cudaStream_t, NULL = the
 *     legacy default stream) are asynchronous and stream-ordered; the others
 *     are synchronous.
 *   - Host layouts are exactly voxelG's: Brick is repr(C) 72 bytes
 *     (src/voxel.rs:296-301), masks are u64 per cell with child bit
 *     x + z*4 + y*16 (src/voxel.rs:282-294), uniform LUTs one byte per cell.
 */
#ifndef VOXRT_H
#define VOXRT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VX_OK 0
#define VX_ERR_INVALID (-1)   /* bad argument, size or dims                  */
#define VX_ERR_CUDA (-2)      /* CUDA runtime error (incl. no device)        */
#define VX_ERR_OOM (-3)       /* device memory exhausted / over budget       */
#define VX_ERR_DEVICE (-4)    /* a kernel reported an error status word      */
#define VX_ERR_BUSY (-5)      /* admission refused (serving loop)            */

#define VX_ABI_VERSION 1

/* ---- plain data -------------------------------------------------------- */

/* src/voxel.rs:296-301 -- occupancy bit i = voxel x + z*4 + y*16. */
typedef struct {
    uint64_t occupancy;
    uint8_t materials[64];
} VxBrick;

/* World dims in bricks (src/world_dims.rs:12-14 made runtime values).
 * bricks_x and bricks_z must be multiples of 64 (whole 256-voxel L4 cells,
 * so toroidal folding keeps every level aligned); bricks_y a multiple of 16. */
typedef struct {
    int32_t bricks_x, bricks_y, bricks_z;
    int32_t device; /* CUDA device ordinal */
} VxWorldDesc;

/* Camera uniform subset the traversal reads (shaders/common.wgsl:7-42). */
typedef struct {
    float origin[3];
    float forward[3];
    float right[3];
    float up[3];
    float tan_half_fov;
    float res_x, res_y;
    float jitter_x, jitter_y;      /* sub-pixel jitter in pixels            */
    int32_t world_origin[3];       /* loaded-window corner, world voxels;
                                      y must be 0: windows move in x/z only
                                      (src/voxel.rs:439-445), every call
                                      taking a window corner rejects y != 0 */
} VxCamera;

/* Method switches.  The reference method is L4|LUT|LOD|BEAM. */
#define VX_F_L4 (1u << 0)      /* L4 + chunk-in-L4 skip (!PROFILE_NO_L4)   */
#define VX_F_LUT (1u << 1)     /* uniform tile/brick early-out             */
#define VX_F_LOD (1u << 2)     /* tile LOD (t>520) + brick LOD (t>400)     */
#define VX_F_BEAM (1u << 3)    /* 1/8-res beam pre-pass fast-forward       */
#define VX_F_SHADOW (1u << 4)  /* one any-hit shadow ray per primary hit   */

typedef struct {
    float max_dist;          /* MAX_RAY_DIST 700    raymarch.wgsl:4501 */
    float lod_brick_t;       /* LOD_BRICK_T 400     raymarch.wgsl:4489 */
    float tile_lod_t;        /* TILE_LOD_T 520      raymarch.wgsl:4494 */
    float shadow_max_dist;   /* SHADOW_MAX_DIST 480 raymarch.wgsl:4517 */
    float beam_margin;       /* 16                  raymarch.wgsl:608  */
    int32_t max_iters;       /* 1024                raymarch.wgsl:4625 */
    int32_t any_max_iters;   /* 768                 raymarch.wgsl:4359 */
    uint32_t flags;          /* VX_F_*                                 */
    float sun[3];            /* unit sun direction                     */
    float sun_tangent[3];    /* raymarch.wgsl:3984-3988                */
    float sun_bitangent[3];
    float cone_tan;          /* tan(cone half-angle)                   */
    float frame;             /* interleaved-gradient-noise frame term  */
} VxTraceParams;

/* One ray's record (24 bytes).  face = 2*axis + (entering along +axis), i.e.
 * 0:+x 1:-x 2:+y 3:-y 4:+z 5:-z outward normal; 0xFF on a miss.  t is the hit
 * distance from the ray origin (camera for primary rays); steps the number
 * of traversal-loop iterations begun, including the last. */
typedef struct {
    int32_t voxel[3];
    uint8_t face;
    uint8_t mat;
    uint8_t flags;    /* bit0 hit, bit1 uniform/LOD early-out */
    uint8_t pad;
    float t;
    uint32_t steps;
} VxHitRecord;

typedef struct {
    uint32_t steps;
    uint8_t occluded;
    uint8_t traced;
    uint16_t pad;
} VxShadowRecord;

/* One pixel's VxHitRecord and VxShadowRecord, losslessly in 16 bytes (half
 * the 32 the pair takes), for frames delivered to host memory.
 *   voxel   a hit's voxel relative to the window corner (world_origin),
 *           rx + wx * (ry + wy * rz) with (wx, wy, wz) the window's voxel
 *           counts; 0 for a miss (whose record voxel is 0, 0, 0)
 *   face, mat, flags, t   as VxHitRecord (pad is always 0)
 *   shadow  bit0 occluded, bit1 traced
 *   steps   primary steps in bits 0-15, shadow steps in bits 16-31
 * Frames packed this way need wx * wy * wz <= 2^32 and max_iters,
 * any_max_iters <= 65535.  vx_unpack_records restores both records. */
typedef struct {
    uint32_t voxel;
    uint8_t face;
    uint8_t mat;
    uint8_t flags;
    uint8_t shadow;
    float t;
    uint32_t steps;
} VxPackedRecord;

/* The same pair losslessly in 12 bytes, for windows of at most 2^30 voxels
 * (the 2048 x 256 x 2048 window has exactly 2^30) and max_iters <= 2047,
 * any_max_iters <= 1023:
 *   w[0]  bits 0-29 voxel (as VxPackedRecord), bit 30 flags bit 1 (a LUT or
 *         LOD early-out), bit 31 shadow occluded
 *   w[1]  bits 0-30 t (a frame's t is never negative: its sign bit is
 *         dropped), bit 31 shadow traced
 *   w[2]  bits 0-10 primary steps, 11-20 shadow steps, 21-23 face (7 for a
 *         miss), 24-31 material
 * A record's flags bit 0 (hit) is face != miss.  A frame holding a record
 * this form cannot hold (which the limits above exclude) is reported as
 * VX_ERR_DEVICE by the next synchronising call instead of being truncated.
 * vx_unpack_compact_records restores both records. */
typedef struct {
    uint32_t w[3];
} VxCompactRecord;

/* src/raycast.rs:13-17 */
typedef struct {
    int32_t voxel[3];
    int32_t normal[3];
} VxPickHit;

/* Generic ray for vx_trace: kind (low two bits; higher bits ignored by
 * vx_trace) 0 first hit (trace), 1 any hit (trace_any,
 * record.flags bit0 = occluded), 2 first non-transparent hit
 * (trace_no_water).  tmax replaces MAX_RAY_DIST / max_dist / t_cap. */
typedef struct {
    float org[3];
    float dir[3];
    float tmax;
    uint32_t kind;
} VxRay;

/* Seeded synthetic terrain: h = floor(base + amp*fbm_2d(x/wl, z/wl, oct)),
 * grass top, dirt_depth dirt, stone below, water (material 12) up to
 * water_level, caves where value_noise_3d(p/cave_wl) > cave_threshold
 * (noise primitives of src/voxel.rs:1163-1232, :1999-2021). */
typedef struct {
    uint64_t seed;
    float base_height;
    float amplitude;
    float inv_wavelength;
    uint32_t octaves;
    int32_t water_level;
    float cave_inv_wavelength;
    float cave_threshold;
    int32_t dirt_depth;
} VxTerrainParams;

typedef struct VxWorld VxWorld;          /* device-resident world pyramid */
typedef struct VxHostWorld VxHostWorld;  /* host mirror of src/voxel.rs World */

/* ---- library ----------------------------------------------------------- */
int vx_abi_version(void);
const char *vx_last_error(void);
/* Fill *p with the reference constants, flags L4|LUT|LOD|BEAM|SHADOW, sun =
 * normalize(0.3, 0.8, 0.5) with its tangent frame, a 0.5-degree cone. */
int vx_default_params(VxTraceParams *p);
/* Camera basis from a pose: src/camera.rs:25-42 (forward/right/up) and
 * :140-166 (CameraUniform::from_camera). */
int vx_camera_from_pose(const float pos[3], float yaw, float pitch, float fov_y,
                        uint32_t width, uint32_t height, const int32_t world_origin[3],
                        VxCamera *out);

/* ---- device world (replaces Renderer::upload_world, renderer.rs:1248) -- */
int vx_world_create(const VxWorldDesc *desc, VxWorld **out);
int vx_world_destroy(VxWorld *w);
/* Full upload from voxelG's host arrays (renderer.rs:1248-1344 all_dirty). */
int vx_world_upload(VxWorld *w, const VxBrick *bricks, const uint64_t *tile_mask,
                    const uint64_t *chunk_mask, const uint64_t *l4_mask,
                    const uint8_t *brick_uniform, const uint8_t *tile_uniform);
/* Copy the device pyramid back into voxelG's host layout (any pointer may
 * be NULL to skip that array). */
int vx_world_download(VxWorld *w, VxBrick *bricks, uint64_t *tile_mask, uint64_t *chunk_mask,
                      uint64_t *l4_mask, uint8_t *brick_uniform, uint8_t *tile_uniform);
/* Generate the seeded synthetic terrain on the device and build masks and
 * uniform LUTs there (src/voxel.rs:946-1000 semantics). */
int vx_world_generate(VxWorld *w, const VxTerrainParams *t);

/* The reference's storage-chunk generator gen_slot_bricks
 * (src/voxel.rs:1322-1500: terrain, biomes, ores, decoration, trees) on the
 * device.  A storage chunk is 8x8x8 bricks (32^3 voxels); world chunk
 * (cx, cy, cz) lives in slot (pos_mod(cx, bricks_x/8), cy,
 * pos_mod(cz, bricks_z/8)), the toroidal mapping of shift_origin
 * (src/voxel.rs:507-537).  Masks and LUTs are rebuilt afterwards.  All three
 * calls are synchronous.
 *
 * vx_world_gen_chunks: generate the n world chunks of `chunks` (n x, y, z
 * triples, host memory; 0 <= y < bricks_y/8, |x|, |z| < 2^24) into their
 * slots; of two chunks for one slot the later wins. */
int vx_world_gen_chunks(VxWorld *w, uint64_t seed, const int32_t *chunks, uint32_t n);
/* fill_demo_terrain (src/voxel.rs:1005-1060) for a window whose lower corner
 * is world chunk (origin_cx, 0, origin_cz): every slot generated.  The
 * camera's world_origin for this window is (32*origin_cx, 0, 32*origin_cz). */
int vx_world_fill_window(VxWorld *w, uint64_t seed, int32_t origin_cx, int32_t origin_cz);
/* shift_origin (src/voxel.rs:507-537) after vx_world_fill_window: only the
 * slots whose world chunk changes are regenerated, with the fill's seed,
 * and get the recorded edits inside them (vx_world_apply_edit); their count
 * goes to *n_regenerated when non-null.  VX_ERR_INVALID when no
 * window was filled, or vx_world_upload / vx_world_generate replaced it. */
int vx_world_shift_origin(VxWorld *w, int32_t origin_cx, int32_t origin_cz,
                          uint32_t *n_regenerated);
/* apply_edit (src/voxel.rs:448-474): a persistent edit at world voxel
 * (wx, wy, wz), |wx|, |wz| < 2^29.  It is kept in the world's edit log (a
 * later edit of the same voxel replaces it) and written on the device now
 * when it lies inside the window -- the one of the last vx_world_fill_window
 * or vx_world_shift_origin, else the window at origin 0.  Every chunk that a
 * later vx_world_fill_window, vx_world_shift_origin or vx_world_gen_chunks
 * generates gets the edits inside it written again (replay_edits_for_chunk,
 * src/voxel.rs:571-603), so edits survive streaming.  mat 0 clears the voxel
 * (Brick::set).  Masks and LUTs are updated.  Synchronous. */
int vx_world_apply_edit(VxWorld *w, int32_t wx, int32_t wy, int32_t wz, uint8_t mat);
/* Forget every recorded edit (the device world is left as it is). */
int vx_world_clear_edits(VxWorld *w);
/* Checkpoint of a device world in a .vxw file: the six arrays in voxelG's
 * host layout, the edit log and the chunk generator's window state.  The
 * reference keeps its world only as (seed, edit log); this dump restores a
 * device world exactly, for debugging and resume.  vx_world_load requires
 * a world of the same dims (VX_ERR_INVALID otherwise, and on a truncated
 * or foreign file).  Both synchronous. */
int vx_world_save(VxWorld *w, const char *path);
int vx_world_load(VxWorld *w, const char *path);
/* Incremental update from dirty bricks (renderer.rs:1345-1394): writes the
 * given bricks and recomputes the touched tile/chunk/L4 masks and uniform
 * LUT entries on the device (voxel.rs:879-946 semantics).  brick_idx and
 * bricks are host arrays of n entries, copied before the call returns;
 * duplicates allowed (the last entry wins, resolved on the device).  With a
 * stream the update is asynchronous and ordered on that stream (and before
 * the library's later calls on this world); stream NULL waits for it. */
int vx_world_apply_dirty(VxWorld *w, const uint32_t *brick_idx, const VxBrick *bricks,
                         size_t n, void *stream);
/* The checked library.  libvoxrt_checked.so is built from the same sources
 * with every world-array load of the traversal compared with the array's
 * length first (a stand-in for a memory checker).  A bad index is not read:
 * the load returns 0 and the first such index is kept in a per-world word,
 * array id << 56 | index (ids: 1 L4 mask, 2 chunk mask, 3 tile mask,
 * 4 tile skip word, 5 tile LUT, 6 occupancy, 7 brick LUT, 8 materials).
 * vx_checked_build returns 1 in the checked library and 0 in libvoxrt.so,
 * whose word stays 0.  vx_world_oob waits for the device, reads the word
 * (0 = no bad index) and clears it when `clear` is nonzero. */
int vx_checked_build(void);
int vx_world_oob(VxWorld *w, uint64_t *word, int32_t clear);
/* Counts of each array: bricks, tiles, chunks, l4 cells. */
int vx_world_counts(const VxWorld *w, uint64_t counts[4]);

/* Launch shape of the frame kernels.  persistent = 0: one CTA per 16x8
 * pixels (default); 1: one wave of CTAs whose warps pull 8x4 pixel tiles from
 * a counter.  Results are identical either way. */
typedef struct {
    int32_t persistent;
    int32_t reserved[7];
} VxTuning;
int vx_world_set_tuning(VxWorld *w, const VxTuning *t);
int vx_world_get_tuning(const VxWorld *w, VxTuning *t);

/* ---- traversal --------------------------------------------------------- */
/* raycast(camera_world, dir, world, world_origin) (src/raycast.rs:21): returns
 * 1 on a hit (fills *out), 0 on a miss, <0 on error.  Synchronous. */
int vx_raycast(VxWorld *w, const float cam[3], const float dir[3], const int32_t origin[3],
               VxPickHit *out);
/* Batched raycast over device arrays: cams/dirs are n*3 floats, hit[i] = 1/0. */
int vx_raycast_batch(VxWorld *w, const int32_t origin[3], const float *cams_dev,
                     const float *dirs_dev, size_t n, VxPickHit *out_dev, int32_t *hit_dev,
                     void *stream);
/* Batched generic rays (trace / trace_any / trace_no_water) over device
 * arrays; origin is the loaded-window corner. */
int vx_trace(VxWorld *w, const int32_t origin[3], const VxRay *rays_dev, size_t n,
             const VxTraceParams *p, VxHitRecord *out_dev, void *stream);
/* One primary frame: beam pre-pass (VX_F_BEAM) + per-pixel trace
 * (raymarch.wgsl:576-631) + one shadow ray per hit (VX_F_SHADOW).
 * rec_dev: res_x*res_y records, row-major; shadow_dev may be NULL when
 * VX_F_SHADOW is off.  The beam scratch is owned by the world. */
int vx_render_primary(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                      VxHitRecord *rec_dev, VxShadowRecord *shadow_dev, void *stream);
/* Contact AO of the primary hits of a frame (compute_ao, raymarch.wgsl
 * :4417-4475): for each record of rec_dev (a vx_render_primary frame of the
 * same camera, any method flags), the hierarchical solid test of the 12
 * neighbours of its entry-face corners, the corner rule and the bilinear
 * mix, with the skip rule of :3862-3863 (beyond 64 voxels, leaf blocks,
 * leaf fringe).  ao_dev[i] = 1 for misses and skipped hits. */
int vx_render_ao(VxWorld *w, const VxCamera *cam, const VxHitRecord *rec_dev, float *ao_dev,
                 void *stream);
/* Rows [y0, y1) of the frame of vx_render_primary (beam over the whole
 * frame): their records and shadow records are written at their frame
 * positions, rec_dev[y * res_x + x], and every other entry is left as it
 * was, so rec_dev must hold y1 * res_x records.  Ranks that split a frame by
 * rows each render their range into a frame-sized buffer and gather the
 * ranges (voxelg_b200/replicas.py render_split).  Records equal the whole
 * frame's.  Asynchronous on `stream`. */
int vx_render_primary_rows(VxWorld *w, const VxCamera *cam, const VxTraceParams *p, uint32_t y0,
                           uint32_t y1, VxHitRecord *rec_dev, VxShadowRecord *shadow_dev,
                           void *stream);
/* Same frame through host buffers: the records are copied to rec_host /
 * shadow_host (pinned memory recommended) before the call returns.  The
 * frame renders in four row bands, each copied while the next renders. */
int vx_render_primary_host(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                           VxHitRecord *rec_host, VxShadowRecord *shadow_host);
/* The same, for frame pipelines: enqueues the frame and returns.  Its
 * records are in rec_host / shadow_host once vx_render_host_wait(w) returns;
 * until then the caller must neither read nor free those buffers (pinned
 * memory, for the copies to overlap).  Frames alternate between two device
 * buffers, so frame N+1's traversal overlaps frame N's copies to the host,
 * and the copies of successive frames land in call order.  Each frame is
 * copied whole (one copy per buffer): in a pipeline, fewer copies are
 * faster than bands. */
int vx_render_primary_host_async(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                                 VxHitRecord *rec_host, VxShadowRecord *shadow_host);
/* Waits until every frame enqueued by vx_render_primary_host_async has
 * landed in its host buffers.
 * Lost staging copies: the beam pre-pass stages the chunk masks in shared
 * memory with one bulk copy and waits for it a bounded time.  A block that
 * gives up reads global memory instead (its beam cells stay exact) and, if
 * the copy has still not landed when it exits, records that in the world.
 * The next synchronising call on the world -- vx_render_primary_host,
 * vx_render_host_wait, vx_render_primary_stats, vx_render_primary_timed or
 * vx_world_oob -- then returns VX_ERR_DEVICE once with a message. */
int vx_render_host_wait(VxWorld *w);
/* vx_render_primary_host / _async with packed records: out_host (res_x *
 * res_y entries, pinned memory recommended) receives the frame as
 * VxPackedRecord, half the bytes of records plus shadow records.  The
 * async form shares the two-buffer pipeline and vx_render_host_wait of
 * vx_render_primary_host_async.  VX_ERR_INVALID when the window has more
 * than 2^32 voxels or max_iters / any_max_iters exceed 65535. */
int vx_render_primary_host_packed(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                                  VxPackedRecord *out_host);
int vx_render_primary_host_packed_async(VxWorld *w, const VxCamera *cam,
                                        const VxTraceParams *p, VxPackedRecord *out_host);
/* The same with VxCompactRecord (12 bytes per pixel).  VX_ERR_INVALID when
 * the window has more than 2^30 voxels, max_iters > 2047 or
 * any_max_iters > 1023. */
int vx_render_primary_host_compact(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                                   VxCompactRecord *out_host);
int vx_render_primary_host_compact_async(VxWorld *w, const VxCamera *cam,
                                         const VxTraceParams *p, VxCompactRecord *out_host);
/* The chunk generator's binary32 transcendentals, equal to the host C
 * library's (as the reference's f32::powf / cos / sin are) on the
 * generator's domains: fn 0 powf(x, 1.15f) and fn 1 powf(x, 0.85f) for
 * every x in [0, 1] (src/voxel.rs:1262, :1623), fn 2 cosf and fn 3 sinf for
 * every branch angle paint_tree forms (:1633-1641, :1689-1697).  Elsewhere
 * in [0, 1] / |x| <= 16 they are the library's own double-precision
 * evaluations rounded to binary32.  Built from an exception table that
 * voxelg_b200/build.py writes beside the library for the C library it runs
 * on; VX_ERR_INVALID when the table is missing or was built for another.
 * vx_gen_math: n device inputs to n device outputs on the world's device
 * (asynchronous on `stream`; NULL = the world's stream, waited for).
 * vx_gen_math_host: the same on the host. */
int vx_gen_math(VxWorld *w, uint32_t fn, const float *in_dev, size_t n, float *out_dev,
                void *stream);
int vx_gen_math_host(uint32_t fn, const float *in, size_t n, float *out);
/* Host: n packed records back to VxHitRecord / VxShadowRecord, byte for
 * byte what vx_render_primary_host writes.  world_origin is the frame
 * camera's world_origin, window_voxels the world's voxel counts
 * (4 * bricks per axis).  Either output pointer may be NULL. */
int vx_unpack_records(const VxPackedRecord *packed, size_t n, const int32_t world_origin[3],
                      const uint32_t window_voxels[3], VxHitRecord *rec, VxShadowRecord *shadow);
/* The same for VxCompactRecord. */
int vx_unpack_compact_records(const VxCompactRecord *compact, size_t n,
                              const int32_t world_origin[3], const uint32_t window_voxels[3],
                              VxHitRecord *rec, VxShadowRecord *shadow);
/* The frame of vx_render_primary, run once more with algorithmic load
 * counters on: bytes the method reads (8 per mask word / occupancy, 1 per
 * LUT or material byte) and loop iterations, summed over all rays.
 * stats = {beam bytes, beam iterations, primary+shadow bytes, primary+shadow
 * iterations}. */
int vx_render_primary_stats(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                            uint64_t stats[4]);
/* vx_render_primary followed by a stream synchronize, with CUDA events
 * recorded on `stream` around each kernel: ms[0] = beam pre-pass,
 * ms[1] = primary (+shadow) kernel. */
int vx_render_primary_timed(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                            VxHitRecord *rec_dev, VxShadowRecord *shadow_dev, void *stream,
                            float ms[2]);

/* ---- mixed ray queue (persistent, graph-captured, autotuned) -------------
 * No single reference function: voxelG traces primary, shadow, GI-probe and
 * picking rays in separate passes (raymarch.wgsl cs_main/trace_any,
 * gi_probes.wgsl, raycast.rs).  Here one persistent launch walks a queue of
 * VxRay of any mix of kinds (VxRay.kind low bits) and lengths (VxRay.tmax);
 * a kind-0 ray flagged VX_RAY_SPAWN_SHADOW that hits continues with one
 * shadow any-hit ray toward VxTraceParams.sun (jitter seeded by the ray
 * index i: ign(i & 0xFFFF, i >> 16, frame)), recorded in shadow_dev[i].
 * rays_dev must be 16-byte aligned; out_dev / shadow_dev 8-byte aligned; when
 * shadow_dev is given every entry is written ({0,0} for rays without a
 * shadow).  Records are identical for every tuning. */
#define VX_RAY_SPAWN_SHADOW (1u << 8)

typedef struct {
    int32_t block_threads;  /* 64, 128 or 256                                  */
    int32_t refill_min;     /* idle lanes a warp waits for before refilling, 1..32 */
    int32_t ctas_per_sm;    /* 0 = as many as fit                              */
    int32_t sort;           /* 1 = reorder by (kind, origin cell, direction) first */
    int32_t reserved[4];
} VxQueueTuning;

int vx_queue_default_tuning(VxQueueTuning *t);
int vx_queue_run(VxWorld *w, const int32_t origin[3], const VxRay *rays_dev, size_t n,
                 const VxTraceParams *p, const VxQueueTuning *t, VxHitRecord *out_dev,
                 VxShadowRecord *shadow_dev, void *stream);
/* Time every candidate tuning on this queue (median of `reps` runs each),
 * check that all give byte-identical outputs (VX_ERR_DEVICE if not), and
 * return the fastest in *best with its time in *best_ms.  Synchronous; the
 * outputs hold the last run's records. */
int vx_queue_autotune(VxWorld *w, const int32_t origin[3], const VxRay *rays_dev, size_t n,
                      const VxTraceParams *p, VxHitRecord *out_dev, VxShadowRecord *shadow_dev,
                      int32_t reps, VxQueueTuning *best, float *best_ms);

/* The queue launch captured once into a CUDA graph (scratch owned by the
 * graph object); each vx_queue_graph_launch replays it on `stream`.  The
 * pointers and parameters are fixed at capture. */
typedef struct VxQueueGraph VxQueueGraph;
int vx_queue_graph_create(VxWorld *w, const int32_t origin[3], const VxRay *rays_dev, size_t n,
                          const VxTraceParams *p, const VxQueueTuning *t, VxHitRecord *out_dev,
                          VxShadowRecord *shadow_dev, VxQueueGraph **out);
int vx_queue_graph_launch(VxQueueGraph *g, void *stream);
int vx_queue_graph_destroy(VxQueueGraph *g);

/* ---- ray-query serving loop ---------------------------------------------
 * The reference's headless server (src/server.rs:6-102) relays edits and
 * poses and holds no world; picking runs client-side (src/app.rs:523-557).
 * This is the device-resident counterpart: clients submit batches of
 * VxRay queries (picking, line-of-sight, physics probes) against one world.
 * World edits enter the same FIFO and are ordered against every request
 * before and after them.  Results are byte-identical to running each
 * request alone through vx_trace on the same world.  Two modes:
 *
 * VX_SERVE_SLOTS: a server thread forms batches continuously from whatever
 * has arrived, admits them into a fixed set of device slots sized by the
 * memory budget (a request waits while no slot is free), and runs each
 * batch on its own stream, so batches that arrive while others are on the
 * GPU overlap on the device.
 *
 * VX_SERVE_RESIDENT: one persistent launch stays on the device and takes
 * requests from a descriptor ring in page-locked host memory mapped into
 * the device's address space; its warps split requests into 32-ray units
 * as they arrive, read the rays and write the records straight from and to
 * host memory (the caller's buffers when they are page-locked, else
 * page-locked staging), and mark each request done in host memory.  The
 * budget bounds the rays in flight (56 B per ray: ray plus record).  The
 * launch ends after idle_us without a request, at an edit (which runs on
 * the same stream after it), or after a fraction of a second (the server
 * starts the next); every wait in it is bounded and a wait that runs out
 * is reported (VX_ERR_DEVICE) instead of hanging. */
#define VX_SERVE_SLOTS 0
#define VX_SERVE_RESIDENT 1
typedef struct {
    uint64_t mem_budget_bytes;  /* bytes for all requests in flight (56 B per ray) */
    int32_t slots;              /* SLOTS: batches in flight at once, 1..16     */
    int32_t max_batch_rays;     /* rays per batch (per request when RESIDENT);
                                   0 = budget / slots / 56 (budget / 56)       */
    int32_t max_batch_requests; /* SLOTS: requests per batch; 0 = as many as fit */
    int32_t mode;               /* VX_SERVE_SLOTS or VX_SERVE_RESIDENT         */
    int32_t idle_us;            /* RESIDENT: idle time before the launch ends;
                                   0 = 2000                                     */
    int32_t wait_us;            /* RESIDENT: bound on a warp's wait for its work;
                                   0 = the launch's lifetime plus one second.  A
                                   wait that runs out stops the server with
                                   VX_ERR_DEVICE (a watchdog: a shorter bound
                                   than idle_us ends idle launches that way)   */
} VxServeConfig;

/* batches: SLOTS batches launched, or RESIDENT launches of the loop. */
typedef struct {
    uint64_t requests, rays, batches, rejected, edits, edited_bricks;
    double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> results in the caller's buffer */
    double seconds;                         /* wall time covered (bench: from the
                                               first arrival to the last request
                                               reaped by its client) */
    double mrays_per_s;
    uint64_t peak_inflight_rays;
} VxServeStats;

typedef struct VxServer VxServer;
int vx_server_create(VxWorld *w, const int32_t origin[3], const VxTraceParams *p,
                     const VxServeConfig *cfg, VxServer **out);
/* Queue n host rays; *out (host, n records) is written before the ticket
 * completes.  Both buffers must stay valid until then.  VX_ERR_BUSY when n
 * exceeds a slot (max_batch_rays). */
int vx_server_submit(VxServer *s, const VxRay *rays, size_t n, VxHitRecord *out,
                     uint64_t *ticket);
/* 1 done, 0 pending, VX_ERR_INVALID for an unknown ticket. */
int vx_server_poll(VxServer *s, uint64_t ticket);
/* Block until done (1) or timeout_s elapses (0). */
int vx_server_wait(VxServer *s, uint64_t ticket, double timeout_s);
/* Queue a dirty-brick update (vx_world_apply_dirty semantics, host arrays
 * copied at the call) between the requests submitted before and after it. */
int vx_server_edit(VxServer *s, const uint32_t *brick_idx, const VxBrick *bricks, size_t n);
/* Latency / throughput of the requests completed since create (or reset). */
int vx_server_stats(VxServer *s, VxServeStats *st, int32_t reset);
int vx_server_destroy(VxServer *s);

/* Built-in load generator: `clients` threads with Poisson arrivals of
 * `rate_per_client` requests/s each for `seconds`; each request has a
 * log-uniform size in [min_rays, max_rays] and max length log-uniform in
 * [min_len, max_len] (kinds: first hit or line of sight), origins / directions
 * seeded; meanwhile `edit_fraction_per_s` of all bricks per second are
 * re-randomized through vx_server_edit.  Fills *st for this run. */
typedef struct {
    int32_t clients;
    float rate_per_client;
    float seconds;
    int32_t min_rays, max_rays;
    float min_len, max_len;
    float edit_fraction_per_s;
    uint64_t seed;
} VxServeLoad;
int vx_serve_bench(VxServer *s, const VxServeLoad *load, VxServeStats *st);

/* ---- temporal differential (src/temporal.rs, src/app.rs:643-767) ------- */
/* Screen tiles are 8x8 pixels, tiles_w = ceil(W/8); bit ti of the u32 word
 * ti/32 of a tile mask marks tile ti dirty (the tile_dirty buffer of
 * shaders/raymarch.wgsl:580-587). */
/* OR into tile_mask_dev the tiles covered by the world AABBs of the given
 * slot bricks as seen by cam (temporal::project_brick_to_tiles,
 * src/temporal.rs:16-111).  brick_idx is a host array; returns after the
 * launch is enqueued and the indices are consumed. */
int vx_project_dirty(VxWorld *w, const VxCamera *cam, const uint32_t *brick_idx, size_t n,
                     uint32_t *tile_mask_dev, void *stream);
/* OR in the rotating hash-scattered refresh set of src/app.rs:706-725 for a
 * width x height frame: tiles with hash % spread == phase. */
int vx_tile_refresh(uint32_t width, uint32_t height, uint32_t spread, uint32_t phase,
                    uint32_t *tile_mask_dev, void *stream);
/* vx_render_primary with cs_main's tile gate: pixels of tiles whose bit is
 * clear are not traced and their records are left as they were. */
int vx_render_primary_gated(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                            const uint32_t *tile_mask_dev, VxHitRecord *rec_dev,
                            VxShadowRecord *shadow_dev, void *stream);

/* ---- frames for callers that cannot allocate ------------------------------
 * No counterpart in the reference: an addition for hosts that reserve all
 * device memory up front and forbid (or cannot afford) cudaMalloc once
 * running -- a plugin handed pre-allocated buffers, a frame loop where the
 * device synchronization of cudaMalloc/cudaFree is a hitch.
 *
 * The caller owns the world in device memory, laid out as this library keeps
 * it: occupancy = one u64 per brick (brick index bx + by*BX + bz*BX*BY),
 * materials = 64 bytes per brick in the same order (voxel x + z*4 + y*16),
 * masks / LUTs exactly as the host arrays of vx_world_upload. */
typedef struct {
    int32_t bricks_x, bricks_y, bricks_z;  /* same rules as VxWorldDesc */
    const uint64_t *occupancy;             /* n_bricks                  */
    const uint8_t *materials;              /* n_bricks * 64             */
    const uint64_t *tile_mask;
    const uint64_t *chunk_mask;
    const uint64_t *l4_mask;
    const uint8_t *brick_uniform;
    const uint8_t *tile_uniform;
} VxWorldView;

/* vx_render_primary over a caller-owned world, allocating nothing: the beam
 * scratch is a static device array of 480x270 cells built into the library
 * (each GPU that loads it holds 512 KiB until exit).  With VX_F_BEAM set, a
 * frame whose beam grid (ceil(w/8) x ceil(h/8) cells) exceeds 129600 cells
 * is rejected with VX_ERR_INVALID; without the beam any resolution up to
 * 32768 passes.  occupancy, the three mask arrays, rec_dev and shadow_dev
 * must be 8-byte aligned (else VX_ERR_INVALID, nothing launched).  Runs on
 * the calling thread's current device and context.  The first call in a
 * context looks up the array's address there (make it before any stream
 * capture); the address is cached with the context's id, so calls after a
 * cudaDeviceReset look it up again.  All calls on a device share the array:
 * calls that overlap on the GPU race on it.  The beam pre-pass reads the
 * chunk masks with plain loads here (no shared-memory staging).
 * Asynchronous on `stream`. */
int vx_render_primary_noalloc(const VxWorldView *world, const VxCamera *cam,
                              const VxTraceParams *p, VxHitRecord *rec_dev,
                              VxShadowRecord *shadow_dev, void *stream);

/* ---- ray-query messages in voxelG's network framing ----------------------
 * For clients of src/net.rs: a frame is a u32 little-endian payload length
 * (at most 16 MiB, net.rs:71-90) and a payload that bincode 1.3.3 writes
 * for two variants appended to net.rs's `Message` (net.rs:46-67) after
 * `Heartbeat`:
 *   RayQuery  { id: u64, rays: Vec<WireRay> }         variant index 10
 *   RayResult { id: u64, records: Vec<WireRecord> }   variant index 11
 *   WireRay    { org: [f32; 3], dir: [f32; 3], tmax: f32, kind: u32 }
 *   WireRecord { voxel: [i32; 3], face: u8, mat: u8, flags: u8, t: f32,
 *                steps: u32 }
 * (variant index u32, fixed-width little-endian fields, Vec as a u64 count
 * and its elements).  The decoders reject frames whose prefix, variant or
 * count disagrees with their length.  Host-only: no device is touched. */
size_t vx_wire_query_bytes(size_t n);    /* whole frame, prefix included */
size_t vx_wire_result_bytes(size_t n);
int vx_wire_encode_query(uint64_t id, const VxRay *rays, size_t n, uint8_t *buf, size_t cap,
                         size_t *len);
int vx_wire_decode_query(const uint8_t *buf, size_t len, uint64_t *id, VxRay *rays, size_t cap,
                         size_t *n);
int vx_wire_encode_result(uint64_t id, const VxHitRecord *rec, size_t n, uint8_t *buf,
                          size_t cap, size_t *len);
int vx_wire_decode_result(const uint8_t *buf, size_t len, uint64_t *id, VxHitRecord *rec,
                          size_t cap, size_t *n);

/* ---- learned start-distance proposal ------------------------------------
 * No counterpart in the reference.  A 70 -> 64 -> 64 -> 64 -> 1 MLP with
 * GELU (tanh form) predicts log(first-hit t) of a ray from 6 ray values
 * (origin mod 64 / 64, direction) and the 64 tile bits of the chunk that
 * holds the origin.  Parameters: VX_MLP_FLOATS f32 in the order
 *   W1[64][80] (columns 70..79 are padding, kept at zero), b1[64],
 *   W2[64][64], b2[64], W3[64][64], b3[64], wo[64], bo
 * -- 12,929 trained values.  Training runs on the device with the library's
 * own forward / backward / Adam kernels on rays labelled by the plain DDA;
 * inference runs on BF16 tensor cores with FP32 accumulation.
 *
 * vx_render_learned uses a proposal only to decide how far a verification
 * walk checks the ray before the DDA restarts past the verified cells; the
 * records equal vx_render_primary's with the same method flags and no beam,
 * except `steps` (the iterations actually executed). */
#define VX_MLP_FLOATS 13569
#define VX_MLP_FEATURES 80
typedef struct VxProposal VxProposal;

typedef struct {
    uint32_t poses;          /* random camera poses                            */
    uint32_t rays_per_pose;  /* random pixel positions per pose                */
    uint32_t steps;          /* Adam steps                                     */
    uint32_t batch;          /* samples per step (<= 65536)                    */
    float lr;                /* peak learning rate (cosine decay to lr/20)     */
    float y_min, y_max;      /* camera height range (window voxels)            */
    float pitch_min, pitch_max; /* radians                                     */
    float fov_y;             /* radians                                        */
    uint32_t width, height;  /* image the random pixels are drawn from         */
    uint32_t flags;          /* method flags of the plain DDA that labels rays */
    uint32_t held_out_poses; /* extra poses for the held-out loss              */
    uint64_t seed;
} VxTrainConfig;

/* 200 poses x 81920 rays (16.4M pairs), 3000 steps of 16384, lr 2e-3,
 * heights 100..200, pitch -40..+10 deg, vfov 70 deg, 1920x1080, flags
 * L4|LUT|LOD, 8 held-out poses, seed 1. */
int vx_proposal_default_config(VxTrainConfig *c);
/* Random initial parameters (seeded) on the world's device. */
int vx_proposal_create(VxWorld *w, uint64_t seed, VxProposal **out);
int vx_proposal_destroy(VxProposal *p);
/* Copy the f32 parameters out / in (n = VX_MLP_FLOATS); set also refreshes
 * the BF16 inference copy and resets the Adam state. */
int vx_proposal_get_params(VxProposal *p, float *host, size_t n);
int vx_proposal_set_params(VxProposal *p, const float *host, size_t n);
/* Features of n rays (n x VX_MLP_FEATURES f32, device) for a window corner. */
int vx_proposal_features(VxProposal *p, VxWorld *w, const int32_t origin[3],
                         const VxRay *rays_dev, size_t n, float *feats_dev, void *stream);
/* FP32 forward + backward of one batch against targets (log t): the mean
 * squared error and its gradient (VX_MLP_FLOATS, host).  Synchronous. */
int vx_proposal_grad(VxProposal *p, const float *feats_dev, const float *target_dev,
                     uint32_t batch, float *grad_host, float *loss);
/* BF16 tensor-core inference: out_dev[i] = predicted log t.  Asynchronous. */
int vx_proposal_infer(VxProposal *p, const float *feats_dev, size_t n, float *out_dev,
                      void *stream);
/* Label rays of random poses with the plain DDA on `w`, then train.
 * loss_curve (c->steps floats, may be NULL) receives every step's batch
 * loss, held_out (may be NULL) the loss over the held-out poses before [0]
 * and after [1] training.  Synchronous. */
int vx_proposal_train(VxProposal *p, VxWorld *w, const VxTrainConfig *c, float *loss_curve,
                      float held_out[2]);

typedef struct {
    uint64_t none;       /* rays whose verification verified no cell           */
    uint64_t partial;    /* stopped before the proposal; restarted earlier     */
    uint64_t accepted;   /* verified up to the proposed distance               */
    uint64_t miss;       /* verified to the window edge / max_dist: a miss     */
    uint64_t cells;      /* verification cells stepped                         */
    uint64_t iters;      /* DDA iterations executed                            */
    uint64_t fallback;   /* restarts that met the iteration cap (plain re-run) */
    uint64_t rays;
    float infer_ms;      /* proposal inference (0 without a proposal)          */
    float trace_ms;      /* verification + traversal                           */
} VxLearnedStats;

/* Primary frame, learned form: proposal inference (skipped when prop is
 * NULL: the verification then runs until it fails) and the verified-restart
 * traversal.  t_target = exp(proposal) * scale.  p->flags must not hold
 * VX_F_BEAM or VX_F_SHADOW.  With stats != NULL the call is synchronous and
 * fills the counters and CUDA-event times; else asynchronous on `stream`.
 * The per-pixel proposals live in the VxProposal: asynchronous calls with
 * one proposal must not overlap on different streams. */
int vx_render_learned(VxWorld *w, VxProposal *prop, const VxCamera *cam,
                      const VxTraceParams *p, float scale, VxHitRecord *rec_dev,
                      VxLearnedStats *stats, void *stream);

/* ---- host world (mirror of src/voxel.rs World, for C/C++ callers) ------ */
int vx_host_world_create(int32_t bricks_x, int32_t bricks_y, int32_t bricks_z,
                         VxHostWorld **out);
int vx_host_world_destroy(VxHostWorld *h);
/* Borrow the array pointers (valid until destroy). */
int vx_host_world_arrays(VxHostWorld *h, VxBrick **bricks, uint64_t **tile_mask,
                         uint64_t **chunk_mask, uint64_t **l4_mask, uint8_t **brick_uniform,
                         uint8_t **tile_uniform);
/* World::set_voxel (voxel.rs:916-935) at slot coords. */
int vx_host_world_set_voxel(VxHostWorld *h, uint32_t x, uint32_t y, uint32_t z, uint8_t mat);
/* World::apply_edit (voxel.rs:450-474) at world coords for a window origin. */
int vx_host_world_apply_edit(VxHostWorld *h, int32_t wx, int32_t wy, int32_t wz, uint8_t mat,
                             const int32_t origin[3]);
/* rebuild_all_masks + rebuild_all_uniform (voxel.rs:946-1000); marks all dirty. */
int vx_host_world_rebuild(VxHostWorld *h);
/* Number of pending dirty bricks (sorted + deduped on read). */
int64_t vx_host_world_dirty_count(VxHostWorld *h);
/* Renderer::upload_world: full upload if all-dirty, else the dirty bricks
 * only through vx_world_apply_dirty; clears the dirty state. */
int vx_world_sync(VxWorld *w, VxHostWorld *h, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* VOXRT_H */
