/*
 * voxoracle.h -- CPU oracle for the voxelG ray-traversal path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithms, used as the checker for the CUDA library (libvoxrt).  Only the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark may
 * load it.  The product never links or calls it.
 *
 * What it restates (reference = marcstampfli1/voxelG):
 *   O1  flat CPU DDA            src/raycast.rs:19-141
 *   O2  hierarchical DDA        shaders/raymarch.wgsl:3321-3448, :4306-4409,
 *                               :4481-4505, :4541-4598, :4600-4864,
 *                               shaders/beam.wgsl:51-113, common.wgsl:49-58
 *   world layout + pyramid      src/voxel.rs:190-301, :879-1000
 *   noise primitives            src/voxel.rs:1163-1232, :1999-2021
 *
 * Parity pinning: the reference is Rust + WGSL and cannot be built or run in
 * this environment (no Rust toolchain, no graphics API).  The oracle is
 * pinned to the reference's own known-answer tests, restated as tests
 * (src/accel.rs:529-572 flat floor, :606-759 clean-hit agreement with
 * raycast(), :837-917 shadow occlusion, :920-942 empty world,
 * tests/worldgen.rs:19-45 determinism).  No numeric golden vectors exist
 * upstream, so bit-level parity of O2 with the WGSL itself rests on the
 * line-by-line restatement ("parity partially unpinned").
 *
 * Build: gcc -O2 -ffp-contract=off -fno-fast-math -fPIC -shared (IEEE f32,
 * no FMA contraction -- the same operation order the CUDA kernels use).
 */
#ifndef VOXORACLE_H
#define VOXORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Brick, repr(C) 72 bytes: src/voxel.rs:296-301.  Voxel bit x + z*4 + y*16. */
typedef struct {
    uint64_t occupancy;
    uint8_t materials[64];
} OrBrick;

/* World arrays in the reference's host layout (src/voxel.rs:328-343).
 * Dims are in bricks; derived counts follow src/world_dims.rs:12-37. */
typedef struct {
    int32_t bx, by, bz;
    OrBrick *bricks;          /* bx*by*bz, index bx + by*BX + bz*BX*BY          */
    uint64_t *tile_mask;      /* (bx/4)*(by/4)*(bz/4)                            */
    uint64_t *chunk_mask;     /* ceil(tx/4)*ceil(ty/4)*ceil(tz/4)                */
    uint64_t *l4_mask;        /* ceil(cx/4)*ceil(cy/4)*ceil(cz/4)                */
    uint8_t *brick_uniform;   /* one byte per brick                              */
    uint8_t *tile_uniform;    /* one byte per tile                               */
} OrWorld;

/* Camera uniform subset the traversal reads (shaders/common.wgsl:7-42). */
typedef struct {
    float origin[3];
    float forward[3];
    float right[3];
    float up[3];
    float tan_half_fov;
    float res_x, res_y;
    float jitter_x, jitter_y;
    int32_t world_origin[3];
} OrCamera;

/* Method switches (reference constants are the defaults). */
enum {
    OR_F_L4 = 1u << 0,        /* !PROFILE_NO_L4 (raymarch.wgsl:403)              */
    OR_F_LUT = 1u << 1,       /* uniform tile/brick early-out                    */
    OR_F_LOD = 1u << 2,       /* tile LOD (t>520) and brick LOD (t>400)          */
    OR_F_BEAM = 1u << 3,      /* beam pre-pass fast-forward                      */
    OR_F_SHADOW = 1u << 4,    /* one shadow (any-hit) ray per primary hit        */
};

typedef struct {
    float max_dist;          /* MAX_RAY_DIST 700        raymarch.wgsl:4501 */
    float lod_brick_t;       /* LOD_BRICK_T 400         :4489            */
    float tile_lod_t;        /* TILE_LOD_T 520          :4494            */
    float shadow_max_dist;   /* SHADOW_MAX_DIST 480     :4517            */
    float beam_margin;       /* 16 voxels               :608             */
    int32_t max_iters;       /* trace cap 1024          :4625            */
    int32_t any_max_iters;   /* trace_any cap 768       :4359            */
    uint32_t flags;          /* OR_F_*                                   */
    /* shadow-ray jitter (config: sun normalize(0.3,0.8,0.5), 0.5 deg cone) */
    float sun[3];
    float sun_tangent[3];
    float sun_bitangent[3];
    float cone_tan;
    float frame;             /* seeded interleaved-gradient-noise frame term */
} OrParams;

/* Hit record: the ray-record contract shared with the CUDA library. */
typedef struct {
    int32_t voxel[3];
    uint8_t face;     /* 2*axis + (step[axis] > 0); 0xFF = miss            */
    uint8_t mat;
    uint8_t flags;    /* bit0 hit, bit1 LOD/uniform early-out               */
    uint8_t pad;
    float t;
    uint32_t steps;   /* loop iterations executed (incl. the final one)     */
} OrRecord;

typedef struct {
    uint32_t steps;
    uint8_t occluded;
    uint8_t traced;
    uint16_t pad;
} OrShadow;

typedef struct {
    int32_t voxel[3];
    int32_t normal[3];
} OrPickHit;

/* Algorithmic load counters (bytes the method reads, by reference widths). */
typedef struct {
    uint64_t bytes;
    uint64_t iters;
} OrStats;

/* ---- world ---- */
void or_rebuild_all_masks(const OrWorld *w);            /* voxel.rs:958-1000 */
void or_rebuild_all_uniform(const OrWorld *w);          /* voxel.rs:946-957  */
uint8_t or_brick_uniform_of(const OrBrick *b);          /* voxel.rs:233-247  */
/* set_voxel at slot coords; returns brick index (dirty) or -1.  voxel.rs:916-935 */
int64_t or_set_voxel(const OrWorld *w, uint32_t x, uint32_t y, uint32_t z, uint8_t mat);

/* ---- noise + synthetic terrain ---- */
void or_seed_offset_xz(uint64_t seed, float out[2]);    /* voxel.rs:1163-1167 */
float or_fbm_2d(float x, float z, uint32_t octaves);    /* voxel.rs:1221-1232 */
float or_value_noise_3d(float x, float y, float z);     /* voxel.rs:1999-2021 */

typedef struct {
    uint64_t seed;
    float base_height;     /* 96  */
    float amplitude;       /* 48  */
    float inv_wavelength;  /* 1/128 */
    uint32_t octaves;      /* 5 */
    int32_t water_level;   /* 80 (water fills h < y <= level) */
    float cave_inv_wavelength; /* 1/32 */
    float cave_threshold;  /* 0.35 */
    int32_t dirt_depth;    /* 3 */
} OrTerrain;
/* Fill bricks (not masks) with the seeded terrain; columns [x0,x1). */
void or_generate_terrain(const OrWorld *w, const OrTerrain *t, int nthreads);

/* ---- the reference's chunk generator gen_slot_bricks (voxel.rs:1322-1500) ---- */
typedef struct {
    int32_t base[3];
    uint32_t ttype;   /* 0 oak, 1 birch, 2 pine, 3 autumn, 4 cactus */
    uint32_t hash;
} OrTree;
/* sample_terrain (voxel.rs:1244-1316): column height; *water_top if non-null */
int32_t or_sample_terrain(float wx, float wz, uint64_t seed, int32_t *water_top);
/* trees_for_chunk (voxel.rs:1537-1591): up to 12 trees, returns the count */
int or_trees_for_chunk(int32_t cx, int32_t cz, uint64_t seed, OrTree out[12]);
/* one storage chunk: 512 bricks, index x + y*8 + z*64 */
void or_gen_slot_bricks(int32_t cx, int32_t cy, int32_t cz, uint64_t seed, OrBrick *out);
/* every slot of a window whose lower corner is world chunk (ox, 0, oz), in
 * the toroidal slot shift_origin assigns (voxel.rs:507-537); then masks and
 * LUTs rebuilt.  World dims must be multiples of 8 bricks. */
void or_fill_window(const OrWorld *w, uint64_t seed, int32_t ox, int32_t oz, int nthreads);

/* ---- rays ---- */
void or_ray_dir_uv(const OrCamera *c, float u, float v, float out[3]);
void or_sincos(float x, float *s, float *c);
float or_ign(float x, float y, float frame);

/* ---- O1: raycast.rs ---- */
int or_raycast(const OrWorld *w, const float cam[3], const float dir[3],
               const int32_t origin[3], OrPickHit *out, uint32_t *steps_out);

/* ---- O2: hierarchical kinds ---- */
void or_trace(const OrWorld *w, const int32_t ro[3], const float origin[3],
              const float dir[3], float max_dist, const OrParams *p,
              OrRecord *out, OrStats *st);
int or_trace_any(const OrWorld *w, const int32_t ro[3], const float origin[3],
                 const float dir[3], float max_dist, const OrParams *p,
                 uint32_t *steps_out, OrStats *st);
void or_trace_no_water(const OrWorld *w, const int32_t ro[3], const float origin[3],
                       const float dir[3], float t_cap, const OrParams *p,
                       OrRecord *out, OrStats *st);
float or_beam_first_tile(const OrWorld *w, const OrCamera *c, const float dir[3],
                         OrStats *st);

/* beam pass over the whole 1/8-res grid (beam.wgsl:30-49) */
void or_beam_pass(const OrWorld *w, const OrCamera *c, float *beam_out, OrStats *st);
/* shadow ray for a primary hit (raymarch.wgsl:3953-3994, config cone) */
void or_shadow_ray(const OrCamera *c, const OrParams *p, uint32_t px, uint32_t py,
                   const float dir[3], const OrRecord *hit,
                   float o_out[3], float d_out[3]);
/* Full primary pass: beam (optional) + trace (+ shadow); rows [y0,y1). */
void or_render_rows(const OrWorld *w, const OrCamera *c, const OrParams *p,
                    const float *beam, uint32_t y0, uint32_t y1,
                    OrRecord *rec, OrShadow *sh, OrStats *st);
/* Multi-threaded full frame; returns wall seconds spent. */
double or_render_frame(const OrWorld *w, const OrCamera *c, const OrParams *p,
                       OrRecord *rec, OrShadow *sh, float *beam, int nthreads,
                       OrStats *st);

/* Temporal tile gating: src/temporal.rs:16-111 and src/app.rs:706-725. */
void or_project_brick_to_tiles(const OrWorld *w, const OrCamera *c, uint32_t bi, uint32_t *mask);
void or_refresh_tiles(uint32_t tiles_w, uint32_t tiles_h, uint32_t spread, uint32_t phase,
                      uint32_t *mask);

/* Contact AO of primary hits: compute_ao / ao_corner / ao_occluder /
 * is_voxel_solid (raymarch.wgsl:4417-4475, :297-322, skip rule :3862-3863).
 * ao[i] = 1 for misses and skipped hits.  Multi-threaded over rows. */
float or_compute_ao(const OrWorld *w, const OrCamera *c, const OrRecord *rec, uint32_t px,
                    uint32_t py);
void or_render_ao(const OrWorld *w, const OrCamera *c, const OrRecord *rec, float *ao,
                  int nthreads);

/* Rows offset + k*stride of a frame on nthreads threads (bounded samples). */
double or_render_row_set(const OrWorld *w, const OrCamera *c, const OrParams *p,
                         const float *beam, uint32_t stride, uint32_t offset, OrRecord *rec,
                         OrShadow *sh, int nthreads, OrStats *st);

/* Batched generic rays (the mixed queue): kind low bits 1 trace_any,
 * 2 trace_no_water, else trace; OR_RAY_SPAWN_SHADOW on a trace ray adds its
 * shadow ray after a hit (shadow record i; sh may be NULL).
 * Ray layout: org[3], dir[3], tmax, kind (32 bytes). */
#define OR_RAY_SPAWN_SHADOW (1u << 8)
typedef struct {
    float org[3];
    float dir[3];
    float tmax;
    uint32_t kind;
} OrRay;
double or_trace_batch(const OrWorld *w, const int32_t ro[3], const OrRay *rays,
                      size_t n, const OrParams *p, OrRecord *out, OrShadow *sh, int nthreads,
                      OrStats *st);
double or_raycast_batch(const OrWorld *w, const int32_t origin[3], const float *cams,
                        const float *dirs, size_t n, OrPickHit *out, int32_t *hit,
                        int nthreads);

#ifdef __cplusplus
}
#endif
/* glibc powf(x, 1.15f) (fn 0), powf(x, 0.85f) (1), cosf (2), sinf (3) on n
 * inputs with nthreads threads: the C library calls of the reference's
 * generator (src/voxel.rs:1262, :1623, :1639-1641, :1695-1697) */
void or_libm_batch(int fn, const float *x, size_t n, float *out, int nthreads);
#endif
