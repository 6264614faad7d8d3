/*
 * voxoracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY; see voxoracle.h).
 *
 * A line-by-line C restatement of the reference traversal.  Every function
 * cites the reference file:line it follows.  Arithmetic is IEEE binary32 with
 * FMA contraction disabled at compile time (-ffp-contract=off), in the
 * reference's operation order, so that the CUDA kernels (built with
 * --fmad=false) reproduce it bit for bit.
 *
 * Conventions shared with the CUDA library (the reference leaves these
 * implementation-defined in WGSL):
 *   - min(a,b) = (b < a) ? b : a ; max(a,b) = (a < b) ? b : a
 *   - normalize(v) = v / sqrt((x*x + y*y) + z*z) with IEEE sqrt and divide
 *   - f32 -> i32 conversion saturates (NaN -> 0), clamped to +-2^30 so the
 *     integer cell arithmetic that follows cannot overflow; such voxels lie
 *     far outside any window and end the ray exactly as a saturated i32 would.
 *   - Sub-voxel shading (water surface, foliage cutouts) is out of scope: a
 *     solid voxel resolves by the reference's far-distance rule at every
 *     distance -- decoration materials never stop a ray, everything else is
 *     an opaque cube (raymarch.wgsl:4541-4545 with t beyond WATER_FAR_T).
 */
#include "voxoracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------ */
/* scalar helpers                                                      */
/* ------------------------------------------------------------------ */
static inline float vmin(float a, float b) { return (b < a) ? b : a; }
static inline float vmax(float a, float b) { return (a < b) ? b : a; }
static inline float clampf(float x, float lo, float hi) { return vmin(vmax(x, lo), hi); }

static inline int32_t f2i(float x) {
    if (x != x) return 0;
    if (x >= 1073741824.0f) return 1073741824;
    if (x <= -1073741824.0f) return -1073741824;
    return (int32_t)x;
}

/* common.wgsl:49-52 */
static inline int32_t pos_mod(int32_t a, int32_t b) {
    if (a >= 0) return a % b;
    return (b - 1) - ((-1 - a) % b);
}

/* common.wgsl:55-58 ; raycast.rs:139-141 */
static inline float safe_inv(float x) {
    if (fabsf(x) < 1e-8f) return 1e30f;
    return 1.0f / x;
}

/* WGSL sign() converted to i32 ; raycast.rs:135-137 */
static inline int32_t sgn(float x) { return x > 0.0f ? 1 : (x < 0.0f ? -1 : 0); }

static inline float fractf(float x) { return x - floorf(x); }

/* Materials: src/voxel.rs:100-157, raymarch.wgsl:875-920 */
enum { MAT_GRASS = 2, MAT_DIRT = 3, MAT_STONE = 4, MAT_WATER = 12, MAT_GLASS = 18,
       MAT_LEAF_FRINGE = 33, MAT_TURF = 35 };
static inline int is_water(uint32_t m) { return m >= 5u && m <= 12u; }
static inline int is_transparent(uint32_t m) { return is_water(m) || m == MAT_GLASS; }
static inline int is_foliage(uint32_t m) {
    return m == 14u || m == 25u || m == 26u || m == 27u || m == 30u || m == 31u ||
           m == 33u || m == 34u || m == 35u || m == 36u || m == 37u;
}
static inline int is_decoration(uint32_t m) {
    return m == 30u || m == 31u || m == 33u || m == 34u || m == 35u || m == 36u || m == 37u;
}
static inline int is_uniform_optimisable(uint32_t m) {
    return !is_foliage(m) && !is_transparent(m);
}
/* resolves_as_opaque_cube (raymarch.wgsl:4541-4545) evaluated beyond both
 * sub-voxel radii: only decoration is non-opaque. */
static inline int resolves_cube(uint32_t m) { return !is_decoration(m); }
/* shadow_voxel_occludes (raymarch.wgsl:4314-4343), far-distance branch. */
static inline int shadow_occludes(uint32_t m) {
    if (m == MAT_LEAF_FRINGE || m == MAT_TURF) return 0;
    if (is_decoration(m)) return 0;
    return 1;
}

/* ------------------------------------------------------------------ */
/* world dims + index functions (world_dims.rs:9-37, voxel.rs:190-294) */
/* ------------------------------------------------------------------ */
typedef struct {
    int32_t bx, by, bz, vx, vy, vz, tx, ty, tz, cx, cy, cz, lx, ly, lz;
} Dims;

static Dims dims_of(const OrWorld *w) {
    Dims d;
    d.bx = w->bx; d.by = w->by; d.bz = w->bz;
    d.vx = d.bx * 4; d.vy = d.by * 4; d.vz = d.bz * 4;
    d.tx = d.bx / 4; d.ty = d.by / 4; d.tz = d.bz / 4;
    d.cx = (d.tx + 3) / 4; d.cy = (d.ty + 3) / 4; d.cz = (d.tz + 3) / 4;
    d.lx = (d.cx + 3) / 4; d.ly = (d.cy + 3) / 4; d.lz = (d.cz + 3) / 4;
    return d;
}
static inline int64_t brick_idx(const Dims *d, int32_t x, int32_t y, int32_t z) {
    return (int64_t)x + (int64_t)y * d->bx + (int64_t)z * d->bx * d->by;
}
static inline int64_t tile_idx(const Dims *d, int32_t x, int32_t y, int32_t z) {
    return (int64_t)x + (int64_t)y * d->tx + (int64_t)z * d->tx * d->ty;
}
static inline int64_t chunk_idx(const Dims *d, int32_t x, int32_t y, int32_t z) {
    return (int64_t)x + (int64_t)y * d->cx + (int64_t)z * d->cx * d->cy;
}
static inline int64_t l4_idx(const Dims *d, int32_t x, int32_t y, int32_t z) {
    return (int64_t)x + (int64_t)y * d->lx + (int64_t)z * d->lx * d->ly;
}
static inline int child_bit(int32_t lx, int32_t ly, int32_t lz) { return lx + lz * 4 + ly * 16; }

/* voxel.rs:233-247 */
uint8_t or_brick_uniform_of(const OrBrick *b) {
    if (b->occupancy != ~0ull) return 0;
    uint8_t m0 = b->materials[0];
    if (m0 == 0) return 0;
    for (int i = 1; i < 64; ++i)
        if (b->materials[i] != m0) return 0;
    return m0;
}

/* voxel.rs:253-272 */
static uint8_t tile_uniform_of(const Dims *d, const uint8_t *bu, int64_t ti) {
    int32_t tx = (int32_t)(ti % d->tx);
    int32_t ty = (int32_t)((ti / d->tx) % d->ty);
    int32_t tz = (int32_t)(ti / ((int64_t)d->tx * d->ty));
    int32_t bx0 = tx * 4, by0 = ty * 4, bz0 = tz * 4;
    uint8_t m0 = bu[brick_idx(d, bx0, by0, bz0)];
    if (m0 == 0) return 0;
    for (int dz = 0; dz < 4; ++dz)
        for (int dy = 0; dy < 4; ++dy)
            for (int dx = 0; dx < 4; ++dx)
                if (bu[brick_idx(d, bx0 + dx, by0 + dy, bz0 + dz)] != m0) return 0;
    return m0;
}

/* voxel.rs:946-957 */
void or_rebuild_all_uniform(const OrWorld *w) {
    Dims d = dims_of(w);
    int64_t nb = (int64_t)d.bx * d.by * d.bz;
    int64_t nt = (int64_t)d.tx * d.ty * d.tz;
    for (int64_t i = 0; i < nb; ++i) w->brick_uniform[i] = or_brick_uniform_of(&w->bricks[i]);
    for (int64_t i = 0; i < nt; ++i) w->tile_uniform[i] = tile_uniform_of(&d, w->brick_uniform, i);
}

/* voxel.rs:958-1000 */
void or_rebuild_all_masks(const OrWorld *w) {
    Dims d = dims_of(w);
    memset(w->tile_mask, 0, sizeof(uint64_t) * (size_t)d.tx * d.ty * d.tz);
    memset(w->chunk_mask, 0, sizeof(uint64_t) * (size_t)d.cx * d.cy * d.cz);
    memset(w->l4_mask, 0, sizeof(uint64_t) * (size_t)d.lx * d.ly * d.lz);
    for (int32_t bz = 0; bz < d.bz; ++bz)
        for (int32_t by = 0; by < d.by; ++by)
            for (int32_t bx = 0; bx < d.bx; ++bx)
                if (w->bricks[brick_idx(&d, bx, by, bz)].occupancy != 0)
                    w->tile_mask[tile_idx(&d, bx / 4, by / 4, bz / 4)] |=
                        1ull << child_bit(bx & 3, by & 3, bz & 3);
    for (int32_t tz = 0; tz < d.tz; ++tz)
        for (int32_t ty = 0; ty < d.ty; ++ty)
            for (int32_t tx = 0; tx < d.tx; ++tx)
                if (w->tile_mask[tile_idx(&d, tx, ty, tz)] != 0)
                    w->chunk_mask[chunk_idx(&d, tx / 4, ty / 4, tz / 4)] |=
                        1ull << child_bit(tx & 3, ty & 3, tz & 3);
    for (int32_t cz = 0; cz < d.cz; ++cz)
        for (int32_t cy = 0; cy < d.cy; ++cy)
            for (int32_t cx = 0; cx < d.cx; ++cx)
                if (w->chunk_mask[chunk_idx(&d, cx, cy, cz)] != 0)
                    w->l4_mask[l4_idx(&d, cx / 4, cy / 4, cz / 4)] |=
                        1ull << child_bit(cx & 3, cy & 3, cz & 3);
}

/* refresh_masks_for_brick, voxel.rs:879-914 */
static void refresh_masks_for_brick(const OrWorld *w, const Dims *d, int32_t bx, int32_t by,
                                    int32_t bz) {
    int64_t bi = brick_idx(d, bx, by, bz);
    int solid = w->bricks[bi].occupancy != 0;
    int32_t tx = bx / 4, ty = by / 4, tz = bz / 4;
    int64_t ti = tile_idx(d, tx, ty, tz);
    int bit = child_bit(bx & 3, by & 3, bz & 3);
    uint64_t prev = w->tile_mask[ti];
    if (solid) w->tile_mask[ti] |= 1ull << bit;
    else w->tile_mask[ti] &= ~(1ull << bit);
    uint64_t now = w->tile_mask[ti];
    if ((prev == 0) != (now == 0)) {
        int32_t cx = tx / 4, cy = ty / 4, cz = tz / 4;
        int64_t ci = chunk_idx(d, cx, cy, cz);
        int cbit = child_bit(tx & 3, ty & 3, tz & 3);
        uint64_t cprev = w->chunk_mask[ci];
        if (now == 0) w->chunk_mask[ci] &= ~(1ull << cbit);
        else w->chunk_mask[ci] |= 1ull << cbit;
        uint64_t cnow = w->chunk_mask[ci];
        if ((cprev == 0) != (cnow == 0)) {
            int64_t li = l4_idx(d, cx / 4, cy / 4, cz / 4);
            int lbit = child_bit(cx & 3, cy & 3, cz & 3);
            if (cnow == 0) w->l4_mask[li] &= ~(1ull << lbit);
            else w->l4_mask[li] |= 1ull << lbit;
        }
    }
}

/* set_voxel, voxel.rs:916-935 (+ Brick::set :309-319) */
int64_t or_set_voxel(const OrWorld *w, uint32_t x, uint32_t y, uint32_t z, uint8_t mat) {
    Dims d = dims_of(w);
    if (x >= (uint32_t)d.vx || y >= (uint32_t)d.vy || z >= (uint32_t)d.vz) return -1;
    int32_t bx = x / 4, by = y / 4, bz = z / 4;
    int vi = child_bit(x % 4, y % 4, z % 4);
    int64_t bi = brick_idx(&d, bx, by, bz);
    OrBrick *b = &w->bricks[bi];
    int was_empty = b->occupancy == 0;
    if (mat == 0) {
        b->occupancy &= ~(1ull << vi);
        b->materials[vi] = 0;
    } else {
        b->occupancy |= 1ull << vi;
        b->materials[vi] = mat;
    }
    int is_empty = b->occupancy == 0;
    if (was_empty != is_empty) refresh_masks_for_brick(w, &d, bx, by, bz);
    w->brick_uniform[bi] = or_brick_uniform_of(b);
    int64_t ti = tile_idx(&d, bx / 4, by / 4, bz / 4);
    w->tile_uniform[ti] = tile_uniform_of(&d, w->brick_uniform, ti);
    return bi;
}

/* ------------------------------------------------------------------ */
/* noise (voxel.rs:1163-1232, :1999-2021)                             */
/* ------------------------------------------------------------------ */
void or_seed_offset_xz(uint64_t seed, float out[2]) {
    float hi = (float)(int32_t)(uint32_t)(seed >> 32);
    float lo = (float)(int32_t)(uint32_t)(seed & 0xFFFFFFFFull);
    out[0] = hi * 0.01734f;
    out[1] = lo * 0.02153f;
}

static inline float hash2(int32_t x, int32_t z) {
    uint32_t h = (uint32_t)x * 0x9E3779B1u + (uint32_t)z * 0x85EBCA77u;
    h = h * 0xC2B2AE3Du;
    h = h ^ (h >> 16);
    h = h * 0x85EBCA6Bu;
    return (((float)(h & 0xFFFFFFu)) / 16777215.0f) * 2.0f - 1.0f;
}

static inline float hash3(int32_t x, int32_t y, int32_t z) {
    uint32_t h = (uint32_t)x * 0x9E3779B1u + (uint32_t)y * 0x85EBCA77u + (uint32_t)z * 0xC2B2AE3Du;
    h = h * 0xD2B74407u;
    h = h ^ (h >> 16);
    h = h * 0x85EBCA6Bu;
    return (((float)(h & 0xFFFFFFu)) / 16777215.0f) * 2.0f - 1.0f;
}

static inline float smooth(float t) { return t * t * (3.0f - 2.0f * t); }

static float value_noise_2d(float x, float z) {
    int32_t xi = f2i(floorf(x));
    int32_t zi = f2i(floorf(z));
    float xf = smooth(x - (float)xi);
    float zf = smooth(z - (float)zi);
    float v00 = hash2(xi, zi);
    float v10 = hash2(xi + 1, zi);
    float v01 = hash2(xi, zi + 1);
    float v11 = hash2(xi + 1, zi + 1);
    float a = v00 * (1.0f - xf) + v10 * xf;
    float b = v01 * (1.0f - xf) + v11 * xf;
    return a * (1.0f - zf) + b * zf;
}

float or_fbm_2d(float x, float z, uint32_t octaves) {
    float total = 0.0f, amp = 1.0f, freq = 1.0f, max_amp = 0.0f;
    for (uint32_t i = 0; i < octaves; ++i) {
        total += value_noise_2d(x * freq, z * freq) * amp;
        max_amp += amp;
        amp *= 0.5f;
        freq *= 2.0f;
    }
    return total / max_amp;
}

float or_value_noise_3d(float x, float y, float z) {
    int32_t xi = f2i(floorf(x)), yi = f2i(floorf(y)), zi = f2i(floorf(z));
    float xf = smooth(x - (float)xi);
    float yf = smooth(y - (float)yi);
    float zf = smooth(z - (float)zi);
    float v000 = hash3(xi, yi, zi);
    float v100 = hash3(xi + 1, yi, zi);
    float v010 = hash3(xi, yi + 1, zi);
    float v110 = hash3(xi + 1, yi + 1, zi);
    float v001 = hash3(xi, yi, zi + 1);
    float v101 = hash3(xi + 1, yi, zi + 1);
    float v011 = hash3(xi, yi + 1, zi + 1);
    float v111 = hash3(xi + 1, yi + 1, zi + 1);
    float a = v000 * (1.0f - xf) + v100 * xf;
    float b = v010 * (1.0f - xf) + v110 * xf;
    float c = v001 * (1.0f - xf) + v101 * xf;
    float d = v011 * (1.0f - xf) + v111 * xf;
    float ab = a * (1.0f - yf) + b * yf;
    float cd = c * (1.0f - yf) + d * yf;
    return ab * (1.0f - zf) + cd * zf;
}

/* ------------------------------------------------------------------ */
/* synthetic terrain (the benchmark worlds).  Noise primitives and the   */
/* seed offset are the reference's; the column recipe is the workload's: */
/* h = floor(base + amp * fbm(x/128, z/128, 5)), grass top, dirt below,  */
/* stone beneath, water up to the level, caves where 3D noise > thr      */
/* (carved only strictly inside the column, the guard of voxel.rs:1128). */
/* ------------------------------------------------------------------ */
typedef struct {
    const OrWorld *w;
    const OrTerrain *t;
    int32_t z0, z1;
} GenJob;

static void gen_columns(const OrWorld *w, const OrTerrain *t, int32_t z0, int32_t z1) {
    Dims d = dims_of(w);
    float off[2];
    or_seed_offset_xz(t->seed, off);
    for (int32_t z = z0; z < z1; ++z) {
        for (int32_t x = 0; x < d.vx; ++x) {
            float fx = (float)x + off[0];
            float fz = (float)z + off[1];
            float n = or_fbm_2d(fx * t->inv_wavelength, fz * t->inv_wavelength, t->octaves);
            int32_t h = f2i(floorf(t->base_height + t->amplitude * n));
            if (h < 1) h = 1;
            if (h > d.vy - 1) h = d.vy - 1;
            for (int32_t y = 0; y <= h; ++y) {
                if (y > 4 && y + 3 < h) {
                    float c = or_value_noise_3d(fx * t->cave_inv_wavelength,
                                                (float)y * t->cave_inv_wavelength,
                                                fz * t->cave_inv_wavelength);
                    if (c > t->cave_threshold) continue;
                }
                uint8_t m = (y == h) ? MAT_GRASS : ((y + t->dirt_depth >= h) ? MAT_DIRT : MAT_STONE);
                OrBrick *b = &w->bricks[brick_idx(&d, x / 4, y / 4, z / 4)];
                int vi = child_bit(x & 3, y & 3, z & 3);
                b->occupancy |= 1ull << vi;
                b->materials[vi] = m;
            }
            for (int32_t y = h + 1; y <= t->water_level && y < d.vy; ++y) {
                OrBrick *b = &w->bricks[brick_idx(&d, x / 4, y / 4, z / 4)];
                int vi = child_bit(x & 3, y & 3, z & 3);
                b->occupancy |= 1ull << vi;
                b->materials[vi] = MAT_WATER;
            }
        }
    }
}

static void *gen_thread(void *arg) {
    GenJob *j = (GenJob *)arg;
    gen_columns(j->w, j->t, j->z0, j->z1);
    return NULL;
}

void or_generate_terrain(const OrWorld *w, const OrTerrain *t, int nthreads) {
    Dims d = dims_of(w);
    memset(w->bricks, 0, sizeof(OrBrick) * (size_t)d.bx * d.by * d.bz);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    /* split along z at brick boundaries so threads never share a brick */
    int32_t nb = d.bz;
    pthread_t th[256];
    GenJob jobs[256];
    int used = 0;
    for (int i = 0; i < nthreads; ++i) {
        int32_t b0 = (int32_t)((int64_t)nb * i / nthreads);
        int32_t b1 = (int32_t)((int64_t)nb * (i + 1) / nthreads);
        if (b1 <= b0) continue;
        jobs[used].w = w; jobs[used].t = t; jobs[used].z0 = b0 * 4; jobs[used].z1 = b1 * 4;
        used++;
    }
    for (int i = 1; i < used; ++i) pthread_create(&th[i], NULL, gen_thread, &jobs[i]);
    if (used > 0) gen_thread(&jobs[0]);
    for (int i = 1; i < used; ++i) pthread_join(th[i], NULL);
}

/* ------------------------------------------------------------------ */
/* gen_slot_bricks: the reference's own chunk generator                */
/* (voxel.rs:1244-1500 terrain/biomes/ores/decoration, :1500-1811      */
/* trees, :1822-1997 biome tables).  Rivers and ravines are disabled   */
/* in the reference (voxel.rs:1267-1306) and are absent here too.      */
/* powf / cosf / sinf are the C library's, the functions the           */
/* reference's f32::powf / cos / sin call on Linux.                    */
/* ------------------------------------------------------------------ */
enum { SG_SEA = 64, SG_WORLD_Y = 256, SG_CV = 32 };
enum { SG_SAND = 1, SG_WOOD = 13, SG_LEAVES = 14, SG_SNOW = 15, SG_COAL = 19, SG_IRON = 20,
       SG_GOLD = 21, SG_DIAMOND = 22, SG_WOOD_BIRCH = 23, SG_WOOD_PINE = 24,
       SG_LEAVES_BIRCH = 25, SG_LEAVES_PINE = 26, SG_LEAVES_AUTUMN = 27, SG_FLOWER = 30,
       SG_TALL_GRASS = 31, SG_CACTUS = 32, SG_GRASS_DRY = 34, SG_BUSH = 36 };
/* Biome (voxel.rs:1810-1820) */
enum { B_TUNDRA, B_PLAINS, B_FOREST, B_JUNGLE, B_SAVANNA, B_DESERT, B_BEACH, B_MOUNTAIN };

static inline float fmaxr(float a, float b) { return a < b ? b : a; }  /* f32::max, no NaN here */
static inline float fminr(float a, float b) { return b < a ? b : a; }

/* sample_terrain, voxel.rs:1244-1316 (ravine_cut 0, rivers off) */
int32_t or_sample_terrain(float wx, float wz, uint64_t seed, int32_t *water_top) {
    float off[2];
    or_seed_offset_xz(seed, off);
    float px = wx + off[0], pz = wz + off[1];
    float warp_x = or_fbm_2d(px * 0.005f, pz * 0.005f, 2) * 8.0f;
    float warp_z = or_fbm_2d(px * 0.005f + 50.0f, pz * 0.005f + 50.0f, 2) * 8.0f;
    float wpx = px + warp_x, wpz = pz + warp_z;
    float base = or_fbm_2d(wpx * 0.012f, wpz * 0.012f, 4) * 22.0f;
    float mountain_mask = fmaxr(or_fbm_2d(wpx * 0.0028f, wpz * 0.0028f, 2) + 0.2f, 0.0f);
    float mountain_amp = fminr(mountain_mask, 1.0f);
    float mountain_h =
        powf(fmaxr(or_fbm_2d(wpx * 0.009f, wpz * 0.009f, 5), 0.0f), 1.15f) * mountain_amp * 110.0f;
    float base_h = 64.0f + 8.0f + base + mountain_h - 0.0f;
    float h = base_h < 2.0f ? 2.0f : (base_h > 255.0f ? 255.0f : base_h);
    int32_t h_i = f2i(h);
    if (water_top) *water_top = h_i < SG_SEA ? SG_SEA : 0;
    return h_i;
}

/* pick_biome, voxel.rs:1822-1832 */
static int pick_biome(float temp, float humid, uint32_t h, uint32_t sea) {
    if (h > sea + 36) return B_MOUNTAIN;
    if (h <= sea + 1) return B_BEACH;
    if (temp < -0.20f) return B_TUNDRA;
    if (temp > 0.25f && humid < -0.05f) return B_DESERT;
    if (temp > 0.15f && humid > 0.25f) return B_JUNGLE;
    if (temp > 0.10f && humid < 0.10f) return B_SAVANNA;
    if (humid > 0.20f) return B_FOREST;
    return B_PLAINS;
}
/* Biome::top_block / subsoil / tree_type / flora_probs / tree_density,
 * voxel.rs:1834-1903 */
static uint8_t top_block(int b, uint32_t h) {
    switch (b) {
    case B_TUNDRA: return SG_SNOW;
    case B_DESERT: case B_BEACH: case B_SAVANNA: return SG_SAND;
    case B_MOUNTAIN: return h > SG_SEA + 55 ? SG_SNOW : MAT_STONE;
    default: return MAT_GRASS;
    }
}
static uint8_t subsoil(int b) {
    switch (b) {
    case B_DESERT: case B_BEACH: return SG_SAND;
    case B_MOUNTAIN: return MAT_STONE;
    default: return MAT_DIRT;
    }
}
static uint32_t tree_type(int b, uint32_t hash) {
    switch (b) {
    case B_TUNDRA: case B_MOUNTAIN: return 2;
    case B_PLAINS: return hash % 3 == 0 ? 1 : 0;
    case B_FOREST: { uint32_t k = hash % 4; return k == 0 ? 1 : (k == 1 ? 3 : 0); }
    case B_JUNGLE: return hash % 4 == 0 ? 3 : 0;
    default: return 0;
    }
}
static void flora_probs(int b, float *fp, float *gp) {
    switch (b) {
    case B_PLAINS: *fp = 0.020f; *gp = 0.08f; break;
    case B_FOREST: *fp = 0.010f; *gp = 0.065f; break;
    case B_JUNGLE: *fp = 0.012f; *gp = 0.09f; break;
    default: *fp = 0.015f; *gp = 0.065f; break;
    }
}
static float tree_density(int b) {
    switch (b) {
    case B_JUNGLE: return 1.2f;
    case B_FOREST: return 0.55f;
    case B_TUNDRA: return 0.30f;
    case B_PLAINS: return 0.20f;
    case B_MOUNTAIN: return 0.14f;
    case B_DESERT: return 0.20f;
    default: return 0.0f;
    }
}

/* stone_or_ore, voxel.rs:1906-1916 */
static uint8_t stone_or_ore(float x, float y, float z, uint32_t h) {
    float depth = fmaxr((float)h - y, 0.0f);
    float n1 = or_value_noise_3d(x * 0.27f, y * 0.27f, z * 0.27f);
    float n2 = or_value_noise_3d(x * 0.55f, y * 0.55f, z * 0.55f);
    float combined = n1 + n2 * 0.30f;
    if (depth > 30.0f && combined > 0.50f) return SG_DIAMOND;
    if (depth > 20.0f && combined > 0.36f) return SG_GOLD;
    if (depth > 10.0f && combined > 0.24f) return SG_IRON;
    if (combined > 0.32f) return SG_COAL;
    return MAT_STONE;
}

/* Brick::set (voxel.rs:315-325) on the chunk scratch, x + y*8 + z*64 */
static void sg_set(OrBrick *s, uint32_t dx, uint32_t dy, uint32_t dz, uint8_t mat) {
    OrBrick *b = &s[(dx / 4) + (dy / 4) * 8 + (dz / 4) * 64];
    int vi = child_bit((int32_t)(dx % 4), (int32_t)(dy % 4), (int32_t)(dz % 4));
    if (mat == 0) {
        b->occupancy &= ~(1ull << vi);
        b->materials[vi] = 0;
    } else {
        b->occupancy |= 1ull << vi;
        b->materials[vi] = mat;
    }
}

/* trees_for_chunk, voxel.rs:1537-1591 */
int or_trees_for_chunk(int32_t cx, int32_t cz, uint64_t seed, OrTree out[12]) {
    float off[2];
    or_seed_offset_xz(seed, off);
    float ccx = ((float)cx + 0.5f) * 32.0f;
    float ccz = ((float)cz + 0.5f) * 32.0f;
    float temperature = or_fbm_2d((ccx + off[0]) * 0.0006f, (ccz + off[1]) * 0.0006f, 3);
    float humidity =
        or_fbm_2d((ccx + off[0]) * 0.0008f + 100.0f, (ccz + off[1]) * 0.0008f + 100.0f, 3);
    int biome = pick_biome(temperature, humidity, SG_SEA + 10, SG_SEA);
    uint32_t n_cand = (uint32_t)f2i(roundf(tree_density(biome) * 5.0f));
    if (n_cand == 0) return 0;
    float patch_mul = 1.0f;
    if (biome != B_DESERT) {
        float patch_raw = or_fbm_2d(ccx * 0.0035f, ccz * 0.0035f, 2);
        patch_mul = fminr(fmaxr(patch_raw + 0.4f, 0.0f) * 1.6f, 2.0f);
    }
    uint32_t n = (uint32_t)f2i((float)n_cand * patch_mul);
    /* hash_chunk, voxel.rs:1593-1601 */
    uint32_t s = (uint32_t)seed ^ (uint32_t)(seed >> 32);
    uint32_t ch = (uint32_t)cx * 0x9E3779B1u;
    ch = ch + (uint32_t)cz * 0x85EBCA77u;
    ch = ch + s * 0xC2B2AE3Du;
    ch = ch ^ (ch >> 16);
    ch = ch * 0xD2B74407u;
    ch = ch ^ (ch >> 13);
    int k = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t h = ch * 2654435761u + i * 7919u;
        int32_t wx = cx * 32 + (int32_t)(h & 31u);
        int32_t wz = cz * 32 + (int32_t)((h >> 5) & 31u);
        int32_t th = or_sample_terrain((float)wx, (float)wz, seed, NULL);
        if ((uint32_t)th <= SG_SEA + 1) continue;
        if (th + 22 >= SG_WORLD_Y) continue;
        float lt = or_fbm_2d(((float)wx + off[0]) * 0.0006f, ((float)wz + off[1]) * 0.0006f, 3);
        float lh = or_fbm_2d(((float)wx + off[0]) * 0.0008f + 100.0f,
                             ((float)wz + off[1]) * 0.0008f + 100.0f, 3);
        int lb = pick_biome(lt, lh, (uint32_t)th, SG_SEA);
        uint32_t tt;
        if (lb == B_BEACH || lb == B_SAVANNA) continue;
        tt = lb == B_DESERT ? 4u : tree_type(lb, h);
        out[k].base[0] = wx; out[k].base[1] = th + 1; out[k].base[2] = wz;
        out[k].ttype = tt; out[k].hash = h;
        ++k;
    }
    return k;
}

typedef struct {
    OrBrick *s;
    int32_t mn[3], mx[3];
} SgChunk;

/* try_write_tree_voxel, voxel.rs:1500-1525 */
static void sg_tree_voxel(const SgChunk *c, int32_t x, int32_t y, int32_t z, uint8_t mat) {
    if (x < c->mn[0] || x >= c->mx[0]) return;
    if (y < c->mn[1] || y >= c->mx[1]) return;
    if (z < c->mn[2] || z >= c->mx[2]) return;
    uint32_t dx = (uint32_t)(x - c->mn[0]), dy = (uint32_t)(y - c->mn[1]), dz = (uint32_t)(z - c->mn[2]);
    const OrBrick *b = &c->s[(dx / 4) + (dy / 4) * 8 + (dz / 4) * 64];
    int vi = child_bit((int32_t)(dx % 4), (int32_t)(dy % 4), (int32_t)(dz % 4));
    int occupied = (b->occupancy >> vi) & 1u;
    int fringe = occupied && b->materials[vi] == MAT_LEAF_FRINGE;
    if (!occupied || (fringe && mat != MAT_LEAF_FRINGE)) sg_set(c->s, dx, dy, dz, mat);
}

/* paint_line with thickness 0, voxel.rs:1744-1776 */
static void sg_line(const SgChunk *c, const int32_t a[3], const int32_t b[3], uint8_t mat) {
    int32_t d0 = b[0] - a[0], d1 = b[1] - a[1], d2 = b[2] - a[2];
    float len = sqrtf((float)(d0 * d0 + d1 * d1 + d2 * d2));
    int32_t steps = f2i(ceilf(len * 1.5f));
    if (steps <= 0) {
        sg_tree_voxel(c, a[0], a[1], a[2], mat);
        return;
    }
    for (int32_t s = 0; s <= steps; ++s) {
        float t = (float)s / (float)steps;
        int32_t x = f2i(roundf((float)a[0] + (float)d0 * t));
        int32_t y = f2i(roundf((float)a[1] + (float)d1 * t));
        int32_t z = f2i(roundf((float)a[2] + (float)d2 * t));
        sg_tree_voxel(c, x, y, z, mat);
    }
}
/* paint_fringe_shell + paint_sphere = paint_canopy, voxel.rs:1715-1742, :1778-1789 */
static void sg_canopy(const SgChunk *c, const int32_t ctr[3], int32_t r, uint8_t mat) {
    int32_t rf = r + 1, r2 = rf * rf;
    for (int32_t dy = -rf; dy <= rf; ++dy)
        for (int32_t dx = -(rf + 1); dx <= rf + 1; ++dx)
            for (int32_t dz = -(rf + 1); dz <= rf + 1; ++dz) {
                int32_t hx = abs(dx) - 1, hz = abs(dz) - 1;
                if (hx < 0) hx = 0;
                if (hz < 0) hz = 0;
                if (hx * hx + dy * dy + hz * hz > r2) continue;
                sg_tree_voxel(c, ctr[0] + dx, ctr[1] + dy, ctr[2] + dz, MAT_LEAF_FRINGE);
            }
    r2 = r * r;
    for (int32_t dy = -r; dy <= r; ++dy)
        for (int32_t dx = -r; dx <= r; ++dx)
            for (int32_t dz = -r; dz <= r; ++dz) {
                if (dx * dx + dy * dy + dz * dz > r2) continue;
                sg_tree_voxel(c, ctr[0] + dx, ctr[1] + dy, ctr[2] + dz, mat);
            }
}
/* branch_jitter, voxel.rs:1791-1797 */
static float branch_jitter(uint32_t hash, uint32_t b, uint32_t salt) {
    uint32_t h = hash * 0x9E3779B1u + b * 2654435761u + salt * 40503u;
    return ((float)(h & 0xFFFFu) / 65535.0f) * 2.0f - 1.0f;
}

/* paint_tree, voxel.rs:1605-1710 */
static void sg_paint_tree(const SgChunk *c, const OrTree *t) {
    const float tau = 6.28318548202514648f; /* std::f32::consts::TAU */
    const int32_t *base = t->base;
    uint32_t h = t->hash;
    if (t->ttype == 2) {
        int32_t trunk_h = 10 + (int32_t)(h % 6);
        int32_t top[3] = {base[0], base[1] + trunk_h, base[2]};
        sg_line(c, base, top, SG_WOOD_PINE);
        for (int32_t i = 0; i < 6; ++i) {
            float tf = (float)i / 6.0f;
            int32_t y = base[1] + f2i((float)trunk_h * (0.35f + tf * 0.78f));
            int32_t r = f2i(powf(1.0f - tf, 0.85f) * 3.5f + 1.0f);
            int32_t ctr[3] = {base[0], y, base[2]};
            sg_canopy(c, ctr, r, SG_LEAVES_PINE);
        }
    } else if (t->ttype == 1) {
        int32_t trunk_h = 8 + (int32_t)(h % 5);
        int32_t top[3] = {base[0], base[1] + trunk_h, base[2]};
        sg_line(c, base, top, SG_WOOD_BIRCH);
        int32_t n = 2 + (int32_t)(h % 2);
        for (int32_t b = 0; b < n; ++b) {
            float angle = ((float)b / (float)n) * tau + branch_jitter(h, (uint32_t)b, 0) * 0.5f;
            int32_t len = 2 + (int32_t)((h * ((uint32_t)b + 1u)) % 3u);
            int32_t sy = base[1] + f2i((float)trunk_h * 0.7f);
            int32_t from[3] = {base[0], sy, base[2]};
            int32_t end[3] = {base[0] + f2i(cosf(angle) * (float)len), sy + 1,
                              base[2] + f2i(sinf(angle) * (float)len)};
            sg_line(c, from, end, SG_WOOD_BIRCH);
            sg_canopy(c, end, 2, SG_LEAVES_BIRCH);
        }
        sg_canopy(c, top, 3, SG_LEAVES_BIRCH);
    } else if (t->ttype == 4) {
        static const int32_t sets[4][2][2] = {{{1, 0}, {0, 1}}, {{-1, 0}, {0, -1}},
                                              {{0, 1}, {-1, 0}}, {{0, -1}, {1, 0}}};
        int32_t col_h = 3 + (int32_t)(h % 6);
        int32_t top[3] = {base[0], base[1] + col_h, base[2]};
        sg_line(c, base, top, SG_CACTUS);
        int32_t n_arms = (int32_t)(h % 3);
        const int32_t(*set)[2] = sets[h & 3u];
        for (int32_t a = 0; a < n_arms; ++a) {
            int32_t dx = set[a % 2][0], dz = set[a % 2][1];
            int32_t sy = base[1] + f2i((float)col_h * 0.4f);
            int32_t arm_top = base[1] + f2i((float)col_h * 0.9f);
            int32_t ax = base[0] + dx * 2, az = base[2] + dz * 2;
            int32_t p0[3] = {base[0], sy, base[2]}, p1[3] = {ax, sy, az}, p2[3] = {ax, arm_top, az};
            sg_line(c, p0, p1, SG_CACTUS);
            sg_line(c, p1, p2, SG_CACTUS);
        }
    } else {
        uint8_t leaf = t->ttype == 3 ? SG_LEAVES_AUTUMN : SG_LEAVES;
        int32_t trunk_h = 8 + (int32_t)(h % 5);
        int32_t top[3] = {base[0], base[1] + trunk_h, base[2]};
        sg_line(c, base, top, SG_WOOD);
        int32_t n = 3 + (int32_t)(h % 2);
        for (int32_t b = 0; b < n; ++b) {
            float angle = ((float)b / (float)n) * tau + branch_jitter(h, (uint32_t)b, 0) * 0.6f;
            int32_t len = 3 + (int32_t)((h * ((uint32_t)b + 7u)) % 3u);
            int32_t sy = base[1] + f2i((float)trunk_h * 0.65f);
            int32_t from[3] = {base[0], sy, base[2]};
            int32_t end[3] = {base[0] + f2i(cosf(angle) * (float)len), sy + f2i((float)len * 0.5f),
                              base[2] + f2i(sinf(angle) * (float)len)};
            sg_line(c, from, end, SG_WOOD);
            sg_canopy(c, end, 3, leaf);
        }
        sg_canopy(c, top, 4, leaf);
    }
}

/* gen_slot_bricks, voxel.rs:1322-1500 */
void or_gen_slot_bricks(int32_t cx, int32_t cy, int32_t cz, uint64_t seed, OrBrick *out) {
    memset(out, 0, sizeof(OrBrick) * 512);
    float off[2];
    or_seed_offset_xz(seed, off);
    const int32_t x0 = cx * SG_CV, y0 = cy * SG_CV, z0 = cz * SG_CV;
    for (int32_t dz = 0; dz < SG_CV; ++dz) {
        for (int32_t dx = 0; dx < SG_CV; ++dx) {
            const int32_t wxi = x0 + dx, wzi = z0 + dz;
            const float wx = (float)wxi, wz = (float)wzi;
            int32_t water_top;
            const int32_t h = or_sample_terrain(wx, wz, seed, &water_top);
            const uint32_t hu = (uint32_t)h;
            const int32_t col_top = h > water_top ? h : water_top;
            if (col_top < y0 || 0 >= y0 + SG_CV) continue;
            float temperature = or_fbm_2d((wx + off[0]) * 0.0006f, (wz + off[1]) * 0.0006f, 3);
            float humidity = or_fbm_2d((wx + off[0]) * 0.0008f + 100.0f,
                                       (wz + off[1]) * 0.0008f + 100.0f, 3);
            int biome = pick_biome(temperature, humidity, hu, SG_SEA);
            const int32_t ys = y0 > 0 ? y0 : 0;
            const int32_t ye = (y0 + SG_CV) < SG_WORLD_Y ? (y0 + SG_CV) : SG_WORLD_Y;
            const int32_t seal = water_top > h ? h - 5 : INT32_MIN;
            for (int32_t y = ys; y < ye; ++y) {
                if (y > h) break;
                if (!(y >= seal)) {
                    float cn = or_value_noise_3d(wx * 0.045f, (float)y * 0.085f, wz * 0.045f);
                    float cn2 = or_value_noise_3d(wx * 0.110f, (float)y * 0.060f, wz * 0.110f);
                    if (y > 4 && y + 3 < h && (cn + cn2 * 0.6f) > 0.30f) continue;
                }
                uint8_t mat;
                if ((uint32_t)y >= hu) mat = top_block(biome, hu);
                else if ((uint32_t)y + 4u >= hu) mat = subsoil(biome);
                else mat = stone_or_ore(wx, (float)y, wz, hu);
                sg_set(out, (uint32_t)dx, (uint32_t)(y - y0), (uint32_t)dz, mat);
            }
            if (water_top > h) {
                int32_t fb = h + 1 > y0 ? h + 1 : y0;
                int32_t fe = water_top < y0 + SG_CV - 1 ? water_top : y0 + SG_CV - 1;
                for (int32_t wy = fb; wy <= fe; ++wy)
                    sg_set(out, (uint32_t)dx, (uint32_t)(wy - y0), (uint32_t)dz, MAT_WATER);
            }
            if (water_top == 0 && hu < SG_WORLD_Y - 1) {
                uint8_t surface = top_block(biome, hu);
                int32_t dec_y = h + 1;
                if (dec_y >= y0 && dec_y < y0 + SG_CV) {
                    float v = hash3(wxi, dec_y, wzi) * 0.5f + 0.5f;
                    uint8_t dec = 0;
                    const int32_t ax = wxi & ~1, az = wzi & ~1;
                    if (surface == MAT_GRASS) {
                        float fp, gp;
                        flora_probs(biome, &fp, &gp);
                        if (or_fbm_2d((float)wxi * 0.02f + 7.0f, (float)wzi * 0.02f - 3.0f, 2) > 0.30f) {
                            fp *= 3.0f;
                            gp *= 12.0f;
                        }
                        if (v > 1.0f - fp) dec = SG_FLOWER;
                        else if (v > 1.0f - fp - gp) dec = SG_TALL_GRASS;
                        else if (hash3(ax, 977, az) * 0.5f + 0.5f > 0.9955f) dec = SG_BUSH;
                        else if (v > 1.0f - fp - gp - 0.004f) dec = SG_BUSH;
                    } else if (surface == SG_SAND && (biome == B_DESERT || biome == B_SAVANNA)) {
                        if (v > 0.99f) dec = SG_GRASS_DRY;
                    } else if (surface == SG_SNOW && biome == B_TUNDRA) {
                        if (v > 0.995f) dec = SG_GRASS_DRY;
                    }
                    if (dec != 0) {
                        uint32_t dy = (uint32_t)(dec_y - y0);
                        sg_set(out, (uint32_t)dx, dy, (uint32_t)dz, dec);
                        if (dec == SG_BUSH) {
                            int big = hash3(ax, 977, az) * 0.5f + 0.5f > 0.9955f;
                            if (big && dec_y + 1 >= y0 && dec_y + 1 < y0 + SG_CV)
                                sg_set(out, (uint32_t)dx, dy + 1, (uint32_t)dz, SG_BUSH);
                        }
                    }
                }
            }
        }
    }
    /* tree pass: trees based in this chunk's column or its 8 xz neighbours */
    SgChunk c;
    c.s = out;
    c.mn[0] = x0; c.mn[1] = y0; c.mn[2] = z0;
    c.mx[0] = x0 + SG_CV; c.mx[1] = y0 + SG_CV; c.mx[2] = z0 + SG_CV;
    for (int32_t ncz = -1; ncz <= 1; ++ncz)
        for (int32_t ncx = -1; ncx <= 1; ++ncx) {
            OrTree trees[12];
            int n = or_trees_for_chunk(cx + ncx, cz + ncz, seed, trees);
            for (int i = 0; i < n; ++i) {
                if (trees[i].base[1] > c.mx[1] || trees[i].base[1] + 22 < c.mn[1]) continue;
                sg_paint_tree(&c, &trees[i]);
            }
        }
}

/* fill_demo_terrain (voxel.rs:1005-1060) generalised to a window whose
 * lower corner is world chunk (ox, 0, oz): the slot (sx, sy, sz) holds the
 * world chunk shift_origin assigns it (voxel.rs:507-537), then the masks
 * and LUTs are rebuilt. */
typedef struct {
    const OrWorld *w;
    uint64_t seed;
    int32_t ox, oz;
    int64_t j0, j1;
} SlotJob;

static void *slot_thread(void *arg) {
    SlotJob *j = (SlotJob *)arg;
    Dims d = dims_of(j->w);
    const int32_t sx_n = d.bx / 8, sy_n = d.by / 8, sz_n = d.bz / 8;
    OrBrick *scratch = (OrBrick *)malloc(sizeof(OrBrick) * 512);
    if (!scratch) return NULL;
    for (int64_t k = j->j0; k < j->j1; ++k) {
        int32_t sx = (int32_t)(k % sx_n), sy = (int32_t)((k / sx_n) % sy_n),
                sz = (int32_t)(k / ((int64_t)sx_n * sy_n));
        int32_t wcx = j->ox + pos_mod(sx - j->ox, sx_n);
        int32_t wcz = j->oz + pos_mod(sz - j->oz, sz_n);
        or_gen_slot_bricks(wcx, sy, wcz, j->seed, scratch);
        for (int32_t bz = 0; bz < 8; ++bz)
            for (int32_t by = 0; by < 8; ++by)
                for (int32_t bx = 0; bx < 8; ++bx)
                    j->w->bricks[brick_idx(&d, sx * 8 + bx, sy * 8 + by, sz * 8 + bz)] =
                        scratch[bx + by * 8 + bz * 64];
    }
    free(scratch);
    return NULL;
}

void or_fill_window(const OrWorld *w, uint64_t seed, int32_t ox, int32_t oz, int nthreads) {
    Dims d = dims_of(w);
    const int64_t n = (int64_t)(d.bx / 8) * (d.by / 8) * (d.bz / 8);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    SlotJob jobs[256];
    int used = 0;
    for (int i = 0; i < nthreads; ++i) {
        int64_t a = n * i / nthreads, b = n * (i + 1) / nthreads;
        if (b <= a) continue;
        jobs[used].w = w; jobs[used].seed = seed; jobs[used].ox = ox; jobs[used].oz = oz;
        jobs[used].j0 = a; jobs[used].j1 = b;
        used++;
    }
    for (int i = 1; i < used; ++i) pthread_create(&th[i], NULL, slot_thread, &jobs[i]);
    if (used > 0) slot_thread(&jobs[0]);
    for (int i = 1; i < used; ++i) pthread_join(th[i], NULL);
    or_rebuild_all_masks(w);
    or_rebuild_all_uniform(w);
}

/* ------------------------------------------------------------------ */
/* ray generation                                                      */
/* ------------------------------------------------------------------ */
static inline void normalize3(const float v[3], float out[3]) {
    float len = sqrtf((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
    out[0] = v[0] / len;
    out[1] = v[1] / len;
    out[2] = v[2] / len;
}

/* ray_dir_uv, raymarch.wgsl:430-438 (beam.wgsl:38-45 is the same formula) */
void or_ray_dir_uv(const OrCamera *c, float u, float v, float out[3]) {
    float ndc_x = u * 2.0f - 1.0f;
    float ndc_y = 1.0f - v * 2.0f;
    float aspect = c->res_x / c->res_y;
    float a = ndc_x * c->tan_half_fov * aspect;
    float b = ndc_y * c->tan_half_fov;
    float r[3];
    for (int k = 0; k < 3; ++k) r[k] = (c->forward[k] + c->right[k] * a) + c->up[k] * b;
    normalize3(r, out);
}

/* ign, raymarch.wgsl:394-396 */
float or_ign(float x, float y, float frame) {
    float a = x + frame * 5.588238f;
    float b = y + frame * 4.182857f;
    return fractf(52.9829189f * fractf(0.06711056f * a + 0.00583715f * b));
}

/* sin/cos by the Maclaurin series, nested in x^2 (terms through x^17 /
 * x^18; truncation < 2e-10 on [0, 2.4]).  Written out so the CPU and the
 * GPU evaluate the identical operation sequence. */
void or_sincos(float x, float *s, float *c) {
    float x2 = x * x;
    float ps = 1.0f - x2 * 0.0036764706f;      /* 1/272 */
    ps = 1.0f - x2 * 0.0047619049f * ps;       /* 1/210 */
    ps = 1.0f - x2 * 0.0064102565f * ps;       /* 1/156 */
    ps = 1.0f - x2 * 0.0090909088f * ps;       /* 1/110 */
    ps = 1.0f - x2 * 0.013888889f * ps;        /* 1/72  */
    ps = 1.0f - x2 * 0.023809524f * ps;        /* 1/42  */
    ps = 1.0f - x2 * 0.050000001f * ps;        /* 1/20  */
    ps = 1.0f - x2 * 0.16666667f * ps;         /* 1/6   */
    *s = x * ps;
    float pc = 1.0f - x2 * 0.0032679739f;      /* 1/306 */
    pc = 1.0f - x2 * 0.0041666669f * pc;       /* 1/240 */
    pc = 1.0f - x2 * 0.0054945056f * pc;       /* 1/182 */
    pc = 1.0f - x2 * 0.0075757578f * pc;       /* 1/132 */
    pc = 1.0f - x2 * 0.011111111f * pc;        /* 1/90  */
    pc = 1.0f - x2 * 0.017857144f * pc;        /* 1/56  */
    pc = 1.0f - x2 * 0.033333335f * pc;        /* 1/30  */
    pc = 1.0f - x2 * 0.083333336f * pc;        /* 1/12  */
    pc = 1.0f - x2 * 0.5f * pc;                /* 1/2   */
    *c = pc;
}

/* ------------------------------------------------------------------ */
/* O2 hierarchical DDA                                                 */
/* ------------------------------------------------------------------ */
typedef struct {
    float org[3], inv[3], tdel[3], tmin3[3], tmax[3];
    float t_enter;
    int32_t step[3], voxel[3], slot[3];
} Dda;

/* dda_init, raymarch.wgsl:3369-3411 */
static int dda_init(const Dims *d, const int32_t ro[3], const float origin[3],
                    const float dir[3], Dda *s) {
    float dims[3] = {(float)d->vx, (float)d->vy, (float)d->vz};
    float tmax3[3];
    for (int k = 0; k < 3; ++k) {
        s->org[k] = origin[k] - (float)ro[k];
        s->inv[k] = safe_inv(dir[k]);
        float t0 = (0.0f - s->org[k]) * s->inv[k];
        float t1 = (dims[k] - s->org[k]) * s->inv[k];
        s->tmin3[k] = vmin(t0, t1);
        tmax3[k] = vmax(t0, t1);
    }
    s->t_enter = vmax(vmax(s->tmin3[0], s->tmin3[1]), vmax(s->tmin3[2], 0.0f));
    float t_exit = vmin(vmin(tmax3[0], tmax3[1]), tmax3[2]);
    if (s->t_enter >= t_exit || t_exit < 0.0f) return 0;
    for (int k = 0; k < 3; ++k) {
        float p = s->org[k] + dir[k] * (s->t_enter + 1e-3f);
        p = clampf(p, 0.01f, dims[k] - 0.01f);
        s->step[k] = sgn(dir[k]);
        s->tdel[k] = fabsf(s->inv[k]);
        int32_t vl0 = f2i(floorf(p));
        s->voxel[k] = vl0 + ro[k];
        if (s->step[k] > 0) s->tmax[k] = ((float)(vl0 + 1) - s->org[k]) * s->inv[k];
        else s->tmax[k] = ((float)vl0 - s->org[k]) * s->inv[k];
    }
    s->slot[0] = pos_mod(s->voxel[0], d->vx);
    s->slot[1] = s->voxel[1];
    s->slot[2] = pos_mod(s->voxel[2], d->vz);
    return 1;
}

/* dda_step, raymarch.wgsl:3416-3448 */
static inline void dda_step(const Dims *d, Dda *s, float *t_cur, int32_t *last_axis) {
    int ax;
    if (s->tmax[0] < s->tmax[1] && s->tmax[0] < s->tmax[2]) ax = 0;
    else if (s->tmax[1] < s->tmax[2]) ax = 1;
    else ax = 2;
    *t_cur = s->tmax[ax];
    s->voxel[ax] += s->step[ax];
    s->slot[ax] += s->step[ax];
    if (ax == 0) {
        if (s->slot[0] >= d->vx) s->slot[0] -= d->vx;
        else if (s->slot[0] < 0) s->slot[0] += d->vx;
    } else if (ax == 2) {
        if (s->slot[2] >= d->vz) s->slot[2] -= d->vz;
        else if (s->slot[2] < 0) s->slot[2] += d->vz;
    }
    s->tmax[ax] = s->tmax[ax] + s->tdel[ax];
    *last_axis = ax;
}

/* skip_to_cell, raymarch.wgsl:4807-4864 */
static void skip_to_cell(const Dims *d, int32_t cell, Dda *s, const int32_t ro[3],
                         const float dir[3], int32_t *last_axis) {
    int32_t co[3];
    float tf[3];
    for (int k = 0; k < 3; ++k) {
        co[k] = s->voxel[k] - pos_mod(s->voxel[k], cell);
        int32_t b = (s->step[k] > 0 ? co[k] + cell : co[k]) - ro[k];
        tf[k] = ((float)b - s->org[k]) * s->inv[k];
    }
    const float eps = 1e-6f;
    float t_min = 1e30f;
    int ax = 0;
    if (s->step[0] != 0 && tf[0] > eps && tf[0] < t_min) { t_min = tf[0]; ax = 0; }
    if (s->step[1] != 0 && tf[1] > eps && tf[1] < t_min) { t_min = tf[1]; ax = 1; }
    if (s->step[2] != 0 && tf[2] > eps && tf[2] < t_min) { t_min = tf[2]; ax = 2; }
    int32_t nv[3];
    for (int k = 0; k < 3; ++k) {
        float p = s->org[k] + dir[k] * (t_min + 1e-3f);
        nv[k] = f2i(floorf(p)) + ro[k];
    }
    nv[ax] = s->step[ax] > 0 ? co[ax] + cell : co[ax] - 1;
    for (int k = 0; k < 3; ++k) {
        s->voxel[k] = nv[k];
        int32_t vl = nv[k] - ro[k];
        if (s->step[k] > 0) s->tmax[k] = ((float)(vl + 1) - s->org[k]) * s->inv[k];
        else s->tmax[k] = ((float)vl - s->org[k]) * s->inv[k];
    }
    *last_axis = ax;
    s->slot[0] = pos_mod(nv[0], d->vx);
    s->slot[1] = nv[1];
    s->slot[2] = pos_mod(nv[2], d->vz);
}

/* last_axis_after_entry, raymarch.wgsl:4800-4805 */
static inline int entry_axis(int32_t la, const float tmin3[3]) {
    if (la >= 0) return la;
    if (tmin3[0] >= tmin3[1] && tmin3[0] >= tmin3[2]) return 0;
    if (tmin3[1] >= tmin3[2]) return 1;
    return 2;
}

/* entry_normal_and_t (raymarch.wgsl:3321-3342) -> record fields */
static void fill_hit(const Dda *s, int32_t last_axis, uint32_t m, int early, OrRecord *out) {
    int ax = entry_axis(last_axis, s->tmin3);
    float t;
    if (last_axis >= 0) t = s->tmax[last_axis] - s->tdel[last_axis];
    else t = s->t_enter;
    out->voxel[0] = s->voxel[0];
    out->voxel[1] = s->voxel[1];
    out->voxel[2] = s->voxel[2];
    out->face = (uint8_t)(2 * ax + (s->step[ax] > 0 ? 1 : 0));
    out->mat = (uint8_t)m;
    out->flags = (uint8_t)(1u | (early ? 2u : 0u));
    out->t = t;
}

static void miss_record(OrRecord *out) {
    memset(out, 0, sizeof(*out));
    out->face = 0xFF;
}

/* brick_topmost_material, raymarch.wgsl:253-295 */
static uint32_t brick_topmost_material(const OrBrick *b, uint64_t *bytes) {
    uint32_t occ_lo = (uint32_t)b->occupancy, occ_hi = (uint32_t)(b->occupancy >> 32);
    uint32_t layers[4] = {(occ_hi >> 16) & 0xFFFFu, occ_hi & 0xFFFFu, (occ_lo >> 16) & 0xFFFFu,
                          occ_lo & 0xFFFFu};
    int base[4] = {48, 32, 16, 0};
    for (int i = 0; i < 4; ++i) {
        if (layers[i] != 0u) {
            int bit = __builtin_ctz(layers[i]);
            uint32_t m = b->materials[base[i] + bit];
            *bytes += 1;
            if (m != MAT_TURF) return m;
        }
    }
    return (occ_lo | occ_hi) != 0u ? (uint32_t)MAT_TURF : 0u;
}

/* tile_representative_material, raymarch.wgsl:4782-4798 */
static uint32_t tile_representative_material(const OrWorld *w, const Dims *d, int64_t ti,
                                             const int32_t tp[3], uint64_t *bytes) {
    uint64_t tm = w->tile_mask[ti];
    *bytes += 8;
    int lin = -1;
    uint32_t lo = (uint32_t)tm, hi = (uint32_t)(tm >> 32);
    if (lo != 0u) lin = __builtin_ctz(lo);
    else if (hi != 0u) lin = 32 + __builtin_ctz(hi);
    if (lin < 0) return 0u;
    int lx = lin & 3, lz = (lin >> 2) & 3, ly = (lin >> 4) & 3;
    int64_t bi = brick_idx(d, tp[0] * 4 + lx, tp[1] * 4 + ly, tp[2] * 4 + lz);
    *bytes += 8;
    return brick_topmost_material(&w->bricks[bi], bytes);
}

static inline int in_window(const Dims *d, const int32_t v[3], const int32_t ro[3]) {
    int32_t rx = v[0] - ro[0], ry = v[1] - ro[1], rz = v[2] - ro[2];
    return !(rx < 0 || rx >= d->vx || ry < 0 || ry >= d->vy || rz < 0 || rz >= d->vz);
}

#define SKIP(cell)                                                          \
    do {                                                                    \
        skip_to_cell(&d, (cell), &s, ro, dir, &last_axis);                  \
        t_cur = s.tmax[last_axis] - s.tdel[last_axis];                      \
    } while (0)

/* trace, raymarch.wgsl:4600-4777 (cube resolution, see file header) */
void or_trace(const OrWorld *w, const int32_t ro[3], const float origin[3],
              const float dir[3], float max_dist, const OrParams *p, OrRecord *out,
              OrStats *st) {
    Dims d = dims_of(w);
    uint64_t bytes = 0, iters = 0;
    miss_record(out);
    Dda s;
    if (!dda_init(&d, ro, origin, dir, &s)) goto done;
    int32_t last_axis = -1;
    float t_cur = s.t_enter;
    const uint32_t fl = p->flags;
    int32_t it;
    for (it = 0; it < p->max_iters; ++it) {
        iters++;
        if (t_cur > max_dist) break;
        if (!in_window(&d, s.voxel, ro)) break;
        int32_t bp[3] = {s.slot[0] >> 2, s.slot[1] >> 2, s.slot[2] >> 2};
        int32_t tp[3] = {s.slot[0] >> 4, s.slot[1] >> 4, s.slot[2] >> 4};
        int32_t cp[3] = {s.slot[0] >> 6, s.slot[1] >> 6, s.slot[2] >> 6};
        if (fl & OR_F_L4) {
            int64_t li = l4_idx(&d, s.slot[0] >> 8, s.slot[1] >> 8, s.slot[2] >> 8);
            uint64_t lw = w->l4_mask[li];
            bytes += 8;
            if (lw == 0) { SKIP(256); continue; }
            if (!((lw >> child_bit(cp[0] & 3, cp[1] & 3, cp[2] & 3)) & 1ull)) { SKIP(64); continue; }
        }
        int64_t ci = chunk_idx(&d, cp[0], cp[1], cp[2]);
        uint64_t cw = w->chunk_mask[ci];
        bytes += 8;
        if (!((cw >> child_bit(tp[0] & 3, tp[1] & 3, tp[2] & 3)) & 1ull)) { SKIP(16); continue; }
        int64_t ti = tile_idx(&d, tp[0], tp[1], tp[2]);
        if ((fl & OR_F_LOD) && t_cur > p->tile_lod_t) {
            uint32_t lm = tile_representative_material(w, &d, ti, tp, &bytes);
            if (lm != 0u && is_uniform_optimisable(lm)) {
                fill_hit(&s, last_axis, lm, 1, out);
                goto hit;
            }
        }
        if (fl & OR_F_LUT) {
            uint32_t tum = w->tile_uniform[ti];
            bytes += 1;
            if (tum != 0u && is_uniform_optimisable(tum)) {
                fill_hit(&s, last_axis, tum, 1, out);
                goto hit;
            }
        }
        uint64_t tw = w->tile_mask[ti];
        bytes += 8;
        if (!((tw >> child_bit(bp[0] & 3, bp[1] & 3, bp[2] & 3)) & 1ull)) { SKIP(4); continue; }
        int64_t bi = brick_idx(&d, bp[0], bp[1], bp[2]);
        if (fl & OR_F_LUT) {
            uint32_t bum = w->brick_uniform[bi];
            bytes += 1;
            if (bum != 0u && is_uniform_optimisable(bum)) {
                fill_hit(&s, last_axis, bum, 1, out);
                goto hit;
            }
        }
        const OrBrick *b = &w->bricks[bi];
        if ((fl & OR_F_LOD) && t_cur > p->lod_brick_t) {
            bytes += 8;
            if (b->occupancy == 0) { SKIP(4); continue; }
            uint32_t m = brick_topmost_material(b, &bytes);
            if (!is_foliage(m)) {
                fill_hit(&s, last_axis, m, 1, out);
                goto hit;
            }
        }
        int vi = child_bit(s.slot[0] - bp[0] * 4, s.slot[1] - bp[1] * 4, s.slot[2] - bp[2] * 4);
        bytes += 8;
        if ((b->occupancy >> vi) & 1ull) {
            uint32_t m = b->materials[vi];
            bytes += 1;
            if (resolves_cube(m)) {
                fill_hit(&s, last_axis, m, 0, out);
                goto hit;
            }
        }
        dda_step(&d, &s, &t_cur, &last_axis);
    }
hit:
done:
    out->steps = (uint32_t)iters; /* iterations begun, including the last */
    if (st) { st->bytes += bytes; st->iters += iters; }
}

/* trace_any, raymarch.wgsl:4345-4409 (far-distance occluder rule) */
int or_trace_any(const OrWorld *w, const int32_t ro[3], const float origin[3],
                 const float dir[3], float max_dist, const OrParams *p,
                 uint32_t *steps_out, OrStats *st) {
    Dims d = dims_of(w);
    uint64_t bytes = 0, iters = 0;
    int occluded = 0;
    uint32_t steps = 0;
    Dda s;
    if (!dda_init(&d, ro, origin, dir, &s)) goto done;
    int32_t last_axis = -1;
    float t_cur = s.t_enter;
    int32_t it;
    for (it = 0; it < p->any_max_iters; ++it) {
        iters++;
        if (t_cur > max_dist) break;
        if (!in_window(&d, s.voxel, ro)) break;
        int32_t bp[3] = {s.slot[0] >> 2, s.slot[1] >> 2, s.slot[2] >> 2};
        int32_t tp[3] = {s.slot[0] >> 4, s.slot[1] >> 4, s.slot[2] >> 4};
        int32_t cp[3] = {s.slot[0] >> 6, s.slot[1] >> 6, s.slot[2] >> 6};
        int64_t li = l4_idx(&d, s.slot[0] >> 8, s.slot[1] >> 8, s.slot[2] >> 8);
        uint64_t lw = w->l4_mask[li];
        bytes += 8;
        if (lw == 0) { SKIP(256); continue; }
        if (!((lw >> child_bit(cp[0] & 3, cp[1] & 3, cp[2] & 3)) & 1ull)) { SKIP(64); continue; }
        uint64_t cw = w->chunk_mask[chunk_idx(&d, cp[0], cp[1], cp[2])];
        bytes += 8;
        if (!((cw >> child_bit(tp[0] & 3, tp[1] & 3, tp[2] & 3)) & 1ull)) { SKIP(16); continue; }
        uint64_t tw = w->tile_mask[tile_idx(&d, tp[0], tp[1], tp[2])];
        bytes += 8;
        if (!((tw >> child_bit(bp[0] & 3, bp[1] & 3, bp[2] & 3)) & 1ull)) { SKIP(4); continue; }
        const OrBrick *b = &w->bricks[brick_idx(&d, bp[0], bp[1], bp[2])];
        int vi = child_bit(s.slot[0] - bp[0] * 4, s.slot[1] - bp[1] * 4, s.slot[2] - bp[2] * 4);
        bytes += 8;
        if ((b->occupancy >> vi) & 1ull) {
            uint32_t m = b->materials[vi];
            bytes += 1;
            if (shadow_occludes(m)) { occluded = 1; break; }
        }
        dda_step(&d, &s, &t_cur, &last_axis);
    }
    steps = (uint32_t)iters;
done:
    if (steps_out) *steps_out = steps;
    if (st) { st->bytes += bytes; st->iters += iters; }
    return occluded;
}

/* trace_no_water, raymarch.wgsl:3450-3532 */
void or_trace_no_water(const OrWorld *w, const int32_t ro[3], const float origin[3],
                       const float dir[3], float t_cap, const OrParams *p, OrRecord *out,
                       OrStats *st) {
    Dims d = dims_of(w);
    uint64_t bytes = 0, iters = 0;
    miss_record(out);
    Dda s;
    if (!dda_init(&d, ro, origin, dir, &s)) goto done;
    int32_t last_axis = -1;
    float t_cur = s.t_enter;
    int32_t it;
    for (it = 0; it < p->max_iters; ++it) {
        iters++;
        if (t_cur > t_cap) break;
        if (!in_window(&d, s.voxel, ro)) break;
        int32_t bp[3] = {s.slot[0] >> 2, s.slot[1] >> 2, s.slot[2] >> 2};
        int32_t tp[3] = {s.slot[0] >> 4, s.slot[1] >> 4, s.slot[2] >> 4};
        int32_t cp[3] = {s.slot[0] >> 6, s.slot[1] >> 6, s.slot[2] >> 6};
        int64_t li = l4_idx(&d, s.slot[0] >> 8, s.slot[1] >> 8, s.slot[2] >> 8);
        uint64_t lw = w->l4_mask[li];
        bytes += 8;
        if (lw == 0) { skip_to_cell(&d, 256, &s, ro, dir, &last_axis); continue; }
        if (!((lw >> child_bit(cp[0] & 3, cp[1] & 3, cp[2] & 3)) & 1ull)) {
            skip_to_cell(&d, 64, &s, ro, dir, &last_axis);
            continue;
        }
        uint64_t cw = w->chunk_mask[chunk_idx(&d, cp[0], cp[1], cp[2])];
        bytes += 8;
        if (!((cw >> child_bit(tp[0] & 3, tp[1] & 3, tp[2] & 3)) & 1ull)) {
            skip_to_cell(&d, 16, &s, ro, dir, &last_axis);
            continue;
        }
        uint64_t tw = w->tile_mask[tile_idx(&d, tp[0], tp[1], tp[2])];
        bytes += 8;
        if (!((tw >> child_bit(bp[0] & 3, bp[1] & 3, bp[2] & 3)) & 1ull)) {
            skip_to_cell(&d, 4, &s, ro, dir, &last_axis);
            continue;
        }
        const OrBrick *b = &w->bricks[brick_idx(&d, bp[0], bp[1], bp[2])];
        int vi = child_bit(s.slot[0] - bp[0] * 4, s.slot[1] - bp[1] * 4, s.slot[2] - bp[2] * 4);
        bytes += 8;
        if ((b->occupancy >> vi) & 1ull) {
            uint32_t m = b->materials[vi];
            bytes += 1;
            if (!is_transparent(m)) {
                fill_hit(&s, last_axis, m, 0, out);
                goto done;
            }
        }
        dda_step(&d, &s, &t_cur, &last_axis);
    }
done:
    out->steps = (uint32_t)iters;
    if (st) { st->bytes += bytes; st->iters += iters; }
}
#undef SKIP

/* trace_first_tile, beam.wgsl:51-113 (world, non-rebased coordinates) */
float or_beam_first_tile(const OrWorld *w, const OrCamera *c, const float dir[3], OrStats *st) {
    Dims d = dims_of(w);
    uint64_t bytes = 0, iters = 0;
    float result = 1e9f;
    float win_min[3], win_max[3], inv[3], tmin3[3], tmax3[3];
    float dims[3] = {(float)d.vx, (float)d.vy, (float)d.vz};
    for (int k = 0; k < 3; ++k) {
        win_min[k] = (float)c->world_origin[k];
        win_max[k] = win_min[k] + dims[k];
        inv[k] = safe_inv(dir[k]);
        float t0 = (win_min[k] - c->origin[k]) * inv[k];
        float t1 = (win_max[k] - c->origin[k]) * inv[k];
        tmin3[k] = vmin(t0, t1);
        tmax3[k] = vmax(t0, t1);
    }
    float t_enter = vmax(vmax(tmin3[0], tmin3[1]), vmax(tmin3[2], 0.0f));
    float t_exit = vmin(vmin(tmax3[0], tmax3[1]), tmax3[2]);
    if (t_enter >= t_exit || t_exit < 0.0f) goto done;
    int32_t tile[3], step[3], origin_tile[3];
    float tdel[3], tmax[3];
    for (int k = 0; k < 3; ++k) {
        float p = c->origin[k] + dir[k] * (t_enter + 0.05f);
        p = clampf(p, win_min[k] + 0.01f, win_max[k] - 0.01f);
        tile[k] = f2i(floorf(p / 16.0f));
        step[k] = sgn(dir[k]);
        tdel[k] = fabsf(inv[k]) * 16.0f;
        if (step[k] > 0) tmax[k] = ((float)((tile[k] + 1) * 16) - c->origin[k]) * inv[k];
        else tmax[k] = ((float)(tile[k] * 16) - c->origin[k]) * inv[k];
        origin_tile[k] = c->world_origin[k] / 16;
    }
    float t_cur = t_enter;
    for (int s = 0; s < 80; ++s) {
        iters++;
        int32_t rx = tile[0] - origin_tile[0], ry = tile[1] - origin_tile[1],
                rz = tile[2] - origin_tile[2];
        if (rx < 0 || rx >= d.tx || ry < 0 || ry >= d.ty || rz < 0 || rz >= d.tz) goto done;
        int32_t st_[3] = {pos_mod(tile[0], d.tx), tile[1], pos_mod(tile[2], d.tz)};
        int64_t ci = chunk_idx(&d, st_[0] / 4, st_[1] / 4, st_[2] / 4);
        int lin = (st_[0] & 3) + (st_[2] & 3) * 4 + (st_[1] & 3) * 16;
        bytes += 8;
        if ((w->chunk_mask[ci] >> lin) & 1ull) { result = t_cur; goto done; }
        if (tmax[0] < tmax[1] && tmax[0] < tmax[2]) {
            tile[0] += step[0]; t_cur = tmax[0]; tmax[0] = tmax[0] + tdel[0];
        } else if (tmax[1] < tmax[2]) {
            tile[1] += step[1]; t_cur = tmax[1]; tmax[1] = tmax[1] + tdel[1];
        } else {
            tile[2] += step[2]; t_cur = tmax[2]; tmax[2] = tmax[2] + tdel[2];
        }
    }
done:
    if (st) { st->bytes += bytes; st->iters += iters; }
    return result;
}

/* cs_beam, beam.wgsl:30-49 */
void or_beam_pass(const OrWorld *w, const OrCamera *c, float *beam_out, OrStats *st) {
    uint32_t bw = ((uint32_t)c->res_x + 7u) / 8u;
    uint32_t bh = ((uint32_t)c->res_y + 7u) / 8u;
    for (uint32_t gy = 0; gy < bh; ++gy)
        for (uint32_t gx = 0; gx < bw; ++gx) {
            float u = ((float)gx * 8.0f + 4.0f) / c->res_x;
            float v = ((float)gy * 8.0f + 4.0f) / c->res_y;
            float dir[3];
            or_ray_dir_uv(c, u, v, dir);
            beam_out[gy * bw + gx] = or_beam_first_tile(w, c, dir, st);
        }
}

/* Shadow ray of raymarch.wgsl:3953-3994 with the workload's cone:
 * theta = ign * golden angle, radius = tan(cone) * sqrt(ign). */
void or_shadow_ray(const OrCamera *c, const OrParams *p, uint32_t px, uint32_t py,
                   const float dir[3], const OrRecord *hit, float o_out[3], float d_out[3]) {
    int ax = hit->face >> 1;
    float nval = (hit->face & 1) ? -1.0f : 1.0f;
    for (int k = 0; k < 3; ++k) {
        float ph = c->origin[k] + dir[k] * hit->t;
        float n = (k == ax) ? nval : 0.0f;
        o_out[k] = ph + n * 0.001f;
    }
    float jit = or_ign((float)px, (float)py, p->frame);
    float theta = jit * 2.39996323f;
    float radius = p->cone_tan * sqrtf(jit);
    float sn, cs;
    or_sincos(theta, &sn, &cs);
    float v[3];
    for (int k = 0; k < 3; ++k) {
        float off = (p->sun_tangent[k] * cs + p->sun_bitangent[k] * sn) * radius;
        v[k] = p->sun[k] + off;
    }
    normalize3(v, d_out);
}

/* cs_main traversal part, raymarch.wgsl:576-631 (all tiles dirty, camera
 * above water) + one shadow ray per hit. */
void or_render_rows(const OrWorld *w, const OrCamera *c, const OrParams *p,
                    const float *beam, uint32_t y0, uint32_t y1, OrRecord *rec,
                    OrShadow *sh, OrStats *st) {
    uint32_t W = (uint32_t)c->res_x;
    uint32_t bw = (W + 7u) / 8u;
    for (uint32_t gy = y0; gy < y1; ++gy) {
        for (uint32_t gx = 0; gx < W; ++gx) {
            size_t i = (size_t)gy * W + gx;
            float u = (((float)gx + 0.5f) + c->jitter_x) / c->res_x;
            float v = (((float)gy + 0.5f) + c->jitter_y) / c->res_y;
            float dir[3];
            or_ray_dir_uv(c, u, v, dir);
            float skip = 0.0f;
            float org[3] = {c->origin[0], c->origin[1], c->origin[2]};
            if (p->flags & OR_F_BEAM) {
                float bt = beam[(gy / 8u) * bw + gx / 8u];
                skip = vmax(0.0f, bt - p->beam_margin);
                for (int k = 0; k < 3; ++k) org[k] = c->origin[k] + dir[k] * skip;
            }
            or_trace(w, c->world_origin, org, dir, p->max_dist, p, &rec[i], st);
            if ((p->flags & OR_F_BEAM) && (rec[i].flags & 1u)) rec[i].t = rec[i].t + skip;
            if (sh) {
                memset(&sh[i], 0, sizeof(OrShadow));
                if ((p->flags & OR_F_SHADOW) && (rec[i].flags & 1u)) {
                    float so[3], sd[3];
                    or_shadow_ray(c, p, gx, gy, dir, &rec[i], so, sd);
                    uint32_t ssteps = 0;
                    sh[i].occluded = (uint8_t)or_trace_any(w, c->world_origin, so, sd,
                                                           p->shadow_max_dist, p, &ssteps, st);
                    sh[i].steps = ssteps;
                    sh[i].traced = 1;
                }
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* temporal tile gating (src/temporal.rs:16-111, src/app.rs:643-725)   */
/* ------------------------------------------------------------------ */

/* project_brick_to_tiles: the world AABB of slot brick bi (window corner
 * c->world_origin; slot -> world fold as the toroidal storage implies) is
 * projected through the camera and the covered 8x8 screen tiles are set in
 * mask (tiles_w = ceil(W/8), bit ti of word ti>>5). */
void or_project_brick_to_tiles(const OrWorld *w, const OrCamera *c, uint32_t bi, uint32_t *mask) {
    Dims d = dims_of(w);
    int32_t bx = (int32_t)(bi % (uint32_t)d.bx);
    int32_t by = (int32_t)((bi / (uint32_t)d.bx) % (uint32_t)d.by);
    int32_t bz = (int32_t)(bi / ((uint32_t)d.bx * (uint32_t)d.by));
    int32_t wx = c->world_origin[0] + pos_mod(bx * 4 - c->world_origin[0], d.vx);
    int32_t wy = by * 4;
    int32_t wz = c->world_origin[2] + pos_mod(bz * 4 - c->world_origin[2], d.vz);
    float base[3] = {(float)wx, (float)wy, (float)wz};
    uint32_t W = (uint32_t)c->res_x, H = (uint32_t)c->res_y;
    uint32_t tiles_w = (W + 7u) / 8u, tiles_h = (H + 7u) / 8u;
    float tan_half = c->tan_half_fov;
    float aspect = (float)W / (float)H;
    float wf = (float)W, hf = (float)H;
    int32_t min_x = INT32_MAX, min_y = INT32_MAX, max_x = INT32_MIN, max_y = INT32_MIN;
    int any_visible = 0, any_behind = 0;
    for (int ci = 0; ci < 8; ++ci) {
        float corner[3] = {base[0] + (float)(ci & 1) * 4.0f, base[1] + (float)((ci >> 1) & 1) * 4.0f,
                           base[2] + (float)((ci >> 2) & 1) * 4.0f};
        float dv[3] = {corner[0] - c->origin[0], corner[1] - c->origin[1], corner[2] - c->origin[2]};
        float z_cam = (dv[0] * c->forward[0] + dv[1] * c->forward[1]) + dv[2] * c->forward[2];
        if (z_cam <= 0.1f) {
            any_behind = 1;
            continue;
        }
        float x_cam = (dv[0] * c->right[0] + dv[1] * c->right[1]) + dv[2] * c->right[2];
        float y_cam = (dv[0] * c->up[0] + dv[1] * c->up[1]) + dv[2] * c->up[2];
        float inv_z = 1.0f / (z_cam * tan_half);
        float ndc_x = (x_cam * inv_z) / aspect;
        float ndc_y = y_cam * inv_z;
        int32_t px = f2i((ndc_x + 1.0f) * 0.5f * wf);
        int32_t py = f2i((1.0f - ndc_y) * 0.5f * hf);
        if (px < min_x) min_x = px;
        if (py < min_y) min_y = py;
        if (px > max_x) max_x = px;
        if (py > max_y) max_y = py;
        any_visible = 1;
    }
    if (!any_visible) return;
    if (any_behind) {
        min_x = 0; min_y = 0;
        max_x = (int32_t)W - 1; max_y = (int32_t)H - 1;
    }
    if (max_x < 0 || max_y < 0 || min_x >= (int32_t)W || min_y >= (int32_t)H) return;
    uint32_t tx_min = (uint32_t)(min_x > 0 ? min_x : 0) / 8u;
    uint32_t ty_min = (uint32_t)(min_y > 0 ? min_y : 0) / 8u;
    uint32_t tx_max = (uint32_t)(max_x < (int32_t)W - 1 ? max_x : (int32_t)W - 1) / 8u;
    uint32_t ty_max = (uint32_t)(max_y < (int32_t)H - 1 ? max_y : (int32_t)H - 1) / 8u;
    if (tx_max > tiles_w - 1u) tx_max = tiles_w - 1u;
    if (ty_max > tiles_h - 1u) ty_max = tiles_h - 1u;
    for (uint32_t ty = ty_min; ty <= ty_max; ++ty)
        for (uint32_t tx = tx_min; tx <= tx_max; ++tx) {
            uint32_t idx = ty * tiles_w + tx;
            mask[idx >> 5] |= 1u << (idx & 31u);
        }
}

/* The rotating, hash-scattered animation refresh (src/app.rs:706-725): tile
 * (tx, ty) is refreshed when ((tx*73856093 ^ ty*19349663) * 2654435761 >> 8)
 * % spread == phase, in 64-bit wrapping arithmetic (usize on the
 * reference's 64-bit targets). */
void or_refresh_tiles(uint32_t tiles_w, uint32_t tiles_h, uint32_t spread, uint32_t phase,
                      uint32_t *mask) {
    if (spread == 0) return;
    for (uint32_t ti = 0; ti < tiles_w * tiles_h; ++ti) {
        uint64_t tx = ti % tiles_w, ty = ti / tiles_w;
        uint64_t h = ((tx * 73856093ull) ^ (ty * 19349663ull)) * 2654435761ull;
        if ((h >> 8) % spread == phase) mask[ti >> 5] |= 1u << (ti & 31u);
    }
}

/* ------------------------------------------------------------------ */
/* threading                                                           */
/* ------------------------------------------------------------------ */
static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

typedef struct {
    const OrWorld *w;
    const OrCamera *c;
    const OrParams *p;
    const float *beam;
    uint32_t H;
    _Atomic uint32_t *next_row;   /* rows are handed out one at a time */
    OrRecord *rec;
    OrShadow *sh;
    OrStats st;
} RowJob;

/* Rows cost very different amounts (sky rows end at once, terrain rows
 * step through surfaces), so every thread takes the next untraced row until
 * none is left. */
static void *row_thread(void *arg) {
    RowJob *j = (RowJob *)arg;
    for (;;) {
        uint32_t y = atomic_fetch_add(j->next_row, 1u);
        if (y >= j->H) break;
        or_render_rows(j->w, j->c, j->p, j->beam, y, y + 1, j->rec, j->sh, &j->st);
    }
    return NULL;
}

double or_render_frame(const OrWorld *w, const OrCamera *c, const OrParams *p, OrRecord *rec,
                       OrShadow *sh, float *beam, int nthreads, OrStats *st) {
    double t0 = now_s();
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    if (p->flags & OR_F_BEAM) or_beam_pass(w, c, beam, st);
    uint32_t H = (uint32_t)c->res_y;
    pthread_t th[256];
    RowJob jobs[256];
    _Atomic uint32_t next_row = 0;
    int used = 0;
    for (int i = 0; i < nthreads && (uint32_t)i < H; ++i) {
        RowJob *j = &jobs[used++];
        j->w = w; j->c = c; j->p = p; j->beam = beam; j->H = H; j->next_row = &next_row;
        j->rec = rec; j->sh = sh;
        j->st.bytes = 0; j->st.iters = 0;
    }
    for (int i = 1; i < used; ++i) pthread_create(&th[i], NULL, row_thread, &jobs[i]);
    if (used > 0) row_thread(&jobs[0]);
    for (int i = 1; i < used; ++i) pthread_join(th[i], NULL);
    if (st)
        for (int i = 0; i < used; ++i) { st->bytes += jobs[i].st.bytes; st->iters += jobs[i].st.iters; }
    return now_s() - t0;
}

/* ------------------------------------------------------------------ */
/* contact AO of primary hits                                           */
/* ------------------------------------------------------------------ */
#define AO_DIST 64.0f /* raymarch.wgsl:4522 */

static inline int is_leaf_block(uint32_t m) {  /* raymarch.wgsl:908-911 */
    return m == 14u || m == 25u || m == 26u || m == 27u;
}

/* is_voxel_solid (raymarch.wgsl:297-322): window test, slot fold, then the
 * chunk -> tile -> brick bits; *mat gets the voxel's material byte
 * (voxel_material_at, :324-346) when solid. */
static int ao_solid(const OrWorld *w, const Dims *d, const int32_t v[3], const int32_t ro[3],
                    uint32_t *mat) {
    int32_t rx = v[0] - ro[0], ry = v[1] - ro[1], rz = v[2] - ro[2];
    if (rx < 0 || rx >= d->vx || ry < 0 || ry >= d->vy || rz < 0 || rz >= d->vz) return 0;
    int32_t sx = pos_mod(v[0], d->vx), sy = v[1], sz = pos_mod(v[2], d->vz);
    int64_t ci = chunk_idx(d, sx >> 6, sy >> 6, sz >> 6);
    int tl = child_bit((sx >> 4) & 3, (sy >> 4) & 3, (sz >> 4) & 3);
    if (!((w->chunk_mask[ci] >> tl) & 1ull)) return 0;
    int64_t ti = tile_idx(d, sx >> 4, sy >> 4, sz >> 4);
    int bl = child_bit((sx >> 2) & 3, (sy >> 2) & 3, (sz >> 2) & 3);
    if (!((w->tile_mask[ti] >> bl) & 1ull)) return 0;
    const OrBrick *b = &w->bricks[brick_idx(d, sx >> 2, sy >> 2, sz >> 2)];
    int vi = child_bit(sx & 3, sy & 3, sz & 3);
    if (!((b->occupancy >> vi) & 1ull)) return 0;
    *mat = b->materials[vi];
    return 1;
}

/* ao_occluder (raymarch.wgsl:4462-4465): solid and not decoration */
static int ao_occluder(const OrWorld *w, const Dims *d, const int32_t v[3], const int32_t ro[3]) {
    uint32_t m = 0;
    if (!ao_solid(w, d, v, ro, &m)) return 0;
    return !is_decoration(m);
}

/* ao_corner (raymarch.wgsl:4467-4475) */
static float ao_corner(const OrWorld *w, const Dims *d, const int32_t base[3],
                       const int32_t da[3], const int32_t db[3], const int32_t ro[3]) {
    int32_t a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) {
        a[k] = base[k] + da[k];
        b[k] = base[k] + db[k];
        c[k] = base[k] + da[k] + db[k];
    }
    int s1 = ao_occluder(w, d, a, ro), s2 = ao_occluder(w, d, b, ro);
    int cd = ao_occluder(w, d, c, ro);
    if (s1 && s2) return 0.35f;
    int cnt = s1 + s2 + cd;
    return 1.0f - (float)cnt * 0.22f;
}

/* WGSL mix(a, b, t) = a * (1 - t) + b * t */
static inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }

/* compute_ao (raymarch.wgsl:4417-4453) for pixel (px, py) of a primary
 * frame: origin = camera origin, dir = ray_dir_uv of the pixel centre,
 * t / voxel / entry face from its record. */
float or_compute_ao(const OrWorld *w, const OrCamera *c, const OrRecord *rec, uint32_t px,
                    uint32_t py) {
    if (!(rec->flags & 1u)) return 1.0f;
    const uint32_t m = rec->mat;
    if (rec->t > AO_DIST || is_leaf_block(m) || m == MAT_LEAF_FRINGE) return 1.0f;
    Dims d = dims_of(w);
    float dir[3];
    float u = (((float)px + 0.5f) + c->jitter_x) / c->res_x;
    float v = (((float)py + 0.5f) + c->jitter_y) / c->res_y;
    or_ray_dir_uv(c, u, v, dir);
    const int na = rec->face >> 1;
    const int32_t n_dir = (rec->face & 1u) ? -1 : 1;  /* -step[na] */
    float lf[3];
    for (int k = 0; k < 3; ++k) lf[k] = (c->origin[k] + dir[k] * rec->t) - (float)rec->voxel[k];
    int32_t da[3] = {0, 0, 0}, db[3] = {0, 0, 0};
    float fa, fb;
    if (na == 0) { da[1] = 1; db[2] = 1; fa = lf[1]; fb = lf[2]; }
    else if (na == 1) { da[0] = 1; db[2] = 1; fa = lf[0]; fb = lf[2]; }
    else { da[0] = 1; db[1] = 1; fa = lf[0]; fb = lf[1]; }
    int32_t dan[3] = {-da[0], -da[1], -da[2]}, dbn[3] = {-db[0], -db[1], -db[2]};
    int32_t base[3] = {rec->voxel[0], rec->voxel[1], rec->voxel[2]};
    base[na] += n_dir;
    const int32_t *ro = c->world_origin;
    float ao00 = ao_corner(w, &d, base, dan, dbn, ro);
    float ao10 = ao_corner(w, &d, base, da, dbn, ro);
    float ao01 = ao_corner(w, &d, base, dan, db, ro);
    float ao11 = ao_corner(w, &d, base, da, db, ro);
    float fa_c = clampf(fa, 0.0f, 1.0f), fb_c = clampf(fb, 0.0f, 1.0f);
    float ao_x0 = mixf(ao00, ao10, fa_c);
    float ao_x1 = mixf(ao01, ao11, fa_c);
    return mixf(ao_x0, ao_x1, fb_c);
}

typedef struct {
    const OrWorld *w;
    const OrCamera *c;
    const OrRecord *rec;
    float *ao;
    uint32_t y0, y1;
} AoJob;

static void *ao_thread(void *arg) {
    AoJob *j = (AoJob *)arg;
    uint32_t W = (uint32_t)j->c->res_x;
    for (uint32_t y = j->y0; y < j->y1; ++y)
        for (uint32_t x = 0; x < W; ++x)
            j->ao[(size_t)y * W + x] = or_compute_ao(j->w, j->c, &j->rec[(size_t)y * W + x], x, y);
    return NULL;
}

void or_render_ao(const OrWorld *w, const OrCamera *c, const OrRecord *rec, float *ao,
                  int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    uint32_t H = (uint32_t)c->res_y;
    pthread_t th[256];
    AoJob jobs[256];
    int used = 0;
    for (int i = 0; i < nthreads; ++i) {
        uint32_t a = (uint32_t)((uint64_t)H * i / nthreads);
        uint32_t b = (uint32_t)((uint64_t)H * (i + 1) / nthreads);
        if (b <= a) continue;
        AoJob *j = &jobs[used++];
        j->w = w; j->c = c; j->rec = rec; j->ao = ao; j->y0 = a; j->y1 = b;
    }
    for (int i = 1; i < used; ++i) pthread_create(&th[i], NULL, ao_thread, &jobs[i]);
    if (used > 0) ao_thread(&jobs[0]);
    for (int i = 1; i < used; ++i) pthread_join(th[i], NULL);
}

typedef struct {
    const OrWorld *w;
    const OrCamera *c;
    const OrParams *p;
    const float *beam;
    uint32_t stride, offset, first, last; /* rows first..last-1 of the set */
    OrRecord *rec;
    OrShadow *sh;
    OrStats st;
} RowSetJob;

static void *rowset_thread(void *arg) {
    RowSetJob *j = (RowSetJob *)arg;
    for (uint32_t k = j->first; k < j->last; ++k) {
        uint32_t y = j->offset + k * j->stride;
        or_render_rows(j->w, j->c, j->p, j->beam, y, y + 1, j->rec, j->sh, &j->st);
    }
    return NULL;
}

/* Rows offset, offset+stride, ... of a frame (the beam buffer is given) on
 * nthreads threads; records land at their full-frame indices.  Returns wall
 * seconds.  Used for bounded CPU samples of a frame. */
double or_render_row_set(const OrWorld *w, const OrCamera *c, const OrParams *p,
                         const float *beam, uint32_t stride, uint32_t offset, OrRecord *rec,
                         OrShadow *sh, int nthreads, OrStats *st) {
    double t0 = now_s();
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    if (stride < 1) stride = 1;
    uint32_t H = (uint32_t)c->res_y;
    uint32_t nrows = offset < H ? (H - offset + stride - 1) / stride : 0;
    pthread_t th[256];
    RowSetJob jobs[256];
    int used = 0;
    for (int i = 0; i < nthreads; ++i) {
        uint32_t a = (uint32_t)((uint64_t)nrows * i / nthreads);
        uint32_t b = (uint32_t)((uint64_t)nrows * (i + 1) / nthreads);
        if (b <= a) continue;
        RowSetJob *j = &jobs[used++];
        j->w = w; j->c = c; j->p = p; j->beam = beam; j->stride = stride; j->offset = offset;
        j->first = a; j->last = b; j->rec = rec; j->sh = sh;
        j->st.bytes = 0; j->st.iters = 0;
    }
    for (int i = 1; i < used; ++i) pthread_create(&th[i], NULL, rowset_thread, &jobs[i]);
    if (used > 0) rowset_thread(&jobs[0]);
    for (int i = 1; i < used; ++i) pthread_join(th[i], NULL);
    if (st)
        for (int i = 0; i < used; ++i) { st->bytes += jobs[i].st.bytes; st->iters += jobs[i].st.iters; }
    return now_s() - t0;
}

typedef struct {
    const OrWorld *w;
    const int32_t *ro;
    const OrRay *rays;
    size_t a, b;
    const OrParams *p;
    OrRecord *out;
    OrShadow *sh;
    OrStats st;
} BatchJob;

/* One queue ray: kind (low 2 bits) 1 trace_any, 2 trace_no_water, else
 * trace; a trace ray flagged OR_RAY_SPAWN_SHADOW that hits is followed by its
 * shadow ray (raymarch.wgsl:3953-3994) with the jitter seeded by the ray
 * index: ign(i & 0xFFFF, i >> 16, frame). */
static void queue_ray(const OrWorld *w, const int32_t *ro, const OrRay *r, size_t i,
                      const OrParams *p, OrRecord *out, OrShadow *sh, OrStats *st) {
    uint32_t kind = r->kind & 3u;
    if (sh) memset(sh, 0, sizeof(*sh));
    if (kind == 1u) {
        uint32_t steps = 0;
        int occ = or_trace_any(w, ro, r->org, r->dir, r->tmax, p, &steps, st);
        miss_record(out);
        out->flags = (uint8_t)(occ ? 1u : 0u);
        out->steps = steps;
        return;
    }
    if (kind == 2u) or_trace_no_water(w, ro, r->org, r->dir, r->tmax, p, out, st);
    else or_trace(w, ro, r->org, r->dir, r->tmax, p, out, st);
    if (sh && (r->kind & OR_RAY_SPAWN_SHADOW) && (out->flags & 1u)) {
        int ax = out->face >> 1;
        float nval = (out->face & 1) ? -1.0f : 1.0f;
        float so[3], v[3], sd[3];
        for (int k = 0; k < 3; ++k) {
            float ph = r->org[k] + r->dir[k] * out->t;
            so[k] = ph + ((k == ax) ? nval : 0.0f) * 0.001f;
        }
        float jit = or_ign((float)(uint32_t)(i & 0xFFFFu), (float)(uint32_t)(i >> 16), p->frame);
        float theta = jit * 2.39996323f;
        float radius = p->cone_tan * sqrtf(jit);
        float sn, cs;
        or_sincos(theta, &sn, &cs);
        for (int k = 0; k < 3; ++k)
            v[k] = p->sun[k] + (p->sun_tangent[k] * cs + p->sun_bitangent[k] * sn) * radius;
        normalize3(v, sd);
        uint32_t ssteps = 0;
        sh->occluded = (uint8_t)or_trace_any(w, ro, so, sd, p->shadow_max_dist, p, &ssteps, st);
        sh->steps = ssteps;
        sh->traced = 1;
    }
}

static void *batch_thread(void *arg) {
    BatchJob *j = (BatchJob *)arg;
    for (size_t i = j->a; i < j->b; ++i)
        queue_ray(j->w, j->ro, &j->rays[i], i, j->p, &j->out[i], j->sh ? &j->sh[i] : NULL, &j->st);
    return NULL;
}

double or_trace_batch(const OrWorld *w, const int32_t ro[3], const OrRay *rays, size_t n,
                      const OrParams *p, OrRecord *out, OrShadow *sh, int nthreads, OrStats *st) {
    double t0 = now_s();
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    BatchJob jobs[256];
    int used = 0;
    for (int i = 0; i < nthreads; ++i) {
        size_t a = n * (size_t)i / (size_t)nthreads, b = n * (size_t)(i + 1) / (size_t)nthreads;
        if (b <= a) continue;
        BatchJob *j = &jobs[used++];
        j->w = w; j->ro = ro; j->rays = rays; j->a = a; j->b = b; j->p = p; j->out = out;
        j->sh = sh;
        j->st.bytes = 0; j->st.iters = 0;
    }
    for (int i = 1; i < used; ++i) pthread_create(&th[i], NULL, batch_thread, &jobs[i]);
    if (used > 0) batch_thread(&jobs[0]);
    for (int i = 1; i < used; ++i) pthread_join(th[i], NULL);
    if (st)
        for (int i = 0; i < used; ++i) { st->bytes += jobs[i].st.bytes; st->iters += jobs[i].st.iters; }
    return now_s() - t0;
}

/* ------------------------------------------------------------------ */
/* O1: flat CPU DDA, src/raycast.rs:21-133                             */
/* ------------------------------------------------------------------ */
static int o1_in_window(const Dims *d, const int32_t v[3], const int32_t o[3]) {
    int32_t rx = v[0] - o[0], ry = v[1] - o[1], rz = v[2] - o[2];
    return rx >= 0 && ry >= 0 && rz >= 0 && (uint32_t)rx < (uint32_t)d->vx &&
           (uint32_t)ry < (uint32_t)d->vy && (uint32_t)rz < (uint32_t)d->vz;
}

static int o1_in_solid(const OrWorld *w, const Dims *d, const int32_t v[3], const int32_t o[3]) {
    if (!o1_in_window(d, v, o)) return 0;
    int32_t sx = pos_mod(v[0], d->vx);  /* rem_euclid */
    int32_t sy = v[1];
    int32_t sz = pos_mod(v[2], d->vz);
    const OrBrick *b = &w->bricks[brick_idx(d, sx / 4, sy / 4, sz / 4)];
    if (b->occupancy == 0) return 0;
    int vi = child_bit(sx % 4, sy % 4, sz % 4);
    if (!((b->occupancy >> vi) & 1ull)) return 0;
    return b->materials[vi] != MAT_LEAF_FRINGE;
}

int or_raycast(const OrWorld *w, const float cam[3], const float dir_in[3],
               const int32_t origin[3], OrPickHit *out, uint32_t *steps_out) {
    Dims d = dims_of(w);
    if (steps_out) *steps_out = 0;
    /* glam 0.29.3 Vec3::normalize_or_zero: self * (1 / sqrt(dot(self, self))) */
    float len = sqrtf((dir_in[0] * dir_in[0] + dir_in[1] * dir_in[1]) + dir_in[2] * dir_in[2]);
    float rcp = 1.0f / len;
    if (!(isfinite(rcp) && rcp > 0.0f)) return 0;
    float dir[3] = {dir_in[0] * rcp, dir_in[1] * rcp, dir_in[2] * rcp};
    if (dir[0] == 0.0f && dir[1] == 0.0f && dir[2] == 0.0f) return 0;
    float dims[3] = {(float)d.vx, (float)d.vy, (float)d.vz};
    float wmin[3], wmax[3], inv[3], tmin[3], tmax[3];
    for (int k = 0; k < 3; ++k) {
        wmin[k] = (float)origin[k];
        wmax[k] = wmin[k] + dims[k];
        inv[k] = safe_inv(dir[k]);
        float t0 = (wmin[k] - cam[k]) * inv[k];
        float t1 = (wmax[k] - cam[k]) * inv[k];
        tmin[k] = vmin(t0, t1);
        tmax[k] = vmax(t0, t1);
    }
    /* max_element / min_element: x.max(y.max(z)) */
    float t_enter = vmax(vmax(tmin[0], vmax(tmin[1], tmin[2])), 0.0f);
    float t_exit = vmin(tmax[0], vmin(tmax[1], tmax[2]));
    if (t_enter >= t_exit || t_exit < 0.0f) return 0;
    int32_t voxel[3], step[3];
    float tdel[3], tm[3];
    for (int k = 0; k < 3; ++k) {
        float p = cam[k] + dir[k] * (t_enter + 1e-3f);
        p = vmin(vmax(p, wmin[k] + 1e-3f), wmax[k] - 1e-3f); /* glam clamp */
        voxel[k] = f2i(floorf(p));
        step[k] = sgn(dir[k]);
        tdel[k] = fabsf(inv[k]);
    }
    for (int k = 0; k < 3; ++k) {
        float nxt = step[k] > 0 ? (float)(voxel[k] + 1) : (float)voxel[k];
        tm[k] = (nxt - cam[k]) * inv[k];
    }
    int32_t last_axis = -1;
    int32_t steps_left = 4096;
#define ARGMIN_STEP(axv)                                                        \
    do {                                                                        \
        int32_t a_ = -1;                                                        \
        float m_ = INFINITY;                                                    \
        for (int k = 0; k < 3; ++k)                                             \
            if (step[k] != 0 && tm[k] < m_) { a_ = k; m_ = tm[k]; }             \
        if (a_ >= 0) { voxel[a_] += step[a_]; tm[a_] += tdel[a_]; }             \
        (axv) = a_;                                                             \
    } while (0)
    while (steps_left > 0 && o1_in_solid(w, &d, voxel, origin)) {
        int32_t ax;
        ARGMIN_STEP(ax);
        if (ax < 0) goto miss;
        last_axis = ax;
        steps_left--;
        if (!o1_in_window(&d, voxel, origin)) goto miss;
    }
    while (steps_left > 0) {
        if (!o1_in_window(&d, voxel, origin)) goto miss;
        if (o1_in_solid(w, &d, voxel, origin)) {
            out->voxel[0] = voxel[0]; out->voxel[1] = voxel[1]; out->voxel[2] = voxel[2];
            out->normal[0] = out->normal[1] = out->normal[2] = 0;
            if (last_axis >= 0) out->normal[last_axis] = -step[last_axis];
            if (steps_out) *steps_out = (uint32_t)(4096 - steps_left);
            return 1;
        }
        int32_t ax;
        ARGMIN_STEP(ax);
        if (ax < 0) goto miss;
        last_axis = ax;
        steps_left--;
    }
#undef ARGMIN_STEP
miss:
    if (steps_out) *steps_out = (uint32_t)(4096 - steps_left);
    return 0;
}

typedef struct {
    const OrWorld *w;
    const int32_t *origin;
    const float *cams, *dirs;
    size_t a, b;
    OrPickHit *out;
    int32_t *hit;
} PickJob;

static void *pick_thread(void *arg) {
    PickJob *j = (PickJob *)arg;
    for (size_t i = j->a; i < j->b; ++i) {
        memset(&j->out[i], 0, sizeof(OrPickHit));
        j->hit[i] = or_raycast(j->w, &j->cams[3 * i], &j->dirs[3 * i], j->origin, &j->out[i], NULL);
    }
    return NULL;
}

double or_raycast_batch(const OrWorld *w, const int32_t origin[3], const float *cams,
                        const float *dirs, size_t n, OrPickHit *out, int32_t *hit, int nthreads) {
    double t0 = now_s();
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    PickJob jobs[256];
    int used = 0;
    for (int i = 0; i < nthreads; ++i) {
        size_t a = n * (size_t)i / (size_t)nthreads, b = n * (size_t)(i + 1) / (size_t)nthreads;
        if (b <= a) continue;
        PickJob *j = &jobs[used++];
        j->w = w; j->origin = origin; j->cams = cams; j->dirs = dirs; j->a = a; j->b = b;
        j->out = out; j->hit = hit;
    }
    for (int i = 1; i < used; ++i) pthread_create(&th[i], NULL, pick_thread, &jobs[i]);
    if (used > 0) pick_thread(&jobs[0]);
    for (int i = 1; i < used; ++i) pthread_join(th[i], NULL);
    return now_s() - t0;
}

/* ------------------------------------------------------------------ */
/* the C library's binary32 transcendentals, batched                   */
/* ------------------------------------------------------------------ */
/* glibc powf / cosf / sinf are what the reference's f32::powf / cos / sin
 * call (src/voxel.rs:1262, :1623, :1639-1641, :1695-1697). */
typedef struct {
    int fn;
    const float *x;
    float *out;
    size_t a, b;
} LibmJob;

static void *libm_thread(void *arg) {
    LibmJob *j = (LibmJob *)arg;
    for (size_t i = j->a; i < j->b; ++i) {
        const float v = j->x[i];
        float r;
        if (j->fn == 0) r = powf(v, 1.15f);
        else if (j->fn == 1) r = powf(v, 0.85f);
        else if (j->fn == 2) r = cosf(v);
        else r = sinf(v);
        j->out[i] = r;
    }
    return NULL;
}

void or_libm_batch(int fn, const float *x, size_t n, float *out, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    LibmJob jobs[256];
    for (int t = 0; t < nthreads; ++t) {
        jobs[t].fn = fn;
        jobs[t].x = x;
        jobs[t].out = out;
        jobs[t].a = n * (size_t)t / (size_t)nthreads;
        jobs[t].b = n * (size_t)(t + 1) / (size_t)nthreads;
        pthread_create(&th[t], NULL, libm_thread, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
}
