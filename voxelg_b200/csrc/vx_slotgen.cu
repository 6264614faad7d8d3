// vx_slotgen.cu -- the reference's storage-chunk generator gen_slot_bricks
// (src/voxel.rs:1322-1500) on the device: terrain columns, biomes, ores,
// surface decoration and the branched trees of the chunk and its eight xz
// neighbours, written straight into the world's toroidal slots.  Compiled
// with --fmad=false so every binary32 operation rounds as the CPU's does.
//
// The reference recomputes, for every storage chunk, the terrain of its
// 32x32 columns and the trees of its 3x3 neighbourhood.  Both depend only on
// x and z, so a batch of chunks is generated by three kernels:
//   k_gen_columns  one thread per column of each distinct xz chunk:
//                  sample_terrain (:1244-1316), the biome (:1342-1344) and
//                  the surface decoration (:1394-1459) packed in one word;
//   k_gen_trees    one thread per tree candidate of each distinct source
//                  chunk (trees_for_chunk, :1537-1591), expanded into its
//                  paint primitives (paint_tree, :1605-1710);
//   k_gen_slot     one 256-thread CTA per storage chunk, four per SM: the
//                  voxels of its columns (cave and ore noise per voxel) in
//                  shared memory, then the primitives of the 3x3 source
//                  chunks in the reference's order -- source chunk (z, x),
//                  tree, primitive -- one primitive at a time with a
//                  barrier between, skipping primitives whose box misses
//                  the chunk.  Every write of one primitive carries one
//                  material, so the order among its voxels cannot change
//                  what try_write_tree_voxel (:1500-1525) leaves.  Last the
//                  512 bricks, their occupancy words (occupancy == material
//                  != 0, the invariant Brick::set keeps, :315-325) and
//                  uniform bytes go to the slot's bricks.
// powf, cosf and sinf give the host C library's binary32 results, as the
// reference's f32::powf / cos / sin do: vx_gmath.h's functions, corrected
// by the exception table (Seed::lmx) on the generator's domains.
#include <cuda_runtime.h>

#include "vx_gmath.h"
#include "vx_internal.h"
#include "vx_noise.cuh"

namespace vx {
namespace {

using noise::fbm_2d;
using noise::hash3;
using noise::value_noise_3d;

constexpr int kCV = 32;          // STORAGE_CHUNK_VOXELS
constexpr int kSea = 64;         // sea_level
constexpr int kWorldY = 256;     // WORLD_VOXELS_Y the generator is written for
constexpr int kCand = 12;        // trees_for_chunk yields at most round(1.2*5)*2
constexpr int kTrees = 9 * kCand;
constexpr int kPrims = 16;       // primitives of one tree (oak: 1 + 4*3 + 2)

enum : uint8_t {
    M_SAND = 1, M_GRASS = 2, M_DIRT = 3, M_STONE = 4, M_WATER = 12, M_WOOD = 13,
    M_LEAVES = 14, M_SNOW = 15, M_COAL = 19, M_IRON = 20, M_GOLD = 21, M_DIAMOND = 22,
    M_WOOD_BIRCH = 23, M_WOOD_PINE = 24, M_LEAVES_BIRCH = 25, M_LEAVES_PINE = 26,
    M_LEAVES_AUTUMN = 27, M_FLOWER = 30, M_TALL_GRASS = 31, M_CACTUS = 32, M_FRINGE = 33,
    M_GRASS_DRY = 34, M_BUSH = 36
};
enum { B_TUNDRA, B_PLAINS, B_FOREST, B_JUNGLE, B_SAVANNA, B_DESERT, B_BEACH, B_MOUNTAIN };

__device__ __forceinline__ int32_t f2i(float x) {
    if (x != x) return 0;
    if (x >= 1073741824.0f) return 1073741824;
    if (x <= -1073741824.0f) return -1073741824;
    return (int32_t)x;
}
__device__ __forceinline__ float fmaxr(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float fminr(float a, float b) { return b < a ? b : a; }
// the C library's powf(x, 1.15f), powf(x, 0.85f), cosf, sinf (vx_gmath.h)
__device__ __forceinline__ float pow115(const uint32_t *lmx, float x) {
    return gm::lmx_fix(lmx, gm::LMX_POW115, x, gm::pow01(x, 1.15f));
}
__device__ __forceinline__ float pow085(const uint32_t *lmx, float x) {
    return gm::lmx_fix(lmx, gm::LMX_POW085, x, gm::pow01(x, 0.85f));
}
__device__ __forceinline__ float cos_f(const uint32_t *lmx, float a) {
    return gm::lmx_fix(lmx, gm::LMX_COS, a, gm::cos_small(a));
}
__device__ __forceinline__ float sin_f(const uint32_t *lmx, float a) {
    return gm::lmx_fix(lmx, gm::LMX_SIN, a, gm::sin_small(a));
}

struct Seed {
    uint64_t seed;
    float offx, offz;      // seed_offset_xz, voxel.rs:1163-1167
    const uint32_t *lmx;   // exception table of vx_gmath.h (device copy)
};

// sample_terrain, voxel.rs:1244-1316 (ravine cut 0, rivers off)
__device__ int32_t sample_terrain(float wx, float wz, float offx, float offz, const uint32_t *lmx,
                                  int32_t *water_top) {
    const float px = wx + offx, pz = wz + offz;
    const float warp_x = fbm_2d(px * 0.005f, pz * 0.005f, 2) * 8.0f;
    const float warp_z = fbm_2d(px * 0.005f + 50.0f, pz * 0.005f + 50.0f, 2) * 8.0f;
    const float wpx = px + warp_x, wpz = pz + warp_z;
    const float base = fbm_2d(wpx * 0.012f, wpz * 0.012f, 4) * 22.0f;
    const float mountain_mask = fmaxr(fbm_2d(wpx * 0.0028f, wpz * 0.0028f, 2) + 0.2f, 0.0f);
    const float mountain_amp = fminr(mountain_mask, 1.0f);
    const float mountain_h =
        pow115(lmx, fmaxr(fbm_2d(wpx * 0.009f, wpz * 0.009f, 5), 0.0f)) * mountain_amp * 110.0f;
    const float base_h = 64.0f + 8.0f + base + mountain_h - 0.0f;
    const float h = base_h < 2.0f ? 2.0f : (base_h > 255.0f ? 255.0f : base_h);
    const int32_t hi = f2i(h);
    *water_top = hi < kSea ? kSea : 0;
    return hi;
}

// pick_biome and the Biome tables, voxel.rs:1822-1903
__device__ __forceinline__ int pick_biome(float temp, float humid, uint32_t h) {
    if (h > kSea + 36) return B_MOUNTAIN;
    if (h <= kSea + 1) return B_BEACH;
    if (temp < -0.20f) return B_TUNDRA;
    if (temp > 0.25f && humid < -0.05f) return B_DESERT;
    if (temp > 0.15f && humid > 0.25f) return B_JUNGLE;
    if (temp > 0.10f && humid < 0.10f) return B_SAVANNA;
    if (humid > 0.20f) return B_FOREST;
    return B_PLAINS;
}
__device__ __forceinline__ uint8_t top_block(int b, uint32_t h) {
    if (b == B_TUNDRA) return M_SNOW;
    if (b == B_DESERT || b == B_BEACH || b == B_SAVANNA) return M_SAND;
    if (b == B_MOUNTAIN) return h > kSea + 55 ? M_SNOW : M_STONE;
    return M_GRASS;
}
__device__ __forceinline__ uint8_t subsoil(int b) {
    if (b == B_DESERT || b == B_BEACH) return M_SAND;
    if (b == B_MOUNTAIN) return M_STONE;
    return M_DIRT;
}
__device__ __forceinline__ uint32_t tree_type(int b, uint32_t hash) {
    if (b == B_TUNDRA || b == B_MOUNTAIN) return 2;
    if (b == B_PLAINS) return hash % 3 == 0 ? 1 : 0;
    if (b == B_FOREST) {
        const uint32_t k = hash % 4;
        return k == 0 ? 1 : (k == 1 ? 3 : 0);
    }
    if (b == B_JUNGLE) return hash % 4 == 0 ? 3 : 0;
    return 0;
}
__device__ __forceinline__ float tree_density(int b) {
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

// shared-memory chunk: brick (x + y*8 + z*64) * 64 + x + z*4 + y*16
__device__ __forceinline__ uint32_t vox(uint32_t dx, uint32_t dy, uint32_t dz) {
    return (((dx >> 2) + (dy >> 2) * 8u + (dz >> 2) * 64u) << 6) +
           ((dx & 3u) + (dz & 3u) * 4u + (dy & 3u) * 16u);
}

// ------------------------------------------------------------------ trees
struct Tree {
    int32_t x, y, z;
    uint32_t ttype, hash;
};

// candidate i of trees_for_chunk(cx, cz) (voxel.rs:1537-1591); false when
// the reference's loop yields no tree for it
__device__ bool tree_candidate(int32_t cx, int32_t cz, uint32_t i, const Seed &g, Tree &t) {
    const float ccx = ((float)cx + 0.5f) * 32.0f, ccz = ((float)cz + 0.5f) * 32.0f;
    const float temperature = fbm_2d((ccx + g.offx) * 0.0006f, (ccz + g.offz) * 0.0006f, 3);
    const float humidity =
        fbm_2d((ccx + g.offx) * 0.0008f + 100.0f, (ccz + g.offz) * 0.0008f + 100.0f, 3);
    const int biome = pick_biome(temperature, humidity, kSea + 10);
    const uint32_t n_cand = (uint32_t)f2i(roundf(tree_density(biome) * 5.0f));
    if (i >= n_cand * 2u) return false;  // n <= n_cand * patch_mul <= 2 n_cand
    float patch_mul = 1.0f;
    if (biome != B_DESERT) {
        const float patch_raw = fbm_2d(ccx * 0.0035f, ccz * 0.0035f, 2);
        patch_mul = fminr(fmaxr(patch_raw + 0.4f, 0.0f) * 1.6f, 2.0f);
    }
    const uint32_t n = (uint32_t)f2i((float)n_cand * patch_mul);
    if (i >= n) return false;
    // hash_chunk, voxel.rs:1593-1601
    const uint32_t s = (uint32_t)g.seed ^ (uint32_t)(g.seed >> 32);
    uint32_t ch = (uint32_t)cx * 0x9E3779B1u;
    ch = ch + (uint32_t)cz * 0x85EBCA77u;
    ch = ch + s * 0xC2B2AE3Du;
    ch = ch ^ (ch >> 16);
    ch = ch * 0xD2B74407u;
    ch = ch ^ (ch >> 13);
    const uint32_t h = ch * 2654435761u + i * 7919u;
    const int32_t wx = cx * kCV + (int32_t)(h & 31u), wz = cz * kCV + (int32_t)((h >> 5) & 31u);
    int32_t wt;
    const int32_t th = sample_terrain((float)wx, (float)wz, g.offx, g.offz, g.lmx, &wt);
    if ((uint32_t)th <= (uint32_t)(kSea + 1)) return false;
    if (th + 22 >= kWorldY) return false;
    const float lt = fbm_2d(((float)wx + g.offx) * 0.0006f, ((float)wz + g.offz) * 0.0006f, 3);
    const float lh = fbm_2d(((float)wx + g.offx) * 0.0008f + 100.0f,
                            ((float)wz + g.offz) * 0.0008f + 100.0f, 3);
    const int lb = pick_biome(lt, lh, (uint32_t)th);
    if (lb == B_BEACH || lb == B_SAVANNA) return false;
    t.x = wx; t.y = th + 1; t.z = wz;
    t.ttype = lb == B_DESERT ? 4u : tree_type(lb, h);
    t.hash = h;
    return true;
}

enum : uint32_t { PR_LINE = 0, PR_SHELL = 1, PR_SPHERE = 2 };
struct Prim {
    int32_t a[3];    // line start / shell or sphere centre
    int32_t b[3];    // line end; b[0] = radius of a shell or sphere
    uint32_t kind_mat;
    int32_t steps;   // line: ceil(len * 1.5)
};

// Appends a tree's primitives in paint_tree order.
struct Emit {
    Prim *out;
    int n;
    // paint_line with thickness 0, voxel.rs:1744-1776
    __device__ void line(int32_t ax, int32_t ay, int32_t az, int32_t bx, int32_t by, int32_t bz,
                         uint8_t mat) {
        const int32_t d0 = bx - ax, d1 = by - ay, d2 = bz - az;
        const float len = sqrtf((float)(d0 * d0 + d1 * d1 + d2 * d2));
        Prim &p = out[n++];
        p.a[0] = ax; p.a[1] = ay; p.a[2] = az;
        p.b[0] = bx; p.b[1] = by; p.b[2] = bz;
        p.kind_mat = (PR_LINE << 8) | mat;
        p.steps = f2i(ceilf(len * 1.5f));
    }
    // paint_fringe_shell(c, r + 1) then paint_sphere(c, r): paint_canopy,
    // voxel.rs:1715-1742, :1778-1789
    __device__ void canopy(int32_t cx, int32_t cy, int32_t cz, int32_t r, uint8_t mat) {
        Prim &f = out[n++];
        f.a[0] = cx; f.a[1] = cy; f.a[2] = cz;
        f.b[0] = r + 1; f.b[1] = f.b[2] = 0;
        f.kind_mat = (PR_SHELL << 8) | M_FRINGE;
        f.steps = 0;
        Prim &p = out[n++];
        p.a[0] = cx; p.a[1] = cy; p.a[2] = cz;
        p.b[0] = r; p.b[1] = p.b[2] = 0;
        p.kind_mat = (PR_SPHERE << 8) | mat;
        p.steps = 0;
    }
};

// Whether a primitive can write into the chunk [lo, lo + 32): its voxels
// lie in the box of the segment (rounding a + d t with t in [0, 1] stays
// between the ends), in c +- (r + 1, r, r + 1) for a shell, c +- r for a
// sphere.
__device__ __forceinline__ bool prim_meets(const Prim &p, const int32_t lo[3]) {
    const uint32_t kind = p.kind_mat >> 8;
    int32_t mn[3], mx[3];
    if (kind == PR_LINE) {
        for (int k = 0; k < 3; ++k) {
            mn[k] = min(p.a[k], p.b[k]);
            mx[k] = max(p.a[k], p.b[k]);
        }
    } else {
        const int32_t r = p.b[0], rh = kind == PR_SHELL ? r + 1 : r;
        mn[0] = p.a[0] - rh; mx[0] = p.a[0] + rh;
        mn[1] = p.a[1] - r;  mx[1] = p.a[1] + r;
        mn[2] = p.a[2] - rh; mx[2] = p.a[2] + rh;
    }
    return mx[0] >= lo[0] && mn[0] < lo[0] + kCV && mx[1] >= lo[1] && mn[1] < lo[1] + kCV &&
           mx[2] >= lo[2] && mn[2] < lo[2] + kCV;
}

// branch_jitter, voxel.rs:1791-1797
__device__ __forceinline__ float branch_jitter(uint32_t hash, uint32_t b) {
    const uint32_t h = hash * 0x9E3779B1u + b * 2654435761u;
    return ((float)(h & 0xFFFFu) / 65535.0f) * 2.0f - 1.0f;
}

// paint_tree, voxel.rs:1605-1710
__device__ void tree_prims(const Tree &t, const uint32_t *lmx, Emit &e) {
    const float tau = 6.28318548202514648f;  // std::f32::consts::TAU
    const uint32_t h = t.hash;
    if (t.ttype == 2) {
        const int32_t trunk_h = 10 + (int32_t)(h % 6);
        e.line(t.x, t.y, t.z, t.x, t.y + trunk_h, t.z, M_WOOD_PINE);
        for (int32_t i = 0; i < 6; ++i) {
            const float tf = (float)i / 6.0f;
            const int32_t y = t.y + f2i((float)trunk_h * (0.35f + tf * 0.78f));
            const int32_t r = f2i(pow085(lmx, 1.0f - tf) * 3.5f + 1.0f);
            e.canopy(t.x, y, t.z, r, M_LEAVES_PINE);
        }
    } else if (t.ttype == 1) {
        const int32_t trunk_h = 8 + (int32_t)(h % 5);
        e.line(t.x, t.y, t.z, t.x, t.y + trunk_h, t.z, M_WOOD_BIRCH);
        const int32_t n = 2 + (int32_t)(h % 2);
        for (int32_t b = 0; b < n; ++b) {
            const float angle = ((float)b / (float)n) * tau + branch_jitter(h, (uint32_t)b) * 0.5f;
            const int32_t len = 2 + (int32_t)((h * ((uint32_t)b + 1u)) % 3u);
            const int32_t sy = t.y + f2i((float)trunk_h * 0.7f);
            const int32_t ex = t.x + f2i(cos_f(lmx, angle) * (float)len);
            const int32_t ez = t.z + f2i(sin_f(lmx, angle) * (float)len);
            e.line(t.x, sy, t.z, ex, sy + 1, ez, M_WOOD_BIRCH);
            e.canopy(ex, sy + 1, ez, 2, M_LEAVES_BIRCH);
        }
        e.canopy(t.x, t.y + trunk_h, t.z, 3, M_LEAVES_BIRCH);
    } else if (t.ttype == 4) {
        // arm directions per h & 3: [(1,0),(0,1)] [(-1,0),(0,-1)] [(0,1),(-1,0)] [(0,-1),(1,0)]
        const int32_t sets[4][2][2] = {{{1, 0}, {0, 1}}, {{-1, 0}, {0, -1}},
                                       {{0, 1}, {-1, 0}}, {{0, -1}, {1, 0}}};
        const int32_t col_h = 3 + (int32_t)(h % 6);
        e.line(t.x, t.y, t.z, t.x, t.y + col_h, t.z, M_CACTUS);
        const int32_t n_arms = (int32_t)(h % 3);
        const uint32_t si = h & 3u;
        for (int32_t a = 0; a < n_arms; ++a) {
            const int32_t dx = sets[si][a % 2][0], dz = sets[si][a % 2][1];
            const int32_t sy = t.y + f2i((float)col_h * 0.4f);
            const int32_t arm_top = t.y + f2i((float)col_h * 0.9f);
            const int32_t ax = t.x + dx * 2, az = t.z + dz * 2;
            e.line(t.x, sy, t.z, ax, sy, az, M_CACTUS);
            e.line(ax, sy, az, ax, arm_top, az, M_CACTUS);
        }
    } else {
        const uint8_t leaf = t.ttype == 3 ? M_LEAVES_AUTUMN : M_LEAVES;
        const int32_t trunk_h = 8 + (int32_t)(h % 5);
        e.line(t.x, t.y, t.z, t.x, t.y + trunk_h, t.z, M_WOOD);
        const int32_t n = 3 + (int32_t)(h % 2);
        for (int32_t b = 0; b < n; ++b) {
            const float angle = ((float)b / (float)n) * tau + branch_jitter(h, (uint32_t)b) * 0.6f;
            const int32_t len = 3 + (int32_t)((h * ((uint32_t)b + 7u)) % 3u);
            const int32_t sy = t.y + f2i((float)trunk_h * 0.65f);
            const int32_t ex = t.x + f2i(cos_f(lmx, angle) * (float)len);
            const int32_t ey = sy + f2i((float)len * 0.5f);
            const int32_t ez = t.z + f2i(sin_f(lmx, angle) * (float)len);
            e.line(t.x, sy, t.z, ex, ey, ez, M_WOOD);
            e.canopy(ex, ey, ez, 3, leaf);
        }
        e.canopy(t.x, t.y + trunk_h, t.z, 4, leaf);
    }
}

// try_write_tree_voxel, voxel.rs:1500-1525, on the shared chunk
__device__ __forceinline__ void tree_voxel(uint8_t *s_mat, const int32_t lo[3], int32_t x,
                                           int32_t y, int32_t z, uint8_t mat) {
    const uint32_t dx = (uint32_t)(x - lo[0]), dy = (uint32_t)(y - lo[1]), dz = (uint32_t)(z - lo[2]);
    if (dx >= (uint32_t)kCV || dy >= (uint32_t)kCV || dz >= (uint32_t)kCV) return;
    const uint32_t v = vox(dx, dy, dz);
    const uint8_t cur = s_mat[v];
    if (cur == 0 || (cur == M_FRINGE && mat != M_FRINGE)) s_mat[v] = mat;
}

// Voxel k of a primitive (any order: one primitive writes one material).
__device__ void paint_prim(uint8_t *s_mat, const int32_t lo[3], const Prim &p, int nthr) {
    const uint32_t kind = p.kind_mat >> 8;
    const uint8_t mat = (uint8_t)(p.kind_mat & 0xFFu);
    if (kind == PR_LINE) {
        if (p.steps <= 0) {
            if (threadIdx.x == 0) tree_voxel(s_mat, lo, p.a[0], p.a[1], p.a[2], mat);
            return;
        }
        const int32_t d0 = p.b[0] - p.a[0], d1 = p.b[1] - p.a[1], d2 = p.b[2] - p.a[2];
        for (int32_t s = (int32_t)threadIdx.x; s <= p.steps; s += nthr) {
            const float t = (float)s / (float)p.steps;
            const int32_t x = f2i(roundf((float)p.a[0] + (float)d0 * t));
            const int32_t y = f2i(roundf((float)p.a[1] + (float)d1 * t));
            const int32_t z = f2i(roundf((float)p.a[2] + (float)d2 * t));
            tree_voxel(s_mat, lo, x, y, z, mat);
        }
    } else if (kind == PR_SHELL) {
        const int32_t r = p.b[0], r2 = r * r, wxz = 2 * r + 3, n = (2 * r + 1) * wxz * wxz;
        for (int32_t k = (int32_t)threadIdx.x; k < n; k += nthr) {
            const int32_t dz = k % wxz - (r + 1), dx = (k / wxz) % wxz - (r + 1),
                          dy = k / (wxz * wxz) - r;
            const int32_t hx = max(abs(dx) - 1, 0), hz = max(abs(dz) - 1, 0);
            if (hx * hx + dy * dy + hz * hz > r2) continue;
            tree_voxel(s_mat, lo, p.a[0] + dx, p.a[1] + dy, p.a[2] + dz, mat);
        }
    } else {
        const int32_t r = p.b[0], r2 = r * r, wd = 2 * r + 1, n = wd * wd * wd;
        for (int32_t k = (int32_t)threadIdx.x; k < n; k += nthr) {
            const int32_t dz = k % wd - r, dx = (k / wd) % wd - r, dy = k / (wd * wd) - r;
            if (dx * dx + dy * dy + dz * dz > r2) continue;
            tree_voxel(s_mat, lo, p.a[0] + dx, p.a[1] + dy, p.a[2] + dz, mat);
        }
    }
}

// ------------------------------------------------------------------ columns
// Column word: bits 0-7 h, 8 water (water_top = sea level), 9-11 biome,
// 12-17 decoration material (0: none), 18 the decoration is a big bush.
// pos_mod(a, n), n > 0
__device__ __forceinline__ int32_t wrap(int32_t a, int32_t n) { return ((a % n) + n) % n; }

// The world chunk (x, z) of column chunk k / source chunk k of a plan.
__device__ __forceinline__ void col_chunk(const GenPlan &p, const Dims &d, uint32_t k,
                                          int32_t &cx, int32_t &cz) {
    if (p.window) {
        const int32_t sxn = d.bx / 8, szn = d.bz / 8;
        const int32_t sx = (int32_t)k % sxn, sz = (int32_t)k / sxn;
        cx = p.ox + wrap(sx - p.ox, sxn);
        cz = p.oz + wrap(sz - p.oz, szn);
    } else {
        cx = p.cols[2 * k];
        cz = p.cols[2 * k + 1];
    }
}
__device__ __forceinline__ void src_chunk(const GenPlan &p, const Dims &d, uint32_t k,
                                          int32_t &cx, int32_t &cz) {
    if (p.window) {
        const int32_t w = d.bx / 8 + 2;
        cx = p.ox - 1 + (int32_t)k % w;
        cz = p.oz - 1 + (int32_t)k / w;
    } else {
        cx = p.srcs[2 * k];
        cz = p.srcs[2 * k + 1];
    }
}

__global__ void __launch_bounds__(256) k_gen_columns(GenPlan p, Dims d, Seed g) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= p.n_cols * (uint32_t)(kCV * kCV)) return;
    const uint32_t k = c >> 10, col = c & 1023u;
    int32_t ccx, ccz;
    col_chunk(p, d, k, ccx, ccz);
    const int32_t wxi = ccx * kCV + (int32_t)(col & 31u);
    const int32_t wzi = ccz * kCV + (int32_t)(col >> 5);
    const float wx = (float)wxi, wz = (float)wzi;
    int32_t water_top;
    const int32_t h = sample_terrain(wx, wz, g.offx, g.offz, g.lmx, &water_top);
    const uint32_t hu = (uint32_t)h;
    const float temperature = fbm_2d((wx + g.offx) * 0.0006f, (wz + g.offz) * 0.0006f, 3);
    const float humidity =
        fbm_2d((wx + g.offx) * 0.0008f + 100.0f, (wz + g.offz) * 0.0008f + 100.0f, 3);
    const int biome = pick_biome(temperature, humidity, hu);
    uint32_t dec = 0, big = 0;
    if (water_top == 0 && hu < (uint32_t)(kWorldY - 1)) {
        const uint8_t surface = top_block(biome, hu);
        const int32_t dec_y = h + 1;
        const float v = hash3(wxi, dec_y, wzi) * 0.5f + 0.5f;
        const bool big_lattice = hash3(wxi & ~1, 977, wzi & ~1) * 0.5f + 0.5f > 0.9955f;
        if (surface == M_GRASS) {
            float fp, gp;
            if (biome == B_PLAINS) { fp = 0.020f; gp = 0.08f; }
            else if (biome == B_FOREST) { fp = 0.010f; gp = 0.065f; }
            else if (biome == B_JUNGLE) { fp = 0.012f; gp = 0.09f; }
            else { fp = 0.015f; gp = 0.065f; }
            if (fbm_2d((float)wxi * 0.02f + 7.0f, (float)wzi * 0.02f - 3.0f, 2) > 0.30f) {
                fp *= 3.0f;
                gp *= 12.0f;
            }
            if (v > 1.0f - fp) dec = M_FLOWER;
            else if (v > 1.0f - fp - gp) dec = M_TALL_GRASS;
            else if (big_lattice) dec = M_BUSH;
            else if (v > 1.0f - fp - gp - 0.004f) dec = M_BUSH;
        } else if (surface == M_SAND && (biome == B_DESERT || biome == B_SAVANNA)) {
            if (v > 0.99f) dec = M_GRASS_DRY;
        } else if (surface == M_SNOW && biome == B_TUNDRA) {
            if (v > 0.995f) dec = M_GRASS_DRY;
        }
        big = (dec == M_BUSH && big_lattice) ? 1u : 0u;
    }
    p.colw[c] = hu | ((water_top != 0 ? 1u : 0u) << 8) | ((uint32_t)biome << 9) | (dec << 12) |
             (big << 18);
}

// ------------------------------------------------------------------ trees
// Per source chunk: kCand headers (primitive count | base y << 8, 0 when the
// candidate yields no tree) and kCand x kPrims primitives.
__global__ void __launch_bounds__(128) k_gen_trees(GenPlan p, Dims d, Seed g) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= p.n_srcs * (uint32_t)kCand) return;
    const uint32_t k = c / kCand, i = c % kCand;
    int32_t scx, scz;
    src_chunk(p, d, k, scx, scz);
    Tree t;
    int32_t h = 0;
    if (tree_candidate(scx, scz, i, g, t)) {
        Emit e;
        e.out = reinterpret_cast<Prim *>(p.prims) + (size_t)c * kPrims;
        e.n = 0;
        tree_prims(t, g.lmx, e);
        h = e.n | (t.y << 8);
    }
    p.hdr[c] = h;
}

// ------------------------------------------------------------------ chunks
constexpr int kSlotThreads = 256;   // four CTAs per SM overlap each other's barriers
static_assert(kTrees <= 9 * kCand && (512 % kSlotThreads) == 0, "write-out covers 512 bricks");

// Job b of a plan (kGenJobInts ints, the layout of explicit plans).
__device__ __forceinline__ void job_of(const GenPlan &p, const Dims &d, uint32_t b,
                                      int32_t job[kGenJobInts]) {
    if (!p.window) {
#pragma unroll
        for (int k = 0; k < kGenJobInts; ++k) job[k] = p.jobs[(size_t)b * kGenJobInts + k];
        return;
    }
    const int32_t sxn = d.bx / 8, syn = d.by / 8, szn = d.bz / 8;
    const int32_t sx = (int32_t)b % sxn, sy = ((int32_t)b / sxn) % syn,
                  sz = (int32_t)b / (sxn * syn);
    const int32_t cx = p.ox + wrap(sx - p.ox, sxn), cz = p.oz + wrap(sz - p.oz, szn);
    job[0] = cx; job[1] = sy; job[2] = cz;
    job[3] = sx; job[4] = sy; job[5] = sz;
    job[6] = sx + sz * sxn;
#pragma unroll
    for (int k = 0; k < 9; ++k)
        job[7 + k] = (cx + k % 3 - 1 - (p.ox - 1)) + (cz + k / 3 - 1 - (p.oz - 1)) * (sxn + 2);
}

__global__ void __launch_bounds__(kSlotThreads, 4) k_gen_slot(DevWorld w, GenPlan pl) {
    __shared__ __align__(16) uint8_t s_mat[kCV * kCV * kCV];
    __shared__ int32_t s_job[kGenJobInts];
    if (threadIdx.x == 0) {
        int32_t j[kGenJobInts];
        job_of(pl, w.d, blockIdx.x, j);
#pragma unroll
        for (int k = 0; k < kGenJobInts; ++k) s_job[k] = j[k];
    }
    const uint32_t tid = threadIdx.x;
    const Prim *prims = reinterpret_cast<const Prim *>(pl.prims);

    uint4 *z4 = reinterpret_cast<uint4 *>(s_mat);
    for (uint32_t i = tid; i < (uint32_t)(kCV * kCV * kCV / 16); i += kSlotThreads)
        z4[i] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    const int32_t *job = s_job;
    const int32_t lo[3] = {job[0] * kCV, job[1] * kCV, job[2] * kCV};
    const uint32_t *colw = pl.colw + (size_t)job[6] * (kCV * kCV);

    // ---- the columns (dx, dz), voxel.rs:1333-1461
    const int32_t y0 = lo[1];
    for (uint32_t col = tid; col < (uint32_t)(kCV * kCV); col += kSlotThreads) {
        const uint32_t word = colw[col];
        const int32_t h = (int32_t)(word & 0xFFu);
        const uint32_t hu = (uint32_t)h;
        const int32_t water_top = (word >> 8) & 1u ? kSea : 0;
        const int col_top = max(h, water_top);
        if (col_top < y0 || 0 >= y0 + kCV) continue;
        const int biome = (int)((word >> 9) & 7u);
        const uint32_t dx = col & 31u, dz = col >> 5;
        const float wx = (float)(lo[0] + (int32_t)dx), wz = (float)(lo[2] + (int32_t)dz);
        const int32_t ys = max(y0, 0), ye = min(y0 + kCV, kWorldY);
        const int32_t seal = water_top > h ? h - 5 : INT32_MIN;
        // stone_or_ore's two noises (voxel.rs:1906-1916) along this column
        // and the two cave noises (:1361-1366)
        noise::ColumnNoise3 ore1, ore2, cave1, cave2;
        ore1.init(wx * 0.27f, wz * 0.27f);
        ore2.init(wx * 0.55f, wz * 0.55f);
        cave1.init(wx * 0.045f, wz * 0.045f);
        cave2.init(wx * 0.110f, wz * 0.110f);
        for (int32_t y = ys; y < ye; ++y) {
            if (y > h) break;
            if (!(y >= seal) && y > 4 && y + 3 < h) {
                const float cn = cave1.eval((float)y * 0.085f);
                const float cn2 = cave2.eval((float)y * 0.060f);
                if ((cn + cn2 * 0.6f) > 0.30f) continue;
            }
            uint8_t mat;
            if ((uint32_t)y >= hu) {
                mat = top_block(biome, hu);
            } else if ((uint32_t)y + 4u >= hu) {
                mat = subsoil(biome);
            } else {
                const float fy = (float)y;
                const float depth = fmaxr((float)hu - fy, 0.0f);
                const float n1 = ore1.eval(fy * 0.27f);
                const float n2 = ore2.eval(fy * 0.55f);
                const float combined = n1 + n2 * 0.30f;
                if (depth > 30.0f && combined > 0.50f) mat = M_DIAMOND;
                else if (depth > 20.0f && combined > 0.36f) mat = M_GOLD;
                else if (depth > 10.0f && combined > 0.24f) mat = M_IRON;
                else if (combined > 0.32f) mat = M_COAL;
                else mat = M_STONE;
            }
            s_mat[vox(dx, (uint32_t)(y - y0), dz)] = mat;
        }
        if (water_top > h) {
            const int32_t fb = max(h + 1, y0), fe = min(water_top, y0 + kCV - 1);
            for (int32_t wy = fb; wy <= fe; ++wy) s_mat[vox(dx, (uint32_t)(wy - y0), dz)] = M_WATER;
        }
        const uint32_t dec = (word >> 12) & 63u;
        const int32_t dec_y = h + 1;
        if (dec != 0u && dec_y >= y0 && dec_y < y0 + kCV) {
            const uint32_t dy = (uint32_t)(dec_y - y0);
            s_mat[vox(dx, dy, dz)] = (uint8_t)dec;
            if (((word >> 18) & 1u) && dec_y + 1 < y0 + kCV) s_mat[vox(dx, dy + 1u, dz)] = M_BUSH;
        }
    }
    __syncthreads();

    // ---- trees of the 3x3 source chunks in the reference's order
    for (int k = 0; k < 9; ++k) {
        const int32_t src = job[7 + k];
        for (int i = 0; i < kCand; ++i) {
            const int32_t hd = pl.hdr[(size_t)src * kCand + i];
            const int np = hd & 0xFF;
            const int32_t base_y = hd >> 8;
            if (np == 0 || base_y > lo[1] + kCV || base_y + 22 < lo[1]) continue;
            const Prim *tp = prims + ((size_t)src * kCand + i) * kPrims;
            for (int p = 0; p < np; ++p) {
                const Prim pr = tp[p];
                if (!prim_meets(pr, lo)) continue;
                paint_prim(s_mat, lo, pr, kSlotThreads);
                __syncthreads();
            }
        }
    }

    // ---- bricks out: material rows, occupancy words, uniform bytes
    const uint32_t sbx = (uint32_t)job[3] * 8u, sby = (uint32_t)job[4] * 8u,
                   sbz = (uint32_t)job[5] * 8u;
    for (uint32_t b = tid; b < 512u; b += kSlotThreads) {
        const uint32_t gbi = (sbx + (b & 7u)) + (sby + ((b >> 3) & 7u)) * (uint32_t)w.d.bx +
                             (sbz + (b >> 6)) * (uint32_t)(w.d.bx * w.d.by);
        const uint4 *src = reinterpret_cast<const uint4 *>(s_mat + b * 64u);
        uint4 *dst = reinterpret_cast<uint4 *>(w.mat + (size_t)gbi * 64u);
        uint64_t occ = 0;
        const uint32_t m0 = s_mat[b * 64u], rep = 0x01010101u * m0;
        bool same = m0 != 0u;
#pragma unroll
        for (int q4 = 0; q4 < 4; ++q4) {
            const uint4 q = src[q4];
            dst[q4] = q;
            const uint32_t qs[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                same = same && qs[m] == rep;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if ((qs[m] >> (8 * j)) & 0xFFu) occ |= 1ull << (16 * q4 + 4 * m + j);
            }
        }
        w.occ[gbi] = occ;
        w.brick_uniform[gbi] = (occ == ~0ull && same) ? (uint8_t)m0 : (uint8_t)0;
    }
}

}  // namespace

namespace {
__global__ void k_gen_math(const uint32_t *lmx, uint32_t fn, const float *__restrict__ in, size_t n,
                           float *__restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = in[i];
    float v;
    if (fn == gm::LMX_POW115) v = pow115(lmx, x);
    else if (fn == gm::LMX_POW085) v = pow085(lmx, x);
    else if (fn == gm::LMX_COS) v = cos_f(lmx, x);
    else v = sin_f(lmx, x);
    out[i] = v;
}
}  // namespace

cudaError_t launch_gen_math(const uint32_t *lmx, uint32_t fn, const float *in, size_t n, float *out,
                            cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_gen_math<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(lmx, fn, in, n, out);
    return cudaGetLastError();
}

size_t gen_prim_bytes_per_src() { return sizeof(Prim) * kCand * kPrims; }

cudaError_t launch_gen_slots(const DevWorld &w, uint64_t seed, const GenPlan &p, cudaStream_t s) {
    if (p.n_jobs == 0) return cudaSuccess;
    Seed g;
    g.seed = seed;
    // seed_offset_xz, voxel.rs:1163-1167
    g.offx = (float)(int32_t)(uint32_t)(seed >> 32) * 0.01734f;
    g.offz = (float)(int32_t)(uint32_t)(seed & 0xFFFFFFFFull) * 0.02153f;
    g.lmx = p.lmx;
    if (!g.lmx) return cudaErrorInvalidValue;
    const uint32_t n_col_threads = p.n_cols * (uint32_t)(kCV * kCV);
    k_gen_columns<<<(n_col_threads + 255) / 256, 256, 0, s>>>(p, w.d, g);
    const uint32_t n_tree_threads = p.n_srcs * (uint32_t)kCand;
    k_gen_trees<<<(n_tree_threads + 127) / 128, 128, 0, s>>>(p, w.d, g);
    k_gen_slot<<<p.n_jobs, kSlotThreads, 0, s>>>(w, p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_rebuild_pyramid(w, s);
}

}  // namespace vx
