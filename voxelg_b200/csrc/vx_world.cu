// vx_world.cu -- device-resident world pyramid: layout conversion, seeded
// terrain generation, mask/LUT construction and the incremental dirty-brick
// update.  Compiled with --fmad=false (the terrain noise must match the CPU
// restatement bit for bit).
//
// Semantics follow src/voxel.rs: brick_uniform_of :233-247, tile_uniform_of
// :253-272, rebuild_all_uniform :946-957, rebuild_all_masks :958-1000,
// refresh_masks_for_brick :879-914 (the incremental update recomputes each
// touched tile/chunk/L4 word from its 64 children, which equals the value
// the reference's incremental bit maintenance keeps), noise :1163-1232,
// :1999-2021.
#include <cuda_runtime.h>

#include "vx_internal.h"
#include "vx_noise.cuh"

namespace vx {
namespace {

__device__ __forceinline__ int32_t f2i(float x) {
    if (x != x) return 0;
    if (x >= 1073741824.0f) return 1073741824;
    if (x <= -1073741824.0f) return -1073741824;
    return (int32_t)x;
}
__device__ __forceinline__ int child_bit(int lx, int ly, int lz) { return lx + lz * 4 + ly * 16; }

// ------------------------------------------------------------- layout
// voxelG's 72-byte Brick (AoS) <-> occupancy array + 64-byte material rows.
__global__ void k_aos_to_soa(DevWorld w, const VxBrick *__restrict__ aos, int64_t first,
                             int64_t count) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint2 *src = reinterpret_cast<const uint2 *>(aos + i);
    const uint2 o = src[0];
    w.occ[first + i] = (uint64_t)o.x | ((uint64_t)o.y << 32);
    uint2 *dst = reinterpret_cast<uint2 *>(w.mat + (first + i) * 64);
#pragma unroll
    for (int k = 0; k < 8; ++k) dst[k] = src[1 + k];
}

__global__ void k_soa_to_aos(DevWorld w, VxBrick *__restrict__ aos, int64_t first,
                             int64_t count) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint2 *dst = reinterpret_cast<uint2 *>(aos + i);
    const uint64_t o = w.occ[first + i];
    dst[0] = make_uint2((uint32_t)o, (uint32_t)(o >> 32));
    const uint2 *src = reinterpret_cast<const uint2 *>(w.mat + (first + i) * 64);
#pragma unroll
    for (int k = 0; k < 8; ++k) dst[1 + k] = src[k];
}

// brick_uniform_of, voxel.rs:233-247
__device__ __forceinline__ uint8_t uniform_of(uint64_t occ, const uint8_t *row) {
    if (occ != ~0ull) return 0;
    const uint4 *r = reinterpret_cast<const uint4 *>(row);
    const uint8_t m0 = row[0];
    if (m0 == 0) return 0;
    const uint32_t rep = 0x01010101u * m0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint4 q = r[k];
        if (q.x != rep || q.y != rep || q.z != rep || q.w != rep) return 0;
    }
    return m0;
}

// ------------------------------------------------------------- terrain
using noise::fbm_2d;
using noise::value_noise_3d;

struct GenArgs {
    DevWorld w;
    VxTerrainParams t;
    float off_x, off_z;   // seed_offset_xz, voxel.rs:1163-1167
    int16_t *heights;     // vx * vz column heights
};

__global__ void k_heights(GenArgs g) {
    const Dims &d = g.w.d;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)d.vx * d.vz) return;
    const int32_t x = (int32_t)(i % d.vx), z = (int32_t)(i / d.vx);
    const float fx = (float)x + g.off_x, fz = (float)z + g.off_z;
    const float n = fbm_2d(fx * g.t.inv_wavelength, fz * g.t.inv_wavelength, g.t.octaves);
    int32_t h = f2i(floorf(g.t.base_height + g.t.amplitude * n));
    if (h < 1) h = 1;
    if (h > d.vy - 1) h = d.vy - 1;
    g.heights[i] = (int16_t)h;
}

// One thread per brick: 64 voxels from the column heights + cave noise.
__global__ void k_gen_bricks(GenArgs g) {
    const Dims &d = g.w.d;
    const int64_t bi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (bi >= d.n_bricks) return;
    const int32_t bx = (int32_t)(bi % d.bx);
    const int32_t by = (int32_t)((bi / d.bx) % d.by);
    const int32_t bz = (int32_t)(bi / ((int64_t)d.bx * d.by));
    uint64_t occ = 0;
    uint32_t words[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) words[k] = 0;
    const float cinv = g.t.cave_inv_wavelength;
    for (int lz = 0; lz < 4; ++lz) {
        for (int lx = 0; lx < 4; ++lx) {
            const int32_t x = bx * 4 + lx, z = bz * 4 + lz;
            const int32_t h = g.heights[(int64_t)z * d.vx + x];
            const float fx = (float)x + g.off_x, fz = (float)z + g.off_z;
            for (int ly = 0; ly < 4; ++ly) {
                const int32_t y = by * 4 + ly;
                uint32_t m = 0;
                if (y <= h) {
                    bool cave = false;
                    if (y > 4 && y + 3 < h)
                        cave = value_noise_3d(fx * cinv, (float)y * cinv, fz * cinv) >
                               g.t.cave_threshold;
                    if (!cave) m = (y == h) ? 2u : ((y + g.t.dirt_depth >= h) ? 3u : 4u);
                } else if (y <= g.t.water_level) {
                    m = 12u;
                }
                if (m != 0u) {
                    const int vi = child_bit(lx, ly, lz);
                    occ |= 1ull << vi;
                    // vi is not a compile-time index here; build the word by shifts
                    const int wi = vi >> 2, sh = (vi & 3) * 8;
#pragma unroll
                    for (int k = 0; k < 16; ++k)
                        if (k == wi) words[k] |= m << sh;
                }
            }
        }
    }
    g.w.occ[bi] = occ;
    uint4 *row = reinterpret_cast<uint4 *>(g.w.mat + bi * 64);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        row[k] = make_uint4(words[4 * k], words[4 * k + 1], words[4 * k + 2], words[4 * k + 3]);
    uint8_t u = 0;
    if (occ == ~0ull) {
        const uint32_t m0 = words[0] & 0xFFu;
        const uint32_t rep = 0x01010101u * m0;
        bool same = m0 != 0u;
#pragma unroll
        for (int k = 0; k < 16; ++k) same = same && (words[k] == rep);
        u = same ? (uint8_t)m0 : 0;
    }
    g.w.brick_uniform[bi] = u;
}

// ------------------------------------------------------------- pyramid
// tile word + tile LUT from the 64 child bricks (voxel.rs:253-272, :964-972)
__device__ void build_tile(const DevWorld &w, int64_t ti) {
    const Dims &d = w.d;
    const int32_t tx = (int32_t)(ti % d.tx);
    const int32_t ty = (int32_t)((ti / d.tx) % d.ty);
    const int32_t tz = (int32_t)(ti / ((int64_t)d.tx * d.ty));
    uint64_t mask = 0;
    const int64_t b0 = (int64_t)(tx * 4) + (int64_t)(ty * 4) * d.bx + (int64_t)(tz * 4) * d.bx * d.by;
    const uint8_t m0 = w.brick_uniform[b0];
    bool uni = m0 != 0;
    for (int lz = 0; lz < 4; ++lz)
        for (int ly = 0; ly < 4; ++ly)
            for (int lx = 0; lx < 4; ++lx) {
                const int64_t bi = b0 + lx + (int64_t)ly * d.bx + (int64_t)lz * d.bx * d.by;
                if (w.occ[bi] != 0ull) mask |= 1ull << child_bit(lx, ly, lz);
                uni = uni && (w.brick_uniform[bi] == m0);
            }
    w.tile_mask[ti] = mask;
    w.tile_uniform[ti] = uni ? m0 : 0;
}

// chunk word from its (up to 64) child tiles (voxel.rs:973-981)
__device__ void build_chunk(const DevWorld &w, int64_t ci) {
    const Dims &d = w.d;
    const int32_t cx = (int32_t)(ci % d.cx);
    const int32_t cy = (int32_t)((ci / d.cx) % d.cy);
    const int32_t cz = (int32_t)(ci / ((int64_t)d.cx * d.cy));
    uint64_t mask = 0;
    for (int lz = 0; lz < 4; ++lz)
        for (int ly = 0; ly < 4; ++ly)
            for (int lx = 0; lx < 4; ++lx) {
                const int32_t tx = cx * 4 + lx, ty = cy * 4 + ly, tz = cz * 4 + lz;
                if (tx >= d.tx || ty >= d.ty || tz >= d.tz) continue;
                const int64_t ti = tx + (int64_t)ty * d.tx + (int64_t)tz * d.tx * d.ty;
                if (w.tile_mask[ti] != 0ull) mask |= 1ull << child_bit(lx, ly, lz);
            }
    w.chunk_mask[ci] = mask;
}

// L4 word from its child chunks (voxel.rs:982-990)
__device__ void build_l4(const DevWorld &w, int64_t li) {
    const Dims &d = w.d;
    const int32_t x = (int32_t)(li % d.lx);
    const int32_t y = (int32_t)((li / d.lx) % d.ly);
    const int32_t z = (int32_t)(li / ((int64_t)d.lx * d.ly));
    uint64_t mask = 0;
    for (int lz = 0; lz < 4; ++lz)
        for (int ly = 0; ly < 4; ++ly)
            for (int lx = 0; lx < 4; ++lx) {
                const int32_t cx = x * 4 + lx, cy = y * 4 + ly, cz = z * 4 + lz;
                if (cx >= d.cx || cy >= d.cy || cz >= d.cz) continue;
                const int64_t ci = cx + (int64_t)cy * d.cx + (int64_t)cz * d.cx * d.cy;
                if (w.chunk_mask[ci] != 0ull) mask |= 1ull << child_bit(lx, ly, lz);
            }
    w.l4_mask[li] = mask;
}

__global__ void k_build_tiles(DevWorld w) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < w.d.n_tiles) build_tile(w, i);
}
__global__ void k_build_chunks(DevWorld w) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < w.d.n_chunks) build_chunk(w, i);
}
__global__ void k_build_l4(DevWorld w) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < w.d.n_l4) build_l4(w, i);
}

// ------------------------------------------------------------- dirty
__device__ __forceinline__ void scatter_brick(const DevWorld &w, int64_t bi, const VxBrick *b) {
    const uint2 *src = reinterpret_cast<const uint2 *>(b);
    const uint2 o = src[0];
    const uint64_t occ = (uint64_t)o.x | ((uint64_t)o.y << 32);
    w.occ[bi] = occ;
    uint2 *dst = reinterpret_cast<uint2 *>(w.mat + bi * 64);
#pragma unroll
    for (int k = 0; k < 8; ++k) dst[k] = src[1 + k];
    w.brick_uniform[bi] = uniform_of(occ, reinterpret_cast<const uint8_t *>(src + 1));
}

__global__ void k_dirty_scatter(DevWorld w, const uint32_t *__restrict__ idx,
                                const VxBrick *__restrict__ bricks, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    scatter_brick(w, idx[i], bricks + i);
}

// Duplicate brick indices in one update, last entry wins: each entry claims
// its brick with its position + 1 (the largest wins), only the winner writes,
// and the claims are cleared again once the update's kernels are done.
__global__ void k_dirty_claim(uint32_t *__restrict__ win, const uint32_t *__restrict__ idx,
                              size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    atomicMax(win + idx[i], (uint32_t)(i + 1));
}
__global__ void k_dirty_scatter_last(DevWorld w, const uint32_t *__restrict__ win,
                                     const uint32_t *__restrict__ idx,
                                     const VxBrick *__restrict__ bricks, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t bi = idx[i];
    if (win[bi] != (uint32_t)(i + 1)) return;
    scatter_brick(w, bi, bricks + i);
}
__global__ void k_dirty_release(uint32_t *__restrict__ win, const uint32_t *__restrict__ idx,
                                size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    win[idx[i]] = 0u;
}

// Each dirty brick re-derives its parent word; threads that share a parent
// write the same value (computed from data finished by the previous launch).
__global__ void k_dirty_tiles(DevWorld w, const uint32_t *__restrict__ idx, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Dims &d = w.d;
    const int64_t bi = idx[i];
    const int32_t bx = (int32_t)(bi % d.bx), by = (int32_t)((bi / d.bx) % d.by),
                  bz = (int32_t)(bi / ((int64_t)d.bx * d.by));
    build_tile(w, (bx / 4) + (int64_t)(by / 4) * d.tx + (int64_t)(bz / 4) * d.tx * d.ty);
}
__global__ void k_dirty_chunks(DevWorld w, const uint32_t *__restrict__ idx, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Dims &d = w.d;
    const int64_t bi = idx[i];
    const int32_t bx = (int32_t)(bi % d.bx), by = (int32_t)((bi / d.bx) % d.by),
                  bz = (int32_t)(bi / ((int64_t)d.bx * d.by));
    build_chunk(w, (bx / 16) + (int64_t)(by / 16) * d.cx + (int64_t)(bz / 16) * d.cx * d.cy);
}
__global__ void k_dirty_l4(DevWorld w, const uint32_t *__restrict__ idx, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Dims &d = w.d;
    const int64_t bi = idx[i];
    const int32_t bx = (int32_t)(bi % d.bx), by = (int32_t)((bi / d.bx) % d.by),
                  bz = (int32_t)(bi / ((int64_t)d.bx * d.by));
    build_l4(w, (bx / 64) + (int64_t)(by / 64) * d.lx + (int64_t)(bz / 64) * d.lx * d.ly);
}

// Persistent edits (apply_edit / replay_edits_for_chunk, voxel.rs:448-474,
// :571-603): edit i sets voxel (ed[i].y & 63) of brick ed[i].x to material
// ed[i].y >> 8, Brick::set semantics (voxel.rs:315-325: material 0 clears the
// occupancy bit).  The edits of one batch name distinct voxels; several may
// share a brick, so the occupancy word is updated atomically.
__global__ void k_edit_voxels(DevWorld w, const uint2 *__restrict__ ed, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint2 e = ed[i];
    const uint32_t vi = e.y & 63u, mat = e.y >> 8;
    w.mat[(size_t)e.x * 64u + vi] = (uint8_t)mat;
    unsigned long long *occ = reinterpret_cast<unsigned long long *>(w.occ + e.x);
    if (mat != 0u) atomicOr(occ, 1ull << vi);
    else atomicAnd(occ, ~(1ull << vi));
}
// the uniform byte of each edited brick, once all its voxels are written
__global__ void k_edit_uniform(DevWorld w, const uint32_t *__restrict__ idx, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t bi = idx[i];
    w.brick_uniform[bi] = uniform_of(w.occ[bi], w.mat + bi * 64);
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_edits(const DevWorld &w, const uint2 *ed, size_t n_edits, const uint32_t *idx,
                         size_t n_bricks, cudaStream_t s) {
    if (n_edits == 0) return cudaSuccess;
    k_edit_voxels<<<blocks_for((int64_t)n_edits, 128), 128, 0, s>>>(w, ed, n_edits);
    const unsigned b = blocks_for((int64_t)n_bricks, 128);
    k_edit_uniform<<<b, 128, 0, s>>>(w, idx, n_bricks);
    k_dirty_tiles<<<b, 128, 0, s>>>(w, idx, n_bricks);
    k_dirty_chunks<<<b, 128, 0, s>>>(w, idx, n_bricks);
    k_dirty_l4<<<b, 128, 0, s>>>(w, idx, n_bricks);
    return launch_tile_meta(w, s);
}

cudaError_t launch_bricks_from_aos(const DevWorld &w, const VxBrick *aos, int64_t first,
                                   int64_t count, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    k_aos_to_soa<<<blocks_for(count, 256), 256, 0, s>>>(w, aos, first, count);
    return cudaGetLastError();
}

cudaError_t launch_bricks_to_aos(const DevWorld &w, VxBrick *aos, int64_t first, int64_t count,
                                 cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    k_soa_to_aos<<<blocks_for(count, 256), 256, 0, s>>>(w, aos, first, count);
    return cudaGetLastError();
}

cudaError_t launch_rebuild_pyramid(const DevWorld &w, cudaStream_t s) {
    k_build_tiles<<<blocks_for(w.d.n_tiles, 128), 128, 0, s>>>(w);
    k_build_chunks<<<blocks_for(w.d.n_chunks, 128), 128, 0, s>>>(w);
    k_build_l4<<<blocks_for(w.d.n_l4, 128), 128, 0, s>>>(w);
    return launch_tile_meta(w, s);
}



cudaError_t launch_generate(const DevWorld &w, const VxTerrainParams &t, int16_t *heights,
                            cudaStream_t s) {
    GenArgs g;
    g.w = w;
    g.t = t;
    // seed_offset_xz, voxel.rs:1163-1167 (same float ops as the device would do)
    const float hi = (float)(int32_t)(uint32_t)(t.seed >> 32);
    const float lo = (float)(int32_t)(uint32_t)(t.seed & 0xFFFFFFFFull);
    g.off_x = hi * 0.01734f;
    g.off_z = lo * 0.02153f;
    g.heights = heights;
    k_heights<<<blocks_for((int64_t)w.d.vx * w.d.vz, 256), 256, 0, s>>>(g);
    k_gen_bricks<<<blocks_for(w.d.n_bricks, 128), 128, 0, s>>>(g);
    return launch_rebuild_pyramid(w, s);
}

cudaError_t launch_apply_dirty_last_wins(const DevWorld &w, uint32_t *win, const uint32_t *idx,
                                         const VxBrick *bricks, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const unsigned b = blocks_for((int64_t)n, 128);
    k_dirty_claim<<<b, 128, 0, s>>>(win, idx, n);
    k_dirty_scatter_last<<<b, 128, 0, s>>>(w, win, idx, bricks, n);
    k_dirty_release<<<b, 128, 0, s>>>(win, idx, n);
    k_dirty_tiles<<<b, 128, 0, s>>>(w, idx, n);
    k_dirty_chunks<<<b, 128, 0, s>>>(w, idx, n);
    k_dirty_l4<<<b, 128, 0, s>>>(w, idx, n);
    return launch_tile_meta(w, s);
}

cudaError_t launch_apply_dirty(const DevWorld &w, const uint32_t *idx, const VxBrick *bricks,
                               size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const unsigned b = blocks_for((int64_t)n, 128);
    k_dirty_scatter<<<b, 128, 0, s>>>(w, idx, bricks, n);
    k_dirty_tiles<<<b, 128, 0, s>>>(w, idx, n);
    k_dirty_chunks<<<b, 128, 0, s>>>(w, idx, n);
    k_dirty_l4<<<b, 128, 0, s>>>(w, idx, n);
    return launch_tile_meta(w, s);
}

}  // namespace vx
