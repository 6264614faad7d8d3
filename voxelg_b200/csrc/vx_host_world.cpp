// vx_host_world.cpp -- host mirror of voxelG's World core (src/voxel.rs) for
// C/C++ callers of libvoxrt: the arrays in the reference's host layout, the
// incremental mask/LUT maintenance of set_voxel, the toroidal apply_edit and
// the dirty-brick list that vx_world_sync turns into a device update
// (the role Renderer::upload_world plays in src/renderer.rs:1248-1394).
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "vx_internal.h"

struct VxHostWorld {
    vx::Dims d;
    std::vector<VxBrick> bricks;
    std::vector<uint64_t> tile_mask, chunk_mask, l4_mask;
    std::vector<uint8_t> brick_uniform, tile_uniform;
    std::vector<uint32_t> dirty;
    bool all_dirty = true;
};

namespace {

inline int child_bit(int32_t lx, int32_t ly, int32_t lz) { return lx + lz * 4 + ly * 16; }
inline int64_t brick_idx(const vx::Dims &d, int32_t x, int32_t y, int32_t z) {
    return (int64_t)x + (int64_t)y * d.bx + (int64_t)z * d.bx * d.by;
}
inline int64_t tile_idx(const vx::Dims &d, int32_t x, int32_t y, int32_t z) {
    return (int64_t)x + (int64_t)y * d.tx + (int64_t)z * d.tx * d.ty;
}
inline int64_t chunk_idx(const vx::Dims &d, int32_t x, int32_t y, int32_t z) {
    return (int64_t)x + (int64_t)y * d.cx + (int64_t)z * d.cx * d.cy;
}
inline int64_t l4_idx(const vx::Dims &d, int32_t x, int32_t y, int32_t z) {
    return (int64_t)x + (int64_t)y * d.lx + (int64_t)z * d.lx * d.ly;
}

// brick_uniform_of, voxel.rs:233-247
uint8_t brick_uniform_of(const VxBrick &b) {
    if (b.occupancy != ~0ull) return 0;
    const uint8_t m0 = b.materials[0];
    if (m0 == 0) return 0;
    for (int i = 1; i < 64; ++i)
        if (b.materials[i] != m0) return 0;
    return m0;
}

// tile_uniform_of, voxel.rs:253-272
uint8_t tile_uniform_of(const VxHostWorld &h, int64_t ti) {
    const vx::Dims &d = h.d;
    const int32_t tx = (int32_t)(ti % d.tx), ty = (int32_t)((ti / d.tx) % d.ty),
                  tz = (int32_t)(ti / ((int64_t)d.tx * d.ty));
    const uint8_t m0 = h.brick_uniform[brick_idx(d, tx * 4, ty * 4, tz * 4)];
    if (m0 == 0) return 0;
    for (int dz = 0; dz < 4; ++dz)
        for (int dy = 0; dy < 4; ++dy)
            for (int dx = 0; dx < 4; ++dx)
                if (h.brick_uniform[brick_idx(d, tx * 4 + dx, ty * 4 + dy, tz * 4 + dz)] != m0)
                    return 0;
    return m0;
}

// refresh_masks_for_brick, voxel.rs:879-914
void refresh_masks_for_brick(VxHostWorld &h, int32_t bx, int32_t by, int32_t bz) {
    const vx::Dims &d = h.d;
    const bool solid = h.bricks[brick_idx(d, bx, by, bz)].occupancy != 0;
    const int32_t tx = bx / 4, ty = by / 4, tz = bz / 4;
    const int64_t ti = tile_idx(d, tx, ty, tz);
    const uint64_t bit = 1ull << child_bit(bx & 3, by & 3, bz & 3);
    const uint64_t prev = h.tile_mask[ti];
    h.tile_mask[ti] = solid ? (prev | bit) : (prev & ~bit);
    const uint64_t now = h.tile_mask[ti];
    if ((prev == 0) == (now == 0)) return;
    const int32_t cx = tx / 4, cy = ty / 4, cz = tz / 4;
    const int64_t ci = chunk_idx(d, cx, cy, cz);
    const uint64_t cbit = 1ull << child_bit(tx & 3, ty & 3, tz & 3);
    const uint64_t cprev = h.chunk_mask[ci];
    h.chunk_mask[ci] = now == 0 ? (cprev & ~cbit) : (cprev | cbit);
    const uint64_t cnow = h.chunk_mask[ci];
    if ((cprev == 0) == (cnow == 0)) return;
    const int64_t li = l4_idx(d, cx / 4, cy / 4, cz / 4);
    const uint64_t lbit = 1ull << child_bit(cx & 3, cy & 3, cz & 3);
    h.l4_mask[li] = cnow == 0 ? (h.l4_mask[li] & ~lbit) : (h.l4_mask[li] | lbit);
}

}  // namespace

extern "C" {

int vx_host_world_create(int32_t bx, int32_t by, int32_t bz, VxHostWorld **out) {
    if (!out || bx <= 0 || by <= 0 || bz <= 0 || bx % 64 || bz % 64 || by % 16) {
        vx::set_error("vx_host_world_create: bricks_x/z must be positive multiples of 64, "
                      "bricks_y a positive multiple of 16");
        return VX_ERR_INVALID;
    }
    VxHostWorld *h = new (std::nothrow) VxHostWorld();
    if (!h) return VX_ERR_OOM;
    try {
        h->d = vx::make_dims(bx, by, bz);
        VxBrick empty;
        std::memset(&empty, 0, sizeof(empty));
        h->bricks.assign((size_t)h->d.n_bricks, empty);
        h->tile_mask.assign((size_t)h->d.n_tiles, 0);
        h->chunk_mask.assign((size_t)h->d.n_chunks, 0);
        h->l4_mask.assign((size_t)h->d.n_l4, 0);
        h->brick_uniform.assign((size_t)h->d.n_bricks, 0);
        h->tile_uniform.assign((size_t)h->d.n_tiles, 0);
    } catch (...) {
        delete h;
        vx::set_error("vx_host_world_create: out of host memory");
        return VX_ERR_OOM;
    }
    *out = h;
    return VX_OK;
}

int vx_host_world_destroy(VxHostWorld *h) {
    delete h;
    return VX_OK;
}

int vx_host_world_arrays(VxHostWorld *h, VxBrick **bricks, uint64_t **tile_mask,
                         uint64_t **chunk_mask, uint64_t **l4_mask, uint8_t **brick_uniform,
                         uint8_t **tile_uniform) {
    if (!h) return VX_ERR_INVALID;
    if (bricks) *bricks = h->bricks.data();
    if (tile_mask) *tile_mask = h->tile_mask.data();
    if (chunk_mask) *chunk_mask = h->chunk_mask.data();
    if (l4_mask) *l4_mask = h->l4_mask.data();
    if (brick_uniform) *brick_uniform = h->brick_uniform.data();
    if (tile_uniform) *tile_uniform = h->tile_uniform.data();
    return VX_OK;
}

// World::set_voxel, voxel.rs:916-935 (Brick::set :309-319)
int vx_host_world_set_voxel(VxHostWorld *h, uint32_t x, uint32_t y, uint32_t z, uint8_t mat) {
    if (!h) return VX_ERR_INVALID;
    const vx::Dims &d = h->d;
    if (x >= (uint32_t)d.vx || y >= (uint32_t)d.vy || z >= (uint32_t)d.vz) return VX_OK;
    const int32_t bx = x / 4, by = y / 4, bz = z / 4;
    const int64_t bi = brick_idx(d, bx, by, bz);
    VxBrick &b = h->bricks[(size_t)bi];
    const int vi = child_bit(x % 4, y % 4, z % 4);
    const bool was_empty = b.occupancy == 0;
    if (mat == 0) {
        b.occupancy &= ~(1ull << vi);
        b.materials[vi] = 0;
    } else {
        b.occupancy |= 1ull << vi;
        b.materials[vi] = mat;
    }
    if (was_empty != (b.occupancy == 0)) refresh_masks_for_brick(*h, bx, by, bz);
    h->brick_uniform[(size_t)bi] = brick_uniform_of(b);
    const int64_t ti = tile_idx(d, bx / 4, by / 4, bz / 4);
    h->tile_uniform[(size_t)ti] = tile_uniform_of(*h, ti);
    if (!h->all_dirty) h->dirty.push_back((uint32_t)bi);  // mark_brick_dirty :871-875
    return VX_OK;
}

// World::apply_edit, voxel.rs:450-474 (toroidal slot mapping)
int vx_host_world_apply_edit(VxHostWorld *h, int32_t wx, int32_t wy, int32_t wz, uint8_t mat,
                             const int32_t origin[3]) {
    if (!h || !origin) return VX_ERR_INVALID;
    const vx::Dims &d = h->d;
    const int32_t rx = wx - origin[0], ry = wy - origin[1], rz = wz - origin[2];
    if (rx < 0 || ry < 0 || rz < 0 || rx >= d.vx || ry >= d.vy || rz >= d.vz) return VX_OK;
    const int32_t lx = ((wx % d.vx) + d.vx) % d.vx;  // rem_euclid
    const int32_t lz = ((wz % d.vz) + d.vz) % d.vz;
    return vx_host_world_set_voxel(h, (uint32_t)lx, (uint32_t)ry, (uint32_t)lz, mat);
}

// rebuild_all_masks + rebuild_all_uniform, voxel.rs:946-1000
int vx_host_world_rebuild(VxHostWorld *h) {
    if (!h) return VX_ERR_INVALID;
    const vx::Dims &d = h->d;
    std::fill(h->tile_mask.begin(), h->tile_mask.end(), 0);
    std::fill(h->chunk_mask.begin(), h->chunk_mask.end(), 0);
    std::fill(h->l4_mask.begin(), h->l4_mask.end(), 0);
    for (int32_t bz = 0; bz < d.bz; ++bz)
        for (int32_t by = 0; by < d.by; ++by)
            for (int32_t bx = 0; bx < d.bx; ++bx)
                if (h->bricks[(size_t)brick_idx(d, bx, by, bz)].occupancy != 0)
                    h->tile_mask[(size_t)tile_idx(d, bx / 4, by / 4, bz / 4)] |=
                        1ull << child_bit(bx & 3, by & 3, bz & 3);
    for (int32_t tz = 0; tz < d.tz; ++tz)
        for (int32_t ty = 0; ty < d.ty; ++ty)
            for (int32_t tx = 0; tx < d.tx; ++tx)
                if (h->tile_mask[(size_t)tile_idx(d, tx, ty, tz)] != 0)
                    h->chunk_mask[(size_t)chunk_idx(d, tx / 4, ty / 4, tz / 4)] |=
                        1ull << child_bit(tx & 3, ty & 3, tz & 3);
    for (int32_t cz = 0; cz < d.cz; ++cz)
        for (int32_t cy = 0; cy < d.cy; ++cy)
            for (int32_t cx = 0; cx < d.cx; ++cx)
                if (h->chunk_mask[(size_t)chunk_idx(d, cx, cy, cz)] != 0)
                    h->l4_mask[(size_t)l4_idx(d, cx / 4, cy / 4, cz / 4)] |=
                        1ull << child_bit(cx & 3, cy & 3, cz & 3);
    for (int64_t i = 0; i < d.n_bricks; ++i) h->brick_uniform[(size_t)i] = brick_uniform_of(h->bricks[(size_t)i]);
    for (int64_t i = 0; i < d.n_tiles; ++i) h->tile_uniform[(size_t)i] = tile_uniform_of(*h, i);
    h->all_dirty = true;
    h->dirty.clear();
    return VX_OK;
}

int64_t vx_host_world_dirty_count(VxHostWorld *h) {
    if (!h) return VX_ERR_INVALID;
    if (h->all_dirty) return h->d.n_bricks;
    std::sort(h->dirty.begin(), h->dirty.end());
    h->dirty.erase(std::unique(h->dirty.begin(), h->dirty.end()), h->dirty.end());
    return (int64_t)h->dirty.size();
}

int vx_world_sync(VxWorld *w, VxHostWorld *h, void *stream) {
    if (!w || !h) {
        vx::set_error("vx_world_sync: null argument");
        return VX_ERR_INVALID;
    }
    uint64_t counts[4];
    int rc = vx_world_counts(w, counts);
    if (rc != VX_OK) return rc;
    if (counts[0] != (uint64_t)h->d.n_bricks || counts[1] != (uint64_t)h->d.n_tiles) {
        vx::set_error("vx_world_sync: host and device world dims differ");
        return VX_ERR_INVALID;
    }
    if (h->all_dirty) {
        rc = vx_world_upload(w, h->bricks.data(), h->tile_mask.data(), h->chunk_mask.data(),
                             h->l4_mask.data(), h->brick_uniform.data(), h->tile_uniform.data());
        if (rc != VX_OK) return rc;
        h->all_dirty = false;
        h->dirty.clear();
        return VX_OK;
    }
    vx_host_world_dirty_count(h);  // sort + dedup
    if (h->dirty.empty()) return VX_OK;
    std::vector<VxBrick> payload(h->dirty.size());
    for (size_t i = 0; i < h->dirty.size(); ++i) payload[i] = h->bricks[h->dirty[i]];
    rc = vx_world_apply_dirty(w, h->dirty.data(), payload.data(), h->dirty.size(), stream);
    if (rc != VX_OK) return rc;
    h->dirty.clear();
    return VX_OK;
}

}  // extern "C"
