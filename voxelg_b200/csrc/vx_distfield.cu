// vx_distfield.cu -- empty-space distance fields over the world pyramid, for
// the learned form's verification walk (vx_learned.cu).
//
// For every brick (and, separately, every tile) the Chebyshev distance, in
// cells of that level, to the nearest non-empty cell: 0 for a non-empty cell,
// k when every cell within Chebyshev distance k-1 is empty and one at
// distance k is not, and R+1 when all cells within R are empty (the cap).
// Distances are taken in slot space: toroidal in x and z (the loaded window
// covers every slot exactly once, so the toroidal distance between two
// window cells is never more than their distance in the world, and a value
// read here is conservative for every window cell), clamped in y (cells
// outside the y range count as empty: the traversal ends there).
//
// The L-infinity distance transform is separable:
//   f1(x,y,z) = min over occupied (x',y,z)            of |x - x'|
//   f2(x,y,z) = min over z'  of max(|z - z'|, f1(x,y,z'))
//   f3(x,y,z) = min over y'  of max(|y - y'|, f2(x,y',z))
// so three 1-D passes give it exactly; each pass scans outward from the
// cell and stops once the distance scanned reaches the best value found.
// Integer work only.  A brick is non-empty when its occupancy word is
// nonzero, a tile when its tile_mask word is (src/voxel.rs:282-335).
#include <cuda_runtime.h>

#include "vx_internal.h"

namespace vx {
namespace {

struct Grid {
    int32_t nx, ny, nz;
};

__device__ __forceinline__ int32_t wrap(int32_t v, int32_t n) {
    return v < 0 ? v + n : (v >= n ? v - n : v);
}

// pass along x from the occupancy words: distance to the nearest nonzero word
__global__ void k_df_x(const uint64_t *__restrict__ occ, uint8_t *__restrict__ out, Grid g,
                       int32_t cap) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)g.nx * g.ny * g.nz;
    if (i >= n) return;
    const int32_t x = (int32_t)(i % g.nx);
    const int64_t row = i - x;
    int32_t best = cap + 1;
    const int32_t reach = min(cap, g.nx / 2);
    for (int32_t k = 0; k <= reach && k < best; ++k) {
        if (__ldg(occ + row + wrap(x + k, g.nx)) != 0ull ||
            __ldg(occ + row + wrap(x - k, g.nx)) != 0ull)
            best = k;
    }
    out[i] = (uint8_t)best;
}

// pass along z (toroidal, AXIS 2) or y (clamped, AXIS 1) over distances
template <int AXIS>
__global__ void k_df_pass(const uint8_t *__restrict__ in, uint8_t *__restrict__ out, Grid g,
                          int32_t cap) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)g.nx * g.ny * g.nz;
    if (i >= n) return;
    const int32_t y = (int32_t)((i / g.nx) % g.ny);
    const int32_t z = (int32_t)(i / ((int64_t)g.nx * g.ny));
    const int64_t stride = AXIS == 2 ? (int64_t)g.nx * g.ny : (int64_t)g.nx;
    const int32_t c = AXIS == 2 ? z : y, len = AXIS == 2 ? g.nz : g.ny;
    const int64_t base = i - (int64_t)c * stride;
    int32_t best = __ldg(in + i);
    const int32_t reach = AXIS == 2 ? min(cap, g.nz / 2) : cap;
    for (int32_t k = 1; k <= reach && k < best; ++k) {
        int32_t a = c + k, b = c - k;
        int32_t va = cap + 1, vb = cap + 1;
        if (AXIS == 2) {
            va = __ldg(in + base + (int64_t)wrap(a, len) * stride);
            vb = __ldg(in + base + (int64_t)wrap(b, len) * stride);
        } else {
            if (a < len) va = __ldg(in + base + (int64_t)a * stride);
            if (b >= 0) vb = __ldg(in + base + (int64_t)b * stride);
        }
        const int32_t m = max(k, min(va, vb));
        if (m < best) best = m;
    }
    out[i] = (uint8_t)best;
}

inline unsigned blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

cudaError_t field(const uint64_t *occ, uint8_t *out, uint8_t *tmp, Grid g, int32_t cap,
                  cudaStream_t s) {
    const int64_t n = (int64_t)g.nx * g.ny * g.nz;
    if (n == 0) return cudaSuccess;
    k_df_x<<<blocks(n), 256, 0, s>>>(occ, out, g, cap);
    k_df_pass<2><<<blocks(n), 256, 0, s>>>(out, tmp, g, cap);
    k_df_pass<1><<<blocks(n), 256, 0, s>>>(tmp, out, g, cap);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_dist_fields(const DevWorld &w, uint8_t *bdf, uint8_t *tdf, uint8_t *tmp,
                               cudaStream_t s) {
    cudaError_t e = field(w.occ, bdf, tmp, Grid{w.d.bx, w.d.by, w.d.bz}, kBrickFieldCap, s);
    if (e != cudaSuccess) return e;
    return field(w.tile_mask, tdf, tmp, Grid{w.d.tx, w.d.ty, w.d.tz}, kTileFieldCap, s);
}

}  // namespace vx
