// vx_pack.cu -- a frame's records and shadow records in the 16-byte
// VxPackedRecord form or the 12-byte VxCompactRecord form, for delivery to
// host memory.
//
// The pair takes 32 bytes per pixel (VxHitRecord 24, VxShadowRecord 8);
// copied to the host over PCIe it is what bounds a host-buffer frame.  The
// packed form keeps every bit a record can hold: the hit voxel relative to
// the window corner as one 32-bit index (a hit is always inside the loaded
// window, and a miss's voxel is 0, 0, 0), face / material / flags and the two
// shadow bits in one word, t, and the primary and shadow step counts in 16
// bits each (the caller bounds max_iters and any_max_iters to 65535).
//
// One thread per pixel: three 8-byte loads of the record, one of the shadow
// record, one 16-byte store; a warp touches 768 + 256 contiguous bytes and
// writes 512, so the kernel runs at HBM rate (48 bytes per pixel).
#include <cuda_runtime.h>

#include "vx_internal.h"

namespace vx {
namespace {

__global__ void __launch_bounds__(256) k_pack(const VxHitRecord *__restrict__ rec,
                                              const VxShadowRecord *__restrict__ sh,
                                              size_t first, size_t n, int32_t rox, int32_t roy,
                                              int32_t roz, uint32_t wx, uint32_t wy,
                                              VxPackedRecord *__restrict__ out) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t i = first + k;
    const uint2 *q = reinterpret_cast<const uint2 *>(rec + i);
    const uint2 a = __ldcs(q), b = __ldcs(q + 1), c = __ldcs(q + 2);
    uint32_t word = b.y;  // face | mat << 8 | flags << 16 (pad byte 0)
    uint32_t vox = 0;
    if ((word >> 16) & 1u) {
        const uint32_t rx = a.x - (uint32_t)rox, ry = a.y - (uint32_t)roy,
                       rz = b.x - (uint32_t)roz;
        vox = rx + wx * (ry + wy * rz);
    }
    uint32_t steps = c.y & 0xFFFFu;
    if (sh) {
        const uint2 s = __ldcs(reinterpret_cast<const uint2 *>(sh + i));
        word |= ((s.y & 1u) | (((s.y >> 8) & 1u) << 1)) << 24;  // occluded, traced
        steps |= s.x << 16;
    }
    __stcs(reinterpret_cast<uint4 *>(out + i), make_uint4(vox, word, c.x, steps));
}

// The 12-byte VxCompactRecord (layout in include/voxrt.h).  One thread per
// pixel, the same loads as k_pack, three 4-byte stores (a warp's 384 bytes
// are contiguous).  Any record outside what the form holds -- a negative t,
// a step count beyond 11 / 10 bits, a voxel index beyond 30 bits, a face,
// flags, pad or shadow bit the frame kernels never write -- sets
// kFaultCompactLossy in the world's fault word (host memory, read by the
// next synchronising call), so the form is lossless or reported.
__global__ void __launch_bounds__(256) k_pack_compact(const VxHitRecord *__restrict__ rec,
                                                      const VxShadowRecord *__restrict__ sh,
                                                      size_t first, size_t n, int32_t rox,
                                                      int32_t roy, int32_t roz, uint32_t wx,
                                                      uint32_t wy,
                                                      uint32_t *__restrict__ out,
                                                      uint32_t *fault) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t i = first + k;
    const uint2 *q = reinterpret_cast<const uint2 *>(rec + i);
    const uint2 a = __ldcs(q), b = __ldcs(q + 1), c = __ldcs(q + 2);
    const uint32_t face = b.y & 0xFFu, mat = (b.y >> 8) & 0xFFu, flags = (b.y >> 16) & 0xFFu;
    const bool hit = (flags & 1u) != 0u;
    uint32_t vox = 0;
    bool lossy = (b.y >> 24) != 0u || (flags & ~3u) != 0u || hit != (face != 0xFFu) ||
                 (hit && face > 5u) || (!hit && (flags != 0u || (a.x | a.y | b.x) != 0u));
    if (hit) {
        const uint32_t rx = a.x - (uint32_t)rox, ry = a.y - (uint32_t)roy,
                       rz = b.x - (uint32_t)roz;
        vox = rx + wx * (ry + wy * rz);
        lossy = lossy || vox >= (1u << 30);
    }
    uint32_t occ = 0, traced = 0, ssteps = 0;
    if (sh) {
        const uint2 sv = __ldcs(reinterpret_cast<const uint2 *>(sh + i));
        occ = sv.y & 1u;
        traced = (sv.y >> 8) & 1u;
        ssteps = sv.x;
        lossy = lossy || (sv.y & ~0x101u) != 0u || ssteps > 1023u;
    }
    const uint32_t psteps = c.y;
    lossy = lossy || (c.x >> 31) != 0u || psteps > 2047u;
    out[3 * i + 0] = (vox & 0x3FFFFFFFu) | (((flags >> 1) & 1u) << 30) | (occ << 31);
    out[3 * i + 1] = (c.x & 0x7FFFFFFFu) | (traced << 31);
    out[3 * i + 2] = (psteps & 0x7FFu) | ((ssteps & 0x3FFu) << 11) |
                     ((hit ? face : 7u) << 21) | (mat << 24);
    if (lossy && fault) {
        // every writer in this launch sets the same bit; earlier bits stay
        volatile uint32_t *f = fault;
        *f = *f | kFaultCompactLossy;
    }
}

}  // namespace

static_assert(sizeof(VxPackedRecord) == 16, "16-byte packed record");
static_assert(sizeof(VxCompactRecord) == 12, "12-byte compact record");

cudaError_t launch_pack_compact(const VxHitRecord *rec, const VxShadowRecord *sh, size_t first,
                                size_t n, const int32_t ro[3], uint32_t wx, uint32_t wy,
                                VxCompactRecord *out, uint32_t *fault, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_pack_compact<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
        rec, sh, first, n, ro[0], ro[1], ro[2], wx, wy, reinterpret_cast<uint32_t *>(out), fault);
    return cudaGetLastError();
}

cudaError_t launch_pack(const VxHitRecord *rec, const VxShadowRecord *sh, size_t first, size_t n,
                        const int32_t ro[3], uint32_t wx, uint32_t wy, VxPackedRecord *out,
                        cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_pack<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(rec, sh, first, n, ro[0], ro[1], ro[2], wx,
                                                       wy, out);
    return cudaGetLastError();
}

}  // namespace vx
