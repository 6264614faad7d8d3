// vx_mlp_infer.cuh -- inference of the learned start-distance proposal's
// network (70 -> 64 -> 64 -> 64 -> 1, GELU), shared by vx_mlp.cu and the
// learned form's pre-pass (vx_learned.cu).
//
//   BF16 tensor cores (mma.sync m16n8k16, FP32 accumulation); one warp per
//   16 rays, the three hidden layers chained in registers (the accumulators
//   of two n8 tiles, packed to bf16x2, are the A operand of one k16 tile);
//   GELU in f32 with the approximate tanh; weights staged in shared memory
//   with padded rows (conflict-free B fragments).
//
// Features (80 columns, 70 used): origin mod 64 / 64 (3), direction (3), the
// 64 child bits of the origin chunk's tile mask (bit x + z*4 + y*16 of
// chunk_mask, src/voxel.rs:282-294), 10 zero columns.  The proposal only
// decides where a ray may restart inside its proven segment; records never
// depend on its value.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "vx_internal.h"

namespace vx {
namespace {

constexpr int kIn = kMlpIn, kH = kMlpHidden;
constexpr int kW1 = 0, kB1 = kW1 + kH * kIn, kW2 = kB1 + kH, kB2 = kW2 + kH * kH,
              kW3 = kB2 + kH, kB3 = kW3 + kH * kH, kWo = kB3 + kH, kBo = kWo + kH;
static_assert(kBo + 1 == kMlpFloats, "parameter layout");
// padded bf16 rows of the inference copy (stride in elements)
constexpr int kS1 = kIn + 8, kS2 = kH + 8;
constexpr int kW16 = kH * kS1 + 2 * kH * kS2;

__device__ __forceinline__ float feature(const float o[3], const float d[3], uint64_t mask,
                                         int col) {
    if (col < 3) return (o[col] - 64.0f * floorf(o[col] * (1.0f / 64.0f))) * (1.0f / 64.0f);
    if (col < 6) return d[col - 3];
    if (col < 70) return (float)((mask >> (col - 6)) & 1ull);
    return 0.0f;
}

// tile bits of the chunk holding the origin (slot coordinates; 0 outside the window)
__device__ __forceinline__ uint64_t origin_chunk_word(const DevWorld &w, const int32_t ro[3],
                                                      const float o[3]) {
    const Dims &d = w.d;
    const float fx = floorf(o[0]), fy = floorf(o[1]), fz = floorf(o[2]);
    if (!(fx >= -1.0e9f && fx <= 1.0e9f && fy >= -1.0e9f && fy <= 1.0e9f && fz >= -1.0e9f &&
          fz <= 1.0e9f))
        return 0ull;
    const int32_t vx = (int32_t)fx, vy = (int32_t)fy, vz = (int32_t)fz;
    if ((uint32_t)(vx - ro[0]) >= (uint32_t)d.vx || (uint32_t)(vy - ro[1]) >= (uint32_t)d.vy ||
        (uint32_t)(vz - ro[2]) >= (uint32_t)d.vz)
        return 0ull;
    const int32_t sx = ((vx % d.vx) + d.vx) % d.vx, sz = ((vz % d.vz) + d.vz) % d.vz;
    if (vy < 0 || vy >= d.vy) return 0ull;
    const int64_t ci = (sx >> 6) + (int64_t)(vy >> 6) * d.cx + (int64_t)(sz >> 6) * d.cx * d.cy;
    return __ldg(w.chunk_mask + ci);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// GELU (tanh form) in f32 with the approximate tanh: 0.5x + 0.5x tanh(u),
// u = x (k0 + k1 x^2).  (bf16 arithmetic here loses the negative tail to
// cancellation in 1 + tanh(u).)
__device__ __forceinline__ float gelu_fast(float x) {
    const float u = x * fmaf(0.0356774081f, x * x, 0.7978845608f);
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
    const float hx = 0.5f * x;
    return fmaf(hx, t, hx);
}
__device__ __forceinline__ uint32_t gelu2(float lo, float hi) {
    return pack_bf16(gelu_fast(lo), gelu_fast(hi));
}

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

struct InferArgs {
    const __nv_bfloat16 *w;  // padded bf16 W1 | W2 | W3
    const float *f32;        // f32 parameters (biases, output layer)
    const float *feats;      // n x 80 features, or nullptr = camera rays
    VxCamera cam;
    uint32_t W, n;
    uint32_t blk_w, blk_h, bw;  // camera rays: one per blk_w x blk_h pixels, bw blocks per row
    DevWorld world;
    int32_t ro[3];
    float *out;              // n: predicted log t
};

// camera ray through the centre of pixel block r (approximate
// normalization: features only)
__device__ __forceinline__ void camera_ray(const InferArgs &a, uint32_t r, float o[3], float d[3]) {
    const VxCamera &c = a.cam;
    const uint32_t px = (r % a.bw) * a.blk_w, py = (r / a.bw) * a.blk_h;
    const float u = (((float)px + 0.5f * (float)a.blk_w) + c.jitter_x) / c.res_x;
    const float v = (((float)py + 0.5f * (float)a.blk_h) + c.jitter_y) / c.res_y;
    const float ax = (u * 2.0f - 1.0f) * c.tan_half_fov * (c.res_x / c.res_y);
    const float by = (1.0f - v * 2.0f) * c.tan_half_fov;
    const float x = (c.forward[0] + c.right[0] * ax) + c.up[0] * by;
    const float y = (c.forward[1] + c.right[1] * ax) + c.up[1] * by;
    const float z = (c.forward[2] + c.right[2] * ax) + c.up[2] * by;
    const float inv = rsqrtf(x * x + y * y + z * z);
    o[0] = c.origin[0]; o[1] = c.origin[1]; o[2] = c.origin[2];
    d[0] = x * inv; d[1] = y * inv; d[2] = z * inv;
}

// One warp = 16 rays per pass: lane g = lane/4 owns rays g and g+8 of the
// pass, t = lane%4 the fragment columns 2t, 2t+1, 2t+8, 2t+9 of a k16 tile.
// FRAME: camera rays of one frame.  Their origin features are the same for
// every ray, so layer 1 is folded to z1 = c1 + W1[:, 3:6] . dir with
// c1 = b1 + W1[:, 0:3] . origin features + W1[:, 6:70] . tile bits, computed
// once per CTA in f32.
// The body of the inference kernel for CTA `cta` of `ctas` (128 threads):
// used by k_mlp_infer and by the learned form's pre-pass, whose grid holds
// other CTAs too.
template <bool FRAME>
__device__ __forceinline__ void mlp_infer_body(const InferArgs &a, uint32_t cta, uint32_t ctas) {
    __shared__ __align__(16) __nv_bfloat16 sw[kW16];
    __shared__ float4 l1[kH];   // FRAME: (W1[j][3], W1[j][4], W1[j][5], c1[j])
    // stage the bf16 weights: 16-byte loads, all of a thread's issued before
    // any is stored (kW16 * 2 bytes is a multiple of 16)
    {
        constexpr int kVec = kW16 * 2 / 16, kPer = (kVec + 127) / 128;
        static_assert(kW16 * 2 % 16 == 0, "16-byte staging");
        const uint4 *src = reinterpret_cast<const uint4 *>(a.w);
        uint4 *dst = reinterpret_cast<uint4 *>(sw);
        uint4 v[kPer];
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int idx = (int)threadIdx.x + 128 * q;
            if (idx < kVec) v[q] = __ldg(src + idx);
        }
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
            const int idx = (int)threadIdx.x + 128 * q;
            if (idx < kVec) dst[idx] = v[q];
        }
    }
    if (FRAME) {
        // camera frames: layer 1's constant terms, two threads per hidden
        // unit j (origin features and tile bits split between them)
        const int j = (int)(threadIdx.x >> 1), half = (int)(threadIdx.x & 1u);
        const float o[3] = {a.cam.origin[0], a.cam.origin[1], a.cam.origin[2]};
        const float zd[3] = {0.f, 0.f, 0.f};
        const uint64_t m = origin_chunk_word(a.world, a.ro, o);
        const float *w1r = a.f32 + kW1 + j * kIn;
        float c = 0.0f;
#pragma unroll
        for (int q = 0; q < 35; ++q) {
            const int col = half + 2 * q;  // 0..69
            if (col < 3 || col >= 6) c += __ldg(w1r + col) * feature(o, zd, m, col);
        }
        c += __shfl_xor_sync(0xFFFFFFFFu, c, 1);
        if (half == 0) l1[j] = make_float4(__ldg(w1r + 3), __ldg(w1r + 4), __ldg(w1r + 5),
                                           c + __ldg(a.f32 + kB1 + j));
    }
    __syncthreads();
    const __nv_bfloat16 *w1 = sw, *w2 = sw + kH * kS1, *w3 = w2 + kH * kS2;
    const uint32_t lane = threadIdx.x & 31u, g = lane >> 2, t = lane & 3u;
    const uint32_t warps = ctas * (blockDim.x >> 5);
    const uint32_t passes = (a.n + 15u) / 16u;
    for (uint32_t pass = cta * (blockDim.x >> 5) + (threadIdx.x >> 5); pass < passes;
         pass += warps) {
        const uint32_t r0 = pass * 16u + g, r1 = r0 + 8u;
        const bool v0 = r0 < a.n, v1 = r1 < a.n;
        float C[8][4];
        if (FRAME) {
            float o[3], d0[3] = {0, 0, 0}, d1[3] = {0, 0, 0};
            if (v0) camera_ray(a, r0, o, d0);
            if (v1) camera_ray(a, r1, o, d1);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const float4 q0 = l1[nt * 8 + 2 * t], q1 = l1[nt * 8 + 2 * t + 1];
                C[nt][0] = q0.w + q0.x * d0[0] + q0.y * d0[1] + q0.z * d0[2];
                C[nt][1] = q1.w + q1.x * d0[0] + q1.y * d0[1] + q1.z * d0[2];
                C[nt][2] = q0.w + q0.x * d1[0] + q0.y * d1[1] + q0.z * d1[2];
                C[nt][3] = q1.w + q1.x * d1[0] + q1.y * d1[1] + q1.z * d1[2];
            }
        } else {
            uint32_t A[5][4];
            const float *p0 = a.feats + (size_t)(v0 ? r0 : 0) * kIn;
            const float *p1 = a.feats + (size_t)(v1 ? r1 : 0) * kIn;
#pragma unroll
            for (int kt = 0; kt < 5; ++kt) {
                const int c0 = kt * 16 + 2 * (int)t, c1 = c0 + 8;
                const float2 z2 = make_float2(0.f, 0.f);
                const float2 f00 = v0 ? *reinterpret_cast<const float2 *>(p0 + c0) : z2;
                const float2 f10 = v1 ? *reinterpret_cast<const float2 *>(p1 + c0) : z2;
                const float2 f01 = v0 ? *reinterpret_cast<const float2 *>(p0 + c1) : z2;
                const float2 f11 = v1 ? *reinterpret_cast<const float2 *>(p1 + c1) : z2;
                A[kt][0] = pack_bf16(f00.x, f00.y);
                A[kt][1] = pack_bf16(f10.x, f10.y);
                A[kt][2] = pack_bf16(f01.x, f01.y);
                A[kt][3] = pack_bf16(f11.x, f11.y);
            }
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const float b0 = a.f32[kB1 + nt * 8 + 2 * t], b1 = a.f32[kB1 + nt * 8 + 2 * t + 1];
                C[nt][0] = b0; C[nt][1] = b1; C[nt][2] = b0; C[nt][3] = b1;
                const __nv_bfloat16 *wr = w1 + (nt * 8 + g) * kS1 + 2 * t;
#pragma unroll
                for (int kt = 0; kt < 5; ++kt)
                    mma_bf16(C[nt], A[kt], *reinterpret_cast<const uint32_t *>(wr + kt * 16),
                             *reinterpret_cast<const uint32_t *>(wr + kt * 16 + 8));
            }
        }
#pragma unroll
        for (int layer = 0; layer < 2; ++layer) {
            const __nv_bfloat16 *wl = layer == 0 ? w2 : w3;
            const int boff = layer == 0 ? kB2 : kB3;
            uint32_t Hf[4][4];
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                Hf[kt][0] = gelu2(C[2 * kt][0], C[2 * kt][1]);
                Hf[kt][1] = gelu2(C[2 * kt][2], C[2 * kt][3]);
                Hf[kt][2] = gelu2(C[2 * kt + 1][0], C[2 * kt + 1][1]);
                Hf[kt][3] = gelu2(C[2 * kt + 1][2], C[2 * kt + 1][3]);
            }
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const float b0 = a.f32[boff + nt * 8 + 2 * t], b1 = a.f32[boff + nt * 8 + 2 * t + 1];
                C[nt][0] = b0; C[nt][1] = b1; C[nt][2] = b0; C[nt][3] = b1;
                const __nv_bfloat16 *wr = wl + (nt * 8 + g) * kS2 + 2 * t;
#pragma unroll
                for (int kt = 0; kt < 4; ++kt)
                    mma_bf16(C[nt], Hf[kt], *reinterpret_cast<const uint32_t *>(wr + kt * 16),
                             *reinterpret_cast<const uint32_t *>(wr + kt * 16 + 8));
            }
        }
        // output: GELU(h3) . wo + bo, reduced over the four lanes of a quad
        float y0 = 0.f, y1 = 0.f;
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const float wa = a.f32[kWo + nt * 8 + 2 * t], wb = a.f32[kWo + nt * 8 + 2 * t + 1];
            y0 += gelu_fast(C[nt][0]) * wa + gelu_fast(C[nt][1]) * wb;
            y1 += gelu_fast(C[nt][2]) * wa + gelu_fast(C[nt][3]) * wb;
        }
        y0 += __shfl_xor_sync(0xFFFFFFFFu, y0, 1);
        y0 += __shfl_xor_sync(0xFFFFFFFFu, y0, 2);
        y1 += __shfl_xor_sync(0xFFFFFFFFu, y1, 1);
        y1 += __shfl_xor_sync(0xFFFFFFFFu, y1, 2);
        if (t == 0) {
            if (v0) a.out[r0] = y0 + a.f32[kBo];
            if (v1) a.out[r1] = y1 + a.f32[kBo];
        }
    }
}


}  // namespace
}  // namespace vx
