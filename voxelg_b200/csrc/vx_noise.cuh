// vx_noise.cuh -- the reference's value-noise primitives (src/voxel.rs
// hash2 :1172-1181, hash3 :1183-1193, smoothstep :1195-1198,
// value_noise_2d :1200-1212, fbm_2d :1220-1232, value_noise_3d :1999-2021,
// seed_offset_xz :1163-1167), shared by the terrain generators.  Users
// compile with --fmad=false so each value equals the CPU's binary32 result.
#pragma once
#include <cstdint>

namespace vx {
namespace noise {

__device__ __forceinline__ int32_t floor_i(float x) {
    x = floorf(x);
    if (x != x) return 0;
    if (x >= 1073741824.0f) return 1073741824;
    if (x <= -1073741824.0f) return -1073741824;
    return (int32_t)x;
}
// The IEEE binary32 quotient u / 16777215.0f for an integer u < 2^24,
// without a division.  u / (2^24 - 1) = u 2^-24 (1 + 2^-24 + 2^-48 + ...):
// with y the 24-bit significand of u, the quotient is (y + f) units in the
// last place of float(u) 2^-24, f = y / (2^24 - 1) in (1/2, 1), so it rounds
// to y + 1 units, still inside the binade (y + 1 < 2^24).  Hence the
// quotient is float(u) 2^-24 with its bit pattern incremented (0 for u = 0).
__device__ __forceinline__ float unit24(uint32_t u) {
    const float p = (float)u * 5.9604644775390625e-8f;   // exact: 2^-24
    return u != 0u ? __int_as_float(__float_as_int(p) + 1) : 0.0f;
}
__device__ __forceinline__ float hash2(int32_t x, int32_t z) {
    uint32_t h = (uint32_t)x * 0x9E3779B1u + (uint32_t)z * 0x85EBCA77u;
    h = h * 0xC2B2AE3Du;
    h = h ^ (h >> 16);
    h = h * 0x85EBCA6Bu;
    return unit24(h & 0xFFFFFFu) * 2.0f - 1.0f;
}
__device__ __forceinline__ float hash3(int32_t x, int32_t y, int32_t z) {
    uint32_t h = (uint32_t)x * 0x9E3779B1u + (uint32_t)y * 0x85EBCA77u + (uint32_t)z * 0xC2B2AE3Du;
    h = h * 0xD2B74407u;
    h = h ^ (h >> 16);
    h = h * 0x85EBCA6Bu;
    return unit24(h & 0xFFFFFFu) * 2.0f - 1.0f;
}
__device__ __forceinline__ float smooth(float t) { return t * t * (3.0f - 2.0f * t); }

__device__ __forceinline__ float value_noise_2d(float x, float z) {
    const int32_t xi = floor_i(x), zi = floor_i(z);
    const float xf = smooth(x - (float)xi), zf = smooth(z - (float)zi);
    const float v00 = hash2(xi, zi), v10 = hash2(xi + 1, zi);
    const float v01 = hash2(xi, zi + 1), v11 = hash2(xi + 1, zi + 1);
    const float a = v00 * (1.0f - xf) + v10 * xf;
    const float b = v01 * (1.0f - xf) + v11 * xf;
    return a * (1.0f - zf) + b * zf;
}

__device__ __forceinline__ float fbm_2d(float x, float z, uint32_t octaves) {
    float total = 0.0f, amp = 1.0f, freq = 1.0f, max_amp = 0.0f;
    for (uint32_t i = 0; i < octaves; ++i) {
        total += value_noise_2d(x * freq, z * freq) * amp;
        max_amp += amp;
        amp *= 0.5f;
        freq *= 2.0f;
    }
    return total / max_amp;
}

__device__ __forceinline__ float value_noise_3d(float x, float y, float z) {
    const int32_t xi = floor_i(x), yi = floor_i(y), zi = floor_i(z);
    const float xf = smooth(x - (float)xi), yf = smooth(y - (float)yi), zf = smooth(z - (float)zi);
    const float v000 = hash3(xi, yi, zi), v100 = hash3(xi + 1, yi, zi);
    const float v010 = hash3(xi, yi + 1, zi), v110 = hash3(xi + 1, yi + 1, zi);
    const float v001 = hash3(xi, yi, zi + 1), v101 = hash3(xi + 1, yi, zi + 1);
    const float v011 = hash3(xi, yi + 1, zi + 1), v111 = hash3(xi + 1, yi + 1, zi + 1);
    const float a = v000 * (1.0f - xf) + v100 * xf;
    const float b = v010 * (1.0f - xf) + v110 * xf;
    const float c = v001 * (1.0f - xf) + v101 * xf;
    const float d = v011 * (1.0f - xf) + v111 * xf;
    const float ab = a * (1.0f - yf) + b * yf;
    const float cd = c * (1.0f - yf) + d * yf;
    return ab * (1.0f - zf) + cd * zf;
}

// value_noise_3d(x, y, z) along a column: x and z fixed, y non-decreasing
// from call to call.  The x-interpolated corner values a, b, c, d of the
// lattice cell are kept; when the cell steps up by one in y its lower
// face's values are the previous upper face's, so four of the eight hashes
// are reused.  Each value is the one value_noise_3d computes, operation for
// operation.
struct ColumnNoise3 {
    int32_t xi, zi, yi;
    float xf, zf;        // smoothed fractions of x and z
    float a, b, c, d;    // lerp_x at (y0, z0), (y1, z0), (y0, z1), (y1, z1)

    __device__ __forceinline__ void init(float x, float z) {
        xi = floor_i(x);
        zi = floor_i(z);
        xf = smooth(x - (float)xi);
        zf = smooth(z - (float)zi);
        yi = INT32_MIN;
    }
    __device__ __forceinline__ float lerp_x(int32_t y, int32_t z) const {
        return hash3(xi, y, z) * (1.0f - xf) + hash3(xi + 1, y, z) * xf;
    }
    __device__ __forceinline__ float eval(float y) {
        const int32_t yn = floor_i(y);
        if (yn != yi) {
            if (yi != INT32_MIN && yn == yi + 1) {
                a = b;
                c = d;
            } else {
                a = lerp_x(yn, zi);
                c = lerp_x(yn, zi + 1);
            }
            b = lerp_x(yn + 1, zi);
            d = lerp_x(yn + 1, zi + 1);
            yi = yn;
        }
        const float yf = smooth(y - (float)yi);
        const float ab = a * (1.0f - yf) + b * yf;
        const float cd = c * (1.0f - yf) + d * yf;
        return ab * (1.0f - zf) + cd * zf;
    }
};

}  // namespace noise
}  // namespace vx
