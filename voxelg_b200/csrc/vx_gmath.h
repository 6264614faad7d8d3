// vx_gmath.h -- the chunk generator's transcendentals, with the host C
// library's binary32 results.
//
// The reference's generator calls f32::powf, f32::cos and f32::sin
// (src/voxel.rs:1262 mountain height, :1623 pine canopy radius, :1639-1641
// and :1695-1697 branch ends); on Linux they are the C library's powf, cosf
// and sinf.  Those are not correctly rounded: on some inputs their binary32
// result is one unit in the last place from the nearest.  The device
// reproduces them in two parts:
//
// 1. Functions of this file, compiled identically for host and device: pow
//    (x in [0, 1], y > 0) as exp(y * log(x)), and sin / cos (|a| <= 16), in
//    double precision from IEEE +, -, *, / only (no contraction: the device
//    objects build with --fmad=false, the host with -ffp-contract=off), so the
//    host and the device compute the same bits.  The methods are the textbook
//    ones: log by x = m * 2^e, m in [sqrt(1/2), sqrt(2)), s = (m - 1) / (m + 1),
//    log(m) = 2 atanh(s) as its odd series to s^23; exp by z = k ln2 + r
//    (Cody-Waite reduction with ln2 split in two, |r| <= ln2 / 2) and the
//    Taylor series of e^r to r^13; sin and cos by a = q pi/2 + r (pi/2 split
//    in three, |r| <= pi/4) and their Taylor series to r^21 / r^20.  Every
//    constant below is derived from its definition (ln 2, pi, 1/(2k+1),
//    1/n!) and written as the binary64 value nearest to it (the ln2 and
//    pi/2 leading parts are truncated so that small multiples stay exact).
// 2. An exception table, built on the host by vx_libmx_gen.cpp, listing the
//    inputs of the generator's domains where the C library's result differs
//    from part 1's, with the C library's value: every float x in [0, 1] for
//    powf(x, 1.15f) and powf(x, 0.85f), and every branch angle paint_tree
//    can form for cosf and sinf (two to four branches, 65536 jitter values).
#pragma once

#include <stdint.h>
#include <string.h>

#include <cmath>

#ifdef __CUDACC__
#define VX_GM __host__ __device__ __forceinline__
#else
#define VX_GM inline
#endif

namespace vx {
namespace gm {

VX_GM uint64_t dbits(double x) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t b;
    memcpy(&b, &x, 8);
    return b;
#endif
}
VX_GM double dfrom(uint64_t b) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double x;
    memcpy(&x, &b, 8);
    return x;
#endif
}
VX_GM uint32_t fbits(float x) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(x);
#else
    uint32_t b;
    memcpy(&b, &x, 4);
    return b;
#endif
}
VX_GM float ffrom(uint32_t b) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float x;
    memcpy(&x, &b, 4);
    return x;
#endif
}
// double -> float, round to nearest even
VX_GM float to_f32(double x) {
#ifdef __CUDA_ARCH__
    return __double2float_rn(x);
#else
    return (float)x;
#endif
}
VX_GM double dfloor(double x) {
#ifdef __CUDA_ARCH__
    return floor(x);
#else
    return std::floor(x);
#endif
}

// ln 2 = LN2_HI + LN2_LO, LN2_HI to 33 significant bits
constexpr double LN2_HI = 0x1.62e42fee00000p-1;
constexpr double LN2_LO = 0x1.a39ef35793c76p-33;
constexpr double INV_LN2 = 0x1.71547652b82fep+0;
constexpr double SQRT2 = 0x1.6a09e667f3bcdp+0;
// pi / 2 = PIO2_1 + PIO2_2 + PIO2_3, the first two to 33 significant bits
constexpr double PIO2_1 = 0x1.921fb54400000p+0;
constexpr double PIO2_2 = 0x1.0b4611a600000p-34;
constexpr double PIO2_3 = 0x1.3198a2e037073p-69;
constexpr double TWO_OVER_PI = 0x1.45f306dc9c883p-1;

// log(x), x a finite positive double (every positive float is a normal double)
VX_GM double log_pos(double x) {
    const uint64_t b = dbits(x);
    int e = (int)((b >> 52) & 0x7FFu) - 1023;
    double m = dfrom((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);  // [1, 2)
    if (m > SQRT2) {
        m = m * 0.5;
        e += 1;
    }
    const double s = (m - 1.0) / (m + 1.0);  // m - 1 is exact
    const double z = s * s;
    // 1 + z/3 + z^2/5 + ... + z^11/23
    double p = 0x1.642c8590b2164p-5;  // 1/23
    p = p * z + 0x1.8618618618618p-5; // 1/21
    p = p * z + 0x1.af286bca1af28p-5; // 1/19
    p = p * z + 0x1.e1e1e1e1e1e1ep-5; // 1/17
    p = p * z + 0x1.1111111111111p-4; // 1/15
    p = p * z + 0x1.3b13b13b13b14p-4; // 1/13
    p = p * z + 0x1.745d1745d1746p-4; // 1/11
    p = p * z + 0x1.c71c71c71c71cp-4; // 1/9
    p = p * z + 0x1.2492492492492p-3; // 1/7
    p = p * z + 0x1.999999999999ap-3; // 1/5
    p = p * z + 0x1.5555555555555p-2; // 1/3
    p = p * z + 1.0;
    const double ed = (double)e;
    return ed * LN2_HI + (ed * LN2_LO + (s + s) * p);
}

// e^z for -708 < z <= 0
VX_GM double exp_neg(double z) {
    const double kd = dfloor(z * INV_LN2 + 0.5);
    const double r = (z - kd * LN2_HI) - kd * LN2_LO;  // kd * LN2_HI is exact
    // sum of r^n / n!, n = 0..13
    double p = 0x1.6124613a86d09p-33;  // 1/13!
    p = p * r + 0x1.1eed8eff8d898p-29; // 1/12!
    p = p * r + 0x1.ae64567f544e4p-26; // 1/11!
    p = p * r + 0x1.27e4fb7789f5cp-22; // 1/10!
    p = p * r + 0x1.71de3a556c734p-19; // 1/9!
    p = p * r + 0x1.a01a01a01a01ap-16; // 1/8!
    p = p * r + 0x1.a01a01a01a01ap-13; // 1/7!
    p = p * r + 0x1.6c16c16c16c17p-10; // 1/6!
    p = p * r + 0x1.1111111111111p-7;  // 1/5!
    p = p * r + 0x1.5555555555555p-5;  // 1/4!
    p = p * r + 0x1.5555555555555p-3;  // 1/3!
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    const int k = (int)kd;
    return p * dfrom((uint64_t)(k + 1023) << 52);
}

// sin and cos of a, |a| <= 16
VX_GM void sincos_small(double a, double *sn, double *cs) {
    const double q = dfloor(a * TWO_OVER_PI + 0.5);
    const double r = ((a - q * PIO2_1) - q * PIO2_2) - q * PIO2_3;  // q * PIO2_1, q * PIO2_2 exact
    const double z = r * r;
    // sin r = r * sum_k (-1)^k z^k / (2k+1)!, k = 0..10
    double s = 0x1.71b8ef6dcf572p-66;   //  1/21!
    s = s * z - 0x1.2f49b46814157p-57;  // -1/19!
    s = s * z + 0x1.952c77030ad4ap-49;  //  1/17!
    s = s * z - 0x1.ae7f3e733b81fp-41;  // -1/15!
    s = s * z + 0x1.6124613a86d09p-33;  //  1/13!
    s = s * z - 0x1.ae64567f544e4p-26;  // -1/11!
    s = s * z + 0x1.71de3a556c734p-19;  //  1/9!
    s = s * z - 0x1.a01a01a01a01ap-13;  // -1/7!
    s = s * z + 0x1.1111111111111p-7;   //  1/5!
    s = s * z - 0x1.5555555555555p-3;   // -1/3!
    s = s * z + 1.0;
    s = r * s;
    // cos r = sum_k (-1)^k z^k / (2k)!, k = 0..10
    double c = 0x1.e542ba4020225p-62;   //  1/20!
    c = c * z - 0x1.6827863b97d97p-53;  // -1/18!
    c = c * z + 0x1.ae7f3e733b81fp-45;  //  1/16!
    c = c * z - 0x1.93974a8c07c9dp-37;  // -1/14!
    c = c * z + 0x1.1eed8eff8d898p-29;  //  1/12!
    c = c * z - 0x1.27e4fb7789f5cp-22;  // -1/10!
    c = c * z + 0x1.a01a01a01a01ap-16;  //  1/8!
    c = c * z - 0x1.6c16c16c16c17p-10;  // -1/6!
    c = c * z + 0x1.5555555555555p-5;   //  1/4!
    c = c * z - 0.5;
    c = c * z + 1.0;
    // a = q pi/2 + r: rotate by the quadrant
    switch ((int)q & 3) {
        case 0: *sn = s; *cs = c; break;
        case 1: *sn = c; *cs = -s; break;
        case 2: *sn = -s; *cs = -c; break;
        default: *sn = -c; *cs = s; break;
    }
}

// ---------------------------------------------------------------- float API
// part 1 in binary32: powf(x, y) for x in [0, 1] and y > 0, cosf / sinf of
// |a| <= 16
VX_GM float pow01(float x, float y) {
    if (x == 0.0f) return 0.0f;
    if (x == 1.0f) return 1.0f;
    return to_f32(exp_neg((double)y * log_pos((double)x)));
}
VX_GM float cos_small(float a) {
    double s, c;
    sincos_small((double)a, &s, &c);
    return to_f32(c);
}
VX_GM float sin_small(float a) {
    double s, c;
    sincos_small((double)a, &s, &c);
    return to_f32(s);
}

// ------------------------------------------------------ exception table
// The table (uint32 words, built by vx_libmx_gen.cpp, loaded by the library):
//   [0] 'VXLM'  [1] version  [2..9] C library version string  [10] functions
//   [11 + f] word offset of function f's section
// A section: [0] n, [1 .. 65537] directory (the entries whose input bits
// have high half below i start at dir[i]), n input bits ascending, n
// result bits.
enum : uint32_t {
    LMX_POW115 = 0,   // powf(x, 1.15f), x in [0, 1]
    LMX_POW085 = 1,   // powf(x, 0.85f), x in [0, 1]
    LMX_COS = 2,      // cosf of paint_tree's branch angles
    LMX_SIN = 3,      // sinf of the same
    LMX_FUNCS = 4,
    LMX_MAGIC = 0x4D4C5856u,  // "VXLM"
    LMX_VERSION = 1,
    LMX_HEADER = 11 + LMX_FUNCS,
    LMX_DIR = 65537,
};

// the C library's value of function f at x, given part 1's value v
VX_GM float lmx_fix(const uint32_t *blob, uint32_t f, float x, float v) {
    const uint32_t *t = blob + blob[11 + f];
    const uint32_t n = t[0];
    const uint32_t *dir = t + 1;
    const uint32_t *key = dir + LMX_DIR;
    const uint32_t b = fbits(x);
    uint32_t lo = dir[b >> 16], hi = dir[(b >> 16) + 1];
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (key[mid] < b) lo = mid + 1;
        else hi = mid;
    }
    if (lo < dir[(b >> 16) + 1] && key[lo] == b) return ffrom(key[n + lo]);
    return v;
}

// paint_tree's branch angle (src/voxel.rs:1633-1634, :1689-1690): branch b of
// n at jitter j (the low 16 bits of the hash), spread 0.5 (birch) or 0.6
VX_GM float branch_angle(int32_t b, int32_t n, uint32_t j, float spread) {
    const float tau = 6.28318548202514648f;  // std::f32::consts::TAU
    const float jit = ((float)j / 65535.0f) * 2.0f - 1.0f;
    return ((float)b / (float)n) * tau + jit * spread;
}

}  // namespace gm
}  // namespace vx
