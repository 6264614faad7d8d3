// vx_libmx_gen.cpp -- builds the exception table of vx_gmath.h: the inputs
// of the chunk generator's domains where the host C library's binary32
// powf / cosf / sinf differ from vx_gmath.h's functions, with the library's
// values (format at LMX_MAGIC in vx_gmath.h).
//
// Usage: vx_libmx_gen OUT.bin      (run by voxelg_b200/build.py)
//
// Domains: every float x in [0, 1] for powf(x, 1.15f) and powf(x, 0.85f)
// (src/voxel.rs:1262, :1623); for cosf and sinf every angle paint_tree can
// form (src/voxel.rs:1633-1641, :1689-1697): branch b of n = 2 or 3 (birch,
// jitter spread 0.5) or n = 3 or 4 (oak and autumn, spread 0.6), each of
// the 65536 jitter values.  Compile with -ffp-contract=off.
#include <gnu/libc-version.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "vx_gmath.h"

using namespace vx::gm;

namespace {

struct Entry {
    uint32_t key, val;
};

// the C library's functions, called through pointers so that no compiler
// folds or replaces them
float (*volatile c_powf)(float, float) = powf;
float (*volatile c_cosf)(float) = cosf;
float (*volatile c_sinf)(float) = sinf;

std::vector<Entry> scan_pow(float y) {
    const uint32_t last = 0x3F800000u;  // 1.0f
    const unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::vector<Entry>> part(nt);
    std::vector<std::thread> th;
    const uint64_t total = (uint64_t)last + 1;
    for (unsigned t = 0; t < nt; ++t) {
        th.emplace_back([&, t] {
            const uint64_t a = total * t / nt, b = total * (t + 1) / nt;
            for (uint64_t i = a; i < b; ++i) {
                const float x = ffrom((uint32_t)i);
                const uint32_t g = fbits(c_powf(x, y)), m = fbits(pow01(x, y));
                if (g != m) part[t].push_back({(uint32_t)i, g});
            }
        });
    }
    for (auto &t : th) t.join();
    std::vector<Entry> out;
    for (auto &p : part) out.insert(out.end(), p.begin(), p.end());
    return out;  // ascending: threads cover ascending ranges
}

std::vector<float> branch_angles() {
    std::vector<float> a;
    const struct { int32_t n0, n1; float spread; } kinds[2] = {{2, 3, 0.5f}, {3, 4, 0.6f}};
    for (const auto &k : kinds)
        for (int32_t n = k.n0; n <= k.n1; ++n)
            for (int32_t b = 0; b < n; ++b)
                for (uint32_t j = 0; j < 65536u; ++j) a.push_back(branch_angle(b, n, j, k.spread));
    std::sort(a.begin(), a.end(), [](float u, float v) { return fbits(u) < fbits(v); });
    a.erase(std::unique(a.begin(), a.end(),
                        [](float u, float v) { return fbits(u) == fbits(v); }),
            a.end());
    return a;
}

std::vector<Entry> scan_trig(const std::vector<float> &angles, bool cosine) {
    std::vector<Entry> out;
    for (float a : angles) {
        const uint32_t g = fbits(cosine ? c_cosf(a) : c_sinf(a));
        const uint32_t m = fbits(cosine ? cos_small(a) : sin_small(a));
        if (g != m) out.push_back({fbits(a), g});
    }
    return out;  // ascending by input bits
}

void section(std::vector<uint32_t> &blob, const std::vector<Entry> &e) {
    blob.push_back((uint32_t)e.size());
    const size_t dir = blob.size();
    blob.resize(dir + LMX_DIR);
    size_t k = 0;
    for (uint32_t i = 0; i < LMX_DIR; ++i) {
        while (k < e.size() && (e[k].key >> 16) < i) ++k;
        blob[dir + i] = (uint32_t)k;
    }
    for (const auto &x : e) blob.push_back(x.key);
    for (const auto &x : e) blob.push_back(x.val);
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s OUT.bin\n", argv[0]);
        return 2;
    }
    std::vector<Entry> fn[LMX_FUNCS];
    fn[LMX_POW115] = scan_pow(1.15f);
    fn[LMX_POW085] = scan_pow(0.85f);
    const std::vector<float> angles = branch_angles();
    fn[LMX_COS] = scan_trig(angles, true);
    fn[LMX_SIN] = scan_trig(angles, false);
    std::vector<uint32_t> blob(LMX_HEADER, 0u);
    blob[0] = LMX_MAGIC;
    blob[1] = LMX_VERSION;
    char ver[32] = {0};
    std::strncpy(ver, gnu_get_libc_version(), sizeof(ver) - 1);
    std::memcpy(&blob[2], ver, sizeof(ver));
    blob[10] = LMX_FUNCS;
    for (uint32_t f = 0; f < LMX_FUNCS; ++f) {
        blob[11 + f] = (uint32_t)blob.size();
        section(blob, fn[f]);
    }
    FILE *o = std::fopen(argv[1], "wb");
    if (!o || std::fwrite(blob.data(), 4, blob.size(), o) != blob.size() || std::fclose(o) != 0) {
        std::fprintf(stderr, "cannot write %s\n", argv[1]);
        return 1;
    }
    std::printf("%s: glibc %s; exceptions pow(x,1.15) %zu, pow(x,0.85) %zu, cos %zu, sin %zu "
                "(of %zu angles)\n",
                argv[1], ver, fn[0].size(), fn[1].size(), fn[2].size(), fn[3].size(),
                angles.size());
    return 0;
}
