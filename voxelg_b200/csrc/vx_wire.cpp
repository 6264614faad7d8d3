// vx_wire.cpp -- the ray-query messages in voxelG's network framing, so
// that clients of the relay protocol (src/net.rs) can reach the serving
// loop.  Framing is net.rs's read_message / write_message (net.rs:71-90): a
// u32 little-endian payload length (at most 16 MiB) followed by the payload.
// The payload is what bincode 1.3.3 (Cargo.lock:185-186) serializes with its
// default configuration for two variants appended to net.rs's `Message`
// enum (net.rs:46-67) after `Heartbeat`:
//
//   RayQuery  { id: u64, rays: Vec<WireRay> }         variant 10
//   RayResult { id: u64, records: Vec<WireRecord> }   variant 11
//   WireRay    { org: [f32; 3], dir: [f32; 3], tmax: f32, kind: u32 }
//   WireRecord { voxel: [i32; 3], face: u8, mat: u8, flags: u8, t: f32, steps: u32 }
//
// i.e. the variant index as u32, integers and floats as fixed-width
// little-endian, fixed arrays without a length, Vec<T> as a u64 length and
// its elements, struct fields in order with no padding.
#include <cstring>
#include <string>

#include "voxrt.h"
#include "vx_internal.h"

namespace {

constexpr uint32_t kMaxPayload = 16u * 1024u * 1024u;  // net.rs:74
constexpr uint32_t kTagQuery = 10, kTagResult = 11;
constexpr size_t kRayBytes = 32, kRecordBytes = 23, kHead = 4 + 4 + 8 + 8;

struct Writer {
    uint8_t *p;
    void u8(uint8_t v) { *p++ = v; }
    void u32(uint32_t v) {
        for (int i = 0; i < 4; ++i) *p++ = (uint8_t)(v >> (8 * i));
    }
    void u64(uint64_t v) {
        for (int i = 0; i < 8; ++i) *p++ = (uint8_t)(v >> (8 * i));
    }
    void f32(float f) {
        uint32_t v;
        std::memcpy(&v, &f, 4);
        u32(v);
    }
};

struct Reader {
    const uint8_t *p;
    uint8_t u8() { return *p++; }
    uint32_t u32() {
        uint32_t v = 0;
        for (int i = 0; i < 4; ++i) v |= (uint32_t)*p++ << (8 * i);
        return v;
    }
    uint64_t u64() {
        uint64_t v = 0;
        for (int i = 0; i < 8; ++i) v |= (uint64_t)*p++ << (8 * i);
        return v;
    }
    float f32() {
        const uint32_t v = u32();
        float f;
        std::memcpy(&f, &v, 4);
        return f;
    }
};

int bad(const char *fn, const char *why) {
    vx::set_error(std::string(fn) + ": " + why);
    return VX_ERR_INVALID;
}

// frame header shared by both messages; returns the element count
int read_head(const uint8_t *buf, size_t len, uint32_t tag, size_t elem, const char *fn,
              uint64_t *id, uint64_t *count) {
    if (!buf || len < kHead) return bad(fn, "frame shorter than its header");
    Reader r{buf};
    const uint32_t payload = r.u32();
    if (payload > kMaxPayload) return bad(fn, "payload over the 16 MiB frame limit");
    if ((size_t)payload + 4 != len) return bad(fn, "frame length does not match its prefix");
    if (r.u32() != tag) return bad(fn, "not this message variant");
    *id = r.u64();
    *count = r.u64();
    if (*count > (kMaxPayload - (kHead - 4)) / elem || kHead + *count * elem != len)
        return bad(fn, "element count does not match the frame length");
    return VX_OK;
}

}  // namespace

extern "C" {

size_t vx_wire_query_bytes(size_t n) { return kHead + n * kRayBytes; }
size_t vx_wire_result_bytes(size_t n) { return kHead + n * kRecordBytes; }

int vx_wire_encode_query(uint64_t id, const VxRay *rays, size_t n, uint8_t *buf, size_t cap,
                         size_t *len) {
    const char *fn = "vx_wire_encode_query";
    if (!buf || !len || (n && !rays)) return bad(fn, "null argument");
    const size_t total = vx_wire_query_bytes(n);
    if (total - 4 > kMaxPayload) return bad(fn, "query over the 16 MiB frame limit");
    if (cap < total) return bad(fn, "buffer too small");
    Writer w{buf};
    w.u32((uint32_t)(total - 4));
    w.u32(kTagQuery);
    w.u64(id);
    w.u64(n);
    for (size_t i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) w.f32(rays[i].org[k]);
        for (int k = 0; k < 3; ++k) w.f32(rays[i].dir[k]);
        w.f32(rays[i].tmax);
        w.u32(rays[i].kind);
    }
    *len = total;
    return VX_OK;
}

int vx_wire_decode_query(const uint8_t *buf, size_t len, uint64_t *id, VxRay *rays, size_t cap,
                         size_t *n) {
    const char *fn = "vx_wire_decode_query";
    if (!id || !n) return bad(fn, "null argument");
    uint64_t count = 0;
    const int rc = read_head(buf, len, kTagQuery, kRayBytes, fn, id, &count);
    if (rc != VX_OK) return rc;
    *n = (size_t)count;
    if (count > cap || (count && !rays)) return bad(fn, "ray buffer too small");
    Reader r{buf + kHead};
    for (uint64_t i = 0; i < count; ++i) {
        for (int k = 0; k < 3; ++k) rays[i].org[k] = r.f32();
        for (int k = 0; k < 3; ++k) rays[i].dir[k] = r.f32();
        rays[i].tmax = r.f32();
        rays[i].kind = r.u32();
    }
    return VX_OK;
}

int vx_wire_encode_result(uint64_t id, const VxHitRecord *rec, size_t n, uint8_t *buf, size_t cap,
                          size_t *len) {
    const char *fn = "vx_wire_encode_result";
    if (!buf || !len || (n && !rec)) return bad(fn, "null argument");
    const size_t total = vx_wire_result_bytes(n);
    if (total - 4 > kMaxPayload) return bad(fn, "result over the 16 MiB frame limit");
    if (cap < total) return bad(fn, "buffer too small");
    Writer w{buf};
    w.u32((uint32_t)(total - 4));
    w.u32(kTagResult);
    w.u64(id);
    w.u64(n);
    for (size_t i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) w.u32((uint32_t)rec[i].voxel[k]);
        w.u8(rec[i].face);
        w.u8(rec[i].mat);
        w.u8(rec[i].flags);
        w.f32(rec[i].t);
        w.u32(rec[i].steps);
    }
    *len = total;
    return VX_OK;
}

int vx_wire_decode_result(const uint8_t *buf, size_t len, uint64_t *id, VxHitRecord *rec,
                          size_t cap, size_t *n) {
    const char *fn = "vx_wire_decode_result";
    if (!id || !n) return bad(fn, "null argument");
    uint64_t count = 0;
    const int rc = read_head(buf, len, kTagResult, kRecordBytes, fn, id, &count);
    if (rc != VX_OK) return rc;
    *n = (size_t)count;
    if (count > cap || (count && !rec)) return bad(fn, "record buffer too small");
    Reader r{buf + kHead};
    for (uint64_t i = 0; i < count; ++i) {
        for (int k = 0; k < 3; ++k) rec[i].voxel[k] = (int32_t)r.u32();
        rec[i].face = r.u8();
        rec[i].mat = r.u8();
        rec[i].flags = r.u8();
        rec[i].pad = 0;
        rec[i].t = r.f32();
        rec[i].steps = r.u32();
    }
    return VX_OK;
}

}  // extern "C"
