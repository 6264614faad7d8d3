// vx_api.cpp -- the C ABI of libvoxrt (include/voxrt.h): device world
// lifetime, uploads, the traversal entry points and error reporting.
#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <dlfcn.h>
#include <gnu/libc-version.h>
#include <thread>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "vx_gmath.h"
#include "vx_internal.h"

namespace vx {
namespace {
thread_local std::string g_last_error;
}
void set_error(const std::string &msg) { g_last_error = msg; }
}  // namespace vx

struct VxWorld {
    int device = 0;
    vx::DevWorld dw{};
    cudaStream_t stream = nullptr;   // library stream for synchronous calls
    std::mutex mu;                   // guards the scratch buffers below
    float *beam = nullptr;
    size_t beam_cap = 0;
    uint32_t *d_idx = nullptr;
    size_t idx_cap = 0;
    VxBrick *d_bricks = nullptr;
    size_t bricks_cap = 0;
    unsigned long long *d_stats = nullptr;
    VxHitRecord *rec = nullptr;
    size_t rec_cap = 0;
    VxShadowRecord *sh = nullptr;
    size_t sh_cap = 0;
    // single-ray picking: pinned, device-mapped host block that the kernel
    // writes its result to (the ray travels in the launch parameters; no
    // copies, one sync)
    struct PickBox {
        VxPickHit out;
        int32_t hit;
        uint32_t fault;               // DevWorld::fault (kFaultBeamCopyLost)
    };
    PickBox *pick = nullptr;          // host address
    PickBox *pick_dev = nullptr;      // device address of the same block
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    uint32_t *d_work = nullptr;      // persistent-schedule counters (self-resetting)
    cudaStream_t copy_stream = nullptr;
    uint32_t *d_gate_idx = nullptr;  // staging of vx_project_dirty
    size_t gate_cap = 0;
    vx::QueueScratch qs;             // scratch of vx_queue_run / vx_queue_autotune
    cudaEvent_t band_ev[4] = {};    // one per row band (kSyncBands at most)
    VxTuning tuning{0, {0, 0, 0, 0, 0, 0, 0}};
    // chunk generator state: the world chunk each storage-chunk slot holds
    // (3 ints per slot, empty until a window is filled), its seed and origin
    std::vector<int32_t> slot_chunk;
    uint64_t gen_seed = 0;
    int32_t gen_origin[2] = {0, 0};
    bool gen_window = false;         // a window fill made the slot table whole
    // persistent edits by world voxel, replayed into regenerated chunks
    std::map<std::array<int32_t, 3>, uint8_t> edits;
    uint2 *d_edits = nullptr;
    size_t edits_cap = 0;
    // host-buffer frames: ping-pong device records, and per buffer the event
    // after its last copy to the host (frame N+1 renders while N copies)
    VxHitRecord *hrec[2] = {nullptr, nullptr};
    VxShadowRecord *hsh[2] = {nullptr, nullptr};
    VxPackedRecord *hpk[2] = {nullptr, nullptr};   // packed frames (vx_pack.cu)
    size_t hrec_cap[2] = {0, 0}, hsh_cap[2] = {0, 0}, hpk_cap[2] = {0, 0};
    cudaEvent_t copy_done[2] = {nullptr, nullptr};
    uint64_t host_frames = 0;
    void *d_gen = nullptr;           // chunk generator scratch: plan, column words, trees
    size_t gen_cap = 0;              // bytes
    void *h_gen = nullptr;           // pinned staging of the generator's plan
    size_t h_gen_cap = 0;            // bytes
    uint32_t *d_lmx = nullptr;       // device copy of the generator's math exception table
    // vx_world_apply_dirty: a claim word per brick (zero between updates),
    // and two staging buffers (pinned host + device), each free again once
    // its update's event has passed; every update waits for the previous one
    uint32_t *d_dirty_win = nullptr;
    struct DirtyStage {
        uint32_t *h_idx = nullptr;
        VxBrick *h_bricks = nullptr;
        uint32_t *d_idx = nullptr;
        VxBrick *d_bricks = nullptr;
        size_t cap = 0;
        cudaEvent_t done = nullptr;
    } dirty[2];
    uint64_t dirty_calls = 0;
    cudaEvent_t dirty_last = nullptr;
    // empty-space distance fields of the learned form, rebuilt on demand when
    // the masks changed (mask_gen) since they were built (df_gen)
    uint8_t *bdf = nullptr, *tdf = nullptr, *df_tmp = nullptr;
    std::atomic<uint64_t> mask_gen{1};
    uint64_t df_gen = 0;
    float *lrn_depth = nullptr;      // per-tile proven depths of learned frames without a proposal
    size_t lrn_depth_cap = 0;
};

namespace vx {
DevWorld world_dev(const VxWorld *w) { return w->dw; }
int world_device(const VxWorld *w) { return w->device; }
void world_masks_changed(VxWorld *w) { w->mask_gen.fetch_add(1, std::memory_order_relaxed); }

int world_dist_fields(VxWorld *w, cudaStream_t s, DevWorld *out) {
    std::lock_guard<std::mutex> lk(w->mu);
    cudaError_t e = cudaSuccess;
    if (!w->bdf) {
        e = cudaMalloc(&w->bdf, (size_t)w->dw.d.n_bricks);
        if (e == cudaSuccess) e = cudaMalloc(&w->tdf, (size_t)w->dw.d.n_tiles);
        if (e == cudaSuccess) e = cudaMalloc(&w->df_tmp, (size_t)w->dw.d.n_bricks);
        if (e != cudaSuccess) {
            cudaFree(w->bdf);
            cudaFree(w->tdf);
            cudaFree(w->df_tmp);
            w->bdf = w->tdf = w->df_tmp = nullptr;
        }
    }
    const uint64_t gen = w->mask_gen.load(std::memory_order_relaxed);
    if (e == cudaSuccess && w->df_gen != gen) {
        e = launch_dist_fields(w->dw, w->bdf, w->tdf, w->df_tmp, s);
        if (e == cudaSuccess) w->df_gen = gen;
    }
    if (e != cudaSuccess) {
        set_error(std::string("distance fields: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? VX_ERR_OOM : VX_ERR_CUDA;
    }
    *out = w->dw;
    out->bdf = w->bdf;
    out->tdf = w->tdf;
    return VX_OK;
}

int world_learned_depth(VxWorld *w, size_t n, float **out) {
    std::lock_guard<std::mutex> lk(w->mu);
    if (w->lrn_depth_cap < n) {
        cudaFree(w->lrn_depth);
        w->lrn_depth = nullptr;
        w->lrn_depth_cap = 0;
        const cudaError_t e = cudaMalloc(&w->lrn_depth, std::max<size_t>(n, 1) * sizeof(float));
        if (e != cudaSuccess) {
            set_error(std::string("learned frame scratch: ") + cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? VX_ERR_OOM : VX_ERR_CUDA;
        }
        w->lrn_depth_cap = n;
    }
    *out = w->lrn_depth;
    return VX_OK;
}
}  // namespace vx

namespace {

#define VX_CK(call)                                                                   \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            vx::set_error(std::string(__func__) + ": " #call " failed: " +           \
                          cudaGetErrorString(e_));                                    \
            return e_ == cudaErrorMemoryAllocation ? VX_ERR_OOM : VX_ERR_CUDA;        \
        }                                                                             \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Row bands of the host-buffer frame path.  A synchronous call copies each
// band while the next one renders.  Pipelined calls overlap whole frames (one
// renders while the previous one copies), so one band, i.e. the fewest
// copies, is fastest there: 1.18 ms per 1080p frame against 1.23 ms with 8
// bands, where the copy engine spends a few microseconds per copy.
constexpr uint32_t kSyncBands = 4;
constexpr uint32_t kAsyncBands = 1;

int use_device(VxWorld *w) {
    VX_CK(cudaSetDevice(w->device));
    return VX_OK;
}

template <typename T>
int ensure(T **p, size_t *cap, size_t n) {
    if (*cap >= n && *p) return VX_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    VX_CK(cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(n, 1) * sizeof(T)));
    *cap = n;
    return VX_OK;
}

void free_world(VxWorld *w) {
    cudaFree(w->dw.occ);
    cudaFree(w->dw.mat);
    cudaFree(w->dw.tile_mask);
    cudaFree(w->dw.chunk_mask);
    cudaFree(w->dw.l4_mask);
    cudaFree(w->dw.brick_uniform);
    cudaFree(w->dw.tile_uniform);
    cudaFree(w->dw.tile_meta);
    cudaFree(w->dw.oob);
    cudaFree(w->beam);
    cudaFree(w->d_idx);
    cudaFree(w->d_bricks);
    cudaFree(w->d_stats);
    cudaFree(w->rec);
    cudaFree(w->sh);
    if (w->pick) cudaFreeHost(w->pick);
    cudaFree(w->d_work);
    cudaFree(w->d_gate_idx);
    cudaFree(w->d_gen);
    cudaFree(w->d_edits);
    cudaFree(w->bdf);
    cudaFree(w->tdf);
    cudaFree(w->df_tmp);
    cudaFree(w->lrn_depth);
    if (w->h_gen) cudaFreeHost(w->h_gen);
    cudaFree(w->d_lmx);
    cudaFree(w->d_dirty_win);
    for (auto &b : w->dirty) {
        if (b.h_idx) cudaFreeHost(b.h_idx);
        if (b.h_bricks) cudaFreeHost(b.h_bricks);
        cudaFree(b.d_idx);
        cudaFree(b.d_bricks);
        if (b.done) cudaEventDestroy(b.done);
    }
    if (w->dirty_last) cudaEventDestroy(w->dirty_last);
    if (w->copy_stream) cudaStreamSynchronize(w->copy_stream);
    for (int i = 0; i < 2; ++i) {
        cudaFree(w->hrec[i]);
        cudaFree(w->hsh[i]);
        cudaFree(w->hpk[i]);
        if (w->copy_done[i]) cudaEventDestroy(w->copy_done[i]);
    }
    w->qs.release();
    for (auto &e : w->ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : w->band_ev)
        if (e) cudaEventDestroy(e);
    if (w->copy_stream) cudaStreamDestroy(w->copy_stream);
    if (w->stream) cudaStreamDestroy(w->stream);
}

// The whole world is replaced: the chunk generator's slot table no longer
// describes it.  Caller holds w->mu.
void forget_generated(VxWorld *w) {
    w->slot_chunk.clear();
    w->gen_window = false;
}

int check_frame(const VxCamera *cam) {
    if (!cam || !(cam->res_x >= 1.0f) || !(cam->res_y >= 1.0f) || cam->res_x > 32768.0f ||
        cam->res_y > 32768.0f || cam->res_x != std::floor(cam->res_x) ||
        cam->res_y != std::floor(cam->res_y)) {
        vx::set_error("camera resolution must be an integer in [1, 32768]");
        return VX_ERR_INVALID;
    }
    if (!vx::origin_ok(cam->world_origin, "camera")) return VX_ERR_INVALID;
    return VX_OK;
}

vx::FrameArgs make_frame(VxWorld *w, const VxCamera *cam, const VxTraceParams *p) {
    vx::FrameArgs fa{};
    fa.ta.w = w->dw;
    fa.ta.p = *p;
    fa.ta.ro[0] = cam->world_origin[0];
    fa.ta.ro[1] = cam->world_origin[1];
    fa.ta.ro[2] = cam->world_origin[2];
    fa.cam = *cam;
    fa.W = (uint32_t)cam->res_x;
    fa.H = (uint32_t)cam->res_y;
    fa.bw = (fa.W + 7u) / 8u;
    fa.bh = (fa.H + 7u) / 8u;
    fa.y0 = 0;
    fa.y1 = fa.H;
    fa.work = w->tuning.persistent ? w->d_work : nullptr;
    return fa;
}

// beam + primary on one stream; caller holds w->mu
int run_frame(VxWorld *w, vx::FrameArgs &fa, cudaStream_t s) {
    if (fa.ta.p.flags & VX_F_BEAM) {
        int rc = ensure(&w->beam, &w->beam_cap, (size_t)fa.bw * fa.bh);
        if (rc != VX_OK) return rc;
        fa.beam = w->beam;
        VX_CK(vx::launch_beam(fa, w->beam, s));
    }
    VX_CK(vx::launch_primary(fa, s));
    return VX_OK;
}

// After a synchronisation: a fault the kernels of this world recorded in its
// mapped fault word (a beam CTA that left before its bulk copy landed) turns
// the call's result into VX_ERR_DEVICE, once.
int take_fault(VxWorld *w, const char *fn) {
    volatile uint32_t *f = &w->pick->fault;
    const uint32_t v = *f;
    if (v == 0u) return VX_OK;
    *f = 0u;
    std::string msg = std::string(fn) + ":";
    if (v & vx::kFaultBeamCopyLost)
        msg += " a beam pre-pass block exited before its bulk copy of the chunk masks "
               "completed (bounded wait ran out); records of the frame are valid, shared "
               "memory of a later block may have been overwritten;";
    if (v & vx::kFaultCompactLossy)
        msg += " a compact frame held a record VxCompactRecord cannot hold (its 12-byte "
               "records are not the frame's);";
    vx::set_error(msg);
    return VX_ERR_DEVICE;
}

int check_params(const VxTraceParams *p) {
    if (!p || p->max_iters < 0 || p->any_max_iters < 0 || p->max_iters > (1 << 20) ||
        p->any_max_iters > (1 << 20)) {
        vx::set_error("invalid VxTraceParams (null or iteration caps outside [0, 2^20])");
        return VX_ERR_INVALID;
    }
    return VX_OK;
}

}  // namespace

extern "C" {

int vx_abi_version(void) { return VX_ABI_VERSION; }

const char *vx_last_error(void) { return vx::g_last_error.c_str(); }

int vx_default_params(VxTraceParams *p) {
    if (!p) return VX_ERR_INVALID;
    std::memset(p, 0, sizeof(*p));
    p->max_dist = 700.0f;
    p->lod_brick_t = 400.0f;
    p->tile_lod_t = 520.0f;
    p->shadow_max_dist = 480.0f;
    p->beam_margin = 16.0f;
    p->max_iters = 1024;
    p->any_max_iters = 768;
    p->flags = VX_F_L4 | VX_F_LUT | VX_F_LOD | VX_F_BEAM | VX_F_SHADOW;
    // sun = normalize(0.3, 0.8, 0.5); tangent frame as raymarch.wgsl:3984-3988
    const float s0 = 0.3f, s1 = 0.8f, s2 = 0.5f;
    const float sl = std::sqrt((s0 * s0 + s1 * s1) + s2 * s2);
    p->sun[0] = s0 / sl;
    p->sun[1] = s1 / sl;
    p->sun[2] = s2 / sl;
    // cross(s, (0,1,0)) = (-s.z, 0, s.x)
    float t0 = -p->sun[2], t1 = 0.0f, t2 = p->sun[0];
    const float tl = std::sqrt((t0 * t0 + t1 * t1) + t2 * t2);
    if (tl < 0.01f) {
        t0 = 1.0f; t1 = 0.0f; t2 = 0.0f;
    } else {
        t0 = t0 / tl; t1 = t1 / tl; t2 = t2 / tl;
    }
    p->sun_tangent[0] = t0;
    p->sun_tangent[1] = t1;
    p->sun_tangent[2] = t2;
    p->sun_bitangent[0] = p->sun[1] * t2 - p->sun[2] * t1;
    p->sun_bitangent[1] = p->sun[2] * t0 - p->sun[0] * t2;
    p->sun_bitangent[2] = p->sun[0] * t1 - p->sun[1] * t0;
    p->cone_tan = 0.0087268678f;  // tan(0.5 degrees)
    p->frame = 0.0f;
    return VX_OK;
}

int vx_camera_from_pose(const float pos[3], float yaw, float pitch, float fov_y, uint32_t width,
                        uint32_t height, const int32_t world_origin[3], VxCamera *out) {
    if (!pos || !out || width == 0 || height == 0) return VX_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    // camera.rs:25-42 with glam's normalize = v * (1 / length)
    auto norm = [](float v[3]) {
        const float r = 1.0f / std::sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
        v[0] = v[0] * r; v[1] = v[1] * r; v[2] = v[2] * r;
    };
    float f[3] = {std::sin(yaw) * std::cos(pitch), std::sin(pitch), std::cos(yaw) * std::cos(pitch)};
    norm(f);
    float r[3] = {f[2], 0.0f, -f[0]};
    norm(r);
    float u[3] = {f[1] * r[2] - r[1] * f[2], f[2] * r[0] - r[2] * f[0], f[0] * r[1] - r[0] * f[1]};
    norm(u);
    for (int k = 0; k < 3; ++k) {
        out->origin[k] = pos[k];
        out->forward[k] = f[k];
        out->right[k] = r[k];
        out->up[k] = u[k];
        out->world_origin[k] = world_origin ? world_origin[k] : 0;
    }
    out->tan_half_fov = std::tan(fov_y * 0.5f);
    out->res_x = (float)width;
    out->res_y = (float)height;
    return VX_OK;
}

int vx_world_create(const VxWorldDesc *desc, VxWorld **out) {
    if (!desc || !out) {
        vx::set_error("vx_world_create: null argument");
        return VX_ERR_INVALID;
    }
    const int32_t bx = desc->bricks_x, by = desc->bricks_y, bz = desc->bricks_z;
    if (bx <= 0 || by <= 0 || bz <= 0 || bx % 64 || bz % 64 || by % 16 || bx > 65536 ||
        bz > 65536 || by > 65536) {
        vx::set_error("vx_world_create: bricks_x/z must be multiples of 64, bricks_y a "
                      "multiple of 16");
        return VX_ERR_INVALID;
    }
    VxWorld *w = new (std::nothrow) VxWorld();
    if (!w) return VX_ERR_OOM;
    w->device = desc->device;
    w->dw.d = vx::make_dims(bx, by, bz);
    const vx::Dims &d = w->dw.d;
    auto fail = [&](int rc) {
        free_world(w);
        delete w;
        return rc;
    };
    int rc = use_device(w);
    if (rc != VX_OK) return fail(rc);
#define VX_CKW(call)                                                                    \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            vx::set_error(std::string("vx_world_create: ") + cudaGetErrorString(e_));   \
            return fail(e_ == cudaErrorMemoryAllocation ? VX_ERR_OOM : VX_ERR_CUDA);    \
        }                                                                               \
    } while (0)
    VX_CKW(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
    VX_CKW(cudaMalloc(&w->dw.occ, d.n_bricks * sizeof(uint64_t)));
    VX_CKW(cudaMalloc(&w->dw.mat, d.n_bricks * 64));
    VX_CKW(cudaMalloc(&w->dw.tile_mask, d.n_tiles * sizeof(uint64_t)));
    VX_CKW(cudaMalloc(&w->dw.chunk_mask, d.n_chunks * sizeof(uint64_t)));
    VX_CKW(cudaMalloc(&w->dw.l4_mask, d.n_l4 * sizeof(uint64_t)));
    VX_CKW(cudaMalloc(&w->dw.brick_uniform, d.n_bricks));
    VX_CKW(cudaMalloc(&w->dw.tile_uniform, d.n_tiles));
    VX_CKW(cudaMalloc(&w->dw.tile_meta, d.n_tiles * sizeof(uint16_t)));
    VX_CKW(cudaMalloc(&w->dw.oob, sizeof(unsigned long long)));
    VX_CKW(cudaMemsetAsync(w->dw.oob, 0, sizeof(unsigned long long), w->stream));
    VX_CKW(cudaMalloc(&w->d_stats, 4 * sizeof(unsigned long long)));
    VX_CKW(cudaMalloc(&w->d_work, 2 * sizeof(uint32_t)));
    VX_CKW(cudaMemsetAsync(w->d_work, 0, 2 * sizeof(uint32_t), w->stream));
    VX_CKW(cudaHostAlloc(reinterpret_cast<void **>(&w->pick), sizeof(VxWorld::PickBox),
                         cudaHostAllocMapped));
    VX_CKW(cudaHostGetDevicePointer(reinterpret_cast<void **>(&w->pick_dev), w->pick, 0));
    w->pick->fault = 0u;
    w->dw.fault = &w->pick_dev->fault;
    VX_CKW(cudaMemsetAsync(w->dw.occ, 0, d.n_bricks * sizeof(uint64_t), w->stream));
    VX_CKW(cudaMemsetAsync(w->dw.mat, 0, d.n_bricks * 64, w->stream));
    VX_CKW(cudaMemsetAsync(w->dw.tile_mask, 0, d.n_tiles * sizeof(uint64_t), w->stream));
    VX_CKW(cudaMemsetAsync(w->dw.chunk_mask, 0, d.n_chunks * sizeof(uint64_t), w->stream));
    VX_CKW(cudaMemsetAsync(w->dw.l4_mask, 0, d.n_l4 * sizeof(uint64_t), w->stream));
    VX_CKW(cudaMemsetAsync(w->dw.brick_uniform, 0, d.n_bricks, w->stream));
    VX_CKW(cudaMemsetAsync(w->dw.tile_uniform, 0, d.n_tiles, w->stream));
    VX_CKW(vx::launch_tile_meta(w->dw, w->stream));
    VX_CKW(cudaStreamSynchronize(w->stream));
#undef VX_CKW
    *out = w;
    return VX_OK;
}

int vx_world_destroy(VxWorld *w) {
    if (!w) return VX_OK;
    cudaSetDevice(w->device);
    if (w->stream) cudaStreamSynchronize(w->stream);
    free_world(w);
    delete w;
    return VX_OK;
}

int vx_world_set_tuning(VxWorld *w, const VxTuning *t) {
    if (!w || !t || (t->persistent != 0 && t->persistent != 1)) {
        vx::set_error("vx_world_set_tuning: persistent must be 0 or 1");
        return VX_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(w->mu);
    w->tuning = *t;
    return VX_OK;
}

int vx_world_get_tuning(const VxWorld *w, VxTuning *t) {
    if (!w || !t) return VX_ERR_INVALID;
    *t = w->tuning;
    return VX_OK;
}

int vx_world_counts(const VxWorld *w, uint64_t counts[4]) {
    if (!w || !counts) return VX_ERR_INVALID;
    counts[0] = (uint64_t)w->dw.d.n_bricks;
    counts[1] = (uint64_t)w->dw.d.n_tiles;
    counts[2] = (uint64_t)w->dw.d.n_chunks;
    counts[3] = (uint64_t)w->dw.d.n_l4;
    return VX_OK;
}

int vx_world_upload(VxWorld *w, const VxBrick *bricks, const uint64_t *tile_mask,
                    const uint64_t *chunk_mask, const uint64_t *l4_mask,
                    const uint8_t *brick_uniform, const uint8_t *tile_uniform) {
    vx::Range nvtx_range("vx_world_upload");
    if (!w || !bricks || !tile_mask || !chunk_mask || !l4_mask || !brick_uniform || !tile_uniform) {
        vx::set_error("vx_world_upload: null argument");
        return VX_ERR_INVALID;
    }
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    forget_generated(w);
    const vx::Dims &d = w->dw.d;
    const size_t chunk = (size_t)1 << 20;  // bricks per staging round (72 MiB)
    rc = ensure(&w->d_bricks, &w->bricks_cap, std::min<size_t>(chunk, (size_t)d.n_bricks));
    if (rc != VX_OK) return rc;
    for (int64_t first = 0; first < d.n_bricks; first += (int64_t)chunk) {
        const int64_t cnt = std::min<int64_t>((int64_t)chunk, d.n_bricks - first);
        VX_CK(cudaMemcpyAsync(w->d_bricks, bricks + first, (size_t)cnt * sizeof(VxBrick),
                              cudaMemcpyHostToDevice, w->stream));
        VX_CK(vx::launch_bricks_from_aos(w->dw, w->d_bricks, first, cnt, w->stream));
    }
    VX_CK(cudaMemcpyAsync(w->dw.tile_mask, tile_mask, d.n_tiles * 8, cudaMemcpyHostToDevice, w->stream));
    VX_CK(cudaMemcpyAsync(w->dw.chunk_mask, chunk_mask, d.n_chunks * 8, cudaMemcpyHostToDevice, w->stream));
    VX_CK(cudaMemcpyAsync(w->dw.l4_mask, l4_mask, d.n_l4 * 8, cudaMemcpyHostToDevice, w->stream));
    VX_CK(cudaMemcpyAsync(w->dw.brick_uniform, brick_uniform, d.n_bricks, cudaMemcpyHostToDevice, w->stream));
    VX_CK(cudaMemcpyAsync(w->dw.tile_uniform, tile_uniform, d.n_tiles, cudaMemcpyHostToDevice, w->stream));
    vx::world_masks_changed(w);
    VX_CK(vx::launch_tile_meta(w->dw, w->stream));
    VX_CK(cudaStreamSynchronize(w->stream));
    return VX_OK;
}

int vx_world_download(VxWorld *w, VxBrick *bricks, uint64_t *tile_mask, uint64_t *chunk_mask,
                      uint64_t *l4_mask, uint8_t *brick_uniform, uint8_t *tile_uniform) {
    if (!w) return VX_ERR_INVALID;
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    const vx::Dims &d = w->dw.d;
    if (bricks) {
        const size_t chunk = (size_t)1 << 20;
        rc = ensure(&w->d_bricks, &w->bricks_cap, std::min<size_t>(chunk, (size_t)d.n_bricks));
        if (rc != VX_OK) return rc;
        const size_t step = std::min(chunk, w->bricks_cap);
        for (int64_t first = 0; first < d.n_bricks; first += (int64_t)step) {
            const int64_t cnt = std::min<int64_t>((int64_t)step, d.n_bricks - first);
            VX_CK(vx::launch_bricks_to_aos(w->dw, w->d_bricks, first, cnt, w->stream));
            VX_CK(cudaMemcpyAsync(bricks + first, w->d_bricks, (size_t)cnt * sizeof(VxBrick),
                                  cudaMemcpyDeviceToHost, w->stream));
            VX_CK(cudaStreamSynchronize(w->stream));
        }
    }
    if (tile_mask) VX_CK(cudaMemcpyAsync(tile_mask, w->dw.tile_mask, d.n_tiles * 8, cudaMemcpyDeviceToHost, w->stream));
    if (chunk_mask) VX_CK(cudaMemcpyAsync(chunk_mask, w->dw.chunk_mask, d.n_chunks * 8, cudaMemcpyDeviceToHost, w->stream));
    if (l4_mask) VX_CK(cudaMemcpyAsync(l4_mask, w->dw.l4_mask, d.n_l4 * 8, cudaMemcpyDeviceToHost, w->stream));
    if (brick_uniform) VX_CK(cudaMemcpyAsync(brick_uniform, w->dw.brick_uniform, d.n_bricks, cudaMemcpyDeviceToHost, w->stream));
    if (tile_uniform) VX_CK(cudaMemcpyAsync(tile_uniform, w->dw.tile_uniform, d.n_tiles, cudaMemcpyDeviceToHost, w->stream));
    VX_CK(cudaStreamSynchronize(w->stream));
    return VX_OK;
}

int vx_world_generate(VxWorld *w, const VxTerrainParams *t) {
    vx::Range nvtx_range("vx_world_generate");
    if (!w || !t || t->octaves > 32) {
        vx::set_error("vx_world_generate: null argument or octaves > 32");
        return VX_ERR_INVALID;
    }
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    forget_generated(w);
    const vx::Dims &d = w->dw.d;
    int16_t *heights = nullptr;
    VX_CK(cudaMallocAsync(&heights, (size_t)d.vx * d.vz * sizeof(int16_t), w->stream));
    vx::world_masks_changed(w);
    cudaError_t e = vx::launch_generate(w->dw, *t, heights, w->stream);
    cudaFreeAsync(heights, w->stream);
    VX_CK(e);
    VX_CK(cudaStreamSynchronize(w->stream));
    return VX_OK;
}

namespace {
// pos_mod(a, n) for n > 0; a mask when n is a power of two
inline int32_t wrap(int32_t a, int32_t n) {
    return (n & (n - 1)) == 0 ? (a & (n - 1)) : ((a % n) + n) % n;
}

// pos_mod / div_euclid by a chunk's 32 voxels
inline int32_t chunk_of(int32_t v) { return v >= 0 ? v / 32 : -((-v + 31) / 32); }

// Writes edits (world voxel + material) into their slot voxels
// (pos_mod(x, VX), y, pos_mod(z, VZ)) on the device and refreshes the
// touched bricks' uniform bytes and parent masks.  Caller holds w->mu.
int write_edits_locked(VxWorld *w, const std::vector<std::array<int32_t, 4>> &list) {
    if (list.empty()) return VX_OK;
    const vx::Dims &d = w->dw.d;
    std::vector<uint2> ed;
    std::vector<uint32_t> bricks;
    ed.reserve(list.size());
    for (const auto &e : list) {
        const uint32_t x = (uint32_t)wrap(e[0], d.vx), y = (uint32_t)e[1],
                       z = (uint32_t)wrap(e[2], d.vz);
        const uint32_t bi = (x >> 2) + (y >> 2) * (uint32_t)d.bx + (z >> 2) * (uint32_t)(d.bx * d.by);
        const uint32_t vi = (x & 3u) + (z & 3u) * 4u + (y & 3u) * 16u;
        ed.push_back(make_uint2(bi, vi | ((uint32_t)e[3] << 8)));
        bricks.push_back(bi);
    }
    std::sort(bricks.begin(), bricks.end());
    bricks.erase(std::unique(bricks.begin(), bricks.end()), bricks.end());
    int rc = ensure(&w->d_edits, &w->edits_cap, ed.size());
    if (rc == VX_OK) rc = ensure(&w->d_idx, &w->idx_cap, bricks.size());
    if (rc != VX_OK) return rc;
    VX_CK(cudaMemcpyAsync(w->d_edits, ed.data(), ed.size() * sizeof(uint2), cudaMemcpyHostToDevice,
                          w->stream));
    VX_CK(cudaMemcpyAsync(w->d_idx, bricks.data(), bricks.size() * sizeof(uint32_t),
                          cudaMemcpyHostToDevice, w->stream));
    vx::world_masks_changed(w);
    VX_CK(vx::launch_edits(w->dw, w->d_edits, ed.size(), w->d_idx, bricks.size(), w->stream));
    VX_CK(cudaStreamSynchronize(w->stream));
    return VX_OK;
}

// The window's lower corner in world voxels: that of the last window fill or
// shift, else 0 (World::world_origin_voxel, voxel.rs:439-445).
inline void window_corner(const VxWorld *w, int32_t &ox, int32_t &oz) {
    ox = w->gen_window ? w->gen_origin[0] * 32 : 0;
    oz = w->gen_window ? w->gen_origin[1] * 32 : 0;
}

// The exception table of vx_gmath.h (built by voxelg_b200/build.py beside
// the library as vx_libm_exceptions.bin), loaded once per process.  It holds
// this host C library's powf / cosf / sinf results where they differ from
// vx_gmath.h's, so it must come from the C library the process runs on.
const std::vector<uint32_t> *lmx_table(std::string *err) {
    static std::mutex mu;
    static std::vector<uint32_t> blob;
    static std::string failure;
    static bool tried = false;
    std::lock_guard<std::mutex> lk(mu);
    if (!tried) {
        tried = true;
        Dl_info info{};
        std::string path = "vx_libm_exceptions.bin";
        if (dladdr(reinterpret_cast<void *>(&vx_gen_math_host), &info) && info.dli_fname) {
            std::string lib = info.dli_fname;
            const size_t slash = lib.rfind('/');
            if (slash != std::string::npos) path = lib.substr(0, slash + 1) + path;
        }
        FILE *f = std::fopen(path.c_str(), "rb");
        if (!f) {
            failure = "generator math table " + path +
                      " missing (python -m voxelg_b200.build writes it)";
        } else {
            std::fseek(f, 0, SEEK_END);
            const long bytes = std::ftell(f);
            std::fseek(f, 0, SEEK_SET);
            if (bytes > 0 && bytes % 4 == 0) {
                blob.resize((size_t)bytes / 4);
                if (std::fread(blob.data(), 4, blob.size(), f) != blob.size()) blob.clear();
            }
            std::fclose(f);
            char ver[33] = {0};
            if (blob.size() > vx::gm::LMX_HEADER) std::memcpy(ver, &blob[2], 32);
            if (blob.size() <= vx::gm::LMX_HEADER || blob[0] != vx::gm::LMX_MAGIC ||
                blob[1] != vx::gm::LMX_VERSION || blob[10] != vx::gm::LMX_FUNCS) {
                failure = "generator math table " + path + " is not a version-" +
                          std::to_string(vx::gm::LMX_VERSION) + " table";
                blob.clear();
            } else if (std::strcmp(ver, gnu_get_libc_version()) != 0) {
                failure = std::string("generator math table was built against C library ") +
                          ver + ", this process runs " + gnu_get_libc_version() +
                          " (rebuild: python -m voxelg_b200.build)";
                blob.clear();
            }
        }
    }
    if (blob.empty()) {
        if (err) *err = failure;
        return nullptr;
    }
    return &blob;
}

// the world's device copy of the table; caller holds w->mu
int world_lmx(VxWorld *w, const char *fn) {
    if (w->d_lmx) return VX_OK;
    std::string err;
    const std::vector<uint32_t> *t = lmx_table(&err);
    if (!t) {
        vx::set_error(std::string(fn) + ": " + err);
        return VX_ERR_INVALID;
    }
    VX_CK(cudaMalloc(&w->d_lmx, t->size() * 4));
    // once per world; synchronous, so that work on any stream may read it
    VX_CK(cudaMemcpy(w->d_lmx, t->data(), t->size() * 4, cudaMemcpyHostToDevice));
    return VX_OK;
}

// Lays out the generator's scratch -- the plan's ints (explicit plans),
// column words, tree headers and primitives -- uploads the ints through the
// pinned staging buffer, runs the kernels and waits.  Caller holds w->mu.
int run_gen_plan(VxWorld *w, uint64_t seed, vx::GenPlan &plan, const std::vector<int32_t> &ints) {
    auto up16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    const size_t plan_bytes = ints.size() * sizeof(int32_t);
    const size_t off_colw = up16(plan_bytes);
    const size_t off_hdr = off_colw + up16((size_t)plan.n_cols * 1024 * sizeof(uint32_t));
    const size_t off_prim = off_hdr + up16((size_t)plan.n_srcs * 12 * sizeof(int32_t));
    const size_t bytes = off_prim + (size_t)plan.n_srcs * vx::gen_prim_bytes_per_src();
    if (bytes > w->gen_cap) {
        VX_CK(cudaStreamSynchronize(w->stream));
        cudaFree(w->d_gen);
        w->d_gen = nullptr;
        w->gen_cap = 0;
        VX_CK(cudaMalloc(&w->d_gen, bytes));
        w->gen_cap = bytes;
    }
    uint8_t *base = static_cast<uint8_t *>(w->d_gen);
    if (plan_bytes > 0) {
        if (plan_bytes > w->h_gen_cap) {
            if (w->h_gen) cudaFreeHost(w->h_gen);
            w->h_gen = nullptr;
            w->h_gen_cap = 0;
            VX_CK(cudaHostAlloc(&w->h_gen, plan_bytes, cudaHostAllocDefault));
            w->h_gen_cap = plan_bytes;
        }
        std::memcpy(w->h_gen, ints.data(), plan_bytes);   // the previous call synchronized
        VX_CK(cudaMemcpyAsync(base, w->h_gen, plan_bytes, cudaMemcpyHostToDevice, w->stream));
        plan.jobs = reinterpret_cast<const int32_t *>(base);
        plan.cols = plan.jobs + (size_t)plan.n_jobs * vx::kGenJobInts;
        plan.srcs = plan.cols + (size_t)plan.n_cols * 2;
    }
    plan.colw = reinterpret_cast<uint32_t *>(base + off_colw);
    plan.hdr = reinterpret_cast<int32_t *>(base + off_hdr);
    plan.prims = base + off_prim;
    int rc = world_lmx(w, "chunk generator");
    if (rc != VX_OK) return rc;
    plan.lmx = w->d_lmx;
    vx::world_masks_changed(w);
    VX_CK(vx::launch_gen_slots(w->dw, seed, plan, w->stream));
    VX_CK(cudaStreamSynchronize(w->stream));
    return VX_OK;
}

// Generates the listed world chunks (x, y, z triples) into their toroidal
// slots: slot = (pos_mod(x, SX), y, pos_mod(z, SZ)), SX/SY/SZ the window in
// storage chunks (voxel.rs:507-537).  Caller holds w->mu.
int gen_chunks_locked(VxWorld *w, uint64_t seed, const int32_t *chunks, uint32_t n,
                      const char *fn) {
    const vx::Dims &d = w->dw.d;
    const int32_t sx_n = d.bx / 8, sy_n = d.by / 8, sz_n = d.bz / 8;
    // one job per slot: a later chunk for the same slot replaces an earlier
    // one, as a later install does in the reference
    std::vector<int64_t> last((size_t)sx_n * sy_n * sz_n, -1);
    std::vector<uint32_t> slot_of(n);
    for (uint32_t i = 0; i < n; ++i) {
        const int32_t cx = chunks[3 * i], cy = chunks[3 * i + 1], cz = chunks[3 * i + 2];
        if (cy < 0 || cy >= sy_n || cx < -(1 << 24) || cx >= (1 << 24) || cz < -(1 << 24) ||
            cz >= (1 << 24)) {
            vx::set_error(std::string(fn) + ": chunk y outside the window or x/z beyond +-2^24");
            return VX_ERR_INVALID;
        }
        slot_of[i] = (uint32_t)wrap(cx, sx_n) + (uint32_t)cy * (uint32_t)sx_n +
                     (uint32_t)wrap(cz, sz_n) * (uint32_t)(sx_n * sy_n);
        last[slot_of[i]] = i;
    }
    // distinct xz chunks (terrain columns) and 3x3 source chunks (trees),
    // numbered through a dense grid over the jobs' bounding box (widened by
    // the neighbour ring) when it is small, else through a hash map
    int32_t x0 = INT32_MAX, x1 = INT32_MIN, z0 = INT32_MAX, z1 = INT32_MIN;
    for (uint32_t i = 0; i < n; ++i) {
        x0 = std::min(x0, chunks[3 * i] - 1);
        x1 = std::max(x1, chunks[3 * i] + 1);
        z0 = std::min(z0, chunks[3 * i + 2] - 1);
        z1 = std::max(z1, chunks[3 * i + 2] + 1);
    }
    const int64_t gw = n ? (int64_t)x1 - x0 + 1 : 0, gh = n ? (int64_t)z1 - z0 + 1 : 0;
    const bool dense = gw * gh <= std::max<int64_t>(1 << 16, (int64_t)n * 16);
    std::vector<int32_t> col_grid(dense ? gw * gh : 0, -1), src_grid(dense ? gw * gh : 0, -1);
    std::unordered_map<uint64_t, int32_t> col_map, src_map;
    std::vector<int32_t> jobs, cols, srcs;
    auto index = [&](std::vector<int32_t> &grid, std::unordered_map<uint64_t, int32_t> &m,
                     std::vector<int32_t> &v, int32_t x, int32_t z) {
        int32_t *slot;
        if (dense) {
            slot = &grid[(size_t)(z - z0) * gw + (size_t)(x - x0)];
        } else {
            slot = &m.emplace(((uint64_t)(uint32_t)x << 32) | (uint32_t)z, -1).first->second;
        }
        if (*slot < 0) {
            *slot = (int32_t)(v.size() / 2);
            v.push_back(x);
            v.push_back(z);
        }
        return *slot;
    };
    jobs.reserve((size_t)n * vx::kGenJobInts);
    for (uint32_t i = 0; i < n; ++i) {
        const int32_t cx = chunks[3 * i], cy = chunks[3 * i + 1], cz = chunks[3 * i + 2];
        if (last[slot_of[i]] != (int64_t)i) continue;
        const int32_t sx = wrap(cx, sx_n), sz = wrap(cz, sz_n);
        int32_t j[vx::kGenJobInts] = {cx, cy, cz, sx, cy, sz,
                                      index(col_grid, col_map, cols, cx, cz)};
        for (int k = 0; k < 9; ++k)
            j[7 + k] = index(src_grid, src_map, srcs, cx + k % 3 - 1, cz + k / 3 - 1);
        jobs.insert(jobs.end(), j, j + vx::kGenJobInts);
    }
    n = (uint32_t)(jobs.size() / vx::kGenJobInts);
    if (w->slot_chunk.empty()) w->slot_chunk.assign((size_t)sx_n * sy_n * sz_n * 3, INT32_MIN);
    if (n == 0) return VX_OK;
    // [jobs | cols | srcs] ints, then column words, headers, primitives
    std::vector<int32_t> ints(jobs);
    ints.insert(ints.end(), cols.begin(), cols.end());
    ints.insert(ints.end(), srcs.begin(), srcs.end());
    vx::GenPlan plan{};
    plan.window = false;
    plan.n_jobs = n;
    plan.n_cols = (uint32_t)(cols.size() / 2);
    plan.n_srcs = (uint32_t)(srcs.size() / 2);
    int rc = run_gen_plan(w, seed, plan, ints);
    if (rc != VX_OK) return rc;
    // replay_edits_for_chunk (voxel.rs:571-603) for every generated chunk
    if (!w->edits.empty()) {
        std::vector<char> generated((size_t)sx_n * sy_n * sz_n, 0);
        std::vector<std::array<int32_t, 3>> gen_chunk((size_t)sx_n * sy_n * sz_n);
        for (uint32_t i = 0; i < n; ++i) {
            const int32_t *j = &jobs[(size_t)i * vx::kGenJobInts];
            const size_t slot = (size_t)j[3] + (size_t)j[4] * sx_n + (size_t)j[5] * sx_n * sy_n;
            generated[slot] = 1;
            gen_chunk[slot] = {j[0], j[1], j[2]};
        }
        std::vector<std::array<int32_t, 4>> replay;
        for (const auto &e : w->edits) {
            const int32_t cx = chunk_of(e.first[0]), cy = chunk_of(e.first[1]),
                          cz = chunk_of(e.first[2]);
            if (cy < 0 || cy >= sy_n) continue;
            const size_t slot = (size_t)wrap(cx, sx_n) + (size_t)cy * sx_n +
                                (size_t)wrap(cz, sz_n) * sx_n * sy_n;
            if (generated[slot] && gen_chunk[slot] == std::array<int32_t, 3>{cx, cy, cz})
                replay.push_back({e.first[0], e.first[1], e.first[2], e.second});
        }
        rc = write_edits_locked(w, replay);
        if (rc != VX_OK) return rc;
    }
    for (uint32_t i = 0; i < n; ++i) {
        const int32_t *j = &jobs[(size_t)i * vx::kGenJobInts];
        const size_t slot = (size_t)j[3] + (size_t)j[4] * sx_n + (size_t)j[5] * sx_n * sy_n;
        w->slot_chunk[slot * 3] = j[0];
        w->slot_chunk[slot * 3 + 1] = j[1];
        w->slot_chunk[slot * 3 + 2] = j[2];
    }
    return VX_OK;
}

// The world chunk shift_origin assigns slot (sx, sy, sz) for a window
// whose lower corner is chunk (ox, oz) (voxel.rs:515-521).
inline void wanted_chunk(const vx::Dims &d, int32_t ox, int32_t oz, int32_t sx, int32_t sy,
                         int32_t sz, int32_t out[3]) {
    out[0] = ox + wrap(sx - ox, d.bx / 8);
    out[1] = sy;
    out[2] = oz + wrap(sz - oz, d.bz / 8);
}

bool origin_in_range(int32_t ox, int32_t oz) {
    return ox > -(1 << 23) && ox < (1 << 23) && oz > -(1 << 23) && oz < (1 << 23);
}
}  // namespace

int vx_world_gen_chunks(VxWorld *w, uint64_t seed, const int32_t *chunks, uint32_t n) {
    vx::Range nvtx_range("vx_world_gen_chunks");
    if (!w || (n > 0 && !chunks)) {
        vx::set_error("vx_world_gen_chunks: null argument");
        return VX_ERR_INVALID;
    }
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    return gen_chunks_locked(w, seed, chunks, n, "vx_world_gen_chunks");
}

int vx_world_fill_window(VxWorld *w, uint64_t seed, int32_t origin_cx, int32_t origin_cz) {
    vx::Range nvtx_range("vx_world_fill_window");
    if (!w || !origin_in_range(origin_cx, origin_cz)) {
        vx::set_error("vx_world_fill_window: null world or origin beyond +-2^23 chunks");
        return VX_ERR_INVALID;
    }
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    const vx::Dims &d = w->dw.d;
    const int32_t sx_n = d.bx / 8, sy_n = d.by / 8, sz_n = d.bz / 8;
    vx::GenPlan plan{};
    plan.window = true;
    plan.ox = origin_cx;
    plan.oz = origin_cz;
    plan.n_jobs = (uint32_t)(sx_n * sy_n * sz_n);
    plan.n_cols = (uint32_t)(sx_n * sz_n);
    plan.n_srcs = (uint32_t)((sx_n + 2) * (sz_n + 2));
    rc = run_gen_plan(w, seed, plan, {});
    if (rc != VX_OK) return rc;
    // replay_edits_for_chunk (voxel.rs:571-603) over the whole window
    std::vector<std::array<int32_t, 4>> replay;
    for (const auto &e : w->edits) {
        const int64_t rx = (int64_t)e.first[0] - (int64_t)origin_cx * 32,
                      rz = (int64_t)e.first[2] - (int64_t)origin_cz * 32;
        if (rx >= 0 && rx < d.vx && e.first[1] >= 0 && e.first[1] < d.vy && rz >= 0 && rz < d.vz)
            replay.push_back({e.first[0], e.first[1], e.first[2], e.second});
    }
    rc = write_edits_locked(w, replay);
    if (rc != VX_OK) return rc;
    w->slot_chunk.resize((size_t)sx_n * sy_n * sz_n * 3);
    for (int32_t sz = 0; sz < sz_n; ++sz)
        for (int32_t sy = 0; sy < sy_n; ++sy)
            for (int32_t sx = 0; sx < sx_n; ++sx) {
                const size_t slot = (size_t)sx + (size_t)sy * sx_n + (size_t)sz * sx_n * sy_n;
                wanted_chunk(d, origin_cx, origin_cz, sx, sy, sz, &w->slot_chunk[slot * 3]);
            }
    w->gen_seed = seed;
    w->gen_origin[0] = origin_cx;
    w->gen_origin[1] = origin_cz;
    w->gen_window = true;
    return VX_OK;
}

int vx_world_shift_origin(VxWorld *w, int32_t origin_cx, int32_t origin_cz,
                          uint32_t *n_regenerated) {
    vx::Range nvtx_range("vx_world_shift_origin");
    if (!w || !origin_in_range(origin_cx, origin_cz)) {
        vx::set_error("vx_world_shift_origin: null world or origin beyond +-2^23 chunks");
        return VX_ERR_INVALID;
    }
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    if (!w->gen_window) {
        vx::set_error("vx_world_shift_origin: the world is not a generated window "
                      "(vx_world_fill_window first; uploads and vx_world_generate replace it)");
        return VX_ERR_INVALID;
    }
    const vx::Dims &d = w->dw.d;
    const int32_t sx_n = d.bx / 8, sy_n = d.by / 8, sz_n = d.bz / 8;
    std::vector<int32_t> chunks;
    for (int32_t sz = 0; sz < sz_n; ++sz)
        for (int32_t sy = 0; sy < sy_n; ++sy)
            for (int32_t sx = 0; sx < sx_n; ++sx) {
                int32_t c[3];
                wanted_chunk(d, origin_cx, origin_cz, sx, sy, sz, c);
                const size_t slot = (size_t)sx + (size_t)sy * sx_n + (size_t)sz * sx_n * sy_n;
                const int32_t *have = &w->slot_chunk[slot * 3];
                if (have[0] != c[0] || have[1] != c[1] || have[2] != c[2])
                    chunks.insert(chunks.end(), c, c + 3);
            }
    rc = gen_chunks_locked(w, w->gen_seed, chunks.data(), (uint32_t)(chunks.size() / 3),
                           "vx_world_shift_origin");
    if (rc != VX_OK) return rc;
    w->gen_origin[0] = origin_cx;
    w->gen_origin[1] = origin_cz;
    if (n_regenerated) *n_regenerated = (uint32_t)(chunks.size() / 3);
    return VX_OK;
}

int vx_checked_build(void) {
#ifdef VX_CHECKED
    return 1;
#else
    return 0;
#endif
}

int vx_world_oob(VxWorld *w, uint64_t *word, int32_t clear) {
    if (!w || !word) {
        vx::set_error("vx_world_oob: null argument");
        return VX_ERR_INVALID;
    }
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    // kernels of this world may run on any stream of the device
    VX_CK(cudaDeviceSynchronize());
    unsigned long long v = 0;
    VX_CK(cudaMemcpy(&v, w->dw.oob, sizeof(v), cudaMemcpyDeviceToHost));
    if (clear) VX_CK(cudaMemset(w->dw.oob, 0, sizeof(v)));
    *word = v;
    return take_fault(w, "vx_world_oob");
}

int vx_world_apply_edit(VxWorld *w, int32_t wx, int32_t wy, int32_t wz, uint8_t mat) {
    vx::Range nvtx_range("vx_world_apply_edit");
    if (!w || wx <= -(1 << 29) || wx >= (1 << 29) || wz <= -(1 << 29) || wz >= (1 << 29)) {
        vx::set_error("vx_world_apply_edit: null world or x/z beyond +-2^29");
        return VX_ERR_INVALID;
    }
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    w->edits[{wx, wy, wz}] = mat;
    int32_t ox, oz;
    window_corner(w, ox, oz);
    const vx::Dims &d = w->dw.d;
    const int64_t rx = (int64_t)wx - ox, rz = (int64_t)wz - oz;
    if (rx < 0 || rx >= d.vx || wy < 0 || wy >= d.vy || rz < 0 || rz >= d.vz) return VX_OK;
    return write_edits_locked(w, {{wx, wy, wz, (int32_t)mat}});
}

int vx_world_clear_edits(VxWorld *w) {
    if (!w) {
        vx::set_error("vx_world_clear_edits: null world");
        return VX_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(w->mu);
    w->edits.clear();
    return VX_OK;
}

namespace {
// .vxw: "VXW1", u32 version, i32 dims[3], u64 counts[4], the six arrays in
// voxelG's host layout, the edit log (u64 n, then i32 x, y, z + u8 mat each),
// the chunk generator's state (u8 window, u64 seed, i32 origin[2], u64 n,
// then n ints of the slot table).
constexpr char kVxwMagic[4] = {'V', 'X', 'W', '1'};
constexpr uint32_t kVxwVersion = 1;

struct File {
    FILE *f = nullptr;
    ~File() {
        if (f) fclose(f);
    }
};
bool put(FILE *f, const void *p, size_t n) { return n == 0 || fwrite(p, 1, n, f) == n; }
bool get(FILE *f, void *p, size_t n) { return n == 0 || fread(p, 1, n, f) == n; }
}  // namespace

int vx_world_save(VxWorld *w, const char *path) {
    if (!w || !path) {
        vx::set_error("vx_world_save: null argument");
        return VX_ERR_INVALID;
    }
    const vx::Dims d = w->dw.d;
    std::vector<VxBrick> bricks((size_t)d.n_bricks);
    std::vector<uint64_t> tm((size_t)d.n_tiles), cm((size_t)d.n_chunks), lm((size_t)d.n_l4);
    std::vector<uint8_t> bu((size_t)d.n_bricks), tu((size_t)d.n_tiles);
    int rc = vx_world_download(w, bricks.data(), tm.data(), cm.data(), lm.data(), bu.data(),
                               tu.data());
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    File out;
    out.f = fopen(path, "wb");
    if (!out.f) {
        vx::set_error(std::string("vx_world_save: cannot open ") + path);
        return VX_ERR_INVALID;
    }
    const int32_t dims[3] = {d.bx, d.by, d.bz};
    const uint64_t counts[4] = {(uint64_t)d.n_bricks, (uint64_t)d.n_tiles, (uint64_t)d.n_chunks,
                                (uint64_t)d.n_l4};
    bool ok = put(out.f, kVxwMagic, 4) && put(out.f, &kVxwVersion, 4) && put(out.f, dims, 12) &&
              put(out.f, counts, 32) && put(out.f, bricks.data(), bricks.size() * sizeof(VxBrick)) &&
              put(out.f, tm.data(), tm.size() * 8) && put(out.f, cm.data(), cm.size() * 8) &&
              put(out.f, lm.data(), lm.size() * 8) && put(out.f, bu.data(), bu.size()) &&
              put(out.f, tu.data(), tu.size());
    const uint64_t ne = w->edits.size();
    ok = ok && put(out.f, &ne, 8);
    for (const auto &e : w->edits) ok = ok && put(out.f, e.first.data(), 12) && put(out.f, &e.second, 1);
    const uint8_t win = w->gen_window ? 1 : 0;
    const uint64_t ns = w->slot_chunk.size();
    ok = ok && put(out.f, &win, 1) && put(out.f, &w->gen_seed, 8) && put(out.f, w->gen_origin, 8) &&
         put(out.f, &ns, 8) && put(out.f, w->slot_chunk.data(), ns * 4);
    ok = ok && fflush(out.f) == 0;
    if (!ok) {
        vx::set_error(std::string("vx_world_save: write failed: ") + path);
        return VX_ERR_INVALID;
    }
    return VX_OK;
}

int vx_world_load(VxWorld *w, const char *path) {
    if (!w || !path) {
        vx::set_error("vx_world_load: null argument");
        return VX_ERR_INVALID;
    }
    const vx::Dims d = w->dw.d;
    File in;
    in.f = fopen(path, "rb");
    if (!in.f) {
        vx::set_error(std::string("vx_world_load: cannot open ") + path);
        return VX_ERR_INVALID;
    }
    char magic[4];
    uint32_t version = 0;
    int32_t dims[3];
    uint64_t counts[4];
    if (!get(in.f, magic, 4) || std::memcmp(magic, kVxwMagic, 4) != 0 || !get(in.f, &version, 4) ||
        version != kVxwVersion || !get(in.f, dims, 12) || !get(in.f, counts, 32)) {
        vx::set_error(std::string("vx_world_load: not a .vxw file of this version: ") + path);
        return VX_ERR_INVALID;
    }
    if (dims[0] != d.bx || dims[1] != d.by || dims[2] != d.bz ||
        counts[0] != (uint64_t)d.n_bricks || counts[1] != (uint64_t)d.n_tiles ||
        counts[2] != (uint64_t)d.n_chunks || counts[3] != (uint64_t)d.n_l4) {
        vx::set_error("vx_world_load: the file's world dims differ from this world's");
        return VX_ERR_INVALID;
    }
    std::vector<VxBrick> bricks((size_t)d.n_bricks);
    std::vector<uint64_t> tm((size_t)d.n_tiles), cm((size_t)d.n_chunks), lm((size_t)d.n_l4);
    std::vector<uint8_t> bu((size_t)d.n_bricks), tu((size_t)d.n_tiles);
    bool ok = get(in.f, bricks.data(), bricks.size() * sizeof(VxBrick)) &&
              get(in.f, tm.data(), tm.size() * 8) && get(in.f, cm.data(), cm.size() * 8) &&
              get(in.f, lm.data(), lm.size() * 8) && get(in.f, bu.data(), bu.size()) &&
              get(in.f, tu.data(), tu.size());
    uint64_t ne = 0;
    ok = ok && get(in.f, &ne, 8) && ne <= ((uint64_t)1 << 32);
    std::map<std::array<int32_t, 3>, uint8_t> edits;
    for (uint64_t i = 0; ok && i < ne; ++i) {
        std::array<int32_t, 3> k;
        uint8_t m = 0;
        ok = get(in.f, k.data(), 12) && get(in.f, &m, 1);
        edits[k] = m;
    }
    uint8_t win = 0;
    uint64_t seed = 0, ns = 0;
    int32_t origin[2] = {0, 0};
    ok = ok && get(in.f, &win, 1) && get(in.f, &seed, 8) && get(in.f, origin, 8) &&
         get(in.f, &ns, 8) && (ns == 0 || ns == (uint64_t)(d.bx / 8) * (d.by / 8) * (d.bz / 8) * 3);
    std::vector<int32_t> slots((size_t)(ok ? ns : 0));
    ok = ok && get(in.f, slots.data(), slots.size() * 4);
    if (!ok) {
        vx::set_error(std::string("vx_world_load: truncated or inconsistent file: ") + path);
        return VX_ERR_INVALID;
    }
    int rc = vx_world_upload(w, bricks.data(), tm.data(), cm.data(), lm.data(), bu.data(),
                             tu.data());
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    w->edits = std::move(edits);
    w->gen_window = win != 0;
    w->gen_seed = seed;
    w->gen_origin[0] = origin[0];
    w->gen_origin[1] = origin[1];
    w->slot_chunk = std::move(slots);
    return VX_OK;
}

int vx_world_apply_dirty(VxWorld *w, const uint32_t *brick_idx, const VxBrick *bricks, size_t n,
                         void *stream) {
    vx::Range nvtx_range("vx_world_apply_dirty");
    if (!w || (n > 0 && (!brick_idx || !bricks))) {
        vx::set_error("vx_world_apply_dirty: null argument");
        return VX_ERR_INVALID;
    }
    if (n == 0) return VX_OK;
    if (n >= 0xFFFFFFFFull) {
        vx::set_error("vx_world_apply_dirty: more than 2^32 - 2 entries");
        return VX_ERR_INVALID;
    }
    const vx::Dims &d = w->dw.d;
    for (size_t i = 0; i < n; ++i) {
        if ((int64_t)brick_idx[i] >= d.n_bricks) {
            vx::set_error("vx_world_apply_dirty: brick index out of range");
            return VX_ERR_INVALID;
        }
    }
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    cudaStream_t s = stream ? as_stream(stream) : w->stream;
    if (!w->d_dirty_win) {
        VX_CK(cudaMalloc(&w->d_dirty_win, (size_t)d.n_bricks * sizeof(uint32_t)));
        VX_CK(cudaMemset(w->d_dirty_win, 0, (size_t)d.n_bricks * sizeof(uint32_t)));
        for (auto &b : w->dirty) VX_CK(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming));
        VX_CK(cudaEventCreateWithFlags(&w->dirty_last, cudaEventDisableTiming));
    }
    VxWorld::DirtyStage &b = w->dirty[w->dirty_calls & 1u];
    // the staging buffer's previous update has finished (usually long ago)
    VX_CK(cudaEventSynchronize(b.done));
    if (b.cap < n) {
        if (b.h_idx) cudaFreeHost(b.h_idx);
        if (b.h_bricks) cudaFreeHost(b.h_bricks);
        cudaFree(b.d_idx);
        cudaFree(b.d_bricks);
        b.h_idx = nullptr;
        b.h_bricks = nullptr;
        b.d_idx = nullptr;
        b.d_bricks = nullptr;
        b.cap = 0;
        VX_CK(cudaHostAlloc(reinterpret_cast<void **>(&b.h_idx), n * sizeof(uint32_t),
                            cudaHostAllocDefault));
        VX_CK(cudaHostAlloc(reinterpret_cast<void **>(&b.h_bricks), n * sizeof(VxBrick),
                            cudaHostAllocDefault));
        VX_CK(cudaMalloc(&b.d_idx, n * sizeof(uint32_t)));
        VX_CK(cudaMalloc(&b.d_bricks, n * sizeof(VxBrick)));
        b.cap = n;
    }
    std::memcpy(b.h_idx, brick_idx, n * sizeof(uint32_t));
    std::memcpy(b.h_bricks, bricks, n * sizeof(VxBrick));
    // updates apply in call order, whatever streams they come on
    if (w->dirty_calls > 0) VX_CK(cudaStreamWaitEvent(s, w->dirty_last, 0));
    VX_CK(cudaMemcpyAsync(b.d_idx, b.h_idx, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    VX_CK(cudaMemcpyAsync(b.d_bricks, b.h_bricks, n * sizeof(VxBrick), cudaMemcpyHostToDevice, s));
    vx::world_masks_changed(w);
    VX_CK(vx::launch_apply_dirty_last_wins(w->dw, w->d_dirty_win, b.d_idx, b.d_bricks, n, s));
    VX_CK(cudaEventRecord(b.done, s));
    VX_CK(cudaEventRecord(w->dirty_last, s));
    ++w->dirty_calls;
    if (!stream) {
        VX_CK(cudaStreamSynchronize(s));
    } else if (s != w->stream) {
        // the library's own calls on the world's stream come after the update
        VX_CK(cudaStreamWaitEvent(w->stream, w->dirty_last, 0));
    }
    return VX_OK;
}

int vx_raycast(VxWorld *w, const float cam[3], const float dir[3], const int32_t origin[3],
               VxPickHit *out) {
    if (!w || !cam || !dir || !origin || !out) {
        vx::set_error("vx_raycast: null argument");
        return VX_ERR_INVALID;
    }
    if (!vx::origin_ok(origin, "vx_raycast")) return VX_ERR_INVALID;
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    // the ray goes in with the launch's parameters and the result comes back
    // through the mapped block: one launch and one synchronization, no copies
    VX_CK(vx::launch_raycast_one(w->dw, origin, cam, dir, &w->pick_dev->out, &w->pick_dev->hit,
                                 w->stream));
    VX_CK(cudaStreamSynchronize(w->stream));
    *out = w->pick->out;
    return w->pick->hit ? 1 : 0;
}

int vx_raycast_batch(VxWorld *w, const int32_t origin[3], const float *cams_dev,
                     const float *dirs_dev, size_t n, VxPickHit *out_dev, int32_t *hit_dev,
                     void *stream) {
    vx::Range nvtx_range("vx_raycast_batch");
    if (!w || !origin || (n > 0 && (!cams_dev || !dirs_dev || !out_dev || !hit_dev))) {
        vx::set_error("vx_raycast_batch: null argument");
        return VX_ERR_INVALID;
    }
    if (!vx::origin_ok(origin, "vx_raycast_batch")) return VX_ERR_INVALID;
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    VX_CK(vx::launch_raycast(w->dw, origin, cams_dev, dirs_dev, n, out_dev, hit_dev,
                             as_stream(stream)));
    return VX_OK;
}

int vx_trace(VxWorld *w, const int32_t origin[3], const VxRay *rays_dev, size_t n,
             const VxTraceParams *p, VxHitRecord *out_dev, void *stream) {
    vx::Range nvtx_range("vx_trace");
    if (!w || !origin || (n > 0 && (!rays_dev || !out_dev))) {
        vx::set_error("vx_trace: null argument");
        return VX_ERR_INVALID;
    }
    if (!vx::origin_ok(origin, "vx_trace")) return VX_ERR_INVALID;
    int rc = check_params(p);
    if (rc != VX_OK) return rc;
    if ((reinterpret_cast<uintptr_t>(rays_dev) & 15u) || (reinterpret_cast<uintptr_t>(out_dev) & 7u)) {
        vx::set_error("vx_trace: rays must be 16-byte and records 8-byte aligned");
        return VX_ERR_INVALID;
    }
    rc = use_device(w);
    if (rc != VX_OK) return rc;
    vx::TraceArgs ta{};
    ta.w = w->dw;
    ta.p = *p;
    ta.ro[0] = origin[0]; ta.ro[1] = origin[1]; ta.ro[2] = origin[2];
    VX_CK(vx::launch_trace_rays(ta, rays_dev, n, out_dev, as_stream(stream)));
    return VX_OK;
}

int vx_render_primary(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                      VxHitRecord *rec_dev, VxShadowRecord *shadow_dev, void *stream) {
    vx::Range nvtx_range("vx_render_primary");
    if (!w || !rec_dev) {
        vx::set_error("vx_render_primary: null argument");
        return VX_ERR_INVALID;
    }
    int rc = check_frame(cam);
    if (rc == VX_OK) rc = check_params(p);
    if (rc != VX_OK) return rc;
    if ((reinterpret_cast<uintptr_t>(rec_dev) & 7u) || (reinterpret_cast<uintptr_t>(shadow_dev) & 7u)) {
        vx::set_error("vx_render_primary: records must be 8-byte aligned");
        return VX_ERR_INVALID;
    }
    rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    vx::FrameArgs fa = make_frame(w, cam, p);
    fa.rec = rec_dev;
    fa.shadow = shadow_dev;
    return run_frame(w, fa, as_stream(stream));
}

int vx_render_primary_rows(VxWorld *w, const VxCamera *cam, const VxTraceParams *p, uint32_t y0,
                           uint32_t y1, VxHitRecord *rec_dev, VxShadowRecord *shadow_dev,
                           void *stream) {
    vx::Range nvtx_range("vx_render_primary_rows");
    if (!w || !rec_dev) {
        vx::set_error("vx_render_primary_rows: null argument");
        return VX_ERR_INVALID;
    }
    int rc = check_frame(cam);
    if (rc == VX_OK) rc = check_params(p);
    if (rc != VX_OK) return rc;
    if (y0 > y1 || y1 > (uint32_t)cam->res_y) {
        vx::set_error("vx_render_primary_rows: need y0 <= y1 <= res_y");
        return VX_ERR_INVALID;
    }
    if ((reinterpret_cast<uintptr_t>(rec_dev) & 7u) || (reinterpret_cast<uintptr_t>(shadow_dev) & 7u)) {
        vx::set_error("vx_render_primary_rows: records must be 8-byte aligned");
        return VX_ERR_INVALID;
    }
    rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    vx::FrameArgs fa = make_frame(w, cam, p);
    fa.work = nullptr;  // the grid form renders a row range; the persistent one whole frames
    fa.y0 = y0;
    fa.y1 = y1;
    fa.rec = rec_dev;
    fa.shadow = shadow_dev;
    return run_frame(w, fa, as_stream(stream));
}

int vx_queue_default_tuning(VxQueueTuning *t) {
    if (!t) return VX_ERR_INVALID;
    std::memset(t, 0, sizeof(*t));
    t->block_threads = 128;
    t->refill_min = 32;
    t->ctas_per_sm = 0;
    t->sort = 1;
    return VX_OK;
}

namespace {
int check_queue(const VxWorld *w, const int32_t origin[3], const VxRay *rays_dev, size_t n,
                const VxTraceParams *p, const VxQueueTuning *t, const VxHitRecord *out_dev,
                const VxShadowRecord *shadow_dev, const char *fn) {
    if (!w || !origin || (n > 0 && (!rays_dev || !out_dev))) {
        vx::set_error(std::string(fn) + ": null argument");
        return VX_ERR_INVALID;
    }
    if (!vx::origin_ok(origin, fn)) return VX_ERR_INVALID;
    if (n >= 0xFFFFFFF0ull) {
        vx::set_error(std::string(fn) + ": at most 2^32 - 16 rays per queue");
        return VX_ERR_INVALID;
    }
    if ((reinterpret_cast<uintptr_t>(rays_dev) & 15u) || (reinterpret_cast<uintptr_t>(out_dev) & 7u) ||
        (reinterpret_cast<uintptr_t>(shadow_dev) & 7u)) {
        vx::set_error(std::string(fn) + ": rays must be 16-byte, records 8-byte aligned");
        return VX_ERR_INVALID;
    }
    if (t && ((t->block_threads != 64 && t->block_threads != 128 && t->block_threads != 256) ||
              t->refill_min < 1 || t->refill_min > 32 || t->ctas_per_sm < 0 ||
              (t->sort != 0 && t->sort != 1))) {
        vx::set_error(std::string(fn) + ": invalid VxQueueTuning");
        return VX_ERR_INVALID;
    }
    return check_params(p);
}

vx::TraceArgs trace_args(const VxWorld *w, const int32_t origin[3], const VxTraceParams *p) {
    vx::TraceArgs ta{};
    ta.w = w->dw;
    ta.p = *p;
    ta.ro[0] = origin[0];
    ta.ro[1] = origin[1];
    ta.ro[2] = origin[2];
    return ta;
}
}  // namespace

int vx_queue_run(VxWorld *w, const int32_t origin[3], const VxRay *rays_dev, size_t n,
                 const VxTraceParams *p, const VxQueueTuning *t, VxHitRecord *out_dev,
                 VxShadowRecord *shadow_dev, void *stream) {
    vx::Range nvtx_range("vx_queue_run");
    VxQueueTuning def;
    vx_queue_default_tuning(&def);
    if (!t) t = &def;
    int rc = check_queue(w, origin, rays_dev, n, p, t, out_dev, shadow_dev, "vx_queue_run");
    if (rc != VX_OK) return rc;
    rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    cudaStream_t s = as_stream(stream);
    if (w->qs.cap < n) VX_CK(cudaStreamSynchronize(s));
    VX_CK(w->qs.reserve(n));
    VX_CK(vx::launch_queue(trace_args(w, origin, p), rays_dev, n, out_dev, shadow_dev, *t, w->qs, s));
    return VX_OK;
}

int vx_queue_autotune(VxWorld *w, const int32_t origin[3], const VxRay *rays_dev, size_t n,
                      const VxTraceParams *p, VxHitRecord *out_dev, VxShadowRecord *shadow_dev,
                      int32_t reps, VxQueueTuning *best, float *best_ms) {
    int rc = check_queue(w, origin, rays_dev, n, p, nullptr, out_dev, shadow_dev,
                         "vx_queue_autotune");
    if (rc != VX_OK) return rc;
    if (!best || !best_ms || reps < 1 || reps > 100) {
        vx::set_error("vx_queue_autotune: need best, best_ms and 1 <= reps <= 100");
        return VX_ERR_INVALID;
    }
    rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    cudaStream_t s = w->stream;
    VX_CK(w->qs.reserve(n));
    if (!w->ev[0])
        for (int k = 0; k < 3; ++k) VX_CK(cudaEventCreate(&w->ev[k]));
    const vx::TraceArgs ta = trace_args(w, origin, p);
    unsigned long long ref_fp = 0;
    bool have_ref = false;
    float best_t = 1e30f;
    for (int bt : {64, 128, 256})
        for (int rm : {1, 8, 16, 24, 32})
            for (int so : {0, 1}) {
                VxQueueTuning t{};
                t.block_threads = bt;
                t.refill_min = rm;
                t.sort = so;
                std::vector<float> ms;
                for (int r = 0; r < reps + 1; ++r) {  // first run warms up
                    VX_CK(cudaEventRecord(w->ev[0], s));
                    VX_CK(vx::launch_queue(ta, rays_dev, n, out_dev, shadow_dev, t, w->qs, s));
                    VX_CK(cudaEventRecord(w->ev[1], s));
                    VX_CK(cudaEventSynchronize(w->ev[1]));
                    float m = 0.f;
                    VX_CK(cudaEventElapsedTime(&m, w->ev[0], w->ev[1]));
                    if (r > 0) ms.push_back(m);
                }
                std::sort(ms.begin(), ms.end());
                const float med = ms[ms.size() / 2];
                unsigned long long fp = 0;
                VX_CK(vx::queue_fingerprint(out_dev, n, shadow_dev, w->qs, s, &fp));
                if (!have_ref) {
                    ref_fp = fp;
                    have_ref = true;
                } else if (fp != ref_fp) {
                    vx::set_error("vx_queue_autotune: a tuning changed the records");
                    return VX_ERR_DEVICE;
                }
                if (med < best_t) {
                    best_t = med;
                    *best = t;
                }
            }
    *best_ms = best_t;
    return VX_OK;
}

int vx_project_dirty(VxWorld *w, const VxCamera *cam, const uint32_t *brick_idx, size_t n,
                     uint32_t *tile_mask_dev, void *stream) {
    if (!w || !tile_mask_dev || (n > 0 && !brick_idx)) {
        vx::set_error("vx_project_dirty: null argument");
        return VX_ERR_INVALID;
    }
    int rc = check_frame(cam);
    if (rc != VX_OK) return rc;
    for (size_t i = 0; i < n; ++i)
        if ((int64_t)brick_idx[i] >= w->dw.d.n_bricks) {
            vx::set_error("vx_project_dirty: brick index out of range");
            return VX_ERR_INVALID;
        }
    if (n == 0) return VX_OK;
    rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    cudaStream_t s = as_stream(stream);
    if (w->gate_cap < n) VX_CK(cudaStreamSynchronize(s));
    rc = ensure(&w->d_gate_idx, &w->gate_cap, n);
    if (rc != VX_OK) return rc;
    VX_CK(cudaMemcpyAsync(w->d_gate_idx, brick_idx, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    VX_CK(vx::launch_project_dirty(w->dw, *cam, w->d_gate_idx, n, tile_mask_dev, s));
    // the staging buffer is reused by the next call: finish this one first
    VX_CK(cudaStreamSynchronize(s));
    return VX_OK;
}

int vx_tile_refresh(uint32_t width, uint32_t height, uint32_t spread, uint32_t phase,
                    uint32_t *tile_mask_dev, void *stream) {
    if (!tile_mask_dev || width == 0 || height == 0 || width > 32768 || height > 32768 ||
        (spread > 0 && phase >= spread)) {
        vx::set_error("vx_tile_refresh: invalid argument");
        return VX_ERR_INVALID;
    }
    VX_CK(vx::launch_refresh_tiles((width + 7) / 8, (height + 7) / 8, spread, phase,
                                   tile_mask_dev, as_stream(stream)));
    return VX_OK;
}

int vx_render_primary_gated(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                            const uint32_t *tile_mask_dev, VxHitRecord *rec_dev,
                            VxShadowRecord *shadow_dev, void *stream) {
    if (!w || !rec_dev || !tile_mask_dev) {
        vx::set_error("vx_render_primary_gated: null argument");
        return VX_ERR_INVALID;
    }
    int rc = check_frame(cam);
    if (rc == VX_OK) rc = check_params(p);
    if (rc != VX_OK) return rc;
    if ((reinterpret_cast<uintptr_t>(rec_dev) & 7u) || (reinterpret_cast<uintptr_t>(shadow_dev) & 7u)) {
        vx::set_error("vx_render_primary_gated: records must be 8-byte aligned");
        return VX_ERR_INVALID;
    }
    rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    vx::FrameArgs fa = make_frame(w, cam, p);
    fa.rec = rec_dev;
    fa.shadow = shadow_dev;
    fa.tile_gate = tile_mask_dev;
    return run_frame(w, fa, as_stream(stream));
}

int vx_render_ao(VxWorld *w, const VxCamera *cam, const VxHitRecord *rec_dev, float *ao_dev,
                 void *stream) {
    vx::Range nvtx_range("vx_render_ao");
    if (!w || !rec_dev || !ao_dev) {
        vx::set_error("vx_render_ao: null argument");
        return VX_ERR_INVALID;
    }
    int rc = check_frame(cam);
    if (rc != VX_OK) return rc;
    if ((reinterpret_cast<uintptr_t>(rec_dev) & 7u) || (reinterpret_cast<uintptr_t>(ao_dev) & 3u)) {
        vx::set_error("vx_render_ao: records must be 8-byte and AO 4-byte aligned");
        return VX_ERR_INVALID;
    }
    rc = use_device(w);
    if (rc != VX_OK) return rc;
    VX_CK(vx::launch_ao(w->dw, *cam, rec_dev, ao_dev, as_stream(stream)));
    return VX_OK;
}

namespace {
// Enqueues one host-buffer frame: beam, then row bands whose copies to the
// host (copy stream) overlap the next band's traversal.  Frames alternate
// between two device buffers; a frame first waits, on the device, for the
// copies of the frame two calls back that used its buffer.  Caller holds
// w->mu.
// One frame into host memory on the world's two streams: the traversal in
// row bands on w->stream, each band copied on copy_stream once it is done.
// rec_host / shadow_host receive the full records; or, with packed_host set,
// each band is packed (16 bytes per pixel, shadows included) and only the
// packed form crosses to the host.
int enqueue_host_frame(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                       VxHitRecord *rec_host, VxShadowRecord *shadow_host,
                       VxPackedRecord *packed_host, uint32_t bands,
                       VxCompactRecord *compact_host = nullptr) {
    static_assert(kSyncBands <= sizeof(w->band_ev) / sizeof(w->band_ev[0]), "one event per band");
    static_assert(kAsyncBands <= kSyncBands, "one event per band");
    vx::FrameArgs fa = make_frame(w, cam, p);
    const size_t n = (size_t)fa.W * fa.H;
    const int buf = (int)(w->host_frames & 1u);
    if (!w->copy_stream) {
        VX_CK(cudaStreamCreateWithFlags(&w->copy_stream, cudaStreamNonBlocking));
        for (auto &e : w->band_ev) VX_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (!w->copy_done[0]) {
        for (auto &e : w->copy_done) VX_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    // the packed and compact forms share the device staging buffer (12 <= 16 bytes)
    const bool compact = compact_host != nullptr;
    const bool packed = packed_host != nullptr || compact;
    if (w->hrec_cap[buf] < n || w->hsh_cap[buf] < n || (packed && w->hpk_cap[buf] < n)) {
        VX_CK(cudaStreamSynchronize(w->copy_stream));   // no copy may read a freed buffer
        int rc = ensure(&w->hrec[buf], &w->hrec_cap[buf], n);
        if (rc == VX_OK) rc = ensure(&w->hsh[buf], &w->hsh_cap[buf], n);
        if (rc == VX_OK && packed) rc = ensure(&w->hpk[buf], &w->hpk_cap[buf], n);
        if (rc != VX_OK) return rc;
    }
    fa.rec = w->hrec[buf];
    fa.shadow = (shadow_host || packed) ? w->hsh[buf] : nullptr;
    VX_CK(cudaStreamWaitEvent(w->stream, w->copy_done[buf], 0));
    // bands of rows (the grid form only; the persistent form renders in one go)
    const uint32_t nb = fa.work ? 1u : bands;
    const uint32_t band = ((fa.H + nb - 1) / nb + 7u) & ~7u;
    if (fa.ta.p.flags & VX_F_BEAM) {
        int rc = ensure(&w->beam, &w->beam_cap, (size_t)fa.bw * fa.bh);
        if (rc != VX_OK) return rc;
        fa.beam = w->beam;
        VX_CK(vx::launch_beam(fa, w->beam, w->stream));
    }
    for (uint32_t b = 0; b < nb; ++b) {
        fa.y0 = std::min(fa.H, b * band);
        fa.y1 = std::min(fa.H, (b + 1) * band);
        if (fa.work) fa.y0 = 0, fa.y1 = fa.H;
        if (fa.y1 <= fa.y0) break;
        VX_CK(vx::launch_primary(fa, w->stream));
        const size_t r0 = (size_t)fa.y0 * fa.W, rn = (size_t)(fa.y1 - fa.y0) * fa.W;
        if (packed) {
            const uint32_t wx = (uint32_t)w->dw.d.vx, wy = (uint32_t)w->dw.d.vy;
            if (compact)
                VX_CK(vx::launch_pack_compact(fa.rec, fa.shadow, r0, rn, fa.ta.ro, wx, wy,
                                              reinterpret_cast<VxCompactRecord *>(w->hpk[buf]),
                                              fa.ta.w.fault, w->stream));
            else
                VX_CK(vx::launch_pack(fa.rec, fa.shadow, r0, rn, fa.ta.ro, wx, wy, w->hpk[buf],
                                      w->stream));
        }
        VX_CK(cudaEventRecord(w->band_ev[b], w->stream));
        VX_CK(cudaStreamWaitEvent(w->copy_stream, w->band_ev[b], 0));
        if (compact) {
            VX_CK(cudaMemcpyAsync(compact_host + r0,
                                  reinterpret_cast<VxCompactRecord *>(w->hpk[buf]) + r0,
                                  rn * sizeof(VxCompactRecord), cudaMemcpyDeviceToHost,
                                  w->copy_stream));
            continue;
        }
        if (packed) {
            VX_CK(cudaMemcpyAsync(packed_host + r0, w->hpk[buf] + r0, rn * sizeof(VxPackedRecord),
                                  cudaMemcpyDeviceToHost, w->copy_stream));
            continue;
        }
        VX_CK(cudaMemcpyAsync(rec_host + r0, fa.rec + r0, rn * sizeof(VxHitRecord),
                              cudaMemcpyDeviceToHost, w->copy_stream));
        if (shadow_host)
            VX_CK(cudaMemcpyAsync(shadow_host + r0, fa.shadow + r0, rn * sizeof(VxShadowRecord),
                                  cudaMemcpyDeviceToHost, w->copy_stream));
    }
    VX_CK(cudaEventRecord(w->copy_done[buf], w->copy_stream));
    ++w->host_frames;
    return VX_OK;
}

int host_frame_args(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                    VxHitRecord *rec_host, const char *fn) {
    if (!w || !rec_host) {
        vx::set_error(std::string(fn) + ": null argument");
        return VX_ERR_INVALID;
    }
    int rc = check_frame(cam);
    if (rc == VX_OK) rc = check_params(p);
    if (rc == VX_OK) rc = use_device(w);
    return rc;
}
}  // namespace

int vx_render_primary_host(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                           VxHitRecord *rec_host, VxShadowRecord *shadow_host) {
    vx::Range nvtx_range("vx_render_primary_host");
    int rc = host_frame_args(w, cam, p, rec_host, "vx_render_primary_host");
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    rc = enqueue_host_frame(w, cam, p, rec_host, shadow_host, nullptr, kSyncBands);
    if (rc != VX_OK) return rc;
    VX_CK(cudaStreamSynchronize(w->copy_stream));
    VX_CK(cudaStreamSynchronize(w->stream));
    return take_fault(w, "vx_render_primary_host");
}

int vx_render_primary_host_async(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                                 VxHitRecord *rec_host, VxShadowRecord *shadow_host) {
    vx::Range nvtx_range("vx_render_primary_host_async");
    int rc = host_frame_args(w, cam, p, rec_host, "vx_render_primary_host_async");
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    return enqueue_host_frame(w, cam, p, rec_host, shadow_host, nullptr, kAsyncBands);
}

int vx_render_host_wait(VxWorld *w) {
    if (!w) {
        vx::set_error("vx_render_host_wait: null world");
        return VX_ERR_INVALID;
    }
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    if (w->copy_stream) VX_CK(cudaStreamSynchronize(w->copy_stream));
    VX_CK(cudaStreamSynchronize(w->stream));
    return take_fault(w, "vx_render_host_wait");
}

namespace {
// the packed form's limits: a 32-bit window voxel index, 16-bit step counts
int packed_args(VxWorld *w, const VxTraceParams *p, const char *fn) {
    const uint64_t nvox = (uint64_t)w->dw.d.vx * (uint64_t)w->dw.d.vy * (uint64_t)w->dw.d.vz;
    if (nvox > (1ull << 32)) {
        vx::set_error(std::string(fn) + ": the window has more than 2^32 voxels");
        return VX_ERR_INVALID;
    }
    if (p->max_iters > 65535 || p->any_max_iters > 65535) {
        vx::set_error(std::string(fn) + ": max_iters and any_max_iters must be <= 65535");
        return VX_ERR_INVALID;
    }
    return VX_OK;
}
}  // namespace

int vx_render_primary_host_packed(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                                  VxPackedRecord *out_host) {
    vx::Range nvtx_range("vx_render_primary_host_packed");
    VxHitRecord *probe = reinterpret_cast<VxHitRecord *>(out_host);
    int rc = host_frame_args(w, cam, p, probe, "vx_render_primary_host_packed");
    if (rc == VX_OK) rc = packed_args(w, p, "vx_render_primary_host_packed");
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    rc = enqueue_host_frame(w, cam, p, nullptr, nullptr, out_host, kSyncBands);
    if (rc != VX_OK) return rc;
    VX_CK(cudaStreamSynchronize(w->copy_stream));
    VX_CK(cudaStreamSynchronize(w->stream));
    return take_fault(w, "vx_render_primary_host_packed");
}

int vx_render_primary_host_packed_async(VxWorld *w, const VxCamera *cam,
                                        const VxTraceParams *p, VxPackedRecord *out_host) {
    vx::Range nvtx_range("vx_render_primary_host_packed_async");
    VxHitRecord *probe = reinterpret_cast<VxHitRecord *>(out_host);
    int rc = host_frame_args(w, cam, p, probe, "vx_render_primary_host_packed_async");
    if (rc == VX_OK) rc = packed_args(w, p, "vx_render_primary_host_packed_async");
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    return enqueue_host_frame(w, cam, p, nullptr, nullptr, out_host, kAsyncBands);
}

namespace {
// the compact form's limits: a 30-bit window voxel index, 11 / 10-bit step counts
int compact_args(VxWorld *w, const VxTraceParams *p, const char *fn) {
    const uint64_t nvox = (uint64_t)w->dw.d.vx * (uint64_t)w->dw.d.vy * (uint64_t)w->dw.d.vz;
    if (nvox > (1ull << 30)) {
        vx::set_error(std::string(fn) + ": the window has more than 2^30 voxels");
        return VX_ERR_INVALID;
    }
    if (p->max_iters > 2047 || p->any_max_iters > 1023) {
        vx::set_error(std::string(fn) + ": max_iters must be <= 2047 and any_max_iters <= 1023");
        return VX_ERR_INVALID;
    }
    return VX_OK;
}
}  // namespace

int vx_render_primary_host_compact(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                                   VxCompactRecord *out_host) {
    vx::Range nvtx_range("vx_render_primary_host_compact");
    VxHitRecord *probe = reinterpret_cast<VxHitRecord *>(out_host);
    int rc = host_frame_args(w, cam, p, probe, "vx_render_primary_host_compact");
    if (rc == VX_OK) rc = compact_args(w, p, "vx_render_primary_host_compact");
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    rc = enqueue_host_frame(w, cam, p, nullptr, nullptr, nullptr, kSyncBands, out_host);
    if (rc != VX_OK) return rc;
    VX_CK(cudaStreamSynchronize(w->copy_stream));
    VX_CK(cudaStreamSynchronize(w->stream));
    return take_fault(w, "vx_render_primary_host_compact");
}

int vx_render_primary_host_compact_async(VxWorld *w, const VxCamera *cam,
                                         const VxTraceParams *p, VxCompactRecord *out_host) {
    vx::Range nvtx_range("vx_render_primary_host_compact_async");
    VxHitRecord *probe = reinterpret_cast<VxHitRecord *>(out_host);
    int rc = host_frame_args(w, cam, p, probe, "vx_render_primary_host_compact_async");
    if (rc == VX_OK) rc = compact_args(w, p, "vx_render_primary_host_compact_async");
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    return enqueue_host_frame(w, cam, p, nullptr, nullptr, nullptr, kAsyncBands, out_host);
}

namespace {
// vx_unpack_compact_records over [i0, i1): the compact words back to the
// 16-byte packed fields, then as vx_unpack_records
void unpack_compact_range(const VxCompactRecord *cr, size_t i0, size_t i1, const int32_t ro[3],
                          uint64_t wx, uint64_t wy, VxHitRecord *rec, VxShadowRecord *shadow);

// vx_unpack_records over [i0, i1)
void unpack_range(const VxPackedRecord *packed, size_t i0, size_t i1, const int32_t ro[3],
                  uint64_t wx, uint64_t wy, VxHitRecord *rec, VxShadowRecord *shadow) {
    // window index -> (rx, ry, rz): shifts and masks when wx and wy are
    // powers of two (every library world), else 32-bit divisions (an index
    // and wx, wy fit 32 bits; wx * wy may not, so it splits in two steps)
    const bool pow2 = (wx & (wx - 1)) == 0 && (wy & (wy - 1)) == 0;
    const uint32_t sx = pow2 ? (uint32_t)__builtin_ctzll(wx) : 0u;
    const uint32_t sy = pow2 ? (uint32_t)__builtin_ctzll(wy) : 0u;
    const uint32_t wx32 = (uint32_t)wx, wy32 = (uint32_t)wy;
    for (size_t i = i0; i < i1; ++i) {
        const VxPackedRecord &q = packed[i];
        if (rec) {
            VxHitRecord r;
            if (q.flags & 1u) {
                uint32_t rx, ry, rz;
                if (pow2) {
                    rx = q.voxel & (wx32 - 1u);
                    ry = (q.voxel >> sx) & (wy32 - 1u);
                    rz = (uint32_t)((uint64_t)q.voxel >> (sx + sy));
                } else {
                    const uint32_t row = q.voxel / wx32;
                    rx = q.voxel - row * wx32;
                    rz = row / wy32;
                    ry = row - rz * wy32;
                }
                r.voxel[0] = ro[0] + (int32_t)rx;
                r.voxel[1] = ro[1] + (int32_t)ry;
                r.voxel[2] = ro[2] + (int32_t)rz;
            } else {
                r.voxel[0] = r.voxel[1] = r.voxel[2] = 0;
            }
            r.face = q.face;
            r.mat = q.mat;
            r.flags = q.flags;
            r.pad = 0;
            r.t = q.t;
            r.steps = q.steps & 0xFFFFu;
            rec[i] = r;
        }
        if (shadow) {
            VxShadowRecord s;
            s.steps = q.steps >> 16;
            s.occluded = (uint8_t)(q.shadow & 1u);
            s.traced = (uint8_t)((q.shadow >> 1) & 1u);
            s.pad = 0;
            shadow[i] = s;
        }
    }
}
}  // namespace

namespace {
void unpack_compact_range(const VxCompactRecord *cr, size_t i0, size_t i1, const int32_t ro[3],
                          uint64_t wx, uint64_t wy, VxHitRecord *rec, VxShadowRecord *shadow) {
    constexpr size_t kBlock = 1024;
    VxPackedRecord tmp[kBlock];
    for (size_t b0 = i0; b0 < i1; b0 += kBlock) {
        const size_t nb = std::min(kBlock, i1 - b0);
        for (size_t j = 0; j < nb; ++j) {
            const uint32_t *w = cr[b0 + j].w;
            const uint32_t face3 = (w[2] >> 21) & 7u;
            const bool hit = face3 != 7u;
            VxPackedRecord &q = tmp[j];
            q.voxel = hit ? (w[0] & 0x3FFFFFFFu) : 0u;
            q.face = (uint8_t)(hit ? face3 : 0xFFu);
            q.mat = (uint8_t)(w[2] >> 24);
            q.flags = (uint8_t)(hit ? (1u | (((w[0] >> 30) & 1u) << 1)) : 0u);
            q.shadow = (uint8_t)((w[0] >> 31) | ((w[1] >> 31) << 1));
            const uint32_t tb = w[1] & 0x7FFFFFFFu;
            std::memcpy(&q.t, &tb, 4);
            q.steps = (w[2] & 0x7FFu) | (((w[2] >> 11) & 0x3FFu) << 16);
        }
        unpack_range(tmp, 0, nb, ro, wx, wy, rec ? rec + b0 : nullptr,
                     shadow ? shadow + b0 : nullptr);
    }
}
}  // namespace

int vx_unpack_compact_records(const VxCompactRecord *compact, size_t n,
                              const int32_t world_origin[3], const uint32_t window_voxels[3],
                              VxHitRecord *rec, VxShadowRecord *shadow) {
    if ((!compact && n) || !world_origin || !window_voxels) {
        vx::set_error("vx_unpack_compact_records: null argument");
        return VX_ERR_INVALID;
    }
    const uint64_t wx = window_voxels[0], wy = window_voxels[1];
    if (wx == 0 || wy == 0 || window_voxels[2] == 0) {
        vx::set_error("vx_unpack_compact_records: empty window");
        return VX_ERR_INVALID;
    }
    const size_t per = (size_t)1 << 18;
    const size_t hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t nt = std::min(hw, (n + per - 1) / per);
    if (nt <= 1) {
        unpack_compact_range(compact, 0, n, world_origin, wx, wy, rec, shadow);
        return VX_OK;
    }
    std::vector<std::thread> th;
    th.reserve(nt - 1);
    const size_t chunk = (n + nt - 1) / nt;
    for (size_t t = 1; t < nt; ++t) {
        const size_t i0 = std::min(n, t * chunk), i1 = std::min(n, (t + 1) * chunk);
        th.emplace_back(unpack_compact_range, compact, i0, i1, world_origin, wx, wy, rec, shadow);
    }
    unpack_compact_range(compact, 0, std::min(n, chunk), world_origin, wx, wy, rec, shadow);
    for (auto &t : th) t.join();
    return VX_OK;
}

int vx_unpack_records(const VxPackedRecord *packed, size_t n, const int32_t world_origin[3],
                      const uint32_t window_voxels[3], VxHitRecord *rec, VxShadowRecord *shadow) {
    if ((!packed && n) || !world_origin || !window_voxels) {
        vx::set_error("vx_unpack_records: null argument");
        return VX_ERR_INVALID;
    }
    const uint64_t wx = window_voxels[0], wy = window_voxels[1];
    if (wx == 0 || wy == 0 || window_voxels[2] == 0) {
        vx::set_error("vx_unpack_records: empty window");
        return VX_ERR_INVALID;
    }
    // host threads over chunks of at least 256k records (memory-bound copy)
    const size_t per = (size_t)1 << 18;
    const size_t hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t nt = std::min(hw, (n + per - 1) / per);
    if (nt <= 1) {
        unpack_range(packed, 0, n, world_origin, wx, wy, rec, shadow);
        return VX_OK;
    }
    std::vector<std::thread> th;
    th.reserve(nt - 1);
    const size_t chunk = (n + nt - 1) / nt;
    for (size_t t = 1; t < nt; ++t) {
        const size_t i0 = std::min(n, t * chunk), i1 = std::min(n, (t + 1) * chunk);
        th.emplace_back(unpack_range, packed, i0, i1, world_origin, wx, wy, rec, shadow);
    }
    unpack_range(packed, 0, std::min(n, chunk), world_origin, wx, wy, rec, shadow);
    for (auto &t : th) t.join();
    return VX_OK;
}

int vx_render_primary_stats(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                            uint64_t stats[4]) {
    if (!w || !stats) {
        vx::set_error("vx_render_primary_stats: null argument");
        return VX_ERR_INVALID;
    }
    int rc = check_frame(cam);
    if (rc == VX_OK) rc = check_params(p);
    if (rc != VX_OK) return rc;
    rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    vx::FrameArgs fa = make_frame(w, cam, p);
    const size_t n = (size_t)fa.W * fa.H;
    rc = ensure(&w->rec, &w->rec_cap, n);
    if (rc == VX_OK) rc = ensure(&w->sh, &w->sh_cap, n);
    if (rc == VX_OK) rc = ensure(&w->beam, &w->beam_cap, (size_t)fa.bw * fa.bh);
    if (rc != VX_OK) return rc;
    fa.rec = w->rec;
    fa.shadow = w->sh;
    fa.beam = w->beam;
    unsigned long long h[4] = {0, 0, 0, 0};
    VX_CK(cudaMemsetAsync(w->d_stats, 0, 4 * sizeof(unsigned long long), w->stream));
    if (fa.ta.p.flags & VX_F_BEAM) {
        fa.stats = w->d_stats;
        VX_CK(vx::launch_beam(fa, w->beam, w->stream));
    }
    fa.stats = w->d_stats + 2;
    VX_CK(vx::launch_primary(fa, w->stream));
    VX_CK(cudaMemcpyAsync(h, w->d_stats, sizeof(h), cudaMemcpyDeviceToHost, w->stream));
    VX_CK(cudaStreamSynchronize(w->stream));
    for (int k = 0; k < 4; ++k) stats[k] = h[k];
    return take_fault(w, "vx_render_primary_stats");
}

int vx_render_primary_timed(VxWorld *w, const VxCamera *cam, const VxTraceParams *p,
                            VxHitRecord *rec_dev, VxShadowRecord *shadow_dev, void *stream,
                            float ms[2]) {
    if (!w || !rec_dev || !ms) {
        vx::set_error("vx_render_primary_timed: null argument");
        return VX_ERR_INVALID;
    }
    int rc = check_frame(cam);
    if (rc == VX_OK) rc = check_params(p);
    if (rc != VX_OK) return rc;
    rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    if (!w->ev[0])
        for (int k = 0; k < 3; ++k) VX_CK(cudaEventCreate(&w->ev[k]));
    cudaStream_t s = as_stream(stream);
    vx::FrameArgs fa = make_frame(w, cam, p);
    fa.rec = rec_dev;
    fa.shadow = shadow_dev;
    VX_CK(cudaEventRecord(w->ev[0], s));
    if (fa.ta.p.flags & VX_F_BEAM) {
        rc = ensure(&w->beam, &w->beam_cap, (size_t)fa.bw * fa.bh);
        if (rc != VX_OK) return rc;
        fa.beam = w->beam;
        VX_CK(vx::launch_beam(fa, w->beam, s));
    }
    VX_CK(cudaEventRecord(w->ev[1], s));
    VX_CK(vx::launch_primary(fa, s));
    VX_CK(cudaEventRecord(w->ev[2], s));
    VX_CK(cudaEventSynchronize(w->ev[2]));
    VX_CK(cudaEventElapsedTime(&ms[0], w->ev[0], w->ev[1]));
    VX_CK(cudaEventElapsedTime(&ms[1], w->ev[1], w->ev[2]));
    return take_fault(w, "vx_render_primary_timed");
}

struct VxQueueGraph {
    int device = 0;
    vx::QueueScratch qs;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

int vx_queue_graph_create(VxWorld *w, const int32_t origin[3], const VxRay *rays_dev, size_t n,
                          const VxTraceParams *p, const VxQueueTuning *t, VxHitRecord *out_dev,
                          VxShadowRecord *shadow_dev, VxQueueGraph **out) {
    VxQueueTuning def;
    vx_queue_default_tuning(&def);
    if (!t) t = &def;
    int rc = check_queue(w, origin, rays_dev, n, p, t, out_dev, shadow_dev, "vx_queue_graph_create");
    if (rc != VX_OK) return rc;
    if (!out) return VX_ERR_INVALID;
    rc = use_device(w);
    if (rc != VX_OK) return rc;
    VxQueueGraph *g = new (std::nothrow) VxQueueGraph();
    if (!g) return VX_ERR_OOM;
    g->device = w->device;
    auto fail = [&](cudaError_t e) {
        vx::set_error(std::string("vx_queue_graph_create: ") + cudaGetErrorString(e));
        if (g->exec) cudaGraphExecDestroy(g->exec);
        if (g->graph) cudaGraphDestroy(g->graph);
        g->qs.release();
        delete g;
        return e == cudaErrorMemoryAllocation ? VX_ERR_OOM : VX_ERR_CUDA;
    };
    cudaError_t e = g->qs.reserve(n);
    if (e != cudaSuccess) return fail(e);
    cudaStream_t cs = nullptr;
    e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(e);
    const vx::TraceArgs ta = trace_args(w, origin, p);
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        // the counters reset themselves; clear them once more as a node so a
        // replay after an interrupted one still starts from zero
        cudaError_t e1 = cudaMemsetAsync(g->qs.work, 0, 2 * sizeof(uint32_t), cs);
        cudaError_t e2 = e1 == cudaSuccess
                             ? vx::launch_queue(ta, rays_dev, n, out_dev, shadow_dev, *t, g->qs, cs)
                             : e1;
        cudaError_t e3 = cudaStreamEndCapture(cs, &g->graph);
        e = e2 != cudaSuccess ? e2 : e3;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
    cudaStreamDestroy(cs);
    if (e != cudaSuccess) return fail(e);
    *out = g;
    return VX_OK;
}

int vx_queue_graph_launch(VxQueueGraph *g, void *stream) {
    if (!g || !g->exec) {
        vx::set_error("vx_queue_graph_launch: null graph");
        return VX_ERR_INVALID;
    }
    VX_CK(cudaSetDevice(g->device));
    VX_CK(cudaGraphLaunch(g->exec, as_stream(stream)));
    return VX_OK;
}

int vx_queue_graph_destroy(VxQueueGraph *g) {
    if (!g) return VX_OK;
    cudaSetDevice(g->device);
    cudaDeviceSynchronize();
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    g->qs.release();
    delete g;
    return VX_OK;
}

}  // extern "C"

int vx_gen_math(VxWorld *w, uint32_t fn, const float *in_dev, size_t n, float *out_dev,
                void *stream) {
    if (!w || fn >= vx::gm::LMX_FUNCS || ((!in_dev || !out_dev) && n)) {
        vx::set_error("vx_gen_math: null argument or unknown function");
        return VX_ERR_INVALID;
    }
    int rc = use_device(w);
    if (rc != VX_OK) return rc;
    std::lock_guard<std::mutex> lk(w->mu);
    rc = world_lmx(w, "vx_gen_math");
    if (rc != VX_OK) return rc;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : w->stream;
    if (!stream) VX_CK(cudaStreamSynchronize(w->stream));
    VX_CK(vx::launch_gen_math(w->d_lmx, fn, in_dev, n, out_dev, s));
    if (!stream) VX_CK(cudaStreamSynchronize(s));
    return VX_OK;
}

int vx_gen_math_host(uint32_t fn, const float *in, size_t n, float *out) {
    if (fn >= vx::gm::LMX_FUNCS || ((!in || !out) && n)) {
        vx::set_error("vx_gen_math_host: null argument or unknown function");
        return VX_ERR_INVALID;
    }
    std::string err;
    const std::vector<uint32_t> *t = lmx_table(&err);
    if (!t) {
        vx::set_error("vx_gen_math_host: " + err);
        return VX_ERR_INVALID;
    }
    const uint32_t *blob = t->data();
    for (size_t i = 0; i < n; ++i) {
        const float x = in[i];
        float v;
        if (fn == vx::gm::LMX_POW115) v = vx::gm::pow01(x, 1.15f);
        else if (fn == vx::gm::LMX_POW085) v = vx::gm::pow01(x, 0.85f);
        else if (fn == vx::gm::LMX_COS) v = vx::gm::cos_small(x);
        else v = vx::gm::sin_small(x);
        out[i] = vx::gm::lmx_fix(blob, fn, x, v);
    }
    return VX_OK;
}
