// vx_proposal.cpp -- C ABI of the learned start-distance proposal: parameter
// management, the on-device training loop (rays of random poses labelled by
// the plain DDA, Adam over strided-permutation batches) and the learned
// form of the primary frame.  Kernels live in vx_mlp.cu and vx_learned.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "voxrt.h"
#include "vx_internal.h"

struct VxProposal {
    int device = 0;
    vx::Mlp m;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    float *pred = nullptr;             // per-block proposals of the last frame
    float *depth = nullptr;            // per-tile proven depths of the last frame
    size_t pred_cap = 0, depth_cap = 0;
    unsigned long long *stats = nullptr;
    // frame timing (frame start / inference start / inference end / frame end)
    // and the fork / join of the inference on `stream` beside the frame
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join = nullptr;
};

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

uint64_t splitmix(uint64_t &x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
double uniform(uint64_t &x) { return (double)(splitmix(x) >> 11) * (1.0 / 9007199254740992.0); }
double normal(uint64_t &x) {
    const double u1 = std::max(uniform(x), 1e-300), u2 = uniform(x);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

// LeCun-normal weights, zero biases, output bias at log(150)
std::vector<float> init_params(uint64_t seed) {
    using namespace vx;
    std::vector<float> p(kMlpFloats, 0.0f);
    uint64_t s = seed ^ 0x5DEECE66Dull;
    const int H = kMlpHidden, I = kMlpIn;
    size_t o = 0;
    for (int r = 0; r < H; ++r)
        for (int c = 0; c < I; ++c) p[o + r * I + c] = c < 70 ? (float)(normal(s) / std::sqrt(70.0)) : 0.0f;
    o += H * I + H;
    for (int l = 0; l < 2; ++l) {
        for (int i = 0; i < H * H; ++i) p[o + i] = (float)(normal(s) / std::sqrt((double)H));
        o += H * H + H;
    }
    for (int i = 0; i < H; ++i) p[o + i] = (float)(normal(s) / std::sqrt((double)H));
    o += H;
    p[o] = std::log(150.0f);
    return p;
}

int check_prop(const VxProposal *p, const char *fn) {
    if (!p) {
        vx::set_error(std::string(fn) + ": null proposal");
        return VX_ERR_INVALID;
    }
    return VX_OK;
}

bool is_prime(uint64_t v) {
    if (v < 2) return false;
    for (uint64_t d = 2; d * d <= v; ++d)
        if (v % d == 0) return false;
    return true;
}

// a stride coprime to n near 0.618 n: k -> k * stride mod n is a permutation
uint64_t permutation_stride(uint64_t n) {
    if (n <= 2) return 1;
    for (uint64_t c = (uint64_t)(0.6180339887 * (double)n); c > 1; --c)
        if (is_prime(c) && std::gcd(c, n) == 1) return c;
    return 1;
}

template <typename T>
struct DevBuf {
    T *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)); }
};

// rays of `poses` random poses (rays_per_pose each) labelled by the plain DDA
int make_set(const vx::DevWorld &dw, const VxTrainConfig &c, uint32_t poses, uint64_t seed,
             VxRay *rays, float *targets, cudaStream_t s) {
    VxTraceParams tp;
    vx_default_params(&tp);
    tp.flags = c.flags & (VX_F_L4 | VX_F_LUT | VX_F_LOD);
    const size_t rpp = c.rays_per_pose, n = (size_t)poses * rpp;
    uint64_t rng = seed;
    const int32_t zero[3] = {0, 0, 0};
    for (uint32_t i = 0; i < poses; ++i) {
        const float pos[3] = {(float)((0.1 + 0.8 * uniform(rng)) * dw.d.vx),
                              (float)(c.y_min + (c.y_max - c.y_min) * uniform(rng)),
                              (float)((0.1 + 0.8 * uniform(rng)) * dw.d.vz)};
        const float yaw = (float)(6.283185307179586 * uniform(rng));
        const float pitch = (float)(c.pitch_min + (c.pitch_max - c.pitch_min) * uniform(rng));
        VxCamera cam;
        vx_camera_from_pose(pos, yaw, pitch, c.fov_y, c.width, c.height, zero, &cam);
        VX_CK(vx::mlp_pose_rays(cam, splitmix(rng), rpp, rays + (size_t)i * rpp, tp.max_dist, s));
    }
    DevBuf<VxHitRecord> rec;
    VX_CK(rec.alloc(n));
    vx::TraceArgs ta{};
    ta.w = dw;
    ta.p = tp;
    VX_CK(vx::launch_trace_rays(ta, rays, n, rec.p, s));
    VX_CK(vx::mlp_targets(rec.p, n, tp.max_dist, targets, s));
    VX_CK(cudaStreamSynchronize(s));
    return VX_OK;
}

// mean loss over a labelled set (batches of B, weighted by batch size)
int set_loss(VxProposal *p, const vx::DevWorld &dw, const VxRay *rays, const float *targets,
             size_t n, uint32_t B, float *feats, float *tgt, float *out) {
    const int32_t zero[3] = {0, 0, 0};
    double acc = 0.0;
    for (size_t b = 0; b < n; b += B) {
        const size_t cnt = std::min<size_t>(B, n - b);
        VX_CK(vx::mlp_features(dw, zero, rays, n, b, 1, cnt, feats, targets, tgt, p->stream));
        VX_CK(vx::mlp_grad(p->m, feats, tgt, (int)cnt, p->stream));
        float l = 0.0f;
        VX_CK(cudaMemcpyAsync(&l, p->m.loss, sizeof(float), cudaMemcpyDeviceToHost, p->stream));
        VX_CK(cudaStreamSynchronize(p->stream));
        acc += (double)l * (double)cnt;
    }
    *out = n ? (float)(acc / (double)n) : 0.0f;
    return VX_OK;
}

}  // namespace

extern "C" {

int vx_proposal_default_config(VxTrainConfig *c) {
    if (!c) return VX_ERR_INVALID;
    std::memset(c, 0, sizeof(*c));
    c->poses = 200;
    c->rays_per_pose = 81920;
    c->steps = 3000;
    c->batch = 16384;
    c->lr = 2e-3f;
    c->y_min = 100.0f;
    c->y_max = 200.0f;
    c->pitch_min = -0.6981317f;  // -40 deg
    c->pitch_max = 0.1745329f;   // +10 deg
    c->fov_y = 1.2217305f;       // 70 deg
    c->width = 1920;
    c->height = 1080;
    c->flags = VX_F_L4 | VX_F_LUT | VX_F_LOD;
    c->held_out_poses = 8;
    c->seed = 1;
    return VX_OK;
}

int vx_proposal_create(VxWorld *w, uint64_t seed, VxProposal **out) {
    if (!w || !out) {
        vx::set_error("vx_proposal_create: null argument");
        return VX_ERR_INVALID;
    }
    *out = nullptr;
    VxProposal *p = new (std::nothrow) VxProposal();
    if (!p) return VX_ERR_OOM;
    p->device = vx::world_device(w);
    auto fail = [&](cudaError_t e) {
        vx::set_error(std::string("vx_proposal_create: ") + cudaGetErrorString(e));
        vx::mlp_free(p->m);
        if (p->stream) cudaStreamDestroy(p->stream);
        delete p;
        return e == cudaErrorMemoryAllocation ? VX_ERR_OOM : VX_ERR_CUDA;
    };
    cudaError_t e = cudaSetDevice(p->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = vx::mlp_alloc(p->m);
    if (e != cudaSuccess) return fail(e);
    const std::vector<float> init = init_params(seed);
    e = cudaMemcpy(p->m.p, init.data(), init.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = vx::mlp_sync_bf16(p->m, p->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) return fail(e);
    *out = p;
    return VX_OK;
}

int vx_proposal_destroy(VxProposal *p) {
    if (!p) return VX_OK;
    cudaSetDevice(p->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    vx::mlp_free(p->m);
    if (p->pred) cudaFree(p->pred);
    if (p->depth) cudaFree(p->depth);
    if (p->stats) cudaFree(p->stats);
    for (auto &e : p->ev)
        if (e) cudaEventDestroy(e);
    if (p->fork) cudaEventDestroy(p->fork);
    if (p->join) cudaEventDestroy(p->join);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
    return VX_OK;
}

int vx_proposal_get_params(VxProposal *p, float *host, size_t n) {
    int rc = check_prop(p, "vx_proposal_get_params");
    if (rc != VX_OK) return rc;
    if (!host || n != (size_t)vx::kMlpFloats) {
        vx::set_error("vx_proposal_get_params: need VX_MLP_FLOATS floats");
        return VX_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(p->mu);
    VX_CK(cudaSetDevice(p->device));
    VX_CK(cudaMemcpyAsync(host, p->m.p, n * sizeof(float), cudaMemcpyDeviceToHost, p->stream));
    VX_CK(cudaStreamSynchronize(p->stream));
    return VX_OK;
}

int vx_proposal_set_params(VxProposal *p, const float *host, size_t n) {
    int rc = check_prop(p, "vx_proposal_set_params");
    if (rc != VX_OK) return rc;
    if (!host || n != (size_t)vx::kMlpFloats) {
        vx::set_error("vx_proposal_set_params: need VX_MLP_FLOATS floats");
        return VX_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(p->mu);
    VX_CK(cudaSetDevice(p->device));
    VX_CK(cudaMemcpyAsync(p->m.p, host, n * sizeof(float), cudaMemcpyHostToDevice, p->stream));
    VX_CK(cudaMemsetAsync(p->m.m, 0, n * sizeof(float), p->stream));
    VX_CK(cudaMemsetAsync(p->m.v, 0, n * sizeof(float), p->stream));
    p->m.adam_t = 0;
    VX_CK(vx::mlp_sync_bf16(p->m, p->stream));
    VX_CK(cudaStreamSynchronize(p->stream));
    return VX_OK;
}

int vx_proposal_features(VxProposal *p, VxWorld *w, const int32_t origin[3],
                         const VxRay *rays_dev, size_t n, float *feats_dev, void *stream) {
    int rc = check_prop(p, "vx_proposal_features");
    if (rc != VX_OK) return rc;
    if (!w || !origin || (n && (!rays_dev || !feats_dev))) {
        vx::set_error("vx_proposal_features: null argument");
        return VX_ERR_INVALID;
    }
    if (!vx::origin_ok(origin, "vx_proposal_features")) return VX_ERR_INVALID;
    VX_CK(cudaSetDevice(p->device));
    VX_CK(vx::mlp_features(vx::world_dev(w), origin, rays_dev, n, 0, 1, n, feats_dev, nullptr,
                           nullptr, as_stream(stream)));
    return VX_OK;
}

int vx_proposal_grad(VxProposal *p, const float *feats_dev, const float *target_dev,
                     uint32_t batch, float *grad_host, float *loss) {
    int rc = check_prop(p, "vx_proposal_grad");
    if (rc != VX_OK) return rc;
    if (!feats_dev || !target_dev || !grad_host || !loss || batch == 0 || batch > (1u << 20)) {
        vx::set_error("vx_proposal_grad: null argument or batch outside [1, 2^20]");
        return VX_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(p->mu);
    VX_CK(cudaSetDevice(p->device));
    VX_CK(vx::mlp_grad(p->m, feats_dev, target_dev, (int)batch, p->stream));
    VX_CK(cudaMemcpyAsync(grad_host, p->m.g, vx::kMlpFloats * sizeof(float),
                          cudaMemcpyDeviceToHost, p->stream));
    VX_CK(cudaMemcpyAsync(loss, p->m.loss, sizeof(float), cudaMemcpyDeviceToHost, p->stream));
    VX_CK(cudaStreamSynchronize(p->stream));
    return VX_OK;
}

int vx_proposal_infer(VxProposal *p, const float *feats_dev, size_t n, float *out_dev,
                      void *stream) {
    int rc = check_prop(p, "vx_proposal_infer");
    if (rc != VX_OK) return rc;
    if (n && (!feats_dev || !out_dev)) {
        vx::set_error("vx_proposal_infer: null argument");
        return VX_ERR_INVALID;
    }
    if (n > 0xFFFFFFF0u) {
        vx::set_error("vx_proposal_infer: n must be below 2^32 - 16");
        return VX_ERR_INVALID;
    }
    VX_CK(cudaSetDevice(p->device));
    VX_CK(vx::mlp_infer_features(p->m, feats_dev, n, out_dev, as_stream(stream)));
    return VX_OK;
}

int vx_proposal_train(VxProposal *p, VxWorld *w, const VxTrainConfig *c, float *loss_curve,
                      float held_out[2]) {
    vx::Range nvtx_range("vx_proposal_train");
    int rc = check_prop(p, "vx_proposal_train");
    if (rc != VX_OK) return rc;
    if (!w || !c || c->poses == 0 || c->rays_per_pose == 0 || c->batch == 0 ||
        c->batch > 65536u || !(c->lr > 0.0f) || c->width == 0 || c->height == 0 ||
        !(c->y_max >= c->y_min) || !(c->pitch_max >= c->pitch_min) ||
        (uint64_t)c->poses * c->rays_per_pose > (1ull << 31)) {
        vx::set_error("vx_proposal_train: invalid config (batch <= 65536, at most 2^31 rays)");
        return VX_ERR_INVALID;
    }
    if (vx::world_device(w) != p->device) {
        vx::set_error("vx_proposal_train: world and proposal on different devices");
        return VX_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(p->mu);
    VX_CK(cudaSetDevice(p->device));
    const vx::DevWorld dw = vx::world_dev(w);
    const size_t n = (size_t)c->poses * c->rays_per_pose;
    const size_t nh = (size_t)c->held_out_poses * std::min<uint32_t>(c->rays_per_pose, 8192u);
    DevBuf<VxRay> rays, rays_h;
    DevBuf<float> tg, tg_h, feats, tb, curve;
    VX_CK(rays.alloc(n));
    VX_CK(tg.alloc(n));
    VX_CK(feats.alloc((size_t)c->batch * vx::kMlpIn));
    VX_CK(tb.alloc(c->batch));
    VX_CK(curve.alloc(std::max<uint32_t>(c->steps, 1)));
    uint64_t seed = c->seed;
    rc = make_set(dw, *c, c->poses, splitmix(seed), rays.p, tg.p, p->stream);
    if (rc != VX_OK) return rc;
    if (nh) {
        VxTrainConfig ch = *c;
        ch.rays_per_pose = std::min<uint32_t>(c->rays_per_pose, 8192u);
        VX_CK(rays_h.alloc(nh));
        VX_CK(tg_h.alloc(nh));
        rc = make_set(dw, ch, c->held_out_poses, splitmix(seed) ^ 0xABCDEFull, rays_h.p, tg_h.p,
                      p->stream);
        if (rc != VX_OK) return rc;
    }
    float hl[2] = {0.0f, 0.0f};
    if (nh) {
        rc = set_loss(p, dw, rays_h.p, tg_h.p, nh, c->batch, feats.p, tb.p, &hl[0]);
        if (rc != VX_OK) return rc;
    }
    const uint64_t stride = permutation_stride(n);
    const int32_t zero[3] = {0, 0, 0};
    for (uint32_t step = 0; step < c->steps; ++step) {
        const double cosf_ = 0.5 * (1.0 + std::cos(3.141592653589793 * (double)step /
                                                   (double)std::max<uint32_t>(c->steps, 1)));
        const float lr = (float)(c->lr * (0.05 + 0.95 * cosf_));
        const uint64_t base = ((uint64_t)step * c->batch) % n;
        const uint32_t B = (uint32_t)std::min<size_t>(c->batch, n);
        VX_CK(vx::mlp_features(dw, zero, rays.p, n, base, stride, B, feats.p, tg.p, tb.p,
                               p->stream));
        VX_CK(vx::mlp_grad(p->m, feats.p, tb.p, (int)B, p->stream));
        VX_CK(cudaMemcpyAsync(curve.p + step, p->m.loss, sizeof(float), cudaMemcpyDeviceToDevice,
                              p->stream));
        VX_CK(vx::mlp_adam(p->m, lr, p->stream));
    }
    VX_CK(vx::mlp_sync_bf16(p->m, p->stream));
    if (loss_curve && c->steps)
        VX_CK(cudaMemcpyAsync(loss_curve, curve.p, c->steps * sizeof(float),
                              cudaMemcpyDeviceToHost, p->stream));
    VX_CK(cudaStreamSynchronize(p->stream));
    if (nh) {
        rc = set_loss(p, dw, rays_h.p, tg_h.p, nh, c->batch, feats.p, tb.p, &hl[1]);
        if (rc != VX_OK) return rc;
    }
    if (held_out) {
        held_out[0] = hl[0];
        held_out[1] = hl[1];
    }
    return VX_OK;
}

int vx_render_learned(VxWorld *w, VxProposal *prop, const VxCamera *cam, const VxTraceParams *p,
                      float scale, VxHitRecord *rec_dev, VxLearnedStats *stats, void *stream) {
    vx::Range nvtx_range("vx_render_learned");
    if (!w || !cam || !p || !rec_dev) {
        vx::set_error("vx_render_learned: null argument");
        return VX_ERR_INVALID;
    }
    if (!(cam->res_x >= 1.0f) || !(cam->res_y >= 1.0f) || cam->res_x > 32768.0f ||
        cam->res_y > 32768.0f || cam->res_x != std::floor(cam->res_x) ||
        cam->res_y != std::floor(cam->res_y)) {
        vx::set_error("vx_render_learned: camera resolution must be an integer in [1, 32768]");
        return VX_ERR_INVALID;
    }
    if (!vx::origin_ok(cam->world_origin, "vx_render_learned")) return VX_ERR_INVALID;
    if ((p->flags & (VX_F_BEAM | VX_F_SHADOW)) || p->max_iters < 0 || p->max_iters > (1 << 20) ||
        !(scale > 0.0f)) {
        vx::set_error("vx_render_learned: flags must not hold VX_F_BEAM / VX_F_SHADOW, "
                      "max_iters in [0, 2^20], scale > 0");
        return VX_ERR_INVALID;
    }
    if (reinterpret_cast<uintptr_t>(rec_dev) & 7u) {
        vx::set_error("vx_render_learned: records must be 8-byte aligned");
        return VX_ERR_INVALID;
    }
    const int device = vx::world_device(w);
    if (prop && prop->device != device) {
        vx::set_error("vx_render_learned: world and proposal on different devices");
        return VX_ERR_INVALID;
    }
    VX_CK(cudaSetDevice(device));
    cudaStream_t s = as_stream(stream);
    vx::TraceArgs ta{};
    // the world with its empty-space distance fields, rebuilt on s when its
    // masks changed since the last learned frame
    int rc = vx::world_dist_fields(w, s, &ta.w);
    if (rc != VX_OK) return rc;
    ta.p = *p;
    for (int k = 0; k < 3; ++k) ta.ro[k] = cam->world_origin[k];
    // one proven depth per 8 x 4 pixel tile (the ray bundle of the frustum
    // pre-pass) and one proposal per 16 x 8 pixels
    const uint32_t W = (uint32_t)cam->res_x, H = (uint32_t)cam->res_y;
    const size_t n_tiles = (size_t)((W + vx::kLearnedTileW - 1u) / vx::kLearnedTileW) *
                           ((H + vx::kLearnedTileH - 1u) / vx::kLearnedTileH);
    const size_t n_props = (size_t)((W + vx::kLearnedPropW - 1u) / vx::kLearnedPropW) *
                           ((H + vx::kLearnedPropH - 1u) / vx::kLearnedPropH);
    // scratch: the proposal's, or the world's (and temporary statistics
    // scratch) for a call without it
    std::unique_lock<std::mutex> lk;
    unsigned long long *d_stats = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    if (prop) {
        lk = std::unique_lock<std::mutex>(prop->mu);
        if (prop->pred_cap < n_props) {
            if (prop->pred) cudaFree(prop->pred);
            prop->pred = nullptr;
            prop->pred_cap = 0;
            VX_CK(cudaMalloc(&prop->pred, n_props * sizeof(float)));
            prop->pred_cap = n_props;
        }
        if (prop->depth_cap < n_tiles) {
            if (prop->depth) cudaFree(prop->depth);
            prop->depth = nullptr;
            prop->depth_cap = 0;
            VX_CK(cudaMalloc(&prop->depth, n_tiles * sizeof(float)));
            prop->depth_cap = n_tiles;
        }
        if (!prop->fork) {
            VX_CK(cudaEventCreateWithFlags(&prop->fork, cudaEventDisableTiming));
            VX_CK(cudaEventCreateWithFlags(&prop->join, cudaEventDisableTiming));
        }
        if (stats) {
            if (!prop->stats) VX_CK(cudaMalloc(&prop->stats, 8 * sizeof(unsigned long long)));
            if (!prop->ev[0])
                for (auto &e : prop->ev) VX_CK(cudaEventCreate(&e));
            d_stats = prop->stats;
            for (int k = 0; k < 4; ++k) ev[k] = prop->ev[k];
        }
    }
    // a statistics call without a proposal uses temporary scratch, released
    // on every path out of this function
    struct Temp {
        unsigned long long *stats = nullptr;
        cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
        ~Temp() {
            if (stats) cudaFree(stats);
            for (auto &x : ev)
                if (x) cudaEventDestroy(x);
        }
    } temp;
    if (!prop && stats) {
        VX_CK(cudaMalloc(&temp.stats, 8 * sizeof(unsigned long long)));
        for (auto &x : temp.ev) VX_CK(cudaEventCreate(&x));
        d_stats = temp.stats;
        for (int k = 0; k < 4; ++k) ev[k] = temp.ev[k];
    }
    float *depth = prop ? prop->depth : nullptr;
    if (!prop) {
        rc = vx::world_learned_depth(w, n_tiles, &depth);
        if (rc != VX_OK) return rc;
    }
    // s: [ev0] pre-pass (proofs + proposals) -> frame [ev3]
    cudaError_t e = cudaSuccess;
    if (stats) e = cudaMemsetAsync(d_stats, 0, 8 * sizeof(unsigned long long), s);
    if (e == cudaSuccess && stats) e = cudaEventRecord(ev[0], s);
    const bool proof = e == cudaSuccess && vx::learned_proof_ok(ta);
    if (proof)
        e = vx::launch_learned_prepass(ta, *cam, depth, prop ? &prop->m : nullptr,
                                       prop ? prop->pred : nullptr, d_stats, s);
    if (e == cudaSuccess)
        e = vx::launch_learned(ta, *cam, proof ? depth : nullptr,
                               proof && prop ? prop->pred : nullptr, scale, rec_dev, d_stats, s);
    if (e == cudaSuccess && stats) e = cudaEventRecord(ev[3], s);
    if (e == cudaSuccess && stats) e = cudaEventSynchronize(ev[3]);
    if (e == cudaSuccess && stats) {
        unsigned long long h[8];
        e = cudaMemcpy(h, d_stats, sizeof(h), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) {
            stats->none = h[0];
            stats->partial = h[1];
            stats->accepted = h[2];
            stats->miss = h[3];
            stats->cells = h[4];
            stats->iters = h[5];
            stats->fallback = h[6];
            stats->rays = h[7];
            stats->infer_ms = 0.0f;  // inside the pre-pass, beside the proofs
            e = cudaEventElapsedTime(&stats->trace_ms, ev[0], ev[3]);
        }
    }
    if (e != cudaSuccess) {
        vx::set_error(std::string("vx_render_learned: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? VX_ERR_OOM : VX_ERR_CUDA;
    }
    return VX_OK;
}

}  // extern "C"
