// vx_noalloc.cu -- vx_render_primary_noalloc: the primary frame for callers
// that cannot allocate device memory.
//
// Who needs it: hosts that reserve their whole device-memory budget up front
// and hand plugins only pre-allocated buffers (a game engine's frame loop, a
// sandboxed plugin host), where a cudaMalloc is either forbidden or a frame
// hitch, because cudaMalloc/cudaFree can synchronize the device.  Such a
// caller owns the world arrays and the output records; the one piece of
// scratch the frame needs -- the beam pre-pass depth grid -- lives here, in a
// file-scope device array that exists for as long as the library is loaded
// (every GPU that loads the module holds its 512 KiB until process exit).
//
// Set-up: the device address of the array is looked up once per CUDA
// context, by the first call made with that context current
// (cudaGetSymbolAddress); make that first call before any stream capture.
// The address is cached together with the context's unique id, so a call
// after cudaDeviceReset (which destroys the primary context and, with it,
// the module that holds the array) looks the address up again instead of
// using a stale one.  Host code must never pass the array's name to a kernel
// -- on the host it is only a stand-in, not a device address.
//
// Sharing: every call on a device uses the same array.  The beam kernel
// rewrites every cell a frame reads before the primary kernel reads it, so
// nothing needs clearing between calls, but calls that overlap on the GPU
// (two streams, or two threads without ordering) race on it.
//
// The beam pre-pass here reads the chunk masks with plain loads: a
// caller-owned world has no fault word through which a shared-memory staging
// copy that never landed could be reported.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "vx_internal.h"

namespace {

// Beam grid of a 3840x2160 frame: 480 x 270 cells.
constexpr size_t kMaxBeamCells = 480u * 270u;

static __device__ __align__(256) float g_beam_scratch[kMaxBeamCells];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct Cached {
    unsigned long long ctx_id;   // cuCtxGetId of the context the address belongs to
    float *addr;
};
Cached g_scratch[kMaxDevices] = {};

// cuCtxGetCurrent / cuCtxGetId through the runtime's driver entry points
// (the library links the static runtime, not libcuda).  Caller holds g_mu.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);
CtxGetCurrentFn g_get_cur = nullptr;
CtxGetIdFn g_get_id = nullptr;

// Unique id of the calling thread's current context, 0 when none is current.
int current_ctx_id(unsigned long long *id) {
    *id = 0;
    if (!g_get_cur || !g_get_id) {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa{}, qb{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
            qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b) {
            vx::set_error("vx_render_primary_noalloc: cuCtxGetCurrent/cuCtxGetId unavailable");
            return VX_ERR_CUDA;
        }
        g_get_cur = reinterpret_cast<CtxGetCurrentFn>(a);
        g_get_id = reinterpret_cast<CtxGetIdFn>(b);
    }
    CUcontext ctx = nullptr;
    if (g_get_cur(&ctx) != CUDA_SUCCESS) {
        vx::set_error("vx_render_primary_noalloc: cuCtxGetCurrent failed");
        return VX_ERR_CUDA;
    }
    if (ctx && g_get_id(ctx, id) != CUDA_SUCCESS) {
        vx::set_error("vx_render_primary_noalloc: cuCtxGetId failed");
        return VX_ERR_CUDA;
    }
    return VX_OK;
}

// Device address of g_beam_scratch in the current context of `dev`, looked
// up again whenever that context is not the one the cached address came
// from (cudaGetSymbolAddress also creates the device's primary context when
// no context is current yet).
int scratch_for(int dev, float **out) {
    std::lock_guard<std::mutex> lk(g_mu);
    unsigned long long id = 0;
    int rc = current_ctx_id(&id);
    if (rc != VX_OK) return rc;
    Cached &c = g_scratch[dev];
    if (!c.addr || id == 0 || c.ctx_id != id) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_beam_scratch);
        if (e != cudaSuccess || !p) {
            vx::set_error(std::string("vx_render_primary_noalloc: cudaGetSymbolAddress failed: ") +
                          cudaGetErrorString(e));
            return VX_ERR_CUDA;
        }
        rc = current_ctx_id(&id);
        if (rc != VX_OK) return rc;
        if (id == 0) {
            vx::set_error("vx_render_primary_noalloc: no current CUDA context");
            return VX_ERR_CUDA;
        }
        c.addr = static_cast<float *>(p);
        c.ctx_id = id;
    }
    *out = c.addr;
    return VX_OK;
}

}  // namespace

extern "C" int vx_render_primary_noalloc(const VxWorldView *view, const VxCamera *cam,
                                         const VxTraceParams *p, VxHitRecord *rec_dev,
                                         VxShadowRecord *shadow_dev, void *stream) {
    if (!view || !cam || !p || !rec_dev) {
        vx::set_error("vx_render_primary_noalloc: null argument");
        return VX_ERR_INVALID;
    }
    const int32_t bx = view->bricks_x, by = view->bricks_y, bz = view->bricks_z;
    if (bx <= 0 || by <= 0 || bz <= 0 || bx % 64 || bz % 64 || by % 16 || bx > 65536 ||
        by > 65536 || bz > 65536) {
        vx::set_error("vx_render_primary_noalloc: bricks_x/z must be multiples of 64, "
                      "bricks_y a multiple of 16");
        return VX_ERR_INVALID;
    }
    if (!view->occupancy || !view->materials || !view->tile_mask || !view->chunk_mask ||
        !view->l4_mask || !view->brick_uniform || !view->tile_uniform) {
        vx::set_error("vx_render_primary_noalloc: every world array must be given");
        return VX_ERR_INVALID;
    }
    if (!(cam->res_x >= 1.0f) || !(cam->res_y >= 1.0f) || cam->res_x > 32768.0f ||
        cam->res_y > 32768.0f || cam->res_x != (float)(uint32_t)cam->res_x ||
        cam->res_y != (float)(uint32_t)cam->res_y) {
        vx::set_error("vx_render_primary_noalloc: resolution must be an integer in [1, 32768]");
        return VX_ERR_INVALID;
    }
    if (!vx::origin_ok(cam->world_origin, "vx_render_primary_noalloc")) return VX_ERR_INVALID;
    if (p->max_iters < 0 || p->any_max_iters < 0 || p->max_iters > (1 << 20) ||
        p->any_max_iters > (1 << 20)) {
        vx::set_error("vx_render_primary_noalloc: iteration caps outside [0, 2^20]");
        return VX_ERR_INVALID;
    }
    // 8-byte loads and stores: a misaligned one faults the device, so refuse
    // it here, before anything is launched
    const uintptr_t mis = (reinterpret_cast<uintptr_t>(rec_dev) |
                           reinterpret_cast<uintptr_t>(shadow_dev) |
                           reinterpret_cast<uintptr_t>(view->occupancy) |
                           reinterpret_cast<uintptr_t>(view->tile_mask) |
                           reinterpret_cast<uintptr_t>(view->chunk_mask) |
                           reinterpret_cast<uintptr_t>(view->l4_mask)) & 7u;
    if (mis) {
        vx::set_error("vx_render_primary_noalloc: records, shadow records, occupancy and the "
                      "three mask arrays must be 8-byte aligned");
        return VX_ERR_INVALID;
    }
    vx::FrameArgs fa{};
    fa.W = (uint32_t)cam->res_x;
    fa.H = (uint32_t)cam->res_y;
    fa.bw = (fa.W + 7u) / 8u;
    fa.bh = (fa.H + 7u) / 8u;
    fa.y0 = 0;
    fa.y1 = fa.H;
    if ((p->flags & VX_F_BEAM) && (size_t)fa.bw * fa.bh > kMaxBeamCells) {
        vx::set_error("vx_render_primary_noalloc: frame too large for the static beam scratch "
                      "(at most 129600 beam cells, e.g. 3840x2160); use vx_render_primary");
        return VX_ERR_INVALID;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        vx::set_error("vx_render_primary_noalloc: no usable current CUDA device");
        return VX_ERR_CUDA;
    }
    float *beam = nullptr;
    if (p->flags & VX_F_BEAM) {
        int rc = scratch_for(dev, &beam);
        if (rc != VX_OK) return rc;
    }
    fa.ta.w.d = vx::make_dims(bx, by, bz);
    fa.ta.w.occ = const_cast<uint64_t *>(view->occupancy);
    fa.ta.w.mat = const_cast<uint8_t *>(view->materials);
    fa.ta.w.tile_mask = const_cast<uint64_t *>(view->tile_mask);
    fa.ta.w.chunk_mask = const_cast<uint64_t *>(view->chunk_mask);
    fa.ta.w.l4_mask = const_cast<uint64_t *>(view->l4_mask);
    fa.ta.w.brick_uniform = const_cast<uint8_t *>(view->brick_uniform);
    fa.ta.w.tile_uniform = const_cast<uint8_t *>(view->tile_uniform);
    fa.ta.p = *p;
    fa.ta.ro[0] = cam->world_origin[0];
    fa.ta.ro[1] = cam->world_origin[1];
    fa.ta.ro[2] = cam->world_origin[2];
    fa.cam = *cam;
    fa.rec = rec_dev;
    fa.shadow = shadow_dev;
    fa.beam = beam;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (p->flags & VX_F_BEAM) {
        e = vx::launch_beam(fa, beam, s);
        if (e != cudaSuccess) {
            vx::set_error(std::string("vx_render_primary_noalloc: beam launch: ") +
                          cudaGetErrorString(e));
            return VX_ERR_CUDA;
        }
    }
    e = vx::launch_primary(fa, s);
    if (e != cudaSuccess) {
        vx::set_error(std::string("vx_render_primary_noalloc: primary launch: ") +
                      cudaGetErrorString(e));
        return VX_ERR_CUDA;
    }
    return VX_OK;
}
