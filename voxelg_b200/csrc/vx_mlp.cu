// vx_mlp.cu -- the learned start-distance proposal: a 70->64->64->64->1 MLP
// with GELU (tanh form) that predicts log(first-hit t) of a ray from 6 ray
// values and the 64 tile bits of the chunk holding the ray origin.
//
//   inference  BF16 tensor cores (mma.sync, FP32 accumulation), in
//              vx_mlp_infer.cuh;
//   training   FP32 kernels: tiled GEMM (split-K with atomics for the weight
//              gradients), bias + GELU forward/backward, MSE loss, Adam.
//
// Features (80 columns, 70 used): origin mod 64 / 64 (3), direction (3), the
// 64 child bits of the origin chunk's tile mask (bit x + z*4 + y*16 of
// chunk_mask, src/voxel.rs:282-294), 10 zero columns.  The proposal only
// decides how far the exact traversal verifies before restarting; records
// never depend on its value, so this file uses ordinary float code
// generation (contraction, approximate tanh).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "vx_internal.h"
#include "vx_mlp_infer.cuh"

namespace vx {

namespace {

template <bool FRAME>
__global__ void __launch_bounds__(128) k_mlp_infer(InferArgs a) {
    mlp_infer_body<FRAME>(a, blockIdx.x, gridDim.x);
}

// ------------------------------------------------------------- training
// C[M][N] = sum_k A(m,k) B(k,n); A(m,k) = A[m*sam + k*sak], B likewise.
// 64x64 tile per CTA, 16x16 threads x 4x4 outputs; blockIdx.z splits K
// (partial sums added with atomics when split > 1; C pre-zeroed then).
__global__ void __launch_bounds__(256) k_sgemm(int M, int N, int K, const float *A, long sam,
                                               long sak, const float *B, long sbk, long sbn,
                                               float *C, long scm, long scn, int split) {
    __shared__ float As[16][65], Bs[16][65];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int kchunk = (K + split - 1) / split;
    const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
    float acc[4][4] = {};
    for (int k0 = kb; k0 < ke; k0 += 16) {
        for (int i = threadIdx.x; i < 16 * 64; i += 256) {
            // walk the contiguous dimension fastest for coalesced loads
            int kk, mm;
            if (sak == 1) { kk = i & 15; mm = i >> 4; } else { kk = i >> 6; mm = i & 63; }
            const int k = k0 + kk;
            As[kk][mm] = (k < ke && m0 + mm < M) ? A[(long)(m0 + mm) * sam + (long)k * sak] : 0.f;
            int kb2, nn;
            if (sbk == 1) { kb2 = i & 15; nn = i >> 4; } else { kb2 = i >> 6; nn = i & 63; }
            const int k2 = k0 + kb2;
            Bs[kb2][nn] = (k2 < ke && n0 + nn < N) ? B[(long)k2 * sbk + (long)(n0 + nn) * sbn] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                av[i] = As[kk][ty * 4 + i];
                bv[i] = Bs[kk][tx * 4 + i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] += av[i] * bv[j];
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int m = m0 + ty * 4 + i, n = n0 + tx * 4 + j;
            if (m < M && n < N) {
                float *c = C + (long)m * scm + (long)n * scn;
                if (split > 1) atomicAdd(c, acc[i][j]);
                else *c = acc[i][j];
            }
        }
}

__device__ __forceinline__ float gelu_f(float x) {
    return 0.5f * x * (1.0f + tanhf(0.7978845608f * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float th = tanhf(0.7978845608f * (x + 0.044715f * x * x * x));
    return 0.5f * (1.0f + th) +
           0.5f * x * (1.0f - th * th) * 0.7978845608f * (1.0f + 3.0f * 0.044715f * x * x);
}

// Z[b][j] += bias[j]; A = GELU(Z)
__global__ void k_bias_gelu(float *Z, float *Aout, const float *bias, long n) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float z = Z[i] + bias[i & (kH - 1)];
    Z[i] = z;
    Aout[i] = gelu_f(z);
}

// dZ = dA * GELU'(Z)
__global__ void k_gelu_back(const float *dA, const float *Z, float *dZ, long n) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dZ[i] = dA[i] * gelu_grad(Z[i]);
}

// y = A3 . wo + bo; dY = 2 (y - target) / B; loss += (y - target)^2 / B
__global__ void k_out_loss(const float *A3, const float *p, const float *target, int B, float *y,
                           float *dY, float *loss) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (b < B) {
        float s = p[kBo];
        for (int j = 0; j < kH; ++j) s += A3[(long)b * kH + j] * p[kWo + j];
        y[b] = s;
        const float e = s - target[b];
        dY[b] = 2.0f * e / (float)B;
        l = e * e / (float)B;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xFFFFFFFFu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// dA3[b][j] = dY[b] wo[j]; g_wo[j] += sum_b dY[b] A3[b][j]; g_bo += sum_b dY[b]
// (blockDim 256 = 4 samples x 64 columns)
__global__ void k_out_back(const float *A3, const float *dY, const float *p, int B, float *dA3,
                           float *grad) {
    const int j = threadIdx.x & 63;
    float gw = 0.f, gb = 0.f;
    for (int b = blockIdx.x * 4 + (threadIdx.x >> 6); b < B; b += gridDim.x * 4) {
        dA3[(long)b * kH + j] = dY[b] * p[kWo + j];
        gw += dY[b] * A3[(long)b * kH + j];
        if (j == 0) gb += dY[b];
    }
    atomicAdd(grad + kWo + j, gw);
    if (j == 0) atomicAdd(grad + kBo, gb);
}

// column sums of dZ [B][64] into grad[off + j]
__global__ void k_bias_grad(const float *dZ, int B, float *grad, int off) {
    const int j = threadIdx.x & 63;
    float s = 0.f;
    for (int b = blockIdx.x * 4 + (threadIdx.x >> 6); b < B; b += gridDim.x * 4)
        s += dZ[(long)b * kH + j];
    atomicAdd(grad + off + j, s);
}

__global__ void k_adam(float *p, const float *g, float *m, float *v, int n, float lr, float b1,
                       float b2, float eps, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// f32 W1, W2, W3 -> padded bf16 rows
__global__ void k_to_bf16(const float *p, __nv_bfloat16 *w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kW16) return;
    float v = 0.f;
    if (i < kH * kS1) {
        const int r = i / kS1, c = i % kS1;
        if (c < kIn) v = p[kW1 + r * kIn + c];
    } else {
        const int j = i - kH * kS1, which = j / (kH * kS2), jj = j % (kH * kS2);
        const int r = jj / kS2, c = jj % kS2;
        if (c < kH) v = p[(which == 0 ? kW2 : kW3) + r * kH + c];
    }
    w[i] = __float2bfloat16_rn(v);
}

// features of rays idx(j) = ((base + j) % n) * mult % n (f32, 80 columns)
// and their targets gathered alongside; mult coprime to n permutes the set
__global__ void k_features(DevWorld w, int32_t rox, int32_t roy, int32_t roz, const VxRay *rays,
                           unsigned long long n, unsigned long long base, unsigned long long mult,
                           unsigned long long count, float *feats, const float *tsrc,
                           float *tdst) {
    const unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const unsigned long long i = (((base + j) % n) * mult) % n;
    const int32_t ro[3] = {rox, roy, roz};
    const VxRay r = rays[i];
    const float o[3] = {r.org[0], r.org[1], r.org[2]};
    const float d[3] = {r.dir[0], r.dir[1], r.dir[2]};
    const uint64_t m = origin_chunk_word(w, ro, o);
    float *f = feats + j * kIn;
#pragma unroll 4
    for (int c = 0; c < kIn; ++c) f[c] = feature(o, d, m, c);
    if (tsrc) tdst[j] = tsrc[i];
}

// target: log of the plain DDA's first-hit t, or of the distance budget for a miss
__global__ void k_targets(const VxHitRecord *rec, size_t n, float max_dist, float *target) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool hit = (rec[i].flags & 1u) != 0u;
    target[i] = logf(fmaxf(hit ? rec[i].t : max_dist, 1.0f));
}

// rays of one camera through hashed random pixel positions
__global__ void k_pose_rays(VxCamera c, unsigned long long seed, size_t n, VxRay *rays,
                            float max_dist) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long h = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    h ^= h >> 30; h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 27; h *= 0x94D049BB133111EBull;
    h ^= h >> 31;
    const float u = (float)(h & 0xFFFFFFull) * (1.0f / 16777216.0f);
    const float v = (float)((h >> 24) & 0xFFFFFFull) * (1.0f / 16777216.0f);
    const float ax = (u * 2.0f - 1.0f) * c.tan_half_fov * (c.res_x / c.res_y);
    const float by = (1.0f - v * 2.0f) * c.tan_half_fov;
    const float x = (c.forward[0] + c.right[0] * ax) + c.up[0] * by;
    const float y = (c.forward[1] + c.right[1] * ax) + c.up[1] * by;
    const float z = (c.forward[2] + c.right[2] * ax) + c.up[2] * by;
    const float l = sqrtf(x * x + y * y + z * z);
    VxRay r;
    r.org[0] = c.origin[0]; r.org[1] = c.origin[1]; r.org[2] = c.origin[2];
    r.dir[0] = x / l; r.dir[1] = y / l; r.dir[2] = z / l;
    r.tmax = max_dist;
    r.kind = 0;
    rays[i] = r;
}

unsigned nblk(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t mlp_alloc(Mlp &m) {
    cudaError_t e = cudaMalloc(&m.p, kMlpFloats * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m.g, kMlpFloats * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m.m, kMlpFloats * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m.v, kMlpFloats * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m.w16, kW16 * sizeof(uint16_t));
    if (e == cudaSuccess) e = cudaMalloc(&m.loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(m.m, 0, kMlpFloats * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(m.v, 0, kMlpFloats * sizeof(float));
    return e;
}

void mlp_free(Mlp &m) {
    for (float *q : {m.p, m.g, m.m, m.v, m.z1, m.a1, m.z2, m.a2, m.z3, m.a3, m.y, m.dy, m.da,
                     m.dz, m.loss})
        if (q) cudaFree(q);
    if (m.w16) cudaFree(m.w16);
    m = Mlp();
}

static cudaError_t mlp_reserve(Mlp &m, size_t B) {
    if (m.cap >= B) return cudaSuccess;
    for (float **q : {&m.z1, &m.a1, &m.z2, &m.a2, &m.z3, &m.a3, &m.da, &m.dz, &m.y, &m.dy}) {
        if (*q) cudaFree(*q);
        *q = nullptr;
    }
    m.cap = 0;
    cudaError_t e = cudaSuccess;
    for (float **q : {&m.z1, &m.a1, &m.z2, &m.a2, &m.z3, &m.a3, &m.da, &m.dz})
        if (e == cudaSuccess) e = cudaMalloc(q, B * kH * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m.y, B * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m.dy, B * sizeof(float));
    if (e == cudaSuccess) m.cap = B;
    return e;
}

cudaError_t mlp_sync_bf16(Mlp &m, cudaStream_t s) {
    k_to_bf16<<<nblk(kW16, 256), 256, 0, s>>>(m.p, reinterpret_cast<__nv_bfloat16 *>(m.w16));
    return cudaGetLastError();
}

cudaError_t mlp_grad(Mlp &m, const float *X, const float *target, int B, cudaStream_t s) {
    if (B <= 0) return cudaErrorInvalidValue;
    cudaError_t e = mlp_reserve(m, (size_t)B);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(m.g, 0, kMlpFloats * sizeof(float), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(m.loss, 0, sizeof(float), s);
    if (e != cudaSuccess) return e;
    const long n = (long)B * kH;
    auto gemm = [&](int M, int N, int K, const float *A, long sam, long sak, const float *Bm,
                    long sbk, long sbn, float *C, long scm, long scn, int split) {
        const dim3 grid((N + 63) / 64, (M + 63) / 64, split);
        k_sgemm<<<grid, 256, 0, s>>>(M, N, K, A, sam, sak, Bm, sbk, sbn, C, scm, scn, split);
    };
    const unsigned bb = std::min<unsigned>(nblk((size_t)B, 4), 1184u);
    // forward: Z = X W^T (+ b), A = GELU(Z)
    gemm(B, kH, kIn, X, kIn, 1, m.p + kW1, 1, kIn, m.z1, kH, 1, 1);
    k_bias_gelu<<<nblk(n, 256), 256, 0, s>>>(m.z1, m.a1, m.p + kB1, n);
    gemm(B, kH, kH, m.a1, kH, 1, m.p + kW2, 1, kH, m.z2, kH, 1, 1);
    k_bias_gelu<<<nblk(n, 256), 256, 0, s>>>(m.z2, m.a2, m.p + kB2, n);
    gemm(B, kH, kH, m.a2, kH, 1, m.p + kW3, 1, kH, m.z3, kH, 1, 1);
    k_bias_gelu<<<nblk(n, 256), 256, 0, s>>>(m.z3, m.a3, m.p + kB3, n);
    k_out_loss<<<nblk((size_t)B, 256), 256, 0, s>>>(m.a3, m.p, target, B, m.y, m.dy, m.loss);
    // backward (weight gradients: split-K over the batch)
    const int split = std::max(1, std::min(148, B / 256));
    k_out_back<<<bb, 256, 0, s>>>(m.a3, m.dy, m.p, B, m.da, m.g);
    k_gelu_back<<<nblk(n, 256), 256, 0, s>>>(m.da, m.z3, m.dz, n);              // dZ3
    gemm(kH, kH, B, m.dz, 1, kH, m.a2, kH, 1, m.g + kW3, kH, 1, split);         // gW3 = dZ3^T A2
    k_bias_grad<<<bb, 256, 0, s>>>(m.dz, B, m.g, kB3);
    gemm(B, kH, kH, m.dz, kH, 1, m.p + kW3, kH, 1, m.da, kH, 1, 1);             // dA2 = dZ3 W3
    k_gelu_back<<<nblk(n, 256), 256, 0, s>>>(m.da, m.z2, m.dz, n);              // dZ2
    gemm(kH, kH, B, m.dz, 1, kH, m.a1, kH, 1, m.g + kW2, kH, 1, split);
    k_bias_grad<<<bb, 256, 0, s>>>(m.dz, B, m.g, kB2);
    gemm(B, kH, kH, m.dz, kH, 1, m.p + kW2, kH, 1, m.da, kH, 1, 1);             // dA1 = dZ2 W2
    k_gelu_back<<<nblk(n, 256), 256, 0, s>>>(m.da, m.z1, m.dz, n);              // dZ1
    gemm(kH, kIn, B, m.dz, 1, kH, X, kIn, 1, m.g + kW1, kIn, 1, split);         // gW1 = dZ1^T X
    k_bias_grad<<<bb, 256, 0, s>>>(m.dz, B, m.g, kB1);
    return cudaGetLastError();
}

cudaError_t mlp_adam(Mlp &m, float lr, cudaStream_t s) {
    m.adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    k_adam<<<nblk(kMlpFloats, 256), 256, 0, s>>>(
        m.p, m.g, m.m, m.v, kMlpFloats, lr, b1, b2, 1e-8f,
        1.f - std::pow(b1, (float)m.adam_t), 1.f - std::pow(b2, (float)m.adam_t));
    return cudaGetLastError();
}

// Grid of the inference kernel: one 16-ray pass per warp (4 per CTA), at
// most eight CTAs per SM; larger batches loop.
static unsigned infer_blocks(size_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t passes = (n + 15) / 16;  // 4 warps per block
    return (unsigned)std::max<size_t>(1, std::min<size_t>((passes + 3) / 4, (size_t)sms * 8));
}

cudaError_t mlp_infer_frame(const Mlp &m, const DevWorld &w, const VxCamera &cam,
                            const int32_t ro[3], uint32_t bw, uint32_t bh, float *out,
                            cudaStream_t s) {
    InferArgs a{};
    a.w = reinterpret_cast<const __nv_bfloat16 *>(m.w16);
    a.f32 = m.p;
    a.cam = cam;
    a.W = (uint32_t)cam.res_x;
    a.blk_w = bw ? bw : 1u;
    a.blk_h = bh ? bh : 1u;
    a.bw = (a.W + a.blk_w - 1u) / a.blk_w;
    a.n = a.bw * (((uint32_t)cam.res_y + a.blk_h - 1u) / a.blk_h);
    a.world = w;
    a.ro[0] = ro[0]; a.ro[1] = ro[1]; a.ro[2] = ro[2];
    a.out = out;
    if (a.n == 0) return cudaSuccess;
    k_mlp_infer<true><<<infer_blocks(a.n), 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t mlp_infer_features(const Mlp &m, const float *feats, size_t n, float *out,
                               cudaStream_t s) {
    InferArgs a{};
    a.w = reinterpret_cast<const __nv_bfloat16 *>(m.w16);
    a.f32 = m.p;
    a.feats = feats;
    a.n = (uint32_t)n;
    a.out = out;
    if (n == 0) return cudaSuccess;
    k_mlp_infer<false><<<infer_blocks(n), 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t mlp_features(const DevWorld &w, const int32_t ro[3], const VxRay *rays, size_t n,
                         uint64_t base, uint64_t mult, size_t count, float *feats,
                         const float *targets_src, float *targets_dst, cudaStream_t s) {
    if (count == 0 || n == 0) return cudaSuccess;
    k_features<<<nblk(count, 128), 128, 0, s>>>(w, ro[0], ro[1], ro[2], rays, n, base, mult,
                                                count, feats, targets_src, targets_dst);
    return cudaGetLastError();
}

cudaError_t mlp_targets(const VxHitRecord *rec, size_t n, float max_dist, float *target,
                        cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_targets<<<nblk(n, 256), 256, 0, s>>>(rec, n, max_dist, target);
    return cudaGetLastError();
}

cudaError_t mlp_pose_rays(const VxCamera &c, uint64_t seed, size_t n, VxRay *rays, float max_dist,
                          cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_pose_rays<<<nblk(n, 256), 256, 0, s>>>(c, seed, n, rays, max_dist);
    return cudaGetLastError();
}

}  // namespace vx
