// Learned path guiding on sm_100a: fused hash-grid encoding + BF16 MLP on tcgen05 tensor cores
// (FP32 accumulation in TMEM) + vMF mixture head; training by a fused forward/backward kernel
// whose weight gradients accumulate in TMEM across tiles, hash-grid gradient scatter, and Adam
// (adam.slang:25-51: m = lerp(g, m, b1), v = lerp(g^2, v, b2), bias-corrected, iter from 1).
//
// One CTA of 128 threads owns one SM (TMEM: 512 columns) and walks 128-row tiles; thread t owns
// row t of the tile.  Every activation, gradient and weight tile is stored once in shared memory
// in the canonical no-swizzle layout and read by the tensor core as a K-major operand in one GEMM
// and as an MN-major operand in the transposed GEMM:
//   forward   Z_l  [128 x out] = X_l [128 x in]  * W_l^T    (A = X_l^T buffer MN-major, B = W_l K-major)
//   backward  dX_l [128 x in]  = dY_l[128 x out] * W_l      (A = dY^T buffer MN-major, B = W_l MN-major)
//             dW_l [out x in] += dY_l^T * X_l               (A = dY^T K-major, padded to 128 rows,
//                                                            B = X_l^T buffer K-major)
#include "ks_guide.cuh"
#include "ks_internal.h"
#include "ks_tc.cuh"

#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <vector>

using namespace ksb;
using namespace ksb::guide;

static_assert(KS_GUIDE_LEVELS == kLevels && KS_GUIDE_TABLE_SIZE == kTableSize && KS_GUIDE_WEIGHTS == kWeights &&
                  KS_GUIDE_OUTPUTS == kOut,
              "C ABI constants out of sync with the guide network");

namespace
{

constexpr int kThreads = 128;
// shared-memory layout (bytes)
__host__ __device__ constexpr uint32_t w_bytes(int l) { return (uint32_t)(layer_out(l) * layer_in(l) * 2); }
__host__ __device__ constexpr uint32_t w_soff(int l)
{
    uint32_t o = 0;
    for (int i = 0; i < l; ++i)
        o += w_bytes(i);
    return o;
}
constexpr uint32_t kWImage = w_soff(kLayers);                // 36864
__host__ __device__ constexpr uint32_t x_bytes(int l) { return (uint32_t)(layer_in(l) / 8) * 2048u; }
__host__ __device__ constexpr uint32_t x_soff(int l)
{
    uint32_t o = 0;
    for (int i = 0; i < l; ++i)
        o += x_bytes(i);
    return o;
}
constexpr uint32_t kSmemW = 0;
constexpr uint32_t kSmemX = kSmemW + kWImage;          // X_l^T buffers, 77824 B
constexpr uint32_t kSmemDY = kSmemX + x_soff(kLayers); // dY^T, 128 x 128 bf16 = 32768 B
constexpr uint32_t kSmemBar = kSmemDY + 32768;
// The allocation is padded so that every descriptor above stays inside it even if the tensor core
// read one of them with its two strides exchanged (furthest reach: the dX A operand, dY^T base +
// 3 K-steps + 16 M-groups x 2048 B = 159744 B).
constexpr uint32_t kSmemTotal = 160u * 1024u;
static_assert(kSmemBar + 64 <= kSmemTotal && kSmemDY + 3u * 4096u + 16u * 2048u <= kSmemTotal,
              "guide MLP shared-memory plan");
// TMEM columns
constexpr uint32_t kColFwd = 0, kColDX = 64, kColDW = 128;
__host__ __device__ constexpr uint32_t dw_col(int l)
{
    uint32_t c = kColDW;
    for (int i = 0; i < l; ++i)
        c += (uint32_t)layer_in(i);
    return c;
}

// element (row, k) of an activation / input tile stored transposed (k rows, row contiguous)
__device__ __forceinline__ uint32_t xt_off(uint32_t k, uint32_t row)
{
    return (k >> 3) * 2048u + (row >> 3) * 128u + (k & 7u) * 16u + (row & 7u) * 2u;
}
// element (n, k) of W_l ([out][in], k contiguous in core matrices)
__host__ __device__ constexpr uint32_t w_off(int l, uint32_t n, uint32_t k)
{
    return (n >> 3) * ((uint32_t)layer_in(l) / 8u * 128u) + (k >> 3) * 128u + (n & 7u) * 16u + (k & 7u) * 2u;
}

struct MlpArgs
{
    GridParams gp;
    const float *grid;          // kLevels * T * 2
    const uint8_t *w_image;     // bf16 weight image (kWImage bytes)
    uint32_t n;                 // rows
    const float *pos, *wo;      // n x 3
    const float *wi, *target;   // training: n x 3, n
    float target_scale;         // multiplies the targets (1 / batch size)
    float *out;                 // inference: n x 40 raw outputs
    float *w_grad;              // training: kWeights
    float *grid_grad;           // training: kLevels * T * 2
    double *loss;               // training
    int *err;
};

__device__ __forceinline__ void store_bf16(uint8_t *base, uint32_t off, float v)
{
    *reinterpret_cast<__nv_bfloat16 *>(base + off) = __float2bfloat16_rn(v);
}
__device__ __forceinline__ float load_bf16(const uint8_t *base, uint32_t off)
{
    return __bfloat162float(*reinterpret_cast<const __nv_bfloat16 *>(base + off));
}

// Waits on the MMA barrier; on timeout records the error.  Returns false when the CTA must stop.
__device__ __forceinline__ bool wait_mma(uint64_t *bar, uint32_t &phase, int *cta_err, int *err)
{
    bool ok = tc::mbar_wait_bounded(bar, phase);
    phase ^= 1u;
    if (!ok) {
        *cta_err = 1;
        atomicOr(err, 1);
    }
    __syncthreads();
    tc::fence_after_sync();
    return *cta_err == 0;
}

template <bool kTrain>
__global__ void __launch_bounds__(kThreads, 1) k_mlp(MlpArgs a)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sw = smem + kSmemW, *sx = smem + kSmemX, *sdy = smem + kSmemDY;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + kSmemBar);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + kSmemBar + 8);
    int *cta_err = reinterpret_cast<int *>(smem + kSmemBar + 12);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    constexpr uint32_t kCols = kTrain ? 512u : 64u;

    // weights -> shared memory; dY buffer zeroed (rows beyond a layer's width stay zero)
    for (uint32_t i = tid; i < kWImage / 16; i += kThreads)
        reinterpret_cast<uint4 *>(sw)[i] = reinterpret_cast<const uint4 *>(a.w_image)[i];
    if (kTrain)
        for (uint32_t i = tid; i < 32768 / 16; i += kThreads)
            reinterpret_cast<uint4 *>(sdy)[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        *cta_err = 0;
    }
    if (warp == 0)
        tc::tmem_alloc(tmem_slot, kCols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    const uint32_t lane_base = (warp * 32u) << 16;
    uint32_t phase = 0;
    bool first_tile = true;
    double loss_acc = 0.0;

    const uint32_t n_tiles = (a.n + kThreads - 1) / kThreads;
    for (uint32_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const uint32_t row = tile * kThreads + tid;
        const bool valid = row < a.n;
        // ---- encoding -> X_0^T ----
        f3 pn = mk(0, 0, 0), wo = mk(0, 0, 1);
        if (valid) {
            pn = normalise_position(a.gp, mk(a.pos[3 * row], a.pos[3 * row + 1], a.pos[3 * row + 2]));
            wo = normalize(mk(a.wo[3 * row], a.wo[3 * row + 1], a.wo[3 * row + 2]));
        }
        uint8_t *x0 = sx + x_soff(0);
        for (int l = 0; l < kLevels; ++l) {
            float f0 = 0.0f, f1 = 0.0f;
            if (valid) {
                Corner c;
                level_corners(a.gp, l, pn, c);
                const float2 *tab = reinterpret_cast<const float2 *>(a.grid) + (size_t)l * kTableSize;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    float2 e = __ldg(&tab[c.idx[k]]);
                    f0 += c.w[k] * e.x;
                    f1 += c.w[k] * e.y;
                }
            }
            store_bf16(x0, xt_off(2 * l, tid), f0);
            store_bf16(x0, xt_off(2 * l + 1, tid), f1);
        }
        float sh[kShCoeffs];
        sh16(wo, sh);
        for (int i = 0; i < kShCoeffs; ++i)
            store_bf16(x0, xt_off(kGridFeatures + i, tid), valid ? sh[i] : 0.0f);

        // ---- forward ----
        float o[kOut];
        for (int l = 0; l < kLayers; ++l) {
            const int in = layer_in(l), out = layer_out(l);
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after_sync();
                const uint32_t idesc = tc::idesc_bf16(128, out, 1, 0);
                for (int s = 0; s < in / 16; ++s) {
                    uint64_t ad = tc::smem_desc(tc::smem_addr(sx + x_soff(l)) + s * 4096u, 2048u, 128u);
                    uint64_t bd = tc::smem_desc(tc::smem_addr(sw + w_soff(l)) + s * 256u, 128u, in / 8 * 128u);
                    tc::mma_bf16(tmem + kColFwd, ad, bd, idesc, s > 0);
                }
                tc::commit(bar);
            }
            if (!wait_mma(bar, phase, cta_err, a.err))
                goto done;
            for (int c0 = 0; c0 < out; c0 += 16) {
                float v[16];
                tc::tmem_ld16(tmem + lane_base + kColFwd + c0, v);
                if (l < kLayers - 1) {
                    uint8_t *xn = sx + x_soff(l + 1);
                    for (int i = 0; i < 16; ++i)
                        store_bf16(xn, xt_off(c0 + i, tid), fmaxf(v[i], 0.0f));
                } else {
                    for (int i = 0; i < 16 && c0 + i < kOut; ++i)
                        o[c0 + i] = v[i];
                }
            }
            tc::fence_before_sync();
        }
        if (!kTrain) {
            if (valid)
                for (int i = 0; i < kOut; ++i)
                    a.out[(size_t)row * kOut + i] = o[i];
            continue;
        }
        // ---- head: loss and dO -> dY_4^T ----
        {
            float g[kOut], loss = 0.0f;
            f3 wi = mk(0, 0, 1);
            float t = 0.0f;
            if (valid) {
                wi = normalize(mk(a.wi[3 * row], a.wi[3 * row + 1], a.wi[3 * row + 2]));
                t = a.target[row] * a.target_scale;
            }
            mixture_loss_grad(o, wi, t, loss, g);
            loss_acc += loss;
            for (int n = 0; n < kOutPad; ++n)
                store_bf16(sdy, xt_off(n, tid), n < kOut ? g[n] : 0.0f);
        }
        // ---- backward ----
        for (int l = kLayers - 1; l >= 0; --l) {
            const int in = layer_in(l), out = layer_out(l);
            tc::fence_smem_to_async();
            tc::fence_before_sync();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after_sync();
                // dW_l += dY_l^T X_l  (M = 128 padded output rows, N = in, K = 128 tile rows)
                const uint32_t idw = tc::idesc_bf16(128, in, 0, 0);
                for (int s = 0; s < 8; ++s) {
                    uint64_t ad = tc::smem_desc(tc::smem_addr(sdy) + s * 256u, 128u, 2048u);
                    uint64_t bd = tc::smem_desc(tc::smem_addr(sx + x_soff(l)) + s * 256u, 128u, 2048u);
                    tc::mma_bf16(tmem + dw_col(l), ad, bd, idw, (!first_tile || s > 0) ? 1u : 0u);
                }
                // dX_l = dY_l W_l  (M = 128 rows, N = in, K = out)
                const uint32_t idx = tc::idesc_bf16(128, in, 1, 1);
                const uint32_t sn = (uint32_t)in / 8u * 128u;
                for (int s = 0; s < out / 16; ++s) {
                    uint64_t ad = tc::smem_desc(tc::smem_addr(sdy) + s * 4096u, 2048u, 128u);
                    uint64_t bd = tc::smem_desc(tc::smem_addr(sw + w_soff(l)) + s * 2u * sn, sn, 128u);
                    tc::mma_bf16(tmem + kColDX, ad, bd, idx, s > 0);
                }
                tc::commit(bar);
            }
            if (!wait_mma(bar, phase, cta_err, a.err))
                goto done;
            for (int c0 = 0; c0 < in; c0 += 16) {
                float v[16];
                tc::tmem_ld16(tmem + lane_base + kColDX + c0, v);
                if (l > 0) {
                    // dY_{l-1} = dX_l * relu'(Z_{l-1}); X_l holds relu(Z_{l-1})
                    const uint8_t *xl = sx + x_soff(l);
                    for (int i = 0; i < 16; ++i) {
                        float act = load_bf16(xl, xt_off(c0 + i, tid));
                        store_bf16(sdy, xt_off(c0 + i, tid), act > 0.0f ? v[i] : 0.0f);
                    }
                } else if (valid && c0 < kGridFeatures) {
                    // gradient of the hash-grid features: scatter to the 8 corners of each level
                    for (int i = 0; i < 16; i += 2) {
                        int lev = (c0 + i) / 2;
                        Corner c;
                        level_corners(a.gp, lev, pn, c);
                        float2 *gt = reinterpret_cast<float2 *>(a.grid_grad) + (size_t)lev * kTableSize;
                        for (int k = 0; k < 8; ++k) {
                            atomicAdd(&gt[c.idx[k]].x, c.w[k] * v[i]);
                            atomicAdd(&gt[c.idx[k]].y, c.w[k] * v[i + 1]);
                        }
                    }
                }
            }
            tc::fence_before_sync();
        }
        first_tile = false;
    }
    if (kTrain) {
        // weight gradients accumulated in TMEM over this CTA's tiles -> global
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (!first_tile && *cta_err == 0) {
            for (int l = 0; l < kLayers; ++l) {
                const int in = layer_in(l), out = layer_out(l);
                for (int c0 = 0; c0 < in; c0 += 16) {
                    float v[16];
                    tc::tmem_ld16(tmem + lane_base + dw_col(l) + c0, v);
                    if ((int)tid < out)
                        for (int i = 0; i < 16; ++i)
                            atomicAdd(&a.w_grad[weight_offset(l) + tid * in + c0 + i], v[i]);
                }
            }
        }
        for (int o2 = 16; o2 > 0; o2 >>= 1)
            loss_acc += __shfl_xor_sync(0xffffffffu, loss_acc, o2);
        if ((tid & 31) == 0)
            atomicAdd(a.loss, loss_acc);
    }
done:
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0)
        tc::tmem_dealloc(tmem, kCols);
}

// fp32 master weights -> bf16 canonical image
__global__ void k_pack(const float *w, uint8_t *image)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kWeights)
        return;
    int l = 0;
    while (l + 1 < kLayers && i >= weight_offset(l + 1))
        ++l;
    int r = i - weight_offset(l);
    uint32_t n = (uint32_t)(r / layer_in(l)), k = (uint32_t)(r % layer_in(l));
    *reinterpret_cast<__nv_bfloat16 *>(image + w_soff(l) + w_off(l, n, k)) = __float2bfloat16_rn(w[i]);
}

// Adam (adam.slang:25-51)
__global__ void k_adam(float *p, float *g, float *m, float *v, size_t n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float gi = g[i];
        float mt = gi + b1 * (m[i] - gi);
        float vt = gi * gi + b2 * (v[i] - gi * gi);
        float mh = mt / c1, vh = vt / c2;
        p[i] -= lr * mh / (sqrtf(vh) + eps);
        m[i] = mt;
        v[i] = vt;
        g[i] = 0.0f;
    }
}

} // namespace

struct ks_guide
{
    ks_context *ctx = nullptr;
    ks_guide_params params{};
    GridParams gp{};
    DevBuf<float> grid, grid_grad, grid_m, grid_v;
    DevBuf<float> w, w_grad, w_m, w_v;
    DevBuf<uint8_t> w_image;
    DevBuf<int> err;
    DevBuf<double> loss;
    int iter = 0;
    bool packed = false;
    int grid_ctas = 148;
};

namespace ksb
{
namespace guide_impl
{
size_t grid_count() { return (size_t)kLevels * kTableSize * kFeatPerLevel; }

ks_status pack(ks_guide *g)
{
    k_pack<<<(kWeights + 255) / 256, 256, 0, g->ctx->stream>>>(g->w.ptr, g->w_image.ptr);
    KS_CUDA_TRY(g->ctx, cudaGetLastError());
    g->packed = true;
    return KS_OK;
}

ks_status check_err(ks_guide *g)
{
    int e = 0;
    KS_CUDA_TRY(g->ctx, cudaMemcpyAsync(&e, g->err.ptr, sizeof(int), cudaMemcpyDeviceToHost, g->ctx->stream));
    KS_CUDA_TRY(g->ctx, cudaStreamSynchronize(g->ctx->stream));
    if (e)
        return fail(g->ctx, KS_ERR_WATCHDOG, "guide MLP: tensor-core completion wait timed out");
    return KS_OK;
}

// Runs the MLP over n device-resident rows.
ks_status run_mlp(ks_guide *g, bool train, uint32_t n, const float *pos, const float *wo, const float *wi,
                  const float *target, float *out)
{
    if (!g->packed) {
        ks_status s = pack(g);
        if (s != KS_OK)
            return s;
    }
    MlpArgs a{};
    a.gp = g->gp;
    a.grid = g->grid.ptr;
    a.w_image = g->w_image.ptr;
    a.n = n;
    a.pos = pos;
    a.wo = wo;
    a.wi = wi;
    a.target = target;
    a.target_scale = n ? 1.0f / (float)n : 0.0f;
    a.out = out;
    a.w_grad = g->w_grad.ptr;
    a.grid_grad = g->grid_grad.ptr;
    a.loss = g->loss.ptr;
    a.err = g->err.ptr;
    uint32_t tiles = (n + kThreads - 1) / kThreads;
    uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)g->grid_ctas);
    if (grid == 0)
        return KS_OK;
    if (train)
        k_mlp<true><<<grid, kThreads, kSmemTotal, g->ctx->stream>>>(a);
    else
        k_mlp<false><<<grid, kThreads, kSmemTotal, g->ctx->stream>>>(a);
    KS_CUDA_TRY(g->ctx, cudaGetLastError());
    return KS_OK;
}

ks_status adam(ks_guide *g)
{
    g->iter += 1;
    const ks_guide_params &p = g->params;
    float c1 = 1.0f - powf(0.9f, (float)g->iter), c2 = 1.0f - powf(0.999f, (float)g->iter);
    cudaStream_t st = g->ctx->stream;
    k_adam<<<g->ctx->sm_count * 8, 256, 0, st>>>(g->w.ptr, g->w_grad.ptr, g->w_m.ptr, g->w_v.ptr, kWeights,
                                                p.learning_rate, 0.9f, 0.999f, 1e-8f, c1, c2);
    k_adam<<<g->ctx->sm_count * 8, 256, 0, st>>>(g->grid.ptr, g->grid_grad.ptr, g->grid_m.ptr, g->grid_v.ptr,
                                                grid_count(), p.learning_rate, 0.9f, 0.999f, 1e-8f, c1, c2);
    KS_CUDA_TRY(g->ctx, cudaGetLastError());
    g->packed = false;
    return KS_OK;
}

} // namespace guide_impl
} // namespace ksb

using namespace ksb::guide_impl;

extern "C" {

ks_status ks_guide_create(ks_context *ctx, const ks_guide_params *params, ks_guide **out)
{
    if (!ctx || !params || !out)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_guide_create: null argument");
    *out = nullptr;
    const float *b = params->bound;
    for (int k = 0; k < 3; ++k)
        if (!(b[3 + k] > b[k]))
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_guide_create: empty bound");
    KS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    ks_guide *g = new (std::nothrow) ks_guide();
    if (!g)
        return fail(ctx, KS_ERR_OUT_OF_MEMORY, "ks_guide_create");
    g->ctx = ctx;
    g->params = *params;
    if (!(g->params.learning_rate > 0.0f))
        g->params.learning_rate = 1e-2f;
    if (!(g->params.base_res > 0.0f))
        g->params.base_res = 16.0f;
    if (!(g->params.max_res > g->params.base_res))
        g->params.max_res = 2048.0f;
    const double lscale = std::log((double)g->params.max_res / (double)g->params.base_res) / (double)(kLevels - 1);
    for (int l = 0; l < kLevels; ++l)
        g->gp.res[l] = (uint32_t)std::floor((double)g->params.base_res * std::exp(lscale * l) + 1e-9);
    for (int k = 0; k < 3; ++k) {
        g->gp.bmin[k] = b[k];
        g->gp.inv_ext[k] = 1.0f / (b[3 + k] - b[k]);
    }
    g->grid_ctas = ctx->sm_count;
    size_t ng = grid_count();
    cudaError_t e = cudaSuccess;
    for (DevBuf<float> *buf : {&g->grid, &g->grid_grad, &g->grid_m, &g->grid_v})
        if (e == cudaSuccess)
            e = buf->alloc(ng);
    for (DevBuf<float> *buf : {&g->w, &g->w_grad, &g->w_m, &g->w_v})
        if (e == cudaSuccess)
            e = buf->alloc(kWeights);
    if (e == cudaSuccess)
        e = g->w_image.alloc(kWImage);
    if (e == cudaSuccess)
        e = g->err.alloc(1);
    if (e == cudaSuccess)
        e = g->loss.alloc(1);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemTotal);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemTotal);
    if (e != cudaSuccess) {
        delete g;
        return cuda_fail(ctx, e, "ks_guide_create");
    }
    // seeded initialisation: hash grid U(-1e-4, 1e-4), weights U(-sqrt(6/fan_in), +), output layer x0.1
    std::mt19937_64 rng(params->seed);
    std::uniform_real_distribution<float> u01(0.0f, 1.0f);
    std::vector<float> hw(kWeights, 0.0f);
    for (int l = 0; l < kLayers; ++l) {
        float lim = std::sqrt(6.0f / (float)layer_in(l)) * (l == kLayers - 1 ? 0.1f : 1.0f);
        int rows = l == kLayers - 1 ? kOut : layer_out(l);
        for (int n = 0; n < rows; ++n)
            for (int k = 0; k < layer_in(l); ++k)
                hw[weight_offset(l) + n * layer_in(l) + k] = (2.0f * u01(rng) - 1.0f) * lim;
    }
    std::vector<float> hg(ng);
    for (auto &x : hg)
        x = (2.0f * u01(rng) - 1.0f) * 1e-4f;
    cudaStream_t st = ctx->stream;
    e = cudaMemcpyAsync(g->w.ptr, hw.data(), g->w.bytes(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g->grid.ptr, hg.data(), g->grid.bytes(), cudaMemcpyHostToDevice, st);
    for (DevBuf<float> *buf : {&g->grid_grad, &g->grid_m, &g->grid_v, &g->w_grad, &g->w_m, &g->w_v})
        if (e == cudaSuccess)
            e = cudaMemsetAsync(buf->ptr, 0, buf->bytes(), st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(g->err.ptr, 0, sizeof(int), st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        delete g;
        return cuda_fail(ctx, e, "ks_guide_create: init");
    }
    *out = g;
    return KS_OK;
}

void ks_guide_destroy(ks_guide *g)
{
    if (!g)
        return;
    cudaSetDevice(g->ctx->device);
    cudaStreamSynchronize(g->ctx->stream);
    delete g;
}

ks_status ks_guide_level_res(const ks_guide *g, uint32_t res[KS_GUIDE_LEVELS])
{
    if (!g || !res)
        return KS_ERR_INVALID_ARGUMENT;
    for (int l = 0; l < kLevels; ++l)
        res[l] = g->gp.res[l];
    return KS_OK;
}

ks_status ks_guide_get_weights(ks_guide *g, float *mlp_weights, float *grid)
{
    if (!g)
        return KS_ERR_INVALID_ARGUMENT;
    KS_CUDA_TRY(g->ctx, cudaSetDevice(g->ctx->device));
    if (mlp_weights)
        KS_CUDA_TRY(g->ctx, cudaMemcpy(mlp_weights, g->w.ptr, g->w.bytes(), cudaMemcpyDeviceToHost));
    if (grid)
        KS_CUDA_TRY(g->ctx, cudaMemcpy(grid, g->grid.ptr, g->grid.bytes(), cudaMemcpyDeviceToHost));
    return KS_OK;
}

ks_status ks_guide_set_weights(ks_guide *g, const float *mlp_weights, const float *grid)
{
    if (!g)
        return KS_ERR_INVALID_ARGUMENT;
    KS_CUDA_TRY(g->ctx, cudaSetDevice(g->ctx->device));
    if (mlp_weights)
        KS_CUDA_TRY(g->ctx, cudaMemcpy(g->w.ptr, mlp_weights, g->w.bytes(), cudaMemcpyHostToDevice));
    if (grid)
        KS_CUDA_TRY(g->ctx, cudaMemcpy(g->grid.ptr, grid, g->grid.bytes(), cudaMemcpyHostToDevice));
    g->packed = false;
    return KS_OK;
}

ks_status ks_guide_infer(ks_guide *g, const float *pos, const float *wo, uint32_t n, float *raw_out)
{
    if (!g || !pos || !wo || !raw_out)
        return KS_ERR_INVALID_ARGUMENT;
    ks_context *ctx = g->ctx;
    KS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    if (n == 0)
        return KS_OK;
    DevBuf<float> dp, dw, dout;
    KS_CUDA_TRY(ctx, dp.alloc(3 * (size_t)n));
    KS_CUDA_TRY(ctx, dw.alloc(3 * (size_t)n));
    KS_CUDA_TRY(ctx, dout.alloc((size_t)kOut * n));
    cudaStream_t st = ctx->stream;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dp.ptr, pos, dp.bytes(), cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dw.ptr, wo, dw.bytes(), cudaMemcpyHostToDevice, st));
    ks_status s = run_mlp(g, false, n, dp.ptr, dw.ptr, nullptr, nullptr, dout.ptr);
    if (s != KS_OK)
        return s;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(raw_out, dout.ptr, dout.bytes(), cudaMemcpyDeviceToHost, st));
    return check_err(g);
}

ks_status ks_guide_gradients(ks_guide *g, const float *pos, const float *wo, const float *wi, const float *target,
                             uint32_t n, int apply_adam, double *loss, float *mlp_grad, float *grid_grad)
{
    if (!g || !pos || !wo || !wi || !target)
        return KS_ERR_INVALID_ARGUMENT;
    ks_context *ctx = g->ctx;
    KS_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    DevBuf<float> dp, dwo, dwi, dt;
    KS_CUDA_TRY(ctx, dp.alloc(3 * (size_t)n + 3));
    KS_CUDA_TRY(ctx, dwo.alloc(3 * (size_t)n + 3));
    KS_CUDA_TRY(ctx, dwi.alloc(3 * (size_t)n + 3));
    KS_CUDA_TRY(ctx, dt.alloc((size_t)n + 1));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dp.ptr, pos, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dwo.ptr, wo, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dwi.ptr, wi, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dt.ptr, target, 4 * (size_t)n, cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemsetAsync(g->loss.ptr, 0, sizeof(double), st));
    ks_status s = run_mlp(g, true, n, dp.ptr, dwo.ptr, dwi.ptr, dt.ptr, nullptr);
    if (s != KS_OK)
        return s;
    if (loss)
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(loss, g->loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (mlp_grad)
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(mlp_grad, g->w_grad.ptr, g->w_grad.bytes(), cudaMemcpyDeviceToHost, st));
    if (grid_grad)
        KS_CUDA_TRY(ctx,
                    cudaMemcpyAsync(grid_grad, g->grid_grad.ptr, g->grid_grad.bytes(), cudaMemcpyDeviceToHost, st));
    s = check_err(g);
    if (s != KS_OK)
        return s;
    if (apply_adam) {
        s = adam(g);
    } else {
        KS_CUDA_TRY(ctx, cudaMemsetAsync(g->w_grad.ptr, 0, g->w_grad.bytes(), st));
        KS_CUDA_TRY(ctx, cudaMemsetAsync(g->grid_grad.ptr, 0, g->grid_grad.bytes(), st));
    }
    if (s != KS_OK)
        return s;
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return KS_OK;
}

} // extern "C"
