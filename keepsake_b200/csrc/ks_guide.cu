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
#include "ks_guide_host.h"
#include "ks_internal.h"
#include "ks_tc.cuh"

#include <cuda_fp16.h>

#include <algorithm>
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
// 3 K-steps + 16 M-groups x 2048 B).
constexpr uint32_t kSmemTotal = 168u * 1024u;
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
    const float *grid;        // kLevels * T * 2
    const __half2 *grid_h;    // its FP16 copy (inference)
    const uint8_t *w_image;   // bf16 weight image (kWImage bytes)
    uint32_t n;               // rows
    uint32_t stride;          // floats between consecutive rows of pos / wo / nrm / wi (3 or 4)
    const float *pos, *wo;    // n rows
    const float *nrm;         // n rows: geometric normal on the side of wo
    const float *wi, *target; // training: n rows, n
    float target_scale;       // multiplies the targets (1 / batch size)
    const float *pb;          // training: BSDF pdf of wi per row (null: 0)
    uint32_t pb_stride;
    float alpha_max;          // selection probability = alpha_max * sigmoid(output kSel)
    float *out;               // row inference: n x 40 raw outputs
    float *w_grad;            // training: kWeights
    float *grid_grad;         // training: kLevels * T * 2
    double *loss;             // training
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

// CTA prologue shared by the kernels: weights -> shared memory, barrier init, TMEM allocation.
// Returns the TMEM base address.
__device__ __forceinline__ uint32_t mlp_prologue(const uint8_t *w_image, uint8_t *sw, uint64_t *bar,
                                                 uint32_t *tmem_slot, int *cta_err, uint32_t cols)
{
    // the weight image into shared memory, kCopyBatch loads in flight per thread (a load-store loop
    // waits for each load: about 20 round trips per thread, most of a small launch's time)
    constexpr uint32_t kCopyBatch = 10, kVecs = kWImage / 16;
    const uint4 *src = reinterpret_cast<const uint4 *>(w_image);
    uint4 *dst = reinterpret_cast<uint4 *>(sw);
    for (uint32_t base = threadIdx.x; base < kVecs; base += kThreads * kCopyBatch) {
        uint4 v[kCopyBatch];
#pragma unroll
        for (uint32_t c = 0; c < kCopyBatch; ++c)
            if (base + c * kThreads < kVecs)
                v[c] = __ldg(&src[base + c * kThreads]);
#pragma unroll
        for (uint32_t c = 0; c < kCopyBatch; ++c)
            if (base + c * kThreads < kVecs)
                dst[base + c * kThreads] = v[c];
    }
    if (threadIdx.x == 0) {
        tc::mbar_init(bar, 1);
        *cta_err = 0;
    }
    if (threadIdx.x < 32)
        tc::tmem_alloc(tmem_slot, cols);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    return *tmem_slot;
}

__device__ __forceinline__ void mlp_epilogue(uint32_t tmem, uint32_t cols)
{
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (threadIdx.x < 32)
        tc::tmem_dealloc(tmem, cols);
}

// Input encoding of this thread's row into X_0^T: 16 hash-grid levels x 2 features, then 16 SH
// coefficients of wo and 16 of the normal.  Invalid rows are zero.
// Hash-grid gathers with an L2 evict-last policy: the 64 MB table is read by every inference and
// training launch, while the wavefront streams gigabytes of path state through L2 in between;
// the hint keeps the table's lines ahead of those streams.
__device__ __forceinline__ uint64_t l2_keep_policy()
{
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ float2 ld_grid(const float2 *ptr, uint64_t pol)
{
    float2 v;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;" : "=f"(v.x), "=f"(v.y) : "l"(ptr), "l"(pol));
    return v;
}

// An entry of the FP16 inference copy of the table (two features in one 32-bit word).
__device__ __forceinline__ float2 ld_grid(const __half2 *ptr, uint64_t pol)
{
    uint32_t u;
    asm volatile("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(u) : "l"(ptr), "l"(pol));
    __half2 h;
    memcpy(&h, &u, 4);
    return __half22float2(h);
}

// Levels whose corner gathers are in flight together (2: within the inference kernel's 128-register
// budget at 4 CTAs per SM; 4 spills).
#ifndef KS_GUIDE_GATHER_GROUP
#define KS_GUIDE_GATHER_GROUP 2
#endif

// Table: float2 (the FP32 master table: training) or __half2 (its FP16 copy: inference).
template <class Entry>
__device__ __forceinline__ void encode_row(const GridParams &gp, const Entry *grid, bool valid, f3 pn, f3 wo,
                                           f3 nrm, uint8_t *x0)
{
    const uint64_t pol = l2_keep_policy();
    const uint32_t tid = threadIdx.x;
    // kGroup levels at a time: all their corner loads are issued before any is consumed, so a
    // thread waits for kLevels / kGroup round trips to L2 instead of kLevels
    constexpr int kGroup = KS_GUIDE_GATHER_GROUP;
    for (int l0 = 0; l0 < kLevels; l0 += kGroup) {
        float f0[kGroup], f1[kGroup];
#pragma unroll
        for (int g = 0; g < kGroup; ++g)
            f0[g] = f1[g] = 0.0f;
        if (valid) {
            Corner c[kGroup];
            float2 e[kGroup][8];
#pragma unroll
            for (int g = 0; g < kGroup; ++g) {
                level_corners(gp, l0 + g, pn, c[g]);
                const Entry *tab = grid + (size_t)(l0 + g) * kTableSize;
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    e[g][k] = ld_grid(&tab[c[g].idx[k]], pol);
            }
#pragma unroll
            for (int g = 0; g < kGroup; ++g)
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    f0[g] += c[g].w[k] * e[g][k].x;
                    f1[g] += c[g].w[k] * e[g][k].y;
                }
        }
#pragma unroll
        for (int g = 0; g < kGroup; ++g) {
            store_bf16(x0, xt_off(2 * (l0 + g), tid), f0[g]);
            store_bf16(x0, xt_off(2 * (l0 + g) + 1, tid), f1[g]);
        }
    }
    float sh[kShCoeffs];
    sh16(wo, sh);
    for (int i = 0; i < kShCoeffs; ++i)
        store_bf16(x0, xt_off(kGridFeatures + i, tid), valid ? sh[i] : 0.0f);
    sh16(nrm, sh);
    for (int i = 0; i < kShCoeffs; ++i)
        store_bf16(x0, xt_off(kGridFeatures + kShCoeffs + i, tid), valid ? sh[i] : 0.0f);
}

// Forward pass of the CTA's 128-row tile: X_l^T lives in xb[l] (written here for l >= 1, X_0 by
// the caller); the raw outputs of this thread's row end in o.  Returns false on an MMA timeout.
__device__ __forceinline__ bool mlp_forward(uint8_t *const xb[kLayers], const uint8_t *sw, uint32_t tmem,
                                            uint64_t *bar, uint32_t &phase, int *cta_err, int *err, float o[kOut])
{
    const uint32_t tid = threadIdx.x, lane_base = ((tid >> 5) * 32u) << 16;
    for (int l = 0; l < kLayers; ++l) {
        const int in = layer_in(l), out = layer_out(l);
        tc::fence_smem_to_async();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t idesc = tc::idesc_bf16(128, out, 1, 0);
            for (int s = 0; s < in / 16; ++s) {
                uint64_t ad = tc::smem_desc(tc::smem_addr(xb[l]) + s * 4096u, 2048u, 128u);
                uint64_t bd = tc::smem_desc(tc::smem_addr(sw + w_soff(l)) + s * 256u, 128u, in / 8 * 128u);
                tc::mma_bf16(tmem + kColFwd, ad, bd, idesc, s > 0);
            }
            tc::commit(bar);
        }
        if (!wait_mma(bar, phase, cta_err, err))
            return false;
        for (int c0 = 0; c0 < out; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem + lane_base + kColFwd + c0, v);
            if (l < kLayers - 1) {
                for (int i = 0; i < 16; ++i)
                    store_bf16(xb[l + 1], xt_off(c0 + i, tid), fmaxf(v[i], 0.0f));
            } else {
                for (int i = 0; i < 16 && c0 + i < kOut; ++i)
                    o[c0 + i] = v[i];
            }
        }
        tc::fence_before_sync();
    }
    return true;
}

__device__ __forceinline__ f3 load_row3(const float *p, uint32_t row, uint32_t stride)
{
    const float *q = p + (size_t)row * stride;
    return mk(q[0], q[1], q[2]);
}

// Row inference (raw outputs) and training (forward, loss, backward; weight gradients accumulate
// in TMEM across the CTA's tiles).
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

    if (kTrain)
        for (uint32_t i = tid; i < 32768 / 16; i += kThreads)
            reinterpret_cast<uint4 *>(sdy)[i] = make_uint4(0, 0, 0, 0);
    const uint32_t tmem = mlp_prologue(a.w_image, sw, bar, tmem_slot, cta_err, kCols);
    const uint32_t lane_base = (warp * 32u) << 16;
    uint8_t *xb[kLayers];
    for (int l = 0; l < kLayers; ++l)
        xb[l] = sx + x_soff(l);
    uint32_t phase = 0;
    bool first_tile = true;
    double loss_acc = 0.0;

    const uint32_t n_tiles = (a.n + kThreads - 1) / kThreads;
    for (uint32_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const uint32_t row = tile * kThreads + tid;
        const bool valid = row < a.n;
        f3 pn = mk(0, 0, 0), wo = mk(0, 0, 1), nrm = mk(0, 0, 1);
        if (valid) {
            pn = normalise_position(a.gp, load_row3(a.pos, row, a.stride));
            wo = normalize(load_row3(a.wo, row, a.stride));
            nrm = normalize(load_row3(a.nrm, row, a.stride));
        }
        // training encodes from the FP32 master table its gradients update; inference from the FP16 copy
        if constexpr (kTrain)
            encode_row(a.gp, reinterpret_cast<const float2 *>(a.grid), valid, pn, wo, nrm, xb[0]);
        else
            encode_row(a.gp, a.grid_h, valid, pn, wo, nrm, xb[0]);
        float o[kOut];
        if (!mlp_forward(xb, sw, tmem, bar, phase, cta_err, a.err, o))
            goto done;
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
            float t = 0.0f, p_b = 0.0f;
            if (valid) {
                wi = normalize(load_row3(a.wi, row, a.stride));
                t = a.target[row] * a.target_scale;
                if (a.pb)
                    p_b = a.pb[(size_t)row * a.pb_stride];
            }
            mixture_loss_grad(o, wi, t, p_b, a.alpha_max, loss, g);
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
                    uint64_t bd = tc::smem_desc(tc::smem_addr(xb[l]) + s * 256u, 128u, 2048u);
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
                    for (int i = 0; i < 16; ++i) {
                        float act = load_bf16(xb[l], xt_off(c0 + i, tid));
                        store_bf16(sdy, xt_off(c0 + i, tid), act > 0.0f ? v[i] : 0.0f);
                    }
                } else if (valid && c0 < kGridFeatures) {
                    // gradient of the hash-grid features: scatter to the 8 corners of each level
                    for (int i = 0; i < 16; i += 2) {
                        int lev = (c0 + i) / 2;
                        Corner c;
                        level_corners(a.gp, lev, pn, c);
                        float2 *gt = reinterpret_cast<float2 *>(a.grid_grad) + (size_t)lev * kTableSize;
                        // one vector reduction per corner (both features of the entry)
                        for (int k = 0; k < 8; ++k)
                            atomicAdd(&gt[c.idx[k]], make_float2(c.w[k] * v[i], c.w[k] * v[i + 1]));
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
    mlp_epilogue(tmem, kCols);
}

// Inference for the hit queue of a wavefront bounce: row = queue entry, input = hit position
// (origin + t * direction) and the reversed ray direction; output = the decoded mixture of the
// path slot (layout in ks_guide_view.cuh).  Two activation buffers alternate between layers, so a
// CTA needs 68 KB of shared memory and three CTAs share an SM.
struct PathArgs
{
    GridParams gp;
    const __half2 *grid_h; // FP16 copy of the table
    const uint8_t *w_image;
    const uint32_t *queue, *queue_count;
    const float4 *o_pdf, *d_info, *hits;
    const float4 *prim_tris; // 3 per SBVH primitive slot (vertices)
    const uint32_t *hit_inst; // instanced scenes: instance of each hit (else null)
    const float *inst_xf;     // 12 floats per instance
    float4 *lobes;
    uint32_t cap;
    float alpha_max;
    int *err;
};
// One activation buffer: layer l's output overwrites its input, which every thread writes only after
// the MMAs that read it have completed (the mbarrier wait in mlp_forward).  52 KB per CTA lets 4 CTAs
// (4 tiles in flight, 256 of the 512 TMEM columns) share an SM.
constexpr uint32_t kPathSmemX0 = kWImage, kPathSmemBar = kPathSmemX0 + 16384u;
constexpr uint32_t kPathSmem = kPathSmemBar + 64;
#ifndef KS_GUIDE_PATH_CTAS
#define KS_GUIDE_PATH_CTAS 4
#endif
constexpr int kPathCtasPerSm = KS_GUIDE_PATH_CTAS;

__global__ void __launch_bounds__(kThreads, kPathCtasPerSm) k_guide_paths(PathArgs a)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sw = smem;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + kPathSmemBar);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + kPathSmemBar + 8);
    int *cta_err = reinterpret_cast<int *>(smem + kPathSmemBar + 12);
    const uint32_t tmem = mlp_prologue(a.w_image, sw, bar, tmem_slot, cta_err, 64u);
    uint8_t *xb[kLayers];
    for (int l = 0; l < kLayers; ++l)
        xb[l] = smem + kPathSmemX0;
    uint32_t phase = 0;
    const uint32_t count = *a.queue_count;
    const uint32_t n_tiles = (count + kThreads - 1) / kThreads;
    for (uint32_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const uint32_t q = tile * kThreads + threadIdx.x;
        const bool valid = q < count;
        uint32_t i = 0;
        f3 pn = mk(0, 0, 0), wo = mk(0, 0, 1), nrm = mk(0, 0, 1);
        if (valid) {
            i = a.queue[q];
            float4 o4 = a.o_pdf[i], d4 = a.d_info[i], h4 = a.hits[i];
            f3 d = mk(d4.x, d4.y, d4.z);
            pn = normalise_position(a.gp, mk(o4.x, o4.y, o4.z) + h4.x * d);
            wo = -normalize(d);
            const float4 *pt = a.prim_tris + 3 * (size_t)__float_as_uint(h4.w);
            float4 v0 = __ldg(pt), v1 = __ldg(pt + 1), v2 = __ldg(pt + 2);
            f3 p0 = mk(v0.x, v0.y, v0.z), p1 = mk(v1.x, v1.y, v1.z), p2 = mk(v2.x, v2.y, v2.z);
            if (a.inst_xf) {
                float m[12];
                const float *src = a.inst_xf + 12 * (size_t)a.hit_inst[i];
                for (int e = 0; e < 12; ++e)
                    m[e] = __ldg(&src[e]);
                p0 = xf_point(m, p0);
                p1 = xf_point(m, p1);
                p2 = xf_point(m, p2);
            }
            nrm = facing_normal(p0, p1, p2, wo);
        }
        encode_row(a.gp, a.grid_h, valid, pn, wo, nrm, xb[0]);
        float o[kOut];
        if (!mlp_forward(xb, sw, tmem, bar, phase, cta_err, a.err, o))
            break;
        if (valid) {
            Lobe lobes[kLobes];
            decode_mixture(o, lobes);
            // weights scaled by the selection probability: they sum to alpha
            const float alpha = a.alpha_max * sigmoid(o[kSel]);
            for (int j = 0; j < kLobes; ++j)
                lobes[j].w *= alpha;
            for (int j = 0; j < kLobes; ++j)
                a.lobes[(size_t)j * a.cap + i] = make_float4(lobes[j].mu.x, lobes[j].mu.y, lobes[j].mu.z, lobes[j].kappa);
            a.lobes[(size_t)8 * a.cap + i] = make_float4(lobes[0].w, lobes[1].w, lobes[2].w, lobes[3].w);
            a.lobes[(size_t)9 * a.cap + i] = make_float4(lobes[4].w, lobes[5].w, lobes[6].w, lobes[7].w);
        }
    }
    mlp_epilogue(tmem, 64u);
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

// FP32 master table -> FP16 copy read by inference (round to nearest even, clamped to the FP16 range)
__global__ void k_pack_grid(const float2 *grid, __half2 *out, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float2 v = grid[i];
        out[i] = __floats2half2_rn(fminf(fmaxf(v.x, -65504.0f), 65504.0f), fminf(fmaxf(v.y, -65504.0f), 65504.0f));
    }
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
    DevBuf<__half2> grid_h; // FP16 copy of grid for inference, refreshed with w_image
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

// The inference images of the parameters: BF16 weights, FP16 table.
ks_status pack(ks_guide *g, cudaStream_t st)
{
    k_pack<<<(kWeights + 255) / 256, 256, 0, st>>>(g->w.ptr, g->w_image.ptr);
    k_pack_grid<<<g->ctx->sm_count * 8, 256, 0, st>>>(reinterpret_cast<const float2 *>(g->grid.ptr), g->grid_h.ptr,
                                                      (size_t)kLevels * kTableSize);
    KS_CUDA_TRY(g->ctx, cudaGetLastError());
    g->packed = true;
    return KS_OK;
}
ks_status pack(ks_guide *g) { return pack(g, g->ctx->stream); }

ks_status check_err(ks_guide *g)
{
    int e = 0;
    KS_CUDA_TRY(g->ctx, cudaMemcpyAsync(&e, g->err.ptr, sizeof(int), cudaMemcpyDeviceToHost, g->ctx->stream));
    KS_CUDA_TRY(g->ctx, cudaStreamSynchronize(g->ctx->stream));
    if (e)
        return fail(g->ctx, KS_ERR_WATCHDOG, "guide MLP: tensor-core completion wait timed out");
    return KS_OK;
}

// Runs the MLP over n device-resident rows (pos / wo / wi rows `stride` floats apart, BSDF pdfs
// pb_stride floats apart).
ks_status run_mlp(ks_guide *g, bool train, uint32_t n, const float *pos, const float *wo, const float *nrm,
                  const float *wi, const float *target, float *out, uint32_t stride = 3, const float *pb = nullptr,
                  uint32_t pb_stride = 1)
{
    if (!g->packed) {
        ks_status s = pack(g);
        if (s != KS_OK)
            return s;
    }
    MlpArgs a{};
    a.gp = g->gp;
    a.grid = g->grid.ptr;
    a.grid_h = g->grid_h.ptr;
    a.w_image = g->w_image.ptr;
    a.n = n;
    a.stride = stride;
    a.pos = pos;
    a.wo = wo;
    a.wi = wi;
    a.target = target;
    a.nrm = nrm;
    a.target_scale = n ? 1.0f / (float)n : 0.0f;
    a.pb = pb;
    a.pb_stride = pb_stride;
    a.alpha_max = g->params.alpha_max;
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

ks_context *context_of(const ks_guide *g) { return g->ctx; }

ks_status infer_paths(ks_guide *g, const uint32_t *queue, const uint32_t *queue_count, const float4 *o_pdf,
                      const float4 *d_info, const float4 *hits, const float4 *prim_tris, const uint32_t *hit_inst,
                      const float *inst_xf, float4 *lobes, uint32_t cap, uint32_t max_rows, cudaStream_t stream)
{
    if (!stream)
        stream = g->ctx->stream;
    if (!g->packed) {
        ks_status s = pack(g, stream);
        if (s != KS_OK)
            return s;
    }
    PathArgs a{};
    a.gp = g->gp;
    a.grid_h = g->grid_h.ptr;
    a.w_image = g->w_image.ptr;
    a.queue = queue;
    a.queue_count = queue_count;
    a.o_pdf = o_pdf;
    a.d_info = d_info;
    a.hits = hits;
    a.prim_tris = prim_tris;
    a.hit_inst = hit_inst;
    a.inst_xf = inst_xf;
    a.lobes = lobes;
    a.cap = cap;
    a.alpha_max = g->params.alpha_max;
    a.err = g->err.ptr;
    // one CTA per 128-row tile up to one wave of resident CTAs (each CTA loads the 39 KB weight
    // image and takes TMEM once, so the late bounces' few rows should not start a full wave)
    const uint32_t tiles = (max_rows + kThreads - 1) / kThreads;
    const uint32_t grid = std::max(1u, std::min(tiles, (uint32_t)g->ctx->sm_count * kPathCtasPerSm));
    k_guide_paths<<<grid, kThreads, kPathSmem, stream>>>(a);
    KS_CUDA_TRY(g->ctx, cudaGetLastError());
    return KS_OK;
}

ks_status train_rows(ks_guide *g, uint32_t n, const float4 *pos, const float4 *wo, const float4 *nrm,
                     const float4 *wi, const float *t, uint32_t batch, uint32_t *steps)
{
    if (batch == 0)
        batch = 1u << 18;
    for (uint32_t off = 0; off < n; off += batch) {
        uint32_t rows = std::min(batch, n - off);
        KS_CUDA_TRY(g->ctx, cudaMemsetAsync(g->loss.ptr, 0, sizeof(double), g->ctx->stream));
        // the BSDF pdf of each record sits in the w component of its wo row
        ks_status s = run_mlp(g, true, rows, reinterpret_cast<const float *>(pos + off),
                              reinterpret_cast<const float *>(wo + off), reinterpret_cast<const float *>(nrm + off),
                              reinterpret_cast<const float *>(wi + off), t + off, nullptr, 4,
                              reinterpret_cast<const float *>(wo + off) + 3, 4);
        if (s == KS_OK)
            s = adam(g);
        if (s != KS_OK)
            return s;
        ++*steps;
    }
    return KS_OK;
}

ks_status status(ks_guide *g) { return check_err(g); }

// The bounded completion wait of wait_mma on its own: one mbarrier for one arrival, which one
// thread makes when `arrive` is set; every thread then polls the phase at most max_polls times.
__global__ void k_mbarrier_probe(uint32_t max_polls, int arrive, int *timed_out)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0)
        tc::mbar_init(&bar, 1);
    __syncthreads();
    if (arrive && threadIdx.x == 0)
        tc::mbar_arrive(&bar);
    if (!tc::mbar_wait_bounded(&bar, 0, max_polls))
        atomicOr(timed_out, 1);
}

} // namespace guide_impl
} // namespace ksb

using namespace ksb::guide_impl;

extern "C" {

ks_status ks_mbarrier_wait_probe(ks_context *ctx, uint32_t max_polls, int arrive)
{
    if (!ctx || max_polls == 0)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_mbarrier_wait_probe: null context or zero polls");
    KS_CUDA_TRY(ctx, enter_device(ctx));
    DevBuf<int> flag;
    KS_CUDA_TRY(ctx, flag.alloc(1));
    KS_CUDA_TRY(ctx, cudaMemsetAsync(flag.ptr, 0, sizeof(int), ctx->stream));
    k_mbarrier_probe<<<1, 64, 0, ctx->stream>>>(max_polls, arrive, flag.ptr);
    KS_CUDA_TRY(ctx, cudaGetLastError());
    int timed_out = 0;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(&timed_out, flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (timed_out)
        return fail(ctx, KS_ERR_WATCHDOG, "ks_mbarrier_wait_probe: the bounded wait ran out of polls");
    return KS_OK;
}

ks_status ks_guide_create(ks_context *ctx, const ks_guide_params *params, ks_guide **out)
{
    if (!ctx || !params || !out)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_guide_create: null argument");
    *out = nullptr;
    const float *b = params->bound;
    for (int k = 0; k < 3; ++k)
        if (!(b[3 + k] > b[k]))
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_guide_create: empty bound");
    KS_CUDA_TRY(ctx, enter_device(ctx));
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
    if (!(g->params.alpha_max > 0.0f && g->params.alpha_max <= 1.0f))
        g->params.alpha_max = 0.8f;
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
        e = g->grid_h.alloc((size_t)kLevels * kTableSize);
    if (e == cudaSuccess)
        e = g->err.alloc(1);
    if (e == cudaSuccess)
        e = g->loss.alloc(1);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemTotal);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemTotal);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guide_paths, cudaFuncAttributeMaxDynamicSharedMemorySize, kPathSmem);
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

ks_status ks_guide_last_loss(ks_guide *g, double *loss)
{
    if (!g || !loss)
        return KS_ERR_INVALID_ARGUMENT;
    KS_CUDA_TRY(g->ctx, enter_device(g->ctx));
    KS_CUDA_TRY(g->ctx, cudaStreamSynchronize(g->ctx->stream));
    KS_CUDA_TRY(g->ctx, cudaMemcpy(loss, g->loss.ptr, sizeof(double), cudaMemcpyDeviceToHost));
    return KS_OK;
}

ks_status ks_guide_get_weights(ks_guide *g, float *mlp_weights, float *grid)
{
    if (!g)
        return KS_ERR_INVALID_ARGUMENT;
    KS_CUDA_TRY(g->ctx, enter_device(g->ctx));
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
    KS_CUDA_TRY(g->ctx, enter_device(g->ctx));
    if (mlp_weights)
        KS_CUDA_TRY(g->ctx, cudaMemcpy(g->w.ptr, mlp_weights, g->w.bytes(), cudaMemcpyHostToDevice));
    if (grid)
        KS_CUDA_TRY(g->ctx, cudaMemcpy(g->grid.ptr, grid, g->grid.bytes(), cudaMemcpyHostToDevice));
    g->packed = false;
    return KS_OK;
}

ks_status ks_guide_infer(ks_guide *g, const float *pos, const float *wo, const float *normal, uint32_t n,
                         float *raw_out)
{
    if (!g || !pos || !wo || !normal || !raw_out)
        return KS_ERR_INVALID_ARGUMENT;
    ks_context *ctx = g->ctx;
    KS_CUDA_TRY(ctx, enter_device(ctx));
    if (n == 0)
        return KS_OK;
    DevBuf<float> dp, dw, dn, dout;
    KS_CUDA_TRY(ctx, dp.alloc(3 * (size_t)n));
    KS_CUDA_TRY(ctx, dw.alloc(3 * (size_t)n));
    KS_CUDA_TRY(ctx, dn.alloc(3 * (size_t)n));
    KS_CUDA_TRY(ctx, dout.alloc((size_t)kOut * n));
    cudaStream_t st = ctx->stream;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dp.ptr, pos, dp.bytes(), cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dw.ptr, wo, dw.bytes(), cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dn.ptr, normal, dn.bytes(), cudaMemcpyHostToDevice, st));
    ks_status s = run_mlp(g, false, n, dp.ptr, dw.ptr, dn.ptr, nullptr, nullptr, dout.ptr);
    if (s != KS_OK)
        return s;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(raw_out, dout.ptr, dout.bytes(), cudaMemcpyDeviceToHost, st));
    return check_err(g);
}

ks_status ks_guide_gradients(ks_guide *g, const float *pos, const float *wo, const float *normal, const float *wi,
                             const float *target, const float *bsdf_pdf, uint32_t n, int apply_adam, double *loss,
                             float *mlp_grad, float *grid_grad)
{
    if (!g || !pos || !wo || !normal || !wi || !target)
        return KS_ERR_INVALID_ARGUMENT;
    ks_context *ctx = g->ctx;
    KS_CUDA_TRY(ctx, enter_device(ctx));
    cudaStream_t st = ctx->stream;
    DevBuf<float> dp, dwo, dn, dwi, dt, dpb;
    KS_CUDA_TRY(ctx, dn.alloc(3 * (size_t)n + 3));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dn.ptr, normal, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, dp.alloc(3 * (size_t)n + 3));
    KS_CUDA_TRY(ctx, dwo.alloc(3 * (size_t)n + 3));
    KS_CUDA_TRY(ctx, dwi.alloc(3 * (size_t)n + 3));
    KS_CUDA_TRY(ctx, dt.alloc((size_t)n + 1));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dp.ptr, pos, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dwo.ptr, wo, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dwi.ptr, wi, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(dt.ptr, target, 4 * (size_t)n, cudaMemcpyHostToDevice, st));
    if (bsdf_pdf) {
        KS_CUDA_TRY(ctx, dpb.alloc((size_t)n + 1));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(dpb.ptr, bsdf_pdf, 4 * (size_t)n, cudaMemcpyHostToDevice, st));
    }
    KS_CUDA_TRY(ctx, cudaMemsetAsync(g->loss.ptr, 0, sizeof(double), st));
    ks_status s = run_mlp(g, true, n, dp.ptr, dwo.ptr, dn.ptr, dwi.ptr, dt.ptr, nullptr, 3, dpb.ptr, 1);
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
