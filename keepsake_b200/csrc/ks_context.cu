// Context lifetime, status strings, the device-memory pool and the Sobol parity kernels.
#include "ks_internal.h"
#include "ks_sampler.cuh"

#include <cstdint>
#include <mutex>
#include <new>

using namespace ksb;

namespace ksb
{
namespace pool_detail
{
// One pool and one allocation stream per GPU, made on first use and kept for the process (they
// may still be needed by buffers freed during process exit).
struct DevicePool
{
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
    bool failed = false; // no pool could be made: plain cudaMalloc / cudaFree
};
constexpr int kMaxDevices = 64;
DevicePool g_pools[kMaxDevices];
std::mutex g_pool_mutex;

DevicePool *pool_of(int device)
{
    if (device < 0 || device >= kMaxDevices)
        return nullptr;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    DevicePool &d = g_pools[device];
    if (d.pool || d.failed)
        return &d;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
    uint64_t keep = UINT64_MAX;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess ||
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess ||
        cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        if (pool)
            cudaMemPoolDestroy(pool);
        d.failed = true;
        return &d;
    }
    d.pool = pool;
    d.stream = stream;
    return &d;
}
} // namespace pool_detail
using pool_detail::DevicePool;
using pool_detail::pool_of;

cudaError_t pool_alloc(void **ptr, size_t bytes)
{
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess)
        return e;
    DevicePool *d = pool_of(device);
    if (!d || d->failed)
        return cudaMalloc(ptr, bytes);
    e = cudaMallocFromPoolAsync(ptr, bytes, d->pool, d->stream);
    if (e == cudaErrorMemoryAllocation) {
        // the pool's free blocks may not fit this size: give them back and try once more
        cudaGetLastError();
        cudaStreamSynchronize(d->stream);
        cudaMemPoolTrimTo(d->pool, 0);
        e = cudaMallocFromPoolAsync(ptr, bytes, d->pool, d->stream);
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(d->stream); // usable from every stream once this returns
    return e;
}

void pool_free(void *ptr, int device)
{
    DevicePool *d = pool_of(device);
    if (!d || d->failed) {
        cudaFree(ptr);
        return;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != device)
        cudaSetDevice(device);
    cudaDeviceSynchronize(); // cudaFree's wait: nothing in flight may still use the block
    cudaFreeAsync(ptr, d->stream);
    if (cur != device)
        cudaSetDevice(cur);
}

void pool_trim(int device)
{
    DevicePool *d = pool_of(device);
    if (!d || d->failed)
        return;
    cudaStreamSynchronize(d->stream);
    cudaMemPoolTrimTo(d->pool, 0);
}
} // namespace ksb

extern "C" {

const char *ks_status_string(ks_status s)
{
    switch (s) {
    case KS_OK:
        return "ok";
    case KS_ERR_INVALID_ARGUMENT:
        return "invalid argument";
    case KS_ERR_OUT_OF_MEMORY:
        return "out of device memory";
    case KS_ERR_CUDA:
        return "CUDA error";
    case KS_ERR_QUEUE_OVERFLOW:
        return "wavefront queue overflow";
    case KS_ERR_WATCHDOG:
        return "watchdog limit reached";
    case KS_ERR_NOT_BUILT:
        return "acceleration structure not built";
    case KS_ERR_UNSUPPORTED:
        return "unsupported configuration";
    case KS_ERR_PARSE:
        return "config parse error";
    case KS_ERR_IO:
        return "file i/o error";
    }
    return "unknown status";
}

ks_status ks_context_create(int device, ks_context **out)
{
    if (!out)
        return KS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess)
        return KS_ERR_CUDA;
    if (device < 0 || device >= n)
        return KS_ERR_INVALID_ARGUMENT;
    ks_context *ctx = new (std::nothrow) ks_context();
    if (!ctx)
        return KS_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    e = cudaSetDevice(device);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        delete ctx;
        return KS_ERR_CUDA;
    }
    *out = ctx;
    return KS_OK;
}

void ks_context_destroy(ks_context *ctx)
{
    if (!ctx)
        return;
    cudaSetDevice(ctx->device);
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    ctx->render_cache.reset();
    ctx->build_cache.reset();
    if (ctx->stream)
        cudaStreamDestroy(ctx->stream);
    const int device = ctx->device;
    delete ctx;
    pool_trim(device);
}

const char *ks_last_error(const ks_context *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

ks_status ks_context_set_limits(ks_context *ctx, const ks_context_limits *limits)
{
    if (!ctx)
        return KS_ERR_INVALID_ARGUMENT;
    ctx->limits = limits ? *limits : ks_context_limits{};
    return KS_OK;
}

} // extern "C"

namespace
{

__global__ void sobol_points_kernel(uint32_t x0, uint32_t y0, uint32_t nx, uint32_t ny, uint32_t s0, uint32_t ns,
                                    uint32_t nd, int log2_spp, int n_digits, uint32_t seed, float *out)
{
    uint64_t total = (uint64_t)nx * ny * ns * nd;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t d = (uint32_t)(i % nd);
        uint64_t r = i / nd;
        uint32_t s = (uint32_t)(r % ns);
        r /= ns;
        uint32_t px = (uint32_t)(r % nx);
        uint32_t py = (uint32_t)(r / nx);
        SobolSampler a = SobolSampler::start(x0 + px, y0 + py, s0 + s, log2_spp, n_digits, seed, (int)d);
        SobolSampler b = a;
        float u = a.next();
        float v0, v1;
        b.next2d(v0, v1);
        out[3 * i + 0] = u;
        out[3 * i + 1] = v0;
        out[3 * i + 2] = v1;
    }
}

__global__ void sobol_bounce_kernel(uint32_t x0, uint32_t y0, uint32_t nx, uint32_t ny, uint32_t s0, uint32_t ns,
                                    uint32_t dim, int log2_spp, int n_digits, uint32_t seed, float *out)
{
    uint64_t total = (uint64_t)nx * ny * ns;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t s = (uint32_t)(i % ns);
        uint64_t r = i / ns;
        uint32_t px = (uint32_t)(r % nx);
        uint32_t py = (uint32_t)(r / nx);
        SobolSampler a = SobolSampler::start(x0 + px, y0 + py, s0 + s, log2_spp, n_digits, seed, (int)dim);
        float u[7];
        a.bounce_values(u);
#pragma unroll
        for (int c = 0; c < 7; ++c)
            out[7 * i + c] = u[c];
    }
}

// Shared by the two hooks: argument checks, one launch, the copy back.
template <class Launch>
ks_status sobol_hook(ks_context *ctx, const char *what, uint32_t full_width, uint32_t full_height, uint32_t spp,
                     uint32_t x0, uint32_t y0, uint32_t nx, uint32_t ny, uint32_t s0, uint32_t ns, uint64_t n_items,
                     uint32_t per_item, float *out, Launch launch)
{
    if (!ctx || !out || full_width == 0 || full_height == 0 || spp == 0)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, std::string(what) + ": null pointer or zero size");
    if ((uint64_t)x0 + nx > full_width || (uint64_t)y0 + ny > full_height || (uint64_t)s0 + ns > spp)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, std::string(what) + ": window outside the image or sample range");
    if (n_items == 0)
        return KS_OK;
    KS_CUDA_TRY(ctx, enter_device(ctx));
    int log2_spp, n_digits;
    sobol_setup((int)spp, (int)full_width, (int)full_height, log2_spp, n_digits);
    DevBuf<float> d_out;
    KS_CUDA_TRY(ctx, d_out.alloc(n_items * per_item));
    uint64_t blocks = (n_items + 255) / 256;
    if (blocks > (uint64_t)ctx->sm_count * 64)
        blocks = (uint64_t)ctx->sm_count * 64;
    launch((unsigned)blocks, log2_spp, n_digits, d_out.ptr);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, d_out.ptr, d_out.bytes(), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(ctx->stream);
    d_out.release();
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, what);
    return KS_OK;
}

} // namespace

extern "C" ks_status ks_sobol_bounce(ks_context *ctx, uint32_t full_width, uint32_t full_height, uint32_t spp,
                                     uint32_t seed, uint32_t x0, uint32_t y0, uint32_t nx, uint32_t ny, uint32_t s0,
                                     uint32_t ns, uint32_t dim, float *out)
{
    return sobol_hook(ctx, "ks_sobol_bounce", full_width, full_height, spp, x0, y0, nx, ny, s0, ns,
                      (uint64_t)nx * ny * ns, 7, out, [&](unsigned blocks, int log2_spp, int n_digits, float *d) {
                          sobol_bounce_kernel<<<blocks, 256, 0, ctx->stream>>>(x0, y0, nx, ny, s0, ns, dim, log2_spp,
                                                                               n_digits, seed, d);
                      });
}

extern "C" ks_status ks_sobol_points(ks_context *ctx, uint32_t full_width, uint32_t full_height, uint32_t spp,
                                     uint32_t seed, uint32_t x0, uint32_t y0, uint32_t nx, uint32_t ny, uint32_t s0,
                                     uint32_t ns, uint32_t nd, float *out)
{
    return sobol_hook(ctx, "ks_sobol_points", full_width, full_height, spp, x0, y0, nx, ny, s0, ns,
                      (uint64_t)nx * ny * ns * nd, 3, out, [&](unsigned blocks, int log2_spp, int n_digits, float *d) {
                          sobol_points_kernel<<<blocks, 256, 0, ctx->stream>>>(x0, y0, nx, ny, s0, ns, nd, log2_spp,
                                                                               n_digits, seed, d);
                      });
}
