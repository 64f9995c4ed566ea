// Context lifetime, status strings and the Sobol parity kernel.
#include "ks_internal.h"
#include "ks_sampler.cuh"

#include <new>

using namespace ksb;

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
    delete ctx;
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

} // namespace

extern "C" ks_status ks_sobol_points(ks_context *ctx, uint32_t full_width, uint32_t full_height, uint32_t spp,
                                     uint32_t seed, uint32_t x0, uint32_t y0, uint32_t nx, uint32_t ny, uint32_t s0,
                                     uint32_t ns, uint32_t nd, float *out)
{
    if (!ctx || !out || full_width == 0 || full_height == 0 || spp == 0)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_sobol_points: null pointer or zero size");
    if ((uint64_t)x0 + nx > full_width || (uint64_t)y0 + ny > full_height || (uint64_t)s0 + ns > spp)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_sobol_points: window outside the image or sample range");
    uint64_t total = (uint64_t)nx * ny * ns * nd;
    if (total == 0)
        return KS_OK;
    KS_CUDA_TRY(ctx, enter_device(ctx));
    int log2_spp, n_digits;
    sobol_setup((int)spp, (int)full_width, (int)full_height, log2_spp, n_digits);
    DevBuf<float> d_out;
    KS_CUDA_TRY(ctx, d_out.alloc(total * 3));
    uint64_t blocks = (total + 255) / 256;
    if (blocks > (uint64_t)ctx->sm_count * 64)
        blocks = (uint64_t)ctx->sm_count * 64;
    sobol_points_kernel<<<(unsigned)blocks, 256, 0, ctx->stream>>>(x0, y0, nx, ny, s0, ns, nd, log2_spp, n_digits,
                                                                    seed, d_out.ptr);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, d_out.ptr, d_out.bytes(), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(ctx->stream);
    d_out.release();
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "ks_sobol_points");
    return KS_OK;
}
