// Internal host-side helpers shared by the C-ABI translation units.
#pragma once
#include <utility>
#include "../../include/ks_b200.h"

#include <cuda_runtime.h>
#include <memory>
#include <string>

struct ks_context
{
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    int sm_count = 148;
    // buffers the renders and the SBVH builder keep between calls (owned by ks_integrator.cu and
    // ks_sbvh_build.cu; freed at destroy)
    std::shared_ptr<void> render_cache, build_cache;
    // failure-detection limits (ks_context_set_limits; 0 = the library's own bound)
    ks_context_limits limits{};
};

namespace ksb
{

// Records a failure on the context and returns its status.
inline ks_status fail(ks_context *ctx, ks_status s, const std::string &msg)
{
    if (ctx)
        ctx->last_error = msg;
    return s;
}

// Makes the context's device current at the start of an entry point and clears a launch error
// left in the thread's CUDA state by earlier code (another library, or a call that already
// reported its failure), so that the checks after this call's launches see only its own errors.
// Errors that poison the context (a fault) are sticky and still surface.
inline cudaError_t enter_device(const ks_context *ctx)
{
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e == cudaSuccess)
        cudaGetLastError();
    return e;
}

inline ks_status cuda_fail(ks_context *ctx, cudaError_t e, const char *what)
{
    return fail(ctx, e == cudaErrorMemoryAllocation ? KS_ERR_OUT_OF_MEMORY : KS_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

// Device buffer owned by the caller of these helpers; freed explicitly.
template <typename T>
struct DevBuf
{
    T *ptr = nullptr;
    size_t count = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    // Grows (never shrinks) to hold n elements; contents are not preserved.
    cudaError_t reserve(size_t n)
    {
        if (n <= count && ptr)
            return cudaSuccess;
        return alloc(n);
    }
    cudaError_t alloc(size_t n)
    {
        release();
        count = n;
        if (n == 0)
            return cudaSuccess;
        return cudaMalloc((void **)&ptr, n * sizeof(T));
    }
    void release()
    {
        if (ptr)
            cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    size_t bytes() const { return count * sizeof(T); }
    void swap(DevBuf &o)
    {
        std::swap(ptr, o.ptr);
        std::swap(count, o.count);
    }
};

} // namespace ksb

#define KS_CUDA_TRY(ctx, expr)                                                                                         \
    do {                                                                                                               \
        cudaError_t _e = (expr);                                                                                       \
        if (_e != cudaSuccess)                                                                                         \
            return ksb::cuda_fail((ctx), _e, #expr);                                                                   \
    } while (0)
