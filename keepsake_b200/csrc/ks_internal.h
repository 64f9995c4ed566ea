// Internal host-side helpers shared by the C-ABI translation units.
#pragma once
#include <utility>
#include "../../include/ks_b200.h"

#include <cuda_runtime.h>
#include <algorithm>
#include <memory>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

// Page-locked host memory a context keeps between calls (grow-only), held by one call at a time:
// the host side of large uploads.  Fresh host vectors pay a page fault per 4 KB on first touch and
// pageable copies go through the driver's own staging, which together cost more than the copy.
struct KsPinned
{
    void *ptr = nullptr;
    size_t bytes = 0;
    bool busy = false;
    KsPinned() = default;
    KsPinned(const KsPinned &) = delete;
    KsPinned &operator=(const KsPinned &) = delete;
    ~KsPinned() { release(); }
    cudaError_t reserve(size_t n)
    {
        if (ptr && n <= bytes)
            return cudaSuccess;
        release();
        cudaError_t e = cudaMallocHost(&ptr, n);
        if (e != cudaSuccess) {
            ptr = nullptr;
            return e;
        }
        bytes = n;
        return cudaSuccess;
    }
    void release()
    {
        if (ptr)
            cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

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
    // host side of ks_scene_create's uploads
    KsPinned upload;
};

namespace ksb
{

// f(begin, end) over contiguous chunks of [0, n) on up to 8 host threads (the caller runs the first
// chunk), for the memory-bound host passes over scene and image arrays; inline below 2 grains, or
// when no thread can be started.
template <class F>
void host_parallel(size_t n, size_t grain, F &&f)
{
    const unsigned hw = std::thread::hardware_concurrency();
    const size_t chunks = std::min<size_t>(std::min<unsigned>(hw ? hw : 1u, 8u), grain ? n / grain : 1);
    if (chunks <= 1) {
        f((size_t)0, n);
        return;
    }
    const size_t step = (n + chunks - 1) / chunks;
    std::vector<std::thread> pool;
    size_t done = step; // [0, done) is the caller's; the rest goes to threads while they start
    for (size_t b = step; b < n; b += step) {
        const size_t e = std::min(n, b + step);
        try {
            pool.emplace_back([&f, b, e] { f(b, e); });
            done = e;
        } catch (const std::system_error &) {
            break;
        }
    }
    f((size_t)0, std::min(n, step));
    if (done < n)
        f(done, n);
    for (auto &t : pool)
        t.join();
}

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

// Device memory of the library: one stream-ordered pool per GPU that keeps the blocks it is given
// back (release threshold unlimited), so scenes, builds and renders created and destroyed in a loop
// reuse memory instead of calling the driver's allocator each time; ks_context_destroy returns the
// free blocks to the driver.  Both calls keep cudaMalloc / cudaFree's host-synchronous behaviour:
// pool_alloc returns usable memory, pool_free first waits for the device (as cudaFree does), so no
// launch still in flight can see the block handed out again.
cudaError_t pool_alloc(void **ptr, size_t bytes);
void pool_free(void *ptr, int device);
void pool_trim(int device);

// Device buffer owned by the caller of these helpers; freed explicitly.
template <typename T>
struct DevBuf
{
    T *ptr = nullptr;
    size_t count = 0;
    int device = 0; // the GPU whose pool the block came from
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
        if (n == 0)
            return cudaSuccess;
        cudaGetDevice(&device);
        cudaError_t e = pool_alloc((void **)&ptr, n * sizeof(T));
        if (e != cudaSuccess) {
            ptr = nullptr;
            return e;
        }
        count = n;
        return cudaSuccess;
    }
    void release()
    {
        if (ptr)
            pool_free(ptr, device);
        ptr = nullptr;
        count = 0;
    }
    size_t bytes() const { return count * sizeof(T); }
    void swap(DevBuf &o)
    {
        std::swap(ptr, o.ptr);
        std::swap(count, o.count);
        std::swap(device, o.device);
    }
};

} // namespace ksb

#define KS_CUDA_TRY(ctx, expr)                                                                                         \
    do {                                                                                                               \
        cudaError_t _e = (expr);                                                                                       \
        if (_e != cudaSuccess)                                                                                         \
            return ksb::cuda_fail((ctx), _e, #expr);                                                                   \
    } while (0)
