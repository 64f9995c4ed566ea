// Ray queries that allocate no device memory.
//
// Some callers of this library cannot allocate device memory: a host application that owns the
// whole device-memory budget through its own allocator (a render-farm worker or a DCC plugin
// running inside another renderer's process), or one that forbids cudaMalloc/cudaFree on its
// frame loop.  ks_trace_rays_noalloc serves them: it stages rays and results in one statically
// sized device array of this translation unit instead of calling cudaMalloc.  The array holds
// kNoAllocMaxRays rays and their results (3.4 MB) and stays resident on every GPU that loads the
// library until the process exits.
#include "ks_scene.h"
#include "ks_traverse.cuh"

#include <mutex>

using namespace ksb;

namespace
{

constexpr uint32_t kNoAllocMaxRays = 65536;

struct NoAllocScratch
{
    float rays[8 * kNoAllocMaxRays];
    uint32_t tri[kNoAllocMaxRays];
    float t[kNoAllocMaxRays];
    float bary[3 * kNoAllocMaxRays];
    int overflow;
};

// One copy per device.  In host code this name is only a stand-in for the device symbol, so the
// kernel receives the address returned by cudaGetSymbolAddress, never &g_noalloc_scratch.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
NoAllocScratch *g_noalloc_ptr[kMaxDevices] = {};

// Set-up, once per device, with that device current.
cudaError_t noalloc_scratch(int device, NoAllocScratch **out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return e;
        g_noalloc_ptr[device] = (NoAllocScratch *)p;
    }
    *out = g_noalloc_ptr[device];
    return cudaSuccess;
}

__global__ void trace_noalloc_kernel(const TravNode *nodes, const float4 *tris, uint32_t root_ref,
                                     uint32_t root_count, float bx0, float by0, float bz0, float bx1, float by1,
                                     float bz1, uint32_t n, int any_hit, int culling, NoAllocScratch *s)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float *r = s->rays + 8 * (size_t)i;
    RayQuery q;
    q.o = mk(r[0], r[1], r[2]);
    q.tmin = r[3];
    q.d = mk(r[4], r[5], r[6]);
    q.tmax = r[7];
    const float bmin[3] = {bx0, by0, bz0}, bmax[3] = {bx1, by1, bz1};
    Hit h;
    int overflow = 0;
    if (any_hit) {
        bool occ = traverse<true>(nodes, tris, root_ref, root_count, bmin, bmax, q, culling, h, overflow);
        s->tri[i] = occ ? 1u : 0u;
    } else {
        traverse<false>(nodes, tris, root_ref, root_count, bmin, bmax, q, culling, h, overflow);
        s->tri[i] = h.tri;
        bool hit = h.tri != ~0u;
        s->t[i] = hit ? h.t : -kInf;
        s->bary[3 * i + 0] = hit ? h.b0 : 0.0f;
        s->bary[3 * i + 1] = hit ? h.b1 : 0.0f;
        s->bary[3 * i + 2] = hit ? h.b2 : 0.0f;
    }
    if (overflow)
        atomicOr(&s->overflow, 1);
}

} // namespace

extern "C" ks_status ks_trace_rays_noalloc(ks_scene *scene, const float *rays, uint32_t n, int any_hit, int culling,
                                           uint32_t *tri_idx, float *t, float *bary)
{
    if (!scene || !rays || !tri_idx || (!any_hit && (!t || !bary)) || culling < 0 || culling > 2)
        return fail(scene ? scene->ctx : nullptr, KS_ERR_INVALID_ARGUMENT, "ks_trace_rays_noalloc: bad argument");
    ks_context *ctx = scene->ctx;
    if (n > kNoAllocMaxRays)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT,
                    "ks_trace_rays_noalloc: at most 65536 rays per call (static device buffer)");
    if (!scene->bvh_built)
        return fail(ctx, KS_ERR_NOT_BUILT, "ks_trace_rays_noalloc: call ks_scene_build_bvh first");
    if (scene->n_instances)
        return fail(ctx, KS_ERR_UNSUPPORTED, "ks_trace_rays_noalloc: instanced scenes use ks_trace_rays");
    if (n == 0)
        return KS_OK;
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return fail(ctx, KS_ERR_UNSUPPORTED, "ks_trace_rays_noalloc: device index too large");
    KS_CUDA_TRY(ctx, enter_device(ctx));
    NoAllocScratch *s = nullptr;
    KS_CUDA_TRY(ctx, noalloc_scratch(ctx->device, &s));
    cudaStream_t st = ctx->stream;
    // the array keeps the previous call's contents: clear the flag that must start at zero
    KS_CUDA_TRY(ctx, cudaMemsetAsync(&s->overflow, 0, sizeof(int), st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->rays, rays, sizeof(float) * 8 * (size_t)n, cudaMemcpyHostToDevice, st));
    const float *b = scene->scene_bound;
    trace_noalloc_kernel<<<(n + 127) / 128, 128, 0, st>>>(scene->trav_nodes.ptr, scene->prim_tris.ptr,
                                                           scene->root_ref, scene->root_count, b[0], b[1], b[2], b[3],
                                                           b[4], b[5], n, any_hit, culling, s);
    KS_CUDA_TRY(ctx, cudaGetLastError());
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(tri_idx, s->tri, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st));
    if (!any_hit) {
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(t, s->t, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(bary, s->bary, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, st));
    }
    int overflow = 0;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(&overflow, &s->overflow, sizeof(int), cudaMemcpyDeviceToHost, st));
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (overflow)
        return fail(ctx, KS_ERR_QUEUE_OVERFLOW, "ks_trace_rays_noalloc: traversal stack depth exceeded");
    return KS_OK;
}
