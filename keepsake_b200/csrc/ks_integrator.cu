// Wavefront small_pt integrator for sm_100a.
//
// SmallPT::run / trace (small_pt.cpp:15-178) restructured as a streaming wavefront:
//
//   raygen  -> new camera paths fill the free queue slots (sample-major over the crop window),
//   extend  -> closest-hit traversal of the SBVH's 4-wide view by persistent warps that fetch rays
//              from a counter (ks_traverse.cuh), then hit and miss queues in path order,
//   sample  -> the bounce's Sobol values and the NEE light sample (ks_shade.cu),
//   shade   -> miss/sky MIS, emitter MIS, BSDF eval of the light sample (Material::sample_with_nee,
//              material.cpp:101-167; next_event_estimate, nee.cpp:11-57), BSDF sample, Russian
//              roulette (ks_shade.cu); surviving paths and shadow rays are appended to compacted
//              SoA queues (ballot + popc within a warp, one atomic per CTA),
//   shadow  -> any-hit traversal of the NEE shadow rays; unoccluded contributions are added to the
//              path (or, for a path that ended this bounce, the path is accumulated).
//
// Per-path arithmetic follows the reference's order: L gains the emitter/sky term of the bounce
// first, then beta * Ld of the same bounce, then the next bounce's terms, exactly like trace().
// Sobol dimensions are carried per path (light select, light uv, lobe, wi, roulette: 6 or 7 per
// bounce), so each path draws the same sample values as the CPU path.  Finished paths are added
// to FP64 pixel accumulators (RenderTarget2::add / add_miss, render_target.cpp:82-107).
#include "ks_guide_host.h"
#include "ks_sampler.cuh"
#include "ks_traverse.cuh"
#include "ks_wavefront.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

namespace ksb
{
SceneView make_view(const ks_scene *s);

namespace
{
using namespace wave;

// Minimum resident CTAs per SM asked of the compiler (a register cap) for the persistent
// traversal kernels: at 8 CTAs of 128 (64 registers) they run a little faster than at 7.
#ifndef KS_TRAV_MIN_BLOCKS
#define KS_TRAV_MIN_BLOCKS 8
#endif
// Persistent traversal with dynamic ray fetch (1) or one thread per ray (0) for flat scenes.
#ifndef KS_PERSISTENT_TRAV
#define KS_PERSISTENT_TRAV 1
#endif
constexpr bool kPersistentTraversal = KS_PERSISTENT_TRAV != 0;
// Tree layouts of the persistent kernels: the SBVH nodes (0) or their 4-wide view (1).  Measured on
// the bench frame: the 4-wide view takes 15 % off the any-hit kernel and 2 % off the closest-hit
// one (whose nearest-first ordering of up to four slots eats most of the saving).
#ifndef KS_WIDE_EXTEND
#define KS_WIDE_EXTEND 1
#endif
#ifndef KS_WIDE_SHADOW
#define KS_WIDE_SHADOW 1
#endif
using ExtendNode = std::conditional_t<KS_WIDE_EXTEND != 0, WideNode, TravNode>;
using ShadowNode = std::conditional_t<KS_WIDE_SHADOW != 0, WideNode, TravNode>;
// Path slots of a single-frame wavefront (log2).  More rays per launch shorten the share of each
// persistent traversal launch that its last rays run alone, and halve the iterations (and host
// round trips) per doubling: on the bench frame 4 M slots 1458 Mrays/s, 16 M 1643, 32 M 1690,
// 64 M 1689.  32 M slots hold about 9.2 GB of path state (plus 5 GB for a guided render).
#ifndef KS_WAVE_LOG2
#define KS_WAVE_LOG2 25
#endif

// Per-iteration counters: paths continuing, shadow rays, hit queue, miss queue, extension-ray
// fetch, shadow-ray fetch.
constexpr uint32_t kCounters = 6;

// ---- kernels --------------------------------------------------------------------------------

// Camera sample s of pixel (px, py) into path slot `slot`: Sobol pixel-filter offset (box: uniform
// over [-r, r]^2; Gaussian / Blackman-Harris: PixelFilterSampleTable::sample, render_target.h:94-101,
// through the tabulated DistribTable2D's sample_linear, distrib.cpp:74-86), ray through the
// projection (Camera::spawn_ray, camera.cpp:129-170; film position small_pt.cpp:50-54).
// pix_word is the pixel index (with the job id in its upper bits for batched renders).
KS_D void camera_path(const RenderParams &rp, int px, int py, int s, uint32_t pix_word, PathBuf &pb, uint32_t slot)
{
    SobolSampler smp = SobolSampler::start((uint32_t)px, (uint32_t)py, (uint32_t)s, rp.log2_spp, rp.n_digits,
                                           (uint32_t)rp.seed, 0);
    float offx = 0.0f, offy = 0.0f;
    if (rp.spp != 1) {
        float u0, u1;
        smp.next2d(u0, u1);
        if (rp.filter_n) {
            const uint32_t n = rp.filter_n;
            float pdf_m, pdf_c;
            uint32_t vi, ui;
            const float vs = distrib_sample_linear(rp.filter_cdf + (size_t)n * (n + 1), n, u1, pdf_m, vi);
            u0 = distrib_sample_linear(rp.filter_cdf + (size_t)vi * (n + 1), n, u0, pdf_c, ui);
            u1 = vs;
        }
        offx = (1.0f - u0) * -rp.filter_r + u0 * rp.filter_r;
        offy = (1.0f - u1) * -rp.filter_r + u1 * rp.filter_r;
    }
    float fx = ((px + 0.5f) + offx) / (float)rp.W;
    float fy = ((py + 0.5f) + offy) / (float)rp.H;
    f3 ndc = mk(fx * 2.0f - 1.0f, fy * 2.0f - 1.0f, 1.0f);
    const float *m = rp.p2w;
    float o[4];
    for (int r = 0; r < 4; ++r)
        o[r] = m[4 * r + 0] * ndc.x + m[4 * r + 1] * ndc.y + m[4 * r + 2] * ndc.z + m[4 * r + 3] * 1.0f;
    f3 wp = mk(o[0] / o[3], o[1] / o[3], o[2] / o[3]);
    f3 cp = mk(rp.cam_pos[0], rp.cam_pos[1], rp.cam_pos[2]);
    f3 dir;
    if (rp.ortho) {
        cp = wp;
        dir = mk(rp.cam_dir[0], rp.cam_dir[1], rp.cam_dir[2]);
    } else {
        dir = normalize(wp - cp);
    }
    pb.o_pdf[slot] = make_float4(cp.x, cp.y, cp.z, 0.0f);
    pb.d_info[slot] = make_float4(dir.x, dir.y, dir.z, fbits(((uint32_t)smp.dimension << 16) | 0u));
    pb.beta_pix[slot] = make_float4(1.0f, 1.0f, 1.0f, fbits(pix_word));
    pb.L_smp[slot] = make_float4(0.0f, 0.0f, 0.0f, fbits((uint32_t)s));
    if (pb.rec)
        pb.rec[slot] = kNoRecord;
}

__global__ void k_raygen(const __grid_constant__ RenderParams rp, PathBuf pb, uint32_t base_slot, uint64_t first_path,
                         uint32_t n_new, int s0, uint32_t n_pix)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_new)
        return;
    uint64_t k = first_path + i;
    int s = s0 + (int)(k / n_pix);
    uint32_t pl = (uint32_t)(k % n_pix);
    int px = rp.cx + (int)(pl % (uint32_t)rp.cw), py = rp.cy + (int)(pl / (uint32_t)rp.cw);
    camera_path(rp, px, py, s, (uint32_t)py * (uint32_t)rp.W + (uint32_t)px, pb, base_slot + i);
}

// Batched refill: new path i of this iteration is global path first_path + i; its job is found in
// the jobs' path ranges, then sample-major over the job's crop window as in k_raygen.
__global__ void k_raygen_batch(BatchView bv, PathBuf pb)
{
    const BatchState &st = *bv.state;
    const uint32_t n_new = st.n_new, base_slot = st.base_slot;
    const unsigned long long first = st.first_path;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_new; i += gridDim.x * blockDim.x) {
        const unsigned long long k = first + i;
        uint32_t lo = 0, hi = bv.n_jobs;
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) / 2;
            if (bv.path_begin[mid] <= k)
                lo = mid;
            else
                hi = mid;
        }
        const RenderParams &rp = bv.params[lo];
        const unsigned long long kk = k - bv.path_begin[lo];
        const uint32_t n_pix = (uint32_t)rp.cw * (uint32_t)rp.ch;
        int s = (int)(kk / n_pix);
        uint32_t pl = (uint32_t)(kk % n_pix);
        int px = rp.cx + (int)(pl % (uint32_t)rp.cw), py = rp.cy + (int)(pl / (uint32_t)rp.cw);
        uint32_t pix = ((uint32_t)py * (uint32_t)rp.W + (uint32_t)px) | (lo << kJobShift);
        camera_path(rp, px, py, s, pix, pb, base_slot + i);
    }
}

// Batched iteration head: paths that continue from the last iteration stay in [0, alive); the
// free slots are refilled with new paths; the queue counters restart.
__global__ void k_batch_prep(BatchState *st, uint32_t *counters, uint32_t capacity)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    BatchState &s = *st;
    const uint32_t alive = counters[0];
    const unsigned long long left = s.total - s.issued;
    const uint32_t n_new = (uint32_t)(left < (unsigned long long)(capacity - alive) ? left : capacity - alive);
    s.cur_count = alive;
    s.base_slot = alive;
    s.n_new = n_new;
    s.first_path = s.issued;
    s.issued += n_new;
    s.count = alive + n_new;
    s.ext_rays += s.count;
    for (uint32_t k = 0; k < kCounters; ++k)
        counters[k] = 0;
}

// Batched iteration tail: counts the shadow rays and decides whether another iteration is
// needed; an iteration limit ends the loop with the error flag set.  In a graph the decision
// drives the while node.
__global__ void k_batch_advance(BatchState *st, const uint32_t *counters, cudaGraphConditionalHandle handle,
                                int use_graph)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    BatchState &s = *st;
    s.shadow_rays += counters[1];
    s.iterations += 1;
    bool more = s.issued < s.total || counters[0] > 0;
    if (s.iterations >= s.max_iterations) {
        if (more)
            s.error = 1;
        more = false;
    }
    if (use_graph)
        cudaGraphSetConditional(handle, more ? 1u : 0u);
}

// Adds a per-thread work count into two 64-bit device counters, one atomic per warp.
KS_D void flush_counts(const TravCount &c, unsigned long long *dst)
{
    unsigned long long n = c.nodes, t = c.tris;
    for (int o = 16; o > 0; o >>= 1) {
        n += __shfl_xor_sync(0xffffffffu, n, o);
        t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(dst, n);
        atomicAdd(dst + 1, t);
    }
}

// Closest hit for every queued ray; the path index goes to the hit queue or the miss queue.
// kInst: two-level traversal of an instanced scene; the instance of each hit goes to hit_inst.
// kBatch: paths of many jobs (flat scenes), the count read from the batch state.
template <bool kInst, bool kBatch = false>
__global__ void __launch_bounds__(128) k_extend(const __grid_constant__ SceneView sv_in, PathBuf pb, uint32_t count,
                                                float4 *hits, uint32_t *hit_inst, uint32_t *hit_queue,
                                                uint32_t *miss_queue, uint32_t *queue_counts, int *overflow,
                                                unsigned long long *work, BatchView bv)
{
    TravCount tc;
    const uint32_t stride = gridDim.x * blockDim.x;
    if constexpr (kBatch)
        count = bv.state->count;
    for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += stride) {
        uint32_t i = base + threadIdx.x;
        bool valid = i < count, is_hit = false;
        if (valid) {
            const uint32_t job = kBatch ? (bits(pb.beta_pix[i].w) >> kJobShift) : 0u;
            const SceneView &sv = job_of<kBatch>(sv_in, bv.views, job);
            float4 a = pb.o_pdf[i], b = pb.d_info[i];
            RayQuery q;
            q.o = mk(a.x, a.y, a.z);
            q.d = mk(b.x, b.y, b.z);
            q.tmin = 0.0f;
            q.tmax = kInf;
            Hit h;
            int of = 0;
            if constexpr (kInst) {
                uint32_t inst = 0;
                traverse_instances<false>(sv.nodes, sv.prim_tris, sv.inst, q, 2, h, inst, of, &tc);
                hit_inst[i] = inst;
            } else {
                traverse<false>(sv.nodes, sv.prim_tris, sv.root_ref, sv.root_count, sv.bmin, sv.bmax, q, 2, h, of,
                                &tc);
            }
            if (of)
                atomicOr(overflow, 1);
            is_hit = h.tri != ~0u;
            hits[i] = is_hit ? make_float4(h.t, h.b1, h.b2, fbits(h.slot)) : make_float4(0, 0, 0, fbits(~0u));
        }
        uint32_t jh = warp_append(queue_counts, valid && is_hit);
        uint32_t jm = warp_append(queue_counts + 1, valid && !is_hit);
        if (valid) {
            if (is_hit)
                hit_queue[jh] = i;
            else
                miss_queue[jm] = i;
        }
    }
    flush_counts(tc, work);
}

// ---- persistent traversal with dynamic ray fetch (flat scenes) --------------------------------
// One thread per ray leaves a warp running until its longest ray ends (about 5 of 32 lanes stay
// busy on average).  k_extend_pt and k_shadow_pt keep the lanes busy instead (warp_fetch and
// trav_step, ks_traverse.cuh).  The grid is one wave of resident CTAs; the fetch counters restart
// every iteration.

// Closest hit of every queued ray into hits[i] (slot ~0u: miss); k_build_queues then sorts the
// paths into the hit and miss queues in index order, so that shading reads the path state in
// order.  kBatch: paths of many jobs, the count read from the batch state.
// kAlpha: the scene has opacity maps; candidate hits go through their stochastic test (SceneAlpha).
template <bool kBatch = false, bool kAlpha = false>
__global__ void __launch_bounds__(128, KS_TRAV_MIN_BLOCKS) k_extend_pt(const __grid_constant__ SceneView sv_in, PathBuf pb, uint32_t count,
                                                   float4 *hits, uint32_t *fetch, int *overflow,
                                                   unsigned long long *work, BatchView bv)
{
    if constexpr (kBatch)
        count = bv.state->count;
    TravCount tc;
    KS_TRAV_STACK(stack);
    TravState s;
    const ExtendNode *nodes = tree_of<ExtendNode>(sv_in);
    const float4 *tris = sv_in.prim_tris;
    uint32_t ray = ~0u;
    bool drained = false;
    int of = 0;
    while (true) {
        const uint32_t id = warp_fetch(fetch, count, ray == ~0u, drained);
        if (id != ~0u) {
            const uint32_t job = kBatch ? (bits(pb.beta_pix[id].w) >> kJobShift) : 0u;
            const SceneView &sv = job_of<kBatch>(sv_in, bv.views, job);
            nodes = tree_of<ExtendNode>(sv);
            tris = sv.prim_tris;
            float4 a = pb.o_pdf[id], b = pb.d_info[id];
            RayQuery q;
            q.o = mk(a.x, a.y, a.z);
            q.d = mk(b.x, b.y, b.z);
            q.tmin = 0.0f;
            q.tmax = kInf;
            if (trav_begin(s, q, sv.root_ref, sv.root_count, sv.bmin, sv.bmax))
                ray = id;
            else
                hits[id] = make_float4(0, 0, 0, fbits(~0u));
        }
        if (__ballot_sync(0xffffffffu, ray != ~0u) == 0) {
            if (drained)
                break;
            continue;
        }
        while (true) {
            bool done;
            if constexpr (kAlpha)
                done = trav_warp_step<false>(nodes, tris, s, stack, 2, of, &tc, ray != ~0u, SceneAlpha{&sv_in});
            else
                done = trav_warp_step<false>(nodes, tris, s, stack, 2, of, &tc, ray != ~0u);
            if (done) {
                hits[ray] = s.hit.tri != ~0u ? make_float4(s.hit.t, s.hit.b1, s.hit.b2, fbits(s.hit.slot))
                                             : make_float4(0, 0, 0, fbits(~0u));
                ray = ~0u;
            }
            const int n_idle = __popc(__ballot_sync(0xffffffffu, ray == ~0u));
            if (n_idle == 32 || (!drained && n_idle >= KS_TRAV_REFILL))
                break;
        }
    }
    if (of)
        atomicOr(overflow, 1);
    flush_counts(tc, work);
}

// Hit and miss queues from the per-ray results of k_extend_pt, one CTA-aggregated append per
// kind (queue order follows the path index within each CTA's tile).
template <bool kBatch = false>
__global__ void __launch_bounds__(256) k_build_queues(const float4 *hits, uint32_t count, uint32_t *hit_queue,
                                                      uint32_t *miss_queue, uint32_t *queue_counts, BatchView bv)
{
    if constexpr (kBatch)
        count = bv.state->count;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t *slot = reinterpret_cast<const uint32_t *>(hits) + 3;
    for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += stride) {
        const uint32_t i = base + threadIdx.x;
        const bool valid = i < count;
        const bool is_hit = valid && slot[4 * (size_t)i] != ~0u;
        uint32_t jh, jm;
        block_append2(queue_counts, is_hit, queue_counts + 1, valid && !is_hit, jh, jm);
        if (valid) {
            if (is_hit)
                hit_queue[jh] = i;
            else
                miss_queue[jm] = i;
        }
    }
}

template <bool kInst, bool kBatch = false>
__global__ void __launch_bounds__(128) k_shadow(const __grid_constant__ SceneView sv_in, ShadowBuf sb,
                                                const uint32_t *shadow_count, PathBuf nxt, double *accum_in,
                                                double *weights_in, int *overflow, unsigned long long *work,
                                                GuideView gv, BatchView bv)
{
    const uint32_t n = *shadow_count;
    TravCount tc;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 c = sb.contrib[i];
        const uint32_t job = kBatch ? bits(c.w) : 0u;
        const SceneView &sv = job_of<kBatch>(sv_in, bv.views, job);
        double *accum = kBatch ? bv.accum[job] : accum_in;
        double *weights = kBatch ? bv.weights[job] : weights_in;
        float4 a = sb.o_tmax[i], b = sb.d_target[i];
        RayQuery q;
        q.o = mk(a.x, a.y, a.z);
        q.d = mk(b.x, b.y, b.z);
        q.tmin = 0.0f;
        q.tmax = a.w;
        Hit h;
        int of = 0;
        bool occ;
        if constexpr (kInst) {
            uint32_t inst = 0;
            occ = traverse_instances<true>(sv.nodes, sv.prim_tris, sv.inst, q, 2, h, inst, of, &tc);
        } else {
            occ = traverse<true>(sv.nodes, sv.prim_tris, sv.root_ref, sv.root_count, sv.bmin, sv.bmax, q, 2, h, of,
                                 &tc);
        }
        if (of)
            atomicOr(overflow, 1);
        uint32_t target = bits(b.w);
        if (gv.rec_cap && !occ && bits(c.w) != kNoRecord)
            record_add(gv, bits(c.w), mk(c.x, c.y, c.z));
        if (target & kTermBit) {
            float4 l = sb.L_term[i];
            f3 L = mk(l.x, l.y, l.z);
            if (!occ)
                L += mk(c.x, c.y, c.z);
            accumulate(accum, weights, kBatch ? (target & kPixMask) : (target & ~kTermBit), L);
        } else if (!occ) {
            float4 l = nxt.L_smp[target];
            l.x += c.x;
            l.y += c.y;
            l.z += c.z;
            nxt.L_smp[target] = l;
        }
    }
    flush_counts(tc, work);
}

// Completion of shadow ray i: records, then the contribution goes to the continuing path or, for a
// path that ended this bounce, the path is accumulated.
template <bool kBatch>
KS_D void shadow_done(const ShadowBuf &sb, uint32_t i, bool occ, PathBuf nxt, double *accum_in, double *weights_in,
                      const GuideView &gv, const BatchView &bv)
{
    const float4 c = sb.contrib[i];
    const uint32_t target = bits(sb.d_target[i].w);
    const uint32_t job = kBatch ? bits(c.w) : 0u;
    if (gv.rec_cap && !occ && bits(c.w) != kNoRecord)
        record_add(gv, bits(c.w), mk(c.x, c.y, c.z));
    if (target & kTermBit) {
        double *accum = kBatch ? bv.accum[job] : accum_in;
        double *weights = kBatch ? bv.weights[job] : weights_in;
        float4 l = sb.L_term[i];
        f3 L = mk(l.x, l.y, l.z);
        if (!occ)
            L += mk(c.x, c.y, c.z);
        accumulate(accum, weights, kBatch ? (target & kPixMask) : (target & ~kTermBit), L);
    } else if (!occ) {
        float4 l = nxt.L_smp[target];
        l.x += c.x;
        l.y += c.y;
        l.z += c.z;
        nxt.L_smp[target] = l;
    }
}

// Any-hit traversal of the NEE shadow rays with dynamic ray fetch (flat scenes); each ray is
// finished by shadow_done as soon as its traversal ends.
template <bool kBatch = false, bool kAlpha = false>
__global__ void __launch_bounds__(128, KS_TRAV_MIN_BLOCKS) k_shadow_pt(const __grid_constant__ SceneView sv_in, ShadowBuf sb,
                                                   const uint32_t *shadow_count, uint32_t *fetch, PathBuf nxt,
                                                   double *accum_in, double *weights_in, int *overflow,
                                                   unsigned long long *work, GuideView gv, BatchView bv)
{
    const uint32_t count = *shadow_count;
    TravCount tc;
    KS_TRAV_STACK(stack);
    TravState s;
    const ShadowNode *nodes = tree_of<ShadowNode>(sv_in);
    const float4 *tris = sv_in.prim_tris;
    uint32_t ray = ~0u;
    bool drained = false;
    int of = 0;
    while (true) {
        const uint32_t id = warp_fetch(fetch, count, ray == ~0u, drained);
        if (id != ~0u) {
            const uint32_t job = kBatch ? bits(sb.contrib[id].w) : 0u;
            const SceneView &sv = job_of<kBatch>(sv_in, bv.views, job);
            nodes = tree_of<ShadowNode>(sv);
            tris = sv.prim_tris;
            float4 a = sb.o_tmax[id], b = sb.d_target[id];
            RayQuery q;
            q.o = mk(a.x, a.y, a.z);
            q.d = mk(b.x, b.y, b.z);
            q.tmin = 0.0f;
            q.tmax = a.w;
            if (trav_begin(s, q, sv.root_ref, sv.root_count, sv.bmin, sv.bmax))
                ray = id;
            else
                shadow_done<kBatch>(sb, id, false, nxt, accum_in, weights_in, gv, bv);
        }
        if (__ballot_sync(0xffffffffu, ray != ~0u) == 0) {
            if (drained)
                break;
            continue;
        }
        while (true) {
            bool done;
            if constexpr (kAlpha)
                done = trav_warp_step<true>(nodes, tris, s, stack, 2, of, &tc, ray != ~0u, SceneAlpha{&sv_in});
            else
                done = trav_warp_step<true>(nodes, tris, s, stack, 2, of, &tc, ray != ~0u);
            if (done) {
                shadow_done<kBatch>(sb, ray, s.hit.tri != ~0u, nxt, accum_in, weights_in, gv, bv);
                ray = ~0u;
            }
            const int n_idle = __popc(__ballot_sync(0xffffffffu, ray == ~0u));
            if (n_idle == 32 || (!drained && n_idle >= KS_TRAV_REFILL))
                break;
        }
    }
    if (of)
        atomicOr(overflow, 1);
    flush_counts(tc, work);
}

// ---- persistent two-level traversal (instanced scenes) ----------------------------------------
#ifndef KS_INST_MIN_BLOCKS
#define KS_INST_MIN_BLOCKS 1
#endif
// BLAS layout of the instanced kernels: the SBVH nodes (0) or their 4-wide view (1).
#ifndef KS_WIDE_INST
#define KS_WIDE_INST 1
#endif
using InstNode = std::conditional_t<KS_WIDE_INST != 0, WideNode, TravNode>;
// The same warp-level ray fetch as k_extend_pt / k_shadow_pt over inst_step (ks_traverse.cuh):
// each ray makes the tests of traverse_instances, in resumable steps.
__global__ void __launch_bounds__(128, KS_INST_MIN_BLOCKS) k_extend_inst_pt(const __grid_constant__ SceneView sv, PathBuf pb,
                                                        uint32_t count, float4 *hits, uint32_t *hit_inst,
                                                        uint32_t *fetch, int *overflow, unsigned long long *work)
{
    TravCount tc;
    KS_TRAV_STACK(stack);
    InstTravState s;
    uint4 tstack[kTlasStackDepth];
    uint32_t ray = ~0u;
    bool drained = false;
    int of = 0;
    while (true) {
        const uint32_t id = warp_fetch(fetch, count, ray == ~0u, drained);
        if (id != ~0u) {
            float4 a = pb.o_pdf[id], b = pb.d_info[id];
            RayQuery q;
            q.o = mk(a.x, a.y, a.z);
            q.d = mk(b.x, b.y, b.z);
            q.tmin = 0.0f;
            q.tmax = kInf;
            if (inst_begin(s, sv.inst, q)) {
                ray = id;
            } else {
                hits[id] = make_float4(0, 0, 0, fbits(~0u));
                hit_inst[id] = 0;
            }
        }
        if (__ballot_sync(0xffffffffu, ray != ~0u) == 0) {
            if (drained)
                break;
            continue;
        }
        while (true) {
            if (inst_warp_step<false>(tree_of<InstNode>(sv), sv.prim_tris, sv.inst, s, tstack, stack, 2, of, &tc,
                                      ray != ~0u)) {
                hits[ray] = s.hit.tri != ~0u ? make_float4(s.hit.t, s.hit.b1, s.hit.b2, fbits(s.hit.slot))
                                             : make_float4(0, 0, 0, fbits(~0u));
                hit_inst[ray] = s.hit_inst;
                ray = ~0u;
            }
            const int n_idle = __popc(__ballot_sync(0xffffffffu, ray == ~0u));
            if (n_idle == 32 || (!drained && n_idle >= KS_TRAV_REFILL))
                break;
        }
    }
    if (of)
        atomicOr(overflow, 1);
    flush_counts(tc, work);
}

__global__ void __launch_bounds__(128, KS_INST_MIN_BLOCKS) k_shadow_inst_pt(const __grid_constant__ SceneView sv, ShadowBuf sb,
                                                        const uint32_t *shadow_count, uint32_t *fetch, PathBuf nxt,
                                                        double *accum, double *weights, int *overflow,
                                                        unsigned long long *work, GuideView gv)
{
    const uint32_t count = *shadow_count;
    TravCount tc;
    KS_TRAV_STACK(stack);
    InstTravState s;
    uint4 tstack[kTlasStackDepth];
    uint32_t ray = ~0u;
    bool drained = false;
    int of = 0;
    while (true) {
        const uint32_t id = warp_fetch(fetch, count, ray == ~0u, drained);
        if (id != ~0u) {
            float4 a = sb.o_tmax[id], b = sb.d_target[id];
            RayQuery q;
            q.o = mk(a.x, a.y, a.z);
            q.d = mk(b.x, b.y, b.z);
            q.tmin = 0.0f;
            q.tmax = a.w;
            if (inst_begin(s, sv.inst, q))
                ray = id;
            else
                shadow_done<false>(sb, id, false, nxt, accum, weights, gv, BatchView{});
        }
        if (__ballot_sync(0xffffffffu, ray != ~0u) == 0) {
            if (drained)
                break;
            continue;
        }
        while (true) {
            if (ray != ~0u &&
                inst_step<true>(tree_of<InstNode>(sv), sv.prim_tris, sv.inst, s, tstack, stack, 2, of, &tc)) {
                shadow_done<false>(sb, ray, s.hit.tri != ~0u, nxt, accum, weights, gv, BatchView{});
                ray = ~0u;
            }
            const int n_idle = __popc(__ballot_sync(0xffffffffu, ray == ~0u));
            if (n_idle == 32 || (!drained && n_idle >= KS_TRAV_REFILL))
                break;
        }
    }
    if (of)
        atomicOr(overflow, 1);
    flush_counts(tc, work);
}

// Guided renders: the hit paths the guide is evaluated for (those that sample a direction at a
// bounce below guided_bounces, the bounces its training records come from, with a material at
// least min_roughness rough) go to gqueue; the others get selection probability 0 (their two
// weight vectors zeroed), so the shading samples their BSDF only.
__global__ void __launch_bounds__(128) k_guide_filter(const __grid_constant__ SceneView sv, int guided_bounces,
                                                      float min_roughness, PathBuf cur, const float4 *hits,
                                                      const uint32_t *queue, const uint32_t *queue_count,
                                                      uint32_t *gqueue, uint32_t *gcount, float4 *lobes,
                                                      uint32_t cap)
{
    const uint32_t count = *queue_count;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += stride) {
        const uint32_t q = base + threadIdx.x;
        bool use = false;
        uint32_t i = 0;
        if (q < count) {
            i = queue[q];
            const int bounce = (int)(bits(cur.d_info[i].w) & 0xffffu);
            if (bounce < guided_bounces) {
                const uint32_t tri = bits(__ldg(&sv.prim_tris[3 * (size_t)bits(hits[i].w)]).w);
                const uint32_t mesh = __ldg(&sv.tri_mesh[tri]);
                use = sv.materials[__ldg(&sv.mesh_material[mesh])].roughness >= min_roughness;
            }
            if (!use) {
                lobes[(size_t)8 * cap + i] = make_float4(0, 0, 0, 0);
                lobes[(size_t)9 * cap + i] = make_float4(0, 0, 0, 0);
            }
        }
        const uint32_t j = warp_append(gcount, use);
        if (use)
            gqueue[j] = i;
    }
}

// Relative MSE of the composited image (RenderTarget2::composite_and_save_to_exr,
// render_target.cpp:181-205) against a reference: sum over pixels and channels of
// (x - r)^2 / (r^2 + eps), accumulated in FP64 (one atomic per warp).
__global__ void k_rel_mse(const double *accum, const double *weights, const double *ref, uint32_t n, double eps,
                          double b0, double b1, double b2, double *out)
{
    double acc = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double w0 = weights[2 * (size_t)i], w1 = weights[2 * (size_t)i + 1];
        double w_sum = (double)(uint32_t)(w0 + w1);
        double w = w_sum == 0.0 ? 0.0 : w0 / fmax(w_sum, 1.0);
        const double bd[3] = {b0, b1, b2};
        for (int c = 0; c < 3; ++c) {
            double fg = w0 == 0.0 ? 0.0 : accum[3 * (size_t)i + c] / w0;
            double x = (1.0 - w) * bd[c] + w * fg;
            double r = ref[3 * (size_t)i + c];
            acc += (x - r) * (x - r) / (r * r + eps);
        }
    }
    for (int o = 16; o > 0; o >>= 1)
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(out, acc);
}

} // namespace
} // namespace ksb

using namespace ksb;

// One wave of resident CTAs of a persistent kernel.
template <class Kernel>
static unsigned resident_grid(Kernel kernel, int block, int sm_count)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return (unsigned)per_sm * (unsigned)sm_count;
}

struct RenderWork
{
    DevBuf<float4> state[2][4];
    DevBuf<float4> hits;
    DevBuf<uint32_t> hit_inst; // instanced scenes: instance of each hit
    DevBuf<float4> samples; // 4 per path slot
    DevBuf<float4> shadow[4];
    DevBuf<uint32_t> counters; // [next, shadow, hit queue, miss queue, extension fetch, shadow fetch]
    DevBuf<uint32_t> queue[2]; // hit / miss path indices
    DevBuf<int> overflow;
    DevBuf<float> filter; // the pixel filter's sample table (Gaussian / Blackman-Harris)
    uint32_t capacity = 0;
    uint32_t *h_counts = nullptr; // pinned: the loop's path counts read back each iteration
    RenderWork() = default;
    RenderWork(const RenderWork &) = delete;
    RenderWork &operator=(const RenderWork &) = delete;
    ~RenderWork()
    {
        if (h_counts)
            cudaFreeHost(h_counts);
    }
};

// Buffers of the single-job renders kept by the context between calls: allocating and freeing the
// wavefront state (about 9.2 GB at 32 M path slots) and the accumulators took tens of milliseconds
// per render.  A render that starts while the cache is in use (from a progress callback) uses
// buffers of its own.
struct RenderCache
{
    RenderWork work;
    bool work_busy = false;
    DevBuf<double> accum, weights; // the host-buffer entry's device accumulators
    double *staging = nullptr;     // pinned host copy of them
    size_t staging_n = 0;
    bool host_busy = false;
    cudaStream_t aux = nullptr;    // guided renders: the guide runs here beside sampling and miss shading
    ~RenderCache()
    {
        if (staging)
            cudaFreeHost(staging);
        if (aux)
            cudaStreamDestroy(aux);
    }
};

static RenderCache &render_cache(ks_context *ctx)
{
    if (!ctx->render_cache)
        ctx->render_cache = std::make_shared<RenderCache>();
    return *static_cast<RenderCache *>(ctx->render_cache.get());
}

// Marks a cached buffer set in use for a scope.
struct CacheLease
{
    bool *flag;
    explicit CacheLease(bool *f) : flag(f)
    {
        if (flag)
            *flag = true;
    }
    ~CacheLease()
    {
        if (flag)
            *flag = false;
    }
};

// RenderParams of one render (SmallPTInput fields + camera); false for an empty crop window.
// DistribTable (distrib.cpp:9-30): the normalised CDF of n values, appended to `out`; returns
// their integral (acc).
static float append_cdf(const float *f, uint32_t n, std::vector<float> &out)
{
    const size_t base = out.size();
    out.resize(base + n + 1);
    float *cdf = &out[base];
    cdf[0] = 0;
    const float invn = 1.0f / (float)n;
    for (uint32_t i = 1; i < n + 1; ++i)
        cdf[i] = cdf[i - 1] + f[i - 1] * invn;
    const float acc = cdf[n];
    if (acc == 0.0f) {
        for (uint32_t i = 0; i < n + 1; ++i)
            cdf[i] = (float)i / (float)n;
    } else {
        const float invacc = 1.0f / acc;
        for (uint32_t i = 0; i < n + 1; ++i)
            cdf[i] *= invacc;
    }
    cdf[n] = 1.0f;
    return acc;
}

// PixelFilterSampleTable (render_target.h:79-92) of a Gaussian (1) or Blackman-Harris (2) filter of
// radius r: the filter at the centres of an n x n grid over [-r, r]^2, n = ceil(32 r), as a
// DistribTable2D (distrib.cpp:61-72): the n conditional CDFs (n + 1 floats each), then the
// marginal one.  The filters as GaussianPixelFilter / BlackmanHarrisPixelFilter evaluate them
// (render_target.h:127-180, gaussian() maths.h:1070-1073), in float.
static std::vector<float> filter_table(int type, float r, float sigma, uint32_t &n_out)
{
    constexpr float pi = 3.14159265359f, two_pi = 6.28318530718f;
    auto gaussian = [&](float x) {
        return 1.0f / std::sqrt(two_pi * sigma * sigma) * std::exp(-((x - 0.0f) * (x - 0.0f)) / (2.0f * sigma * sigma));
    };
    const float threshold = type == 1 ? gaussian(r) : 0.0f;
    auto eval = [&](float x, float y) {
        if (x < -r || x > r || y < -r || y > r)
            return 0.0f;
        if (type == 1)
            return (gaussian(x) - threshold) * (gaussian(y) - threshold);
        constexpr float a0 = 0.35875f, a1 = 0.48829f, a2 = 0.14128f, a3 = 0.01168f;
        const float tx = (x + r) / (2.0f * r);
        const float fx = a0 - a1 * std::cos(2.0f * pi * tx) + a2 * std::cos(4.0f * pi * tx) - a3 * std::cos(6.0f * pi * tx);
        const float ty = (y + r) / (2.0f * r);
        const float fy = a0 - a1 * std::cos(2.0f * pi * ty) + a2 * std::cos(4.0f * pi * ty) - a3 * std::cos(6.0f * pi * ty);
        return fx * fy;
    };
    const uint32_t n = (uint32_t)(int)std::ceil(32 * r);
    std::vector<float> f((size_t)n * n);
    for (uint32_t y = 0; y < n; ++y)
        for (uint32_t x = 0; x < n; ++x)
            f[(size_t)y * n + x] = eval(std::lerp(-r, r, (x + 0.5f) / n), std::lerp(-r, r, (y + 0.5f) / n));
    std::vector<float> out, margin(n);
    out.reserve((size_t)(n + 1) * (n + 1));
    for (uint32_t y = 0; y < n; ++y)
        margin[y] = append_cdf(&f[(size_t)y * n], n, out);
    append_cdf(margin.data(), n, out);
    n_out = n;
    return out;
}

// The pixel filter of the parameters: false for bad values (unknown type, width <= 0, a table
// of more than 256 x 256 cells, a Gaussian sigma <= 0).
static bool pixel_filter_table(const ks_small_pt_params *in, std::vector<float> &table, uint32_t &n)
{
    table.clear();
    n = 0;
    const float width = in->pixel_filter_width > 0.0f ? in->pixel_filter_width : 1.0f;
    if (in->pixel_filter == 0)
        return true;
    if (in->pixel_filter < 0 || in->pixel_filter > 2 || !(width <= 16.0f) ||
        (in->pixel_filter == 1 && !(in->pixel_filter_sigma > 0.0f)))
        return false;
    table = filter_table(in->pixel_filter, 0.5f * width, in->pixel_filter_sigma, n);
    return true;
}

static bool fill_params(const ks_camera_desc *cam, const ks_small_pt_params *in, RenderParams &rp)
{
    const int W = in->render_width, H = in->render_height;
    rp = RenderParams{};
    rp.W = W;
    rp.H = H;
    rp.cx = 0;
    rp.cy = 0;
    rp.cw = W;
    rp.ch = H;
    if (in->crop_width > 0 && in->crop_height > 0) {
        rp.cx = std::max(in->crop_start_x, 0);
        rp.cy = std::max(in->crop_start_y, 0);
        rp.cw = std::min(in->crop_width, W - rp.cx);
        rp.ch = std::min(in->crop_height, H - rp.cy);
        if (rp.cw <= 0 || rp.ch <= 0)
            return false;
    }
    rp.spp = in->spp;
    rp.seed = in->rng_seed;
    sobol_setup(in->spp, W, H, rp.log2_spp, rp.n_digits);
    rp.bounces = in->bounces;
    rp.include_background = in->include_background;
    rp.clamp_direct = in->clamp_direct;
    rp.clamp_indirect = in->clamp_indirect;
    rp.filter_r = 0.5f * (in->pixel_filter_width > 0.0f ? in->pixel_filter_width : 1.0f);
    rp.ortho = cam->orthographic ? 1 : 0;
    {
        // Camera::direction: -(column 2 of camera_to_world).normalized()
        const float x = cam->camera_to_world[2], y = cam->camera_to_world[6], z = cam->camera_to_world[10];
        const float n = std::sqrt(x * x + y * y + z * z);
        rp.cam_dir[0] = -(x / n);
        rp.cam_dir[1] = -(y / n);
        rp.cam_dir[2] = -(z / n);
    }
    rp.cam_pos[0] = cam->camera_to_world[3];
    rp.cam_pos[1] = cam->camera_to_world[7];
    rp.cam_pos[2] = cam->camera_to_world[11];
    std::memcpy(rp.p2w, cam->proj_to_world, sizeof(rp.p2w));
    return true;
}

// Guided renders: per-slot mixtures, record index per path, training records.
struct GuideWork
{
    DevBuf<float4> lobes;
    DevBuf<uint32_t> gqueue, gcount; // hit paths the guide is evaluated for
    DevBuf<uint32_t> rec[2];
    DevBuf<float4> rec_f4[5]; // pos, wo, wi, ibeta, normal
    DevBuf<float> rec_t;
    DevBuf<uint32_t> rec_count;
};

static ks_status render_impl(ks_scene *scene, const ks_camera_desc *cam, const ks_small_pt_params *in,
                             ks_progress_fn cb, void *user, double *d_accum, double *d_weights, double *h_accum,
                             double *h_weights, ks_guide *guide = nullptr,
                             const ks_guide_render_options *gopt = nullptr, ks_device_progress_fn dcb = nullptr,
                             void *duser = nullptr)
{
    ks_context *ctx = scene->ctx;
    if (guide && scene->any_subsurface)
        return fail(ctx, KS_ERR_UNSUPPORTED, "guided renders of scenes with subsurface scattering");
    if (guide && guide_impl::context_of(guide) != ctx)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render_guided: guide and scene on different contexts");
    cudaStream_t st = ctx->stream;
    if (!scene->bvh_built || !scene->lights_built)
        return fail(ctx, KS_ERR_NOT_BUILT, "ks_small_pt_render: call ks_scene_build_bvh first");
    if (scene->light_count == 0)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render: the scene has no light");
    const int W = in->render_width, H = in->render_height;
    if (W <= 0 || H <= 0 || in->spp <= 0 || in->bounces < 0 || in->bounces > 0xfffe || in->spp_prog_interval <= 0)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render: bad resolution, spp, bounces or interval");
    if ((uint64_t)W * H >= (1ull << 31))
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render: resolution too large");
    RenderParams rp{};
    if (cam->orthographic != 0 && cam->orthographic != 1)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render: camera.orthographic must be 0 or 1 (fill the "
                                                  "descriptor with ks_camera_perspective / ks_camera_orthographic)");
    if (!fill_params(cam, in, rp))
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render: empty crop window");
    std::vector<float> ftab;
    if (!pixel_filter_table(in, ftab, rp.filter_n))
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render: bad pixel filter");

    SceneView sv = make_view(scene);
    const int variant = sv.shade_variant;
    const uint32_t n_pix = (uint32_t)rp.cw * (uint32_t)rp.ch;
    const uint64_t max_interval = (uint64_t)n_pix * (uint64_t)std::min(in->spp, in->spp_prog_interval);
    RenderCache &rc = render_cache(ctx);
    RenderWork own;
    RenderWork &w = rc.work_busy ? own : rc.work;
    CacheLease lease(rc.work_busy ? nullptr : &rc.work_busy);
    w.capacity = (uint32_t)std::min<uint64_t>(max_interval, 1u << KS_WAVE_LOG2);
    for (int b = 0; b < 2; ++b)
        for (int f = 0; f < 4; ++f)
            KS_CUDA_TRY(ctx, w.state[b][f].reserve(w.capacity));
    KS_CUDA_TRY(ctx, w.hits.reserve(w.capacity));
    if (scene->n_instances)
        KS_CUDA_TRY(ctx, w.hit_inst.reserve(w.capacity));
    KS_CUDA_TRY(ctx, w.samples.reserve(4 * (size_t)w.capacity));
    if (rp.filter_n) {
        KS_CUDA_TRY(ctx, w.filter.reserve(ftab.size()));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(w.filter.ptr, ftab.data(), sizeof(float) * ftab.size(),
                                         cudaMemcpyHostToDevice, st));
        rp.filter_cdf = w.filter.ptr;
    }
    KS_CUDA_TRY(ctx, w.queue[0].reserve(w.capacity));
    KS_CUDA_TRY(ctx, w.queue[1].reserve(w.capacity));
    for (int f = 0; f < 4; ++f)
        KS_CUDA_TRY(ctx, w.shadow[f].reserve(w.capacity));
    KS_CUDA_TRY(ctx, w.counters.reserve(kCounters));
    KS_CUDA_TRY(ctx, w.overflow.reserve(1));
    DevBuf<unsigned long long> work; // ext nodes, ext tris, shadow nodes, shadow tris
    KS_CUDA_TRY(ctx, work.alloc(4));
    KS_CUDA_TRY(ctx, cudaMemsetAsync(work.ptr, 0, 4 * sizeof(unsigned long long), st));
    KS_CUDA_TRY(ctx, cudaMemsetAsync(w.overflow.ptr, 0, sizeof(int), st));
    PathBuf pb[2];
    for (int b = 0; b < 2; ++b)
        pb[b] = PathBuf{w.state[b][0].ptr, w.state[b][1].ptr, w.state[b][2].ptr, w.state[b][3].ptr, nullptr};
    GuideWork gw;
    GuideView gv{};
    ks_guide_render_options go{};
    if (guide) {
        go = *gopt;
        if (go.guide_from_pass < 0 || go.train_passes < 0)
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render_guided: negative pass count");
        if (go.max_records == 0)
            go.max_records = 1u << 19;
        if (go.record_bounces <= 0)
            go.record_bounces = 6;
        if (!(go.min_roughness >= 0.0f))
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render_guided: negative or NaN min_roughness");
        KS_CUDA_TRY(ctx, gw.lobes.alloc((size_t)kGuideLobeVecs * w.capacity));
        KS_CUDA_TRY(ctx, gw.gqueue.alloc(w.capacity));
        KS_CUDA_TRY(ctx, gw.gcount.alloc(1));
        for (int b = 0; b < 2; ++b) {
            KS_CUDA_TRY(ctx, gw.rec[b].alloc(w.capacity));
            pb[b].rec = gw.rec[b].ptr;
        }
        if (go.train_passes > 0) {
            for (auto &f : gw.rec_f4)
                KS_CUDA_TRY(ctx, f.alloc(go.max_records));
            KS_CUDA_TRY(ctx, gw.rec_t.alloc(go.max_records));
        }
        KS_CUDA_TRY(ctx, gw.rec_count.alloc(1));
        KS_CUDA_TRY(ctx, cudaMemsetAsync(gw.rec_count.ptr, 0, sizeof(uint32_t), st));
        gv.lobes = gw.lobes.ptr;
        gv.cap = w.capacity;
        gv.rec_pos = gw.rec_f4[0].ptr;
        gv.rec_wo = gw.rec_f4[1].ptr;
        gv.rec_wi = gw.rec_f4[2].ptr;
        gv.rec_ibeta = gw.rec_f4[3].ptr;
        gv.rec_n = gw.rec_f4[4].ptr;
        gv.rec_t = gw.rec_t.ptr;
        gv.rec_count = gw.rec_count.ptr;
        gv.rec_bounces = (uint32_t)std::max(1, std::min(go.record_bounces, in->bounces));
        gv.min_roughness = go.min_roughness;
        // about twice max_records candidates per pass; paths that end early record nothing
        const double per_pass = (double)n_pix * std::min(in->spp, in->spp_prog_interval);
        gv.rec_threshold = (uint32_t)std::min(65536.0, std::ceil(65536.0 * 2.0 * go.max_records / per_pass));
    }
    ShadowBuf sb{w.shadow[0].ptr, w.shadow[1].ptr, w.shadow[2].ptr, w.shadow[3].ptr};
    // kept with the wavefront buffers: a pinned allocation and free per render cost milliseconds,
    // now and then far more
    if (!w.h_counts)
        KS_CUDA_TRY(ctx, cudaMallocHost((void **)&w.h_counts, sizeof(uint32_t) * 4));
    uint32_t *h_counts = w.h_counts;
    h_counts[2] = 0;
    // guided renders: the guide's filter and inference run on a second stream, overlapping the
    // sampling and the miss shading, and join before the hit shading
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_g0 = nullptr, ev_g1 = nullptr;
    if (guide) {
        if (!rc.aux)
            KS_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&rc.aux, cudaStreamNonBlocking));
        aux = rc.aux;
        cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming);
        cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming);
        cudaEventCreate(&ev_g0);
        cudaEventCreate(&ev_g1);
    }
    cudaEvent_t ev[6];
    for (auto &e : ev)
        cudaEventCreate(&e);
    cudaEvent_t t_begin, t_end;
    cudaEventCreate(&t_begin);
    cudaEventCreate(&t_end);
    cudaEventRecord(t_begin, st);
    ks_render_stats stats{};
    const unsigned max_grid = (unsigned)ctx->sm_count * 16;
    // opacity maps: the traversal kernels with the candidate-hit filter (flat scenes)
    const bool alpha = scene->any_opacity;
    const unsigned ext_grid = alpha ? resident_grid(k_extend_pt<false, true>, 128, ctx->sm_count)
                                    : resident_grid(k_extend_pt<false>, 128, ctx->sm_count);
    const unsigned shadow_grid = alpha ? resident_grid(k_shadow_pt<false, true>, 128, ctx->sm_count)
                                       : resident_grid(k_shadow_pt<false>, 128, ctx->sm_count);
    const unsigned inst_ext_grid = resident_grid(k_extend_inst_pt, 128, ctx->sm_count);
    const unsigned inst_shadow_grid = resident_grid(k_shadow_inst_pt, 128, ctx->sm_count);
    int cur = 0;
    cudaError_t err = cudaSuccess;
    std::vector<double> cb_acc, cb_w;
    int pass = 0;
    for (int s0 = 0; s0 < in->spp && err == cudaSuccess; s0 += in->spp_prog_interval, ++pass) {
        int batch = std::min(in->spp_prog_interval, in->spp - s0);
        const bool recording = guide && pass < go.train_passes;
        if (guide) {
            gv.active = pass >= go.guide_from_pass ? 1 : 0;
            gv.rec_cap = recording ? go.max_records : 0u;
        }
        uint64_t total = (uint64_t)n_pix * (uint64_t)batch, issued = 0;
        uint32_t cur_count = 0;
        // every path ends after at most bounces + 1 extension rays
        uint64_t watchdog = (total / w.capacity + 2) * (uint64_t)(in->bounces + 2) + 64;
        if (ctx->limits.wavefront_max_iterations)
            watchdog = std::min<uint64_t>(watchdog, ctx->limits.wavefront_max_iterations);
        uint64_t it_interval = 0;
        while ((issued < total || cur_count > 0) && err == cudaSuccess) {
            if (++it_interval > watchdog) {
                err = cudaErrorUnknown;
                stats.iterations = 0xffffffffu;
                break;
            }
            uint32_t n_new = (uint32_t)std::min<uint64_t>(w.capacity - cur_count, total - issued);
            cudaEventRecord(ev[0], st);
            if (n_new) {
                k_raygen<<<(n_new + 255) / 256, 256, 0, st>>>(rp, pb[cur], cur_count, issued, n_new, s0, n_pix);
                stats.kernel_launches++;
            }
            issued += n_new;
            uint32_t count = cur_count + n_new;
            stats.extension_rays += count;
            // counters: [0] next paths, [1] shadow rays, [2] hit queue, [3] miss queue, [4], [5] ray fetch
            cudaMemsetAsync(w.counters.ptr, 0, sizeof(uint32_t) * kCounters, st);
            unsigned grid = std::min<unsigned>((count + 127) / 128, max_grid);
            cudaEventRecord(ev[1], st);
            if (scene->n_instances) {
                if (kPersistentTraversal) {
                    k_extend_inst_pt<<<std::min(grid, inst_ext_grid), 128, 0, st>>>(
                        sv, pb[cur], count, w.hits.ptr, w.hit_inst.ptr, w.counters.ptr + 4, w.overflow.ptr, work.ptr);
                    k_build_queues<false><<<std::min((count + 255) / 256, max_grid), 256, 0, st>>>(
                        w.hits.ptr, count, w.queue[0].ptr, w.queue[1].ptr, w.counters.ptr + 2, BatchView{});
                    stats.kernel_launches++;
                } else {
                    k_extend<true><<<grid, 128, 0, st>>>(sv, pb[cur], count, w.hits.ptr, w.hit_inst.ptr,
                                                         w.queue[0].ptr, w.queue[1].ptr, w.counters.ptr + 2,
                                                         w.overflow.ptr, work.ptr, BatchView{});
                }
            } else if (!kPersistentTraversal)
                k_extend<false><<<grid, 128, 0, st>>>(sv, pb[cur], count, w.hits.ptr, nullptr, w.queue[0].ptr,
                                                      w.queue[1].ptr, w.counters.ptr + 2, w.overflow.ptr, work.ptr,
                                                      BatchView{});
            else {
                if (alpha)
                    k_extend_pt<false, true><<<std::min(grid, ext_grid), 128, 0, st>>>(
                        sv, pb[cur], count, w.hits.ptr, w.counters.ptr + 4, w.overflow.ptr, work.ptr, BatchView{});
                else
                    k_extend_pt<false><<<std::min(grid, ext_grid), 128, 0, st>>>(sv, pb[cur], count, w.hits.ptr,
                                                                                 w.counters.ptr + 4, w.overflow.ptr,
                                                                                 work.ptr, BatchView{});
                k_build_queues<false><<<std::min((count + 255) / 256, max_grid), 256, 0, st>>>(
                    w.hits.ptr, count, w.queue[0].ptr, w.queue[1].ptr, w.counters.ptr + 2, BatchView{});
                stats.kernel_launches++;
            }
            cudaEventRecord(ev[2], st);
            const bool guiding = guide && gv.active;
            if (guiding) {
                // the guide only at vertices that sample a direction with a rough enough BSDF
                cudaEventRecord(ev_fork, st);
                cudaStreamWaitEvent(aux, ev_fork, 0);
                cudaEventRecord(ev_g0, aux);
                cudaMemsetAsync(gw.gcount.ptr, 0, sizeof(uint32_t), aux);
                k_guide_filter<<<grid, 128, 0, aux>>>(sv, std::min<int>(rp.bounces, (int)gv.rec_bounces),
                                                      gv.min_roughness, pb[cur], w.hits.ptr,
                                                      w.queue[0].ptr, w.counters.ptr + 2, gw.gqueue.ptr,
                                                      gw.gcount.ptr, gw.lobes.ptr, w.capacity);
                stats.kernel_launches++;
                ks_status gs = guide_impl::infer_paths(guide, gw.gqueue.ptr, gw.gcount.ptr, pb[cur].o_pdf,
                                                       pb[cur].d_info, w.hits.ptr, sv.prim_tris, w.hit_inst.ptr,
                                                       sv.inst.xf, gw.lobes.ptr, w.capacity, count, aux);
                cudaEventRecord(ev_g1, aux);
                cudaEventRecord(ev_join, aux);
                if (gs != KS_OK) {
                    cudaStreamWaitEvent(st, ev_join, 0);
                    err = cudaErrorLaunchFailure;
                    break;
                }
                stats.kernel_launches++;
            }
            cudaEventRecord(ev[5], st);
            if (scene->any_subsurface) {
                launch_subsurface(grid, st, sv, rp, pb[cur], w.hits.ptr, w.queue[0].ptr, w.counters.ptr + 2,
                                  w.overflow.ptr);
                stats.kernel_launches++;
            }
            launch_sample(false, grid, st, sv, rp, pb[cur], w.hits.ptr, w.hit_inst.ptr, w.queue[0].ptr,
                          w.counters.ptr + 2, w.samples.ptr, BatchView{});
            // misses first (they do not read the guide), then the hits once the guide has joined
            for (int miss = 1; miss >= 0; --miss) {
                if (!miss && guiding)
                    cudaStreamWaitEvent(st, ev_join, 0);
                launch_shade(miss != 0, guide != nullptr, false, variant, grid, st, sv, rp, pb[cur], pb[1 - cur], w.hits.ptr,
                             w.hit_inst.ptr, w.samples.ptr, w.queue[miss].ptr, w.counters.ptr + 2 + miss,
                             w.counters.ptr, sb, w.counters.ptr + 1, d_accum, d_weights, gv, BatchView{});
            }
            cudaEventRecord(ev[3], st);
            if (scene->n_instances) {
                if (kPersistentTraversal)
                    k_shadow_inst_pt<<<std::min(grid, inst_shadow_grid), 128, 0, st>>>(
                        sv, sb, w.counters.ptr + 1, w.counters.ptr + 5, pb[1 - cur], d_accum, d_weights,
                        w.overflow.ptr, work.ptr + 2, gv);
                else
                    k_shadow<true><<<grid, 128, 0, st>>>(sv, sb, w.counters.ptr + 1, pb[1 - cur], d_accum, d_weights,
                                                         w.overflow.ptr, work.ptr + 2, gv, BatchView{});
            } else if (!kPersistentTraversal)
                k_shadow<false><<<grid, 128, 0, st>>>(sv, sb, w.counters.ptr + 1, pb[1 - cur], d_accum, d_weights,
                                                      w.overflow.ptr, work.ptr + 2, gv, BatchView{});
            else if (alpha)
                k_shadow_pt<false, true><<<std::min(grid, shadow_grid), 128, 0, st>>>(
                    sv, sb, w.counters.ptr + 1, w.counters.ptr + 5, pb[1 - cur], d_accum, d_weights, w.overflow.ptr,
                    work.ptr + 2, gv, BatchView{});
            else
                k_shadow_pt<false><<<std::min(grid, shadow_grid), 128, 0, st>>>(sv, sb, w.counters.ptr + 1, w.counters.ptr + 5,
                                                                pb[1 - cur], d_accum, d_weights, w.overflow.ptr,
                                                                work.ptr + 2, gv, BatchView{});
            cudaEventRecord(ev[4], st);
            stats.kernel_launches += 5;
            cudaMemcpyAsync(h_counts, w.counters.ptr, sizeof(uint32_t) * 2, cudaMemcpyDeviceToHost, st);
            if (guide && gv.active)
                cudaMemcpyAsync(h_counts + 2, gw.gcount.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
            err = cudaStreamSynchronize(st);
            if (err != cudaSuccess)
                break;
            err = cudaGetLastError();
            float ms;
            cudaEventElapsedTime(&ms, ev[0], ev[1]);
            stats.ms_shade += ms;
            cudaEventElapsedTime(&ms, ev[1], ev[2]);
            stats.ms_extend += ms;
            if (guiding) {
                cudaEventElapsedTime(&ms, ev_g0, ev_g1);
                stats.ms_guide_infer += ms;
            }
            cudaEventElapsedTime(&ms, ev[5], ev[3]);
            stats.ms_shade += ms;
            cudaEventElapsedTime(&ms, ev[3], ev[4]);
            stats.ms_shadow += ms;
            stats.shadow_rays += h_counts[1];
            if (guide && gv.active)
                stats.guide_rows += h_counts[2];
            stats.iterations++;
            cur_count = h_counts[0];
            cur = 1 - cur;
        }
        stats.paths += total;
        if (err == cudaSuccess && recording) {
            // train on the records of this pass, then start the next pass's capture from zero
            uint32_t n_rec = 0;
            err = cudaMemcpyAsync(&n_rec, gw.rec_count.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
            if (err == cudaSuccess)
                err = cudaStreamSynchronize(st);
            if (err != cudaSuccess)
                break;
            n_rec = std::min(n_rec, go.max_records);
            stats.guide_records += n_rec;
            cudaEventRecord(ev[0], st);
            ks_status gs = guide_impl::train_rows(guide, n_rec, gw.rec_f4[0].ptr, gw.rec_f4[1].ptr, gw.rec_f4[4].ptr,
                                                  gw.rec_f4[2].ptr, gw.rec_t.ptr, go.train_batch,
                                                  &stats.guide_train_steps);
            cudaEventRecord(ev[1], st);
            if (gs != KS_OK) {
                err = cudaErrorLaunchFailure;
                break;
            }
            err = cudaMemsetAsync(gw.rec_count.ptr, 0, sizeof(uint32_t), st);
            if (err == cudaSuccess)
                err = cudaEventSynchronize(ev[1]);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev[0], ev[1]);
            stats.ms_guide_train += ms;
        }
        if (err == cudaSuccess && dcb) {
            err = cudaStreamSynchronize(st);
            if (err == cudaSuccess && dcb(s0 + batch, duser) != 0)
                break;
        }
        if (err == cudaSuccess && cb && h_accum) {
            size_t na = (size_t)W * H * 3, nw = (size_t)W * H * 2;
            cb_acc.resize(na);
            cb_w.resize(nw);
            err = cudaMemcpyAsync(cb_acc.data(), d_accum, na * sizeof(double), cudaMemcpyDeviceToHost, st);
            if (err == cudaSuccess)
                err = cudaMemcpyAsync(cb_w.data(), d_weights, nw * sizeof(double), cudaMemcpyDeviceToHost, st);
            if (err == cudaSuccess)
                err = cudaStreamSynchronize(st);
            if (err == cudaSuccess) {
                // the callback sees the caller's running totals (initial contents + this render)
                for (size_t k = 0; k < na; ++k)
                    cb_acc[k] += h_accum[k];
                for (size_t k = 0; k < nw; ++k)
                    cb_w[k] += h_weights[k];
                cb(s0 + batch, cb_acc.data(), cb_w.data(), user);
            }
        }
    }
    cudaEventRecord(t_end, st);
    cudaEventSynchronize(t_end);
    cudaEventElapsedTime(&stats.ms_total, t_begin, t_end);
    for (auto &e : ev)
        cudaEventDestroy(e);
    for (cudaEvent_t e : {ev_fork, ev_join, ev_g0, ev_g1})
        if (e)
            cudaEventDestroy(e);
    cudaEventDestroy(t_begin);
    cudaEventDestroy(t_end);
    int overflow = 0;
    if (err == cudaSuccess)
        err = cudaMemcpy(&overflow, w.overflow.ptr, sizeof(int), cudaMemcpyDeviceToHost);
    unsigned long long h_work[4] = {0, 0, 0, 0};
    if (err == cudaSuccess)
        err = cudaMemcpy(h_work, work.ptr, sizeof(h_work), cudaMemcpyDeviceToHost);
    stats.ext_nodes = h_work[0];
    stats.ext_tris = h_work[1];
    stats.shadow_nodes = h_work[2];
    stats.shadow_tris = h_work[3];
    scene->last_stats = stats;
    if (stats.iterations == 0xffffffffu)
        return fail(ctx, KS_ERR_WATCHDOG, "ks_small_pt_render: wavefront iteration limit reached");
    if (err != cudaSuccess)
        return cuda_fail(ctx, err, "ks_small_pt_render");
    if (overflow)
        return fail(ctx, KS_ERR_QUEUE_OVERFLOW, "ks_small_pt_render: traversal stack depth exceeded");
    if (guide)
        return guide_impl::status(guide);
    return KS_OK;
}

// ---- batched rendering ----------------------------------------------------------------------
struct BatchWork
{
    DevBuf<float4> state[2][4];
    DevBuf<float4> hits, samples, shadow[4];
    DevBuf<uint32_t> counters, queue[2];
    DevBuf<int> overflow;
    DevBuf<unsigned long long> work;
    DevBuf<SceneView> views;
    DevBuf<RenderParams> params;
    DevBuf<double *> accum, weights;
    DevBuf<unsigned long long> path_begin;
    DevBuf<BatchState> state_dev;
    DevBuf<float> filters; // the jobs' pixel-filter sample tables, concatenated
    unsigned ext_grid = 0, shadow_grid = 0; // one wave of resident CTAs of the traversal kernels
    int variant = kShadePlain;              // the shading kernel variant of the most demanding job
};

// Validates the jobs and fills the per-job tables; returns the total path count in *total.
static ks_status batch_tables(ks_context *ctx, const ks_batch_job *jobs, uint32_t n, BatchWork &w,
                              unsigned long long *total, int *max_bounces)
{
    if (!jobs || n == 0 || n > kMaxJobs)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_batch_render_device: 1 to 1024 jobs");
    std::vector<SceneView> views(n);
    std::vector<RenderParams> params(n);
    std::vector<double *> acc(n), wts(n);
    std::vector<unsigned long long> begin(n + 1, 0);
    std::vector<float> filter_host;
    std::vector<size_t> filter_off(n, 0);
    *max_bounces = 0;
    w.variant = kShadePlain;
    for (uint32_t j = 0; j < n; ++j) {
        const ks_batch_job &jb = jobs[j];
        const ks_small_pt_params &in = jb.params;
        if (!jb.scene || jb.scene->ctx != ctx || !jb.accum_rgb_device || !jb.weights_device)
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_batch_render_device: job " + std::to_string(j) +
                                                          ": null scene/buffer or scene of another context");
        if (!jb.scene->bvh_built || !jb.scene->lights_built)
            return fail(ctx, KS_ERR_NOT_BUILT, "ks_batch_render_device: job " + std::to_string(j) +
                                                   ": call ks_scene_build_bvh first");
        if (jb.scene->light_count == 0 || jb.scene->n_instances)
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_batch_render_device: job " + std::to_string(j) +
                                                          ": scene without lights or instanced");
        if (in.render_width <= 0 || in.render_height <= 0 || in.spp <= 0 || in.bounces < 0 || in.bounces > 0xfffe ||
            (uint64_t)in.render_width * in.render_height > (1ull << kJobShift))
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_batch_render_device: job " + std::to_string(j) +
                                                          ": bad resolution (at most 2^21 pixels), spp or bounces");
        if (jb.camera.orthographic != 0 && jb.camera.orthographic != 1)
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_batch_render_device: job " + std::to_string(j) +
                                                          ": camera.orthographic must be 0 or 1");
        if (!fill_params(&jb.camera, &in, params[j]))
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_batch_render_device: empty crop window");
        std::vector<float> ftab;
        if (!pixel_filter_table(&in, ftab, params[j].filter_n))
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_batch_render_device: job " + std::to_string(j) +
                                                          ": bad pixel filter");
        filter_off[j] = filter_host.size();
        filter_host.insert(filter_host.end(), ftab.begin(), ftab.end());
        if (jb.scene->any_opacity || jb.scene->any_subsurface)
            return fail(ctx, KS_ERR_UNSUPPORTED, "ks_batch_render_device: job " + std::to_string(j) +
                                                     ": opacity maps or subsurface scattering (render the scene "
                                                     "with ks_small_pt_render)");
        views[j] = make_view(jb.scene);
        w.variant = std::max(w.variant, views[j].shade_variant);
        acc[j] = jb.accum_rgb_device;
        wts[j] = jb.weights_device;
        begin[j + 1] = begin[j] + (unsigned long long)params[j].cw * params[j].ch * (unsigned long long)in.spp;
        *max_bounces = std::max(*max_bounces, in.bounces);
    }
    *total = begin[n];
    cudaStream_t st = ctx->stream;
    if (!filter_host.empty()) {
        KS_CUDA_TRY(ctx, w.filters.alloc(filter_host.size()));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(w.filters.ptr, filter_host.data(), sizeof(float) * filter_host.size(),
                                         cudaMemcpyHostToDevice, ctx->stream));
        for (uint32_t j = 0; j < n; ++j)
            if (params[j].filter_n)
                params[j].filter_cdf = w.filters.ptr + filter_off[j];
    }
    KS_CUDA_TRY(ctx, w.views.alloc(n));
    KS_CUDA_TRY(ctx, w.params.alloc(n));
    KS_CUDA_TRY(ctx, w.accum.alloc(n));
    KS_CUDA_TRY(ctx, w.weights.alloc(n));
    KS_CUDA_TRY(ctx, w.path_begin.alloc(n + 1));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(w.views.ptr, views.data(), w.views.bytes(), cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(w.params.ptr, params.data(), w.params.bytes(), cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(w.accum.ptr, acc.data(), w.accum.bytes(), cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(w.weights.ptr, wts.data(), w.weights.bytes(), cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(w.path_begin.ptr, begin.data(), w.path_begin.bytes(), cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return KS_OK;
}

// One wavefront iteration of a batch, enqueued on the stream (captured into the graph body).
static void batch_iteration(ks_context *ctx, BatchWork &w, const BatchView &bv, PathBuf *pb, const ShadowBuf &sb,
                            int cur, uint32_t capacity, unsigned grid, cudaGraphConditionalHandle handle, int use_graph)
{
    cudaStream_t st = ctx->stream;
    uint32_t *cnt = w.counters.ptr;
    const GuideView gv{};
    k_batch_prep<<<1, 32, 0, st>>>(bv.state, cnt, capacity);
    k_raygen_batch<<<(unsigned)ctx->sm_count * 8, 256, 0, st>>>(bv, pb[cur]);
    k_extend_pt<true><<<w.ext_grid, 128, 0, st>>>(SceneView{}, pb[cur], 0u, w.hits.ptr, cnt + 4, w.overflow.ptr,
                                                w.work.ptr, bv);
    k_build_queues<true><<<grid, 256, 0, st>>>(w.hits.ptr, 0u, w.queue[0].ptr, w.queue[1].ptr, cnt + 2, bv);
    launch_sample(true, grid, st, SceneView{}, RenderParams{}, pb[cur], w.hits.ptr, nullptr, w.queue[0].ptr, cnt + 2,
                  w.samples.ptr, bv);
    for (int miss = 0; miss < 2; ++miss)
        launch_shade(miss != 0, false, true, w.variant, grid, st, SceneView{}, RenderParams{}, pb[cur], pb[1 - cur], w.hits.ptr,
                     nullptr, w.samples.ptr, w.queue[miss].ptr, cnt + 2 + miss, cnt, sb, cnt + 1, nullptr, nullptr,
                     gv, bv);
    k_shadow_pt<true><<<w.shadow_grid, 128, 0, st>>>(SceneView{}, sb, cnt + 1, cnt + 5, pb[1 - cur], nullptr, nullptr,
                                                   w.overflow.ptr, w.work.ptr + 2, gv, bv);
    k_batch_advance<<<1, 32, 0, st>>>(bv.state, cnt, handle, use_graph);
}

static ks_status batch_render(ks_context *ctx, const ks_batch_job *jobs, uint32_t n, const ks_batch_options &o,
                              ks_batch_stats *out)
{
    cudaStream_t st = ctx->stream;
    BatchWork w;
    unsigned long long total = 0;
    int max_bounces = 0;
    ks_status s = batch_tables(ctx, jobs, n, w, &total, &max_bounces);
    if (s != KS_OK)
        return s;
    const uint32_t capacity =
        (uint32_t)std::max<unsigned long long>(1, std::min<unsigned long long>(o.capacity ? o.capacity : 1u << 22,
                                                                               total));
    const unsigned grid = (unsigned)ctx->sm_count * (o.grid_per_sm ? std::min(o.grid_per_sm, 64u) : 16u);
    w.ext_grid = resident_grid(k_extend_pt<true>, 128, ctx->sm_count);
    w.shadow_grid = resident_grid(k_shadow_pt<true>, 128, ctx->sm_count);
    for (int b = 0; b < 2; ++b)
        for (int f = 0; f < 4; ++f)
            KS_CUDA_TRY(ctx, w.state[b][f].alloc(capacity));
    KS_CUDA_TRY(ctx, w.hits.alloc(capacity));
    KS_CUDA_TRY(ctx, w.samples.alloc(4 * (size_t)capacity));
    for (auto &q : w.queue)
        KS_CUDA_TRY(ctx, q.alloc(capacity));
    for (auto &f : w.shadow)
        KS_CUDA_TRY(ctx, f.alloc(capacity));
    KS_CUDA_TRY(ctx, w.counters.alloc(kCounters));
    KS_CUDA_TRY(ctx, w.overflow.alloc(1));
    KS_CUDA_TRY(ctx, w.work.alloc(4));
    KS_CUDA_TRY(ctx, w.state_dev.alloc(1));
    BatchState init{};
    init.total = total;
    // every path ends after at most bounces + 1 extension rays
    init.max_iterations = (uint32_t)std::min<unsigned long long>((total / capacity + 2) * (max_bounces + 2) + 64,
                                                                  0x7fffffffull);
    if (ctx->limits.wavefront_max_iterations)
        init.max_iterations = std::min(init.max_iterations, ctx->limits.wavefront_max_iterations);
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(w.state_dev.ptr, &init, sizeof(init), cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemsetAsync(w.counters.ptr, 0, sizeof(uint32_t) * kCounters, st));
    KS_CUDA_TRY(ctx, cudaMemsetAsync(w.overflow.ptr, 0, sizeof(int), st));
    KS_CUDA_TRY(ctx, cudaMemsetAsync(w.work.ptr, 0, sizeof(unsigned long long) * 4, st));
    BatchView bv{w.views.ptr, w.params.ptr, w.accum.ptr, w.weights.ptr, w.path_begin.ptr, n, w.state_dev.ptr};
    PathBuf pb[2];
    for (int b = 0; b < 2; ++b)
        pb[b] = PathBuf{w.state[b][0].ptr, w.state[b][1].ptr, w.state[b][2].ptr, w.state[b][3].ptr, nullptr};
    ShadowBuf sb{w.shadow[0].ptr, w.shadow[1].ptr, w.shadow[2].ptr, w.shadow[3].ptr};

    cudaEvent_t e0, e1;
    KS_CUDA_TRY(ctx, cudaEventCreate(&e0));
    KS_CUDA_TRY(ctx, cudaEventCreate(&e1));
    cudaError_t err = cudaSuccess;
    uint32_t graph_launches = 0;
    if (o.use_graph) {
        // while (more) { iteration(buffers 0 -> 1); iteration(buffers 1 -> 0); }
        cudaGraph_t graph = nullptr, body = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaGraphConditionalHandle handle{};
        err = cudaGraphCreate(&graph, 0);
        if (err == cudaSuccess)
            err = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        if (err == cudaSuccess)
            err = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
        if (err == cudaSuccess) {
            body = cp.conditional.phGraph_out[0];
            err = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
            if (err == cudaSuccess) {
                batch_iteration(ctx, w, bv, pb, sb, 0, capacity, grid, handle, 1);
                batch_iteration(ctx, w, bv, pb, sb, 1, capacity, grid, handle, 1);
                cudaError_t launch_err = cudaGetLastError();
                err = cudaStreamEndCapture(st, &body);
                if (err == cudaSuccess)
                    err = launch_err;
            }
        }
        if (err == cudaSuccess)
            err = cudaGraphInstantiate(&exec, graph, 0);
        if (err == cudaSuccess) {
            cudaEventRecord(e0, st);
            err = cudaGraphLaunch(exec, st);
            cudaEventRecord(e1, st);
            graph_launches = 1;
        }
        if (err == cudaSuccess)
            err = cudaStreamSynchronize(st);
        if (exec)
            cudaGraphExecDestroy(exec);
        if (graph)
            cudaGraphDestroy(graph);
    } else {
        cudaEventRecord(e0, st);
        for (uint32_t pair = 0; err == cudaSuccess; ++pair) {
            batch_iteration(ctx, w, bv, pb, sb, 0, capacity, grid, cudaGraphConditionalHandle{}, 0);
            batch_iteration(ctx, w, bv, pb, sb, 1, capacity, grid, cudaGraphConditionalHandle{}, 0);
            BatchState hs{};
            uint32_t next = 0;
            err = cudaMemcpyAsync(&hs, w.state_dev.ptr, sizeof(hs), cudaMemcpyDeviceToHost, st);
            if (err == cudaSuccess)
                err = cudaMemcpyAsync(&next, w.counters.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
            if (err == cudaSuccess)
                err = cudaStreamSynchronize(st);
            if (err != cudaSuccess || hs.error || hs.iterations >= hs.max_iterations ||
                !(hs.issued < hs.total || next > 0))
                break;
        }
        cudaEventRecord(e1, st);
        if (err == cudaSuccess)
            err = cudaStreamSynchronize(st);
    }
    float ms = 0.0f;
    if (err == cudaSuccess)
        cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess)
        return cuda_fail(ctx, err, "ks_batch_render_device");
    BatchState hs{};
    int overflow = 0;
    KS_CUDA_TRY(ctx, cudaMemcpy(&hs, w.state_dev.ptr, sizeof(hs), cudaMemcpyDeviceToHost));
    KS_CUDA_TRY(ctx, cudaMemcpy(&overflow, w.overflow.ptr, sizeof(int), cudaMemcpyDeviceToHost));
    if (out) {
        *out = ks_batch_stats{};
        out->paths = hs.issued;
        out->extension_rays = hs.ext_rays;
        out->shadow_rays = hs.shadow_rays;
        out->iterations = hs.iterations;
        out->graph_launches = graph_launches;
        out->ms_total = ms;
    }
    if (hs.error)
        return fail(ctx, KS_ERR_WATCHDOG, "ks_batch_render_device: wavefront iteration limit reached");
    if (overflow)
        return fail(ctx, KS_ERR_QUEUE_OVERFLOW, "ks_batch_render_device: traversal stack depth exceeded");
    return KS_OK;
}

extern "C" {

ks_status ks_small_pt_render_device(ks_scene *scene, const ks_camera_desc *camera, const ks_small_pt_params *params,
                                    double *accum_rgb_device, double *weights_device)
{
    if (!scene || !camera || !params || !accum_rgb_device || !weights_device)
        return fail(scene ? scene->ctx : nullptr, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render_device: null");
    KS_CUDA_TRY(scene->ctx, enter_device(scene->ctx));
    return render_impl(scene, camera, params, nullptr, nullptr, accum_rgb_device, weights_device, nullptr, nullptr);
}

static ks_status render_host(ks_scene *scene, const ks_camera_desc *camera, const ks_small_pt_params *params,
                             ks_progress_fn cb, void *user, double *accum_rgb, double *weights, ks_guide *guide,
                             const ks_guide_render_options *gopt)
{
    if (!scene || !camera || !params || !accum_rgb || !weights)
        return fail(scene ? scene->ctx : nullptr, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render: null");
    ks_context *ctx = scene->ctx;
    KS_CUDA_TRY(ctx, enter_device(ctx));
    if (params->render_width <= 0 || params->render_height <= 0)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render: bad resolution");
    size_t na = (size_t)params->render_width * params->render_height * 3;
    size_t nw = (size_t)params->render_width * params->render_height * 2;
    RenderCache &rc = render_cache(ctx);
    DevBuf<double> own_a, own_w;
    const bool cached = !rc.host_busy;
    CacheLease lease(cached ? &rc.host_busy : nullptr);
    DevBuf<double> &da = cached ? rc.accum : own_a, &dw = cached ? rc.weights : own_w;
    KS_CUDA_TRY(ctx, da.reserve(na));
    KS_CUDA_TRY(ctx, dw.reserve(nw));
    KS_CUDA_TRY(ctx, cudaMemsetAsync(da.ptr, 0, na * sizeof(double), ctx->stream));
    KS_CUDA_TRY(ctx, cudaMemsetAsync(dw.ptr, 0, nw * sizeof(double), ctx->stream));
    ks_status s = render_impl(scene, camera, params, cb, user, da.ptr, dw.ptr, accum_rgb, weights, guide, gopt);
    if (s != KS_OK)
        return s;
    // through pinned staging (pageable copies run at a fraction of the link's speed)
    std::vector<double> own_h;
    double *h = nullptr;
    if (cached) {
        if (rc.staging_n < na + nw) {
            if (rc.staging)
                cudaFreeHost(rc.staging);
            rc.staging = nullptr;
            rc.staging_n = 0;
            KS_CUDA_TRY(ctx, cudaMallocHost((void **)&rc.staging, (na + nw) * sizeof(double)));
            rc.staging_n = na + nw;
        }
        h = rc.staging;
    } else {
        own_h.resize(na + nw);
        h = own_h.data();
    }
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(h, da.ptr, na * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(h + na, dw.ptr, nw * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    host_parallel(na, 1u << 17, [&](size_t b, size_t e) {
        for (size_t k = b; k < e; ++k)
            accum_rgb[k] += h[k];
    });
    host_parallel(nw, 1u << 17, [&](size_t b, size_t e) {
        for (size_t k = b; k < e; ++k)
            weights[k] += h[na + k];
    });
    return KS_OK;
}

ks_status ks_small_pt_render(ks_scene *scene, const ks_camera_desc *camera, const ks_small_pt_params *params,
                             ks_progress_fn cb, void *user, double *accum_rgb, double *weights)
{
    return render_host(scene, camera, params, cb, user, accum_rgb, weights, nullptr, nullptr);
}

void ks_guide_render_options_default(ks_guide_render_options *o)
{
    if (!o)
        return;
    o->guide_from_pass = 1;
    o->train_passes = 8;
    o->max_records = 1u << 19;
    o->train_batch = 1u << 18;
    o->record_bounces = 6;
    o->min_roughness = 0.3f;
}

ks_status ks_small_pt_render_guided(ks_scene *scene, const ks_camera_desc *camera, const ks_small_pt_params *params,
                                    ks_guide *guide, const ks_guide_render_options *options, ks_progress_fn cb,
                                    void *user, double *accum_rgb, double *weights)
{
    if (!guide || !options)
        return fail(scene ? scene->ctx : nullptr, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render_guided: null");
    return render_host(scene, camera, params, cb, user, accum_rgb, weights, guide, options);
}

ks_status ks_small_pt_render_guided_device(ks_scene *scene, const ks_camera_desc *camera,
                                           const ks_small_pt_params *params, ks_guide *guide,
                                           const ks_guide_render_options *options, double *accum_rgb_device,
                                           double *weights_device)
{
    if (!scene || !camera || !params || !guide || !options || !accum_rgb_device || !weights_device)
        return fail(scene ? scene->ctx : nullptr, KS_ERR_INVALID_ARGUMENT, "ks_small_pt_render_guided_device: null");
    KS_CUDA_TRY(scene->ctx, enter_device(scene->ctx));
    return render_impl(scene, camera, params, nullptr, nullptr, accum_rgb_device, weights_device, nullptr, nullptr,
                       guide, options);
}

ks_status ks_small_pt_render_device_progress(ks_scene *scene, const ks_camera_desc *camera,
                                             const ks_small_pt_params *params, ks_guide *guide,
                                             const ks_guide_render_options *options, ks_device_progress_fn progress,
                                             void *user, double *accum_rgb_device, double *weights_device)
{
    if (!scene || !camera || !params || !progress || !accum_rgb_device || !weights_device || (guide && !options))
        return fail(scene ? scene->ctx : nullptr, KS_ERR_INVALID_ARGUMENT,
                    "ks_small_pt_render_device_progress: null argument");
    KS_CUDA_TRY(scene->ctx, enter_device(scene->ctx));
    return render_impl(scene, camera, params, nullptr, nullptr, accum_rgb_device, weights_device, nullptr, nullptr,
                       guide, guide ? options : nullptr, progress, user);
}

ks_status ks_image_rel_mse_device(ks_context *ctx, const double *accum_rgb_device, const double *weights_device,
                                  const double *reference_rgb_device, uint32_t n_pixels, double eps,
                                  const float backdrop[3], double *rel_mse)
{
    if (!ctx || !accum_rgb_device || !weights_device || !reference_rgb_device || !rel_mse)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_image_rel_mse_device: null argument");
    KS_CUDA_TRY(ctx, enter_device(ctx));
    *rel_mse = 0.0;
    if (n_pixels == 0)
        return KS_OK;
    DevBuf<double> sum;
    KS_CUDA_TRY(ctx, sum.alloc(1));
    KS_CUDA_TRY(ctx, cudaMemsetAsync(sum.ptr, 0, sizeof(double), ctx->stream));
    const double b0 = backdrop ? backdrop[0] : 0.0, b1 = backdrop ? backdrop[1] : 0.0,
                 b2 = backdrop ? backdrop[2] : 0.0;
    unsigned grid = (unsigned)std::min<uint32_t>((n_pixels + 255) / 256, (uint32_t)ctx->sm_count * 8);
    k_rel_mse<<<grid, 256, 0, ctx->stream>>>(accum_rgb_device, weights_device, reference_rgb_device, n_pixels, eps,
                                             b0, b1, b2, sum.ptr);
    KS_CUDA_TRY(ctx, cudaGetLastError());
    double total = 0.0;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(&total, sum.ptr, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    *rel_mse = total / (3.0 * (double)n_pixels);
    return KS_OK;
}

ks_status ks_render_stats_last(const ks_scene *scene, ks_render_stats *out)
{
    if (!scene || !out)
        return KS_ERR_INVALID_ARGUMENT;
    *out = scene->last_stats;
    return KS_OK;
}

ks_status ks_batch_render_device(ks_context *ctx, const ks_batch_job *jobs, uint32_t n_jobs,
                                 const ks_batch_options *options, ks_batch_stats *stats)
{
    if (!ctx)
        return KS_ERR_INVALID_ARGUMENT;
    KS_CUDA_TRY(ctx, enter_device(ctx));
    ks_batch_options o{0, 0, 1};
    if (options)
        o = *options;
    return batch_render(ctx, jobs, n_jobs, o, stats);
}

ks_status ks_batch_autotune(ks_context *ctx, const ks_batch_job *jobs, uint32_t n_jobs, ks_batch_options *best,
                            float *best_ms)
{
    if (!ctx || !jobs || !best || n_jobs == 0)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_batch_autotune: null argument");
    KS_CUDA_TRY(ctx, enter_device(ctx));
    // sample: up to 8 evenly spaced jobs at no more than 4 spp, into scratch images
    const uint32_t m = std::min<uint32_t>(n_jobs, 8);
    std::vector<ks_batch_job> sample(m);
    std::vector<DevBuf<double>> scratch(2 * m);
    for (uint32_t k = 0; k < m; ++k) {
        sample[k] = jobs[(uint64_t)k * n_jobs / m];
        sample[k].params.spp = std::min(sample[k].params.spp, 4);
        size_t px = (size_t)std::max(0, sample[k].params.render_width) * std::max(0, sample[k].params.render_height);
        KS_CUDA_TRY(ctx, scratch[2 * k].alloc(3 * px + 1));
        KS_CUDA_TRY(ctx, scratch[2 * k + 1].alloc(2 * px + 1));
        sample[k].accum_rgb_device = scratch[2 * k].ptr;
        sample[k].weights_device = scratch[2 * k + 1].ptr;
    }
    const uint32_t caps[] = {1u << 21, 1u << 22, 1u << 23, 1u << 24, 1u << 25};
    const uint32_t grids[] = {4, 8, 16, 32};
    ks_batch_options bo = *best;
    float bms = 0.0f;
    bool have = false;
    // one untimed run first (first-launch costs)
    ks_batch_options warm{1u << 21, 16, best->use_graph};
    ks_status s = batch_render(ctx, sample.data(), m, warm, nullptr);
    if (s != KS_OK)
        return s;
    for (uint32_t c : caps)
        for (uint32_t g : grids) {
            ks_batch_options o{c, g, best->use_graph};
            ks_batch_stats st{};
            s = batch_render(ctx, sample.data(), m, o, &st);
            if (s != KS_OK)
                return s;
            if (!have || st.ms_total < bms) {
                have = true;
                bms = st.ms_total;
                bo = o;
            }
        }
    *best = bo;
    if (best_ms)
        *best_ms = bms;
    return KS_OK;
}

} // extern "C"
