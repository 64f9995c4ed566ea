// Types and device helpers shared by the wavefront kernels of ks_integrator.cu (ray generation,
// traversal, batching, host loop) and ks_shade.cu (sampling and shading, compiled with fast
// division and square root), plus the host launchers of the shading kernels.
#pragma once
#include "ks_guide_view.cuh"
#include "ks_lights.cuh"

namespace ksb
{
namespace wave
{

struct RenderParams
{
    int W, H, cx, cy, cw, ch;
    int spp, seed, log2_spp, n_digits;
    int bounces, include_background;
    float clamp_direct, clamp_indirect;
    float filter_r;
    const float *filter_cdf; // Gaussian / Blackman-Harris: filter_n conditional CDFs (filter_n + 1
                             // each), then the marginal CDF; null for the box filter
    uint32_t filter_n;
    int ortho;          // orthographic camera: origin on the film plane, direction cam_dir
    float cam_dir[3];   // -z of camera_to_world, normalised (Camera::direction, camera.h:24-27)
    float cam_pos[3];
    float p2w[16];
};

// Path state, structure of arrays, one float4 per field (16-byte vector loads/stores).
struct PathBuf
{
    float4 *o_pdf;    // ray origin, pdf_wi_bsdf of the previous bounce
    float4 *d_info;   // ray direction, (sobol dimension << 16 | bounce)
    float4 *beta_pix; // throughput, pixel index
    float4 *L_smp;    // radiance so far, sample index
    uint32_t *rec;    // guided renders: training record of the path (kNoRecord: none); else null
};

struct ShadowBuf
{
    float4 *o_tmax;   // origin, tmax
    float4 *d_target; // direction, target (next-queue slot, or kTermBit | pixel)
    float4 *contrib;  // beta * clamped Ld
    float4 *L_term;   // radiance of a path that ended this bounce
};

constexpr uint32_t kTermBit = 0x80000000u;

// ---- batched rendering: many (scene, camera, params) jobs in one wavefront --------------------
// A path's job id rides in bits 21..30 of its pixel word (per-job frames of at most 2^21 pixels,
// up to 1024 jobs); the scene view, render parameters and accumulators of a job are read from
// device arrays.  The iteration's counts live on the device (BatchState), so the loop needs no
// host round trip and runs as a CUDA graph with a device-side while condition.
constexpr uint32_t kJobShift = 21;
constexpr uint32_t kPixMask = (1u << kJobShift) - 1u;
constexpr uint32_t kMaxJobs = 1024;

struct BatchState
{
    unsigned long long total, issued, first_path; // paths of all jobs, paths issued, first of this refill
    unsigned long long ext_rays, shadow_rays;     // work counters
    uint32_t cur_count, n_new, count, base_slot;  // paths alive, refilled, traced this iteration
    uint32_t iterations, max_iterations, error;
};

struct BatchView
{
    const SceneView *views;       // per job
    const RenderParams *params;   // per job
    double *const *accum;         // per job: W * H * 3
    double *const *weights;       // per job: W * H * 2
    const unsigned long long *path_begin; // n_jobs + 1: first global path index of each job
    uint32_t n_jobs;
    BatchState *state;
};

template <bool kBatch, class T>
KS_D const T &job_of(const T &single, const T *table, uint32_t job)
{
    if constexpr (kBatch)
        return table[job];
    else
        return single;
}

KS_D uint32_t bits(float f) { return __float_as_uint(f); }
KS_D float fbits(uint32_t u) { return __uint_as_float(u); }

// One atomic per warp; every lane of the warp must call this.
KS_D uint32_t warp_append(uint32_t *counter, bool pred)
{
    uint32_t mask = __ballot_sync(0xffffffffu, pred);
    if (mask == 0)
        return 0;
    uint32_t lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if ((int)lane == leader)
        base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}

// Appends to two queues with one atomic per CTA and queue instead of one per warp (the queue
// counters are single addresses that every CTA hits, and same-address atomics serialise in L2).
// Slots follow the CTA's threads in order.  Every thread of the CTA must call it (it synchronises
// the CTA); blockDim.x is a multiple of 32.
KS_D void block_append2(uint32_t *c0, bool p0, uint32_t *c1, bool p1, uint32_t &j0, uint32_t &j1)
{
    __shared__ uint32_t s_off[2][32];
    __shared__ uint32_t s_base[2];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
    const uint32_t m0 = __ballot_sync(0xffffffffu, p0), m1 = __ballot_sync(0xffffffffu, p1);
    if (lane == 0) {
        s_off[0][warp] = __popc(m0);
        s_off[1][warp] = __popc(m1);
    }
    __syncthreads();
    if (warp == 0) {
        const uint32_t a = lane < n_warps ? s_off[0][lane] : 0u, b = lane < n_warps ? s_off[1][lane] : 0u;
        uint32_t sa = a, sb = b; // inclusive prefix sums over the warps
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t ta = __shfl_up_sync(0xffffffffu, sa, o), tb = __shfl_up_sync(0xffffffffu, sb, o);
            if ((int)lane >= o) {
                sa += ta;
                sb += tb;
            }
        }
        const uint32_t na = __shfl_sync(0xffffffffu, sa, 31), nb = __shfl_sync(0xffffffffu, sb, 31);
        if (lane == 0) {
            s_base[0] = na ? atomicAdd(c0, na) : 0u;
            s_base[1] = nb ? atomicAdd(c1, nb) : 0u;
        }
        if (lane < n_warps) {
            s_off[0][lane] = sa - a;
            s_off[1][lane] = sb - b;
        }
    }
    __syncthreads();
    const uint32_t below = (1u << lane) - 1u;
    j0 = s_base[0] + s_off[0][warp] + __popc(m0 & below);
    j1 = s_base[1] + s_off[1][warp] + __popc(m1 & below);
    __syncthreads(); // the next call reuses the shared arrays
}

KS_D void accumulate(double *accum, double *weights, uint32_t pix, f3 L)
{
    atomicAdd(&weights[2 * (size_t)pix], 1.0);
    atomicAdd(&accum[3 * (size_t)pix + 0], (double)L.x);
    atomicAdd(&accum[3 * (size_t)pix + 1], (double)L.y);
    atomicAdd(&accum[3 * (size_t)pix + 2], (double)L.z);
}

// ---- hit record (geometry.cpp:68-163 + transform_it with the identity instance) ----------------
struct ShadeFrame
{
    f3 p;
    f3 t, b, n;    // geometric frame (after re-orthonormalisation)
    f3 st, sb, sn; // shading frame (flat shading: same as the geometric one)
};

KS_D void reortho(f3 &t, f3 &b, f3 &n)
{
    // Transform::frame (maths.h:989-996) with identity: t' = normalize(t),
    // b' = normalize(b - dot(b, t') t'), n' = normalize(cross(t', b'))
    f3 tt = normalize(t);
    f3 bb = normalize(b - dot(b, tt) * tt);
    n = normalize(cross(tt, bb));
    t = tt;
    b = bb;
}

// Hit point from the barycentrics of vertices 1 and 2 (geometry.cpp:68-163).
KS_D f3 hit_point(f3 p0, f3 p1, f3 p2, float u, float v)
{
    float w0 = 1.0f - u - v;
    return w0 * p0 + u * p1 + v * p2;
}

// dP/du from the triangle's texture coordinates (geometry.cpp:94-116); the positional dP/du
// (p1 - p0) when the uv parameterisation is degenerate.
KS_D f3 uv_dpdu(f3 p0, f3 p1, f3 p2, float2 t0, float2 t1, float2 t2, f3 dpdu)
{
    const float du02 = t0.x - t2.x, dv02 = t0.y - t2.y;
    const float du12 = t1.x - t2.x, dv12 = t1.y - t2.y;
    const float det = du02 * dv12 - dv02 * du12;
    if (!(fabsf(det) < 1e-8f)) {
        const float inv = 1.0f / det;
        dpdu = (dv12 * (p0 - p2) - dv02 * (p1 - p2)) * inv;
    }
    return dpdu;
}

// compute_intersection (geometry.cpp:68-163) for a hit at barycentrics (u, v) of the triangle
// (p0, p1, p2), all in the space the frame is built in.  `dpdu` is p1 - p0 or the uv-derived
// tangent.  Smooth shading: `vn` is the interpolated vertex normal carried into that space (the
// zero vector for flat shading); a non-finite normal falls back to the geometric frame.
KS_D ShadeFrame make_frame(f3 p0, f3 p1, f3 p2, float u, float v, f3 ray_dir, bool twosided, f3 dpdu, bool smooth,
                           f3 vn)
{
    ShadeFrame f;
    f3 rd = normalize(ray_dir);
    f3 wo_object = -rd;
    f3 ng = normalize(cross(p1 - p0, p2 - p0));
    f.p = hit_point(p0, p1, p2, u, v);
    f3 b = normalize(cross(ng, dpdu));
    f3 t = normalize(cross(b, ng));
    if (twosided && dot(wo_object, ng) < 0.0f) {
        ng = -ng;
        dpdu = -dpdu;
        t = -t;
    }
    f3 ft = t, fb = b, fn = ng;
    reortho(ft, fb, fn);
    f.t = ft;
    f.b = fb;
    f.n = fn;
    if (smooth) {
        vn = normalize(vn);
        if (isfinite(vn.x) && isfinite(vn.y) && isfinite(vn.z)) {
            // the vertex normal on the side of the face normal, the frame re-orthogonalised
            // around it (geometry.cpp:142-155)
            if (dot(vn, ng) < 0.0f)
                vn = -vn;
            f3 vb = normalize(cross(vn, dpdu));
            f3 vt = normalize(cross(vb, vn));
            reortho(vt, vb, vn);
            f.st = vt;
            f.sb = vb;
            f.sn = vn;
            return f;
        }
    }
    // flat shading: sh_frame = frame (geometry.cpp:139-141), re-orthonormalised identically
    f.st = ft;
    f.sb = fb;
    f.sn = fn;
    return f;
}

// The per-vertex attributes of a hit: dP/du (from texcoords) and the interpolated vertex normal.
// Instanced hits pass the world-space vertices and the instance's object-to-world rows `m` (12
// floats); the vertex normal goes to world space through the cofactor matrix of m, which is what
// the reference's Transform::frame makes of a frame built around it in object space
// (maths.h:989-996).
struct HitAttribs
{
    f3 dpdu, vn;
};
KS_D HitAttribs hit_attribs(const SceneView &sv, uint32_t tri, int flags, f3 p0, f3 p1, f3 p2,
                                               float u, float v, const float *m)
{
    HitAttribs a{p1 - p0, mk(0.0f, 0.0f, 0.0f)};
    const uint32_t i0 = __ldg(&sv.indices[3 * (size_t)tri]), i1 = __ldg(&sv.indices[3 * (size_t)tri + 1]),
                   i2 = __ldg(&sv.indices[3 * (size_t)tri + 2]);
    if (flags & kMeshTexcoords) {
        const float2 *tc = reinterpret_cast<const float2 *>(sv.texcoords);
        a.dpdu = uv_dpdu(p0, p1, p2, __ldg(&tc[i0]), __ldg(&tc[i1]), __ldg(&tc[i2]), a.dpdu);
    }
    if (flags & kMeshSmooth) {
        auto ld = [&](uint32_t k) {
            return mk(__ldg(&sv.normals[3 * (size_t)k]), __ldg(&sv.normals[3 * (size_t)k + 1]),
                      __ldg(&sv.normals[3 * (size_t)k + 2]));
        };
        // rtcInterpolate0 of the vertex-normal buffer: (1 - u - v) n0 + u n1 + v n2
        a.vn = hit_point(ld(i0), ld(i1), ld(i2), u, v);
        if (m) {
            const f3 c0 = mk(m[0], m[4], m[8]), c1 = mk(m[1], m[5], m[9]), c2 = mk(m[2], m[6], m[10]);
            a.vn = a.vn.x * cross(c1, c2) + a.vn.y * cross(c2, c0) + a.vn.z * cross(c0, c1);
        }
    }
    return a;
}

// The hit's frames from the scene's per-mesh flags and per-vertex attributes.  kAttribs = false
// (no mesh of the scene has vertex normals or texcoords) compiles to the flat-shading frame only:
// a separate shading frame keeps three more values live through the BSDF code.
template <bool kAttribs>
KS_D ShadeFrame hit_frame(const SceneView &sv, uint32_t tri, int flags, f3 p0, f3 p1, f3 p2, float u, float v,
                          f3 ray_dir, const float *m)
{
    HitAttribs a{p1 - p0, mk(0.0f, 0.0f, 0.0f)};
    if (!kAttribs)
        flags &= kMeshTwosided;
    else if (flags & (kMeshSmooth | kMeshTexcoords))
        a = hit_attribs(sv, tri, flags, p0, p1, p2, u, v, m);
    return make_frame(p0, p1, p2, u, v, ray_dir, (flags & kMeshTwosided) != 0, a.dpdu, (flags & kMeshSmooth) != 0,
                      a.vn);
}

// The hit's texture coordinates: the mesh's interpolated texcoords (rtcInterpolate0 of the
// texcoord buffer, geometry.cpp:92-99; MeshGeometry::compute_hit_texcoord), else the barycentrics
// (u, v) of vertices 1 and 2.
// Texture coordinate of a hit: the mesh's texcoords interpolated, else the hit's barycentrics
// (compute_intersection, geometry.cpp:78-101) or, for the opacity test and light samples, zero
// (compute_hit_texcoord / interpolate_texcoord, geometry.cpp:165-191).
KS_D void hit_uv(const SceneView &sv, uint32_t tri, int flags, float u, float v, float &tu, float &tv,
                 bool bary_fallback = true)
{
    tu = bary_fallback ? u : 0.0f;
    tv = bary_fallback ? v : 0.0f;
    if (flags & kMeshTexcoords) {
        const float2 *tc = reinterpret_cast<const float2 *>(sv.texcoords);
        const uint32_t i0 = __ldg(&sv.indices[3 * (size_t)tri]), i1 = __ldg(&sv.indices[3 * (size_t)tri + 1]),
                       i2 = __ldg(&sv.indices[3 * (size_t)tri + 2]);
        const float2 t0 = __ldg(&tc[i0]), t1 = __ldg(&tc[i1]), t2 = __ldg(&tc[i2]);
        const float w = 1.0f - u - v;
        tu = w * t0.x + u * t1.x + v * t2.x;
        tv = w * t0.y + u * t1.y + v * t2.y;
    }
}

// hash_float(ro, rd) (hash.h:140-258): murmur_hash_64A of the 24 bytes of the ray's origin and
// direction (seed 0), its low 32 bits times 2^-32
KS_D float hash_float_ray(f3 o, f3 d)
{
    const uint64_t k[3] = {(uint64_t)__float_as_uint(o.x) | ((uint64_t)__float_as_uint(o.y) << 32),
                           (uint64_t)__float_as_uint(o.z) | ((uint64_t)__float_as_uint(d.x) << 32),
                           (uint64_t)__float_as_uint(d.y) | ((uint64_t)__float_as_uint(d.z) << 32)};
    const uint64_t m = 0xc6a4a7935bd1e995ull;
    uint64_t h = 24ull * m;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        uint64_t x = k[i] * m;
        x ^= x >> 47;
        x *= m;
        h ^= x;
        h *= m;
    }
    h ^= h >> 47;
    h *= m;
    h ^= h >> 47;
    return (float)(uint32_t)h * 0x1p-32f;
}

// The opacity maps' candidate-hit filter (Embree filter_opacity_map, scene.cpp:175-208, with
// OpacityMap::stochastic_test, opacity_map.cpp:20-30): a hit on a triangle whose material has an
// opacity map counts with probability saturate(map(uv)), decided by the ray's own hash.
struct SceneAlpha
{
    const SceneView *sv;
    KS_D bool operator()(uint32_t tri, float u, float v, const RayQuery &ray) const
    {
        const uint32_t mesh = __ldg(&sv->tri_mesh[tri]);
        const MaterialGPU &mat = sv->materials[__ldg(&sv->mesh_material[mesh])];
        if (!(mat.tex_flags & kMatOpacityMap))
            return true;
        int k = 0;
        while (sv->bindings[mat.bind_begin + k].field != KS_FIELD_OPACITY_MAP)
            ++k;
        float tu, tv;
        hit_uv(*sv, tri, __ldg(&sv->mesh_flags[mesh]), u, v, tu, tv, false);
        const float opacity = saturate(field_eval(sv->tex_texels, sv->tex_info, sv->bindings[mat.bind_begin + k], tu,
                                                  tv).x);
        if (opacity <= 0.0f)
            return false;
        if (opacity >= 1.0f)
            return true;
        return hash_float_ray(ray.o, ray.d) < opacity;
    }
};

KS_D f3 sh_to_local(const ShadeFrame &f, f3 w)
{
    bool hw = dot(f.n, w) >= 0.0f;
    f3 l = mk(dot(f.st, w), dot(f.sb, w), dot(f.sn, w));
    bool hl = l.z >= 0.0f;
    if (hw != hl)
        l.z *= -1.0f;
    return l;
}

KS_D f3 sh_to_world(const ShadeFrame &f, f3 l)
{
    bool hl = l.z >= 0.0f;
    f3 w = f.st * l.x + f.sb * l.y + f.sn * l.z;
    bool hw = dot(f.n, w) >= 0.0f;
    if (hl != hw)
        w = w - 2.0f * dot(f.n, w) * f.n;
    return w;
}

// offset_ray (ray.h:66-81)
KS_D f3 offset_ray(f3 p, f3 n)
{
    const float origin = 1.0f / 32.0f, float_scale = 1.0f / 65536.0f, int_scale = 256.0f;
    int ox = (int)(int_scale * n.x), oy = (int)(int_scale * n.y), oz = (int)(int_scale * n.z);
    f3 pi = mk(__int_as_float(__float_as_int(p.x) + ((p.x < 0) ? -ox : ox)),
               __int_as_float(__float_as_int(p.y) + ((p.y < 0) ? -oy : oy)),
               __int_as_float(__float_as_int(p.z) + ((p.z < 0) ? -oz : oz)));
    return mk(fabsf(p.x) < origin ? p.x + float_scale * n.x : pi.x,
              fabsf(p.y) < origin ? p.y + float_scale * n.y : pi.y,
              fabsf(p.z) < origin ? p.z + float_scale * n.z : pi.z);
}

// spawn_ray<OffsetType::NextBounce> origin (ray.h:89-96)
KS_D f3 spawn_origin(f3 p, f3 dir, f3 n) { return offset_ray(p, dot(dir, n) > 0.0f ? n : -n); }

KS_D float power_heur(float pf, float pg)
{
    float f2 = pf * pf, g2 = pg * pg;
    return f2 / (f2 + g2);
}

KS_D f3 clamp_contrib(f3 v, int bounce_for_direct, const RenderParams &rp, bool is_nee)
{
    // trace(): NEE uses bounce==0 -> clamp_direct, bounce>=1 -> clamp_indirect (small_pt.cpp:153-157);
    // unidirectional hits use bounce==1 -> direct, bounce>=2 -> indirect (:97-103, :128-133).
    int b = bounce_for_direct;
    if (is_nee) {
        if (b == 0 && rp.clamp_direct > 0.0f)
            return cwise_min(v, rp.clamp_direct);
        if (b >= 1 && rp.clamp_indirect > 0.0f)
            return cwise_min(v, rp.clamp_indirect);
        return v;
    }
    if (b == 1 && rp.clamp_direct > 0.0f)
        return cwise_min(v, rp.clamp_direct);
    if (b >= 2 && rp.clamp_indirect > 0.0f)
        return cwise_min(v, rp.clamp_indirect);
    return v;
}

// The tree a kernel traverses: the SBVH nodes or their 4-wide view.
template <class Node>
KS_D const Node *tree_of(const SceneView &sv);
template <>
KS_D const TravNode *tree_of<TravNode>(const SceneView &sv)
{
    return sv.nodes;
}
template <>
KS_D const WideNode *tree_of<WideNode>(const SceneView &sv)
{
    return sv.wide;
}

// ---- shading launchers (ks_shade.cu) ----------------------------------------------------------
// k_sample: Sobol values and the NEE light sample of every path in the hit queue.
// Subsurface entries of a bounce's hit queue (k_subsurface, ks_shade.cu), before its light samples.
void launch_subsurface(unsigned grid, cudaStream_t st, const SceneView &sv, const RenderParams &rp, PathBuf cur,
                       float4 *hits, const uint32_t *queue, const uint32_t *queue_count, int *overflow);
void launch_sample(bool batch, unsigned grid, cudaStream_t st, const SceneView &sv, const RenderParams &rp,
                   PathBuf cur, const float4 *hits, const uint32_t *hit_inst, const uint32_t *queue,
                   const uint32_t *queue_count, float4 *samples, const BatchView &bv);
// k_shade: hit (miss = false) or miss shading of the paths in a queue; guided and batched
// renders are not combined.  variant: the shading kernel's feature set (kShadePlain,
// kShadeAttribs, kShadeGeneral) that the scene (of every job) needs, SceneView::shade_variant.
void launch_shade(bool miss, bool guided, bool batch, int variant, unsigned grid, cudaStream_t st, const SceneView &sv,
                  const RenderParams &rp, PathBuf cur, PathBuf nxt, const float4 *hits, const uint32_t *hit_inst,
                  const float4 *samples, const uint32_t *queue, const uint32_t *queue_count, uint32_t *next_count,
                  ShadowBuf sb, uint32_t *shadow_count, double *accum, double *weights, const GuideView &gv,
                  const BatchView &bv);

} // namespace wave
} // namespace ksb
