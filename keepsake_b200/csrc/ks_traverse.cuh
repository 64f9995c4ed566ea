// SBVH traversal and the watertight ray/triangle test on the device.
//
// Hit semantics follow the reference exactly:
//   * RayTriHelper + isect_ray_tri: shear/scale watertight test of Woop et al. with the FP64
//     edge fallback (cuda/ray_tri.cuh:8-97),
//   * RayBoundHelper + isect_ray_aabb: slab test with the 0*inf guard (cuda/aabb.cuh:155-252),
//   * SBVH::intersect / intersectBool: near child first by the sign of the ray direction on the
//     node's split axis, leaf primitives in order, a hit replaces the current one only if
//     tHit < tmax (cuda/sbvh.cu:512-603).
// The node layout differs (both children's boxes are stored in the parent, so a child box is
// tested when its parent is expanded and re-checked against the current tmax when popped).
// Because the slab interval of a box does not depend on tmax, that re-check makes exactly the
// decision the reference makes when it visits the child, so the sequence of triangle tests -
// and therefore the hit, including ties - is the reference's.
#pragma once
#include "ks_math.cuh"
#include "ks_scene.h"

namespace ksb
{

struct RayQuery
{
    f3 o, d;
    float tmin, tmax;
};

struct TriHelper
{
    int kx, ky, kz;
    float shx, shy, shz;
};

struct BoxHelper
{
    f3 inv;
    int neg[3];
};

KS_D TriHelper make_tri_helper(f3 dir)
{
    TriHelper h;
    float ax = fabsf(dir.x), ay = fabsf(dir.y), az = fabsf(dir.z);
    if (ax >= ay && ax >= az)
        h.kz = 0;
    else if (ay >= ax && ay >= az)
        h.kz = 1;
    else
        h.kz = 2;
    h.kx = (h.kz + 1) % 3;
    h.ky = (h.kx + 1) % 3;
    if (get(dir, h.kz) < 0.0f) {
        int t = h.kx;
        h.kx = h.ky;
        h.ky = t;
    }
    float dz = get(dir, h.kz);
    h.shx = get(dir, h.kx) / dz;
    h.shy = get(dir, h.ky) / dz;
    h.shz = 1.0f / dz;
    return h;
}

KS_D BoxHelper make_box_helper(f3 dir)
{
    BoxHelper b;
    b.inv = mk(1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z);
    b.neg[0] = dir.x < 0.0f || (dir.x == 0.0f && signbit(dir.x));
    b.neg[1] = dir.y < 0.0f || (dir.y == 0.0f && signbit(dir.y));
    b.neg[2] = dir.z < 0.0f || (dir.z == 0.0f && signbit(dir.z));
    return b;
}

// ksc::difference_of_products (cuda/math.cuh:189-195)
KS_D float diff_of_products(float a, float b, float c, float d)
{
    float cd = c * d;
    float dop = fmaf(a, b, -cd);
    float err = fmaf(-c, d, cd);
    return dop + err;
}

// isect_ray_tri (cuda/ray_tri.cuh:46-97).  Returns true on a hit inside (tmin, tmax).
KS_D bool isect_tri(const RayQuery &ray, const TriHelper &h, f3 v0, f3 v1, f3 v2, float &t_out, float &b0, float &b1,
                    float &b2)
{
    f3 A0 = v0 - ray.o, B0 = v1 - ray.o, C0 = v2 - ray.o;
    f3 A = mk(get(A0, h.kx), get(A0, h.ky), get(A0, h.kz));
    f3 B = mk(get(B0, h.kx), get(B0, h.ky), get(B0, h.kz));
    f3 C = mk(get(C0, h.kx), get(C0, h.ky), get(C0, h.kz));
    f3 sx = mk(A.x - h.shx * A.z, B.x - h.shx * B.z, C.x - h.shx * C.z);
    f3 sy = mk(A.y - h.shy * A.z, B.y - h.shy * B.z, C.y - h.shy * C.z);
    // bc = cross(sy, sx) with difference_of_products
    float bx = diff_of_products(sy.y, sx.z, sy.z, sx.y);
    float by = diff_of_products(sy.z, sx.x, sy.x, sx.z);
    float bz = diff_of_products(sy.x, sx.y, sy.y, sx.x);
    if (bx == 0.0f || by == 0.0f || bz == 0.0f) {
        bx = (float)((double)sx.z * (double)sy.y - (double)sy.z * (double)sx.y);
        by = (float)((double)sx.x * (double)sy.z - (double)sy.x * (double)sx.z);
        bz = (float)((double)sx.y * (double)sy.x - (double)sy.y * (double)sx.x);
    }
    if ((bx < 0.0f || by < 0.0f || bz < 0.0f) && (bx > 0.0f || by > 0.0f || bz > 0.0f))
        return false;
    float det = bx + by + bz;
    if (det == 0.0f)
        return false;
    float szx = h.shz * A.z, szy = h.shz * B.z, szz = h.shz * C.z;
    float T = bx * szx + by * szy + bz * szz;
    if (det < 0.0f && (T >= ray.tmin * det || T <= ray.tmax * det))
        return false;
    if (det > 0.0f && (T <= ray.tmin * det || T >= ray.tmax * det))
        return false;
    float inv_det = 1.0f / det;
    b0 = bx * inv_det;
    b1 = by * inv_det;
    b2 = bz * inv_det;
    t_out = T * inv_det;
    return true;
}

// Slab part of isect_ray_aabb (cuda/aabb.cuh:171-236): returns false if the slabs do not
// overlap, else the clipped-free entry/exit times.
KS_D bool slab(const RayQuery &ray, const BoxHelper &h, const float bmin[3], const float bmax[3], float &t0,
               float &t1)
{
    // every value is computed and the early outs become one condition: the same results without
    // data-dependent branches
    float tmin = (h.neg[0] ? bmax[0] : bmin[0]) - ray.o.x;
    tmin = tmin != 0.0f ? tmin * h.inv.x : tmin;
    float tmax = (h.neg[0] ? bmin[0] : bmax[0]) - ray.o.x;
    tmax = tmax != 0.0f ? tmax * h.inv.x : tmax;
    float tymin = (h.neg[1] ? bmax[1] : bmin[1]) - ray.o.y;
    tymin = tymin != 0.0f ? tymin * h.inv.y : tymin;
    float tymax = (h.neg[1] ? bmin[1] : bmax[1]) - ray.o.y;
    tymax = tymax != 0.0f ? tymax * h.inv.y : tymax;
    const bool miss_y = tmin > tymax || tymin > tmax;
    tmin = tymin > tmin ? tymin : tmin;
    tmax = tymax < tmax ? tymax : tmax;
    float tzmin = (h.neg[2] ? bmax[2] : bmin[2]) - ray.o.z;
    tzmin = tzmin != 0.0f ? tzmin * h.inv.z : tzmin;
    float tzmax = (h.neg[2] ? bmin[2] : bmax[2]) - ray.o.z;
    tzmax = tzmax != 0.0f ? tzmax * h.inv.z : tzmax;
    const bool miss_z = tmin > tzmax || tzmin > tmax;
    t0 = tzmin > tmin ? tzmin : tmin;
    t1 = tzmax < tmax ? tzmax : tmax;
    return !miss_y && !miss_z;
}

enum class Culling : int
{
    Back = 0,
    Front = 1,
    None = 2,
};

KS_D bool cull_tri(const RayQuery &ray, f3 v0, f3 v1, f3 v2, int culling)
{
    if (culling == (int)Culling::None)
        return false;
    // check = dot(dir, cross(v1 - v0, v2 - v1)) with difference_of_products (cuda/sbvh.cu:478-484)
    f3 e0 = v1 - v0, e1 = v2 - v1;
    f3 c = mk(diff_of_products(e0.y, e1.z, e0.z, e1.y), diff_of_products(e0.z, e1.x, e0.x, e1.z),
              diff_of_products(e0.x, e1.y, e0.y, e1.x));
    float check = ray.d.x * c.x + ray.d.y * c.y + ray.d.z * c.z;
    if (check >= 0.0f && culling == (int)Culling::Back)
        return true;
    if (check <= 0.0f && culling == (int)Culling::Front)
        return true;
    return false;
}

struct Hit
{
    uint32_t tri;  // global triangle index, ~0u on miss
    uint32_t slot; // primitive slot of the hit (index into the leaf-ordered triangle array)
    float t, b0, b1, b2;
};

constexpr int kStackDepth = 64;

// Closest hit (any_hit = false) or occlusion (any_hit = true) against the scene's SBVH.
// Work counters of one query: interior nodes fetched (64 B each) and triangles tested (48 B each).
struct TravCount
{
    uint32_t nodes = 0, tris = 0;
};

// Candidate-hit filter of the traversal (the role of Embree's intersection filter that runs the
// opacity maps' stochastic test, scene.cpp:175-208): a hit on triangle tri at barycentrics (u, v)
// counts only when the filter accepts it.  NoAlpha accepts every hit and compiles away.
struct NoAlpha
{
    KS_D bool operator()(uint32_t, float, float, const RayQuery &) const { return true; }
};

template <bool kAnyHit, class Alpha = NoAlpha>
KS_D bool traverse(const TravNode *__restrict__ nodes, const float4 *__restrict__ tris, uint32_t root_ref,
                   uint32_t root_count, const float root_bmin[3], const float root_bmax[3], RayQuery ray,
                   int culling, Hit &hit, int &overflow, TravCount *count = nullptr, const Alpha &alpha = Alpha{})
{
    hit.tri = ~0u;
    const TriHelper th = make_tri_helper(ray.d);
    const BoxHelper bh = make_box_helper(ray.d);
    uint4 stack[kStackDepth]; // (ref, count, entry t bits, -): one 16-byte access per push or pop
    int sp = 0;
    // the root's own box (cuda/sbvh.cu:520-527)
    float t0, t1;
    if (!slab(ray, bh, root_bmin, root_bmax, t0, t1) || !(t0 < ray.tmax && t1 > ray.tmin))
        return false;
    uint32_t ref = root_ref, cnt = root_count;
    while (true) {
        if (ref & kLeafBit) {
            uint32_t first = ref & ~kLeafBit;
            for (uint32_t k = 0; k < cnt; ++k) {
                if (count)
                    count->tris++;
                const float4 *p = tris + 3 * (size_t)(first + k);
                float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
                f3 v0 = mk(a.x, a.y, a.z), v1 = mk(b.x, b.y, b.z), v2 = mk(c.x, c.y, c.z);
                if (cull_tri(ray, v0, v1, v2, culling))
                    continue;
                float t, b0, b1, b2;
                if (isect_tri(ray, th, v0, v1, v2, t, b0, b1, b2)) {
                    if (kAnyHit) {
                        if (!alpha(__float_as_uint(a.w), b1, b2, ray))
                            continue;
                        hit.tri = __float_as_uint(a.w);
                        return true;
                    }
                    if (t < ray.tmax && alpha(__float_as_uint(a.w), b1, b2, ray)) {
                        ray.tmax = t;
                        hit.tri = __float_as_uint(a.w);
                        hit.slot = first + k;
                        hit.t = t;
                        hit.b0 = b0;
                        hit.b1 = b1;
                        hit.b2 = b2;
                    }
                }
            }
        } else {
            const TravNode *n = nodes + ref;
            if (count)
                count->nodes++;
            float4 A = __ldg(&n->a), B = __ldg(&n->b), C = __ldg(&n->c);
            uint4 D = __ldg(&n->d);
            float lmin[3] = {A.x, A.y, A.z}, lmax[3] = {A.w, B.x, B.y};
            float rmin[3] = {B.z, B.w, C.x}, rmax[3] = {C.y, C.z, C.w};
            float lt0, lt1, rt0, rt1;
            bool lok = slab(ray, bh, lmin, lmax, lt0, lt1) && lt1 > ray.tmin && lt0 < ray.tmax;
            bool rok = slab(ray, bh, rmin, rmax, rt0, rt1) && rt1 > ray.tmin && rt0 < ray.tmax;
            uint32_t axis = D.z >> 30;
            uint32_t lcnt = D.z & 0x3fffffffu, rcnt = D.w;
            bool right_first = bh.neg[axis] != 0;
            uint32_t near_ref = right_first ? D.y : D.x, far_ref = right_first ? D.x : D.y;
            uint32_t near_cnt = right_first ? rcnt : lcnt, far_cnt = right_first ? lcnt : rcnt;
            bool near_ok = right_first ? rok : lok, far_ok = right_first ? lok : rok;
            float far_t = right_first ? lt0 : rt0;
            if (near_ok) {
                if (far_ok) {
                    if (sp >= kStackDepth) {
                        overflow = 1;
                        return !kAnyHit && hit.tri != ~0u;
                    }
                    stack[sp++] = make_uint4(far_ref, far_cnt, __float_as_uint(far_t), 0u);
                }
                ref = near_ref;
                cnt = near_cnt;
                continue;
            }
            if (far_ok) {
                ref = far_ref;
                cnt = far_cnt;
                continue;
            }
        }
        // pop, re-checking the entry time against the current tmax
        bool found = false;
        while (sp > 0) {
            const uint4 e = stack[--sp];
            if (__uint_as_float(e.z) < ray.tmax) {
                ref = e.x;
                cnt = e.y;
                found = true;
                break;
            }
        }
        if (!found)
            break;
    }
    return hit.tri != ~0u;
}

// ---- resumable traversal (persistent warps with dynamic ray fetch) ---------------------------
// The same traversal as traverse(), cut into steps so that a warp can hand finished lanes a new
// ray and keep its lanes busy: trav_begin does the root test, every trav_step visits the current
// node (an interior node, or a leaf and its triangles) and then descends or pops, exactly as one
// pass of traverse()'s loop.  Each ray therefore makes the same sequence of box and triangle tests
// (same hits, same distances); only the interleaving of rays changes.  The stack lives in the
// caller's array.
struct TravState
{
    RayQuery ray;
    TriHelper th;
    BoxHelper bh;
    uint32_t ref, cnt;
    int sp;
    Hit hit;
};

// Traversal stack of the persistent kernels (blocks of kTravBlock threads): each thread's first
// KS_SMEM_STACK entries live in shared memory, laid out [entry][thread] so that a warp whose lanes
// sit at different depths still touches distinct banks; deeper entries spill to local memory.
// 8 entries (16 KB per CTA, 128 KB per SM at 8 CTAs) measured best on the bench frame: +3.7 %
// over a local-memory stack; 12 or 16 take L1 capacity from the node cache and lose.
constexpr int kTravBlock = 128;
#ifndef KS_SMEM_STACK
#define KS_SMEM_STACK 8
#endif
// Capacity: the binary traversal pushes at most one entry per level and stops at kStackDepth; the
// 4-wide one pushes up to three per wide level and stops at kWideStackDepth.
constexpr int kWideStackDepth = 96;
constexpr int kSmemStack = KS_SMEM_STACK < kStackDepth ? KS_SMEM_STACK : kStackDepth;
struct TravStack
{
    uint4 *sm; // this thread's column of the block's shared array: entry i at sm[i * kTravBlock]
    uint4 loc[kWideStackDepth - kSmemStack];
    KS_D void set(int i, uint4 e)
    {
        if (i < kSmemStack)
            sm[i * kTravBlock] = e;
        else
            loc[i - kSmemStack] = e;
    }
    KS_D uint4 get(int i) const { return i < kSmemStack ? sm[i * kTravBlock] : loc[i - kSmemStack]; }
};
// The shared part of a block's stacks; every persistent traversal kernel declares one and points
// each thread's TravStack at its column.
#define KS_TRAV_STACK(name)                                                                                       \
    __shared__ uint4 name##_smem[kSmemStack > 0 ? kSmemStack * kTravBlock : 1];                                  \
    TravStack name;                                                                                                \
    name.sm = name##_smem + threadIdx.x

// Returns false when the ray misses the root box (the traversal is then over, without a hit).
KS_D bool trav_begin(TravState &s, const RayQuery &ray, uint32_t root_ref, uint32_t root_count,
                     const float root_bmin[3], const float root_bmax[3])
{
    s.hit.tri = ~0u;
    s.ray = ray;
    s.th = make_tri_helper(ray.d);
    s.bh = make_box_helper(ray.d);
    s.sp = 0;
    s.ref = root_ref;
    s.cnt = root_count;
    float t0, t1;
    return slab(s.ray, s.bh, root_bmin, root_bmax, t0, t1) && t0 < s.ray.tmax && t1 > s.ray.tmin;
}

// Interior node test of trav_step: descends to the near child (pushing the far one when both are
// hit) and returns 1, returns 0 when neither child is hit, and -1 with the overflow flag set when
// the stack is full (the caller then ends the ray).
KS_D int trav_interior(const TravNode *__restrict__ nodes, TravState &s, TravStack &stack, int &overflow,
                        TravCount *count)
{
    const TravNode *n = nodes + s.ref;
    if (count)
        count->nodes++;
    float4 A = __ldg(&n->a), B = __ldg(&n->b), C = __ldg(&n->c);
    uint4 D = __ldg(&n->d);
    float lmin[3] = {A.x, A.y, A.z}, lmax[3] = {A.w, B.x, B.y};
    float rmin[3] = {B.z, B.w, C.x}, rmax[3] = {C.y, C.z, C.w};
    float lt0, lt1, rt0, rt1;
    bool lok = slab(s.ray, s.bh, lmin, lmax, lt0, lt1) && lt1 > s.ray.tmin && lt0 < s.ray.tmax;
    bool rok = slab(s.ray, s.bh, rmin, rmax, rt0, rt1) && rt1 > s.ray.tmin && rt0 < s.ray.tmax;
    uint32_t axis = D.z >> 30;
    uint32_t lcnt = D.z & 0x3fffffffu, rcnt = D.w;
    bool right_first = s.bh.neg[axis] != 0;
    uint32_t near_ref = right_first ? D.y : D.x, far_ref = right_first ? D.x : D.y;
    uint32_t near_cnt = right_first ? rcnt : lcnt, far_cnt = right_first ? lcnt : rcnt;
    bool near_ok = right_first ? rok : lok, far_ok = right_first ? lok : rok;
    float far_t = right_first ? lt0 : rt0;
    if (near_ok && far_ok) {
        if (s.sp >= kStackDepth) {
            overflow = 1;
            return -1;
        }
        stack.set(s.sp++, make_uint4(far_ref, far_cnt, __float_as_uint(far_t), 0u));
    }
    if (!near_ok && !far_ok)
        return 0;
    s.ref = near_ok ? near_ref : far_ref;
    s.cnt = near_ok ? near_cnt : far_cnt;
    return 1;
}

// Interior step of the 4-wide view (WideNode): the slots' boxes are tested with the same slab test,
// the ray descends into the nearest hit slot (smallest entry time, then lowest slot) and the other
// hit slots are pushed farthest first, each with its entry time (re-checked against tmax when
// popped, as in trav_interior); any-hit queries take them in slot order.  Returns 1 / 0 / -1 like
// trav_interior.  The set of leaves a closest-hit ray can reach is that of the binary tree (a
// slot's slab interval lies inside its parent's: same operations, monotone rounding), so the
// closest hit is the binary traversal's up to the order of exact ties.
template <bool kAnyHit>
KS_D int trav_wide(const WideNode *__restrict__ wide, TravState &s, TravStack &stack, int &overflow,
                   TravCount *count)
{
    const WideNode *n = wide + s.ref;
    if (count)
        count->nodes += 2; // 128 bytes: two 64-byte node units
    const float4 lx = __ldg(&n->lo[0]), ly = __ldg(&n->lo[1]), lz = __ldg(&n->lo[2]);
    const float4 hx = __ldg(&n->hi[0]), hy = __ldg(&n->hi[1]), hz = __ldg(&n->hi[2]);
    const uint4 ref = __ldg(&n->ref), cnt = __ldg(&n->cnt);
    const float blo[3][4] = {{lx.x, lx.y, lx.z, lx.w}, {ly.x, ly.y, ly.z, ly.w}, {lz.x, lz.y, lz.z, lz.w}};
    const float bhi[3][4] = {{hx.x, hx.y, hx.z, hx.w}, {hy.x, hy.y, hy.z, hy.w}, {hz.x, hz.y, hz.z, hz.w}};
    // counts are below 2^30 (the bound TravNode's packed counts have); masked to those bits, the
    // kernel measured 0.6 % faster on the bench frame (the compiler keeps it free of spills)
    constexpr uint32_t kCount = 0x3fffffffu;
    const uint32_t refs[4] = {ref.x, ref.y, ref.z, ref.w};
    const uint32_t cnts[4] = {cnt.x & kCount, cnt.y & kCount, cnt.z & kCount, cnt.w & kCount};
    float t0[4];
    bool ok[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float bmin[3] = {blo[0][k], blo[1][k], blo[2][k]}, bmax[3] = {bhi[0][k], bhi[1][k], bhi[2][k]};
        float a, b;
        ok[k] = slab(s.ray, s.bh, bmin, bmax, a, b) && b > s.ray.tmin && a < s.ray.tmax;
        t0[k] = a;
    }
    int n_hit = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        n_hit += ok[k] ? 1 : 0;
    if (n_hit == 0)
        return 0;
    if (s.sp + n_hit - 1 > kWideStackDepth) {
        overflow = 1;
        return -1;
    }
    if constexpr (kAnyHit) {
        // any-hit: the first slot hit next, the others pushed in slot order.  Nearest first (the
        // network below) took 2.5 % off the bench frame's shadow rays but made a pass of the
        // occluded glossy scene 17 % slower: shadow rays blocked by a distant occluder then search
        // the nearby geometry's subtrees first.
        const int f = ok[0] ? 0 : (ok[1] ? 1 : (ok[2] ? 2 : 3));
        s.ref = f == 0 ? refs[0] : (f == 1 ? refs[1] : (f == 2 ? refs[2] : refs[3]));
        s.cnt = f == 0 ? cnts[0] : (f == 1 ? cnts[1] : (f == 2 ? cnts[2] : cnts[3]));
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (ok[k] && k != f)
                stack.set(s.sp++, make_uint4(refs[k], cnts[k], __float_as_uint(t0[k]), 0u));
    } else {
        // the slots in visiting order (entry time, then slot index; the slots not hit last) by a
        // 4-input sorting network: the same instructions in every lane, where branches on the
        // number of slots hit split the warp (measured 6 % off the closest-hit kernel)
        float kt[4];
        uint32_t kr[4], kc[4], ks[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            kt[k] = ok[k] ? t0[k] : kInf;
            ks[k] = ok[k] ? (uint32_t)k : 4u + k;
            kr[k] = refs[k];
            kc[k] = cnts[k];
        }
        auto cex = [&](int i, int j) {
            const bool sw = kt[j] < kt[i] || (kt[j] == kt[i] && ks[j] < ks[i]);
            const float t = sw ? kt[j] : kt[i];
            kt[j] = sw ? kt[i] : kt[j];
            kt[i] = t;
            const uint32_t a = sw ? ks[j] : ks[i], b = sw ? kr[j] : kr[i], c = sw ? kc[j] : kc[i];
            ks[j] = sw ? ks[i] : ks[j];
            kr[j] = sw ? kr[i] : kr[j];
            kc[j] = sw ? kc[i] : kc[j];
            ks[i] = a;
            kr[i] = b;
            kc[i] = c;
        };
        cex(0, 1);
        cex(2, 3);
        cex(0, 2);
        cex(1, 3);
        cex(1, 2);
#pragma unroll
        for (int r = 3; r >= 1; --r)
            if (r < n_hit)
                stack.set(s.sp++, make_uint4(kr[r], kc[r], __float_as_uint(kt[r]), 0u));
        s.ref = kr[0];
        s.cnt = kc[0];
    }
    return 1;
}

// Interior step for either tree layout.
template <bool kAnyHit>
KS_D int trav_node(const TravNode *__restrict__ nodes, TravState &s, TravStack &stack, int &overflow,
                   TravCount *count)
{
    return trav_interior(nodes, s, stack, overflow, count);
}
template <bool kAnyHit>
KS_D int trav_node(const WideNode *__restrict__ nodes, TravState &s, TravStack &stack, int &overflow,
                   TravCount *count)
{
    return trav_wide<kAnyHit>(nodes, s, stack, overflow, count);
}

// Pops the next node whose entry time is below the current tmax; false when the stack is empty.
KS_D bool trav_pop(TravState &s, const TravStack &stack)
{
    while (s.sp > 0) {
        const uint4 e = stack.get(--s.sp);
        if (__uint_as_float(e.z) < s.ray.tmax) {
            s.ref = e.x;
            s.cnt = e.y;
            return true;
        }
    }
    return false;
}

// Leaf triangles of trav_step; true when an any-hit query found an occluder.
template <bool kAnyHit, class Alpha = NoAlpha>
KS_D bool trav_leaf(const float4 *__restrict__ tris, TravState &s, int culling, TravCount *count,
                    const Alpha &alpha = Alpha{})
{
    const uint32_t first = s.ref & ~kLeafBit;
    for (uint32_t k = 0; k < s.cnt; ++k) {
        if (count)
            count->tris++;
        const float4 *p = tris + 3 * (size_t)(first + k);
        float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
        f3 v0 = mk(a.x, a.y, a.z), v1 = mk(b.x, b.y, b.z), v2 = mk(c.x, c.y, c.z);
        if (cull_tri(s.ray, v0, v1, v2, culling))
            continue;
        float t, b0, b1, b2;
        if (isect_tri(s.ray, s.th, v0, v1, v2, t, b0, b1, b2)) {
            if (kAnyHit) {
                if (!alpha(__float_as_uint(a.w), b1, b2, s.ray))
                    continue;
                s.hit.tri = __float_as_uint(a.w);
                return true;
            }
            if (t < s.ray.tmax && alpha(__float_as_uint(a.w), b1, b2, s.ray)) {
                s.ray.tmax = t;
                s.hit.tri = __float_as_uint(a.w);
                s.hit.slot = first + k;
                s.hit.t = t;
                s.hit.b0 = b0;
                s.hit.b1 = b1;
                s.hit.b2 = b2;
            }
        }
    }
    return false;
}

// One step; returns true when the traversal of the ray is over (any-hit: found an occluder).
// A step visits one node (an interior node or a leaf), then descends or pops.
template <bool kAnyHit, class Node, class Alpha = NoAlpha>
KS_D bool trav_step(const Node *__restrict__ nodes, const float4 *__restrict__ tris, TravState &s,
                    TravStack &stack, int culling, int &overflow, TravCount *count, const Alpha &alpha = Alpha{})
{
    if (s.ref & kLeafBit) {
        if (trav_leaf<kAnyHit>(tris, s, culling, count, alpha))
            return true;
    } else {
        const int r = trav_node<kAnyHit>(nodes, s, stack, overflow, count);
        if (r != 0)
            return r < 0;
    }
    return !trav_pop(s, stack);
}

// One warp-wide traversal step; every lane of the warp calls it (busy: the lane holds a ray).
// Closest-hit queries: lanes whose current node is a leaf wait until at least KS_LEAF_BATCH of
// them (or all busy lanes) are at a leaf, then test their leaves together; the others descend
// through interior nodes meanwhile.  Each ray's own sequence of tests is that of trav_step (a
// waiting ray just pauses), but a warp runs the large triangle test with many lanes at once
// instead of with the two or three that reach a leaf in the same step (about 10 % less time for
// extension rays).  Any-hit queries step without waiting: holding back a leaf that may end the
// ray costs them more than the batching saves.  Returns true when this lane's ray is over.
#ifndef KS_LEAF_BATCH
#define KS_LEAF_BATCH 8
#endif
#ifndef KS_LEAF_BATCH_ANY
#define KS_LEAF_BATCH_ANY 0
#endif
template <bool kAnyHit, class Node, class Alpha = NoAlpha>
KS_D bool trav_warp_step(const Node *__restrict__ nodes, const float4 *__restrict__ tris, TravState &s,
                         TravStack &stack, int culling, int &overflow, TravCount *count, bool busy,
                         const Alpha &alpha = Alpha{})
{
    constexpr int kBatch = kAnyHit ? KS_LEAF_BATCH_ANY : KS_LEAF_BATCH;
    if constexpr (kBatch == 0) {
        return busy && trav_step<kAnyHit>(nodes, tris, s, stack, culling, overflow, count, alpha);
    } else {
        const bool at_leaf = busy && (s.ref & kLeafBit);
        const uint32_t leaves = __ballot_sync(0xffffffffu, at_leaf);
        const uint32_t inner = __ballot_sync(0xffffffffu, busy && !at_leaf);
        if (__popc(leaves) >= kBatch || inner == 0) {
            if (!at_leaf)
                return false;
            if (trav_leaf<kAnyHit>(tris, s, culling, count, alpha))
                return true;
            return !trav_pop(s, stack);
        }
        if (!busy || at_leaf)
            return false;
        const int r = trav_node<kAnyHit>(nodes, s, stack, overflow, count);
        if (r != 0)
            return r < 0;
        return !trav_pop(s, stack);
    }
}

// Dynamic ray fetch for trav_step: each warp takes rays from a global counter and hands every lane
// that finished a new ray once at least KS_TRAV_REFILL lanes are idle, so a warp no longer runs
// until its longest ray ends with most lanes masked off.
#ifndef KS_TRAV_REFILL
#define KS_TRAV_REFILL 12
#endif

// Hands the idle lanes of the warp rays [base, base + popc(idle)) in lane order; every lane calls
// it.  Returns this lane's ray (or ~0u) and sets drained once the counter has passed count.
KS_D uint32_t warp_fetch(uint32_t *fetch, uint32_t count, bool idle, bool &drained)
{
    const uint32_t mask = __ballot_sync(0xffffffffu, idle);
    if (drained || mask == 0)
        return ~0u;
    const uint32_t lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == (uint32_t)(__ffs(mask) - 1))
        base = atomicAdd(fetch, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
    if (base + (uint32_t)__popc(mask) >= count)
        drained = true;
    if (!idle)
        return ~0u;
    const uint32_t id = base + __popc(mask & ((1u << lane) - 1u));
    return id < count ? id : ~0u;
}

// ---- two-level traversal (instances) --------------------------------------------------------
// The TLAS has the TravNode layout; its leaves list instance ids (items).  At an instance the ray
// is carried into object space by the inverse transform without renormalising its direction, so
// the hit distance t is the same in both spaces, and the prototype's BLAS is traversed with the
// closest distance found so far as tmax.
struct InstanceView
{
    uint32_t n;                  // instances; 0 = flat scene
    const TravNode *tlas;
    const uint32_t *items;
    uint32_t root_ref, root_count;
    float bmin[3], bmax[3];
    const float *xf, *inv;       // 12 floats (row-major 3x4) per instance
    const uint32_t *proto;       // prototype of each instance
    const uint4 *proto_root;     // (root ref, root count) per prototype
    const float *proto_bound;    // 6 floats per prototype
};
constexpr int kTlasStackDepth = 32;

template <bool kAnyHit>
KS_D bool traverse_instances(const TravNode *__restrict__ nodes, const float4 *__restrict__ tris,
                             const InstanceView &iv, RayQuery ray, int culling, Hit &hit, uint32_t &inst,
                             int &overflow, TravCount *count = nullptr)
{
    hit.tri = ~0u;
    inst = 0;
    const BoxHelper bh = make_box_helper(ray.d);
    uint4 stack[kTlasStackDepth];
    int sp = 0;
    float t0, t1;
    if (!slab(ray, bh, iv.bmin, iv.bmax, t0, t1) || !(t0 < ray.tmax && t1 > ray.tmin))
        return false;
    uint32_t ref = iv.root_ref, cnt = iv.root_count;
    while (true) {
        if (ref & kLeafBit) {
            uint32_t first = ref & ~kLeafBit;
            for (uint32_t k = 0; k < cnt; ++k) {
                const uint32_t id = __ldg(&iv.items[first + k]);
                const float *m = iv.inv + 12 * (size_t)id;
                float mi[12];
#pragma unroll
                for (int e = 0; e < 12; ++e)
                    mi[e] = __ldg(&m[e]);
                RayQuery q;
                q.o = xf_point(mi, ray.o);
                q.d = xf_dir(mi, ray.d);
                q.tmin = ray.tmin;
                q.tmax = ray.tmax;
                const uint32_t pr = __ldg(&iv.proto[id]);
                const uint4 r = __ldg(&iv.proto_root[pr]);
                float pb[6];
#pragma unroll
                for (int e = 0; e < 6; ++e)
                    pb[e] = __ldg(&iv.proto_bound[6 * (size_t)pr + e]);
                Hit h;
                if (traverse<kAnyHit>(nodes, tris, r.x, r.y, pb, pb + 3, q, culling, h, overflow, count)) {
                    if (kAnyHit) {
                        hit.tri = h.tri;
                        inst = id;
                        return true;
                    }
                    if (h.t < ray.tmax) {
                        ray.tmax = h.t;
                        hit = h;
                        inst = id;
                    }
                }
            }
        } else {
            const TravNode *n = iv.tlas + ref;
            if (count)
                count->nodes++;
            float4 A = __ldg(&n->a), B = __ldg(&n->b), C = __ldg(&n->c);
            uint4 D = __ldg(&n->d);
            float lmin[3] = {A.x, A.y, A.z}, lmax[3] = {A.w, B.x, B.y};
            float rmin[3] = {B.z, B.w, C.x}, rmax[3] = {C.y, C.z, C.w};
            float lt0, lt1, rt0, rt1;
            bool lok = slab(ray, bh, lmin, lmax, lt0, lt1) && lt1 > ray.tmin && lt0 < ray.tmax;
            bool rok = slab(ray, bh, rmin, rmax, rt0, rt1) && rt1 > ray.tmin && rt0 < ray.tmax;
            uint32_t axis = D.z >> 30;
            uint32_t lcnt = D.z & 0x3fffffffu, rcnt = D.w;
            bool right_first = bh.neg[axis] != 0;
            uint32_t near_ref = right_first ? D.y : D.x, far_ref = right_first ? D.x : D.y;
            uint32_t near_cnt = right_first ? rcnt : lcnt, far_cnt = right_first ? lcnt : rcnt;
            bool near_ok = right_first ? rok : lok, far_ok = right_first ? lok : rok;
            float far_t = right_first ? lt0 : rt0;
            if (near_ok) {
                if (far_ok) {
                    if (sp >= kTlasStackDepth) {
                        overflow = 1;
                        return !kAnyHit && hit.tri != ~0u;
                    }
                    stack[sp++] = make_uint4(far_ref, far_cnt, __float_as_uint(far_t), 0u);
                }
                ref = near_ref;
                cnt = near_cnt;
                continue;
            }
            if (far_ok) {
                ref = far_ref;
                cnt = far_cnt;
                continue;
            }
        }
        bool found = false;
        while (sp > 0) {
            const uint4 e = stack[--sp];
            if (__uint_as_float(e.z) < ray.tmax) {
                ref = e.x;
                cnt = e.y;
                found = true;
                break;
            }
        }
        if (!found)
            break;
    }
    return hit.tri != ~0u;
}


// ---- resumable two-level traversal (persistent kernels, instanced scenes) -------------------
// traverse_instances cut into steps: a step visits one TLAS node, starts the BLAS traversal of
// the next instance of a TLAS leaf, or advances that BLAS traversal by one trav_step.  With the
// BLAS in its binary layout (Node = TravNode) each ray makes the same TLAS and BLAS tests as
// traverse_instances (identical hits, distances and instances); with the 4-wide view (WideNode)
// the BLAS visiting order differs, which only matters for exact ties.  The BLAS stack is the caller's TravStack, the
// TLAS stack (kTlasStackDepth entries) a separate caller array, so that the scalar state can stay
// in registers.
struct InstTravState
{
    RayQuery ray;       // world-space ray; tmax shrinks with the hits found
    BoxHelper bh;       // of the world-space ray (TLAS boxes)
    uint32_t ref, cnt;  // current TLAS node
    uint32_t item;      // next instance of the current TLAS leaf
    int sp;             // TLAS stack size
    bool in_blas;       // a BLAS traversal is running in blas
    uint32_t inst;      // its instance
    TravState blas;
    Hit hit;            // best hit so far
    uint32_t hit_inst;  // its instance
};

// False when the ray misses the TLAS root box.
KS_D bool inst_begin(InstTravState &s, const InstanceView &iv, const RayQuery &ray)
{
    s.hit.tri = ~0u;
    s.hit_inst = 0;
    s.ray = ray;
    s.bh = make_box_helper(ray.d);
    s.sp = 0;
    s.item = 0;
    s.in_blas = false;
    s.ref = iv.root_ref;
    s.cnt = iv.root_count;
    float t0, t1;
    return slab(s.ray, s.bh, iv.bmin, iv.bmax, t0, t1) && t0 < s.ray.tmax && t1 > s.ray.tmin;
}

// TLAS pop with the tmax re-check; false when the TLAS stack is empty (the ray is done).
KS_D bool inst_pop(InstTravState &s, const uint4 *tstack)
{
    while (s.sp > 0) {
        const uint4 e = tstack[--s.sp];
        if (__uint_as_float(e.z) < s.ray.tmax) {
            s.ref = e.x;
            s.cnt = e.y;
            s.item = 0;
            return true;
        }
    }
    return false;
}

// One step; true when the ray's traversal is over (any-hit: an occluder was found).
template <bool kAnyHit, class Node>
KS_D bool inst_step(const Node *__restrict__ nodes, const float4 *__restrict__ tris, const InstanceView &iv,
                    InstTravState &s, uint4 *tstack, TravStack &blas_stack, int culling, int &overflow,
                    TravCount *count)
{
    if (s.in_blas) {
        if (!trav_step<kAnyHit>(nodes, tris, s.blas, blas_stack, culling, overflow, count))
            return false;
        s.in_blas = false;
        const Hit &h = s.blas.hit;
        if (h.tri != ~0u) {
            if (kAnyHit) {
                s.hit.tri = h.tri;
                s.hit_inst = s.inst;
                return true;
            }
            if (h.t < s.ray.tmax) {
                s.ray.tmax = h.t;
                s.hit = h;
                s.hit_inst = s.inst;
            }
        }
        ++s.item;
        return false;
    }
    if (s.ref & kLeafBit) {
        if (s.item < s.cnt) {
            // the next instance of the leaf: the ray in object space, then its prototype's BLAS
            const uint32_t id = __ldg(&iv.items[(s.ref & ~kLeafBit) + s.item]);
            const float *m = iv.inv + 12 * (size_t)id;
            float mi[12];
#pragma unroll
            for (int e = 0; e < 12; ++e)
                mi[e] = __ldg(&m[e]);
            RayQuery q;
            q.o = xf_point(mi, s.ray.o);
            q.d = xf_dir(mi, s.ray.d);
            q.tmin = s.ray.tmin;
            q.tmax = s.ray.tmax;
            const uint32_t pr = __ldg(&iv.proto[id]);
            const uint4 r = __ldg(&iv.proto_root[pr]);
            float pb[6];
#pragma unroll
            for (int e = 0; e < 6; ++e)
                pb[e] = __ldg(&iv.proto_bound[6 * (size_t)pr + e]);
            if (trav_begin(s.blas, q, r.x, r.y, pb, pb + 3)) {
                s.in_blas = true;
                s.inst = id;
            } else {
                ++s.item;
            }
            return false;
        }
        return !inst_pop(s, tstack);
    }
    const TravNode *n = iv.tlas + s.ref;
    if (count)
        count->nodes++;
    float4 A = __ldg(&n->a), B = __ldg(&n->b), C = __ldg(&n->c);
    uint4 D = __ldg(&n->d);
    float lmin[3] = {A.x, A.y, A.z}, lmax[3] = {A.w, B.x, B.y};
    float rmin[3] = {B.z, B.w, C.x}, rmax[3] = {C.y, C.z, C.w};
    float lt0, lt1, rt0, rt1;
    bool lok = slab(s.ray, s.bh, lmin, lmax, lt0, lt1) && lt1 > s.ray.tmin && lt0 < s.ray.tmax;
    bool rok = slab(s.ray, s.bh, rmin, rmax, rt0, rt1) && rt1 > s.ray.tmin && rt0 < s.ray.tmax;
    uint32_t axis = D.z >> 30;
    uint32_t lcnt = D.z & 0x3fffffffu, rcnt = D.w;
    bool right_first = s.bh.neg[axis] != 0;
    uint32_t near_ref = right_first ? D.y : D.x, far_ref = right_first ? D.x : D.y;
    uint32_t near_cnt = right_first ? rcnt : lcnt, far_cnt = right_first ? lcnt : rcnt;
    bool near_ok = right_first ? rok : lok, far_ok = right_first ? lok : rok;
    float far_t = right_first ? lt0 : rt0;
    if (near_ok && far_ok) {
        if (s.sp >= kTlasStackDepth) {
            overflow = 1;
            return true;
        }
        tstack[s.sp++] = make_uint4(far_ref, far_cnt, __float_as_uint(far_t), 0u);
    }
    if (near_ok || far_ok) {
        s.ref = near_ok ? near_ref : far_ref;
        s.cnt = near_ok ? near_cnt : far_cnt;
        s.item = 0;
        return false;
    }
    return !inst_pop(s, tstack);
}

// Warp-wide step of the two-level traversal (every lane calls it; busy: the lane holds a ray).
// Closest-hit queries batch their BLAS leaf tests like trav_warp_step: a lane whose BLAS node is
// a leaf waits until KS_LEAF_BATCH lanes (or all busy lanes) are at one.  Each ray's own sequence
// of tests is that of inst_step.
template <bool kAnyHit, class Node>
KS_D bool inst_warp_step(const Node *__restrict__ nodes, const float4 *__restrict__ tris, const InstanceView &iv,
                         InstTravState &s, uint4 *tstack, TravStack &blas_stack, int culling, int &overflow,
                         TravCount *count, bool busy)
{
    if constexpr (kAnyHit || KS_LEAF_BATCH == 0) {
        return busy && inst_step<kAnyHit>(nodes, tris, iv, s, tstack, blas_stack, culling, overflow, count);
    } else {
        const bool at_leaf = busy && s.in_blas && (s.blas.ref & kLeafBit);
        const uint32_t leaves = __ballot_sync(0xffffffffu, at_leaf);
        const uint32_t others = __ballot_sync(0xffffffffu, busy && !at_leaf);
        const bool leaf_phase = __popc(leaves) >= KS_LEAF_BATCH || others == 0;
        if (leaf_phase ? !at_leaf : (!busy || at_leaf))
            return false;
        return inst_step<false>(nodes, tris, iv, s, tstack, blas_stack, culling, overflow, count);
    }
}

} // namespace ksb
