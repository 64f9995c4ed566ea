// Parallel SBVH builder for sm_100a.
//
// Produces the same tree as the reference's sequential builder ksc::SBVH::build
// (cuda/sbvh.cu:81-440): same SAH object-split estimate (:81-136), same spatial-split estimate
// (:138-216) and skip test (:132-134), same leaf rule (:351-354), same reference un-splitting
// (:257-287), same depth-first flattening (:375-393).  Every split decision of the reference
// depends only on the *multiset* of references of a node (min/max unions, integer counts, and
// per-reference tests against fixed per-node values), so the tree can be built breadth-first,
// one level of nodes at a time, with all references of the level processed in parallel:
//
//   per level:  bounds -> prep -> object bins -> object eval -> spatial bins -> decide
//               -> spatial classes -> spatial costs -> count -> scan -> scatter -> children
//
// Floating-point expressions are written exactly as in the reference (std::min/std::max
// argument order, std::lerp, float(count) * area, ...) and the translation unit is compiled with
// -fmad=false, so every cost and comparison rounds as on the reference's host.
// Min/max accumulation across threads uses an order-preserving integer encoding of floats and
// integer atomics, which is exact and deterministic.  Only the order of primitives inside a leaf
// can differ from the reference (it depends on std::partition's swap order).
#include "ks_scan.cuh"
#include "ks_scene.h"

#include <algorithm>
#include <cstring>

namespace ksb
{
namespace
{

constexpr int kMaxBuckets = 16;
constexpr uint32_t kChunk = 1024; // references per work item (one warp each)
constexpr int kWarpsPerBlock = 8;

enum NodeKind : int
{
    kPending = 0,
    kLeaf = 1,
    kObject = 2,
    kSpatial = 3,
};

struct BRef
{
    float4 lo; // min xyz, original triangle index (bits) in w
    float4 hi; // max xyz
};

struct LevelNode
{
    uint32_t ref_begin, ref_count, build_id, first_item;
};

struct Item
{
    uint32_t node, begin, count, single;
};

struct NodeInfo
{
    float bmin[3], bmax[3], cmin[3], cmax[3];
    int kind, dim, skip;
    int os_bucket;
    float os_cost;
    float osL[6], osR[6];
    int ss_bucket;
    float ss_cost;
    float ssL[6], ssR[6];
    float clip[kMaxBuckets + 1];
    float split_clip;
    int n1, n2;
    float full_cost, saL, saR;
    uint32_t cls[3];
    uint32_t n_left, n_right;
};

struct BuildRec
{
    float bmin[3], bmax[3];
    uint32_t left, right, axis, leaf;
    uint32_t leaf_begin, leaf_count;
    uint32_t size, prims;
    uint32_t dfs, prim_off;
};

struct Params
{
    uint32_t max_prims;
    uint32_t buckets;
    float trav_weight;
    float alpha;
};

// ---- float helpers with the reference's host semantics -------------------------------------
KS_D float smin(float a, float b) { return (b < a) ? b : a; } // std::min(a, b)
KS_D float smax(float a, float b) { return (a < b) ? b : a; } // std::max(a, b)

// Order-preserving map float -> uint32 (total order, -0 < +0), exact round trip.
KS_D uint32_t f2o(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
KS_D float o2f(uint32_t o) { return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o); }
constexpr uint32_t kOInf = 0xFF800000u;    // f2o(+inf): identity for min
constexpr uint32_t kONegInf = 0x007FFFFFu; // f2o(-inf): identity for max

KS_D float surface_area(const float mn[3], const float mx[3])
{
    float ex = mx[0] - mn[0], ey = mx[1] - mn[1], ez = mx[2] - mn[2];
    return 2.0f * (ex * ey + ey * ez + ex * ez);
}
KS_D void box_empty(float b[6])
{
    b[0] = b[1] = b[2] = kInf;
    b[3] = b[4] = b[5] = -kInf;
}
KS_D void box_expand(float b[6], const float o[6])
{
    for (int k = 0; k < 3; ++k) {
        b[k] = smin(b[k], o[k]);
        b[3 + k] = smax(b[3 + k], o[3 + k]);
    }
}
KS_D float ref_lo(const BRef &r, int d) { return d == 0 ? r.lo.x : (d == 1 ? r.lo.y : r.lo.z); }
KS_D float ref_hi(const BRef &r, int d) { return d == 0 ? r.hi.x : (d == 1 ? r.hi.y : r.hi.z); }
KS_D float ref_center(const BRef &r, int d) { return 0.5f * (ref_lo(r, d) + ref_hi(r, d)); }

// Bucket of a reference for the object split (cuda/sbvh.cu:98-100).
KS_D uint32_t object_bucket(const BRef &r, const NodeInfo &n, uint32_t buckets)
{
    int d = n.dim;
    float ext = n.cmax[d] - n.cmin[d];
    float off = ext == 0.0f ? 0.0f : (ref_center(r, d) - n.cmin[d]) / ext;
    uint32_t b = (uint32_t)floorf((float)buckets * off);
    return b < buckets - 1 ? b : buckets - 1;
}

// Reference un-splitting decision for a straddling reference (cuda/sbvh.cu:257-287).
// Returns 0 = move left, 1 = move right, 2 = split.
KS_D int unsplit_decision(const BRef &r, const NodeInfo &n)
{
    float rb[6] = {r.lo.x, r.lo.y, r.lo.z, r.hi.x, r.hi.y, r.hi.z};
    float jl[6], jr[6];
    for (int k = 0; k < 6; ++k) {
        jl[k] = n.ssL[k];
        jr[k] = n.ssR[k];
    }
    // join(a, b) = AABB3(min(a.min, b.min), max(a.max, b.max)) with ksc::min/max = std::min/max
    for (int k = 0; k < 3; ++k) {
        jl[k] = smin(jl[k], rb[k]);
        jl[3 + k] = smax(jl[3 + k], rb[3 + k]);
        jr[k] = smin(jr[k], rb[k]);
        jr[3 + k] = smax(jr[3 + k], rb[3 + k]);
    }
    float move_left = surface_area(jl, jl + 3) * (float)n.n1 + n.saR * (float)(n.n2 - 1);
    float move_right = n.saL * (float)(n.n1 - 1) + surface_area(jr, jr + 3) * (float)n.n2;
    float m = smin(n.full_cost, smin(move_left, move_right));
    if (m == move_left)
        return 0;
    if (m == move_right)
        return 1;
    return 2;
}

// Destination of a reference: bit0 = goes left, bit1 = goes right, bit2 = to leaf pool.
KS_D int ref_destination(const BRef &r, const NodeInfo &n, uint32_t buckets)
{
    if (n.kind == kLeaf)
        return 4;
    if (n.kind == kObject)
        return object_bucket(r, n, buckets) <= (uint32_t)n.os_bucket ? 1 : 2;
    int d = n.dim;
    if (ref_hi(r, d) <= n.split_clip)
        return 1;
    if (ref_lo(r, d) >= n.split_clip)
        return 2;
    int u = unsplit_decision(r, n);
    return u == 0 ? 1 : (u == 1 ? 2 : 3);
}

// ---- kernels --------------------------------------------------------------------------------

__global__ void k_init_refs(const float *verts, const uint32_t *idx, uint32_t tri_begin, uint32_t n_tris, BRef *refs)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_tris)
        return;
    float b[6];
    box_empty(b);
    for (int v = 0; v < 3; ++v) {
        uint32_t vi = idx[3 * (tri_begin + i) + v];
        float p[6] = {verts[3 * vi], verts[3 * vi + 1], verts[3 * vi + 2], 0, 0, 0};
        p[3] = p[0];
        p[4] = p[1];
        p[5] = p[2];
        box_expand(b, p);
    }
    refs[i].lo = make_float4(b[0], b[1], b[2], __uint_as_float(tri_begin + i));
    refs[i].hi = make_float4(b[3], b[4], b[5], 0.0f);
}

__global__ void k_item_counts(const LevelNode *nodes, uint32_t n, uint32_t *counts)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        counts[i] = (nodes[i].ref_count + kChunk - 1) / kChunk;
}

__global__ void k_items_fill(LevelNode *nodes, uint32_t n, const uint32_t *item_off, Item *items)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    LevelNode nd = nodes[i];
    uint32_t first = item_off[i], cnt = item_off[i + 1] - first;
    nodes[i].first_item = first;
    for (uint32_t k = 0; k < cnt; ++k) {
        Item it;
        it.node = i;
        it.begin = nd.ref_begin + k * kChunk;
        uint32_t rem = nd.ref_count - k * kChunk;
        it.count = rem < kChunk ? rem : kChunk;
        it.single = cnt == 1;
        items[first + k] = it;
    }
}

__global__ void k_acc_init(const LevelNode *nodes, uint32_t *bnd, uint32_t *obj, uint32_t *sp, NodeInfo *info,
                           uint32_t n, uint32_t buckets)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    info[i].cls[0] = info[i].cls[1] = info[i].cls[2] = 0;
    if (nodes[i].ref_count <= kChunk)
        return; // single work item: every accumulator is written with plain stores
    for (int k = 0; k < 12; ++k)
        bnd[12 * i + k] = (k < 3 || (k >= 6 && k < 9)) ? kOInf : kONegInf;
    for (uint32_t b = 0; b < buckets; ++b) {
        uint32_t *o = obj + (size_t)(i * buckets + b) * 7;
        o[0] = 0;
        for (int k = 0; k < 3; ++k) {
            o[1 + k] = kOInf;
            o[4 + k] = kONegInf;
        }
        uint32_t *s = sp + (size_t)(i * buckets + b) * 8;
        s[0] = s[1] = 0;
        for (int k = 0; k < 3; ++k) {
            s[2 + k] = kOInf;
            s[5 + k] = kONegInf;
        }
    }
}

KS_D float warp_min(float v)
{
    for (int o = 16; o > 0; o >>= 1)
        v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
KS_D float warp_max(float v)
{
    for (int o = 16; o > 0; o >>= 1)
        v = smax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Node bounds and centroid bounds (cuda/sbvh.cu:308-313, 330-333).
__global__ void k_bounds(const Item *items, uint32_t n_items, const BRef *refs, uint32_t *bnd)
{
    uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n_items)
        return;
    Item it = items[w];
    float v[12];
    for (int k = 0; k < 3; ++k) {
        v[k] = kInf;
        v[3 + k] = -kInf;
        v[6 + k] = kInf;
        v[9 + k] = -kInf;
    }
    for (uint32_t j = lane; j < it.count; j += 32) {
        BRef r = refs[it.begin + j];
        float lo[3] = {r.lo.x, r.lo.y, r.lo.z}, hi[3] = {r.hi.x, r.hi.y, r.hi.z};
        for (int k = 0; k < 3; ++k) {
            v[k] = smin(v[k], lo[k]);
            v[3 + k] = smax(v[3 + k], hi[k]);
            float c = 0.5f * (lo[k] + hi[k]);
            v[6 + k] = smin(v[6 + k], c);
            v[9 + k] = smax(v[9 + k], c);
        }
    }
    for (int k = 0; k < 3; ++k) {
        v[k] = warp_min(v[k]);
        v[3 + k] = warp_max(v[3 + k]);
        v[6 + k] = warp_min(v[6 + k]);
        v[9 + k] = warp_max(v[9 + k]);
    }
    if (lane < 12) {
        float x = v[0];
        for (int k = 1; k < 12; ++k)
            if ((int)lane == k)
                x = v[k];
        bool is_min = lane < 3 || (lane >= 6 && lane < 9);
        uint32_t *dst = bnd + 12 * it.node + lane;
        if (it.single)
            *dst = f2o(x);
        else if (is_min)
            atomicMin(dst, f2o(x));
        else
            atomicMax(dst, f2o(x));
    }
}

__device__ float g_root_sa;

// Leaf tests before any split estimate (cuda/sbvh.cu:301-338) + node record.
__global__ void k_prep(const LevelNode *nodes, uint32_t n, const uint32_t *bnd, NodeInfo *info, BuildRec *recs,
                       int is_root_level)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    NodeInfo &ni = info[i];
    for (int k = 0; k < 3; ++k) {
        ni.bmin[k] = o2f(bnd[12 * i + k]);
        ni.bmax[k] = o2f(bnd[12 * i + 3 + k]);
        ni.cmin[k] = o2f(bnd[12 * i + 6 + k]);
        ni.cmax[k] = o2f(bnd[12 * i + 9 + k]);
    }
    if (is_root_level)
        g_root_sa = surface_area(ni.bmin, ni.bmax);
    BuildRec &rec = recs[nodes[i].build_id];
    for (int k = 0; k < 3; ++k) {
        rec.bmin[k] = ni.bmin[k];
        rec.bmax[k] = ni.bmax[k];
    }
    ni.kind = kPending;
    ni.skip = 1;
    if (nodes[i].ref_count == 1) {
        ni.kind = kLeaf;
        return;
    }
    float ex = ni.cmax[0] - ni.cmin[0], ey = ni.cmax[1] - ni.cmin[1], ez = ni.cmax[2] - ni.cmin[2];
    int dim = (ex >= ey && ex >= ez) ? 0 : ((ey >= ex && ey >= ez) ? 1 : 2);
    ni.dim = dim;
    if (ni.cmax[dim] == ni.cmin[dim])
        ni.kind = kLeaf;
}

// Object-split bucket statistics (cuda/sbvh.cu:95-102).
__global__ void k_obj_bins(const Item *items, uint32_t n_items, const BRef *refs, const NodeInfo *info,
                           uint32_t buckets, uint32_t *obj)
{
    __shared__ uint32_t sbins[kWarpsPerBlock][kMaxBuckets * 7];
    uint32_t wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t w = blockIdx.x * kWarpsPerBlock + wl;
    if (w >= n_items)
        return;
    Item it = items[w];
    const NodeInfo &ni = info[it.node];
    if (ni.kind != kPending)
        return;
    uint32_t *sb = sbins[wl];
    for (uint32_t k = lane; k < buckets * 7; k += 32) {
        uint32_t f = k % 7;
        sb[k] = f == 0 ? 0u : (f < 4 ? kOInf : kONegInf);
    }
    __syncwarp();
    for (uint32_t j = lane; j < it.count; j += 32) {
        BRef r = refs[it.begin + j];
        uint32_t b = object_bucket(r, ni, buckets);
        uint32_t *o = sb + b * 7;
        atomicAdd(o, 1u);
        atomicMin(o + 1, f2o(r.lo.x));
        atomicMin(o + 2, f2o(r.lo.y));
        atomicMin(o + 3, f2o(r.lo.z));
        atomicMax(o + 4, f2o(r.hi.x));
        atomicMax(o + 5, f2o(r.hi.y));
        atomicMax(o + 6, f2o(r.hi.z));
    }
    __syncwarp();
    uint32_t *dst = obj + (size_t)it.node * buckets * 7;
    for (uint32_t k = lane; k < buckets * 7; k += 32) {
        uint32_t f = k % 7;
        if (it.single)
            dst[k] = sb[k];
        else if (f == 0)
            atomicAdd(dst + k, sb[k]);
        else if (f < 4)
            atomicMin(dst + k, sb[k]);
        else
            atomicMax(dst + k, sb[k]);
    }
}

// Picks the cheapest split of a bucket table (cuda/sbvh.cu:104-130, 190-216).
// bins: per bucket [count-like for left, count-like for right, min xyz, max xyz] accessors.
template <typename LeftCount, typename RightCount, typename BoxOf>
KS_D void best_split(uint32_t buckets, float travw, float node_sa, LeftCount lc, RightCount rc, BoxOf box,
                     int &best_bucket, float &best_cost, float bl[6], float br[6])
{
    for (uint32_t i = 0; i + 1 < buckets; ++i) {
        float L[6], R[6];
        box_empty(L);
        box_empty(R);
        uint32_t c0 = 0, c1 = 0;
        for (uint32_t j = 0; j <= i; ++j) {
            float b[6];
            box(j, b);
            box_expand(L, b);
            c0 += lc(j);
        }
        for (uint32_t j = i + 1; j < buckets; ++j) {
            float b[6];
            box(j, b);
            box_expand(R, b);
            c1 += rc(j);
        }
        float cost = travw + ((float)c0 * surface_area(L, L + 3) + (float)c1 * surface_area(R, R + 3)) / node_sa;
        if (i == 0 || cost < best_cost) {
            best_cost = cost;
            best_bucket = (int)i;
            for (int k = 0; k < 6; ++k) {
                bl[k] = L[k];
                br[k] = R[k];
            }
        }
    }
}

__global__ void k_obj_eval(uint32_t n, const uint32_t *obj, NodeInfo *info, Params p)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    NodeInfo &ni = info[i];
    if (ni.kind != kPending)
        return;
    const uint32_t *o = obj + (size_t)i * p.buckets * 7;
    float node_sa = surface_area(ni.bmin, ni.bmax);
    auto cnt = [&](uint32_t j) { return o[j * 7]; };
    auto box = [&](uint32_t j, float b[6]) {
        for (int k = 0; k < 6; ++k)
            b[k] = o2f(o[j * 7 + 1 + k]);
    };
    best_split(p.buckets, p.trav_weight, node_sa, cnt, cnt, box, ni.os_bucket, ni.os_cost, ni.osL, ni.osR);
    // skipSpatialSplit (cuda/sbvh.cu:132-134)
    float imn[3], imx[3];
    bool empty = false;
    for (int k = 0; k < 3; ++k) {
        imn[k] = smax(ni.osL[k], ni.osR[k]);
        imx[k] = smin(ni.osL[3 + k], ni.osR[3 + k]);
    }
    if (imn[0] > imx[0] || imn[1] > imx[1] || imn[2] > imx[2])
        empty = true; // intersect() returns an empty AABB3, whose is_empty() is true
    float isa = empty ? 0.0f : surface_area(imn, imx);
    ni.skip = (isa / g_root_sa <= p.alpha) ? 1 : 0;
    if (!ni.skip) {
        int d = ni.dim;
        for (uint32_t b = 0; b <= p.buckets; ++b)
            ni.clip[b] = std_lerp(ni.bmin[d], ni.bmax[d], (float)b / (float)p.buckets);
    }
}

// Spatial-split bucket statistics (cuda/sbvh.cu:154-176).
__global__ void k_sp_bins(const Item *items, uint32_t n_items, const BRef *refs, const NodeInfo *info,
                          uint32_t buckets, uint32_t *sp)
{
    __shared__ uint32_t sbins[kWarpsPerBlock][kMaxBuckets * 8];
    uint32_t wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t w = blockIdx.x * kWarpsPerBlock + wl;
    if (w >= n_items)
        return;
    Item it = items[w];
    const NodeInfo &ni = info[it.node];
    if (ni.kind != kPending || ni.skip)
        return;
    uint32_t *sb = sbins[wl];
    for (uint32_t k = lane; k < buckets * 8; k += 32) {
        uint32_t f = k % 8;
        sb[k] = f < 2 ? 0u : (f < 5 ? kOInf : kONegInf);
    }
    __syncwarp();
    int d = ni.dim;
    for (uint32_t j = lane; j < it.count; j += 32) {
        BRef r = refs[it.begin + j];
        float lo[3] = {r.lo.x, r.lo.y, r.lo.z}, hi[3] = {r.hi.x, r.hi.y, r.hi.z};
        uint32_t enter = buckets - 1, exit = 0;
        for (uint32_t b = 0; b < buckets; ++b) {
            if (lo[d] > ni.clip[b + 1])
                continue;
            if (hi[d] < ni.clip[b])
                break;
            exit = exit < b ? b : exit;   // std::max(exit, b)
            enter = b < enter ? b : enter; // std::min(enter, b)
            float cl[3] = {lo[0], lo[1], lo[2]}, ch[3] = {hi[0], hi[1], hi[2]};
            cl[d] = smax(cl[d], ni.clip[b]);
            ch[d] = smin(ch[d], ni.clip[b + 1]);
            uint32_t *s = sb + b * 8;
            for (int k = 0; k < 3; ++k) {
                atomicMin(s + 2 + k, f2o(cl[k]));
                atomicMax(s + 5 + k, f2o(ch[k]));
            }
        }
        atomicAdd(sb + enter * 8 + 0, 1u);
        atomicAdd(sb + exit * 8 + 1, 1u);
    }
    __syncwarp();
    uint32_t *dst = sp + (size_t)it.node * buckets * 8;
    for (uint32_t k = lane; k < buckets * 8; k += 32) {
        uint32_t f = k % 8;
        if (it.single)
            dst[k] = sb[k];
        else if (f < 2)
            atomicAdd(dst + k, sb[k]);
        else if (f < 5)
            atomicMin(dst + k, sb[k]);
        else
            atomicMax(dst + k, sb[k]);
    }
}

// Spatial estimate + leaf/object/spatial decision (cuda/sbvh.cu:347-360).
__global__ void k_decide(const LevelNode *nodes, uint32_t n, const uint32_t *sp, NodeInfo *info, Params p)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    NodeInfo &ni = info[i];
    if (ni.kind != kPending)
        return;
    if (!ni.skip) {
        const uint32_t *s = sp + (size_t)i * p.buckets * 8;
        float node_sa = surface_area(ni.bmin, ni.bmax);
        auto enter = [&](uint32_t j) { return s[j * 8 + 0]; };
        auto exitc = [&](uint32_t j) { return s[j * 8 + 1]; };
        auto box = [&](uint32_t j, float b[6]) {
            for (int k = 0; k < 6; ++k)
                b[k] = o2f(s[j * 8 + 2 + k]);
        };
        best_split(p.buckets, p.trav_weight, node_sa, enter, exitc, box, ni.ss_bucket, ni.ss_cost, ni.ssL, ni.ssR);
    }
    uint32_t ref_count = nodes[i].ref_count;
    float leaf_cost = (float)ref_count;
    if (ref_count <= p.max_prims && leaf_cost <= ni.os_cost && (ni.skip || leaf_cost <= ni.ss_cost)) {
        ni.kind = kLeaf;
        return;
    }
    if (ni.skip || ni.os_cost <= ni.ss_cost) {
        ni.kind = kObject;
    } else {
        ni.kind = kSpatial;
        int d = ni.dim;
        ni.split_clip = std_lerp(ni.bmin[d], ni.bmax[d], (float)(ni.ss_bucket + 1) / (float)p.buckets);
    }
}

// Left / right / straddling counts of a spatial split (cuda/sbvh.cu:242-251).
__global__ void k_sp_classes(const Item *items, uint32_t n_items, const BRef *refs, NodeInfo *info)
{
    uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n_items)
        return;
    Item it = items[w];
    NodeInfo &ni = info[it.node];
    if (ni.kind != kSpatial)
        return;
    uint32_t c[3] = {0, 0, 0};
    int d = ni.dim;
    for (uint32_t j = lane; j < it.count; j += 32) {
        BRef r = refs[it.begin + j];
        if (ref_hi(r, d) <= ni.split_clip)
            c[0]++;
        else if (ref_lo(r, d) >= ni.split_clip)
            c[1]++;
        else
            c[2]++;
    }
    for (int k = 0; k < 3; ++k) {
        uint32_t v = c[k];
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && v)
            atomicAdd(&ni.cls[k], v);
    }
}

__global__ void k_sp_costs(uint32_t n, NodeInfo *info)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    NodeInfo &ni = info[i];
    if (ni.kind != kSpatial)
        return;
    // n1 = rightStart (left + straddling), n2 = N - leftEnd (right + straddling) (cuda/sbvh.cu:256-258)
    ni.n1 = (int)(ni.cls[0] + ni.cls[2]);
    ni.n2 = (int)(ni.cls[1] + ni.cls[2]);
    ni.saL = surface_area(ni.ssL, ni.ssL + 3);
    ni.saR = surface_area(ni.ssR, ni.ssR + 3);
    ni.full_cost = ni.saL * (float)ni.n1 + ni.saR * (float)ni.n2;
}

// Per work item: how many references go left, right, or into the leaf pool.
__global__ void k_count(const Item *items, uint32_t n_items, const BRef *refs, const NodeInfo *info,
                        uint32_t buckets, uint32_t *cl, uint32_t *cr, uint32_t *cp)
{
    uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n_items)
        return;
    Item it = items[w];
    const NodeInfo &ni = info[it.node];
    uint32_t l = 0, r = 0, p = 0;
    for (uint32_t j = lane; j < it.count; j += 32) {
        int dst = ref_destination(refs[it.begin + j], ni, buckets);
        l += dst & 1;
        r += (dst >> 1) & 1;
        p += (dst >> 2) & 1;
    }
    for (int o = 16; o > 0; o >>= 1) {
        l += __shfl_xor_sync(0xffffffffu, l, o);
        r += __shfl_xor_sync(0xffffffffu, r, o);
        p += __shfl_xor_sync(0xffffffffu, p, o);
    }
    if (lane == 0) {
        cl[w] = l;
        cr[w] = r;
        cp[w] = p;
    }
}

// Child reference counts of every node, from the per-item scans.  A spatial split that leaves
// one side empty trips the reference's assertion (cuda/sbvh.cu:295); such a node falls back to
// its object split and the level is recounted.
__global__ void k_child_counts(uint32_t n, const uint32_t *item_off, const uint32_t *sl, const uint32_t *sr,
                               NodeInfo *info, uint32_t *flag)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    NodeInfo &ni = info[i];
    uint32_t a = item_off[i], b = item_off[i + 1];
    ni.n_left = sl[b] - sl[a];
    ni.n_right = sr[b] - sr[a];
    if (ni.kind == kSpatial && (ni.n_left == 0 || ni.n_right == 0)) {
        ni.kind = kObject;
        atomicAdd(flag, 1u);
    }
}

__global__ void k_scatter(const Item *items, uint32_t n_items, const BRef *refs, const NodeInfo *info,
                          uint32_t buckets, const uint32_t *sl, const uint32_t *sr, const uint32_t *spool,
                          uint32_t left_total, BRef *next, uint32_t pool_base, uint32_t *pool)
{
    uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n_items)
        return;
    Item it = items[w];
    const NodeInfo &ni = info[it.node];
    uint32_t ol = sl[w], orr = left_total + sr[w], op = pool_base + spool[w];
    uint32_t lt_mask = (1u << lane) - 1u;
    for (uint32_t j0 = 0; j0 < it.count; j0 += 32) {
        uint32_t j = j0 + lane;
        bool valid = j < it.count;
        BRef r;
        int dst = 0;
        if (valid) {
            r = refs[it.begin + j];
            dst = ref_destination(r, ni, buckets);
        }
        uint32_t bl = __ballot_sync(0xffffffffu, dst & 1);
        uint32_t br = __ballot_sync(0xffffffffu, (dst >> 1) & 1);
        uint32_t bp = __ballot_sync(0xffffffffu, (dst >> 2) & 1);
        if (dst & 4)
            pool[op + __popc(bp & lt_mask)] = __float_as_uint(r.lo.w);
        if (dst & 1) {
            BRef x = r;
            if (dst == 3) {
                int d = ni.dim;
                if (d == 0)
                    x.hi.x = ni.split_clip;
                else if (d == 1)
                    x.hi.y = ni.split_clip;
                else
                    x.hi.z = ni.split_clip;
            }
            next[ol + __popc(bl & lt_mask)] = x;
        }
        if (dst & 2) {
            BRef x = r;
            if (dst == 3) {
                int d = ni.dim;
                if (d == 0)
                    x.lo.x = ni.split_clip;
                else if (d == 1)
                    x.lo.y = ni.split_clip;
                else
                    x.lo.z = ni.split_clip;
            }
            next[orr + __popc(br & lt_mask)] = x;
        }
        ol += __popc(bl);
        orr += __popc(br);
        op += __popc(bp);
    }
}

__global__ void k_split_flags(const NodeInfo *info, uint32_t n, uint32_t *flags)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        flags[i] = (info[i].kind == kObject || info[i].kind == kSpatial) ? 1u : 0u;
}

__global__ void k_children(const LevelNode *nodes, uint32_t n, const NodeInfo *info, const uint32_t *split_scan,
                           uint32_t n_split, const uint32_t *sl, const uint32_t *sr, const uint32_t *spool,
                           uint32_t left_total, uint32_t pool_base, uint32_t next_build_base, BuildRec *recs,
                           LevelNode *next_nodes)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const NodeInfo &ni = info[i];
    LevelNode nd = nodes[i];
    BuildRec &rec = recs[nd.build_id];
    if (ni.kind == kLeaf) {
        rec.leaf = 1;
        rec.left = rec.right = 0;
        rec.axis = 0;
        rec.leaf_begin = pool_base + spool[nd.first_item];
        rec.leaf_count = nd.ref_count;
        return;
    }
    uint32_t k = split_scan[i];
    LevelNode L, R;
    L.ref_begin = sl[nd.first_item];
    L.ref_count = ni.n_left;
    L.build_id = next_build_base + k;
    L.first_item = 0;
    R.ref_begin = left_total + sr[nd.first_item];
    R.ref_count = ni.n_right;
    R.build_id = next_build_base + n_split + k;
    R.first_item = 0;
    next_nodes[k] = L;
    next_nodes[n_split + k] = R;
    rec.leaf = 0;
    rec.left = L.build_id;
    rec.right = R.build_id;
    rec.axis = (uint32_t)ni.dim;
}

// ---- flattening ------------------------------------------------------------------------------

__global__ void k_subtree(BuildRec *recs, uint32_t begin, uint32_t end)
{
    uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end)
        return;
    BuildRec &r = recs[i];
    if (r.leaf) {
        r.size = 1;
        r.prims = r.leaf_count;
    } else {
        r.size = 1 + recs[r.left].size + recs[r.right].size;
        r.prims = recs[r.left].prims + recs[r.right].prims;
    }
}

__global__ void k_dfs(BuildRec *recs, uint32_t begin, uint32_t end)
{
    uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end)
        return;
    BuildRec &r = recs[i];
    if (i == 0) {
        r.dfs = 0;
        r.prim_off = 0;
    }
    if (!r.leaf) {
        BuildRec &L = recs[r.left];
        BuildRec &R = recs[r.right];
        L.dfs = r.dfs + 1;
        L.prim_off = r.prim_off;
        R.dfs = r.dfs + 1 + L.size;
        R.prim_off = r.prim_off + L.prims;
    }
}

__global__ void k_emit(const BuildRec *recs, uint32_t n, const uint32_t *pool, RefNode *out, uint32_t *prims,
                       uint32_t *interior_flag)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const BuildRec &r = recs[i];
    RefNode node;
    for (int k = 0; k < 3; ++k) {
        node.bmin[k] = r.bmin[k];
        node.bmax[k] = r.bmax[k];
    }
    node.axis = r.leaf ? 0 : r.axis;
    node.right = r.leaf ? 0 : recs[r.right].dfs;
    node.prim_offset = r.prim_off;
    out[r.dfs] = node;
    interior_flag[r.dfs] = r.leaf ? 0u : 1u;
    if (r.leaf)
        for (uint32_t k = 0; k < r.leaf_count; ++k)
            prims[r.prim_off + k] = pool[r.leaf_begin + k];
}

// Traversal layout: one 64-byte record per interior node (DFS order), children boxes inline.
// Leaf children carry their primitive count (the count the reference's traversal derives from
// primOffset differences, cuda/sbvh.cu:546-552).
__global__ void k_trav(const BuildRec *recs, uint32_t n, const uint32_t *interior_scan, TravNode *trav)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const BuildRec &p = recs[i];
    if (p.leaf)
        return;
    const BuildRec &L = recs[p.left];
    const BuildRec &R = recs[p.right];
    auto ref_of = [&](const BuildRec &c) { return c.leaf ? (kLeafBit | c.prim_off) : interior_scan[c.dfs]; };
    TravNode t;
    t.a = make_float4(L.bmin[0], L.bmin[1], L.bmin[2], L.bmax[0]);
    t.b = make_float4(L.bmax[1], L.bmax[2], R.bmin[0], R.bmin[1]);
    t.c = make_float4(R.bmin[2], R.bmax[0], R.bmax[1], R.bmax[2]);
    t.d = make_uint4(ref_of(L), ref_of(R), L.prims | (p.axis << 30), R.prims);
    trav[interior_scan[p.dfs]] = t;
}

__global__ void k_prim_tris(const uint32_t *prims, uint32_t n_prims, const float *verts, const uint32_t *idx,
                            float4 *out)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_prims)
        return;
    uint32_t t = prims[i];
    float4 v[3];
    for (int k = 0; k < 3; ++k) {
        uint32_t vi = idx[3 * t + k];
        v[k] = make_float4(verts[3 * vi], verts[3 * vi + 1], verts[3 * vi + 2], 0.0f);
    }
    v[0].w = __uint_as_float(t);
    out[3 * i + 0] = v[0];
    out[3 * i + 1] = v[1];
    out[3 * i + 2] = v[2];
}

inline unsigned grid_for(uint64_t n, unsigned block) { return (unsigned)((n + block - 1) / block); }

} // namespace

// One SBVH over the triangles [tri_begin, tri_begin + n_tris) of the global arrays; primitive
// references keep global triangle indices.
struct RangeOut
{
    DevBuf<RefNode> ref_nodes;
    DevBuf<uint32_t> prims;
    DevBuf<TravNode> trav;
    DevBuf<float4> prim_tris;
    uint32_t n_nodes = 0, n_prims = 0, n_trav = 0;
    float bound[6] = {0, 0, 0, 0, 0, 0};
};

// `done` (may be null) is recorded on the stream after the last build kernel, before the scratch
// buffers are released.
// Scratch of build_range, kept by the context between builds: growing these buffers level by level
// costs a few hundred allocations per build (each replaced buffer's cudaFree waits for the
// device), so a context reuses them; they grow to the largest tree built on it and are freed with
// the context.
struct BuildScratch
{
    DevBuf<BRef> refs_a, refs_b;
    DevBuf<LevelNode> nodes_a, nodes_b;
    DevBuf<Item> items;
    DevBuf<NodeInfo> info;
    DevBuf<uint32_t> bnd, obj, sp, item_cnt, item_off, cl, cr, cp, sl, sr, spool, split_flag, split_scan, pool, flag;
    DevBuf<uint32_t> interior_flag, interior_scan;
    DevBuf<BuildRec> recs;
    ScanScratch scan;
};

static BuildScratch &build_scratch(ks_context *ctx)
{
    if (!ctx->build_cache)
        ctx->build_cache = std::make_shared<BuildScratch>();
    return *static_cast<BuildScratch *>(ctx->build_cache.get());
}

static ks_status build_range(ks_context *ctx, const float *verts, const uint32_t *indices, uint32_t tri_begin,
                             uint32_t n_tris, const Params &p, RangeOut &out, cudaEvent_t done = nullptr)
{
    cudaStream_t st = ctx->stream;
    BuildScratch &bs = build_scratch(ctx);
    auto &refs_a = bs.refs_a, &refs_b = bs.refs_b;
    auto &nodes_a = bs.nodes_a, &nodes_b = bs.nodes_b;
    auto &items = bs.items;
    auto &info = bs.info;
    auto &bnd = bs.bnd, &obj = bs.obj, &sp = bs.sp, &item_cnt = bs.item_cnt, &item_off = bs.item_off;
    auto &cl = bs.cl, &cr = bs.cr, &cp = bs.cp, &sl = bs.sl, &sr = bs.sr, &spool = bs.spool;
    auto &split_flag = bs.split_flag, &split_scan = bs.split_scan, &pool = bs.pool, &flag = bs.flag;
    auto &recs = bs.recs;
    auto &scan = bs.scan;

    size_t ref_cap = (size_t)n_tris * 2 + 1024;
    KS_CUDA_TRY(ctx, refs_a.reserve(ref_cap));
    KS_CUDA_TRY(ctx, refs_b.reserve(ref_cap));
    KS_CUDA_TRY(ctx, pool.reserve(ref_cap));
    size_t rec_cap = (size_t)n_tris * 4 + 1024;
    KS_CUDA_TRY(ctx, recs.reserve(rec_cap));
    KS_CUDA_TRY(ctx, flag.reserve(1));

    k_init_refs<<<grid_for(n_tris, 256), 256, 0, st>>>(verts, indices, tri_begin, n_tris, refs_a.ptr);
    LevelNode root{0, n_tris, 0, 0};
    KS_CUDA_TRY(ctx, nodes_a.reserve(1));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(nodes_a.ptr, &root, sizeof(root), cudaMemcpyHostToDevice, st));

    uint32_t n_active = 1, n_refs = n_tris, build_base = 0, pool_used = 0;
    std::vector<uint32_t> level_begin;
    BRef *cur = refs_a.ptr, *nxt = refs_b.ptr;
    DevBuf<BRef> *cur_buf = &refs_a, *nxt_buf = &refs_b;
    DevBuf<LevelNode> *cur_nodes = &nodes_a, *nxt_nodes = &nodes_b;
    int level = 0;
    while (n_active > 0) {
        level_begin.push_back(build_base);
        if ((size_t)build_base + n_active > rec_cap)
            return fail(ctx, KS_ERR_OUT_OF_MEMORY, "sbvh build: node record capacity exceeded");
        // work items
        KS_CUDA_TRY(ctx, item_cnt.reserve(n_active));
        KS_CUDA_TRY(ctx, item_off.reserve(n_active + 1));
        k_item_counts<<<grid_for(n_active, 256), 256, 0, st>>>(cur_nodes->ptr, n_active, item_cnt.ptr);
        KS_CUDA_TRY(ctx, exclusive_scan(item_cnt.ptr, item_off.ptr, n_active, scan, st));
        uint32_t n_items = 0;
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(&n_items, item_off.ptr + n_active, 4, cudaMemcpyDeviceToHost, st));
        KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        KS_CUDA_TRY(ctx, items.reserve(n_items));
        k_items_fill<<<grid_for(n_active, 256), 256, 0, st>>>(cur_nodes->ptr, n_active, item_off.ptr, items.ptr);
        // accumulators
        KS_CUDA_TRY(ctx, info.reserve(n_active));
        KS_CUDA_TRY(ctx, bnd.reserve((size_t)n_active * 12));
        KS_CUDA_TRY(ctx, obj.reserve((size_t)n_active * p.buckets * 7));
        KS_CUDA_TRY(ctx, sp.reserve((size_t)n_active * p.buckets * 8));
        k_acc_init<<<grid_for(n_active, 128), 128, 0, st>>>(cur_nodes->ptr, bnd.ptr, obj.ptr, sp.ptr, info.ptr,
                                                            n_active, p.buckets);
        unsigned wgrid = grid_for((uint64_t)n_items * 32, 256);
        unsigned wgrid8 = grid_for(n_items, kWarpsPerBlock);
        k_bounds<<<wgrid, 256, 0, st>>>(items.ptr, n_items, cur, bnd.ptr);
        k_prep<<<grid_for(n_active, 128), 128, 0, st>>>(cur_nodes->ptr, n_active, bnd.ptr, info.ptr, recs.ptr + 0,
                                                        level == 0);
        k_obj_bins<<<wgrid8, kWarpsPerBlock * 32, 0, st>>>(items.ptr, n_items, cur, info.ptr, p.buckets, obj.ptr);
        k_obj_eval<<<grid_for(n_active, 128), 128, 0, st>>>(n_active, obj.ptr, info.ptr, p);
        k_sp_bins<<<wgrid8, kWarpsPerBlock * 32, 0, st>>>(items.ptr, n_items, cur, info.ptr, p.buckets, sp.ptr);
        k_decide<<<grid_for(n_active, 128), 128, 0, st>>>(cur_nodes->ptr, n_active, sp.ptr, info.ptr, p);
        k_sp_classes<<<wgrid, 256, 0, st>>>(items.ptr, n_items, cur, info.ptr);
        k_sp_costs<<<grid_for(n_active, 128), 128, 0, st>>>(n_active, info.ptr);
        KS_CUDA_TRY(ctx, cl.reserve(n_items));
        KS_CUDA_TRY(ctx, cr.reserve(n_items));
        KS_CUDA_TRY(ctx, cp.reserve(n_items));
        KS_CUDA_TRY(ctx, sl.reserve(n_items + 1));
        KS_CUDA_TRY(ctx, sr.reserve(n_items + 1));
        KS_CUDA_TRY(ctx, spool.reserve(n_items + 1));
        for (int pass = 0;; ++pass) {
            k_count<<<wgrid, 256, 0, st>>>(items.ptr, n_items, cur, info.ptr, p.buckets, cl.ptr, cr.ptr, cp.ptr);
            KS_CUDA_TRY(ctx, exclusive_scan(cl.ptr, sl.ptr, n_items, scan, st));
            KS_CUDA_TRY(ctx, exclusive_scan(cr.ptr, sr.ptr, n_items, scan, st));
            KS_CUDA_TRY(ctx, exclusive_scan(cp.ptr, spool.ptr, n_items, scan, st));
            KS_CUDA_TRY(ctx, cudaMemsetAsync(flag.ptr, 0, 4, st));
            k_child_counts<<<grid_for(n_active, 128), 128, 0, st>>>(n_active, item_off.ptr, sl.ptr, sr.ptr, info.ptr,
                                                                    flag.ptr);
            uint32_t changed = 0;
            KS_CUDA_TRY(ctx, cudaMemcpyAsync(&changed, flag.ptr, 4, cudaMemcpyDeviceToHost, st));
            KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
            if (!changed)
                break;
            if (pass > 0)
                return fail(ctx, KS_ERR_INVALID_ARGUMENT, "sbvh build: degenerate split could not be resolved");
        }
        KS_CUDA_TRY(ctx, split_flag.reserve(n_active));
        KS_CUDA_TRY(ctx, split_scan.reserve(n_active + 1));
        k_split_flags<<<grid_for(n_active, 256), 256, 0, st>>>(info.ptr, n_active, split_flag.ptr);
        KS_CUDA_TRY(ctx, exclusive_scan(split_flag.ptr, split_scan.ptr, n_active, scan, st));
        uint32_t totals[4] = {0, 0, 0, 0};
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(&totals[0], sl.ptr + n_items, 4, cudaMemcpyDeviceToHost, st));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(&totals[1], sr.ptr + n_items, 4, cudaMemcpyDeviceToHost, st));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(&totals[2], spool.ptr + n_items, 4, cudaMemcpyDeviceToHost, st));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(&totals[3], split_scan.ptr + n_active, 4, cudaMemcpyDeviceToHost, st));
        KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        uint32_t left_total = totals[0], right_total = totals[1], leaf_total = totals[2], n_split = totals[3];
        size_t next_refs = (size_t)left_total + right_total;
        if (next_refs > nxt_buf->count) {
            // grow the next-level buffer (contents are rewritten by the scatter)
            KS_CUDA_TRY(ctx, nxt_buf->alloc(next_refs + next_refs / 2));
            nxt = nxt_buf->ptr;
        }
        if ((size_t)pool_used + leaf_total > pool.count)
            return fail(ctx, KS_ERR_OUT_OF_MEMORY, "sbvh build: leaf pool capacity exceeded");
        k_scatter<<<wgrid, 256, 0, st>>>(items.ptr, n_items, cur, info.ptr, p.buckets, sl.ptr, sr.ptr, spool.ptr,
                                         left_total, nxt, pool_used, pool.ptr);
        KS_CUDA_TRY(ctx, nxt_nodes->reserve((size_t)2 * n_split + 1));
        uint32_t next_build_base = build_base + n_active;
        k_children<<<grid_for(n_active, 128), 128, 0, st>>>(cur_nodes->ptr, n_active, info.ptr, split_scan.ptr, n_split,
                                                            sl.ptr, sr.ptr, spool.ptr, left_total, pool_used,
                                                            next_build_base, recs.ptr, nxt_nodes->ptr);
        // the level's node list is read by k_children above; keep the swap after it
        KS_CUDA_TRY(ctx, cudaGetLastError());
        pool_used += leaf_total;
        build_base = next_build_base;
        n_active = 2 * n_split;
        n_refs = (uint32_t)next_refs;
        std::swap(cur, nxt);
        std::swap(cur_buf, nxt_buf);
        std::swap(cur_nodes, nxt_nodes);
        ++level;
        if ((uint32_t)level > (ctx->limits.sbvh_max_levels ? ctx->limits.sbvh_max_levels : 4096u))
            return fail(ctx, KS_ERR_WATCHDOG, "sbvh build: level limit reached");
    }
    (void)n_refs;
    const uint32_t n_nodes = build_base;
    level_begin.push_back(build_base);
    // subtree sizes bottom-up, DFS numbering top-down
    for (int l = (int)level_begin.size() - 2; l >= 0; --l) {
        uint32_t b = level_begin[l], e = level_begin[l + 1];
        k_subtree<<<grid_for(e - b, 256), 256, 0, st>>>(recs.ptr, b, e);
    }
    for (size_t l = 0; l + 1 < level_begin.size(); ++l) {
        uint32_t b = level_begin[l], e = level_begin[l + 1];
        k_dfs<<<grid_for(e - b, 256), 256, 0, st>>>(recs.ptr, b, e);
    }
    KS_CUDA_TRY(ctx, out.ref_nodes.alloc(n_nodes));
    KS_CUDA_TRY(ctx, out.prims.alloc(pool_used));
    auto &interior_flag = bs.interior_flag, &interior_scan = bs.interior_scan;
    KS_CUDA_TRY(ctx, interior_flag.reserve(n_nodes));
    KS_CUDA_TRY(ctx, interior_scan.reserve(n_nodes + 1));
    k_emit<<<grid_for(n_nodes, 256), 256, 0, st>>>(recs.ptr, n_nodes, pool.ptr, out.ref_nodes.ptr, out.prims.ptr,
                                                   interior_flag.ptr);
    KS_CUDA_TRY(ctx, exclusive_scan(interior_flag.ptr, interior_scan.ptr, n_nodes, scan, st));
    uint32_t n_trav = 0;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(&n_trav, interior_scan.ptr + n_nodes, 4, cudaMemcpyDeviceToHost, st));
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    KS_CUDA_TRY(ctx, out.trav.alloc(n_trav > 0 ? n_trav : 1));
    k_trav<<<grid_for(n_nodes, 256), 256, 0, st>>>(recs.ptr, n_nodes, interior_scan.ptr, out.trav.ptr);
    KS_CUDA_TRY(ctx, out.prim_tris.alloc((size_t)pool_used * 3));
    k_prim_tris<<<grid_for(pool_used, 256), 256, 0, st>>>(out.prims.ptr, pool_used, verts, indices,
                                                          out.prim_tris.ptr);
    KS_CUDA_TRY(ctx, cudaGetLastError());
    if (done)
        KS_CUDA_TRY(ctx, cudaEventRecord(done, st));
    RefNode root_node;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(&root_node, out.ref_nodes.ptr, sizeof(RefNode), cudaMemcpyDeviceToHost, st));
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    for (int k = 0; k < 3; ++k) {
        out.bound[k] = root_node.bmin[k];
        out.bound[3 + k] = root_node.bmax[k];
    }
    out.n_nodes = n_nodes;
    out.n_prims = pool_used;
    out.n_trav = n_trav;
    return KS_OK;
}

// BLAS concatenation: interior refs move by the node base, leaf refs by the slot base.
// Wide node i from interior node i: its leaf children as they are, its interior children replaced
// by their two children (boxes and refs read from the child's node).
__global__ void k_widen(const TravNode *nodes, uint32_t n, WideNode *wide)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    float lo[3][4], hi[3][4];
    uint32_t ref[4], cnt[4];
    for (int k = 0; k < 4; ++k) {
        for (int a = 0; a < 3; ++a) {
            lo[a][k] = __int_as_float(0x7f800000);  // +inf
            hi[a][k] = __int_as_float(0xff800000);  // -inf
        }
        ref[k] = kLeafBit;
        cnt[k] = 0;
    }
    int m = 0;
    auto put = [&](const TravNode &nd, int side) {
        const float4 A = nd.a, B = nd.b, C = nd.c;
        const float l0[3] = {A.x, A.y, A.z}, h0[3] = {A.w, B.x, B.y};
        const float l1[3] = {B.z, B.w, C.x}, h1[3] = {C.y, C.z, C.w};
        for (int a = 0; a < 3; ++a) {
            lo[a][m] = side ? l1[a] : l0[a];
            hi[a][m] = side ? h1[a] : h0[a];
        }
        ref[m] = side ? nd.d.y : nd.d.x;
        cnt[m] = side ? nd.d.w : (nd.d.z & 0x3fffffffu);
        ++m;
    };
    const TravNode nd = nodes[i];
    for (int side = 0; side < 2; ++side) {
        const uint32_t r = side ? nd.d.y : nd.d.x;
        if (r & kLeafBit) {
            put(nd, side);
        } else {
            const TravNode c = nodes[r];
            put(c, 0);
            put(c, 1);
        }
    }
    WideNode w;
    for (int a = 0; a < 3; ++a) {
        w.lo[a] = make_float4(lo[a][0], lo[a][1], lo[a][2], lo[a][3]);
        w.hi[a] = make_float4(hi[a][0], hi[a][1], hi[a][2], hi[a][3]);
    }
    w.ref = make_uint4(ref[0], ref[1], ref[2], ref[3]);
    w.cnt = make_uint4(cnt[0], cnt[1], cnt[2], cnt[3]);
    wide[i] = w;
}

__global__ void k_offset_trav(const TravNode *src, uint32_t n, uint32_t node_base, uint32_t slot_base, TravNode *dst)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    TravNode t = src[i];
    t.d.x = (t.d.x & kLeafBit) ? (kLeafBit | ((t.d.x & ~kLeafBit) + slot_base)) : t.d.x + node_base;
    t.d.y = (t.d.y & kLeafBit) ? (kLeafBit | ((t.d.y & ~kLeafBit) + slot_base)) : t.d.y + node_base;
    dst[i] = t;
}

// ---- TLAS over instance boxes (host, binned SAH; leaves of at most 2 instances) ---------------
struct InstBox
{
    float lo[3], hi[3], c[3];
    uint32_t id;
};

struct TlasBuilder
{
    std::vector<InstBox> items;
    std::vector<TravNode> nodes;

    static void unite(float *lo, float *hi, const InstBox &b)
    {
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], b.lo[k]);
            hi[k] = std::max(hi[k], b.hi[k]);
        }
    }
    static float area(const float *lo, const float *hi)
    {
        float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.0f * (dx * dy + dy * dz + dz * dx);
    }
    // returns (ref, count); box of the subtree in lo/hi
    std::pair<uint32_t, uint32_t> build(uint32_t b, uint32_t e, float *lo, float *hi)
    {
        for (int k = 0; k < 3; ++k) {
            lo[k] = kInf;
            hi[k] = -kInf;
        }
        for (uint32_t i = b; i < e; ++i)
            unite(lo, hi, items[i]);
        if (e - b <= 2)
            return {kLeafBit | b, e - b};
        float clo[3] = {kInf, kInf, kInf}, chi[3] = {-kInf, -kInf, -kInf};
        for (uint32_t i = b; i < e; ++i)
            for (int k = 0; k < 3; ++k) {
                clo[k] = std::min(clo[k], items[i].c[k]);
                chi[k] = std::max(chi[k], items[i].c[k]);
            }
        int axis = 0;
        for (int k = 1; k < 3; ++k)
            if (chi[k] - clo[k] > chi[axis] - clo[axis])
                axis = k;
        uint32_t mid = (b + e) / 2;
        float ext = chi[axis] - clo[axis];
        if (ext > 0.0f) {
            constexpr int kBins = 12;
            float blo[kBins][3], bhi[kBins][3];
            uint32_t bcnt[kBins] = {};
            for (int q = 0; q < kBins; ++q)
                for (int k = 0; k < 3; ++k) {
                    blo[q][k] = kInf;
                    bhi[q][k] = -kInf;
                }
            auto bin_of = [&](const InstBox &x) {
                int q = (int)((x.c[axis] - clo[axis]) / ext * kBins);
                return std::min(std::max(q, 0), kBins - 1);
            };
            for (uint32_t i = b; i < e; ++i) {
                int q = bin_of(items[i]);
                ++bcnt[q];
                unite(blo[q], bhi[q], items[i]);
            }
            float best = kInf;
            int best_q = -1;
            for (int q = 1; q < kBins; ++q) {
                float llo[3] = {kInf, kInf, kInf}, lhi[3] = {-kInf, -kInf, -kInf};
                float rlo[3] = {kInf, kInf, kInf}, rhi[3] = {-kInf, -kInf, -kInf};
                uint32_t nl = 0, nr = 0;
                for (int j = 0; j < kBins; ++j) {
                    if (!bcnt[j])
                        continue;
                    float *L = j < q ? llo : rlo, *H = j < q ? lhi : rhi;
                    for (int k = 0; k < 3; ++k) {
                        L[k] = std::min(L[k], blo[j][k]);
                        H[k] = std::max(H[k], bhi[j][k]);
                    }
                    (j < q ? nl : nr) += bcnt[j];
                }
                if (!nl || !nr)
                    continue;
                float cost = area(llo, lhi) * nl + area(rlo, rhi) * nr;
                if (cost < best) {
                    best = cost;
                    best_q = q;
                }
            }
            if (best_q > 0) {
                auto it = std::partition(items.begin() + b, items.begin() + e,
                                         [&](const InstBox &x) { return bin_of(x) < best_q; });
                mid = (uint32_t)(it - items.begin());
            }
        }
        if (mid == b || mid == e) {
            mid = (b + e) / 2;
            std::nth_element(items.begin() + b, items.begin() + mid, items.begin() + e,
                             [&](const InstBox &x, const InstBox &y) { return x.c[axis] < y.c[axis]; });
        }
        uint32_t me = (uint32_t)nodes.size();
        nodes.emplace_back();
        float llo[3], lhi[3], rlo[3], rhi[3];
        auto L = build(b, mid, llo, lhi);
        auto R = build(mid, e, rlo, rhi);
        TravNode &n = nodes[me];
        n.a = make_float4(llo[0], llo[1], llo[2], lhi[0]);
        n.b = make_float4(lhi[1], lhi[2], rlo[0], rlo[1]);
        n.c = make_float4(rlo[2], rhi[0], rhi[1], rhi[2]);
        n.d = make_uint4(L.first, R.first, L.second | ((uint32_t)axis << 30), R.second);
        return {me, 0u};
    }
};

static ks_status build_instanced(ks_scene *scene, const Params &p)
{
    ks_context *ctx = scene->ctx;
    cudaStream_t st = ctx->stream;
    const SceneHost &h = scene->host;
    const uint32_t n_protos = scene->n_protos;
    std::vector<RangeOut> blas(n_protos);
    uint32_t total_trav = 0, total_slots = 0;
    for (uint32_t q = 0; q < n_protos; ++q) {
        uint32_t b = h.proto_tri_begin[q], n = h.proto_tri_end[q] - b;
        ks_status s = build_range(ctx, scene->verts.ptr, scene->indices.ptr, b, n, p, blas[q]);
        if (s != KS_OK)
            return s;
        total_trav += blas[q].n_trav;
        total_slots += blas[q].n_prims;
    }
    KS_CUDA_TRY(ctx, scene->trav_nodes.alloc(total_trav > 0 ? total_trav : 1));
    KS_CUDA_TRY(ctx, scene->prim_tris.alloc((size_t)total_slots * 3));
    std::vector<uint4> roots(n_protos);
    std::vector<float> pbound(6 * (size_t)n_protos);
    uint32_t node_base = 0, slot_base = 0;
    for (uint32_t q = 0; q < n_protos; ++q) {
        const RangeOut &r = blas[q];
        if (r.n_trav)
            k_offset_trav<<<grid_for(r.n_trav, 256), 256, 0, st>>>(r.trav.ptr, r.n_trav, node_base, slot_base,
                                                                  scene->trav_nodes.ptr + node_base);
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(scene->prim_tris.ptr + 3 * (size_t)slot_base, r.prim_tris.ptr,
                                         sizeof(float4) * 3 * (size_t)r.n_prims, cudaMemcpyDeviceToDevice, st));
        roots[q] = make_uint4(r.n_trav ? node_base : (kLeafBit | slot_base), r.n_prims, 0, 0);
        std::memcpy(&pbound[6 * (size_t)q], r.bound, sizeof(r.bound));
        node_base += r.n_trav;
        slot_base += r.n_prims;
    }
    KS_CUDA_TRY(ctx, cudaGetLastError());
    // the renderer's 4-wide view of the concatenated BLAS nodes (their refs are already global)
    KS_CUDA_TRY(ctx, scene->wide_nodes.alloc(total_trav > 0 ? total_trav : 1));
    if (total_trav > 0)
        k_widen<<<grid_for(total_trav, 256), 256, 0, st>>>(scene->trav_nodes.ptr, total_trav, scene->wide_nodes.ptr);
    // instance boxes: the 8 corners of the prototype box, transformed, padded by a relative epsilon
    TlasBuilder tb;
    for (uint32_t i = 0; i < scene->n_instances; ++i) {
        const float *xf = &h.inst_xf[12 * (size_t)i];
        const float *pb = &pbound[6 * (size_t)h.inst_proto[i]];
        InstBox ib{{kInf, kInf, kInf}, {-kInf, -kInf, -kInf}, {0, 0, 0}, i};
        for (int c = 0; c < 8; ++c) {
            f3 corner = mk(pb[(c & 1) ? 3 : 0], pb[(c & 2) ? 4 : 1], pb[(c & 4) ? 5 : 2]);
            f3 w = xf_point(xf, corner);
            float wv[3] = {w.x, w.y, w.z};
            for (int k = 0; k < 3; ++k) {
                ib.lo[k] = std::min(ib.lo[k], wv[k]);
                ib.hi[k] = std::max(ib.hi[k], wv[k]);
            }
        }
        for (int k = 0; k < 3; ++k) {
            float pad = 1e-6f * (ib.hi[k] - ib.lo[k] + std::fabs(ib.lo[k]) + std::fabs(ib.hi[k])) + 1e-30f;
            ib.lo[k] -= pad;
            ib.hi[k] += pad;
            ib.c[k] = 0.5f * (ib.lo[k] + ib.hi[k]);
        }
        tb.items.push_back(ib);
    }
    float lo[3], hi[3];
    auto root = tb.build(0, (uint32_t)tb.items.size(), lo, hi);
    std::vector<uint32_t> items(tb.items.size());
    for (size_t k = 0; k < items.size(); ++k)
        items[k] = tb.items[k].id;
    KS_CUDA_TRY(ctx, scene->tlas_nodes.alloc(std::max<size_t>(tb.nodes.size(), 1)));
    KS_CUDA_TRY(ctx, scene->tlas_items.alloc(items.size()));
    KS_CUDA_TRY(ctx, scene->proto_root.alloc(n_protos));
    KS_CUDA_TRY(ctx, scene->proto_bound.alloc(pbound.size()));
    if (!tb.nodes.empty())
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(scene->tlas_nodes.ptr, tb.nodes.data(), sizeof(TravNode) * tb.nodes.size(),
                                         cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(scene->tlas_items.ptr, items.data(), sizeof(uint32_t) * items.size(),
                                     cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(scene->proto_root.ptr, roots.data(), sizeof(uint4) * roots.size(),
                                     cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(scene->proto_bound.ptr, pbound.data(), sizeof(float) * pbound.size(),
                                     cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    scene->tlas_root_ref = root.first;
    scene->tlas_root_count = root.second;
    for (int k = 0; k < 3; ++k) {
        scene->scene_bound[k] = lo[k];
        scene->scene_bound[3 + k] = hi[k];
    }
    scene->ref_nodes.release();
    scene->prims.release();
    scene->n_nodes = 0;
    scene->n_prims = total_slots;
    scene->n_trav = total_trav;
    scene->root_ref = 0;
    scene->root_count = 0;
    return KS_OK;
}

ks_status build_sbvh(ks_scene *scene, const ks_sbvh_options &o, float *build_ms)
{
    ks_context *ctx = scene->ctx;
    cudaStream_t st = ctx->stream;
    Params p;
    // option clamps (cuda/sbvh.cu:411-414)
    p.max_prims = std::min(o.max_prims_in_node, 8u);
    p.buckets = std::min(o.bucket_count, 16u);
    p.trav_weight = std::clamp(o.trav_weight, 0.0f, 10.0f);
    p.alpha = std::clamp(o.alpha, 0.0f, 1.0f);
    if (p.buckets < 2)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_build_bvh: bucket_count must be >= 2");
    if (scene->n_tris == 0)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_build_bvh: scene has no triangles");
    cudaEvent_t ev0, ev1, ev2, ev3;
    KS_CUDA_TRY(ctx, cudaEventCreate(&ev0));
    KS_CUDA_TRY(ctx, cudaEventCreate(&ev1));
    KS_CUDA_TRY(ctx, cudaEventCreate(&ev2));
    KS_CUDA_TRY(ctx, cudaEventCreate(&ev3));
    bool widened = false;
    KS_CUDA_TRY(ctx, cudaEventRecord(ev0, st));
    ks_status s = KS_OK;
    if (scene->n_instances > 0) {
        s = build_instanced(scene, p);
        if (s == KS_OK)
            cudaEventRecord(ev1, st);
    } else {
        RangeOut r;
        s = build_range(ctx, scene->verts.ptr, scene->indices.ptr, 0, scene->n_tris, p, r, ev1);
        if (s == KS_OK) {
            scene->ref_nodes.swap(r.ref_nodes);
            scene->prims.swap(r.prims);
            scene->trav_nodes.swap(r.trav);
            scene->prim_tris.swap(r.prim_tris);
            std::memcpy(scene->scene_bound, r.bound, sizeof(r.bound));
            scene->n_nodes = r.n_nodes;
            scene->n_prims = r.n_prims;
            scene->n_trav = r.n_trav;
            scene->root_count = r.n_prims;
            scene->root_ref = r.n_trav > 0 ? 0u : kLeafBit;
            // the renderer's 4-wide view of the tree (timed with the build)
            if (scene->wide_nodes.alloc(r.n_trav > 0 ? r.n_trav : 1) != cudaSuccess) {
                s = fail(ctx, KS_ERR_OUT_OF_MEMORY, "ks_scene_build_bvh: wide nodes");
            } else if (r.n_trav > 0) {
                cudaEventRecord(ev2, st);
                k_widen<<<grid_for(r.n_trav, 256), 256, 0, st>>>(scene->trav_nodes.ptr, r.n_trav,
                                                                  scene->wide_nodes.ptr);
                cudaEventRecord(ev3, st);
                widened = true;
            }
        }
    }
    float ms = 0;
    if (s == KS_OK) {
        cudaEventSynchronize(ev1);
        cudaEventElapsedTime(&ms, ev0, ev1);
        if (widened) {
            float mw = 0;
            cudaEventSynchronize(ev3);
            cudaEventElapsedTime(&mw, ev2, ev3);
            ms += mw;
        }
    } else {
        // a build that stopped early leaves its work on the stream: let it finish before the
        // scratch is reused, and keep no error of it for the next call
        cudaStreamSynchronize(st);
        cudaGetLastError();
    }
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    cudaEventDestroy(ev2);
    cudaEventDestroy(ev3);
    if (s != KS_OK)
        return s;
    if (build_ms)
        *build_ms = ms;
    scene->bvh_built = true;
    return KS_OK;
}

} // namespace ksb
