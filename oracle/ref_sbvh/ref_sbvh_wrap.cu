// Test-only C wrapper around the reference's own SBVH (cuda/sbvh.cu, cuda/sbvh.cuh),
// compiled unmodified from the reference tree by oracle/ref_sbvh/Makefile.
//
// This file is part of the parity oracle, never of the product.  It exposes:
//   * the reference builder  ksc::SBVH::SBVH(option, vertices, indices)   (cuda/sbvh.cu:396-440)
//   * the flattened node array and the ordered primitive list             (cuda/sbvh.cuh:18-28,90-93)
//   * closest-hit and any-hit queries ksc::SBVH::intersect / intersectBool (cuda/sbvh.cu:512-603)
// so that tests can pin the CUDA builder's topology and the CUDA traversal's hit IDs
// against the reference itself.
#include "ray_tri.cuh"
#include "sbvh.cuh"

#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace
{
struct RefHandle
{
    std::vector<ksc::vec3> verts;
    std::vector<uint32_t> idx;
    ksc::SBVH bvh;
};
} // namespace

extern "C" {

int ksref_sbvh_build(const float *vertices, uint32_t n_vertices, const uint32_t *indices, uint32_t n_tris,
                     uint32_t max_prims_in_node, uint32_t bucket_count, float trav_weight, float alpha,
                     void **out_handle, uint32_t *out_n_nodes, uint32_t *out_n_prims)
{
    if (!vertices || !indices || !out_handle || n_tris == 0)
        return 1;
    auto *h = new RefHandle();
    h->verts.resize(n_vertices);
    for (uint32_t i = 0; i < n_vertices; ++i)
        h->verts[i] = ksc::vec3(vertices[3 * i + 0], vertices[3 * i + 1], vertices[3 * i + 2]);
    h->idx.assign(indices, indices + 3 * (size_t)n_tris);
    ksc::SBVHBuildOption opt;
    opt.maxPrimsInNode = max_prims_in_node;
    opt.bucketCount = bucket_count;
    opt.travWeight = trav_weight;
    opt.alpha = alpha;
    h->bvh = ksc::SBVH(opt, ksc::span<const ksc::vec3>(h->verts.data(), h->verts.size()),
                       ksc::span<const uint32_t>(h->idx.data(), h->idx.size()));
    *out_handle = h;
    *out_n_nodes = (uint32_t)h->bvh.nodes.size;
    *out_n_prims = (uint32_t)h->bvh.primitives.size;
    return 0;
}

// node_bounds: 6 floats per node (min xyz, max xyz); axis/right/prim_offset: one uint32 per node;
// prims: ordered primitive (triangle) indices.
int ksref_sbvh_export(void *handle, float *node_bounds, uint32_t *node_axis, uint32_t *node_right,
                      uint32_t *node_prim_offset, uint32_t *prims)
{
    auto *h = (RefHandle *)handle;
    for (size_t i = 0; i < h->bvh.nodes.size; ++i) {
        const ksc::SBVHNode &n = h->bvh.nodes[i];
        node_bounds[6 * i + 0] = n.bound.min.x;
        node_bounds[6 * i + 1] = n.bound.min.y;
        node_bounds[6 * i + 2] = n.bound.min.z;
        node_bounds[6 * i + 3] = n.bound.max.x;
        node_bounds[6 * i + 4] = n.bound.max.y;
        node_bounds[6 * i + 5] = n.bound.max.z;
        node_axis[i] = n.splitAxis;
        node_right[i] = n.rightChildOffset;
        node_prim_offset[i] = n.primOffset;
    }
    for (size_t i = 0; i < h->bvh.primitives.size; ++i)
        prims[i] = h->bvh.primitives[i].shapeIndex;
    return 0;
}

// rays: 8 floats per ray (ox oy oz tmin dx dy dz tmax).  any_hit=0: closest hit, writes tri index
// (~0u on miss), t and the three barycentric weights; any_hit=1: writes 1/0 in tri_idx.
// culling: 0 back-face, 1 front-face, 2 none (ksc::SBVHCulling).
int ksref_sbvh_intersect(void *handle, const float *rays, uint32_t n, int any_hit, int culling, uint32_t *tri_idx,
                         float *t, float *bary, int n_threads)
{
    auto *h = (RefHandle *)handle;
    ksc::SBVHIsectOption opt;
    opt.culling = (ksc::SBVHCulling)culling;
    auto work = [&](uint32_t begin, uint32_t end) {
        for (uint32_t i = begin; i < end; ++i) {
            const float *r = rays + 8 * (size_t)i;
            ksc::Ray ray(ksc::vec3(r[0], r[1], r[2]), ksc::vec3(r[4], r[5], r[6]), r[3], r[7]);
            if (any_hit) {
                tri_idx[i] = h->bvh.intersectBool(ray, opt) ? 1u : 0u;
            } else {
                ksc::SBVHIsectRecord rec = h->bvh.intersect(ray, opt);
                tri_idx[i] = rec.tri_idx;
                if (t)
                    t[i] = rec.thit;
                if (bary) {
                    bary[3 * i + 0] = rec.coord.x;
                    bary[3 * i + 1] = rec.coord.y;
                    bary[3 * i + 2] = rec.coord.z;
                }
            }
        }
    };
    if (n_threads <= 1 || n < 4096) {
        work(0, n);
    } else {
        std::vector<std::thread> pool;
        uint32_t chunk = (n + n_threads - 1) / n_threads;
        for (int k = 0; k < n_threads; ++k) {
            uint32_t b = k * chunk, e = std::min(n, b + chunk);
            if (b < e)
                pool.emplace_back(work, b, e);
        }
        for (auto &th : pool)
            th.join();
    }
    return 0;
}

// One ray (8 floats as above).  Returns the triangle index (~0u on miss) or, for any_hit, 1/0.
uint32_t ksref_sbvh_intersect1(void *handle, const float *r, int any_hit, float *t, float *bary)
{
    auto *h = (RefHandle *)handle;
    ksc::SBVHIsectOption opt;
    opt.culling = ksc::SBVHCulling::None;
    ksc::Ray ray(ksc::vec3(r[0], r[1], r[2]), ksc::vec3(r[4], r[5], r[6]), r[3], r[7]);
    if (any_hit)
        return h->bvh.intersectBool(ray, opt) ? 1u : 0u;
    ksc::SBVHIsectRecord rec = h->bvh.intersect(ray, opt);
    if (rec.tri_idx != ~0u) {
        *t = rec.thit;
        bary[0] = rec.coord.x;
        bary[1] = rec.coord.y;
        bary[2] = rec.coord.z;
    }
    return rec.tri_idx;
}

// SBVH::intersect / intersectBool (cuda/sbvh.cu:512-603) restated over the reference's own node and
// primitive arrays, with the same bound and triangle tests (isect_ray_aabb with RayBoundHelper,
// cuda/aabb.cuh:155-252; the culling check and isect_ray_tri of IsectQuery, cuda/sbvh.cu:485-504)
// in the same order, counting the work of the query: counts[0] += nodes whose bound is tested,
// counts[1] += triangles tested.  These are the algorithmic units of a query (32-byte nodes,
// triangles of three vertices + an index triple).  The stack holds 64 entries like the reference's;
// a deeper push ends the query and sets counts[2].  Returns what ksref_sbvh_intersect1 returns.
// filter (may be NULL): a candidate hit on triangle tri at barycentrics (u, v) of vertices 1 and 2
// counts only when filter(user, tri, u, v) is nonzero (the role of Embree's intersection filter,
// scene.cpp:175-208, which the reference's own SBVH queries do not have).
typedef int (*ksref_filter_fn)(void *user, uint32_t tri, float u, float v);
uint32_t ksref_sbvh_intersect1_counted(void *handle, const float *r, int any_hit, int culling, float *t, float *bary,
                                       uint64_t *counts, ksref_filter_fn filter, void *user)
{
    auto *h = (RefHandle *)handle;
    const ksc::SBVH &b = h->bvh;
    ksc::Ray ray(ksc::vec3(r[0], r[1], r[2]), ksc::vec3(r[4], r[5], r[6]), r[3], r[7]);
    const ksc::RayBoundHelper rb(ray);
    const ksc::RayTriHelper rt(ray);
    const ksc::SBVHCulling cull = (ksc::SBVHCulling)culling;
    auto tri_test = [&](uint32_t tri, ksc::RayTriIsect *isect) {
        auto v = b.tri_verts(tri);
        float check = ksc::dot(ray.dir, ksc::cross(v[1] - v[0], v[2] - v[1]));
        if (check >= 0.0f && cull == ksc::SBVHCulling::CullBackface)
            return false;
        if (check <= 0.0f && cull == ksc::SBVHCulling::CullFrontFace)
            return false;
        return ksc::isect_ray_tri(ray, rt, v[0], v[1], v[2], isect);
    };
    uint32_t stack_node[64], stack_cnt[64];
    int sp = 0;
    uint32_t node_i = 0, cnt = (uint32_t)b.primitives.size, result = ~0u;
    float thit = 0.0f;
    ksc::vec3 coord(0.0f);
    while (true) {
        const ksc::SBVHNode &node = b.nodes[node_i];
        ++counts[0];
        bool pop = false;
        if (!ksc::isect_ray_aabb(ray, node.bound, rb)) {
            pop = true;
        } else if (node.is_leaf()) {
            for (uint32_t i = 0; i < cnt; ++i) {
                const uint32_t tri = b.primitives[i + node.primOffset].shapeIndex;
                ++counts[1];
                ksc::RayTriIsect isect;
                if (any_hit) {
                    if (tri_test(tri, &isect) && (!filter || filter(user, tri, isect.coord.y, isect.coord.z)))
                        return 1u;
                } else if (tri_test(tri, &isect) && isect.tHit < ray.tmax &&
                           (!filter || filter(user, tri, isect.coord.y, isect.coord.z))) {
                    ray.tmax = isect.tHit;
                    thit = isect.tHit;
                    coord = isect.coord;
                    result = tri;
                }
            }
            pop = true;
        } else {
            const uint32_t right = node.rightChildOffset;
            const uint32_t left_cnt = b.nodes[right].primOffset - node.primOffset, right_cnt = cnt - left_cnt;
            if (sp == 64) {
                counts[2] = 1;
                break;
            }
            if (rb.dir_is_neg[node.splitAxis]) {
                stack_node[sp] = node_i + 1;
                stack_cnt[sp++] = left_cnt;
                node_i = right;
                cnt = right_cnt;
            } else {
                stack_node[sp] = right;
                stack_cnt[sp++] = right_cnt;
                node_i = node_i + 1;
                cnt = left_cnt;
            }
        }
        if (pop) {
            if (sp == 0)
                break;
            --sp;
            node_i = stack_node[sp];
            cnt = stack_cnt[sp];
        }
    }
    if (any_hit)
        return 0u;
    if (result != ~0u) {
        *t = thit;
        bary[0] = coord.x;
        bary[1] = coord.y;
        bary[2] = coord.z;
    }
    return result;
}

// The reference's own watertight ray/triangle test (cuda/ray_tri.cuh:46-97, through the query of
// cuda/sbvh.cu with culling off) of triangle tri[i] against ray i over the ray's [tmin, tmax]:
// hit[i] = 1 and t[i] = its distance on a hit, else hit[i] = 0.  Used to prove a hit-id
// difference a tie: the other triangle is a candidate of the reference at (nearly) the same t.
void ksref_tri_test(void *handle, const float *rays, const uint32_t *tri, uint32_t n, float *t, uint32_t *hit)
{
    auto *h = (RefHandle *)handle;
    for (uint32_t i = 0; i < n; ++i) {
        const float *r = rays + 8 * (size_t)i;
        ksc::Ray ray(ksc::vec3(r[0], r[1], r[2]), ksc::vec3(r[4], r[5], r[6]), r[3], r[7]);
        ksc::RayTriHelper help(ray);
        auto v = h->bvh.tri_verts(tri[i]);
        ksc::RayTriIsect isect;
        hit[i] = ksc::isect_ray_tri(ray, help, v[0], v[1], v[2], &isect) ? 1u : 0u;
        t[i] = hit[i] ? isect.tHit : 0.0f;
    }
}

// Root bounds (min xyz, max xyz).
void ksref_sbvh_bound(void *handle, float *out)
{
    auto *h = (RefHandle *)handle;
    ksc::AABB3 b = h->bvh.bound();
    out[0] = b.min.x;
    out[1] = b.min.y;
    out[2] = b.min.z;
    out[3] = b.max.x;
    out[4] = b.max.y;
    out[5] = b.max.z;
}

void ksref_sbvh_destroy(void *handle) { delete (RefHandle *)handle; }

} // extern "C"
