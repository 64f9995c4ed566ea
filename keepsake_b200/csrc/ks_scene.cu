// Scene lifetime, SBVH build/export entry points and the ray-query parity kernel.
#include "ks_lights.cuh"
#include "ks_scene.h"
#include "ks_traverse.cuh"

#include <atomic>
#include <cmath>

#include <cstring>
#include <new>

using namespace ksb;

namespace ksb
{
SceneView make_view(const ks_scene *s);
}

namespace
{

__global__ void trace_kernel(const TravNode *nodes, const float4 *tris, uint32_t root_ref, uint32_t root_count,
                             float bx0, float by0, float bz0, float bx1, float by1, float bz1, const float *rays,
                             uint32_t n, int any_hit, int culling, uint32_t *tri_out, float *t_out, float *bary_out,
                             int *overflow_flag, InstanceView iv)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float *r = rays + 8 * (size_t)i;
    RayQuery q;
    q.o = mk(r[0], r[1], r[2]);
    q.tmin = r[3];
    q.d = mk(r[4], r[5], r[6]);
    q.tmax = r[7];
    const float bmin[3] = {bx0, by0, bz0}, bmax[3] = {bx1, by1, bz1};
    Hit h;
    int overflow = 0;
    uint32_t inst = 0;
    if (any_hit) {
        bool occ = iv.n ? traverse_instances<true>(nodes, tris, iv, q, culling, h, inst, overflow)
                        : traverse<true>(nodes, tris, root_ref, root_count, bmin, bmax, q, culling, h, overflow);
        tri_out[i] = occ ? 1u : 0u;
    } else {
        if (iv.n)
            traverse_instances<false>(nodes, tris, iv, q, culling, h, inst, overflow);
        else
            traverse<false>(nodes, tris, root_ref, root_count, bmin, bmax, q, culling, h, overflow);
        tri_out[i] = h.tri;
        if (h.tri != ~0u) {
            t_out[i] = h.t;
            bary_out[3 * i + 0] = h.b0;
            bary_out[3 * i + 1] = h.b1;
            bary_out[3 * i + 2] = h.b2;
        } else {
            t_out[i] = -kInf;
            bary_out[3 * i + 0] = bary_out[3 * i + 1] = bary_out[3 * i + 2] = 0.0f;
        }
    }
    if (overflow)
        atomicOr(overflow_flag, 1);
}

// ks_trace_rays for flat scenes: the same queries as trace_kernel, traversed by trav_step with
// dynamic ray fetch.  Node = TravNode: each ray makes the same tests as traverse() (same triangle, t
// and barycentrics); Node = WideNode (ks_trace_rays_wide): the renderer's 4-wide traversal.
template <class Node>
__global__ void __launch_bounds__(128) trace_kernel_pt(const Node *nodes, const float4 *tris, uint32_t root_ref,
                                                       uint32_t root_count, float bx0, float by0, float bz0, float bx1,
                                                       float by1, float bz1, const float *rays, uint32_t n, int any_hit,
                                                       int culling, uint32_t *tri_out, float *t_out, float *bary_out,
                                                       int *overflow_flag, uint32_t *fetch)
{
    const float bmin[3] = {bx0, by0, bz0}, bmax[3] = {bx1, by1, bz1};
    KS_TRAV_STACK(stack);
    TravState s;
    uint32_t ray = ~0u;
    bool drained = false;
    int overflow = 0;
    auto finish = [&](uint32_t i, const Hit &h) {
        if (any_hit) {
            tri_out[i] = h.tri != ~0u ? 1u : 0u;
            return;
        }
        tri_out[i] = h.tri;
        t_out[i] = h.tri != ~0u ? h.t : -kInf;
        bary_out[3 * i + 0] = h.tri != ~0u ? h.b0 : 0.0f;
        bary_out[3 * i + 1] = h.tri != ~0u ? h.b1 : 0.0f;
        bary_out[3 * i + 2] = h.tri != ~0u ? h.b2 : 0.0f;
    };
    while (true) {
        const uint32_t id = warp_fetch(fetch, n, ray == ~0u, drained);
        if (id != ~0u) {
            const float *r = rays + 8 * (size_t)id;
            RayQuery q;
            q.o = mk(r[0], r[1], r[2]);
            q.tmin = r[3];
            q.d = mk(r[4], r[5], r[6]);
            q.tmax = r[7];
            if (trav_begin(s, q, root_ref, root_count, bmin, bmax))
                ray = id;
            else
                finish(id, s.hit);
        }
        if (__ballot_sync(0xffffffffu, ray != ~0u) == 0) {
            if (drained)
                break;
            continue;
        }
        while (true) {
            const bool done =
                any_hit ? trav_warp_step<true>(nodes, tris, s, stack, culling, overflow, nullptr, ray != ~0u)
                        : trav_warp_step<false>(nodes, tris, s, stack, culling, overflow, nullptr, ray != ~0u);
            if (done) {
                finish(ray, s.hit);
                ray = ~0u;
            }
            const int n_idle = __popc(__ballot_sync(0xffffffffu, ray == ~0u));
            if (n_idle == 32 || (!drained && n_idle >= KS_TRAV_REFILL))
                break;
        }
    }
    if (overflow)
        atomicOr(overflow_flag, 1);
}

// ks_trace_rays_wide for instanced scenes: the renderer's persistent two-level traversal
// (inst_step over the 4-wide view of the BLAS nodes).
__global__ void __launch_bounds__(128) trace_inst_kernel_pt(const WideNode *nodes, const float4 *tris,
                                                            InstanceView iv, const float *rays, uint32_t n,
                                                            int any_hit, int culling, uint32_t *tri_out,
                                                            float *t_out, float *bary_out, int *overflow_flag,
                                                            uint32_t *fetch)
{
    KS_TRAV_STACK(stack);
    InstTravState s;
    uint4 tstack[kTlasStackDepth];
    uint32_t ray = ~0u;
    bool drained = false;
    int overflow = 0;
    auto finish = [&](uint32_t i, const Hit &h) {
        if (any_hit) {
            tri_out[i] = h.tri != ~0u ? 1u : 0u;
            return;
        }
        tri_out[i] = h.tri;
        t_out[i] = h.tri != ~0u ? h.t : -kInf;
        bary_out[3 * i + 0] = h.tri != ~0u ? h.b0 : 0.0f;
        bary_out[3 * i + 1] = h.tri != ~0u ? h.b1 : 0.0f;
        bary_out[3 * i + 2] = h.tri != ~0u ? h.b2 : 0.0f;
    };
    while (true) {
        const uint32_t id = warp_fetch(fetch, n, ray == ~0u, drained);
        if (id != ~0u) {
            const float *r = rays + 8 * (size_t)id;
            RayQuery q;
            q.o = mk(r[0], r[1], r[2]);
            q.tmin = r[3];
            q.d = mk(r[4], r[5], r[6]);
            q.tmax = r[7];
            if (inst_begin(s, iv, q))
                ray = id;
            else
                finish(id, s.hit);
        }
        if (__ballot_sync(0xffffffffu, ray != ~0u) == 0) {
            if (drained)
                break;
            continue;
        }
        while (true) {
            if (ray != ~0u) {
                const bool done = any_hit ? inst_step<true>(nodes, tris, iv, s, tstack, stack, culling, overflow, nullptr)
                                          : inst_step<false>(nodes, tris, iv, s, tstack, stack, culling, overflow, nullptr);
                if (done) {
                    finish(ray, s.hit);
                    ray = ~0u;
                }
            }
            const int n_idle = __popc(__ballot_sync(0xffffffffu, ray == ~0u));
            if (n_idle == 32 || (!drained && n_idle >= KS_TRAV_REFILL))
                break;
        }
    }
    if (overflow)
        atomicOr(overflow_flag, 1);
}

bool valid_material(const ks_material_desc &m)
{
    auto finite = [](float x) { return x == x && x < 3.0e38f && x > -3.0e38f; };
    for (int c = 0; c < 3; ++c)
        if (!finite(m.basecolor[c]) || !finite(m.emission[c]))
            return false;
    if (!(finite(m.roughness) && finite(m.metallic) && finite(m.ior) && finite(m.specular_r0_mul) &&
          finite(m.specular_trans) && finite(m.diffuse_trans) && finite(m.diffuse_trans_fwd) && finite(m.specular)))
        return false;
    if (m.has_subsurface < 0 || m.has_subsurface > 1)
        return false;
    if (m.has_subsurface) {
        for (int c = 0; c < 3; ++c)
            if (!finite(m.ss_albedo[c]) || !finite(m.ss_radius[c]) || !(m.ss_radius[c] >= 0.0f))
                return false;
        if (!(m.ss_anisotropy > -1.0f && m.ss_anisotropy < 1.0f) || !(m.ss_ior > 0.0f) || !finite(m.ss_ior) ||
            !(m.ss_rfr_entry_prob >= 0.0f && m.ss_rfr_entry_prob <= 1.0f))
            return false;
    }
    return true;
}

// srgb_to_linear (maths.h:631-638) in float; for 8-bit texels the reference reads a 256-entry table
// of the same curve evaluated in double precision (texture.cpp:369-401), which the table below is.
float srgb_to_linear_f(float x) { return x < 0.04045f ? x / 12.92f : std::pow((x + 0.055f) / 1.055f, 2.4f); }

const float *srgb_u8_table()
{
    static const std::vector<float> table = [] {
        std::vector<float> t(256);
        for (int i = 0; i < 256; ++i) {
            const double c = i / 255.0;
            t[i] = (float)(c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4));
        }
        return t;
    }();
    return table.data();
}

// Texture::fetch_as_float (texture.cpp:403-460) of every texel: 4 floats per texel, unused 0.
bool convert_texture(const ks_texture_desc &t, std::vector<float4> &out)
{
    if (!t.texels || t.width == 0 || t.height == 0 || t.channels < 1 || t.channels > 4 || t.format < 0 ||
        t.format > 2 || (uint64_t)t.width * t.height > (1ull << 28))
        return false;
    const size_t n = (size_t)t.width * t.height, nc = t.channels;
    const float *lut = srgb_u8_table();
    for (size_t i = 0; i < n; ++i) {
        float v[4] = {0, 0, 0, 0};
        for (size_t c = 0; c < nc; ++c) {
            const size_t k = i * nc + c;
            if (t.format == 0) {
                const uint8_t u = ((const uint8_t *)t.texels)[k];
                v[c] = t.srgb ? lut[u] : (float)u / 255.0f;
            } else if (t.format == 1) {
                const float f = (float)((const uint16_t *)t.texels)[k] / 65535.0f;
                v[c] = t.srgb ? srgb_to_linear_f(f) : f;
            } else {
                const float f = ((const float *)t.texels)[k];
                v[c] = t.srgb ? srgb_to_linear_f(f) : f;
            }
        }
        out.push_back(make_float4(v[0], v[1], v[2], v[3]));
    }
    return true;
}

// A binding's device form; false for an index or enum out of range or a non-finite value.
bool binding_to_gpu(const ks_texture_binding &b, const ks_scene_desc &d, BindingGPU &g)
{
    if (b.material >= d.n_materials || b.texture >= d.n_textures || b.field < 0 || b.field > KS_FIELD_EMISSION ||
        (b.field == KS_FIELD_EMISSION && !d.materials[b.material].has_emission) ||
        b.filter < 0 || b.filter > 2 || b.cubic_kernel < 0 || b.cubic_kernel > 2 || b.wrap_u < 0 || b.wrap_u > 1 ||
        b.wrap_v < 0 || b.wrap_v > 1 || b.normal_space < 0 || b.normal_space > 1)
        return false;
    auto finite = [](float x) { return std::isfinite(x); };
    for (int k = 0; k < 2; ++k)
        if (!finite(b.uv_scale[k]) || !finite(b.uv_offset[k]))
            return false;
    for (int k = 0; k < 4; ++k)
        if (!finite(b.scale[k]) || b.swizzle[k] < -1 || b.swizzle[k] > 3)
            return false;
    if (!finite(b.strength))
        return false;
    g = BindingGPU{};
    g.tex = (int)b.texture;
    g.field = b.field;
    g.filter = b.filter;
    g.wrap_u = b.wrap_u;
    g.wrap_v = b.wrap_v;
    g.flip_v = b.flip_v != 0;
    for (int k = 0; k < 4; ++k) {
        g.swz[k] = b.swizzle[k];
        g.scale[k] = b.scale[k];
    }
    for (int k = 0; k < 2; ++k) {
        g.uv_scale[k] = b.uv_scale[k];
        g.uv_offset[k] = b.uv_offset[k];
    }
    // CubicSampler's kernels (texture.h:91-121): Mitchell-Netravali (B = C = 1/3), cubic B-spline,
    // Catmull-Rom, as polynomials in (x^3, x^2, x, 1) for |x| < 1 (ca) and 1 <= |x| < 2 (cb)
    static const double kCa[3][4] = {{21, -36, 0, 16}, {3, -6, 0, 4}, {3, -5, 0, 2}};
    static const double kCb[3][4] = {{-7, 36, -60, 32}, {-1, 6, -12, 8}, {-1, 5, -8, 4}};
    static const double kDiv[3] = {18, 6, 2};
    for (int k = 0; k < 4; ++k) {
        g.ca[k] = (float)(kCa[b.cubic_kernel][k] / kDiv[b.cubic_kernel]);
        g.cb[k] = (float)(kCb[b.cubic_kernel][k] / kDiv[b.cubic_kernel]);
    }
    g.space = b.normal_space;
    g.range01 = b.range01 != 0;
    g.strength = b.strength;
    if (b.field == KS_FIELD_NORMAL_MAP && b.normal_space == 1) {
        // Transform::normal (maths.h:987): the inverse transpose of the 3x3 part
        double m[3][3], inv[3][3];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                m[r][c] = b.to_world[4 * r + c];
        const double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                           m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
        if (!(std::fabs(det) > 0.0) || !std::isfinite(det))
            return false;
        inv[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) / det;
        inv[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) / det;
        inv[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det;
        inv[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) / det;
        inv[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) / det;
        inv[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / det;
        inv[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) / det;
        inv[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / det;
        inv[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) / det;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                g.nrm[3 * r + c] = (float)inv[c][r];
    }
    return true;
}

} // namespace

// The device copy of a material; false for a non-finite field or an enum out of range.
bool ksb::material_to_gpu(const ks_material_desc &m, MaterialGPU &g)
{
    if (!valid_material(m) || m.microfacet < 0 || m.microfacet > 1 || m.bsdf < 0 || m.bsdf > 2 ||
        m.has_emission < 0 || m.has_emission > 1)
        return false;
    g = MaterialGPU{};
    for (int c = 0; c < 3; ++c) {
        g.basecolor[c] = m.basecolor[c];
        g.emission[c] = m.emission[c];
    }
    g.roughness = m.roughness;
    g.metallic = m.metallic;
    g.ior = m.ior;
    g.specular_r0_mul = m.specular_r0_mul;
    g.specular_trans = m.specular_trans;
    g.diffuse_trans = m.diffuse_trans;
    g.diffuse_trans_fwd = m.diffuse_trans_fwd;
    g.microfacet = m.microfacet;
    g.bsdf = m.bsdf;
    g.specular = m.specular;
    g.has_emission = m.has_emission;
    g.mesh_light = -1;
    g.has_ss = m.has_subsurface;
    for (int c = 0; c < 3; ++c) {
        // BSSRDF::sample clamps the albedo to [0, 1] (subsurface.cpp:526-527)
        g.ss_albedo[c] = std::min(std::max(m.ss_albedo[c], 0.0f), 1.0f);
        g.ss_radius[c] = m.ss_radius[c];
    }
    g.ss_g = m.ss_anisotropy;
    g.ss_ior = m.ss_ior;
    g.ss_rfr = m.ss_rfr_entry_prob;
    return true;
}

namespace
{
// Per triangle: its mesh (from the meshes' first-triangle offsets; offset[0] = 0, strictly
// increasing: meshes are not empty), the check of its three vertex indices against the mesh's
// vertex count, and the indices made global by the mesh's first vertex.  *bad_mesh ends as the
// lowest mesh with an index out of range (untouched when there is none).
// mesh_info: [0, n] first triangle, [n + 1, 2n] first vertex, [2n + 1, 3n] vertex count.
__global__ void k_mesh_fixup(const uint32_t *mesh_info, uint32_t n_meshes, uint32_t n_tris, uint32_t *indices,
                             uint32_t *tri_mesh, int *bad_mesh)
{
    const uint32_t *offset = mesh_info, *first_vert = mesh_info + n_meshes + 1,
                   *n_verts = mesh_info + 2 * n_meshes + 1;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n_tris; t += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n_meshes;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (offset[mid] <= t)
                lo = mid;
            else
                hi = mid;
        }
        tri_mesh[t] = lo;
        const uint32_t nv = n_verts[lo], base = first_vert[lo];
        uint32_t *ix = indices + 3 * (size_t)t;
        const uint32_t a = ix[0], b = ix[1], c = ix[2];
        if (a >= nv || b >= nv || c >= nv)
            atomicMin(bad_mesh, (int)lo);
        ix[0] = a + base;
        ix[1] = b + base;
        ix[2] = c + base;
    }
}

// Holds the context's pinned upload memory for a scope.
struct KsPinnedLease
{
    bool *flag;
    explicit KsPinnedLease(bool *f) : flag(f)
    {
        if (flag)
            *flag = true;
    }
    ~KsPinnedLease()
    {
        if (flag)
            *flag = false;
    }
};
} // namespace

extern "C" {

// Validates the prototypes and instances and keeps them on the host (with inverse transforms).
static ks_status store_instances(ks_scene *s, const ks_scene_desc *desc)
{
    ks_context *ctx = s->ctx;
    if (!desc->instances || !desc->prototypes || desc->n_prototypes == 0)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: instances need prototypes");
    std::vector<int> owner(desc->n_meshes, -1);
    for (uint32_t p = 0; p < desc->n_prototypes; ++p) {
        const ks_prototype_desc &pd = desc->prototypes[p];
        if (pd.n_meshes == 0 || (uint64_t)pd.first_mesh + pd.n_meshes > desc->n_meshes)
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: prototype mesh range out of bounds");
        for (uint32_t m = pd.first_mesh; m < pd.first_mesh + pd.n_meshes; ++m) {
            if (owner[m] >= 0)
                return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: prototypes overlap");
            owner[m] = (int)p;
        }
        s->host.proto_tri_begin.push_back(s->host.mesh_tri_offset[pd.first_mesh]);
        s->host.proto_tri_end.push_back(s->host.mesh_tri_offset[pd.first_mesh + pd.n_meshes]);
    }
    for (uint32_t i = 0; i < desc->n_instances; ++i) {
        const ks_instance_desc &id = desc->instances[i];
        if (id.prototype >= desc->n_prototypes)
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: instance prototype out of range");
        double m[3][4];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 4; ++c) {
                m[r][c] = id.to_world[4 * r + c];
                if (!std::isfinite(m[r][c]))
                    return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: non-finite instance transform");
            }
        // inverse of the affine map: [A t]^-1 = [A^-1, -A^-1 t]
        double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                     m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                     m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
        if (!(std::fabs(det) > 1e-30))
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: singular instance transform");
        double inv[3][3];
        inv[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) / det;
        inv[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) / det;
        inv[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det;
        inv[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) / det;
        inv[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) / det;
        inv[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / det;
        inv[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) / det;
        inv[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / det;
        inv[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) / det;
        for (int r = 0; r < 3; ++r) {
            double t = -(inv[r][0] * m[0][3] + inv[r][1] * m[1][3] + inv[r][2] * m[2][3]);
            for (int c = 0; c < 3; ++c)
                s->host.inst_inv.push_back((float)inv[r][c]);
            s->host.inst_inv.push_back((float)t);
        }
        for (int k = 0; k < 12; ++k)
            s->host.inst_xf.push_back(id.to_world[k]);
        s->host.inst_proto.push_back(id.prototype);
    }
    s->n_instances = desc->n_instances;
    s->n_protos = desc->n_prototypes;
    cudaStream_t st = ctx->stream;
    KS_CUDA_TRY(ctx, s->inst_xf.alloc(s->host.inst_xf.size()));
    KS_CUDA_TRY(ctx, s->inst_inv.alloc(s->host.inst_inv.size()));
    KS_CUDA_TRY(ctx, s->inst_proto.alloc(s->host.inst_proto.size()));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->inst_xf.ptr, s->host.inst_xf.data(), s->inst_xf.bytes(),
                                     cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->inst_inv.ptr, s->host.inst_inv.data(), s->inst_inv.bytes(),
                                     cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(s->inst_proto.ptr, s->host.inst_proto.data(), s->inst_proto.bytes(),
                                     cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return KS_OK;
}

ks_status ks_scene_create(ks_context *ctx, const ks_scene_desc *desc, ks_scene **out)
{
    if (!ctx || !desc || !out)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: null argument");
    *out = nullptr;
    if (desc->n_meshes == 0 || !desc->meshes)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: no meshes");
    if (desc->n_materials == 0 || !desc->materials)
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: no materials");
    uint64_t n_tris = 0, n_verts = 0;
    for (uint32_t m = 0; m < desc->n_meshes; ++m) {
        const ks_mesh_desc &md = desc->meshes[m];
        if (!md.vertices || !md.indices || md.n_triangles == 0 || md.n_vertices == 0)
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: empty mesh " + std::to_string(m));
        if (md.material >= desc->n_materials)
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: material index out of range");
        n_tris += md.n_triangles;
        n_verts += md.n_vertices;
    }
    if (n_tris >= (1ull << 30) || n_verts >= (1ull << 31))
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: scene too large");
    for (uint32_t k = 0; k < desc->n_materials; ++k) {
        MaterialGPU g;
        if (!material_to_gpu(desc->materials[k], g))
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: material " + std::to_string(k) +
                                                          ": a non-finite field, or microfacet, bsdf or "
                                                          "has_emission out of range (zero-initialise the "
                                                          "descriptor)");
    }
    if ((desc->n_textures && !desc->textures) || (desc->n_bindings && !desc->bindings))
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: n_textures / n_bindings without arrays");
    for (uint32_t k = 0; k < desc->n_textures; ++k) {
        const ks_texture_desc &t = desc->textures[k];
        if (!t.texels || t.width == 0 || t.height == 0 || t.channels < 1 || t.channels > 4 || t.format < 0 ||
            t.format > 2 || (uint64_t)t.width * t.height > (1ull << 28))
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: bad texture " + std::to_string(k));
    }
    for (uint32_t k = 0; k < desc->n_materials; ++k) {
        const ks_material_desc &m = desc->materials[k];
        if (m.has_subsurface && (m.has_emission || desc->n_instances))
            return fail(ctx, KS_ERR_UNSUPPORTED, "ks_scene_create: material " + std::to_string(k) +
                                                     ": subsurface scattering with emission or in an instanced scene");
    }
    for (uint32_t k = 0; k < desc->n_bindings; ++k) {
        BindingGPU g;
        if (!binding_to_gpu(desc->bindings[k], *desc, g))
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: bad texture binding " + std::to_string(k));
        if (g.field == KS_FIELD_OPACITY_MAP && desc->n_instances)
            return fail(ctx, KS_ERR_UNSUPPORTED, "ks_scene_create: opacity maps in instanced scenes");
    }
    KS_CUDA_TRY(ctx, enter_device(ctx));
    ks_scene *s = new (std::nothrow) ks_scene();
    if (!s)
        return fail(ctx, KS_ERR_OUT_OF_MEMORY, "ks_scene_create");
    s->ctx = ctx;
    s->n_tris = (uint32_t)n_tris;
    s->n_verts = (uint32_t)n_verts;
    // sky (checked before the uploads are laid out: the map is one of them)
    const ks_sky_desc &sd = desc->sky;
    if (sd.kind < 0 || sd.kind > 3 || (sd.kind >= 2 && (!sd.map_rgb || sd.width == 0 || sd.height == 0)) ||
        (sd.kind == 3 && (sd.width != sd.height || (sd.width & (sd.width - 1)) != 0 || sd.width > (1u << 14)))) {
        delete s;
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: bad sky description (an equal-area map is a "
                                                  "square of a power-of-two side, at most 16384)");
    }
    const size_t n_sky = sd.kind >= 2 ? 3 * (size_t)sd.width * sd.height : 0;
    // per-vertex shading attributes: only meshes that shade smooth contribute normals (a mesh with
    // use_smooth_normal off or no vertex normals shades flat, geometry.cpp:139-141)
    bool any_smooth = false, any_uv = false;
    for (uint32_t m = 0; m < desc->n_meshes; ++m) {
        any_smooth |= desc->meshes[m].use_smooth_normal && desc->meshes[m].vertex_normals;
        any_uv |= desc->meshes[m].texcoords != nullptr;
    }
    // The concatenated vertex, index, normal and texcoord arrays and the sky map are assembled in
    // the context's pinned upload memory when it is free (else in host vectors), then copied.
    auto align = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t off_i = align(sizeof(float) * 3 * n_verts), off_n = off_i + align(sizeof(uint32_t) * 3 * n_tris);
    const size_t off_t = off_n + (any_smooth ? align(sizeof(float) * 3 * n_verts) : 0);
    const size_t off_s = off_t + (any_uv ? align(sizeof(float) * 2 * n_verts) : 0);
    const size_t stage_bytes = off_s + sizeof(float) * n_sky;
    const bool staged = !ctx->upload.busy && ctx->upload.reserve(stage_bytes) == cudaSuccess;
    if (!staged)
        cudaGetLastError(); // a failed pinned allocation only means the pageable path
    KsPinnedLease upload_lease(staged ? &ctx->upload.busy : nullptr);
    std::vector<char> own_stage;
    if (!staged)
        own_stage.resize(stage_bytes);
    char *stage = staged ? static_cast<char *>(ctx->upload.ptr) : own_stage.data();
    float *verts = reinterpret_cast<float *>(stage);
    uint32_t *idx = reinterpret_cast<uint32_t *>(stage + off_i);
    float *normals = any_smooth ? reinterpret_cast<float *>(stage + off_n) : nullptr;
    float *texcoords = any_uv ? reinterpret_cast<float *>(stage + off_t) : nullptr;
    float *sky_map = n_sky ? reinterpret_cast<float *>(stage + off_s) : nullptr;
    uint64_t vo = 0, to = 0;
    for (uint32_t m = 0; m < desc->n_meshes; ++m) {
        const ks_mesh_desc &md = desc->meshes[m];
        const uint64_t nv = md.n_vertices, v0 = vo;
        host_parallel(3 * nv, 1u << 17, [&](size_t b, size_t e) {
            std::memcpy(verts + 3 * v0 + b, md.vertices + b, sizeof(float) * (e - b));
        });
        // the indices as given: k_mesh_fixup checks them and adds the mesh's first vertex
        uint32_t *dst = idx + 3 * to;
        host_parallel(3ull * md.n_triangles, 1u << 17, [&](size_t b, size_t e) {
            std::memcpy(dst + b, md.indices + b, sizeof(uint32_t) * (e - b));
        });
        int flags = md.twosided ? kMeshTwosided : 0;
        if (md.use_smooth_normal && md.vertex_normals) {
            flags |= kMeshSmooth;
            float *dn = normals + 3 * vo;
            host_parallel(3 * nv, 1u << 17, [&](size_t b, size_t e) {
                std::memcpy(dn + b, md.vertex_normals + b, sizeof(float) * (e - b));
            });
        } else if (normals) {
            std::memset(normals + 3 * vo, 0, sizeof(float) * 3 * nv);
        }
        if (md.texcoords) {
            flags |= kMeshTexcoords;
            float *dt = texcoords + 2 * vo;
            host_parallel(2 * nv, 1u << 17, [&](size_t b, size_t e) {
                std::memcpy(dt + b, md.texcoords + b, sizeof(float) * (e - b));
            });
        } else if (texcoords) {
            std::memset(texcoords + 2 * vo, 0, sizeof(float) * 2 * nv);
        }
        s->host.mesh_tri_offset.push_back((uint32_t)to);
        s->host.mesh_material.push_back(md.material);
        s->host.mesh_flags.push_back(flags);
        vo += md.n_vertices;
        to += md.n_triangles;
    }
    s->host.mesh_tri_offset.push_back((uint32_t)to);
    if (n_sky)
        host_parallel(n_sky, 1u << 17, [&](size_t b, size_t e) {
            std::memcpy(sky_map + b, sd.map_rgb + b, sizeof(float) * (e - b));
        });
    s->host.materials.assign(desc->materials, desc->materials + desc->n_materials);
    // instancing
    if (desc->n_instances > 0) {
        ks_status st = store_instances(s, desc);
        if (st != KS_OK) {
            delete s;
            return st;
        }
    }
    if (sd.kind == 3) // the alias table over the texels is built on the host
        s->sky_host.assign(sky_map, sky_map + n_sky);
    s->sky_desc = sd;
    if (desc->n_lights && !desc->lights) {
        delete s;
        return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: n_lights without lights");
    }
    for (uint32_t k = 0; k < desc->n_lights; ++k) {
        const ks_light_desc &l = desc->lights[k];
        bool ok = l.type == 0 || l.type == 1;
        for (int c = 0; c < 3; ++c)
            ok = ok && std::isfinite(l.color[c]) && std::isfinite(l.vec[c]);
        if (!ok) {
            delete s;
            return fail(ctx, KS_ERR_INVALID_ARGUMENT, "ks_scene_create: bad light " + std::to_string(k));
        }
        s->lights.push_back(l);
    }
    s->sky_desc.map_rgb = nullptr;
    std::vector<MaterialGPU> mats(desc->n_materials);
    for (uint32_t k = 0; k < desc->n_materials; ++k) {
        const ks_material_desc &m = desc->materials[k];
        material_to_gpu(m, mats[k]);
        s->ext_materials |= m.bsdf != 0 || m.microfacet != 0 || m.has_subsurface != 0;
        s->any_subsurface |= m.has_subsurface != 0;
    }
    // textures and bindings (validated above), the bindings grouped by material in their order
    std::vector<float4> texels;
    std::vector<TexInfo> tex_info;
    std::vector<BindingGPU> binds;
    for (uint32_t k = 0; k < desc->n_textures; ++k) {
        const ks_texture_desc &t = desc->textures[k];
        tex_info.push_back(TexInfo{(uint32_t)texels.size(), (int)t.width, (int)t.height, (int)t.channels});
        convert_texture(t, texels);
    }
    for (uint32_t m = 0; m < desc->n_materials; ++m) {
        mats[m].bind_begin = (int)binds.size();
        for (uint32_t k = 0; k < desc->n_bindings; ++k)
            if (desc->bindings[k].material == m) {
                BindingGPU g;
                binding_to_gpu(desc->bindings[k], *desc, g);
                binds.push_back(g);
                if (g.field == KS_FIELD_NORMAL_MAP)
                    mats[m].tex_flags |= kMatNormalMap;
                else if (g.field == KS_FIELD_OPACITY_MAP)
                    mats[m].tex_flags |= kMatOpacityMap;
                else if (g.field == KS_FIELD_EMISSION)
                    mats[m].tex_flags |= kMatEmissionMap;
            }
        mats[m].bind_count = (int)binds.size() - mats[m].bind_begin;
        s->any_opacity |= (mats[m].tex_flags & kMatOpacityMap) != 0;
        s->any_emission_map |= (mats[m].tex_flags & kMatEmissionMap) != 0;
    }
    s->any_bindings = !binds.empty();
    if (s->any_emission_map) {
        s->emit_tex.texels = texels;
        s->emit_tex.info = tex_info;
        s->emit_tex.binds = binds;
        s->emit_tex.mats = mats;
        if (texcoords)
            s->emit_tex.texcoords.assign(texcoords, texcoords + 2 * n_verts);
    }
    cudaError_t e = s->materials.alloc(mats.size());
    if (e == cudaSuccess)
        e = s->mesh_material.alloc(s->host.mesh_material.size());
    if (e == cudaSuccess)
        e = s->mesh_flags.alloc(s->host.mesh_flags.size());
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->materials.ptr, mats.data(), s->materials.bytes(), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->mesh_material.ptr, s->host.mesh_material.data(), s->mesh_material.bytes(),
                            cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->mesh_flags.ptr, s->host.mesh_flags.data(), s->mesh_flags.bytes(),
                            cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && !binds.empty()) {
        e = s->tex_texels.alloc(texels.size());
        if (e == cudaSuccess)
            e = s->tex_info.alloc(tex_info.size());
        if (e == cudaSuccess)
            e = s->bindings.alloc(binds.size());
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->tex_texels.ptr, texels.data(), s->tex_texels.bytes(), cudaMemcpyHostToDevice,
                                ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->tex_info.ptr, tex_info.data(), s->tex_info.bytes(), cudaMemcpyHostToDevice,
                                ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->bindings.ptr, binds.data(), s->bindings.bytes(), cudaMemcpyHostToDevice,
                                ctx->stream);
    }
    if (e == cudaSuccess && any_smooth) {
        e = s->normals.alloc(3 * n_verts);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->normals.ptr, normals, s->normals.bytes(), cudaMemcpyHostToDevice,
                                ctx->stream);
    }
    if (e == cudaSuccess && any_uv) {
        e = s->texcoords.alloc(2 * n_verts);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->texcoords.ptr, texcoords, s->texcoords.bytes(), cudaMemcpyHostToDevice,
                                ctx->stream);
    }
    DevBuf<uint32_t> mesh_info; // k_mesh_fixup's per-mesh table
    DevBuf<int> bad_mesh;
    std::vector<uint32_t> info(s->host.mesh_tri_offset);
    for (uint32_t m = 0, v = 0; m < desc->n_meshes; v += desc->meshes[m].n_vertices, ++m)
        info.push_back(v);
    for (uint32_t m = 0; m < desc->n_meshes; ++m)
        info.push_back(desc->meshes[m].n_vertices);
    if (e == cudaSuccess)
        e = s->verts.alloc(3 * n_verts);
    if (e == cudaSuccess)
        e = s->indices.alloc(3 * n_tris);
    if (e == cudaSuccess)
        e = s->tri_mesh.alloc(n_tris);
    if (e == cudaSuccess)
        e = mesh_info.alloc(info.size());
    if (e == cudaSuccess)
        e = bad_mesh.alloc(1);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->verts.ptr, verts, s->verts.bytes(), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->indices.ptr, idx, s->indices.bytes(), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(mesh_info.ptr, info.data(), mesh_info.bytes(), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(bad_mesh.ptr, 0x7f, sizeof(int), ctx->stream); // 0x7f7f7f7f: no mesh
    if (e == cudaSuccess) {
        k_mesh_fixup<<<(unsigned)std::min<uint64_t>((n_tris + 255) / 256, (uint64_t)ctx->sm_count * 16), 256, 0,
                       ctx->stream>>>(mesh_info.ptr, desc->n_meshes, (uint32_t)n_tris, s->indices.ptr,
                                      s->tri_mesh.ptr, bad_mesh.ptr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && n_sky) {
        e = s->sky_rgb.alloc(n_sky);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(s->sky_rgb.ptr, sky_map, sizeof(float) * n_sky, cudaMemcpyHostToDevice, ctx->stream);
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(ctx->stream);
    int bad = 0x7f7f7f7f;
    if (e == cudaSuccess)
        e = cudaMemcpy(&bad, bad_mesh.ptr, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        delete s;
        return cuda_fail(ctx, e, "ks_scene_create: upload");
    }
    if (bad != 0x7f7f7f7f) {
        delete s;
        return fail(ctx, KS_ERR_INVALID_ARGUMENT,
                    "ks_scene_create: vertex index out of range in mesh " + std::to_string(bad));
    }
    *out = s;
    return KS_OK;
}

void ks_scene_destroy(ks_scene *scene)
{
    if (!scene)
        return;
    cudaSetDevice(scene->ctx->device);
    cudaStreamSynchronize(scene->ctx->stream);
    delete scene;
}

ks_status ks_scene_build_bvh(ks_scene *scene, const ks_sbvh_options *opts, float *build_ms)
{
    if (!scene)
        return KS_ERR_INVALID_ARGUMENT;
    ks_sbvh_options o{4, 12, 1.0f, 1e-5f};
    if (opts)
        o = *opts;
    KS_CUDA_TRY(scene->ctx, enter_device(scene->ctx));
    scene->bvh_built = false;
    scene->lights_built = false;
    ks_status st = build_sbvh(scene, o, build_ms);
    if (st != KS_OK)
        return st;
    // the light sampler needs the scene bound (PowerLightSampler(scene_bound), small_pt.cpp:201)
    return build_lights(scene);
}

ks_status ks_sbvh_counts(const ks_scene *scene, uint32_t *n_nodes, uint32_t *n_prims)
{
    if (!scene || !n_nodes || !n_prims)
        return KS_ERR_INVALID_ARGUMENT;
    if (!scene->bvh_built)
        return fail(scene->ctx, KS_ERR_NOT_BUILT, "ks_sbvh_counts: call ks_scene_build_bvh first");
    *n_nodes = scene->n_nodes;
    *n_prims = scene->n_prims;
    return KS_OK;
}

ks_status ks_sbvh_export(const ks_scene *scene, float *node_bounds, uint32_t *node_axis, uint32_t *node_right,
                         uint32_t *node_prim_offset, uint32_t *prims)
{
    if (!scene)
        return KS_ERR_INVALID_ARGUMENT;
    ks_context *ctx = scene->ctx;
    if (!scene->bvh_built)
        return fail(ctx, KS_ERR_NOT_BUILT, "ks_sbvh_export: call ks_scene_build_bvh first");
    if (scene->n_instances)
        return fail(ctx, KS_ERR_UNSUPPORTED, "ks_sbvh_export: instanced scenes have one SBVH per prototype");
    KS_CUDA_TRY(ctx, enter_device(ctx));
    std::vector<RefNode> nodes(scene->n_nodes);
    KS_CUDA_TRY(ctx, cudaMemcpy(nodes.data(), scene->ref_nodes.ptr, sizeof(RefNode) * nodes.size(),
                                cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < nodes.size(); ++i) {
        if (node_bounds)
            for (int k = 0; k < 3; ++k) {
                node_bounds[6 * i + k] = nodes[i].bmin[k];
                node_bounds[6 * i + 3 + k] = nodes[i].bmax[k];
            }
        if (node_axis)
            node_axis[i] = nodes[i].axis;
        if (node_right)
            node_right[i] = nodes[i].right;
        if (node_prim_offset)
            node_prim_offset[i] = nodes[i].prim_offset;
    }
    if (prims)
        KS_CUDA_TRY(ctx, cudaMemcpy(prims, scene->prims.ptr, sizeof(uint32_t) * scene->n_prims,
                                    cudaMemcpyDeviceToHost));
    return KS_OK;
}

} // extern "C"

// ks_trace_rays and ks_trace_rays_wide (wide: the renderer's traversal kernels: the 4-wide view for
// flat scenes, the persistent two-level traversal for instanced ones).
static ks_status trace_rays_impl(ks_scene *scene, const float *rays, uint32_t n, int any_hit, int culling,
                                 uint32_t *tri_idx, float *t, float *bary, bool wide, const char *name)
{
    if (!scene || !rays || !tri_idx || (!any_hit && (!t || !bary)) || culling < 0 || culling > 2)
        return fail(scene ? scene->ctx : nullptr, KS_ERR_INVALID_ARGUMENT, std::string(name) + ": bad argument");
    ks_context *ctx = scene->ctx;
    if (!scene->bvh_built)
        return fail(ctx, KS_ERR_NOT_BUILT, std::string(name) + ": call ks_scene_build_bvh first");
    if (n == 0)
        return KS_OK;
    KS_CUDA_TRY(ctx, enter_device(ctx));
    DevBuf<float> d_rays, d_t, d_bary;
    DevBuf<uint32_t> d_tri, d_fetch;
    DevBuf<int> d_flag;
    KS_CUDA_TRY(ctx, d_rays.alloc((size_t)n * 8));
    KS_CUDA_TRY(ctx, d_tri.alloc(n));
    KS_CUDA_TRY(ctx, d_t.alloc(n));
    KS_CUDA_TRY(ctx, d_bary.alloc((size_t)n * 3));
    KS_CUDA_TRY(ctx, d_flag.alloc(1));
    cudaStream_t st = ctx->stream;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(d_rays.ptr, rays, d_rays.bytes(), cudaMemcpyHostToDevice, st));
    KS_CUDA_TRY(ctx, cudaMemsetAsync(d_flag.ptr, 0, sizeof(int), st));
    const float *b = scene->scene_bound;
    if (scene->n_instances && wide) {
        KS_CUDA_TRY(ctx, d_fetch.alloc(1));
        KS_CUDA_TRY(ctx, cudaMemsetAsync(d_fetch.ptr, 0, sizeof(uint32_t), st));
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_inst_kernel_pt, 128, 0);
        const unsigned grid = std::min<unsigned>((n + 127) / 128, (unsigned)std::max(per_sm, 1) * ctx->sm_count);
        trace_inst_kernel_pt<<<grid, 128, 0, st>>>(scene->wide_nodes.ptr, scene->prim_tris.ptr, make_view(scene).inst,
                                                   d_rays.ptr, n, any_hit, culling, d_tri.ptr, d_t.ptr, d_bary.ptr,
                                                   d_flag.ptr, d_fetch.ptr);
    } else if (scene->n_instances) {
        trace_kernel<<<(n + 127) / 128, 128, 0, st>>>(scene->trav_nodes.ptr, scene->prim_tris.ptr, scene->root_ref,
                                                       scene->root_count, b[0], b[1], b[2], b[3], b[4], b[5],
                                                       d_rays.ptr, n, any_hit, culling, d_tri.ptr, d_t.ptr,
                                                       d_bary.ptr, d_flag.ptr, make_view(scene).inst);
    } else {
        KS_CUDA_TRY(ctx, d_fetch.alloc(1));
        KS_CUDA_TRY(ctx, cudaMemsetAsync(d_fetch.ptr, 0, sizeof(uint32_t), st));
        int per_sm = 1;
        if (wide)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_kernel_pt<WideNode>, 128, 0);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_kernel_pt<TravNode>, 128, 0);
        const unsigned grid = std::min<unsigned>((n + 127) / 128, (unsigned)std::max(per_sm, 1) * ctx->sm_count);
        if (wide)
            trace_kernel_pt<<<grid, 128, 0, st>>>(scene->wide_nodes.ptr, scene->prim_tris.ptr, scene->root_ref,
                                                  scene->root_count, b[0], b[1], b[2], b[3], b[4], b[5], d_rays.ptr,
                                                  n, any_hit, culling, d_tri.ptr, d_t.ptr, d_bary.ptr, d_flag.ptr,
                                                  d_fetch.ptr);
        else
            trace_kernel_pt<<<grid, 128, 0, st>>>(scene->trav_nodes.ptr, scene->prim_tris.ptr, scene->root_ref,
                                                  scene->root_count, b[0], b[1], b[2], b[3], b[4], b[5], d_rays.ptr,
                                                  n, any_hit, culling, d_tri.ptr, d_t.ptr, d_bary.ptr, d_flag.ptr,
                                                  d_fetch.ptr);
    }
    KS_CUDA_TRY(ctx, cudaGetLastError());
    int overflow = 0;
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(tri_idx, d_tri.ptr, d_tri.bytes(), cudaMemcpyDeviceToHost, st));
    if (!any_hit) {
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(t, d_t.ptr, d_t.bytes(), cudaMemcpyDeviceToHost, st));
        KS_CUDA_TRY(ctx, cudaMemcpyAsync(bary, d_bary.ptr, d_bary.bytes(), cudaMemcpyDeviceToHost, st));
    }
    KS_CUDA_TRY(ctx, cudaMemcpyAsync(&overflow, d_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    KS_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    if (overflow)
        return fail(ctx, KS_ERR_QUEUE_OVERFLOW, std::string(name) + ": traversal stack depth exceeded");
    return KS_OK;
}

extern "C" {

ks_status ks_trace_rays(ks_scene *scene, const float *rays, uint32_t n, int any_hit, int culling, uint32_t *tri_idx,
                        float *t, float *bary)
{
    return trace_rays_impl(scene, rays, n, any_hit, culling, tri_idx, t, bary, false, "ks_trace_rays");
}

ks_status ks_trace_rays_wide(ks_scene *scene, const float *rays, uint32_t n, int any_hit, int culling,
                             uint32_t *tri_idx, float *t, float *bary)
{
    return trace_rays_impl(scene, rays, n, any_hit, culling, tri_idx, t, bary, true, "ks_trace_rays_wide");
}

} // extern "C"
