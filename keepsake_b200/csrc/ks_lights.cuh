// Lights and light selection on the device.
//
//   SkyLight eval / sample / pdf      light.cpp:59-134 (lat-long map, bilinear, thresholded PMF)
//   MeshTriLight sample / pdf         light.cpp:567-628 (uniform barycentric area sampling)
//   PowerLightSampler sample / probability   light.cpp:674-689
//   DistribTable(2D) sample_linear / pdf     distrib.cpp:32-107
//   lerp_helper                        maths.h:760-780
#pragma once
#include "ks_math.cuh"
#include "ks_scene.h"
#include "ks_traverse.cuh"

namespace ksb
{

// Flat, read-only view of everything the shading kernels read (passed by value).
enum : int
{
    kShadePlain = 0,
    kShadeAttribs = 1,
    kShadeGeneral = 2
};

struct SceneView
{
    InstanceView inst; // instances (inst.n == 0: flat scene)
    const TravNode *nodes;
    const WideNode *wide; // 4-wide view of nodes (instanced scenes: of the concatenated BLAS nodes)
    const float4 *prim_tris;
    const float *verts;      // global vertex positions (3 floats each)
    const uint32_t *indices; // global triangle vertex ids (3 each)
    uint32_t root_ref, root_count;
    float bmin[3], bmax[3];
    const uint32_t *tri_mesh;
    const uint32_t *mesh_material;
    const int *mesh_flags;   // per mesh: kMeshTwosided | kMeshSmooth | kMeshTexcoords
    const float *normals;    // global vertex normals (3 floats each; null when no mesh shades smooth)
    const float *texcoords;  // global texture coordinates (2 floats each; null when no mesh has them)
    const MaterialGPU *materials;
    // the shading kernel variant the scene needs: kShadePlain; kShadeAttribs for vertex normals or
    // texcoords; kShadeGeneral for a material other than the GGX PrincipledBSDF
    int shade_variant;
    // lights
    uint32_t light_count;
    uint32_t n_nonmesh; // the sky (light 0, when there is one) and the point / directional lights
    uint32_t n_sky;     // 1 when a sky light exists
    const float4 *punctual; // per point / directional light: (vec, type), (color, 0)
    const float *power_cdf;   // light_count + 1
    const int32_t *tri_light; // per triangle: flat light index or -1 (nullptr if no emitters)
    const uint32_t *ml_tri;   // per mesh-light triangle (flat index - n_nonmesh): global triangle
    const float *ml_area;
    const float4 *ml_emission;
    const float4 *ml_verts;         // 3 per mesh-light triangle: world-space vertices
    const int32_t *inst_light_base; // instanced scenes: flat light index of each instance's first mesh light
    // sky
    int sky_kind; // 0 none, 1 ambient, 2 map
    int sky_w, sky_h;
    float sky_l2w[9], sky_w2l[9];
    int sky_y_up;
    float sky_strength;
    const float4 *sky_map;
    const float *sky_cond;   // sky_h rows of sky_w + 1
    const float *sky_margin; // sky_h + 1
    const uint32_t *sky_cond_guide;   // sky_h rows of kGuide
    const uint32_t *sky_margin_guide; // kGuide
};

// ---- distribution tables ----------------------------------------------------------------------
// std::upper_bound over cdf[0..n] for u, minus one.
KS_D uint32_t cdf_find(const float *cdf, uint32_t n, float u)
{
    uint32_t lo = 0, count = n + 1; // first index with cdf[i] > u
    while (count > 0) {
        uint32_t step = count / 2, mid = lo + step;
        if (!(u < cdf[mid])) {
            lo = mid + 1;
            count -= step + 1;
        } else {
            count = step;
        }
    }
    return lo - 1;
}

KS_D float clamp_u(float u)
{
    const float hi = 0x1.fffffep-1f; // std::nextafter(1.0f, 0.0f)
    return u < 0.0f ? 0.0f : (hi < u ? hi : u);
}

KS_D float distrib_sample_linear(const float *cdf, uint32_t n, float u, float &pdf, uint32_t &index)
{
    u = clamp_u(u);
    index = cdf_find(cdf, n, u);
    float nf = (float)n;
    float c0 = cdf[index], c1 = cdf[index + 1];
    pdf = (c1 - c0) * nf;
    float du = (u - c0) / (c1 - c0);
    return ((float)index + du) / nf;
}

// Guide (cut-point) table of a CDF: guide[k] = upper_bound(cdf, k / G) - 1 for k < G.  For u in
// [k/G, (k+1)/G) the bin upper_bound(cdf, u) - 1 lies in [guide[k], guide[k+1]] (guide[G] = n-1),
// so the search touches a few entries instead of log2(n) dependent loads, with the same result.
constexpr uint32_t kGuide = 128;

KS_D uint32_t cdf_find_guided(const float *cdf, uint32_t n, const uint32_t *guide, float u)
{
    uint32_t k = (uint32_t)(u * (float)kGuide); // exact: kGuide is a power of two, u < 1
    uint32_t lo = __ldg(&guide[k]);
    uint32_t hi = k + 1 < kGuide ? __ldg(&guide[k + 1]) : n - 1;
    // largest i in [lo, hi] with cdf[i] <= u
    while (lo < hi) {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&cdf[mid]) <= u)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

KS_D float distrib_sample_linear_guided(const float *cdf, uint32_t n, const uint32_t *guide, float u, float &pdf,
                                        uint32_t &index)
{
    u = clamp_u(u);
    index = cdf_find_guided(cdf, n, guide, u);
    float nf = (float)n;
    float c0 = __ldg(&cdf[index]), c1 = __ldg(&cdf[index + 1]);
    pdf = (c1 - c0) * nf;
    float du = (u - c0) / (c1 - c0);
    return ((float)index + du) / nf;
}

KS_D float distrib_pdf(const float *cdf, uint32_t n, uint32_t index)
{
    return (cdf[index + 1] - cdf[index]) * (float)n;
}

// PowerLightSampler::probability (light.cpp:681-684)
KS_D float light_probability(const SceneView &s, uint32_t light)
{
    return distrib_pdf(s.power_cdf, s.light_count, light) / (float)s.light_count;
}

// ---- sky ------------------------------------------------------------------------------------
KS_D f3 mat3_apply(const float m[9], f3 v)
{
    return mk(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
              m[6] * v.x + m[7] * v.y + m[8] * v.z);
}

KS_D void sky_spherical(const SceneView &s, f3 wl, float &phi, float &theta)
{
    if (s.sky_y_up) {
        theta = acosf(clampf(wl.y, -1.0f, 1.0f));
        phi = atan2f(wl.z, wl.x);
    } else {
        theta = acosf(clampf(wl.z, -1.0f, 1.0f));
        phi = atan2f(wl.y, wl.x);
    }
    if (phi < 0.0f)
        phi += kTwoPi;
}

KS_D void lerp_helper(float u, int res, bool repeat, int &u0, int &u1, float &t)
{
    float us = u * (float)res - 0.5f;
    u0 = (int)floorf(us);
    u1 = u0 + 1;
    t = us - u0;
    if (repeat) {
        u0 = (u0 + res) % res;
        u1 = (u1 + res) % res;
        // u is in [0, 1] for every direction; guard the fetch against non-finite input anyway
        u0 = u0 < 0 ? 0 : u0;
        u1 = u1 < 0 ? 0 : u1;
    } else {
        u0 = u0 < 0 ? 0 : (u0 > res - 1 ? res - 1 : u0);
        u1 = u1 < 0 ? 0 : (u1 > res - 1 ? res - 1 : u1);
    }
}

KS_D f3 sky_texel(const SceneView &s, int u, int v)
{
    float4 c = __ldg(&s.sky_map[(size_t)v * s.sky_w + u]);
    return mk(c.x, c.y, c.z);
}

KS_D f3 sky_eval(const SceneView &s, f3 wi)
{
    f3 wl = mat3_apply(s.sky_w2l, wi);
    float phi, theta;
    sky_spherical(s, wl, phi, theta);
    float uv0 = phi * kInvPi * 0.5f, uv1 = theta * kInvPi;
    int u0, u1, v0, v1;
    float t0, t1;
    lerp_helper(uv0, s.sky_w, true, u0, u1, t0);
    lerp_helper(uv1, s.sky_h, false, v0, v1, t1);
    f3 L = mk(0, 0, 0);
    L += (1.0f - t0) * (1.0f - t1) * sky_texel(s, u0, v0);
    L += (1.0f - t0) * t1 * sky_texel(s, u0, v1);
    L += t0 * (1.0f - t1) * sky_texel(s, u1, v0);
    L += t0 * t1 * sky_texel(s, u1, v1);
    L *= s.sky_strength;
    return L;
}

KS_D f3 sky_sample(const SceneView &s, float u0, float u1, f3 &wi, float &wi_dist, float &pdf)
{
    float pdf_m, pdf_c;
    uint32_t vi, ui;
    float vs = distrib_sample_linear_guided(s.sky_margin, (uint32_t)s.sky_h, s.sky_margin_guide, u1, pdf_m, vi);
    float us = distrib_sample_linear_guided(s.sky_cond + (size_t)vi * (s.sky_w + 1), (uint32_t)s.sky_w,
                                            s.sky_cond_guide + (size_t)vi * kGuide, u0, pdf_c, ui);
    pdf = pdf_m * pdf_c;
    if (pdf == 0.0f)
        return mk(0, 0, 0);
    float phi = us * 2.0f * kPi;
    float theta = vs * kPi;
    float ct = cosf(theta), st = sinf(theta), cp = cosf(phi), sp = sinf(phi);
    f3 wl = s.sky_y_up ? mk(cp * st, ct, sp * st) : mk(cp * st, sp * st, ct);
    float sin_theta = sinf(theta);
    pdf /= (2.0f * kPi * kPi * sin_theta);
    if (sin_theta == 0.0f) {
        pdf = 0.0f;
        return mk(0, 0, 0);
    }
    wi = mat3_apply(s.sky_l2w, wl);
    wi_dist = kInf;
    return sky_eval(s, wi) / pdf;
}

KS_D float sky_pdf(const SceneView &s, f3 wi)
{
    f3 wl = mat3_apply(s.sky_w2l, wi);
    float phi, theta;
    sky_spherical(s, wl, phi, theta);
    float sin_theta = sinf(theta);
    if (sin_theta == 0.0f)
        return 0.0f;
    float p0 = phi * kInvPi * 0.5f, p1 = theta * kInvPi;
    int x = (int)(p0 * (float)s.sky_w);
    x = x < 0 ? 0 : (x > s.sky_w - 1 ? s.sky_w - 1 : x);
    int y = (int)(p1 * (float)s.sky_h);
    y = y < 0 ? 0 : (y > s.sky_h - 1 ? s.sky_h - 1 : y);
    float p = distrib_pdf(s.sky_margin, (uint32_t)s.sky_h, (uint32_t)y) *
              distrib_pdf(s.sky_cond + (size_t)y * (s.sky_w + 1), (uint32_t)s.sky_w, (uint32_t)x);
    p /= (2.0f * kPi * kPi * sin_theta);
    return p;
}

// ---- mesh lights ----------------------------------------------------------------------------
// MeshData::compute_geometry_normal (geometry.h:45-60) followed by Transform::normal with the
// identity instance transform (normalised twice).
KS_D f3 light_normal(f3 v0, f3 v1, f3 v2)
{
    f3 e01 = v1 - v0, e12 = v2 - v1;
    return normalize(normalize(cross(e01, e12)));
}

struct TriVerts
{
    f3 v0, v1, v2;
};

KS_D f3 mesh_light_sample(const SceneView &s, uint32_t k, const TriVerts &tv, f3 p_shade, float u0, float u1,
                          f3 &wi, float &wi_dist, float &pdf)
{
    float b0, b1;
    if (u0 < u1) {
        b0 = u0 / 2;
        b1 = u1 - b0;
    } else {
        b1 = u1 / 2;
        b0 = u0 - b1;
    }
    float w0 = 1.0f - b0 - b1;
    f3 position = w0 * tv.v0 + b0 * tv.v1 + b1 * tv.v2;
    f3 n = light_normal(tv.v0, tv.v1, tv.v2);
    wi = position - p_shade;
    float d2 = sqnorm(wi);
    if (d2 == 0.0f) {
        wi_dist = 0.0f;
        pdf = 0.0f;
        return mk(0, 0, 0);
    }
    wi_dist = sqrtf(d2);
    wi /= wi_dist;
    pdf = 1.0f / s.ml_area[k];
    float absdot = fabsf(dot(n, wi));
    if (absdot == 0.0f) {
        wi_dist = 0.0f;
        pdf = 0.0f;
        return mk(0, 0, 0);
    }
    pdf *= (d2 / absdot);
    wi_dist = wi_dist - 1e-4f;
    wi_dist = wi_dist < 0.0f ? 0.0f : wi_dist;
    float4 e = __ldg(&s.ml_emission[k]);
    return mk(e.x, e.y, e.z) / pdf;
}

KS_D float mesh_light_pdf(const SceneView &s, uint32_t k, const TriVerts &tv, f3 wi, float wi_dist)
{
    if (wi_dist == 0.0f)
        return 0.0f;
    f3 n = light_normal(tv.v0, tv.v1, tv.v2);
    float pdf = 1.0f / s.ml_area[k];
    float absdot = fabsf(dot(n, wi));
    if (absdot == 0.0f)
        return 0.0f;
    pdf *= (sqr(wi_dist) / absdot);
    return pdf;
}

} // namespace ksb
