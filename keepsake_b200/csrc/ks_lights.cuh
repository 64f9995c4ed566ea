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
    const float4 *tex_texels;        // textures: linear float texels
    const TexInfo *tex_info;         // per texture
    const BindingGPU *bindings;      // per material binding (MaterialGPU::bind_begin / bind_count)
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
    int sky_kind; // 0 none, 1 ambient, 2 lat-long map, 3 equal-area map (sky_w = sky_h = res)
    int sky_w, sky_h;
    float sky_l2w[9], sky_w2l[9];
    int sky_y_up;
    float sky_strength;
    const float4 *sky_map;
    const float *sky_cond;   // sky_h rows of sky_w + 1
    const float *sky_margin; // sky_h + 1
    const uint32_t *sky_cond_guide;   // sky_h rows of kGuide
    const uint32_t *sky_margin_guide; // kGuide
    const float4 *sky_alias;          // equal-area map: res^2 alias-table bins (q, p, alias bits, 0)
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

KS_D f3 latlong_sky_eval(const SceneView &s, f3 wi)
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

KS_D f3 latlong_sky_sample(const SceneView &s, float u0, float u1, f3 &wi, float &wi_dist, float &pdf)
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
    return latlong_sky_eval(s, wi) / pdf;
}

KS_D float latlong_sky_pdf(const SceneView &s, f3 wi)
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

// ---- equal-area sky (EqualAreaSkyLight: light.cpp:161-206; sample / pdf / eval as the
// reference's GPU path defines them, gpu/shaders/light.slang:92-186) ------------------------------
// The map is a res x res square in the equal-area octahedral parameterisation of the sphere; a
// direction is drawn by an alias table over the texels' luminance, then uniformly inside the texel
// (the second uniform split into two by bit de-interleaving), so the density is constant per texel.

// equal_area_square_to_sphere (gpu/shaders/common.slang:245-265; pbrt-v4's mapping)
KS_D f3 ea_square_to_sphere(float px, float py)
{
    float u = 2 * px - 1, v = 2 * py - 1;
    float up = fabsf(u), vp = fabsf(v);
    float signed_distance = 1 - (up + vp);
    float d = fabsf(signed_distance);
    float r = 1 - d;
    float phi = (r == 0 ? 1 : (vp - up) / r + 1) * kPi / 4;
    float z = copysignf(1 - sqr(r), signed_distance);
    float cos_phi = copysignf(cosf(phi), u);
    float sin_phi = copysignf(sinf(phi), v);
    float s2 = 2 - sqr(r);
    float st = r * sqrtf(s2 > 0.0f ? s2 : 0.0f);
    return mk(cos_phi * st, sin_phi * st, z);
}

// equal_area_sphere_to_square (gpu/shaders/common.slang:267-322): Clarberg's inverse with a 6th
// degree minimax polynomial for atan(x) 2 / pi, evaluated with fused multiply-adds
KS_D void ea_sphere_to_square(f3 dir, float &ou, float &ov)
{
    float x = fabsf(dir.x), y = fabsf(dir.y), z = fabsf(dir.z);
    float r2 = 1 - z;
    float r = sqrtf(r2 > 0.0f ? r2 : 0.0f);
    float a = fmaxf(x, y), b = fminf(x, y);
    b = a == 0 ? 0 : b / a;
    const float t1 = 0.406758566246788489601959989e-5f, t2 = 0.636226545274016134946890922156f,
                t3 = 0.61572017898280213493197203466e-2f, t4 = -0.247333733281268944196501420480f,
                t5 = 0.881770664775316294736387951347e-1f, t6 = 0.419038818029165735901852432784e-1f,
                t7 = -0.251390972343483509333252996350e-1f;
    float phi = fmaf(t7, b, t6);
    phi = fmaf(phi, b, t5);
    phi = fmaf(phi, b, t4);
    phi = fmaf(phi, b, t3);
    phi = fmaf(phi, b, t2);
    phi = fmaf(phi, b, t1);
    if (x < y)
        phi = 1 - phi;
    float v = phi * r;
    float u = r - v;
    if (dir.z < 0) {
        const float t = u;
        u = 1 - v;
        v = 1 - t;
    }
    u = copysignf(u, dir.x);
    v = copysignf(v, dir.y);
    ou = 0.5f * (u + 1);
    ov = 0.5f * (v + 1);
}

// equal_area_bilerp (gpu/shaders/common.slang:350-395): the four texels around uv with bilinear
// weights, folded across the square's edges the way the octahedral parameterisation wraps
KS_D void ea_bilerp(float ux, float uy, int N, int ix[4], int iy[4], float w[4])
{
    float x = ux * N - 0.5f, y = uy * N - 0.5f;
    int x0 = (int)floorf(x), y0 = (int)floorf(y);
    float tx = x - x0, ty = y - y0;
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = x0 < 0 ? 0 : (x0 > N - 1 ? N - 1 : x0);
    y0 = y0 < 0 ? 0 : (y0 > N - 1 ? N - 1 : y0);
    x1 = x1 < 0 ? 0 : (x1 > N - 1 ? N - 1 : x1);
    y1 = y1 < 0 ? 0 : (y1 > N - 1 ? N - 1 : y1);
    w[0] = (1.0f - tx) * (1.0f - ty);
    w[1] = tx * (1.0f - ty);
    w[2] = (1.0f - tx) * ty;
    w[3] = tx * ty;
    const int xs[4] = {x0, x1, x0, x1}, ys[4] = {y0, y0, y1, y1}, m = N - 1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const bool mirror = ((xs[k] ^ ys[k]) & N) != 0;
        const int a = xs[k] & m, b = ys[k] & m;
        ix[k] = mirror ? m - a : a;
        iy[k] = mirror ? m - b : b;
    }
}

// demux_float (gpu/shaders/common.slang:569-576): the even and odd bits of f's 32-bit fixed-point
// form, each as a 16-bit fraction
KS_D uint32_t compact_1_by_1(uint32_t x)
{
    x &= 0x55555555u;
    x = (x ^ (x >> 1)) & 0x33333333u;
    x = (x ^ (x >> 2)) & 0x0f0f0f0fu;
    x = (x ^ (x >> 4)) & 0x00ff00ffu;
    x = (x ^ (x >> 8)) & 0x0000ffffu;
    return x;
}

KS_D void demux_float(float f, float &a, float &b)
{
    const uint32_t v = (uint32_t)(f * 4294967296.0f);
    a = (float)compact_1_by_1(v) / 65536.0f;
    b = (float)compact_1_by_1(v >> 1) / 65536.0f;
}

// EqualAreaSkyLight::eval(p_square) (light.slang:160-178): texels read at their centres
KS_D f3 ea_sky_eval_square(const SceneView &s, float px, float py)
{
    int ix[4], iy[4];
    float w[4];
    ea_bilerp(px, py, s.sky_w, ix, iy, w);
    f3 L = mk(0, 0, 0);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        L += w[k] * sky_texel(s, ix[k], iy[k]);
    L *= s.sky_strength;
    return L;
}

KS_D f3 ea_sky_eval(const SceneView &s, f3 wi)
{
    const f3 wl = mat3_apply(s.sky_w2l, wi); // the transposed rotation (light.slang:153-156)
    float px, py;
    ea_sphere_to_square(wl, px, py);
    return ea_sky_eval_square(s, px, py);
}

// AliasTable::sample (distrib.cpp:167-193; gpu/shaders/alias_table.slang): bins (q, p, alias, -)
KS_D uint32_t alias_sample(const float4 *bins, uint32_t n, float u, float &pmf)
{
    const float un = u * (float)n;
    uint32_t offset = (uint32_t)floorf(un);
    offset = offset < n - 1 ? offset : n - 1;
    float up = un - (float)offset;
    up = up < kOneMinusEps ? up : kOneMinusEps;
    const float4 b = __ldg(&bins[offset]);
    if (up < b.x) {
        pmf = b.y;
        return offset;
    }
    const uint32_t alias = __float_as_uint(b.z);
    pmf = __ldg(&bins[alias]).y;
    return alias;
}

// EqualAreaSkyLight::sample (light.slang:114-135)
KS_D f3 ea_sky_sample(const SceneView &s, float u0, float u1, f3 &wi, float &wi_dist, float &pdf)
{
    const uint32_t res = (uint32_t)s.sky_w;
    float pmf;
    const uint32_t index = alias_sample(s.sky_alias, res * res, u0, pmf);
    const uint32_t iy = index / res, ix = index % res;
    float dx, dy;
    demux_float(u1, dx, dy);
    const float px = ((float)ix + dx) / (float)res, py = ((float)iy + dy) / (float)res;
    pdf = pmf * (float)(res * res) / (4.0f * kPi);
    wi = mat3_apply(s.sky_l2w, ea_square_to_sphere(px, py));
    wi_dist = kInf;
    if (pdf == 0.0f)
        return mk(0, 0, 0);
    return ea_sky_eval_square(s, px, py) / pdf;
}

// EqualAreaSkyLight::pdf (light.slang:138-150)
KS_D float ea_sky_pdf(const SceneView &s, f3 wi)
{
    const int res = s.sky_w;
    const f3 wl = mat3_apply(s.sky_w2l, wi);
    float px, py;
    ea_sphere_to_square(wl, px, py);
    int iy = (int)floorf(py * res), ix = (int)floorf(px * res);
    iy = iy < 0 ? 0 : (iy > res - 1 ? res - 1 : iy);
    ix = ix < 0 ? 0 : (ix > res - 1 ? res - 1 : ix);
    return __ldg(&s.sky_alias[(size_t)iy * res + ix]).y * (float)(res * res) / (4.0f * kPi);
}

// The scene's sky light, lat-long (SkyLight) or equal-area (EqualAreaSkyLight).
KS_D f3 sky_eval(const SceneView &s, f3 wi)
{
    return s.sky_kind == 3 ? ea_sky_eval(s, wi) : latlong_sky_eval(s, wi);
}
KS_D f3 sky_sample(const SceneView &s, float u0, float u1, f3 &wi, float &wi_dist, float &pdf)
{
    return s.sky_kind == 3 ? ea_sky_sample(s, u0, u1, wi, wi_dist, pdf)
                           : latlong_sky_sample(s, u0, u1, wi, wi_dist, pdf);
}
KS_D float sky_pdf(const SceneView &s, f3 wi)
{
    return s.sky_kind == 3 ? ea_sky_pdf(s, wi) : latlong_sky_pdf(s, wi);
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

// MeshTriLight::eval (light.cpp:560-565): the emission of mesh light k at barycentrics (u, v) of its
// triangle; a constant, or the emission texture (ml_emission.w holds its binding, -1 for none) at
// the texture coordinate there: the mesh's texcoords interpolated, else the barycentrics for a hit
// (compute_intersection) and zero for a light sample (interpolate_texcoord, geometry.cpp:182-191).
KS_D f3 mesh_light_Le(const SceneView &s, uint32_t k, float u, float v, bool bary_fallback)
{
    const float4 e = __ldg(&s.ml_emission[k]);
    const int b = __float_as_int(e.w);
    if (b < 0)
        return mk(e.x, e.y, e.z);
    const uint32_t tri = __ldg(&s.ml_tri[k]);
    float tu = bary_fallback ? u : 0.0f, tv = bary_fallback ? v : 0.0f;
    if (__ldg(&s.mesh_flags[__ldg(&s.tri_mesh[tri])]) & kMeshTexcoords) {
        const float2 *tc = reinterpret_cast<const float2 *>(s.texcoords);
        const uint32_t i0 = __ldg(&s.indices[3 * (size_t)tri]), i1 = __ldg(&s.indices[3 * (size_t)tri + 1]),
                       i2 = __ldg(&s.indices[3 * (size_t)tri + 2]);
        const float2 t0 = __ldg(&tc[i0]), t1 = __ldg(&tc[i1]), t2 = __ldg(&tc[i2]);
        const float w = 1.0f - u - v;
        tu = w * t0.x + u * t1.x + v * t2.x;
        tv = w * t0.y + u * t1.y + v * t2.y;
    }
    const float4 c = field_eval(s.tex_texels, s.tex_info, s.bindings[b], tu, tv);
    return mk(c.x, c.y, c.z);
}

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
    return mesh_light_Le(s, k, b0, b1, false) / pdf;
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
