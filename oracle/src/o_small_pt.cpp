// ORACLE (test infrastructure only).  CPU restatement of keepsake's small_pt path:
//
//   SmallPT::run / trace          small_pt.cpp:15-178
//   next_event_estimate           nee.cpp:11-57, power_heur nee.h:18-23
//   Material::sample_with_nee     material.cpp:101-167 (subsurface: o_subsurface.h)
//   Camera::spawn_ray             camera.cpp:129-170 (perspective, no ray differentials: the
//                                 constant shader fields never read them)
//   pixel filters                 render_target.h:79-180 (box, Gaussian, Blackman-Harris)
//   MeshGeometry::compute_intersection  geometry.cpp:68-163 (texcoord tangents, smooth normals)
//   transform_it / Transform::frame      ray.h:166-183, maths.h:989-996
//   SkyLight                      light.cpp:19-159 (in-memory lat-long map instead of a file)
//   MeshLightShared / MeshTriLight light.cpp:307-628 (constant emission: uniform importance)
//   PowerLightSampler             light.cpp:636-701
//   DistribTable / DistribTable2D distrib.cpp:9-107
//   RenderTarget2::add / add_miss render_target.cpp:82-107 (FP64 accumulation)
//
// Ray queries go through the reference's own SBVH (cuda/sbvh.cu, oracle/_ref).
// The two float atomics of the reference (the sky luminance threshold light.cpp:35-48 and the
// sky power light.cpp:136-159) have no fixed order there; here both are summed in a fixed order
// (rows sequentially in double) so the product can reproduce them exactly.
#include "../../include/ks_b200.h"
#include "o_bsdf.h"
#include "o_texture.h"
#include "o_subsurface.h"
#include "o_math.h"
#include "o_sampler.h"

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

extern "C" {
int ksref_sbvh_build(const float *, uint32_t, const uint32_t *, uint32_t, uint32_t, uint32_t, float, float, void **,
                     uint32_t *, uint32_t *);
uint32_t ksref_sbvh_intersect1(void *, const float *, int, float *, float *);
uint32_t ksref_sbvh_intersect1_counted(void *, const float *, int, int, float *, float *, uint64_t *,
                                       int (*)(void *, uint32_t, float, float), void *);
void ksref_sbvh_bound(void *, float *);
void ksref_sbvh_destroy(void *);
}

namespace oracle
{

// ---- DistribTable (distrib.cpp:9-75) ----------------------------------------------------------
struct DistribTable
{
    std::vector<float> cdf;
    float acc = 0.0f;
    DistribTable() = default;
    DistribTable(const float *f, uint32_t n) : cdf(n + 1)
    {
        cdf[0] = 0;
        float invn = 1.0f / (float)n;
        for (uint32_t i = 1; i < n + 1; ++i)
            cdf[i] = cdf[i - 1] + f[i - 1] * invn;
        acc = cdf[n];
        if (acc == 0.0f) {
            for (uint32_t i = 0; i < n + 1; ++i)
                cdf[i] = (float)i / (float)n;
        } else {
            float invacc = 1.0f / acc;
            for (uint32_t i = 0; i < n + 1; ++i)
                cdf[i] *= invacc;
        }
        cdf[n] = 1.0f;
    }
    uint32_t sample(float u, float &prob) const
    {
        u = std::clamp(u, 0.0f, std::nextafter(1.0f, 0.0f));
        auto it = std::upper_bound(cdf.begin(), cdf.end(), u);
        uint32_t index = (uint32_t)std::distance(cdf.begin(), std::prev(it));
        prob = cdf[index + 1] - cdf[index];
        return index;
    }
    float sample_linear(float u, float &pdf, uint32_t &index) const
    {
        u = std::clamp(u, 0.0f, std::nextafter(1.0f, 0.0f));
        auto it = std::upper_bound(cdf.begin(), cdf.end(), u);
        index = (uint32_t)std::distance(cdf.begin(), std::prev(it));
        float n = (float)(cdf.size() - 1);
        pdf = (cdf[index + 1] - cdf[index]) * n;
        float du = (u - cdf[index]) / (cdf[index + 1] - cdf[index]);
        return (index + du) / n;
    }
    float pdf(uint32_t index) const
    {
        uint32_t n = (uint32_t)(cdf.size() - 1);
        return (cdf[index + 1] - cdf[index]) * (float)n;
    }
};

struct DistribTable2D
{
    std::vector<DistribTable> cond;
    DistribTable margin;
    DistribTable2D() = default;
    DistribTable2D(const float *f, uint32_t nx, uint32_t ny)
    {
        cond.resize(ny);
        for (uint32_t y = 0; y < ny; ++y)
            cond[y] = DistribTable(f + (size_t)y * nx, nx);
        std::vector<float> marginPmf(ny);
        for (uint32_t y = 0; y < ny; ++y)
            marginPmf[y] = cond[y].acc;
        margin = DistribTable(marginPmf.data(), ny);
    }
    void sample_linear(float u0, float u1, float &pdf, float &s0, float &s1) const
    {
        float pdfMargin, pdfCond;
        uint32_t uIndex, vIndex;
        float vSample = margin.sample_linear(u1, pdfMargin, vIndex);
        float uSample = cond[vIndex].sample_linear(u0, pdfCond, uIndex);
        pdf = pdfMargin * pdfCond;
        s0 = uSample;
        s1 = vSample;
    }
    float pdf(float p0, float p1) const
    {
        int x = std::clamp(int(p0 * (cond[0].cdf.size() - 1)), 0, (int)cond[0].cdf.size() - 2);
        int y = std::clamp(int(p1 * cond.size()), 0, (int)cond.size() - 1);
        return margin.pdf(y) * cond[y].pdf(x);
    }
};

// GaussianPixelFilter / BlackmanHarrisPixelFilter::eval (render_target.h:127-180; gaussian(),
// maths.h:1070-1073) tabulated as PixelFilterSampleTable (render_target.h:79-106): n = ceil(32 r)
// cells per side over [-r, r]^2, sampled through DistribTable2D::sample_linear.
struct PixelFilterTable
{
    float r = 0.5f;
    uint32_t n = 0;
    DistribTable2D distrib;
    PixelFilterTable(int type, float width, float sigma) : r(0.5f * width)
    {
        if (type == 0)
            return;
        const float pi = 3.14159265359f, two_pi = 6.28318530718f;
        auto gaussian = [&](float x, float mu) {
            return 1.0f / std::sqrt(two_pi * sigma * sigma) * std::exp(-((x - mu) * (x - mu)) / (2.0f * sigma * sigma));
        };
        const float threshold = gaussian(r, 0.0f);
        auto eval = [&](float x, float y) {
            if (x < -r || x > r || y < -r || y > r)
                return 0.0f;
            if (type == 1)
                return (gaussian(x, 0.0f) - threshold) * (gaussian(y, 0.0f) - threshold);
            const float a0 = 0.35875f, a1 = 0.48829f, a2 = 0.14128f, a3 = 0.01168f;
            float tx = (x + r) / (2.0f * r);
            float fx = a0 - a1 * std::cos(2.0f * pi * tx) + a2 * std::cos(4.0f * pi * tx) - a3 * std::cos(6.0f * pi * tx);
            float ty = (y + r) / (2.0f * r);
            float fy = a0 - a1 * std::cos(2.0f * pi * ty) + a2 * std::cos(4.0f * pi * ty) - a3 * std::cos(6.0f * pi * ty);
            return fx * fy;
        };
        n = (uint32_t)(int)std::ceil(32 * r);
        std::vector<float> f((size_t)n * n);
        for (uint32_t y = 0; y < n; ++y)
            for (uint32_t x = 0; x < n; ++x)
                f[(size_t)y * n + x] = eval(std::lerp(-r, r, (x + 0.5f) / n), std::lerp(-r, r, (y + 0.5f) / n));
        distrib = DistribTable2D(f.data(), n, n);
    }
    // PixelFilterSampleTable::sample / BoxPixelFilter::sample: lerp(-r, r, .) = (1 - t) * -r + t * r
    void sample(float u0, float u1, float &offx, float &offy) const
    {
        if (n) {
            float pdf;
            distrib.sample_linear(u0, u1, pdf, u0, u1);
        }
        offx = (1.0f - u0) * -r + u0 * r;
        offy = (1.0f - u1) * -r + u1 * r;
    }
};

// ---- SkyLight -----------------------------------------------------------------------------------
// ---- EqualAreaSkyLight (light.cpp:161-206; its sample / pdf / eval are defined by the reference's
// GPU path, gpu/shaders/light.slang:92-186, which this restates) ---------------------------------
// equal_area_square_to_sphere (gpu/shaders/common.slang:245-265)
inline V3 ea_square_to_sphere(float px, float py)
{
    float u = 2 * px - 1, v = 2 * py - 1;
    float up = std::abs(u), vp = std::abs(v);
    float signed_distance = 1 - (up + vp);
    float d = std::abs(signed_distance);
    float r = 1 - d;
    float phi = (r == 0 ? 1 : (vp - up) / r + 1) * pi / 4;
    float z = std::copysign(1 - sqr(r), signed_distance);
    float cos_phi = std::copysign(std::cos(phi), u);
    float sin_phi = std::copysign(std::sin(phi), v);
    return V3(cos_phi * r * safe_sqrt(2 - sqr(r)), sin_phi * r * safe_sqrt(2 - sqr(r)), z);
}

// equal_area_sphere_to_square (gpu/shaders/common.slang:267-322)
inline void ea_sphere_to_square(V3 d, float &ou, float &ov)
{
    float x = std::abs(d.x), y = std::abs(d.y), z = std::abs(d.z);
    float r = safe_sqrt(1 - z);
    float a = std::max(x, y), b = std::min(x, y);
    b = a == 0 ? 0 : b / a;
    const float t1 = 0.406758566246788489601959989e-5f, t2 = 0.636226545274016134946890922156f,
                t3 = 0.61572017898280213493197203466e-2f, t4 = -0.247333733281268944196501420480f,
                t5 = 0.881770664775316294736387951347e-1f, t6 = 0.419038818029165735901852432784e-1f,
                t7 = -0.251390972343483509333252996350e-1f;
    float phi = std::fma(t7, b, t6);
    phi = std::fma(phi, b, t5);
    phi = std::fma(phi, b, t4);
    phi = std::fma(phi, b, t3);
    phi = std::fma(phi, b, t2);
    phi = std::fma(phi, b, t1);
    if (x < y)
        phi = 1 - phi;
    float v = phi * r;
    float u = r - v;
    if (d.z < 0) {
        std::swap(u, v);
        u = 1 - u;
        v = 1 - v;
    }
    u = std::copysign(u, d.x);
    v = std::copysign(v, d.y);
    ou = 0.5f * (u + 1);
    ov = 0.5f * (v + 1);
}

// equal_area_bilerp (gpu/shaders/common.slang:350-395)
inline void ea_bilerp(float ux, float uy, int N, int ix[4], int iy[4], float w[4])
{
    float x = ux * N - 0.5f, y = uy * N - 0.5f;
    int x0 = (int)std::floor(x), y0 = (int)std::floor(y);
    float tx = x - x0, ty = y - y0;
    int x1 = x0 + 1, y1 = y0 + 1;
    x0 = std::clamp(x0, 0, N - 1);
    y0 = std::clamp(y0, 0, N - 1);
    x1 = std::clamp(x1, 0, N - 1);
    y1 = std::clamp(y1, 0, N - 1);
    float inv_tx = 1.0f - tx, inv_ty = 1.0f - ty;
    w[0] = inv_tx * inv_ty;
    w[1] = tx * inv_ty;
    w[2] = inv_tx * ty;
    w[3] = tx * ty;
    const int xs[4] = {x0, x1, x0, x1}, ys[4] = {y0, y0, y1, y1}, n1 = N - 1;
    for (int k = 0; k < 4; ++k) {
        bool mirror = (xs[k] ^ ys[k]) & N;
        int a = xs[k] & n1, b = ys[k] & n1;
        ix[k] = mirror ? n1 - a : a;
        iy[k] = mirror ? n1 - b : b;
    }
}

// compact_1_by_1 / demux_float (gpu/shaders/common.slang:529-537, 569-576)
inline uint32_t compact_1_by_1(uint32_t x)
{
    x &= 0x55555555u;
    x = (x ^ (x >> 1)) & 0x33333333u;
    x = (x ^ (x >> 2)) & 0x0f0f0f0fu;
    x = (x ^ (x >> 4)) & 0x00ff00ffu;
    x = (x ^ (x >> 8)) & 0x0000ffffu;
    return x;
}
inline void demux_float(float f, float &a, float &b)
{
    uint32_t v = (uint32_t)(f * (float)(1ull << 32));
    a = compact_1_by_1(v) / float(1 << 16);
    b = compact_1_by_1(v >> 1) / float(1 << 16);
}

// AliasTable (distrib.cpp:109-193)
struct AliasTable
{
    struct Bin
    {
        float q = 0, p = 0;
        int alias = -1;
    };
    std::vector<Bin> bins;
    AliasTable() = default;
    explicit AliasTable(const std::vector<float> &weights) : bins(weights.size())
    {
        double sum = std::accumulate(weights.begin(), weights.end(), 0.);
        for (size_t i = 0; i < weights.size(); ++i)
            bins[i].p = weights[i] / sum;
        struct Outcome
        {
            float pHat;
            size_t index;
        };
        std::vector<Outcome> under, over;
        for (size_t i = 0; i < bins.size(); ++i) {
            float pHat = bins[i].p * bins.size();
            if (pHat < 1)
                under.push_back(Outcome{pHat, i});
            else
                over.push_back(Outcome{pHat, i});
        }
        while (!under.empty() && !over.empty()) {
            Outcome un = under.back(), ov = over.back();
            under.pop_back();
            over.pop_back();
            bins[un.index].q = un.pHat;
            bins[un.index].alias = (int)ov.index;
            float pExcess = un.pHat + ov.pHat - 1;
            if (pExcess < 1)
                under.push_back(Outcome{pExcess, ov.index});
            else
                over.push_back(Outcome{pExcess, ov.index});
        }
        while (!over.empty()) {
            Outcome ov = over.back();
            over.pop_back();
            bins[ov.index].q = 1;
            bins[ov.index].alias = -1;
        }
        while (!under.empty()) {
            Outcome un = under.back();
            under.pop_back();
            bins[un.index].q = 1;
            bins[un.index].alias = -1;
        }
    }
    int sample(float u, float *pmf) const
    {
        size_t offset = std::min((size_t)std::floor(u * bins.size()), bins.size() - 1);
        float up = std::min(u * bins.size() - offset, fp32_before_one);
        if (up < bins[offset].q) {
            *pmf = bins[offset].p;
            return (int)offset;
        }
        int alias = bins[offset].alias;
        *pmf = bins[alias].p;
        return alias;
    }
};

struct Sky
{
    int kind = 0; // 1 ambient, 2 lat-long map, 3 equal-area map
    AliasTable ea_pmf; // kind 3: over the texels' luminance
    int w = 1, h = 1;
    std::vector<V3> map; // row-major, map(u, v) = map[v * w + u]
    float l2w[16], w2l[16];
    bool y_up = true;
    float strength = 1.0f;
    DistribTable2D distrib;

    static void to_spherical_yup(V3 d, float &phi, float &theta)
    {
        theta = std::acos(std::clamp(d.y, -1.0f, 1.0f));
        phi = std::atan2(d.z, d.x);
        if (phi < 0.0f)
            phi += two_pi;
    }
    static void to_spherical(V3 d, float &phi, float &theta)
    {
        theta = std::acos(std::clamp(d.z, -1.0f, 1.0f));
        phi = std::atan2(d.y, d.x);
        if (phi < 0.0f)
            phi += two_pi;
    }
    static V3 to_cartesian_yup(float phi, float theta)
    {
        float ct = std::cos(theta), st = std::sin(theta), cp = std::cos(phi), sp = std::sin(phi);
        return V3(cp * st, ct, sp * st);
    }
    static V3 to_cartesian(float phi, float theta)
    {
        float ct = std::cos(theta), st = std::sin(theta), cp = std::cos(phi), sp = std::sin(phi);
        return V3(cp * st, sp * st, ct);
    }
    // lerp_helper (maths.h:760-780), TickMode::Middle
    static void lerp_helper(float u, int res, bool repeat, int &u0, int &u1, float &t)
    {
        float u_scaled = u * (float)res - 0.5f;
        u0 = (int)std::floor(u_scaled);
        u1 = u0 + 1;
        t = u_scaled - u0;
        if (repeat) {
            u0 = (u0 + res) % res;
            u1 = (u1 + res) % res;
        } else {
            u0 = std::clamp(u0, 0, res - 1);
            u1 = std::clamp(u1, 0, res - 1);
        }
    }
    V3 at(int u, int v) const { return map[(size_t)v * w + u]; }
    // kind 3 (light.slang:138-178): the light-to-world rotation's transpose takes wi to the map
    V3 ea_local(V3 wi) const
    {
        return V3(l2w[0] * wi.x + l2w[4] * wi.y + l2w[8] * wi.z, l2w[1] * wi.x + l2w[5] * wi.y + l2w[9] * wi.z,
                  l2w[2] * wi.x + l2w[6] * wi.y + l2w[10] * wi.z);
    }
    V3 ea_eval_square(float px, float py) const
    {
        int ix[4], iy[4];
        float wt[4];
        ea_bilerp(px, py, w, ix, iy, wt);
        V3 L;
        for (int k = 0; k < 4; ++k)
            L += wt[k] * at(ix[k], iy[k]);
        L *= strength;
        return L;
    }
    V3 eval(V3 wi) const
    {
        if (kind == 3) {
            float px, py;
            ea_sphere_to_square(ea_local(wi), px, py);
            return ea_eval_square(px, py);
        }
        V3 wl = transform_dir(w2l, wi);
        float phi, theta;
        if (y_up)
            to_spherical_yup(wl, phi, theta);
        else
            to_spherical(wl, phi, theta);
        float uv0 = phi * inv_pi * 0.5f, uv1 = theta * inv_pi;
        int u0, u1, v0, v1;
        float t0, t1;
        lerp_helper(uv0, w, true, u0, u1, t0);
        lerp_helper(uv1, h, false, v0, v1, t1);
        V3 L;
        L += (1.0f - t0) * (1.0f - t1) * at(u0, v0);
        L += (1.0f - t0) * t1 * at(u0, v1);
        L += t0 * (1.0f - t1) * at(u1, v0);
        L += t0 * t1 * at(u1, v1);
        L *= strength;
        return L;
    }
    V3 sample(float u0, float u1, V3 &wi, float &wi_dist, float &pdf) const
    {
        if (kind == 3) {
            float pmf;
            int index = ea_pmf.sample(u0, &pmf);
            int iy = index / w, ix = index % w;
            float dx, dy;
            demux_float(u1, dx, dy);
            float px = (ix + dx) / w, py = (iy + dy) / w;
            pdf = pmf * sqr((float)w) / (4.0f * pi);
            V3 wl = ea_square_to_sphere(px, py);
            wi = V3(l2w[0] * wl.x + l2w[1] * wl.y + l2w[2] * wl.z, l2w[4] * wl.x + l2w[5] * wl.y + l2w[6] * wl.z,
                    l2w[8] * wl.x + l2w[9] * wl.y + l2w[10] * wl.z);
            wi_dist = inf;
            if (pdf == 0.0f)
                return V3();
            return ea_eval_square(px, py) / pdf;
        }
        float s0, s1;
        distrib.sample_linear(u0, u1, pdf, s0, s1);
        if (pdf == 0.0f)
            return V3();
        float phi = s0 * 2.0f * pi;
        float theta = s1 * pi;
        V3 wl = y_up ? to_cartesian_yup(phi, theta) : to_cartesian(phi, theta);
        float sin_theta = std::sin(theta);
        pdf /= (2.0f * pi * pi * sin_theta);
        if (sin_theta == 0.0f) {
            pdf = 0.0f;
            return V3();
        }
        wi = transform_dir(l2w, wl);
        wi_dist = inf;
        return eval(wi) / pdf;
    }
    float pdf(V3 wi) const
    {
        if (kind == 3) {
            float px, py;
            ea_sphere_to_square(ea_local(wi), px, py);
            int iy = std::clamp((int)std::floor(py * w), 0, w - 1);
            int ix = std::clamp((int)std::floor(px * w), 0, w - 1);
            return ea_pmf.bins[(size_t)iy * w + ix].p * sqr((float)w) / (4.0f * pi);
        }
        V3 wl = transform_dir(w2l, wi);
        float phi, theta;
        if (y_up)
            to_spherical_yup(wl, phi, theta);
        else
            to_spherical(wl, phi, theta);
        float sin_theta = std::sin(theta);
        if (sin_theta == 0.0f)
            return 0.0f;
        float p = distrib.pdf(phi * inv_pi * 0.5f, theta * inv_pi);
        p /= (2.0f * pi * pi * sin_theta);
        return p;
    }
    // SkyLight::power (light.cpp:136-159); the rows' float sums are added in row order in double.
    V3 power(const float bound[6]) const
    {
        if (kind == 3) {
            // EqualAreaSkyLight::unit_power / power (light.cpp:182-206): float row sums, the rows
            // added in row order in double
            double sum[3] = {0, 0, 0};
            for (int row = 0; row < w; ++row) {
                V3 row_sum;
                for (int col = 0; col < w; ++col)
                    row_sum += at(col, row);
                for (int c = 0; c < 3; ++c)
                    sum[c] += row_sum[c];
            }
            V3 Phi((float)sum[0], (float)sum[1], (float)sum[2]);
            Phi *= (4 * pi) / sqr((float)w);
            V3 ext(bound[3] - bound[0], bound[4] - bound[1], bound[5] - bound[2]);
            float scene_radius = 0.5f * norm(ext);
            Phi *= pi * sqr(scene_radius);
            return Phi;
        }
        double sum[3] = {0, 0, 0};
        for (int row = 0; row < h; ++row) {
            float theta = (row + 0.5f) / (float)h * pi;
            float sin_theta = std::sin(theta);
            V3 row_sum;
            for (int col = 0; col < w; ++col) {
                float phi = (col + 0.5f) / (float)w * two_pi;
                V3 dir = to_cartesian(phi, theta);
                row_sum += eval(dir) * sin_theta;
            }
            for (int c = 0; c < 3; ++c)
                sum[c] += row_sum[c];
        }
        V3 Phi((float)sum[0], (float)sum[1], (float)sum[2]);
        Phi *= (pi / h) * (two_pi / w);
        V3 ext(bound[3] - bound[0], bound[4] - bound[1], bound[5] - bound[2]);
        float scene_radius = 0.5f * norm(ext);
        Phi *= pi * sqr(scene_radius);
        return Phi;
    }
};

inline bool invert_rigid_or_general(const float *m, float *out)
{
    double a[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 8; ++c)
            a[r][c] = c < 4 ? m[4 * r + c] : (c - 4 == r ? 1.0 : 0.0);
    for (int col = 0; col < 4; ++col) {
        int piv = col;
        for (int r = col + 1; r < 4; ++r)
            if (std::fabs(a[r][col]) > std::fabs(a[piv][col]))
                piv = r;
        if (a[piv][col] == 0.0)
            return false;
        for (int c = 0; c < 8; ++c)
            std::swap(a[piv][c], a[col][c]);
        double inv = 1.0 / a[col][col];
        for (int c = 0; c < 8; ++c)
            a[col][c] *= inv;
        for (int r = 0; r < 4; ++r)
            if (r != col) {
                double f = a[r][col];
                for (int c = 0; c < 8; ++c)
                    a[r][c] -= f * a[col][c];
            }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
            out[4 * r + c] = (float)a[r][c + 4];
    return true;
}

// ---- mesh lights (light.cpp:307-628) ------------------------------------------------------------
struct MeshLight
{
    uint32_t mesh = 0;
    V3 emission;
    int em_binding = -1; // the emission texture's binding in the material's list, -1: constant
    std::vector<uint32_t> prim_ids; // local triangle ids of the mesh
    std::vector<float> importance;
    std::vector<float> areas;
};

// ---- scene ------------------------------------------------------------------------------------
struct Scene
{
    std::vector<float> verts;
    std::vector<uint32_t> idx;
    std::vector<uint32_t> tri_mesh;
    std::vector<uint32_t> mesh_tri_off;
    std::vector<uint32_t> mesh_material;
    std::vector<int> mesh_twosided, mesh_smooth, mesh_uv;
    std::vector<float> normals;   // 3 per vertex (zeros for meshes without)
    std::vector<float> texcoords; // 2 per vertex (zeros for meshes without)
    std::vector<ks_material_desc> materials;
    std::vector<Texture> textures;
    std::vector<std::vector<Binding>> mat_bindings; // per material, in the order given
    bool any_opacity = false;
    void *bvh = nullptr;
    float bound[6];
    std::unique_ptr<Sky> sky;
    std::vector<MeshLight> mesh_lights;
    std::vector<int32_t> tri_light; // global triangle -> flat light index, -1 if none
    std::vector<uint32_t> index_psum;
    std::vector<ks_light_desc> lights; // point / directional lights, after the sky
    DistribTable power_distrib;
    uint32_t light_count = 0;
    std::vector<float> powers;

    ~Scene()
    {
        if (bvh)
            ksref_sbvh_destroy(bvh);
    }
    V3 vert(uint32_t v) const { return V3(verts[3 * v], verts[3 * v + 1], verts[3 * v + 2]); }
    V3 tri_vert(uint32_t t, int k) const { return vert(idx[3 * t + k]); }

    float probability(uint32_t light_index) const { return power_distrib.pdf(light_index) / (float)light_count; }
};

struct Intersection
{
    float thit;
    V3 p;
    float uv[2]; // the mesh's interpolated texcoords, else the barycentrics of vertices 1 and 2
    Frame frame, sh_frame;
    V3 sh_to_local(V3 w) const
    {
        bool hw = dot(frame.n, w) >= 0.0f;
        V3 l = sh_frame.to_local(w);
        bool hl = l.z >= 0.0f;
        if (hw != hl)
            l.z *= -1.0f;
        return l;
    }
    V3 sh_to_world(V3 l) const
    {
        bool hl = l.z >= 0.0f;
        V3 w = sh_frame.to_world(l);
        bool hw = dot(frame.n, w) >= 0.0f;
        if (hl != hw)
            w -= 2.0f * dot(frame.n, w) * frame.n;
        return w;
    }
};

// Transform::frame with the identity instance transform (maths.h:989-996): re-orthonormalises.
inline Frame identity_transform_frame(const Frame &f)
{
    Frame o;
    o.t = normalized(f.t);
    V3 b = f.b;
    b = normalized(b - dot(b, o.t) * o.t);
    o.b = b;
    o.n = normalized(cross(o.t, o.b));
    return o;
}

// compute_intersection for a triangle hit with barycentrics (w0, w1, w2) (geometry.cpp:68-163).
inline Intersection make_intersection(const Scene &s, uint32_t tri, float t, float w1, float w2, V3 ray_dir)
{
    Intersection it;
    it.thit = t;
    V3 rd = normalized(ray_dir);
    V3 wo_object = -rd;
    V3 p0 = s.tri_vert(tri, 0), p1 = s.tri_vert(tri, 1), p2 = s.tri_vert(tri, 2);
    V3 ng = normalized(cross(p1 - p0, p2 - p0));
    float u = w1, v = w2;
    float w0 = 1.0f - u - v;
    it.p = w0 * p0 + u * p1 + v * p2;
    V3 dpdu = p1 - p0;
    const uint32_t mesh = s.tri_mesh[tri];
    const uint32_t i0 = s.idx[3 * tri], i1 = s.idx[3 * tri + 1], i2 = s.idx[3 * tri + 2];
    it.uv[0] = u;
    it.uv[1] = v;
    if (s.mesh_uv[mesh]) {
        // dP/du of the texture parameterisation (geometry.cpp:94-116)
        const float *tc = s.texcoords.data();
        it.uv[0] = w0 * tc[2 * i0] + u * tc[2 * i1] + v * tc[2 * i2];
        it.uv[1] = w0 * tc[2 * i0 + 1] + u * tc[2 * i1 + 1] + v * tc[2 * i2 + 1];
        float du02 = tc[2 * i0] - tc[2 * i2], dv02 = tc[2 * i0 + 1] - tc[2 * i2 + 1];
        float du12 = tc[2 * i1] - tc[2 * i2], dv12 = tc[2 * i1 + 1] - tc[2 * i2 + 1];
        V3 dp02 = p0 - p2, dp12 = p1 - p2;
        float det = du02 * dv12 - dv02 * du12;
        if (!(std::abs(det) < 1e-8f)) {
            float inv = 1.0f / det;
            dpdu = (dv12 * dp02 - dv02 * dp12) * inv;
        }
    }
    V3 b = normalized(cross(ng, dpdu));
    V3 tt = normalized(cross(b, ng));
    if (s.mesh_twosided[mesh]) {
        if (dot(wo_object, ng) < 0.0f) {
            ng = -ng;
            dpdu = -dpdu;
            tt = -tt;
        }
    }
    it.frame.t = tt;
    it.frame.b = b;
    it.frame.n = ng;
    it.sh_frame = it.frame;
    if (s.mesh_smooth[mesh]) {
        // interpolated vertex normal; a non-finite one keeps the face frame (geometry.cpp:139-156)
        auto nrm = [&](uint32_t k) { return V3(s.normals[3 * k], s.normals[3 * k + 1], s.normals[3 * k + 2]); };
        V3 vn = normalized(w0 * nrm(i0) + u * nrm(i1) + v * nrm(i2));
        if (std::isfinite(vn.x) && std::isfinite(vn.y) && std::isfinite(vn.z)) {
            if (dot(vn, it.frame.n) < 0.0f)
                vn = -vn;
            V3 vb = normalized(cross(vn, dpdu));
            V3 vt = normalized(cross(vb, vn));
            it.sh_frame.t = vt;
            it.sh_frame.b = vb;
            it.sh_frame.n = vn;
        }
    }
    // transform_it with the identity instance transform
    it.frame = identity_transform_frame(it.frame);
    it.sh_frame = identity_transform_frame(it.sh_frame);
    return it;
}

// NormalMap::apply (normal_map.cpp:9-40) to the hit's shading frame.
inline void apply_normal_map(const Scene &s, const Binding &bd, Intersection &it)
{
    float c[4];
    bd.eval(s.textures[bd.b.texture], it.uv[0], it.uv[1], c);
    V3 smp(c[0], c[1], c[2]);
    if (bd.b.range01)
        smp = V3(smp.x * 2.0f - 1.0f, smp.y * 2.0f - 1.0f, smp.z * 2.0f - 1.0f);
    V3 normal = normalized(smp);
    if (bd.b.normal_space == 0 && bd.b.strength < 1.0f)
        normal = normalized(lerp3(V3(0.0f, 0.0f, 1.0f), normal, bd.b.strength));
    V3 n_perturb;
    if (bd.b.normal_space == 0) {
        n_perturb = it.sh_frame.to_world(normal);
    } else {
        // Transform::normal (maths.h:987): the inverse transpose of to_world's 3x3, normalised
        double m[3][3];
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k)
                m[r][k] = bd.b.to_world[4 * r + k];
        const double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                           m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
        // rows of inv^T are the cofactor rows over det
        const double it_[3][3] = {{(m[1][1] * m[2][2] - m[1][2] * m[2][1]) / det,
                                   (m[1][2] * m[2][0] - m[1][0] * m[2][2]) / det,
                                   (m[1][0] * m[2][1] - m[1][1] * m[2][0]) / det},
                                  {(m[0][2] * m[2][1] - m[0][1] * m[2][2]) / det,
                                   (m[0][0] * m[2][2] - m[0][2] * m[2][0]) / det,
                                   (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / det},
                                  {(m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det,
                                   (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / det,
                                   (m[0][0] * m[1][1] - m[0][1] * m[1][0]) / det}};
        float f[9];
        for (int r = 0; r < 3; ++r)
            for (int k = 0; k < 3; ++k)
                f[3 * r + k] = (float)it_[r][k];
        n_perturb = normalized(V3(f[0] * normal.x + f[1] * normal.y + f[2] * normal.z,
                                  f[3] * normal.x + f[4] * normal.y + f[5] * normal.z,
                                  f[6] * normal.x + f[7] * normal.y + f[8] * normal.z));
    }
    V3 bump_deriv = -normal / normal.z;
    V3 t_perturb = normalized(it.sh_frame.t + bump_deriv.x * it.sh_frame.n);
    V3 b_perturb = normalized(cross(n_perturb, t_perturb));
    t_perturb = normalized(cross(b_perturb, n_perturb));
    it.sh_frame.t = t_perturb;
    it.sh_frame.b = b_perturb;
    it.sh_frame.n = n_perturb;
}

// The material at a hit: its textured shader fields (TextureField at the hit's uv) over the constant
// ones; the normal map applied to the hit's shading frame.
inline ks_material_desc textured_material(const Scene &s, uint32_t m, Intersection &it)
{
    ks_material_desc mat = s.materials[m];
    for (const Binding &bd : s.mat_bindings[m]) {
        const int f = bd.b.field;
        if (f == KS_FIELD_OPACITY_MAP || f == KS_FIELD_EMISSION)
            continue;
        if (f == KS_FIELD_NORMAL_MAP) {
            apply_normal_map(s, bd, it);
            continue;
        }
        float c[4];
        bd.eval(s.textures[bd.b.texture], it.uv[0], it.uv[1], c);
        switch (f) {
        case KS_FIELD_BASECOLOR: mat.basecolor[0] = c[0]; mat.basecolor[1] = c[1]; mat.basecolor[2] = c[2]; break;
        case KS_FIELD_ROUGHNESS: mat.roughness = c[0]; break;
        case KS_FIELD_METALLIC: mat.metallic = c[0]; break;
        case KS_FIELD_IOR: mat.ior = c[0]; break;
        case KS_FIELD_SPECULAR_R0_MUL: mat.specular_r0_mul = c[0]; break;
        case KS_FIELD_SPECULAR_TRANS: mat.specular_trans = c[0]; break;
        case KS_FIELD_DIFFUSE_TRANS: mat.diffuse_trans = c[0]; break;
        case KS_FIELD_DIFFUSE_TRANS_FWD: mat.diffuse_trans_fwd = c[0]; break;
        default: mat.specular = c[0]; break;
        }
    }
    return mat;
}

// Work of the ray queries, counted by the restatement of the reference traversal (nodes whose
// bound is tested, triangles tested), and the queries where that restatement's answer differed
// from the reference's own SBVH::intersect / intersectBool (none expected).
struct Work
{
    uint64_t ext[3] = {0, 0, 0}, shadow[3] = {0, 0, 0}; // nodes, triangles, stack overflows
    uint64_t mismatches = 0;
};

// The opacity maps' candidate-hit filter (filter_opacity_map, scene.cpp:175-208, with
// OpacityMap::stochastic_test, opacity_map.cpp:20-30) for one ray.
struct AlphaFilter
{
    const Scene *s;
    V3 ro, rd;
    static int call(void *user, uint32_t tri, float u, float v)
    {
        const AlphaFilter &f = *(const AlphaFilter *)user;
        const Scene &s = *f.s;
        const uint32_t m = s.mesh_material[s.tri_mesh[tri]];
        for (const Binding &bd : s.mat_bindings[m]) {
            if (bd.b.field != KS_FIELD_OPACITY_MAP)
                continue;
            // MeshGeometry::compute_hit_texcoord (geometry.cpp:165-173): zero without texcoords
            float tu = 0.0f, tv = 0.0f;
            const uint32_t mesh = s.tri_mesh[tri];
            if (s.mesh_uv[mesh]) {
                const uint32_t i0 = s.idx[3 * tri], i1 = s.idx[3 * tri + 1], i2 = s.idx[3 * tri + 2];
                const float *tc = s.texcoords.data();
                const float w = 1.0f - u - v;
                tu = w * tc[2 * i0] + u * tc[2 * i1] + v * tc[2 * i2];
                tv = w * tc[2 * i0 + 1] + u * tc[2 * i1 + 1] + v * tc[2 * i2 + 1];
            }
            float c[4];
            bd.eval(s.textures[bd.b.texture], tu, tv, c);
            const float opacity = std::clamp(c[0], 0.0f, 1.0f);
            if (opacity <= 0.0f)
                return 0;
            if (opacity >= 1.0f)
                return 1;
            return hash_float_ray(f.ro, f.rd) < opacity;
        }
        return 1;
    }
};

inline bool intersect(const Scene &s, V3 o, V3 d, float tmax, uint32_t &tri, float &t, float bary[3],
                      Work *work = nullptr)
{
    float r[8] = {o.x, o.y, o.z, 0.0f, d.x, d.y, d.z, tmax};
    if (s.any_opacity) {
        // the reference's SBVH queries take no filter: its traversal restated, with the filter
        AlphaFilter f{&s, o, d};
        uint64_t dummy[3] = {0, 0, 0};
        tri = ksref_sbvh_intersect1_counted(s.bvh, r, 0, 2, &t, bary, work ? work->ext : dummy, AlphaFilter::call, &f);
        return tri != ~0u;
    }
    tri = ksref_sbvh_intersect1(s.bvh, r, 0, &t, bary);
    if (work) {
        float t2 = 0.0f, b2[3] = {0, 0, 0};
        uint32_t tri2 = ksref_sbvh_intersect1_counted(s.bvh, r, 0, 2, &t2, b2, work->ext, nullptr, nullptr);
        if (tri2 != tri || (tri != ~0u && std::memcmp(&t2, &t, sizeof(float)) != 0))
            ++work->mismatches;
    }
    return tri != ~0u;
}
inline bool occluded(const Scene &s, V3 o, V3 d, float tmax, Work *work = nullptr)
{
    float r[8] = {o.x, o.y, o.z, 0.0f, d.x, d.y, d.z, tmax};
    if (s.any_opacity) {
        AlphaFilter f{&s, o, d};
        uint64_t dummy[3] = {0, 0, 0};
        return ksref_sbvh_intersect1_counted(s.bvh, r, 1, 2, nullptr, nullptr, work ? work->shadow : dummy,
                                             AlphaFilter::call, &f) != 0;
    }
    const bool occ = ksref_sbvh_intersect1(s.bvh, r, 1, nullptr, nullptr) != 0;
    if (work && (ksref_sbvh_intersect1_counted(s.bvh, r, 1, 2, nullptr, nullptr, work->shadow, nullptr, nullptr) !=
                 0) != occ)
        ++work->mismatches;
    return occ;
}

// spawn_ray<OffsetType::NextBounce> (ray.h:89-96): returns the offset origin
inline V3 spawn_origin(V3 p, V3 dir, V3 ng) { return offset_ray(p, dot(dir, ng) > 0.0f ? ng : -ng); }

// MeshData::compute_geometry_normal (geometry.h:45-60), then Transform::normal with identity.
inline V3 light_normal(const Scene &s, uint32_t tri)
{
    V3 v0 = s.tri_vert(tri, 0), v1 = s.tri_vert(tri, 1), v2 = s.tri_vert(tri, 2);
    V3 e01 = v1 - v0, e12 = v2 - v1;
    V3 ng = normalized(cross(e01, e12));
    return normalized(ng);
}

// compute_mesh_light_importance (light.cpp:307-522), per triangle: the factor of 2 pi x area.
// Uniform branch (constant emission, no opacity texture): luminance(emission).  Textured branch:
// the luminance of emission x opacity at the texel centres of the larger texture in a
// SummedAreaTable (sat.h: double sums, corners looked up bilinearly with clamping over the
// (n + 1)^2 grid), each triangle's mean over the tiles of its texcoord bounding box (flip_v, uv
// scale and offset of the texture field; repeat: mod 1, clamp: saturate; degenerate boxes widened
// by one cell), weighted by the unwrapped tile areas.  Tiles whose wrapped box is empty are skipped
// (the reference asserts there).  Lookups that disagree in those settings: the grid's mean.
struct OracleSat
{
    int nx, ny;
    std::vector<double> t;
    double at(int x, int y) const
    {
        if (x == 0 || y == 0)
            return 0.0;
        return t[(size_t)std::min(y - 1, ny - 1) * nx + std::min(x - 1, nx - 1)];
    }
    double corner(float px, float py) const
    {
        auto split = [](float p, int res, int &a, int &b, float &w) {
            const float q = p * (float)(res - 1);
            a = (int)std::floor(q);
            b = a + 1;
            w = q - (float)a;
            a = std::clamp(a, 0, res - 1);
            b = std::clamp(b, 0, res - 1);
        };
        int x0, x1, y0, y1;
        float wx, wy;
        split(px, nx + 1, x0, x1, wx);
        split(py, ny + 1, y0, y1, wy);
        return at(x0, y0) * (1.0 - wx) * (1.0 - wy) + at(x1, y0) * (wx) * (1.0 - wy) + at(x0, y1) * (1.0 - wx) * (wy) +
               at(x1, y1) * (wx) * (wy);
    }
};

inline std::vector<float> mesh_importance_factor(const Scene &s, uint32_t material, uint32_t first, uint32_t n)
{
    const ks_material_desc &mat = s.materials[material];
    const V3 emission(mat.emission[0], mat.emission[1], mat.emission[2]);
    const Binding *em = nullptr, *op = nullptr;
    for (const Binding &b : s.mat_bindings[material]) {
        if (b.b.field == KS_FIELD_EMISSION)
            em = &b;
        if (b.b.field == KS_FIELD_OPACITY_MAP)
            op = &b;
    }
    if (!em && !op)
        return std::vector<float>(n, luminance(emission));
    int rx = 1, ry = 1;
    if (em) {
        rx = s.textures[em->b.texture].w;
        ry = s.textures[em->b.texture].h;
    }
    bool fallback = false;
    if (op) {
        rx = std::max(rx, s.textures[op->b.texture].w);
        ry = std::max(ry, s.textures[op->b.texture].h);
        if (em && (em->b.wrap_u != op->b.wrap_u || em->b.wrap_v != op->b.wrap_v || (em->b.flip_v != 0) != (op->b.flip_v != 0) ||
                   em->b.uv_scale[0] != op->b.uv_scale[0] || em->b.uv_scale[1] != op->b.uv_scale[1] ||
                   em->b.uv_offset[0] != op->b.uv_offset[0] || em->b.uv_offset[1] != op->b.uv_offset[1]))
            fallback = true;
    }
    std::vector<float> grid((size_t)rx * ry);
    double total = 0.0;
    for (int y = 0; y < ry; ++y)
        for (int x = 0; x < rx; ++x) {
            const float u = (x + 0.5f) / (float)rx, v = (y + 0.5f) / (float)ry;
            float c[4];
            float lum = luminance(emission);
            if (em) {
                em->eval(s.textures[em->b.texture], u, v, c);
                lum = luminance(V3(c[0], c[1], c[2]));
            }
            if (op) {
                op->eval(s.textures[op->b.texture], u, v, c);
                lum *= c[0];
            }
            grid[(size_t)y * rx + x] = lum;
            total += lum;
        }
    if (fallback)
        return std::vector<float>(n, (float)(total / (double)grid.size()));
    OracleSat sat{rx, ry, std::vector<double>(grid.size())};
    for (int y = 0; y < ry; ++y)
        for (int x = 0; x < rx; ++x) {
            double v = grid[(size_t)y * rx + x];
            if (x > 0)
                v += sat.t[(size_t)y * rx + x - 1];
            if (y > 0)
                v += sat.t[(size_t)(y - 1) * rx + x];
            if (x > 0 && y > 0)
                v -= sat.t[(size_t)(y - 1) * rx + x - 1];
            sat.t[(size_t)y * rx + x] = v;
        }
    const Binding &lb = em ? *em : *op;
    const float before_one = std::nextafter(1.0f, 0.0f);
    std::vector<float> out(n, 0.0f);
    for (uint32_t k = 0; k < n; ++k) {
        float lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
        for (int c = 0; c < 3; ++c) {
            const uint32_t vi = s.idx[3 * (first + k) + c];
            float t[2] = {s.texcoords[2 * vi], s.texcoords[2 * vi + 1]};
            if (lb.b.flip_v)
                t[1] = 1.0f - t[1];
            for (int a = 0; a < 2; ++a) {
                t[a] = t[a] * lb.b.uv_scale[a] + lb.b.uv_offset[a];
                lo[a] = std::min(lo[a], t[a]);
                hi[a] = std::max(hi[a], t[a]);
            }
        }
        float acc = 0.0f, area_sum = 0.0f;
        for (int ty = (int)std::floor(lo[1]); ty < (int)std::ceil(hi[1]); ++ty)
            for (int tx = (int)std::floor(lo[0]); tx < (int)std::ceil(hi[0]); ++tx) {
                float b0[2] = {std::max(lo[0], (float)tx), std::max(lo[1], (float)ty)};
                float b1[2] = {std::min(hi[0], tx + before_one), std::min(hi[1], ty + before_one)};
                if (b0[0] > b1[0] || b0[1] > b1[1])
                    continue;
                const float unwrapped = (b1[0] - b0[0]) * (b1[1] - b0[1]);
                if (unwrapped == 0.0f)
                    continue;
                const int wrap[2] = {lb.b.wrap_u, lb.b.wrap_v}, res[2] = {rx, ry};
                for (int a = 0; a < 2; ++a) {
                    if (wrap[a] == 0) {
                        for (float *p : {&b0[a], &b1[a]}) {
                            float r = *p - std::floor(*p / 1.0f) * 1.0f;
                            *p = r < 0 ? r + 1.0f : r;
                        }
                    } else {
                        b0[a] = std::clamp(b0[a], 0.0f, 1.0f);
                        b1[a] = std::clamp(b1[a], 0.0f, 1.0f);
                    }
                    if (b0[a] == 0.0f && b1[a] == 0.0f)
                        b1[a] = 1.0f / (res[a] + 1);
                    if (b0[a] == 1.0f && b1[a] == 1.0f)
                        b0[a] = 1.0f - 1.0f / (res[a] + 1);
                }
                if (b0[0] > b1[0] || b0[1] > b1[1] || (b1[0] - b0[0]) * (b1[1] - b0[1]) == 0.0f)
                    continue;
                const double box = (sat.corner(b1[0], b1[1]) - sat.corner(b0[0], b1[1])) +
                                   (sat.corner(b0[0], b0[1]) - sat.corner(b1[0], b0[1]));
                const float mean = std::max((float)box, 0.0f) / (((b1[0] - b0[0]) * (float)rx) * ((b1[1] - b0[1]) * (float)ry));
                acc += mean * unwrapped;
                area_sum += unwrapped;
            }
        if (area_sum > 0.0f)
            acc /= area_sum;
        out[k] = acc;
    }
    return out;
}

// MeshTriLight::eval (light.cpp:560-565) at barycentrics (u, v): the emission texture at the
// interpolated texcoords, or (without texcoords) at the barycentrics for a hit record
// (compute_intersection) and at zero for a light sample (interpolate_texcoord, geometry.cpp:182-191)
inline V3 light_Le(const Scene &s, const MeshLight &ml, uint32_t tri, float u, float v, bool bary_fallback)
{
    if (ml.em_binding < 0)
        return ml.emission;
    float tu = bary_fallback ? u : 0.0f, tv = bary_fallback ? v : 0.0f;
    if (s.mesh_uv[s.tri_mesh[tri]]) {
        const uint32_t i0 = s.idx[3 * tri], i1 = s.idx[3 * tri + 1], i2 = s.idx[3 * tri + 2];
        const float *tc = s.texcoords.data();
        const float w0 = 1.0f - u - v;
        tu = w0 * tc[2 * i0] + u * tc[2 * i1] + v * tc[2 * i2];
        tv = w0 * tc[2 * i0 + 1] + u * tc[2 * i1 + 1] + v * tc[2 * i2 + 1];
    }
    const Binding &bd = s.mat_bindings[s.mesh_material[ml.mesh]][ml.em_binding];
    float c[4];
    bd.eval(s.textures[bd.b.texture], tu, tv, c);
    return V3(c[0], c[1], c[2]);
}

inline V3 mesh_light_sample(const Scene &s, uint32_t light_flat, V3 p_shade, float u0, float u1, V3 &wi,
                            float &wi_dist, float &pdf)
{
    uint32_t g = (uint32_t)(std::upper_bound(s.index_psum.begin(), s.index_psum.end(), light_flat) -
                            s.index_psum.begin()) - 1;
    uint32_t k = light_flat - s.index_psum[g];
    const MeshLight &ml = s.mesh_lights[g - 1];
    // sample_triangle_bary (rng.h:379-390)
    float b0, b1;
    if (u0 < u1) {
        b0 = u0 / 2;
        b1 = u1 - b0;
    } else {
        b1 = u1 / 2;
        b0 = u0 - b1;
    }
    uint32_t tri = s.mesh_tri_off[ml.mesh] + ml.prim_ids[k];
    V3 p0 = s.tri_vert(tri, 0), p1 = s.tri_vert(tri, 1), p2 = s.tri_vert(tri, 2);
    float w0 = 1.0f - b0 - b1;
    V3 position = w0 * p0 + b0 * p1 + b1 * p2;
    V3 n = light_normal(s, tri);
    wi = position - p_shade;
    float wi_dist2 = sqnorm(wi);
    if (wi_dist2 == 0.0f) {
        wi_dist = 0.0f;
        pdf = 0.0f;
        return V3();
    }
    wi_dist = std::sqrt(wi_dist2);
    wi /= wi_dist;
    pdf = 1.0f / ml.areas[k];
    float absdot = std::abs(dot(n, wi));
    if (absdot == 0.0f) {
        wi_dist = 0.0f;
        pdf = 0.0f;
        return V3();
    }
    pdf *= (wi_dist2 / absdot);
    constexpr float shadow_eps = 1e-4f;
    wi_dist = std::max(0.0f, wi_dist - shadow_eps);
    return light_Le(s, ml, tri, b0, b1, false) / pdf;
}

inline float mesh_light_pdf(const Scene &s, uint32_t tri, uint32_t k, const MeshLight &ml, V3 wi, float wi_dist)
{
    if (wi_dist == 0.0f)
        return 0.0f;
    V3 n = light_normal(s, tri);
    float pdf = 1.0f / ml.areas[k];
    float absdot = std::abs(dot(n, wi));
    if (absdot == 0.0f)
        return 0.0f;
    pdf *= (sqr(wi_dist) / absdot);
    return pdf;
}

struct Counters
{
    uint64_t extension = 0, shadow = 0;
};

struct Camera
{
    float c2w[16], p2w[16];
    bool ortho = false;
    V3 position() const { return V3(c2w[3], c2w[7], c2w[11]); }
    // Camera::direction (camera.h:24-27)
    V3 direction() const { return -normalized(V3(c2w[2], c2w[6], c2w[10])); }
};

struct Tracer
{
    const Scene &s;
    const ks_small_pt_params &in;
    Counters cnt;
    Work *work = nullptr; // counts the queries' nodes and triangles when set

    // next_event_estimate (nee.cpp:11-57)
    V3 nee(const Bsdf &bsdf, const Intersection &hit, V3 wo, OwenScrambledSobol02Morton &sobol)
    {
        float pr_light;
        uint32_t light = s.power_distrib.sample(sobol.next(), pr_light);
        float u0, u1;
        sobol.next2d(u0, u1);
        V3 wi;
        float wi_dist = 0.0f, pdf_wi_light = 0.0f;
        V3 Le_beta;
        uint32_t n_nonmesh = s.index_psum[1], n_sky = s.sky ? 1u : 0u;
        bool delta_light = false;
        if (light < n_sky) {
            Le_beta = s.sky->sample(u0, u1, wi, wi_dist, pdf_wi_light);
        } else if (light < n_nonmesh) {
            // PointLight / DirectionalLight::sample (light.cpp:208-236)
            const ks_light_desc &l = s.lights[light - n_sky];
            delta_light = true;
            pdf_wi_light = 1.0f;
            if (l.type == 0) {
                wi = V3(l.vec[0], l.vec[1], l.vec[2]) - hit.p;
                float l2 = dot(wi, wi);
                if (l2 == 0.0f) {
                    Le_beta = V3(0.0f, 0.0f, 0.0f);
                    pdf_wi_light = 0.0f;
                } else {
                    float len = std::sqrt(l2);
                    wi = wi / len;
                    wi_dist = len;
                    Le_beta = V3(l.color[0] / l2, l.color[1] / l2, l.color[2] / l2);
                }
            } else {
                wi = V3(l.vec[0], l.vec[1], l.vec[2]);
                wi_dist = std::numeric_limits<float>::infinity();
                Le_beta = V3(l.color[0], l.color[1], l.color[2]);
            }
        } else {
            Le_beta = mesh_light_sample(s, light, hit.p, u0, u1, wi, wi_dist, pdf_wi_light);
        }
        V3 beta_nee;
        if (!is_zero(Le_beta) && pdf_wi_light > 0.0f) {
            V3 wo_local = hit.sh_to_local(wo);
            V3 wi_local = hit.sh_to_local(wi);
            V3 f;
            float pdf_wi_bsdf;
            bsdf.eval_and_pdf(wo_local, wi_local, f, pdf_wi_bsdf);
            if (!is_zero(f) && pdf_wi_bsdf > 0.0f) {
                V3 o = spawn_origin(hit.p, wi, hit.frame.n);
                cnt.shadow++;
                if (!occluded(s, o, wi, wi_dist, work)) {
                    float mis_weight = delta_light ? 1.0f : power_heur(pdf_wi_light, pdf_wi_bsdf);
                    beta_nee += Le_beta * f * mis_weight / pr_light;
                }
            }
        }
        return beta_nee;
    }

    bool trace(V3 ro, V3 rd, OwenScrambledSobol02Morton &sobol, Pcg32 &rng, V3 &Lout)
    {
        V3 L;
        V3 beta(1, 1, 1);
        float pdf_wi_bsdf = 0.0f;
        for (int bounce = 0; bounce < in.bounces + 1; ++bounce) {
            uint32_t tri;
            float t, bary[3];
            cnt.extension++;
            bool isect_geom = intersect(s, ro, rd, inf, tri, t, bary, work);
            if (!isect_geom) {
                if (s.sky) {
                    uint32_t light_index = 0;
                    V3 wi = normalized(rd);
                    V3 Le = s.sky->eval(wi);
                    if (bounce == 0) {
                        if (in.include_background)
                            L += beta * Le;
                    } else {
                        float pr_light = s.probability(light_index);
                        float pdf_wi_light = s.sky->pdf(wi);
                        float mis_weight = power_heur(pdf_wi_bsdf, pdf_wi_light * pr_light);
                        V3 beta_uni = Le * mis_weight;
                        if (bounce == 1 && in.clamp_direct > 0.0f)
                            beta_uni = cwise_min(beta_uni, in.clamp_direct);
                        else if (bounce >= 2 && in.clamp_indirect > 0.0f)
                            beta_uni = cwise_min(beta_uni, in.clamp_indirect);
                        L += beta * beta_uni;
                    }
                }
                if (bounce == 0 && !in.include_background) {
                    Lout = V3();
                    return false;
                }
                break;
            }
            Intersection it = make_intersection(s, tri, t, bary[1], bary[2], rd);
            uint32_t mesh = s.tri_mesh[tri];
            const ks_material_desc mat = textured_material(s, s.mesh_material[mesh], it);
            if (mat.has_emission) {
                int32_t light = s.tri_light[tri];
                if (light >= 0) {
                    float pr_light = s.probability((uint32_t)light);
                    V3 wi = normalized(rd);
                    uint32_t g = (uint32_t)(std::upper_bound(s.index_psum.begin(), s.index_psum.end(),
                                                             (uint32_t)light) -
                                            s.index_psum.begin()) - 1;
                    const MeshLight &ml = s.mesh_lights[g - 1];
                    const V3 Le = light_Le(s, ml, tri, bary[1], bary[2], true);
                    if (bounce == 0) {
                        L += beta * Le;
                    } else if (pr_light > 0.0f) {
                        uint32_t k = (uint32_t)light - s.index_psum[g];
                        float pdf_wi_light = mesh_light_pdf(s, tri, k, ml, wi, it.thit);
                        float mis_weight = power_heur(pdf_wi_bsdf, pdf_wi_light * pr_light);
                        V3 beta_uni = Le * mis_weight;
                        if (bounce == 1 && in.clamp_direct > 0.0f)
                            beta_uni = cwise_min(beta_uni, in.clamp_direct);
                        else if (bounce >= 2 && in.clamp_indirect > 0.0f)
                            beta_uni = cwise_min(beta_uni, in.clamp_indirect);
                        L += beta * beta_uni;
                    }
                }
            }
            if (bounce == in.bounces)
                break;
            V3 wo = -normalized(rd);
            Bsdf bsdf{eval_closure(mat)};
            // Material::sample_with_nee (material.cpp:101-167): with a BSSRDF, the BSDF or (1/2) a
            // random walk whose exit shades with the Lambertian exit lobe
            V3 ss_beta(1.0f, 1.0f, 1.0f);
            if (mat.has_subsurface) {
                if (sobol.next() < 0.5f) {
                    ss_beta *= 2.0f;
                } else {
                    ss_beta *= 2.0f;
                    ss_beta /= mat.ss_ior * mat.ss_ior;
                    auto cast = [&](V3 o, V3 d, float tmax, uint32_t &tri_out, float &t_out, float &b1, float &b2) {
                        float r[8] = {o.x, o.y, o.z, 0.0f, d.x, d.y, d.z, tmax};
                        struct MeshFilter
                        {
                            const Scene *s;
                            uint32_t mesh;
                            static int call(void *user, uint32_t tri, float, float)
                            {
                                const MeshFilter &f = *(const MeshFilter *)user;
                                return f.s->tri_mesh[tri] == f.mesh;
                            }
                        } mf{&s, mesh};
                        float bary[3];
                        uint64_t dummy[3] = {0, 0, 0};
                        tri_out = ksref_sbvh_intersect1_counted(s.bvh, r, 0, 2, &t_out, bary, dummy, MeshFilter::call,
                                                                &mf);
                        b1 = bary[1];
                        b2 = bary[2];
                        return tri_out != ~0u;
                    };
                    const V3 alb(std::clamp(mat.ss_albedo[0], 0.0f, 1.0f), std::clamp(mat.ss_albedo[1], 0.0f, 1.0f),
                                 std::clamp(mat.ss_albedo[2], 0.0f, 1.0f));
                    const V3 rad(mat.ss_radius[0], mat.ss_radius[1], mat.ss_radius[2]);
                    uint32_t etri = 0;
                    float et = 0.0f, eb1 = 0.0f, eb2 = 0.0f;
                    V3 ss_wi;
                    if (!ss_walk(alb, rad, mat.ss_anisotropy, mat.ss_ior, mat.ss_rfr_entry_prob, it.p, it.sh_frame.n,
                                 it.frame.n, rng, cast, ss_beta, etri, et, eb1, eb2, ss_wi))
                        break; // MaterialSample {0, 0}: no light and a zero throughput end the path
                    wo = -ss_wi;
                    it = make_intersection(s, etri, et, eb1, eb2, ss_wi);
                    (void)textured_material(s, s.mesh_material[s.tri_mesh[etri]], it); // the exit's normal map
                    Closure ce{};
                    ce.bsdf = 3;
                    ce.ior = mat.ss_ior;
                    bsdf = Bsdf{ce};
                }
            }
            V3 Ld = ss_beta * nee(bsdf, it, wo, sobol);
            V3 wo_local = it.sh_to_local(wo);
            float u_lobe = sobol.next();
            float u0, u1;
            sobol.next2d(u0, u1);
            V3 wi_local;
            float pdf_wi = 0.0f;
            V3 sbeta = ss_beta * bsdf.sample(wo_local, wi_local, u_lobe, u0, u1, pdf_wi);
            V3 wi;
            if (!(max_coeff(sbeta) == 0.0f || pdf_wi == 0.0f))
                wi = it.sh_to_world(wi_local);
            if (bounce == 0 && in.clamp_direct > 0.0f)
                Ld = cwise_min(Ld, in.clamp_direct);
            else if (bounce >= 1 && in.clamp_indirect > 0.0f)
                Ld = cwise_min(Ld, in.clamp_indirect);
            L += beta * Ld;
            beta *= sbeta;
            if (max_coeff(beta) == 0.0f)
                break;
            pdf_wi_bsdf = pdf_wi;
            ro = spawn_origin(it.p, wi, it.frame.n);
            rd = wi;
            if (max_coeff(beta) < 1.0f && bounce >= 1) {
                float q = std::max(0.0f, 1.0f - max_coeff(beta));
                if (sobol.next() < q)
                    break;
                beta /= 1.0f - q;
            }
        }
        Lout = L;
        return true;
    }
};

Scene *create_scene(const ks_scene_desc *d, const ks_sbvh_options *opts)
{
    auto s = std::make_unique<Scene>();
    uint32_t vo = 0;
    for (uint32_t m = 0; m < d->n_meshes; ++m) {
        const ks_mesh_desc &md = d->meshes[m];
        s->mesh_tri_off.push_back((uint32_t)s->tri_mesh.size());
        s->verts.insert(s->verts.end(), md.vertices, md.vertices + 3 * md.n_vertices);
        for (uint32_t k = 0; k < 3 * md.n_triangles; ++k)
            s->idx.push_back(md.indices[k] + vo);
        s->tri_mesh.insert(s->tri_mesh.end(), md.n_triangles, m);
        s->mesh_material.push_back(md.material);
        s->mesh_twosided.push_back(md.twosided);
        s->mesh_smooth.push_back(md.use_smooth_normal && md.vertex_normals ? 1 : 0);
        s->mesh_uv.push_back(md.texcoords ? 1 : 0);
        if (md.use_smooth_normal && md.vertex_normals)
            s->normals.insert(s->normals.end(), md.vertex_normals, md.vertex_normals + 3 * md.n_vertices);
        else
            s->normals.insert(s->normals.end(), 3 * (size_t)md.n_vertices, 0.0f);
        if (md.texcoords)
            s->texcoords.insert(s->texcoords.end(), md.texcoords, md.texcoords + 2 * md.n_vertices);
        else
            s->texcoords.insert(s->texcoords.end(), 2 * (size_t)md.n_vertices, 0.0f);
        vo += md.n_vertices;
    }
    s->mesh_tri_off.push_back((uint32_t)s->tri_mesh.size());
    s->materials.assign(d->materials, d->materials + d->n_materials);
    for (uint32_t k = 0; k < d->n_textures; ++k)
        s->textures.emplace_back(d->textures[k]);
    s->mat_bindings.resize(d->n_materials);
    for (uint32_t k = 0; k < d->n_bindings; ++k) {
        s->mat_bindings[d->bindings[k].material].emplace_back(d->bindings[k]);
        s->any_opacity |= d->bindings[k].field == KS_FIELD_OPACITY_MAP;
    }
    ks_sbvh_options o{4, 12, 1.0f, 1e-5f};
    if (opts)
        o = *opts;
    uint32_t nn, np;
    if (ksref_sbvh_build(s->verts.data(), vo, s->idx.data(), (uint32_t)s->tri_mesh.size(), o.max_prims_in_node,
                         o.bucket_count, o.trav_weight, o.alpha, &s->bvh, &nn, &np) != 0)
        return nullptr;
    ksref_sbvh_bound(s->bvh, s->bound);

    // sky light (light.cpp:19-57)
    const ks_sky_desc &sd = d->sky;
    if (sd.kind == 3) {
        auto sky = std::make_unique<Sky>();
        sky->kind = 3;
        sky->w = sky->h = (int)sd.width;
        sky->map.resize((size_t)sky->w * sky->h);
        std::vector<float> lum(sky->map.size());
        for (size_t i = 0; i < sky->map.size(); ++i) {
            sky->map[i] = V3(sd.map_rgb[3 * i], sd.map_rgb[3 * i + 1], sd.map_rgb[3 * i + 2]);
            lum[i] = luminance(sky->map[i]);
        }
        std::memcpy(sky->l2w, sd.to_world, sizeof(float) * 16);
        sky->strength = sd.strength;
        sky->ea_pmf = AliasTable(lum);
        s->sky = std::move(sky);
    }
    if (sd.kind == 1 || sd.kind == 2) {
        auto sky = std::make_unique<Sky>();
        sky->kind = sd.kind;
        if (sd.kind == 1) {
            sky->w = sky->h = 1;
            sky->map = {V3(sd.ambient[0], sd.ambient[1], sd.ambient[2])};
            float id[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
            std::memcpy(sky->l2w, id, sizeof(id));
            std::memcpy(sky->w2l, id, sizeof(id));
            sky->y_up = true;
            sky->strength = 1.0f;
            float lum = luminance(sky->map[0]);
            sky->distrib = DistribTable2D(&lum, 1, 1);
        } else {
            sky->w = (int)sd.width;
            sky->h = (int)sd.height;
            sky->map.resize((size_t)sky->w * sky->h);
            for (size_t i = 0; i < sky->map.size(); ++i)
                sky->map[i] = V3(sd.map_rgb[3 * i], sd.map_rgb[3 * i + 1], sd.map_rgb[3 * i + 2]);
            std::memcpy(sky->l2w, sd.to_world, sizeof(float) * 16);
            invert_rigid_or_general(sky->l2w, sky->w2l);
            sky->y_up = sd.transform_y_up != 0;
            sky->strength = sd.strength;
            std::vector<float> lum((size_t)sky->w * sky->h);
            double lum_sum = 0.0;
            for (int y = 0; y < sky->h; ++y) {
                float theta = (y + 0.5f) / (float)sky->h * pi;
                float sin_theta = std::sin(theta);
                double row = 0.0;
                for (int x = 0; x < sky->w; ++x) {
                    size_t i = (size_t)y * sky->w + x;
                    lum[i] = sin_theta * luminance(sky->map[i]);
                    row += lum[i];
                }
                lum_sum += row;
            }
            float average = (float)lum_sum / lum.size();
            for (auto &l : lum)
                l = std::max(l - average, 0.0f);
            sky->distrib = DistribTable2D(lum.data(), sky->w, sky->h);
        }
        s->sky = std::move(sky);
    }
    // mesh lights (scene.cpp:315-336, light.cpp:307-560): constant emission -> uniform importance;
    // emission / opacity textures -> the summed-area-table importance (mesh_importance_factor)
    for (uint32_t m = 0; m < d->n_meshes; ++m) {
        const ks_material_desc &mat = s->materials[s->mesh_material[m]];
        if (!mat.has_emission)
            continue;
        MeshLight ml;
        ml.mesh = m;
        ml.emission = V3(mat.emission[0], mat.emission[1], mat.emission[2]);
        const auto &mb = s->mat_bindings[s->mesh_material[m]];
        for (size_t b = 0; b < mb.size(); ++b)
            if (mb[b].b.field == KS_FIELD_EMISSION)
                ml.em_binding = (int)b;
        uint32_t first = s->mesh_tri_off[m], n = s->mesh_tri_off[m + 1] - first;
        const std::vector<float> factor = mesh_importance_factor(*s, s->mesh_material[m], first, n);
        std::vector<float> importance(n), areas(n);
        for (uint32_t k = 0; k < n; ++k) {
            V3 v0 = s->tri_vert(first + k, 0), v1 = s->tri_vert(first + k, 1), v2 = s->tri_vert(first + k, 2);
            V3 e01 = v1 - v0, e12 = v2 - v1;
            float area = 0.5f * norm(cross(e01, e12));
            importance[k] = two_pi * area * factor[k];
            areas[k] = area;
        }
        std::vector<uint32_t> prim_ids(n);
        for (uint32_t k = 0; k < n; ++k)
            prim_ids[k] = k;
        uint32_t N = n;
        for (uint32_t i = 0; i < N;) {
            if (importance[i] == 0.0f) {
                std::swap(prim_ids[N - 1], prim_ids[i]);
                std::swap(importance[N - 1], importance[i]);
                std::swap(areas[N - 1], areas[i]);
                --N;
            } else {
                ++i;
            }
        }
        prim_ids.resize(N);
        importance.resize(N);
        areas.resize(N);
        ml.prim_ids = prim_ids;
        ml.importance = importance;
        ml.areas = areas;
        s->mesh_lights.push_back(std::move(ml));
    }
    // PowerLightSampler::build (light.cpp:636-672)
    if (d->n_lights)
        s->lights.assign(d->lights, d->lights + d->n_lights);
    uint32_t n_nonmesh = (s->sky ? 1u : 0u) + (uint32_t)s->lights.size();
    s->index_psum.assign(1 + s->mesh_lights.size() + 1, 0);
    uint32_t sum = 0;
    for (uint32_t i = 0; i < (uint32_t)s->index_psum.size(); ++i) {
        s->index_psum[i] = sum;
        if (i < (uint32_t)s->index_psum.size() - 1)
            sum += (i == 0 ? n_nonmesh : (uint32_t)s->mesh_lights[i - 1].prim_ids.size());
    }
    s->light_count = sum;
    s->powers.assign(sum, 0.0f);
    s->tri_light.assign(s->tri_mesh.size(), -1);
    uint32_t flat = 0;
    if (s->sky) {
        V3 P = s->sky->power(s->bound);
        s->powers[flat++] = (P.x + P.y + P.z) / 3.0f;
    }
    for (const ks_light_desc &l : s->lights) {
        // PointLight::power 4 pi I, DirectionalLight::power L pi r^2 (light.cpp:218-240)
        float P[3];
        if (l.type == 0) {
            for (int c = 0; c < 3; ++c)
                P[c] = 4.0f * pi * l.color[c];
        } else {
            float ex = s->bound[3] - s->bound[0], ey = s->bound[4] - s->bound[1], ez = s->bound[5] - s->bound[2];
            float r = 0.5f * std::sqrt(ex * ex + ey * ey + ez * ez);
            for (int c = 0; c < 3; ++c)
                P[c] = l.color[c] * pi * (r * r);
        }
        s->powers[flat++] = (P[0] + P[1] + P[2]) / 3.0f;
    }
    for (const MeshLight &ml : s->mesh_lights)
        for (uint32_t j = 0; j < ml.prim_ids.size(); ++j) {
            s->tri_light[s->mesh_tri_off[ml.mesh] + ml.prim_ids[j]] = (int32_t)flat;
            float pw = ml.importance[j];
            s->powers[flat++] = (pw + pw + pw) / 3.0f;
        }
    if (sum > 0)
        s->power_distrib = DistribTable(s->powers.data(), sum);
    return s.release();
}

} // namespace oracle

using namespace oracle;

extern "C" {

void *oracle_scene_create(const ks_scene_desc *desc, const ks_sbvh_options *opts)
{
    return oracle::create_scene(desc, opts);
}

void oracle_scene_destroy(void *s) { delete (Scene *)s; }

// Light tables for parity checks: powers (light_count floats) and the power CDF
// (light_count + 1 floats); returns light_count.
uint32_t oracle_light_table(void *sp, float *powers, float *cdf)
{
    Scene *s = (Scene *)sp;
    for (uint32_t i = 0; i < s->light_count; ++i) {
        if (powers)
            powers[i] = s->powers[i];
    }
    if (cdf)
        for (size_t i = 0; i < s->power_distrib.cdf.size(); ++i)
            cdf[i] = s->power_distrib.cdf[i];
    return s->light_count;
}

// Sky distribution for parity checks: conditional CDFs (h rows of w+1) and marginal CDF (h+1).
int oracle_sky_tables(void *sp, float *cond, float *margin)
{
    Scene *s = (Scene *)sp;
    if (!s->sky)
        return 1;
    const Sky &k = *s->sky;
    for (int y = 0; y < k.h; ++y)
        for (int x = 0; x <= k.w; ++x)
            cond[(size_t)y * (k.w + 1) + x] = k.distrib.cond[y].cdf[x];
    for (int y = 0; y <= k.h; ++y)
        margin[y] = k.distrib.margin.cdf[y];
    return 0;
}

int oracle_render_range(void *sp, const ks_camera_desc *cam, const ks_small_pt_params *in, int s_begin, int s_end,
                        double *accum, double *weights, int n_threads, uint64_t *counts, uint64_t *work_out);

// SmallPT::run (small_pt.cpp:15-70) on n_threads host threads over 4x4 pixel tiles
// (parallel.h:93-113).  accum: W*H*3 doubles, weights: W*H*2 doubles (both zero-initialised by
// the caller and accumulated into).  counts[0..1] receive extension and shadow ray counts.
int oracle_render(void *sp, const ks_camera_desc *cam, const ks_small_pt_params *in, double *accum, double *weights,
                  int n_threads, uint64_t *counts)
{
    return oracle_render_range(sp, cam, in, 0, in->spp, accum, weights, n_threads, counts, nullptr);
}

// The same render restricted to the sample indices [s_begin, s_end) of the in->spp samples per
// pixel (one spp interval of SmallPT::run, small_pt.cpp:56-66, or any bounded part of the frame's
// samples).  work_out (7 values, may be NULL): the extension queries' nodes, triangles and stack
// overflows, the shadow queries' nodes, triangles and overflows, counted by the restatement of the
// reference traversal, then the number of queries where it disagreed with the reference's own.
int oracle_render_range(void *sp, const ks_camera_desc *cam, const ks_small_pt_params *in, int s_begin, int s_end,
                        double *accum, double *weights, int n_threads, uint64_t *counts, uint64_t *work_out)
{
    if (s_begin < 0 || s_end > in->spp || s_begin > s_end)
        return 1;
    Scene &s = *(Scene *)sp;
    const int W = in->render_width, H = in->render_height;
    int cx = 0, cy = 0, cw = W, ch = H;
    if (in->crop_width > 0 && in->crop_height > 0) {
        cx = std::max(in->crop_start_x, 0);
        cy = std::max(in->crop_start_y, 0);
        cw = std::min(in->crop_width, W - cx);
        ch = std::min(in->crop_height, H - cy);
    }
    Camera camera;
    std::memcpy(camera.c2w, cam->camera_to_world, sizeof(float) * 16);
    std::memcpy(camera.p2w, cam->proj_to_world, sizeof(float) * 16);
    camera.ortho = cam->orthographic != 0;
    const int tiles_x = (cw + 3) / 4, tiles_y = (ch + 3) / 4;
    std::atomic<int> next_tile{0};
    std::atomic<uint64_t> n_ext{0}, n_shadow{0};
    std::mutex work_mutex;
    Work work_total;
    const PixelFilterTable filter(in->pixel_filter, in->pixel_filter_width, in->pixel_filter_sigma);
    auto worker = [&]() {
        Tracer tr{s, *in, {}};
        Work work;
        if (work_out)
            tr.work = &work;
        while (true) {
            int tile = next_tile.fetch_add(1);
            if (tile >= tiles_x * tiles_y)
                break;
            int tx = tile % tiles_x, ty = tile / tiles_x;
            for (int oy = ty * 4; oy < std::min(ch, ty * 4 + 4); ++oy)
                for (int ox = tx * 4; ox < std::min(cw, tx * 4 + 4); ++ox) {
                    int px = cx + ox, py = cy + oy;
                    size_t pix = (size_t)py * W + px;
                    for (int smp = s_begin; smp < s_end; ++smp) {
                        PTRenderSampler sampler(W, H, px, py, in->spp, smp, in->rng_seed);
                        float offx = 0.0f, offy = 0.0f;
                        if (in->spp != 1) {
                            float u0, u1;
                            sampler.sobol.next2d(u0, u1);
                            filter.sample(u0, u1, offx, offy);
                        }
                        float fx = ((px + 0.5f) + offx) / (float)W;
                        float fy = ((py + 0.5f) + offy) / (float)H;
                        V3 ndc(fx * 2.0f - 1.0f, fy * 2.0f - 1.0f, 1.0f);
                        V3 cp = camera.position();
                        V3 world_pos = point_hdiv(camera.p2w, ndc);
                        V3 dir;
                        if (camera.ortho) { // Camera::spawn_ray, orthographic (camera.cpp:155-160)
                            cp = world_pos;
                            dir = camera.direction();
                        } else {
                            dir = normalized(world_pos - cp);
                        }
                        V3 L;
                        Pcg32 rng = sample_rng(px, py, (uint32_t)in->rng_seed, smp);
                        bool hit = tr.trace(cp, dir, sampler.sobol, rng, L);
                        if (hit) {
                            weights[2 * pix + 0] += 1.0;
                            weights[2 * pix + 1] += 0.0;
                            accum[3 * pix + 0] += (double)L.x * 1.0;
                            accum[3 * pix + 1] += (double)L.y * 1.0;
                            accum[3 * pix + 2] += (double)L.z * 1.0;
                        } else {
                            weights[2 * pix + 1] += 1.0;
                        }
                    }
                }
        }
        n_ext += tr.cnt.extension;
        n_shadow += tr.cnt.shadow;
        std::lock_guard<std::mutex> lock(work_mutex);
        for (int k = 0; k < 3; ++k) {
            work_total.ext[k] += work.ext[k];
            work_total.shadow[k] += work.shadow[k];
        }
        work_total.mismatches += work.mismatches;
    };
    int nt = std::max(1, n_threads);
    std::vector<std::thread> pool;
    for (int k = 0; k < nt; ++k)
        pool.emplace_back(worker);
    for (auto &t : pool)
        t.join();
    if (counts) {
        counts[0] = n_ext.load();
        counts[1] = n_shadow.load();
    }
    if (work_out) {
        for (int k = 0; k < 3; ++k) {
            work_out[k] = work_total.ext[k];
            work_out[3 + k] = work_total.shadow[k];
        }
        work_out[6] = work_total.mismatches;
    }
    return 0;
}

// Sky-light hooks for tests: n samples from uniforms u (2 per sample): direction, pdf and
// radiance / pdf; and pdf and radiance of n given directions.  1 when the scene has no sky.
int oracle_sky_sample(void *sp, const float *u, uint32_t n, float *wi, float *pdf, float *Le_beta)
{
    const Scene &s = *(Scene *)sp;
    if (!s.sky)
        return 1;
    for (uint32_t i = 0; i < n; ++i) {
        V3 w, L;
        float dist = 0.0f, p = 0.0f;
        L = s.sky->sample(u[2 * i], u[2 * i + 1], w, dist, p);
        wi[3 * i] = w.x;
        wi[3 * i + 1] = w.y;
        wi[3 * i + 2] = w.z;
        pdf[i] = p;
        Le_beta[3 * i] = L.x;
        Le_beta[3 * i + 1] = L.y;
        Le_beta[3 * i + 2] = L.z;
    }
    return 0;
}

int oracle_sky_eval(void *sp, const float *wi, uint32_t n, float *pdf, float *Le)
{
    const Scene &s = *(Scene *)sp;
    if (!s.sky)
        return 1;
    for (uint32_t i = 0; i < n; ++i) {
        V3 w(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        pdf[i] = s.sky->pdf(w);
        V3 L = s.sky->eval(w);
        Le[3 * i] = L.x;
        Le[3 * i + 1] = L.y;
        Le[3 * i + 2] = L.z;
    }
    return 0;
}

// BSDF parity hooks on batches of local directions.
void oracle_bsdf_eval(const ks_material_desc *mat, const float *wo, const float *wi, uint32_t n, float *f,
                      float *pdf)
{
    Bsdf b{eval_closure(*mat)};
    for (uint32_t i = 0; i < n; ++i) {
        V3 o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), w(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        V3 fv;
        float p;
        b.eval_and_pdf(o, w, fv, p);
        f[3 * i] = fv.x;
        f[3 * i + 1] = fv.y;
        f[3 * i + 2] = fv.z;
        pdf[i] = p;
    }
}

void oracle_bsdf_sample(const ks_material_desc *mat, const float *wo, const float *u, uint32_t n, float *wi,
                        float *beta, float *pdf)
{
    Bsdf b{eval_closure(*mat)};
    for (uint32_t i = 0; i < n; ++i) {
        V3 o(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        V3 w;
        float p = 0.0f;
        V3 bt = b.sample(o, w, u[3 * i], u[3 * i + 1], u[3 * i + 2], p);
        wi[3 * i] = w.x;
        wi[3 * i + 1] = w.y;
        wi[3 * i + 2] = w.z;
        beta[3 * i] = bt.x;
        beta[3 * i + 1] = bt.y;
        beta[3 * i + 2] = bt.z;
        pdf[i] = p;
    }
}

} // extern "C"
