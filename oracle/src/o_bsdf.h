// ORACLE (test infrastructure only).  Restatement of keepsake's BSDFs with constant shader fields:
// PrincipledBSDF and PrincipledBRDF with the GGX or Beckmann microfacet distribution, Lambertian.
//
// Follows: principled_bsdf.cpp:246-705 (PrincipledBSDF: closure, eval, sample, pdf, lobe weights,
// per-lobe functions), principled_bsdf.cpp:11-225 (PrincipledBRDF), bsdf.cpp:13-41 (Lambertian),
// microfacet.h:20-147 (GGX D, lambda, G1, G2 with std::beta, VNDF sample), microfacet.h:155-318
// (Beckmann, BeckmannSample11, BeckmannSample), maths.h:598-627 (erfinv),
// fresnel.h:9-37, bsdf.h:47-52 + bsdf.cpp:64-92 (Henyey-Greenstein), rng.h:243-265
// (sample_disk, sample_cosine_hemisphere), rng.h:399-434 (sample_small_distrib),
// maths.h:1037-1049 (reflect, refract), maths.h:813-821 (orthonormal_basis).
#pragma once
#include "../../include/ks_b200.h"
#include "o_math.h"

#include <cmath>

namespace oracle
{

struct Closure
{
    V3 basecolor;
    float roughness, ax, ay, metallic, ior, specular_r0_mul, specular_trans, diffuse_trans, diffuse_trans_fwd;
    int microfacet;
    int bsdf;       // 0 PrincipledBSDF, 1 PrincipledBRDF, 2 Lambertian
    float specular; // PrincipledBRDF: clamp(specular, 0, 1) * 0.08 (principled_bsdf.cpp:22-23)
};

inline Closure eval_closure(const ks_material_desc &m)
{
    Closure c;
    c.basecolor = V3(std::clamp(m.basecolor[0], 0.0f, 1.0f), std::clamp(m.basecolor[1], 0.0f, 1.0f),
                     std::clamp(m.basecolor[2], 0.0f, 1.0f));
    c.roughness = std::clamp(m.roughness, 0.0f, 1.0f);
    c.ax = sqr(c.roughness);
    c.ay = c.ax;
    c.metallic = std::clamp(m.metallic, 0.0f, 1.0f);
    c.ior = std::clamp(m.ior, 1.0f, 4.0f);
    c.specular_r0_mul = m.specular_r0_mul * 2.0f;
    c.specular_r0_mul = std::max(c.specular_r0_mul, 0.0f);
    c.specular_trans = std::clamp(m.specular_trans, 0.0f, 1.0f);
    c.diffuse_trans = std::clamp(m.diffuse_trans, 0.0f, 1.0f);
    c.diffuse_trans_fwd = std::clamp(m.diffuse_trans_fwd, 0.0f, 1.0f);
    c.microfacet = m.microfacet;
    c.bsdf = m.bsdf;
    c.specular = std::clamp(m.specular, 0.0f, 1.0f) * 0.08f;
    return c;
}

// ---- GGX (microfacet.h:20-147) ---------------------------------------------------------------
struct GGX
{
    static constexpr float min_alpha = 1e-3f;
    float alpha_x, alpha_y;
    GGX(float ax, float ay) : alpha_x(std::clamp(ax, min_alpha, 1.0f)), alpha_y(std::clamp(ay, min_alpha, 1.0f)) {}
    bool isotropic() const { return alpha_x == alpha_y; }
    float D(V3 wm) const
    {
        if (wm.z <= 0.0f)
            return 0.0f;
        if (isotropic()) {
            float alpha = alpha_x;
            float a2 = alpha * alpha;
            float t = 1.0f + (a2 - 1.0f) * wm.z * wm.z;
            return a2 / (pi * t * t);
        }
        float hx = wm.x / alpha_x, hy = wm.y / alpha_y;
        float t = sqr(hx) + sqr(hy) + sqr(wm.z);
        return 1.0f / (pi * alpha_x * alpha_y * sqr(t));
    }
    float lambda(V3 w) const
    {
        if (w.z >= 1.0f || w.z <= -1.0f)
            return 0.0f;
        float alpha;
        if (isotropic()) {
            alpha = alpha_x;
        } else {
            float inv_sin_theta2 = 1.0f / (1.0f - w.z * w.z);
            float cos_phi2 = w.x * w.x * inv_sin_theta2;
            float sin_phi2 = w.y * w.y * inv_sin_theta2;
            alpha = std::sqrt(cos_phi2 * alpha_x * alpha_x + sin_phi2 * alpha_y * alpha_y);
        }
        float alpha2 = alpha * alpha;
        float NdotV2 = w.z * w.z;
        float t = (1.0f - NdotV2) * alpha2 / NdotV2;
        return 0.5f * (-1.0f + std::sqrt(1.0f + t));
    }
    float G1(V3 w) const { return 1.0f / (1.0f + lambda(w)); }
    float G2(V3 wo, V3 wi) const
    {
        if (wo.z * wi.z >= 0.0f)
            return 1.0f / (1.0f + lambda(wo) + lambda(wi));
        return (float)std::beta(1.0f + lambda(wo), 1.0f + lambda(wi));
    }
    V3 sample(V3 wo, float u0, float u1) const
    {
        V3 Vh = normalized(V3(alpha_x * wo.x, alpha_y * wo.y, wo.z));
        float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
        V3 T1 = lensq > 0 ? V3(-Vh.y, Vh.x, 0.0f) * (1.0f / std::sqrt(lensq)) : V3(1.0f, 0.0f, 0.0f);
        V3 T2 = cross(Vh, T1);
        float r = std::sqrt(u0);
        float phi = two_pi * u1;
        float t1 = r * std::cos(phi);
        float t2 = r * std::sin(phi);
        float s = 0.5f * (1.0f + Vh.z);
        t2 = (1.0f - s) * std::sqrt(1.0f - t1 * t1) + s * t2;
        V3 Nh = t1 * T1 + t2 * T2 + std::sqrt(std::max(0.0f, 1.0f - t1 * t1 - t2 * t2)) * Vh;
        return normalized(V3(alpha_x * Nh.x, alpha_y * Nh.y, std::max(0.0f, Nh.z)));
    }
};

// ---- erfinv (maths.h:598-627) -----------------------------------------------------------------
inline float erfinv(float x)
{
    float w, p;
    x = std::clamp(x, -.99999f, .99999f);
    w = -std::log((1 - x) * (1 + x));
    if (w < 5) {
        w = w - 2.5f;
        p = 2.81022636e-08f;
        p = 3.43273939e-07f + p * w;
        p = -3.5233877e-06f + p * w;
        p = -4.39150654e-06f + p * w;
        p = 0.00021858087f + p * w;
        p = -0.00125372503f + p * w;
        p = -0.00417768164f + p * w;
        p = 0.246640727f + p * w;
        p = 1.50140941f + p * w;
    } else {
        w = std::sqrt(w) - 3;
        p = -0.000200214257f;
        p = 0.000100950558f + p * w;
        p = 0.00134934322f + p * w;
        p = -0.00367342844f + p * w;
        p = 0.00573950773f + p * w;
        p = -0.0076224613f + p * w;
        p = 0.00943887047f + p * w;
        p = 1.00167406f + p * w;
        p = 2.83297682f + p * w;
    }
    return p * x;
}

// ---- Beckmann (microfacet.h:155-318) -----------------------------------------------------------
inline void beckmann_sample11(float cos_theta_i, float U1, float U2, float *slope_x, float *slope_y)
{
    if (cos_theta_i > .9999) {
        float r = std::sqrt(-std::log(1.0f - U1));
        float sin_phi = std::sin(2 * pi * U2);
        float cos_phi = std::cos(2 * pi * U2);
        *slope_x = r * cos_phi;
        *slope_y = r * sin_phi;
        return;
    }
    float sin_theta_i = std::sqrt(std::max((float)0, (float)1 - cos_theta_i * cos_theta_i));
    float tan_theta_i = sin_theta_i / cos_theta_i;
    float cot_theta_i = 1 / tan_theta_i;
    float a = -1, c = std::erf(cot_theta_i);
    float sample_x = std::max(U1, (float)1e-6f);
    float theta_i = std::acos(cos_theta_i);
    float fit = 1 + theta_i * (-0.876f + theta_i * (0.4265f - 0.0594f * theta_i));
    float b = c - (1 + c) * std::pow(1 - sample_x, fit);
    static const float sqrt_pi_inv = 1.f / std::sqrt(pi);
    float normalization = 1 / (1 + c + sqrt_pi_inv * tan_theta_i * std::exp(-cot_theta_i * cot_theta_i));
    int it = 0;
    while (++it < 10) {
        if (!(b >= a && b <= c))
            b = 0.5f * (a + c);
        float inv_erf = erfinv(b);
        float value = normalization * (1 + b + sqrt_pi_inv * tan_theta_i * std::exp(-inv_erf * inv_erf)) - sample_x;
        float derivative = normalization * (1 - inv_erf * tan_theta_i);
        if (std::abs(value) < 1e-5f)
            break;
        if (value > 0)
            c = b;
        else
            a = b;
        b -= value / derivative;
    }
    *slope_x = erfinv(b);
    *slope_y = erfinv(2.0f * std::max(U2, (float)1e-6f) - 1.0f);
}

struct Beckmann
{
    static constexpr float min_alpha = 1e-3f;
    float alpha_x, alpha_y;
    Beckmann(float ax, float ay)
        : alpha_x(std::clamp(ax, min_alpha, 1.0f)), alpha_y(std::clamp(ay, min_alpha, 1.0f))
    {
    }
    float D(V3 wm) const
    {
        float cos_theta2 = sqr(wm.z);
        float sin_theta2 = std::max(1.0f - cos_theta2, 0.0f);
        float tan_theta2 = sin_theta2 / cos_theta2;
        if (std::isinf(tan_theta2))
            return 0.0f;
        float cos_theta4 = sqr(cos_theta2);
        float sin_theta = std::sqrt(sin_theta2);
        float cos_phi = (sin_theta == 0) ? 1 : std::clamp(wm.x / sin_theta, -1.0f, 1.0f);
        float cos_phi2 = sqr(cos_phi);
        float sin_phi = (sin_theta == 0) ? 0 : std::clamp(wm.y / sin_theta, -1.0f, 1.0f);
        float sin_phi2 = sqr(sin_phi);
        return std::exp(-tan_theta2 * (cos_phi2 / sqr(alpha_x) + sin_phi2 / sqr(alpha_y))) /
               (pi * alpha_x * alpha_y * cos_theta4);
    }
    float lambda(V3 w) const
    {
        float cos_theta2 = sqr(w.z);
        float sin_theta2 = std::max(1.0f - cos_theta2, 0.0f);
        float sin_theta = std::sqrt(sin_theta2);
        float tan_theta = sin_theta / w.z;
        float abs_tan_theta = std::abs(tan_theta);
        if (std::isinf(abs_tan_theta))
            return 0.;
        float cos_phi = (sin_theta == 0) ? 1 : std::clamp(w.x / sin_theta, -1.0f, 1.0f);
        float cos_phi2 = sqr(cos_phi);
        float sin_phi = (sin_theta == 0) ? 0 : std::clamp(w.y / sin_theta, -1.0f, 1.0f);
        float sin_phi2 = sqr(sin_phi);
        float alpha = std::sqrt(cos_phi2 * sqr(alpha_x) + sin_phi2 * sqr(alpha_y));
        float a = 1 / (alpha * abs_tan_theta);
        if (a >= 1.6f)
            return 0;
        return (1 - 1.259f * a + 0.396f * a * a) / (3.535f * a + 2.181f * a * a);
    }
    float G1(V3 w) const { return 1.0f / (1.0f + lambda(w)); }
    float G2(V3 wo, V3 wi) const
    {
        if (wo.z * wi.z >= 0.0f)
            return 1.0f / (1.0f + lambda(wo) + lambda(wi));
        return (float)std::beta(1.0f + lambda(wo), 1.0f + lambda(wi));
    }
    V3 sample(V3 wo, float u0, float u1) const
    {
        bool flip = wo.z < 0;
        V3 wi = flip ? -wo : wo;
        // BeckmannSample (microfacet.h:217-245)
        V3 stretched = normalized(V3(alpha_x * wi.x, alpha_y * wi.y, wi.z));
        float slope_x, slope_y;
        beckmann_sample11(stretched.z, u0, u1, &slope_x, &slope_y);
        float cos_theta2 = sqr(stretched.z);
        float sin_theta2 = std::max(1.0f - cos_theta2, 0.0f);
        float sin_theta = std::sqrt(sin_theta2);
        float cos_phi = (sin_theta == 0) ? 1 : std::clamp(stretched.x / sin_theta, -1.0f, 1.0f);
        float sin_phi = (sin_theta == 0) ? 0 : std::clamp(stretched.y / sin_theta, -1.0f, 1.0f);
        float tmp = cos_phi * slope_x - sin_phi * slope_y;
        slope_y = sin_phi * slope_x + cos_phi * slope_y;
        slope_x = tmp;
        slope_x = alpha_x * slope_x;
        slope_y = alpha_y * slope_y;
        V3 wh = normalized(V3(-slope_x, -slope_y, 1.f));
        if (flip)
            wh = -wh;
        return wh;
    }
};

// ---- helpers ---------------------------------------------------------------------------------
inline float fresnel_dielectric(float cos_theta_i, float eta)
{
    float sin_theta_t_2 = eta * eta * (1.0f - cos_theta_i * cos_theta_i);
    if (sin_theta_t_2 > 1.0)
        return 1.0;
    float cos_theta_t = std::sqrt(std::max(1.0f - sin_theta_t_2, 0.0f));
    float rs = (eta * cos_theta_t - cos_theta_i) / (eta * cos_theta_t + cos_theta_i);
    float rp = (eta * cos_theta_i - cos_theta_t) / (eta * cos_theta_i + cos_theta_t);
    return 0.5f * (rs * rs + rp * rp);
}

inline float fresnel_schlick(float cos_theta_i)
{
    float schlick = saturate(1.0f - cos_theta_i);
    float schlick2 = sqr(schlick);
    schlick = schlick2 * schlick2 * schlick;
    return schlick;
}

inline V3 reflect(V3 w, V3 n) { return 2.0f * dot(n, w) * n - w; }

inline bool refract(V3 wi, V3 n, float eta, V3 &wt)
{
    float NdotI = dot(n, wi);
    float k = 1.0f - eta * eta * (1.0f - sqr(NdotI));
    if (k < 0.0f)
        return false;
    wt = -eta * wi + (eta * NdotI - std::sqrt(k)) * n;
    return true;
}

inline void sample_disk(float u0, float u1, float &dx, float &dy)
{
    float a = 2.0f * u0 - 1.0f;
    float b = 2.0f * u1 - 1.0f;
    if (a == 0.0f && b == 0.0f) {
        dx = dy = 0.0f;
        return;
    }
    float r, phi;
    if (a * a > b * b) {
        r = a;
        phi = 0.25f * pi * (b / a);
    } else {
        r = b;
        phi = half_pi - 0.25f * pi * (a / b);
    }
    dx = r * std::cos(phi);
    dy = r * std::sin(phi);
}

inline V3 sample_cosine_hemisphere(float u0, float u1)
{
    float dx, dy;
    sample_disk(u0, u1, dx, dy);
    float z = std::sqrt(std::max(0.0f, 1.0f - (dx * dx + dy * dy)));
    return V3(dx, dy, z);
}

inline float single_peaked_henyey_greenstein(float cos_theta, float g)
{
    return ((1.0f - g * g) / safe_pow(1.0f + g * g - 2.0f * g * cos_theta, 1.5f)) * (inv_pi * 0.25f);
}

inline void orthonormal_basis(V3 N, V3 &X, V3 &Y)
{
    float sign = std::copysign(1.0f, N.z);
    const float a = -1.0f / (sign + N.z);
    const float b = N.x * N.y * a;
    X = V3(1.0f + sign * N.x * N.x * a, sign * b, -sign * N.x);
    Y = V3(b, sign + N.y * N.y * a, -N.y);
}

inline V3 sample_henyey_greenstein(V3 D, float g, float randu, float randv, float *pdf)
{
    float cos_theta;
    bool isotropic = std::fabs(g) < 1e-3f;
    if (isotropic) {
        cos_theta = (1.0f - 2.0f * randu);
        if (pdf)
            *pdf = inv_pi * 0.25f;
    } else {
        float k = (1.0f - g * g) / (1.0f - g + 2.0f * g * randu);
        cos_theta = (1.0f + g * g - k * k) / (2.0f * g);
        if (pdf)
            *pdf = single_peaked_henyey_greenstein(cos_theta, g);
    }
    float sin_theta = safe_sqrt(1.0f - cos_theta * cos_theta);
    float phi = two_pi * randv;
    V3 dir(sin_theta * std::cos(phi), sin_theta * std::sin(phi), cos_theta);
    V3 T, B;
    orthonormal_basis(D, T, B);
    return dir.x * T + dir.y * B + dir.z * D;
}

inline int sample_small_distrib4(const float *data, float u, float *u_remap)
{
    const int N = 4;
    float sum_w = 0.0f;
    int last_positive = 0;
    for (int i = 0; i < N; ++i) {
        sum_w += data[i];
        if (data[i] > 0.0f)
            last_positive = i;
    }
    float inv_sum_w = 1.0f / sum_w;
    float cdf = 0.0f;
    int selected = -1;
    for (int i = 0; i < N; ++i) {
        float dcdf = data[i] * inv_sum_w;
        float cdf_next = cdf + dcdf;
        if (u < cdf_next) {
            selected = i;
            if (u_remap)
                *u_remap = (u - cdf) / (cdf_next - cdf);
            break;
        }
        cdf = cdf_next;
    }
    if (selected == -1)
        selected = last_positive;
    return selected;
}

// ---- PrincipledBSDF::internal (principled_bsdf.cpp:320-705) ---------------------------------
template <class MF>
struct PrincipledT
{
    Closure c;
    MF mf() const { return MF(c.ax, c.ay); }

    V3 eval_diffuse(V3 wo, V3 wi) const
    {
        float lobe_weight = (1.0f - c.metallic) * (1.0f - c.specular_trans) * (1.0f - c.diffuse_trans);
        if (lobe_weight == 0.0f)
            return V3();
        V3 wh = normalized(wo + wi);
        float Fd90 = 0.5f + 2.0f * c.roughness * wh.z;
        float disney_retro =
            std::lerp(1.0f, Fd90, fresnel_schlick(wi.z)) * std::lerp(1.0f, Fd90, fresnel_schlick(wo.z));
        return lobe_weight * c.basecolor * inv_pi * disney_retro * wi.z;
    }
    V3 eval_diffuse_transmission(V3 wo, V3 wi) const
    {
        float lobe_weight = (1.0f - c.metallic) * (1.0f - c.specular_trans) * c.diffuse_trans;
        if (lobe_weight == 0.0f)
            return V3();
        float fwd_scatter = single_peaked_henyey_greenstein(dot(wo, -wi), c.diffuse_trans_fwd);
        return lobe_weight * c.basecolor * inv_pi * (-wi.z) * fwd_scatter;
    }
    V3 eval_metallic_specular(V3 wo, V3 wi) const
    {
        float lobe_weight = c.metallic;
        if (lobe_weight == 0.0f)
            return V3();
        V3 wh = normalized(wo + wi);
        float D = mf().D(wh);
        float G = mf().G2(wo, wi);
        float fs = fresnel_schlick(dot(wo, wh));
        V3 Fr = lerp3(c.basecolor, V3(1, 1, 1), fs);
        return lobe_weight * D * G * Fr / (4.0f * wo.z);
    }
    float dielectric_specular_adjust(float wo_dot_wh) const
    {
        float R0 = sqr((1.0f - c.ior) / (1.0f + c.ior));
        float schlick = fresnel_schlick(wo_dot_wh);
        // ior 1 (R0 = 0) at wo = wh: 0 / 0 in the reference (principled_bsdf.cpp:508-513); the
        // ratio's limit there is 1
        const float den = std::lerp(R0, 1.0f, schlick);
        return den == 0.0f ? 1.0f : std::lerp(c.specular_r0_mul * R0, 1.0f, schlick) / den;
    }
    V3 eval_dielectric_specular(V3 wo, V3 wi) const
    {
        float lobe_weight = (1.0f - c.metallic);
        if (lobe_weight == 0.0f)
            return V3();
        bool refl = wo.z * wi.z >= 0.0f;
        float eta = wo.z >= 0.0f ? c.ior : (1.0f / c.ior);
        V3 wh;
        if (refl) {
            wh = normalized(wo + wi);
        } else {
            wh = normalized(wo + wi * eta);
            lobe_weight *= c.specular_trans;
        }
        if (wh.z < 0.0f)
            wh = -wh;
        float D = mf().D(wh);
        float G = mf().G2(wo, wi);
        float abs_wo_dot_wh = std::abs(dot(wo, wh));
        float Fr = fresnel_dielectric(abs_wo_dot_wh, 1.0f / eta);
        float f;
        if (refl) {
            float Fr_adj = dielectric_specular_adjust(abs_wo_dot_wh);
            f = D * G * (Fr * Fr_adj) / (4.0f * std::abs(wo.z));
        } else {
            float denom = sqr(dot(wo, wh) + eta * dot(wi, wh));
            float specular = D * G * (1.0f - Fr) * dot(wo, wh) * dot(wi, wh) / (denom * wo.z);
            // wi = -wo through ior 1 makes wo + eta wi vanish: 0 / 0, which the reference asserts
            // against (principled_bsdf.cpp:500); no transmission is counted there
            f = denom == 0.0f ? 0.0f : std::abs(specular);
        }
        V3 out(f, f, f);
        out *= lobe_weight;
        return out;
    }
    void lobe_weights(V3 wo, float w[4]) const
    {
        float lum = luminance(c.basecolor);
        float wd = wo.z > 0.0f ? (1.0f - c.metallic) * (1.0f - c.specular_trans) * lum * inv_pi : 0.0f;
        float weight_diffuse = wd * (1.0f - c.diffuse_trans);
        float weight_diffuse_transmission = wd * c.diffuse_trans;
        float weight_metallic = wo.z > 0.0f ? c.metallic * std::lerp(lum, 1.0f, fresnel_schlick(wo.z)) : 0.0f;
        float eta = wo.z >= 0.0f ? c.ior : (1.0f / c.ior);
        float weight_dielectric = (1.0f - c.metallic) * fresnel_dielectric(std::abs(wo.z), 1.0f / eta);
        float sum = weight_diffuse + weight_diffuse_transmission + weight_metallic + weight_dielectric;
        if (sum == 0.0f) {
            w[0] = w[1] = w[2] = w[3] = 0.0f;
            return;
        }
        w[0] = weight_diffuse / sum;
        w[1] = weight_diffuse_transmission / sum;
        w[2] = weight_metallic / sum;
        w[3] = weight_dielectric / sum;
    }
    float pdf_diffuse(V3, V3 wi) const { return wi.z * inv_pi; }
    float pdf_diffuse_transmission(V3 wo, V3 wi) const
    {
        if (c.diffuse_trans_fwd > 0.05f)
            return single_peaked_henyey_greenstein(dot(wo, -wi), c.diffuse_trans_fwd);
        return -wi.z * inv_pi;
    }
    float pdf_metallic_specular(V3 wo, V3 wi) const
    {
        V3 wh = normalized(wo + wi);
        return mf().D(wh) * mf().G1(wo) / (4.0f * std::abs(wo.z));
    }
    float pdf_dielectric_specular(V3 wo, V3 wi) const
    {
        bool refl = wo.z * wi.z >= 0.0f;
        float eta = wo.z >= 0.0f ? c.ior : (1.0f / c.ior);
        V3 wh = refl ? normalized(wo + wi) : normalized(wo + wi * eta);
        if (wh.z < 0.0f)
            wh = -wh;
        float D = mf().D(wh);
        float G1 = mf().G1(wo);
        float abs_wo_dot_wh = std::abs(dot(wo, wh));
        float Fr = fresnel_dielectric(std::abs(dot(wo, wh)), 1.0f / eta);
        float Fr_adj = dielectric_specular_adjust(abs_wo_dot_wh);
        float Fr_refl = Fr * Fr_adj;
        float Fr_refr = (1.0f - Fr) * c.specular_trans;
        if (Fr_refr == 0.0f)
            Fr_refl = 1.0f;
        float pdf;
        if (refl) {
            pdf = D * G1 / (4.0f * std::abs(wo.z));
            pdf *= Fr_refl / (Fr_refl + Fr_refr);
        } else {
            float denom = sqr(dot(wo, wh) + eta * dot(wi, wh));
            float jacobian = eta * eta * std::abs(dot(wi, wh)) / denom;
            pdf = denom == 0.0f ? 0.0f : D * G1 * std::abs(dot(wo, wh)) / std::abs(wo.z) * jacobian;
            pdf *= Fr_refr / (Fr_refl + Fr_refr);
        }
        return pdf;
    }
    V3 eval(V3 wo, V3 wi) const
    {
        if (wo.z == 0.0f || wi.z == 0.0f)
            return V3();
        V3 f;
        if (wo.z > 0.0f && wi.z > 0.0f) {
            f += eval_diffuse(wo, wi);
            f += eval_metallic_specular(wo, wi);
        }
        if (wo.z > 0.0f && wi.z < 0.0f)
            f += eval_diffuse_transmission(wo, wi);
        f += eval_dielectric_specular(wo, wi);
        return f;
    }
    float pdf(V3 wo, V3 wi) const
    {
        if (wo.z == 0.0f || wi.z == 0.0f)
            return 0.0f;
        float w[4];
        lobe_weights(wo, w);
        if (w[0] == 0.0f && w[1] == 0.0f && w[2] == 0.0f && w[3] == 0.0f)
            return 0.0f;
        float p[4] = {0, 0, 0, 0};
        if (wo.z > 0.0f && wi.z > 0.0f) {
            p[0] = pdf_diffuse(wo, wi);
            p[2] = pdf_metallic_specular(wo, wi);
        }
        if (wo.z > 0.0f && wi.z < 0.0f)
            p[1] = pdf_diffuse_transmission(wo, wi);
        p[3] = pdf_dielectric_specular(wo, wi);
        return p[0] * w[0] + p[1] * w[1] + p[2] * w[2] + p[3] * w[3];
    }
    // eval_and_pdf (principled_bsdf.cpp:297-307)
    void eval_and_pdf(V3 wo, V3 wi, V3 &f, float &p) const
    {
        f = eval(wo, wi);
        if (is_zero(f)) {
            p = 0.0f;
            return;
        }
        p = pdf(wo, wi);
    }
    V3 sample_metallic_specular(V3 wo, float u0, float u1, float &pdf) const
    {
        if (wo.z == 0.0f) {
            pdf = 0.0f;
            return V3();
        }
        V3 wh = mf().sample(sgn(wo.z) * wo, u0, u1);
        V3 wi = reflect(wo, wh);
        if (wo.z * wi.z < 0.0f) {
            pdf = 0.0f;
            return V3();
        }
        pdf = mf().D(wh) * mf().G1(wo) / (4.0f * std::abs(wo.z));
        return wi;
    }
    V3 sample_dielectric_specular(V3 wo, float u_lobe, float u0, float u1, float &pdf) const
    {
        if (wo.z == 0.0f) {
            pdf = 0.0f;
            return V3();
        }
        V3 wh = mf().sample(sgn(wo.z) * wo, u0, u1);
        float D = mf().D(wh);
        float G1 = mf().G1(wo);
        float eta = wo.z >= 0.0f ? c.ior : (1.0f / c.ior);
        float abs_wo_dot_wh = std::abs(dot(wo, wh));
        float Fr = fresnel_dielectric(std::abs(dot(wo, wh)), 1.0f / eta);
        float Fr_adj = dielectric_specular_adjust(abs_wo_dot_wh);
        float Fr_refl = Fr * Fr_adj;
        float Fr_refr = (1.0f - Fr) * c.specular_trans;
        if (Fr_refr == 0.0f)
            Fr_refl = 1.0f;
        V3 wi;
        if (u_lobe < Fr_refl / (Fr_refl + Fr_refr)) {
            wi = reflect(wo, wh);
            if (wo.z * wi.z < 0.0f) {
                pdf = 0.0f;
                return V3();
            }
            pdf = D * G1 / (4.0f * std::abs(wo.z));
            pdf *= Fr_refl / (Fr_refl + Fr_refr);
        } else {
            if (!refract(wo, sgn(wo.z) * wh, 1.0f / eta, wi)) {
                pdf = 0.0f;
                return V3();
            }
            if (wo.z * wi.z > 0.0f) {
                pdf = 0.0f;
                return V3();
            }
            float denom = sqr(dot(wo, wh) + eta * dot(wi, wh));
            if (denom == 0.0f) { // wi = -wo through ior 1: no density (the reference asserts a finite pdf)
                pdf = 0.0f;
                return V3();
            }
            float jacobian = eta * eta * std::abs(dot(wi, wh)) / denom;
            pdf = D * G1 * std::abs(dot(wo, wh)) / std::abs(wo.z) * jacobian;
            pdf *= Fr_refr / (Fr_refl + Fr_refr);
        }
        return wi;
    }
    V3 sample_diffuse_transmission(V3 wo, float u0, float u1, float &pdf) const
    {
        if (c.diffuse_trans_fwd > 0.05f)
            return sample_henyey_greenstein(-wo, c.diffuse_trans_fwd, u0, u1, &pdf);
        V3 wi = sample_cosine_hemisphere(u0, u1);
        pdf = wi.z * inv_pi;
        wi.z = -wi.z;
        return wi;
    }
    // sample (principled_bsdf.cpp:326-393): returns f / pdf, writes wi and pdf
    V3 sample(V3 wo, V3 &wi, float u_lobe, float u0, float u1, float &pdf) const
    {
        if (wo.z == 0.0f) {
            pdf = 0.0f;
            return V3();
        }
        float w[4];
        lobe_weights(wo, w);
        if (w[0] == 0.0f && w[1] == 0.0f && w[2] == 0.0f && w[3] == 0.0f) {
            pdf = 0.0f;
            return V3();
        }
        float u_remap = 0.0f;
        int lobe = sample_small_distrib4(w, u_lobe, &u_remap);
        float p[4] = {0, 0, 0, 0};
        if (lobe == 0) {
            wi = sample_cosine_hemisphere(u0, u1);
            p[0] = wi.z * inv_pi;
            if (is_zero(wi) || p[0] == 0.0f) {
                pdf = 0.0f;
                return V3();
            }
            if (wo.z > 0.0f && wi.z > 0.0f)
                p[2] = pdf_metallic_specular(wo, wi);
            p[3] = pdf_dielectric_specular(wo, wi);
        } else if (lobe == 1) {
            wi = sample_diffuse_transmission(wo, u0, u1, p[1]);
            if (is_zero(wi) || p[1] == 0.0f) {
                pdf = 0.0f;
                return V3();
            }
            p[3] = pdf_dielectric_specular(wo, wi);
        } else if (lobe == 2) {
            wi = sample_metallic_specular(wo, u0, u1, p[2]);
            if (is_zero(wi) || p[2] == 0.0f) {
                pdf = 0.0f;
                return V3();
            }
            if (wo.z > 0.0f && wi.z > 0.0f)
                p[0] = pdf_diffuse(wo, wi);
            p[3] = pdf_dielectric_specular(wo, wi);
        } else {
            wi = sample_dielectric_specular(wo, u_remap, u0, u1, p[3]);
            if (is_zero(wi) || p[3] == 0.0f) {
                pdf = 0.0f;
                return V3();
            }
            if (wo.z > 0.0f && wi.z > 0.0f) {
                p[0] = pdf_diffuse(wo, wi);
                p[2] = pdf_metallic_specular(wo, wi);
            }
            if (wo.z > 0.0f && wi.z < 0.0f)
                p[1] = pdf_diffuse_transmission(wo, wi);
        }
        pdf = p[0] * w[0] + p[1] * w[1] + p[2] * w[2] + p[3] * w[3];
        return eval(wo, wi) / pdf;
    }
};

using Principled = PrincipledT<GGX>;

// ---- PrincipledBRDF::internal (principled_bsdf.cpp:61-225) -----------------------------------
template <class MF>
struct PrincipledBrdfT
{
    Closure c;
    MF mf() const { return MF(c.ax, c.ay); }
    V3 eval_diffuse(V3, V3 wi) const
    {
        float lobe_weight = (1.0f - c.metallic);
        if (lobe_weight == 0.0f)
            return V3();
        return lobe_weight * c.basecolor * inv_pi * wi.z;
    }
    V3 eval_specular(V3 wo, V3 wi) const
    {
        V3 wh = normalized(wo + wi);
        float D = mf().D(wh);
        float G = mf().G2(wo, wi);
        V3 R0 = lerp3(V3(c.specular, c.specular, c.specular), c.basecolor, c.metallic);
        V3 Fr = lerp3(R0, V3(1, 1, 1), fresnel_schlick(dot(wo, wh)));
        return D * G * Fr / (4.0f * wo.z);
    }
    void lobe_sample_weights(V3 wo, float w[2]) const
    {
        float lum_basecolor = luminance(c.basecolor);
        float lum_R0 = std::lerp(c.specular, lum_basecolor, c.metallic);
        float weight_diffuse = wo.z > 0.0f ? (1.0f - c.metallic) * lum_basecolor * inv_pi : 0.0f;
        float weight_specular = wo.z > 0.0f ? std::lerp(lum_R0, 1.0f, fresnel_schlick(wo.z)) : 0.0f;
        float sum = weight_diffuse + weight_specular;
        if (sum == 0.0f) {
            w[0] = w[1] = 0.0f;
            return;
        }
        float inv_sum = 1.0f / sum;
        w[0] = weight_diffuse * inv_sum;
        w[1] = weight_specular * inv_sum;
    }
    float pdf_diffuse(V3, V3 wi) const { return wi.z * inv_pi; }
    float pdf_specular(V3 wo, V3 wi) const
    {
        V3 wh = normalized(wo + wi);
        float D = mf().D(wh);
        float G1 = mf().G1(wo);
        return D * G1 / (4.0f * std::abs(wo.z));
    }
    V3 eval(V3 wo, V3 wi) const
    {
        if (wo.z == 0.0f || wi.z == 0.0f)
            return V3();
        V3 f;
        if (wo.z > 0.0f && wi.z > 0.0f) {
            f += eval_diffuse(wo, wi);
            f += eval_specular(wo, wi);
        }
        return f;
    }
    float pdf(V3 wo, V3 wi) const
    {
        if (wo.z == 0.0f || wi.z == 0.0f)
            return 0.0f;
        float w[2];
        lobe_sample_weights(wo, w);
        if (w[0] == 0.0f && w[1] == 0.0f)
            return 0.0f;
        if (wo.z <= 0.0f || wi.z <= 0.0f)
            return 0.0f;
        float p[2] = {0.0f, 0.0f};
        if (wo.z > 0.0f && wi.z > 0.0f) {
            p[0] = pdf_diffuse(wo, wi);
            p[1] = pdf_specular(wo, wi);
        }
        return p[0] * w[0] + p[1] * w[1];
    }
    void eval_and_pdf(V3 wo, V3 wi, V3 &f, float &p) const
    {
        f = eval(wo, wi);
        if (is_zero(f)) {
            p = 0.0f;
            return;
        }
        p = pdf(wo, wi);
    }
    V3 sample_specular(V3 wo, float u0, float u1, float &pdf) const
    {
        if (wo.z == 0.0f) {
            pdf = 0.0f;
            return V3();
        }
        V3 wh = mf().sample(sgn(wo.z) * wo, u0, u1);
        V3 wi = reflect(wo, wh);
        if (wo.z * wi.z < 0.0f) {
            pdf = 0.0f;
            return V3();
        }
        float D = mf().D(wh);
        float G1 = mf().G1(wo);
        pdf = D * G1 / (4.0f * std::abs(wo.z));
        return wi;
    }
    V3 sample(V3 wo, V3 &wi, float u_lobe, float u0, float u1, float &pdf) const
    {
        if (wo.z == 0.0f) {
            pdf = 0.0f;
            return V3();
        }
        float w[2];
        lobe_sample_weights(wo, w);
        if (w[0] == 0.0f && w[1] == 0.0f) {
            pdf = 0.0f;
            return V3();
        }
        // sample_small_distrib over the two weights (rng.h:399-432)
        float w4[4] = {w[0], w[1], 0.0f, 0.0f};
        int lobe = sample_small_distrib4(w4, u_lobe, nullptr);
        float p[2] = {0.0f, 0.0f};
        if (lobe == 0) {
            wi = sample_cosine_hemisphere(u0, u1);
            p[0] = wi.z * inv_pi;
            if (is_zero(wi) || p[0] == 0.0f) {
                pdf = 0.0f;
                return V3();
            }
            if (wo.z > 0.0f && wi.z > 0.0f)
                p[1] = pdf_specular(wo, wi);
        } else {
            wi = sample_specular(wo, u0, u1, p[1]);
            if (is_zero(wi)) {
                pdf = 0.0f;
                return V3();
            }
            if (wo.z > 0.0f && wi.z > 0.0f)
                p[0] = pdf_diffuse(wo, wi);
        }
        pdf = p[0] * w[0] + p[1] * w[1];
        return eval(wo, wi) / pdf;
    }
};

// ---- Lambertian (bsdf.cpp:13-41) -------------------------------------------------------------
struct Lambertian
{
    Closure c;
    V3 eval(V3 wo, V3 wi) const
    {
        if (wo.z <= 0.0f || wi.z <= 0.0f)
            return V3();
        return inv_pi * c.basecolor * wi.z;
    }
    float pdf(V3 wo, V3 wi) const
    {
        if (wo.z <= 0.0f || wi.z <= 0.0f)
            return 0.0f;
        return wi.z * inv_pi;
    }
    // BSDF::eval_and_pdf (bsdf.cpp:8-11)
    void eval_and_pdf(V3 wo, V3 wi, V3 &f, float &p) const
    {
        f = eval(wo, wi);
        p = pdf(wo, wi);
    }
    V3 sample(V3 wo, V3 &wi, float, float u0, float u1, float &pdf) const
    {
        if (wo.z <= 0.0f) {
            pdf = 0.0f;
            return V3();
        }
        wi = sample_cosine_hemisphere(u0, u1);
        pdf = wi.z * inv_pi;
        return c.basecolor;
    }
};

// A material's BSDF (Material::bsdf, material.h:39), by type and microfacet distribution.
// LambertianSubsurfaceExitAdapter (subsurface.cpp:502-532): the cosine lobe at a random walk's
// exit, times eta^2 (c.ior holds eta); only wi is read.
struct SubsurfaceExit
{
    Closure c;
    void eval_and_pdf(V3, V3 wi, V3 &f, float &p) const
    {
        if (wi.z <= 0.0f) {
            f = V3();
            p = 0.0f;
            return;
        }
        f = V3(inv_pi * wi.z, inv_pi * wi.z, inv_pi * wi.z);
        f *= c.ior * c.ior;
        p = wi.z * inv_pi;
    }
    V3 sample(V3, V3 &wi, float, float u0, float u1, float &pdf) const
    {
        wi = sample_cosine_hemisphere(u0, u1);
        pdf = wi.z * inv_pi;
        const float e2 = c.ior * c.ior;
        return V3(e2, e2, e2);
    }
};

struct Bsdf
{
    Closure c;
    template <class F>
    auto visit(F &&fn) const
    {
        if (c.bsdf == 3)
            return fn(SubsurfaceExit{c});
        if (c.bsdf == 2)
            return fn(Lambertian{c});
        if (c.bsdf == 1)
            return c.microfacet == 1 ? fn(PrincipledBrdfT<Beckmann>{c}) : fn(PrincipledBrdfT<GGX>{c});
        return c.microfacet == 1 ? fn(PrincipledT<Beckmann>{c}) : fn(PrincipledT<GGX>{c});
    }
    void eval_and_pdf(V3 wo, V3 wi, V3 &f, float &p) const
    {
        visit([&](const auto &b) { b.eval_and_pdf(wo, wi, f, p); return 0; });
    }
    V3 sample(V3 wo, V3 &wi, float u_lobe, float u0, float u1, float &pdf) const
    {
        return visit([&](const auto &b) { return b.sample(wo, wi, u_lobe, u0, u1, pdf); });
    }
};

} // namespace oracle
