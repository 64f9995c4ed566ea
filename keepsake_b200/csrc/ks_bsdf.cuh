// The BSDFs of the small_pt path on the device: PrincipledBSDF, PrincipledBRDF and Lambertian,
// each principled one with the GGX or the Beckmann microfacet distribution.
//
// Follows principled_bsdf.cpp:246-705 (PrincipledBSDF: closure, eval, sample, pdf, lobe weights),
// principled_bsdf.cpp:11-225 (PrincipledBRDF), bsdf.cpp:13-41 (Lambertian), microfacet.h:20-147
// (GGX D, lambda, G1, G2, VNDF sample), microfacet.h:155-257 (Beckmann D, lambda, G1, G2 and the
// visible-slope sampling of BeckmannSample11 / BeckmannSample), maths.h:598-627 (erfinv: M. Giles'
// single-precision approximation, "Approximating the erfinv function", GPU Computing Gems 2011),
// fresnel.h:9-37, bsdf.h:47-52 + bsdf.cpp:64-92 (Henyey-Greenstein), rng.h:243-265 (concentric
// disk, cosine hemisphere) and rng.h:399-434 (sample_small_distrib).  Floating-point expressions
// keep the reference's operand order; the transcendental functions are CUDA's (sinf, cosf, powf,
// expf, logf, erff, acosf, lgammaf), whose last-ulp differences from the host libm are the only
// source of divergence from the CPU path.
#pragma once
#include "ks_math.cuh"
#include "ks_scene.h"

namespace ksb
{

// BSDF kinds: MaterialGPU::bsdf * 2 + MaterialGPU::microfacet, Lambertian last.
enum : int
{
    kBsdfPrincipledGGX = 0,
    kBsdfPrincipledBeckmann = 1,
    kBrdfPrincipledGGX = 2,
    kBrdfPrincipledBeckmann = 3,
    kBsdfLambertian = 4,
    kBsdfSubsurfaceExit = 5 // LambertianSubsurfaceExitAdapter: basecolor holds eta^2
};

struct Closure
{
    f3 basecolor;
    float roughness, ax, ay, metallic, ior, specular_r0_mul, specular_trans, diffuse_trans, diffuse_trans_fwd;
    float specular; // PrincipledBRDF: clamp(specular, 0, 1) * 0.08 (principled_bsdf.cpp:22-23)
    int kind;
};

KS_D int bsdf_kind(const MaterialGPU &m)
{
    return m.bsdf == 2 ? kBsdfLambertian : m.bsdf * 2 + m.microfacet;
}

// PrincipledBSDF::eval_closure (principled_bsdf.cpp:245-276) for the principled BSDF; the
// PrincipledBRDF closure (principled_bsdf.cpp:11-29) and Lambertian's clamped albedo
// (bsdf.cpp:17-18) reuse basecolor, ax / ay and metallic.
KS_D Closure make_closure(const MaterialGPU &m)
{
    Closure c;
    c.kind = bsdf_kind(m);
    c.specular = clampf(m.specular, 0.0f, 1.0f) * 0.08f;
    c.basecolor = mk(clampf(m.basecolor[0], 0.0f, 1.0f), clampf(m.basecolor[1], 0.0f, 1.0f),
                     clampf(m.basecolor[2], 0.0f, 1.0f));
    c.roughness = clampf(m.roughness, 0.0f, 1.0f);
    c.ax = sqr(c.roughness);
    c.ay = c.ax;
    c.metallic = clampf(m.metallic, 0.0f, 1.0f);
    c.ior = clampf(m.ior, 1.0f, 4.0f);
    c.specular_r0_mul = m.specular_r0_mul * 2.0f;
    c.specular_r0_mul = c.specular_r0_mul < 0.0f ? 0.0f : c.specular_r0_mul;
    c.specular_trans = clampf(m.specular_trans, 0.0f, 1.0f);
    c.diffuse_trans = clampf(m.diffuse_trans, 0.0f, 1.0f);
    c.diffuse_trans_fwd = clampf(m.diffuse_trans_fwd, 0.0f, 1.0f);
    return c;
}

struct GGXd
{
    float ax, ay;
    KS_D GGXd(float a, float b)
    {
        ax = clampf(a, 1e-3f, 1.0f);
        ay = clampf(b, 1e-3f, 1.0f);
    }
    KS_D bool iso() const { return ax == ay; }
    KS_D float D(f3 wm) const
    {
        if (wm.z <= 0.0f)
            return 0.0f;
        if (iso()) {
            float a2 = ax * ax;
            float t = 1.0f + (a2 - 1.0f) * wm.z * wm.z;
            return a2 / (kPi * t * t);
        }
        float hx = wm.x / ax, hy = wm.y / ay;
        float t = sqr(hx) + sqr(hy) + sqr(wm.z);
        return 1.0f / (kPi * ax * ay * sqr(t));
    }
    KS_D float lambda(f3 w) const
    {
        if (w.z >= 1.0f || w.z <= -1.0f)
            return 0.0f;
        float alpha;
        if (iso()) {
            alpha = ax;
        } else {
            float inv_sin_theta2 = 1.0f / (1.0f - w.z * w.z);
            float cos_phi2 = w.x * w.x * inv_sin_theta2;
            float sin_phi2 = w.y * w.y * inv_sin_theta2;
            alpha = sqrtf(cos_phi2 * ax * ax + sin_phi2 * ay * ay);
        }
        float alpha2 = alpha * alpha;
        float NdotV2 = w.z * w.z;
        float t = (1.0f - NdotV2) * alpha2 / NdotV2;
        return 0.5f * (-1.0f + sqrtf(1.0f + t));
    }
    KS_D float G1(f3 w) const { return 1.0f / (1.0f + lambda(w)); }
    KS_D float G2(f3 wo, f3 wi) const
    {
        if (wo.z * wi.z >= 0.0f)
            return 1.0f / (1.0f + lambda(wo) + lambda(wi));
        // std::beta(a, b) for float arguments: exp(lgamma(a) + lgamma(b) - lgamma(a + b)) in float
        float a = 1.0f + lambda(wo), b = 1.0f + lambda(wi);
        return expf(lgammaf(a) + lgammaf(b) - lgammaf(a + b));
    }
    KS_D f3 sample(f3 wo, float u0, float u1) const
    {
        f3 Vh = normalize(mk(ax * wo.x, ay * wo.y, wo.z));
        float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
        f3 T1 = lensq > 0 ? mk(-Vh.y, Vh.x, 0.0f) * (1.0f / sqrtf(lensq)) : mk(1.0f, 0.0f, 0.0f);
        f3 T2 = cross(Vh, T1);
        float r = sqrtf(u0);
        float phi = kTwoPi * u1;
        float t1 = r * cosf(phi);
        float t2 = r * sinf(phi);
        float s = 0.5f * (1.0f + Vh.z);
        t2 = (1.0f - s) * sqrtf(1.0f - t1 * t1) + s * t2;
        float nz = 1.0f - t1 * t1 - t2 * t2;
        f3 Nh = t1 * T1 + t2 * T2 + sqrtf(nz > 0.0f ? nz : 0.0f) * Vh;
        return normalize(mk(ax * Nh.x, ay * Nh.y, Nh.z > 0.0f ? Nh.z : 0.0f));
    }
};

// erfinv (maths.h:598-627): M. Giles' single-precision approximation of the inverse error
// function on x clamped to +-0.99999, two polynomials in w = -log((1 - x)(1 + x)).
KS_D float erfinv_giles(float x)
{
    x = clampf(x, -.99999f, .99999f);
    float w = -logf((1 - x) * (1 + x)), p;
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
        w = sqrtf(w) - 3;
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

// Beckmann microfacet distribution (microfacet.h:155-257).  Visible normals are drawn by
// stretching wo to the unit-roughness configuration, sampling the slope distribution P22 of
// Jakob's numerical CDF inversion (Newton steps guarded by bisection in the erf domain, from the
// fitted first guess; BeckmannSample11) and un-stretching.
struct Beckmannd
{
    float ax, ay;
    KS_D Beckmannd(float a, float b)
    {
        ax = clampf(a, 1e-3f, 1.0f);
        ay = clampf(b, 1e-3f, 1.0f);
    }
    KS_D float D(f3 wm) const
    {
        float cos_theta2 = sqr(wm.z);
        float sin_theta2 = fmaxf(1.0f - cos_theta2, 0.0f);
        float tan_theta2 = sin_theta2 / cos_theta2;
        if (isinf(tan_theta2))
            return 0.0f;
        float cos_theta4 = sqr(cos_theta2);
        float sin_theta = sqrtf(sin_theta2);
        float cos_phi = (sin_theta == 0) ? 1.0f : clampf(wm.x / sin_theta, -1.0f, 1.0f);
        float sin_phi = (sin_theta == 0) ? 0.0f : clampf(wm.y / sin_theta, -1.0f, 1.0f);
        return expf(-tan_theta2 * (sqr(cos_phi) / sqr(ax) + sqr(sin_phi) / sqr(ay))) /
               (kPi * ax * ay * cos_theta4);
    }
    KS_D float lambda(f3 w) const
    {
        float cos_theta2 = sqr(w.z);
        float sin_theta2 = fmaxf(1.0f - cos_theta2, 0.0f);
        float sin_theta = sqrtf(sin_theta2);
        float abs_tan = fabsf(sin_theta / w.z);
        if (isinf(abs_tan))
            return 0.0f;
        float cos_phi = (sin_theta == 0) ? 1.0f : clampf(w.x / sin_theta, -1.0f, 1.0f);
        float sin_phi = (sin_theta == 0) ? 0.0f : clampf(w.y / sin_theta, -1.0f, 1.0f);
        float alpha = sqrtf(sqr(cos_phi) * sqr(ax) + sqr(sin_phi) * sqr(ay));
        float a = 1 / (alpha * abs_tan);
        if (a >= 1.6f)
            return 0.0f;
        return (1 - 1.259f * a + 0.396f * a * a) / (3.535f * a + 2.181f * a * a);
    }
    KS_D float G1(f3 w) const { return 1.0f / (1.0f + lambda(w)); }
    KS_D float G2(f3 wo, f3 wi) const
    {
        if (wo.z * wi.z >= 0.0f)
            return 1.0f / (1.0f + lambda(wo) + lambda(wi));
        float a = 1.0f + lambda(wo), b = 1.0f + lambda(wi);
        return expf(lgammaf(a) + lgammaf(b) - lgammaf(a + b));
    }
    // BeckmannSample11 (microfacet.h:155-215): slopes of unit roughness for cos(theta_i)
    KS_D static void sample11(float cos_i, float U1, float U2, float &sx, float &sy)
    {
        if ((double)cos_i > .9999) {
            float r = sqrtf(-logf(1.0f - U1));
            float phi = 2 * kPi * U2;
            sx = r * cosf(phi);
            sy = r * sinf(phi);
            return;
        }
        float sin_i = sqrtf(fmaxf(0.0f, 1.0f - cos_i * cos_i));
        float tan_i = sin_i / cos_i;
        float cot_i = 1 / tan_i;
        float a = -1, c = erff(cot_i);
        float sample_x = fmaxf(U1, 1e-6f);
        float theta_i = acosf(cos_i);
        float fit = 1 + theta_i * (-0.876f + theta_i * (0.4265f - 0.0594f * theta_i));
        float b = c - (1 + c) * powf(1 - sample_x, fit);
        const float sqrt_pi_inv = 1.f / sqrtf(kPi);
        float normalization = 1 / (1 + c + sqrt_pi_inv * tan_i * expf(-cot_i * cot_i));
        for (int it = 1; it < 10; ++it) {
            if (!(b >= a && b <= c))
                b = 0.5f * (a + c);
            float inv_erf = erfinv_giles(b);
            float value = normalization * (1 + b + sqrt_pi_inv * tan_i * expf(-inv_erf * inv_erf)) - sample_x;
            float derivative = normalization * (1 - inv_erf * tan_i);
            if (fabsf(value) < 1e-5f)
                break;
            if (value > 0)
                c = b;
            else
                a = b;
            b -= value / derivative;
        }
        sx = erfinv_giles(b);
        sy = erfinv_giles(2.0f * fmaxf(U2, 1e-6f) - 1.0f);
    }
    // Beckmann::sample(wo, u) with BeckmannSample (microfacet.h:217-245, 310-318)
    KS_D f3 sample(f3 wo, float u0, float u1) const
    {
        const bool flip = wo.z < 0;
        const f3 w = flip ? -wo : wo;
        f3 ws = normalize(mk(ax * w.x, ay * w.y, w.z));
        float sx, sy;
        sample11(ws.z, u0, u1, sx, sy);
        float sin_theta = sqrtf(fmaxf(1.0f - sqr(ws.z), 0.0f));
        float cos_phi = (sin_theta == 0) ? 1.0f : clampf(ws.x / sin_theta, -1.0f, 1.0f);
        float sin_phi = (sin_theta == 0) ? 0.0f : clampf(ws.y / sin_theta, -1.0f, 1.0f);
        float tmp = cos_phi * sx - sin_phi * sy;
        sy = sin_phi * sx + cos_phi * sy;
        sx = tmp;
        sx = ax * sx;
        sy = ay * sy;
        f3 wh = normalize(mk(-sx, -sy, 1.0f));
        return flip ? -wh : wh;
    }
};

KS_D float fresnel_dielectric(float cos_theta_i, float eta)
{
    float sin_theta_t_2 = eta * eta * (1.0f - cos_theta_i * cos_theta_i);
    if (sin_theta_t_2 > 1.0f)
        return 1.0f;
    float x = 1.0f - sin_theta_t_2;
    float cos_theta_t = sqrtf(x > 0.0f ? x : 0.0f);
    float rs = (eta * cos_theta_t - cos_theta_i) / (eta * cos_theta_t + cos_theta_i);
    float rp = (eta * cos_theta_i - cos_theta_t) / (eta * cos_theta_i + cos_theta_t);
    return 0.5f * (rs * rs + rp * rp);
}

KS_D float fresnel_schlick(float c)
{
    float s = saturate(1.0f - c);
    float s2 = sqr(s);
    return s2 * s2 * s;
}

KS_D f3 reflect(f3 w, f3 n) { return 2.0f * dot(n, w) * n - w; }

KS_D bool refract(f3 wi, f3 n, float eta, f3 &wt)
{
    float NdotI = dot(n, wi);
    float k = 1.0f - eta * eta * (1.0f - sqr(NdotI));
    if (k < 0.0f)
        return false;
    wt = -eta * wi + (eta * NdotI - sqrtf(k)) * n;
    return true;
}

KS_D f3 sample_cosine_hemisphere(float u0, float u1)
{
    float a = 2.0f * u0 - 1.0f, b = 2.0f * u1 - 1.0f;
    float dx = 0.0f, dy = 0.0f;
    if (!(a == 0.0f && b == 0.0f)) {
        float r, phi;
        if (a * a > b * b) {
            r = a;
            phi = 0.25f * kPi * (b / a);
        } else {
            r = b;
            phi = kHalfPi - 0.25f * kPi * (a / b);
        }
        dx = r * cosf(phi);
        dy = r * sinf(phi);
    }
    float z2 = 1.0f - (dx * dx + dy * dy);
    return mk(dx, dy, sqrtf(z2 > 0.0f ? z2 : 0.0f));
}

KS_D float hg_pdf(float cos_theta, float g)
{
    float base = 1.0f + g * g - 2.0f * g * cos_theta;
    float p = (base == 0.0f) ? 0.0f : powf(base, 1.5f);
    return ((1.0f - g * g) / p) * (kInvPi * 0.25f);
}

KS_D f3 sample_hg(f3 D, float g, float randu, float randv, float &pdf)
{
    float cos_theta;
    if (fabsf(g) < 1e-3f) {
        cos_theta = (1.0f - 2.0f * randu);
        pdf = kInvPi * 0.25f;
    } else {
        float k = (1.0f - g * g) / (1.0f - g + 2.0f * g * randu);
        cos_theta = (1.0f + g * g - k * k) / (2.0f * g);
        pdf = hg_pdf(cos_theta, g);
    }
    float x = 1.0f - cos_theta * cos_theta;
    float sin_theta = sqrtf(x > 0.0f ? x : 0.0f);
    float phi = kTwoPi * randv;
    f3 dir = mk(sin_theta * cosf(phi), sin_theta * sinf(phi), cos_theta);
    float sign = copysignf(1.0f, D.z);
    const float a = -1.0f / (sign + D.z);
    const float b = D.x * D.y * a;
    f3 T = mk(1.0f + sign * D.x * D.x * a, sign * b, -sign * D.x);
    f3 B = mk(b, sign + D.y * D.y * a, -D.y);
    return dir.x * T + dir.y * B + dir.z * D;
}

// PrincipledBSDF::internal (principled_bsdf.cpp:320-705) over a microfacet distribution MF.
template <class MF>
struct PrincipledT
{
    Closure c;
    KS_D MF mf() const { return MF(c.ax, c.ay); }

    KS_D f3 eval_diffuse(f3 wo, f3 wi) const
    {
        float lw = (1.0f - c.metallic) * (1.0f - c.specular_trans) * (1.0f - c.diffuse_trans);
        if (lw == 0.0f)
            return mk(0, 0, 0);
        f3 wh = normalize(wo + wi);
        float Fd90 = 0.5f + 2.0f * c.roughness * wh.z;
        float retro = std_lerp(1.0f, Fd90, fresnel_schlick(wi.z)) * std_lerp(1.0f, Fd90, fresnel_schlick(wo.z));
        return lw * c.basecolor * kInvPi * retro * wi.z;
    }
    KS_D f3 eval_diffuse_transmission(f3 wo, f3 wi) const
    {
        float lw = (1.0f - c.metallic) * (1.0f - c.specular_trans) * c.diffuse_trans;
        if (lw == 0.0f)
            return mk(0, 0, 0);
        float fwd = hg_pdf(dot(wo, -wi), c.diffuse_trans_fwd);
        return lw * c.basecolor * kInvPi * (-wi.z) * fwd;
    }
    KS_D f3 eval_metallic_specular(f3 wo, f3 wi) const
    {
        float lw = c.metallic;
        if (lw == 0.0f)
            return mk(0, 0, 0);
        f3 wh = normalize(wo + wi);
        float D = mf().D(wh);
        float G = mf().G2(wo, wi);
        float fs = fresnel_schlick(dot(wo, wh));
        f3 Fr = (1.0f - fs) * c.basecolor + fs * mk(1.0f, 1.0f, 1.0f);
        return lw * D * G * Fr / (4.0f * wo.z);
    }
    KS_D float dielectric_specular_adjust(float wo_dot_wh) const
    {
        float R0 = sqr((1.0f - c.ior) / (1.0f + c.ior));
        float schlick = fresnel_schlick(wo_dot_wh);
        // ior 1 (R0 = 0) at wo = wh: 0 / 0 in the reference; the ratio's limit there is 1
        const float den = std_lerp(R0, 1.0f, schlick);
        return den == 0.0f ? 1.0f : std_lerp(c.specular_r0_mul * R0, 1.0f, schlick) / den;
    }
    KS_D f3 eval_dielectric_specular(f3 wo, f3 wi) const
    {
        float lw = (1.0f - c.metallic);
        if (lw == 0.0f)
            return mk(0, 0, 0);
        bool refl = wo.z * wi.z >= 0.0f;
        float eta = wo.z >= 0.0f ? c.ior : (1.0f / c.ior);
        f3 wh;
        if (refl) {
            wh = normalize(wo + wi);
        } else {
            wh = normalize(wo + wi * eta);
            lw *= c.specular_trans;
        }
        if (wh.z < 0.0f)
            wh = -wh;
        float D = mf().D(wh);
        float G = mf().G2(wo, wi);
        float awh = fabsf(dot(wo, wh));
        float Fr = fresnel_dielectric(awh, 1.0f / eta);
        float f;
        if (refl) {
            float Fr_adj = dielectric_specular_adjust(awh);
            f = D * G * (Fr * Fr_adj) / (4.0f * fabsf(wo.z));
        } else {
            float denom = sqr(dot(wo, wh) + eta * dot(wi, wh));
            float spec = D * G * (1.0f - Fr) * dot(wo, wh) * dot(wi, wh) / (denom * wo.z);
            // wi = -wo through ior 1: wo + eta wi vanishes (0 / 0, asserted against by the reference)
            f = denom == 0.0f ? 0.0f : fabsf(spec);
        }
        f3 out = mk(f, f, f);
        out *= lw;
        return out;
    }
    KS_D void lobe_weights(f3 wo, float w[4]) const
    {
        float lum = luminance(c.basecolor);
        float wd = wo.z > 0.0f ? (1.0f - c.metallic) * (1.0f - c.specular_trans) * lum * kInvPi : 0.0f;
        float w0 = wd * (1.0f - c.diffuse_trans);
        float w1 = wd * c.diffuse_trans;
        float w2 = wo.z > 0.0f ? c.metallic * std_lerp(lum, 1.0f, fresnel_schlick(wo.z)) : 0.0f;
        float eta = wo.z >= 0.0f ? c.ior : (1.0f / c.ior);
        float w3 = (1.0f - c.metallic) * fresnel_dielectric(fabsf(wo.z), 1.0f / eta);
        float sum = w0 + w1 + w2 + w3;
        if (sum == 0.0f) {
            w[0] = w[1] = w[2] = w[3] = 0.0f;
            return;
        }
        w[0] = w0 / sum;
        w[1] = w1 / sum;
        w[2] = w2 / sum;
        w[3] = w3 / sum;
    }
    KS_D float pdf_diffuse_transmission(f3 wo, f3 wi) const
    {
        if (c.diffuse_trans_fwd > 0.05f)
            return hg_pdf(dot(wo, -wi), c.diffuse_trans_fwd);
        return -wi.z * kInvPi;
    }
    KS_D float pdf_metallic_specular(f3 wo, f3 wi) const
    {
        f3 wh = normalize(wo + wi);
        return mf().D(wh) * mf().G1(wo) / (4.0f * fabsf(wo.z));
    }
    KS_D float pdf_dielectric_specular(f3 wo, f3 wi) const
    {
        bool refl = wo.z * wi.z >= 0.0f;
        float eta = wo.z >= 0.0f ? c.ior : (1.0f / c.ior);
        f3 wh = refl ? normalize(wo + wi) : normalize(wo + wi * eta);
        if (wh.z < 0.0f)
            wh = -wh;
        float D = mf().D(wh);
        float G1 = mf().G1(wo);
        float awh = fabsf(dot(wo, wh));
        float Fr = fresnel_dielectric(fabsf(dot(wo, wh)), 1.0f / eta);
        float Fr_adj = dielectric_specular_adjust(awh);
        float Fr_refl = Fr * Fr_adj;
        float Fr_refr = (1.0f - Fr) * c.specular_trans;
        if (Fr_refr == 0.0f)
            Fr_refl = 1.0f;
        float pdf;
        if (refl) {
            pdf = D * G1 / (4.0f * fabsf(wo.z));
            pdf *= Fr_refl / (Fr_refl + Fr_refr);
        } else {
            float denom = sqr(dot(wo, wh) + eta * dot(wi, wh));
            float jac = eta * eta * fabsf(dot(wi, wh)) / denom;
            pdf = denom == 0.0f ? 0.0f : D * G1 * fabsf(dot(wo, wh)) / fabsf(wo.z) * jac;
            pdf *= Fr_refr / (Fr_refl + Fr_refr);
        }
        return pdf;
    }
    KS_BIG f3 eval(f3 wo, f3 wi) const
    {
        if (wo.z == 0.0f || wi.z == 0.0f)
            return mk(0, 0, 0);
        f3 f = mk(0, 0, 0);
        if (wo.z > 0.0f && wi.z > 0.0f) {
            f += eval_diffuse(wo, wi);
            f += eval_metallic_specular(wo, wi);
        }
        if (wo.z > 0.0f && wi.z < 0.0f)
            f += eval_diffuse_transmission(wo, wi);
        f += eval_dielectric_specular(wo, wi);
        return f;
    }
    KS_BIG float pdf(f3 wo, f3 wi) const
    {
        if (wo.z == 0.0f || wi.z == 0.0f)
            return 0.0f;
        float w[4];
        lobe_weights(wo, w);
        if (w[0] == 0.0f && w[1] == 0.0f && w[2] == 0.0f && w[3] == 0.0f)
            return 0.0f;
        float p[4] = {0, 0, 0, 0};
        if (wo.z > 0.0f && wi.z > 0.0f) {
            p[0] = wi.z * kInvPi;
            p[2] = pdf_metallic_specular(wo, wi);
        }
        if (wo.z > 0.0f && wi.z < 0.0f)
            p[1] = pdf_diffuse_transmission(wo, wi);
        p[3] = pdf_dielectric_specular(wo, wi);
        return p[0] * w[0] + p[1] * w[1] + p[2] * w[2] + p[3] * w[3];
    }
    KS_D void eval_and_pdf(f3 wo, f3 wi, f3 &f, float &p) const
    {
        f = eval(wo, wi);
        if (is_zero(f)) {
            p = 0.0f;
            return;
        }
        p = pdf(wo, wi);
    }
    KS_D f3 sample_metallic(f3 wo, float u0, float u1, float &pdf) const
    {
        if (wo.z == 0.0f) {
            pdf = 0.0f;
            return mk(0, 0, 0);
        }
        f3 wh = mf().sample(fsign(wo.z) * wo, u0, u1);
        f3 wi = reflect(wo, wh);
        if (wo.z * wi.z < 0.0f) {
            pdf = 0.0f;
            return mk(0, 0, 0);
        }
        pdf = mf().D(wh) * mf().G1(wo) / (4.0f * fabsf(wo.z));
        return wi;
    }
    KS_D f3 sample_dielectric(f3 wo, float u_lobe, float u0, float u1, float &pdf) const
    {
        if (wo.z == 0.0f) {
            pdf = 0.0f;
            return mk(0, 0, 0);
        }
        f3 wh = mf().sample(fsign(wo.z) * wo, u0, u1);
        float D = mf().D(wh);
        float G1 = mf().G1(wo);
        float eta = wo.z >= 0.0f ? c.ior : (1.0f / c.ior);
        float awh = fabsf(dot(wo, wh));
        float Fr = fresnel_dielectric(fabsf(dot(wo, wh)), 1.0f / eta);
        float Fr_adj = dielectric_specular_adjust(awh);
        float Fr_refl = Fr * Fr_adj;
        float Fr_refr = (1.0f - Fr) * c.specular_trans;
        if (Fr_refr == 0.0f)
            Fr_refl = 1.0f;
        f3 wi;
        if (u_lobe < Fr_refl / (Fr_refl + Fr_refr)) {
            wi = reflect(wo, wh);
            if (wo.z * wi.z < 0.0f) {
                pdf = 0.0f;
                return mk(0, 0, 0);
            }
            pdf = D * G1 / (4.0f * fabsf(wo.z));
            pdf *= Fr_refl / (Fr_refl + Fr_refr);
        } else {
            if (!refract(wo, fsign(wo.z) * wh, 1.0f / eta, wi)) {
                pdf = 0.0f;
                return mk(0, 0, 0);
            }
            if (wo.z * wi.z > 0.0f) {
                pdf = 0.0f;
                return mk(0, 0, 0);
            }
            float denom = sqr(dot(wo, wh) + eta * dot(wi, wh));
            if (denom == 0.0f) { // wi = -wo through ior 1: no density (the reference asserts, :668)
                pdf = 0.0f;
                return mk(0, 0, 0);
            }
            float jac = eta * eta * fabsf(dot(wi, wh)) / denom;
            pdf = D * G1 * fabsf(dot(wo, wh)) / fabsf(wo.z) * jac;
            pdf *= Fr_refr / (Fr_refl + Fr_refr);
        }
        return wi;
    }
    // sample(): returns f / pdf (principled_bsdf.cpp:326-393)
    KS_BIG f3 sample(f3 wo, f3 &wi, float u_lobe, float u0, float u1, float &pdf) const
    {
        if (wo.z == 0.0f) {
            pdf = 0.0f;
            return mk(0, 0, 0);
        }
        float w[4];
        lobe_weights(wo, w);
        if (w[0] == 0.0f && w[1] == 0.0f && w[2] == 0.0f && w[3] == 0.0f) {
            pdf = 0.0f;
            return mk(0, 0, 0);
        }
        // sample_small_distrib over the 4 lobe weights (rng.h:399-434)
        float sum_w = 0.0f;
        int last_positive = 0;
        for (int i = 0; i < 4; ++i) {
            sum_w += w[i];
            if (w[i] > 0.0f)
                last_positive = i;
        }
        float inv_sum = 1.0f / sum_w;
        float cdf = 0.0f, u_remap = 0.0f;
        int lobe = -1;
        for (int i = 0; i < 4; ++i) {
            float cdf_next = cdf + w[i] * inv_sum;
            if (u_lobe < cdf_next) {
                lobe = i;
                u_remap = (u_lobe - cdf) / (cdf_next - cdf);
                break;
            }
            cdf = cdf_next;
        }
        if (lobe == -1)
            lobe = last_positive;
        // only the direction is drawn in a per-lobe branch; the other lobes' densities come after
        // it, so that lanes of a warp that drew different lobes evaluate them together (the
        // densities and conditions of principled_bsdf.cpp:326-393; on the bench frame the shading
        // stage took 8 ms per frame less than with a branch per lobe that evaluated them inside)
        float ps = 0.0f; // density of the drawn lobe
        if (lobe == 0) {
            wi = sample_cosine_hemisphere(u0, u1);
            ps = wi.z * kInvPi;
        } else if (lobe == 1) {
            if (c.diffuse_trans_fwd > 0.05f) {
                wi = sample_hg(-wo, c.diffuse_trans_fwd, u0, u1, ps);
            } else {
                wi = sample_cosine_hemisphere(u0, u1);
                ps = wi.z * kInvPi;
                wi.z = -wi.z;
            }
        } else if (lobe == 2) {
            wi = sample_metallic(wo, u0, u1, ps);
        } else {
            wi = sample_dielectric(wo, u_remap, u0, u1, ps);
        }
        if (is_zero(wi) || ps == 0.0f) {
            pdf = 0.0f;
            return mk(0, 0, 0);
        }
        const bool up = wo.z > 0.0f && wi.z > 0.0f, down = wo.z > 0.0f && wi.z < 0.0f;
        const float pd = pdf_dielectric_specular(wo, wi);
        const float pm = up && lobe != 1 ? pdf_metallic_specular(wo, wi) : 0.0f;
        const float q0 = lobe == 0 ? ps : (lobe >= 2 && up ? wi.z * kInvPi : 0.0f);
        const float q1 = lobe == 1 ? ps : (lobe == 3 && down ? pdf_diffuse_transmission(wo, wi) : 0.0f);
        const float q2 = lobe == 2 ? ps : ((lobe == 0 || lobe == 3) ? pm : 0.0f);
        const float q3 = lobe == 3 ? ps : pd;
        pdf = q0 * w[0] + q1 * w[1] + q2 * w[2] + q3 * w[3];
        return eval(wo, wi) / pdf;
    }
};

using Principled = PrincipledT<GGXd>;

// sample_small_distrib (rng.h:399-432) over N weights; u_remap as the reference computes it.
template <int N>
KS_D int sample_small_distrib_n(const float *w, float u, float *u_remap)
{
    float sum_w = 0.0f;
    int last_positive = 0;
    for (int i = 0; i < N; ++i) {
        sum_w += w[i];
        if (w[i] > 0.0f)
            last_positive = i;
    }
    float inv_sum = 1.0f / sum_w;
    float cdf = 0.0f;
    for (int i = 0; i < N; ++i) {
        float cdf_next = cdf + w[i] * inv_sum;
        if (u < cdf_next) {
            if (u_remap)
                *u_remap = (u - cdf) / (cdf_next - cdf);
            return i;
        }
        cdf = cdf_next;
    }
    return last_positive;
}

// PrincipledBRDF::internal (principled_bsdf.cpp:61-225): Lambertian diffuse plus a microfacet
// specular lobe whose normal-incidence reflectance lerps from `specular` to the base colour with
// metallic; no transmission.
template <class MF>
struct PrincipledBrdfT
{
    Closure c;
    KS_D MF mf() const { return MF(c.ax, c.ay); }
    KS_D f3 eval_diffuse(f3, f3 wi) const
    {
        float lw = (1.0f - c.metallic);
        if (lw == 0.0f)
            return mk(0, 0, 0);
        return lw * c.basecolor * kInvPi * wi.z;
    }
    KS_D f3 eval_specular(f3 wo, f3 wi) const
    {
        f3 wh = normalize(wo + wi);
        float D = mf().D(wh);
        float G = mf().G2(wo, wi);
        // lerp(a, b, t) = (1 - t) a + t b (maths.h:681-690)
        f3 R0 = (1.0f - c.metallic) * mk(c.specular, c.specular, c.specular) + c.metallic * c.basecolor;
        float fs = fresnel_schlick(dot(wo, wh));
        f3 Fr = (1.0f - fs) * R0 + fs * mk(1.0f, 1.0f, 1.0f);
        return D * G * Fr / (4.0f * wo.z);
    }
    KS_D void lobe_weights(f3 wo, float w[2]) const
    {
        float lum = luminance(c.basecolor);
        float lum_R0 = std_lerp(c.specular, lum, c.metallic);
        float wd = wo.z > 0.0f ? (1.0f - c.metallic) * lum * kInvPi : 0.0f;
        float ws = wo.z > 0.0f ? std_lerp(lum_R0, 1.0f, fresnel_schlick(wo.z)) : 0.0f;
        float sum = wd + ws;
        if (sum == 0.0f) {
            w[0] = w[1] = 0.0f;
            return;
        }
        float inv_sum = 1.0f / sum;
        w[0] = wd * inv_sum;
        w[1] = ws * inv_sum;
    }
    KS_D float pdf_specular(f3 wo, f3 wi) const
    {
        f3 wh = normalize(wo + wi);
        return mf().D(wh) * mf().G1(wo) / (4.0f * fabsf(wo.z));
    }
    KS_BIG f3 eval(f3 wo, f3 wi) const
    {
        if (wo.z == 0.0f || wi.z == 0.0f)
            return mk(0, 0, 0);
        f3 f = mk(0, 0, 0);
        if (wo.z > 0.0f && wi.z > 0.0f) {
            f += eval_diffuse(wo, wi);
            f += eval_specular(wo, wi);
        }
        return f;
    }
    KS_BIG float pdf(f3 wo, f3 wi) const
    {
        if (wo.z == 0.0f || wi.z == 0.0f)
            return 0.0f;
        float w[2];
        lobe_weights(wo, w);
        if (w[0] == 0.0f && w[1] == 0.0f)
            return 0.0f;
        if (wo.z <= 0.0f || wi.z <= 0.0f)
            return 0.0f;
        return (wi.z * kInvPi) * w[0] + pdf_specular(wo, wi) * w[1];
    }
    KS_D void eval_and_pdf(f3 wo, f3 wi, f3 &f, float &p) const
    {
        f = eval(wo, wi);
        p = is_zero(f) ? 0.0f : pdf(wo, wi);
    }
    KS_BIG f3 sample(f3 wo, f3 &wi, float u_lobe, float u0, float u1, float &pdf) const
    {
        if (wo.z == 0.0f) {
            pdf = 0.0f;
            return mk(0, 0, 0);
        }
        float w[2];
        lobe_weights(wo, w);
        if (w[0] == 0.0f && w[1] == 0.0f) {
            pdf = 0.0f;
            return mk(0, 0, 0);
        }
        const int lobe = sample_small_distrib_n<2>(w, u_lobe, nullptr);
        float p[2] = {0.0f, 0.0f};
        if (lobe == 0) {
            wi = sample_cosine_hemisphere(u0, u1);
            p[0] = wi.z * kInvPi;
            if (is_zero(wi) || p[0] == 0.0f) {
                pdf = 0.0f;
                return mk(0, 0, 0);
            }
            if (wo.z > 0.0f && wi.z > 0.0f)
                p[1] = pdf_specular(wo, wi);
        } else {
            // sample_specular (principled_bsdf.cpp:176-196)
            f3 wh = mf().sample(fsign(wo.z) * wo, u0, u1);
            wi = reflect(wo, wh);
            if (wo.z * wi.z < 0.0f)
                wi = mk(0, 0, 0);
            if (is_zero(wi)) {
                pdf = 0.0f;
                return mk(0, 0, 0);
            }
            p[1] = mf().D(wh) * mf().G1(wo) / (4.0f * fabsf(wo.z));
            if (wo.z > 0.0f && wi.z > 0.0f)
                p[0] = wi.z * kInvPi;
        }
        pdf = p[0] * w[0] + p[1] * w[1];
        return eval(wo, wi) / pdf;
    }
};

// Lambertian (bsdf.cpp:13-41) with the clamped base colour as albedo.
struct LambertianD
{
    Closure c;
    KS_D void eval_and_pdf(f3 wo, f3 wi, f3 &f, float &p) const
    {
        if (wo.z <= 0.0f || wi.z <= 0.0f) {
            f = mk(0, 0, 0);
            p = 0.0f;
            return;
        }
        f = kInvPi * c.basecolor * wi.z;
        p = wi.z * kInvPi;
    }
    KS_D f3 sample(f3 wo, f3 &wi, float, float u0, float u1, float &pdf) const
    {
        if (wo.z <= 0.0f) {
            pdf = 0.0f;
            return mk(0, 0, 0);
        }
        wi = sample_cosine_hemisphere(u0, u1);
        pdf = wi.z * kInvPi;
        return c.basecolor;
    }
};

// LambertianSubsurfaceExitAdapter (subsurface.cpp:502-532): the cosine lobe at a random walk's exit
// point, scaled by eta^2 (undoing the 1 / eta^2 of the entry); it reads wi only.
KS_D Closure subsurface_exit_closure(float eta)
{
    Closure c{};
    c.kind = kBsdfSubsurfaceExit;
    c.basecolor = mk(eta * eta, eta * eta, eta * eta);
    return c;
}

struct SubsurfaceExitD
{
    Closure c;
    KS_D void eval_and_pdf(f3, f3 wi, f3 &f, float &p) const
    {
        if (wi.z <= 0.0f) {
            f = mk(0, 0, 0);
            p = 0.0f;
            return;
        }
        f = (kInvPi * wi.z) * c.basecolor;
        p = wi.z * kInvPi;
    }
    KS_D f3 sample(f3, f3 &wi, float, float u0, float u1, float &pdf) const
    {
        wi = sample_cosine_hemisphere(u0, u1);
        pdf = wi.z * kInvPi;
        return c.basecolor;
    }
};

// Any BSDF of a material (the Material::bsdf pointer of material.h:39, dispatched on the kind).
// Its two entry points stay out of line: the general shading kernel then calls one function per
// use instead of holding five inlined variants' live state around each call.
struct AnyBsdf
{
    Closure c;
    KS_BIG void eval_and_pdf(f3 wo, f3 wi, f3 &f, float &p) const
    {
        switch (c.kind) {
        case kBsdfPrincipledGGX:
            PrincipledT<GGXd>{c}.eval_and_pdf(wo, wi, f, p);
            break;
        case kBsdfPrincipledBeckmann:
            PrincipledT<Beckmannd>{c}.eval_and_pdf(wo, wi, f, p);
            break;
        case kBrdfPrincipledGGX:
            PrincipledBrdfT<GGXd>{c}.eval_and_pdf(wo, wi, f, p);
            break;
        case kBrdfPrincipledBeckmann:
            PrincipledBrdfT<Beckmannd>{c}.eval_and_pdf(wo, wi, f, p);
            break;
        case kBsdfSubsurfaceExit:
            SubsurfaceExitD{c}.eval_and_pdf(wo, wi, f, p);
            break;
        default:
            LambertianD{c}.eval_and_pdf(wo, wi, f, p);
            break;
        }
    }
    KS_BIG f3 sample(f3 wo, f3 &wi, float u_lobe, float u0, float u1, float &pdf) const
    {
        switch (c.kind) {
        case kBsdfPrincipledGGX:
            return PrincipledT<GGXd>{c}.sample(wo, wi, u_lobe, u0, u1, pdf);
        case kBsdfPrincipledBeckmann:
            return PrincipledT<Beckmannd>{c}.sample(wo, wi, u_lobe, u0, u1, pdf);
        case kBrdfPrincipledGGX:
            return PrincipledBrdfT<GGXd>{c}.sample(wo, wi, u_lobe, u0, u1, pdf);
        case kBrdfPrincipledBeckmann:
            return PrincipledBrdfT<Beckmannd>{c}.sample(wo, wi, u_lobe, u0, u1, pdf);
        case kBsdfSubsurfaceExit:
            return SubsurfaceExitD{c}.sample(wo, wi, u_lobe, u0, u1, pdf);
        default:
            return LambertianD{c}.sample(wo, wi, u_lobe, u0, u1, pdf);
        }
    }
};

} // namespace ksb
