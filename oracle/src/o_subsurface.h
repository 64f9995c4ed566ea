// ORACLE (test infrastructure only).  Restatement of keepsake's subsurface scattering on the CPU:
// the per-sample RNG of PTRenderSampler (sobol.h:237-244; RNG, rng.h:19-106; hash, hash.h:140-252)
// and subsurface_random_walk with its helpers (subsurface.cpp:12-500), drawn from one stream per
// sample along the whole path, as the reference draws it.
#pragma once
#include "o_bsdf.h"
#include "o_math.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle
{

struct Pcg32
{
    uint64_t state = 0x853c49e6748fea9bull, inc = 0xda3e39cb94b95bdbull;
    static constexpr uint64_t kMult = 0x5851f42d4c957f2dull;
    uint32_t next_u32()
    {
        uint64_t old = state;
        state = old * kMult + inc;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((~rot + 1u) & 31));
    }
    float next() { return std::min<float>(std::nextafter(1.0f, 0.0f), next_u32() * 0x1p-32f); }
    void set_seq(uint64_t seq, uint64_t offset)
    {
        state = 0u;
        inc = (seq << 1u) | 1u;
        next_u32();
        state += offset;
        next_u32();
    }
    void advance(int64_t idelta)
    {
        uint64_t cur_mult = kMult, cur_plus = inc, acc_mult = 1u, acc_plus = 0u, delta = (uint64_t)idelta;
        while (delta > 0) {
            if (delta & 1) {
                acc_mult *= cur_mult;
                acc_plus = acc_plus * cur_mult + cur_plus;
            }
            cur_plus = (cur_mult + 1) * cur_plus;
            cur_mult *= cur_mult;
            delta /= 2;
        }
        state = acc_mult * state + acc_plus;
    }
};

inline uint64_t murmur64a(const unsigned char *key, size_t len, uint64_t seed)
{
    const uint64_t m = 0xc6a4a7935bd1e995ull;
    const int r = 47;
    uint64_t h = seed ^ (len * m);
    const unsigned char *end = key + 8 * (len / 8);
    while (key != end) {
        uint64_t k;
        std::memcpy(&k, key, 8);
        key += 8;
        k *= m;
        k ^= k >> r;
        k *= m;
        h ^= k;
        h *= m;
    }
    const size_t rem = len & 7;
    if (rem) {
        for (size_t i = rem; i-- > 0;)
            h ^= uint64_t(key[i]) << (8 * i);
        h *= m;
    }
    h ^= h >> r;
    h *= m;
    h ^= h >> r;
    return h;
}

inline uint64_t mix_bits_u64(uint64_t v)
{
    v ^= (v >> 31);
    v *= 0x7fb5d329728ea185ull;
    v ^= (v >> 27);
    v *= 0x81dadef4bc2dd44dull;
    v ^= (v >> 33);
    return v;
}

// PTRenderSampler's rng: RNG(hash(pixel, seed)) advanced by sample_index * 65536
inline Pcg32 sample_rng(uint32_t px, uint32_t py, uint32_t seed, uint64_t sample_index)
{
    unsigned char buf[12];
    std::memcpy(buf, &px, 4);
    std::memcpy(buf + 4, &py, 4);
    std::memcpy(buf + 8, &seed, 4);
    const uint64_t seq = murmur64a(buf, 12, 0);
    Pcg32 r;
    r.set_seq(seq, mix_bits_u64(seq));
    r.advance((int64_t)(sample_index * 65536ull));
    return r;
}

inline float ss_rd(float ap, float fa)
{
    float s = std::sqrt(3.0f * (1.0f - ap));
    return 0.5f * ap * (1.0f + std::exp(-fa * s)) * std::exp(-s);
}

inline float ss_alpha_prime(float rd, float fa)
{
    if (rd < 1e-4f)
        return 0.0f;
    if (rd >= 0.995f)
        return 0.999999f;
    float x0 = 0.0f, x1 = 1.0f, xmid = 0.0f;
    for (int i = 0; i < 12; ++i) {
        xmid = 0.5f * (x0 + x1);
        if (ss_rd(xmid, fa) < rd)
            x0 = xmid;
        else
            x1 = xmid;
    }
    return xmid;
}

inline void ss_remap(float albedo, float d, float g, float &sigma_t, float &alpha)
{
    const float g2 = g * g, g3 = g2 * g, g4 = g3 * g, g5 = g4 * g, g6 = g5 * g, g7 = g6 * g;
    const float A = 1.8260523782f + -1.28451056436f * g + -1.79904629312f * g2 + 9.19393289202f * g3 +
                    -22.8215585862f * g4 + 32.0234874259f * g5 + -23.6264803333f * g6 + 7.21067002658f * g7;
    const float B = 4.98511194385f + 0.127355959438f * std::exp(31.1491581433f * g + -201.847017512f * g2 +
                                                                841.576016723f * g3 + -2018.09288505f * g4 +
                                                                2731.71560286f * g5 + -1935.41424244f * g6 +
                                                                559.009054474f * g7);
    const float C = 1.09686102424f + -0.394704063468f * g + 1.05258115941f * g2 + -8.83963712726f * g3 +
                    28.8643230661f * g4 + -46.8802913581f * g5 + 38.5402837518f * g6 + -12.7181042538f * g7;
    const float D = 0.496310210422f + 0.360146581622f * g + -2.15139309747f * g2 + 17.8896899217f * g3 +
                    -55.2984010333f * g4 + 82.065982243f * g5 + -58.5106008578f * g6 + 15.8478295021f * g7;
    const float E = 4.23190299701f + 0.00310603949088f * std::exp(76.7316253952f * g + -594.356773233f * g2 +
                                                                  2448.8834203f * g3 + -5576.68528998f * g4 +
                                                                  7116.60171912f * g5 + -4763.54467887f * g6 +
                                                                  1303.5318055f * g7);
    const float F = 2.40602999408f + -2.51814844609f * g + 9.18494908356f * g2 + -79.2191708682f * g3 +
                    259.082868209f * g4 + -403.613804597f * g5 + 302.85712436f * g6 + -87.4370473567f * g7;
    const float blend = std::pow(albedo, 0.25f);
    alpha = (1.0f - blend) * A * std::pow(std::atan(B * albedo), C) + blend * D * std::pow(std::atan(E * albedo), F);
    alpha = std::clamp(alpha, 0.0f, 0.999999f);
    sigma_t = (1.0f / std::max(d, 1e-16f)) / (1.0f - g);
}

inline V3 cwise_div(V3 a, V3 b) { return V3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline V3 cwise_exp(V3 a) { return V3(std::exp(a.x), std::exp(a.y), std::exp(a.z)); }

// The walk (subsurface_random_walk with D = 0, subsurface.cpp:222-500).  cast(o, d, tmax, tri, t, b1,
// b2) is LocalGeometry::intersect1 (the entry mesh only).
template <class Cast>
bool ss_walk(V3 albedo, V3 radius, float g0, float ior, float rfr_prob, V3 P, V3 N, V3 Ng, Pcg32 &rng,
             const Cast &cast, V3 &throughput, uint32_t &exit_tri, float &exit_t, float &exit_b1, float &exit_b2,
             V3 &wi)
{
    {
        const float eta = ior, inv_eta = 1.0f / eta;
        const float F_dr = inv_eta * (-1.440f * inv_eta + 0.710f) + 0.668f + 0.0636f * eta;
        const float fa = (4.0f / 3.0f) * (1.0f + F_dr) / (1.0f - F_dr);
        for (int c = 0; c < 3; ++c)
            radius[c] *= std::sqrt(3.0f * (1.0f - ss_alpha_prime(albedo[c], fa)));
    }
    if (rng.next() < rfr_prob)
        return false; // wo = -D = 0: the refractive entry ends the walk (subsurface.cpp:241-246)
    float e0 = rng.next(), e1 = rng.next();
    V3 D;
    {
        // sample_cosine_hemisphere(u, -N) (rng.h:269-282)
        V3 n = -N;
        float a = 1.0f - 2.0f * e0;
        float b = safe_sqrt(1.0f - a * a);
        a *= 0.999f;
        b *= 0.999f;
        float phi = two_pi * e1;
        D = normalized(V3(n.x + b * std::cos(phi), n.y + b * std::sin(phi), n.z + a));
    }
    if (-dot(Ng, D) <= 0.0f)
        return false;
    V3 ro = offset_ray(P, dot(D, Ng) > 0.0f ? Ng : -Ng), rd = D;
    float tmax = inf;
    V3 sigma_t, alpha;
    for (int c = 0; c < 3; ++c)
        ss_remap(albedo[c], radius[c], g0, sigma_t[c], alpha[c]);
    for (int c = 0; c < 3; ++c)
        if (alpha[c] < 0.2f) {
            throughput[c] *= alpha[c] / 0.2f;
            alpha[c] = 0.2f;
        }
    const V3 sigma_s = sigma_t * alpha;
    const float amax = std::max(alpha.x, std::max(alpha.y, alpha.z));
    const float dl = 1.0f / std::sqrt(1.0f - std::pow(amax, 2.44294f - 0.0215813f * amax + 0.578637f / amax));
    if (dl == 1.0f)
        return false;
    const float phase_log = std::log((dl + 1.0f) / (dl - 1.0f));
    bool hit = false, have_opposite = false;
    float opposite_distance = 0.0f;
    const float guided_fraction_org = 1.0f - std::max(0.5f, std::pow(std::abs(g0), 0.125f));
    const V3 sigma_s_star = sigma_s * (1.0f - g0);
    const V3 sigma_t_star = sigma_t - sigma_s + sigma_s_star;
    for (int bounce = 0; bounce < 256; ++bounce) {
        const bool late = bounce > 9;
        const float g = late ? 0.0f : g0;
        const float guided_fraction = late ? 0.75f : guided_fraction_org;
        const V3 st = late ? sigma_t_star : sigma_t, ss = late ? sigma_s_star : sigma_s;
        // volume_sample_channel
        const float rphase = rng.next();
        V3 w(std::abs(throughput.x * alpha.x), std::abs(throughput.y * alpha.y), std::abs(throughput.z * alpha.z));
        const float wsum = w.x + w.y + w.z;
        const V3 channel_pdf = wsum > 0.0f ? w / wsum : V3(1.0f / 3.0f, 1.0f / 3.0f, 1.0f / 3.0f);
        int channel = 2;
        float acc = 0.0f;
        for (int c = 0; c < 3; ++c) {
            acc += channel_pdf[c];
            if (rphase < acc) {
                channel = c;
                break;
            }
        }
        float sample_sigma_t = st[channel];
        const float randt = rng.next();
        float backward_fraction = 0.0f, fwd_factor = 0.0f, fwd_stretch = 1.0f, back_factor = 0.0f, back_stretch = 1.0f;
        if (bounce > 0) {
            const bool guided = rng.next() < guided_fraction;
            bool guide_backward = false;
            if (have_opposite) {
                const float x = std::clamp(dot(ro - P, -N), 0.0f, opposite_distance);
                backward_fraction = 1.0f / (1.0f + std::exp((opposite_distance - 2.0f * x) / dl));
                guide_backward = rng.next() < backward_fraction;
            }
            const float r0 = rng.next(), r1 = rng.next();
            float cos_theta, hgp;
            if (guided) {
                cos_theta = dl - (dl + 1.0f) * std::exp(-r0 * phase_log);
                if (guide_backward)
                    cos_theta = -cos_theta;
                // direction_from_cosine
                const float sin_theta = safe_sqrt(1.0f - cos_theta * cos_theta);
                const float phi = two_pi * r1;
                V3 T, B;
                orthonormal_basis(N, T, B);
                const V3 nd = (sin_theta * std::cos(phi)) * T + (sin_theta * std::sin(phi)) * B + cos_theta * N;
                hgp = single_peaked_henyey_greenstein(dot(rd, nd), g);
                rd = nd;
            } else {
                const V3 nd = sample_henyey_greenstein(rd, g, r0, r1, &hgp);
                cos_theta = dot(nd, N);
                rd = nd;
            }
            fwd_factor = (1.0f / two_pi) * (1.0f / ((dl - cos_theta) * phase_log)) / hgp;
            back_factor = (1.0f / two_pi) * (1.0f / ((dl + cos_theta) * phase_log)) / hgp;
            fwd_stretch = 1.0f - cos_theta / dl;
            back_stretch = 1.0f + cos_theta / dl;
            if (guided)
                sample_sigma_t *= guide_backward ? back_stretch : fwd_stretch;
        }
        float t = -std::log(1.0f - randt) / sample_sigma_t;
        tmax = bounce == 0 ? std::max(t, 10.0f / std::min(sigma_t.x, std::min(sigma_t.y, sigma_t.z))) : t;
        uint32_t tri;
        float th, b1, b2;
        hit = cast(ro, rd, tmax, tri, th, b1, b2);
        if (hit) {
            tmax = th;
            exit_tri = tri;
            exit_t = th;
            exit_b1 = b1;
            exit_b2 = b2;
        }
        if (bounce == 0) {
            if (hit) {
                have_opposite = true;
                opposite_distance = dot(ro + tmax * rd - P, -N);
            }
            hit = tmax < t;
        }
        if (hit)
            t = tmax;
        ro += t * rd;
        const V3 transmittance = cwise_exp(-t * st);
        V3 pdf = hit ? transmittance : st * transmittance;
        if (bounce > 0) {
            const V3 tf = cwise_exp(-t * (fwd_stretch * st));
            V3 guided_pdf = hit ? tf : (fwd_stretch * st) * tf;
            if (have_opposite) {
                const V3 tb = cwise_exp(-t * (back_stretch * st));
                const V3 back_pdf = hit ? tb : (back_stretch * st) * tb;
                guided_pdf = (1.0f - backward_fraction) * (guided_pdf * fwd_factor) +
                             backward_fraction * (back_pdf * back_factor);
            } else {
                guided_pdf = guided_pdf * fwd_factor;
            }
            pdf = (1.0f - guided_fraction) * pdf + guided_fraction * guided_pdf;
        }
        const V3 num = hit ? transmittance : ss * transmittance;
        const V3 cp = channel_pdf * pdf;
        throughput = throughput * (num / (cp.x + cp.y + cp.z));
        if (hit)
            break;
        if (std::max(throughput.x, std::max(throughput.y, throughput.z)) < 1e-6f)
            break;
    }
    wi = rd;
    return hit;
}

} // namespace oracle
