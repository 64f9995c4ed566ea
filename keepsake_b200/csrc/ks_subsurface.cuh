// Subsurface scattering of keepsake's BSSRDF (subsurface.cpp: a random walk inside the mesh after
// Blender Cycles' random-walk subsurface, with Dwivedi guiding, channel sampling and the similarity
// relation past the ninth bounce), the PCG32 stream the walk draws from (RNG, rng.h:19-106), and the
// Lambertian exit lobe (LambertianSubsurfaceExitAdapter, subsurface.cpp:502-532).  The published
// fits of Chiang, Kutz and Burley (the albedo-to-single-scattering-albedo remap) and of d'Eon and
// Krivanek (the Dwivedi diffusion length) are restated as the reference writes them.
#pragma once
#include "ks_math.cuh"
#include "ks_sampler.cuh"
#include "ks_wavefront.cuh"

namespace ksb
{

constexpr float kBeforeOneF = 0x1.fffffep-1f; // fp32_before_one

// PCG32 (rng.h:19-106): set_seq, next_u32, next (clamped below 1), advance.
struct Pcg32
{
    uint64_t state = 0, inc = 1;
    static constexpr uint64_t kMult = 0x5851f42d4c957f2dull;
    KS_HD uint32_t next_u32()
    {
        const uint64_t old = state;
        state = old * kMult + inc;
        const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((~rot + 1u) & 31));
    }
    KS_HD float next()
    {
        const float f = (float)next_u32() * 0x1p-32f;
        return f < kBeforeOneF ? f : kBeforeOneF;
    }
    KS_HD void set_seq(uint64_t seq, uint64_t offset)
    {
        state = 0u;
        inc = (seq << 1u) | 1u;
        next_u32();
        state += offset;
        next_u32();
    }
    KS_HD void advance(uint64_t delta)
    {
        uint64_t cur_mult = kMult, cur_plus = inc, acc_mult = 1u, acc_plus = 0u;
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

// hash(pixel, seed) (hash.h:243-252): murmur_hash_64A of the 12 bytes (x, y, seed), seed 0.
KS_HD uint64_t hash_pixel_seed(uint32_t x, uint32_t y, uint32_t seed)
{
    const uint64_t m = 0xc6a4a7935bd1e995ull;
    uint64_t h = 12ull * m;
    uint64_t k = (uint64_t)x | ((uint64_t)y << 32);
    k *= m;
    k ^= k >> 47;
    k *= m;
    h ^= k;
    h *= m;
    h ^= (uint64_t)seed; // the 4-byte tail
    h *= m;
    h ^= h >> 47;
    h *= m;
    h ^= h >> 47;
    return h;
}

// The per-sample stream of PTRenderSampler (sobol.h:237-244): RNG(hash(pixel, seed)) advanced by
// sample_index x 65536.  The wavefront draws each walk from its own stretch of that stream (4096
// values per bounce, more than a walk of 256 steps takes), so a walk needs no state from earlier
// vertices of its path; the reference continues one stream along the path.
KS_HD Pcg32 subsurface_stream(uint32_t px, uint32_t py, uint32_t seed, uint64_t sample_index, uint32_t bounce)
{
    const uint64_t seq = hash_pixel_seed(px, py, seed);
    Pcg32 r;
    r.set_seq(seq, mix_bits64(seq));
    r.advance(sample_index * 65536ull + (uint64_t)bounce * 4096ull);
    return r;
}

struct SsProfile
{
    f3 albedo, radius;
    float g, ior, rfr_entry_prob;
};

// bssrdf_dipole_compute_Rd / _alpha_prime (subsurface.cpp:146-183)
KS_D float ss_dipole_rd(float ap, float fourthird_a)
{
    const float s = sqrtf(3.0f * (1.0f - ap));
    return 0.5f * ap * (1.0f + expf(-fourthird_a * s)) * expf(-s);
}

KS_D float ss_alpha_prime(float rd, float fourthird_a)
{
    if (rd < 1e-4f)
        return 0.0f;
    if (rd >= 0.995f)
        return 0.999999f;
    float x0 = 0.0f, x1 = 1.0f, xmid = 0.0f;
    for (int i = 0; i < 12; ++i) {
        xmid = 0.5f * (x0 + x1);
        if (ss_dipole_rd(xmid, fourthird_a) < rd)
            x0 = xmid;
        else
            x1 = xmid;
    }
    return xmid;
}

// subsurface_random_walk_remap (subsurface.cpp:44-80)
KS_D void ss_remap(float albedo, float d, float g, float &sigma_t, float &alpha)
{
    const float g2 = g * g, g3 = g2 * g, g4 = g3 * g, g5 = g4 * g, g6 = g5 * g, g7 = g6 * g;
    const float A = 1.8260523782f + -1.28451056436f * g + -1.79904629312f * g2 + 9.19393289202f * g3 +
                    -22.8215585862f * g4 + 32.0234874259f * g5 + -23.6264803333f * g6 + 7.21067002658f * g7;
    const float B = 4.98511194385f + 0.127355959438f * expf(31.1491581433f * g + -201.847017512f * g2 +
                                                           841.576016723f * g3 + -2018.09288505f * g4 +
                                                           2731.71560286f * g5 + -1935.41424244f * g6 +
                                                           559.009054474f * g7);
    const float C = 1.09686102424f + -0.394704063468f * g + 1.05258115941f * g2 + -8.83963712726f * g3 +
                    28.8643230661f * g4 + -46.8802913581f * g5 + 38.5402837518f * g6 + -12.7181042538f * g7;
    const float D = 0.496310210422f + 0.360146581622f * g + -2.15139309747f * g2 + 17.8896899217f * g3 +
                    -55.2984010333f * g4 + 82.065982243f * g5 + -58.5106008578f * g6 + 15.8478295021f * g7;
    const float E = 4.23190299701f + 0.00310603949088f * expf(76.7316253952f * g + -594.356773233f * g2 +
                                                             2448.8834203f * g3 + -5576.68528998f * g4 +
                                                             7116.60171912f * g5 + -4763.54467887f * g6 +
                                                             1303.5318055f * g7);
    const float F = 2.40602999408f + -2.51814844609f * g + 9.18494908356f * g2 + -79.2191708682f * g3 +
                    259.082868209f * g4 + -403.613804597f * g5 + 302.85712436f * g6 + -87.4370473567f * g7;
    const float blend = powf(albedo, 0.25f);
    alpha = (1.0f - blend) * A * powf(atanf(B * albedo), C) + blend * D * powf(atanf(E * albedo), F);
    alpha = fminf(fmaxf(alpha, 0.0f), 0.999999f);
    sigma_t = (1.0f / fmaxf(d, 1e-16f)) / (1.0f - g);
}

KS_D float f3_get(f3 v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }
KS_D f3 f3_exp(f3 v) { return mk(expf(v.x), expf(v.y), expf(v.z)); }
KS_D f3 f3_lerp(f3 a, f3 b, float t) { return (1.0f - t) * a + t * b; }
KS_D float f3_sum(f3 v) { return v.x + v.y + v.z; }

// sample_cosine_hemisphere(u, n) (rng.h:269-282): about the direction n
KS_D f3 cosine_about(float u0, float u1, f3 n)
{
    float a = 1.0f - 2.0f * u0;
    float b = sqrtf(fmaxf(1.0f - a * a, 0.0f));
    a *= 0.999f;
    b *= 0.999f;
    const float phi = 6.28318530718f * u1;
    return normalize(mk(n.x + b * cosf(phi), n.y + b * sinf(phi), n.z + a));
}

// orthonormal_basis (maths.h:814-821): T, B of a unit N
KS_D void basis(f3 N, f3 &T, f3 &B)
{
    const float sign = copysignf(1.0f, N.z);
    const float a = -1.0f / (sign + N.z);
    const float b = N.x * N.y * a;
    T = mk(1.0f + sign * N.x * N.x * a, sign * b, -sign * N.x);
    B = mk(b, sign + N.y * N.y * a, -N.y);
}

// sample_henyey_greenstein (bsdf.cpp:64-92); its density is hg_pdf (single_peaked_henyey_greenstein,
// ks_bsdf.cuh)
KS_D f3 hg_sample(f3 D, float g, float ru, float rv, float &pdf)
{
    float cos_theta;
    if (fabsf(g) < 1e-3f) {
        cos_theta = 1.0f - 2.0f * ru;
        pdf = 0.31830988618f * 0.25f;
    } else {
        const float k = (1.0f - g * g) / (1.0f - g + 2.0f * g * ru);
        cos_theta = (1.0f + g * g - k * k) / (2.0f * g);
        pdf = hg_pdf(cos_theta, g);
    }
    const float sin_theta = sqrtf(fmaxf(1.0f - cos_theta * cos_theta, 0.0f));
    const float phi = 6.28318530718f * rv;
    f3 T, B;
    basis(D, T, B);
    return (sin_theta * cosf(phi)) * T + (sin_theta * sinf(phi)) * B + cos_theta * D;
}

// direction_from_cosine (subsurface.cpp:128-137)
KS_D f3 from_cosine(f3 D, float cos_theta, float rv)
{
    const float sin_theta = sqrtf(fmaxf(1.0f - cos_theta * cos_theta, 0.0f));
    const float phi = 6.28318530718f * rv;
    f3 T, B;
    basis(D, T, B);
    return (sin_theta * cosf(phi)) * T + (sin_theta * sinf(phi)) * B + cos_theta * D;
}

struct WalkExit
{
    uint32_t slot; // primitive slot of the exit triangle
    float t, b1, b2;
};

// subsurface_random_walk (subsurface.cpp:222-500) from an entry point P with shading normal N and
// geometric normal Ng (the hit frame's).  cast(o, d, tmax, exit) is the mesh-local closest-hit
// query (LocalGeometry::intersect1: only the entry mesh's triangles).  The walk starts with D = 0,
// as BSSRDF::sample calls it (material.cpp:136-140): the refractive entry then reads a zero wo and
// ends the walk (with probability rfr_entry_prob), else the entry direction is cosine-distributed
// about -N.  On success the exit, the last direction (wi) and the throughput are returned.
template <class Cast>
KS_D bool subsurface_walk(SsProfile prof, f3 P, f3 N, f3 Ng, Pcg32 &rng, const Cast &cast, f3 &throughput,
                          WalkExit &exit, f3 &wi)
{
    // bssrdf_setup_radius (subsurface.cpp:202-216)
    {
        const float eta = prof.ior, inv_eta = 1.0f / eta;
        const float F_dr = inv_eta * (-1.440f * inv_eta + 0.710f) + 0.668f + 0.0636f * eta;
        const float fourthird_a = (4.0f / 3.0f) * (1.0f + F_dr) / (1.0f - F_dr);
        const f3 ap = mk(ss_alpha_prime(prof.albedo.x, fourthird_a), ss_alpha_prime(prof.albedo.y, fourthird_a),
                         ss_alpha_prime(prof.albedo.z, fourthird_a));
        prof.radius = mk(prof.radius.x * sqrtf(3.0f * (1.0f - ap.x)), prof.radius.y * sqrtf(3.0f * (1.0f - ap.y)),
                         prof.radius.z * sqrtf(3.0f * (1.0f - ap.z)));
    }
    // the entry direction
    if (rng.next() < prof.rfr_entry_prob)
        return false; // wo = -D = 0: its local z is 0 (subsurface.cpp:241-246)
    const float e0 = rng.next(), e1 = rng.next();
    f3 D = cosine_about(e0, e1, -N);
    if (-dot(Ng, D) <= 0.0f)
        return false;
    RayQuery ray;
    ray.o = wave::spawn_origin(P, D, Ng);
    ray.d = D;
    ray.tmin = 0.0f;
    ray.tmax = kInf;
    // subsurface_random_walk_coefficients (subsurface.cpp:82-106)
    float st[3], al[3];
    for (int c = 0; c < 3; ++c)
        ss_remap(f3_get(prof.albedo, c), f3_get(prof.radius, c), prof.g, st[c], al[c]);
    f3 sigma_t = mk(st[0], st[1], st[2]), alpha = mk(al[0], al[1], al[2]);
    const float min_alpha = 0.2f;
    if (alpha.x < min_alpha) {
        throughput.x *= alpha.x / min_alpha;
        alpha.x = min_alpha;
    }
    if (alpha.y < min_alpha) {
        throughput.y *= alpha.y / min_alpha;
        alpha.y = min_alpha;
    }
    if (alpha.z < min_alpha) {
        throughput.z *= alpha.z / min_alpha;
        alpha.z = min_alpha;
    }
    const f3 sigma_s = mk(sigma_t.x * alpha.x, sigma_t.y * alpha.y, sigma_t.z * alpha.z);
    // diffusion_length_dwivedi (subsurface.cpp:121-125) of the largest alpha
    const float amax = fmaxf(alpha.x, fmaxf(alpha.y, alpha.z));
    const float diffusion_length = 1.0f / sqrtf(1.0f - powf(amax, 2.44294f - 0.0215813f * amax + 0.578637f / amax));
    if (diffusion_length == 1.0f)
        return false;
    const float phase_log = logf((diffusion_length + 1.0f) / (diffusion_length - 1.0f));
    bool hit = false, have_opposite = false;
    float opposite_distance = 0.0f;
    const float guided_fraction_org = 1.0f - fmaxf(0.5f, powf(fabsf(prof.g), 0.125f));
    // the similarity relation past bounce 9 (SUBSURFACE_RANDOM_WALK_SIMILARITY_LEVEL)
    const f3 sigma_s_star = sigma_s * (1.0f - prof.g);
    const f3 sigma_t_star = sigma_t - sigma_s + sigma_s_star;
    for (int bounce = 0; bounce < 256; ++bounce) {
        const bool late = bounce > 9;
        const float g = late ? 0.0f : prof.g;
        const float guided_fraction = late ? 0.75f : guided_fraction_org;
        const f3 s_t = late ? sigma_t_star : sigma_t;
        const f3 s_s = late ? sigma_s_star : sigma_s;
        // volume_sample_channel (subsurface.cpp:17-42)
        const float rphase = rng.next();
        f3 w = mk(fabsf(throughput.x * alpha.x), fabsf(throughput.y * alpha.y), fabsf(throughput.z * alpha.z));
        const float wsum = f3_sum(w);
        const f3 channel_pdf = wsum > 0.0f ? w / wsum : mk(1.0f / 3.0f, 1.0f / 3.0f, 1.0f / 3.0f);
        int channel = 2;
        {
            float acc = 0.0f;
            for (int c = 0; c < 3; ++c) {
                acc += f3_get(channel_pdf, c);
                if (rphase < acc) {
                    channel = c;
                    break;
                }
            }
        }
        float sample_sigma_t = f3_get(s_t, channel);
        const float randt = rng.next();
        float backward_fraction = 0.0f, forward_pdf_factor = 0.0f, forward_stretching = 1.0f;
        float backward_pdf_factor = 0.0f, backward_stretching = 1.0f;
        if (bounce > 0) {
            const bool guided = rng.next() < guided_fraction;
            bool guide_backward = false;
            if (have_opposite) {
                const float x = fminf(fmaxf(dot(ray.o - P, -N), 0.0f), opposite_distance);
                backward_fraction = 1.0f / (1.0f + expf((opposite_distance - 2.0f * x) / diffusion_length));
                guide_backward = rng.next() < backward_fraction;
            }
            const float r0 = rng.next(), r1 = rng.next();
            float cos_theta, hgp;
            if (guided) {
                cos_theta = diffusion_length - (diffusion_length + 1.0f) * expf(-r0 * phase_log);
                if (guide_backward)
                    cos_theta = -cos_theta;
                const f3 nd = from_cosine(N, cos_theta, r1);
                hgp = hg_pdf(dot(ray.d, nd), g);
                ray.d = nd;
            } else {
                const f3 nd = hg_sample(ray.d, g, r0, r1, hgp);
                cos_theta = dot(nd, N);
                ray.d = nd;
            }
            forward_pdf_factor = (1.0f / 6.28318530718f) * (1.0f / ((diffusion_length - cos_theta) * phase_log)) / hgp;
            backward_pdf_factor = (1.0f / 6.28318530718f) * (1.0f / ((diffusion_length + cos_theta) * phase_log)) / hgp;
            forward_stretching = 1.0f - cos_theta / diffusion_length;
            backward_stretching = 1.0f + cos_theta / diffusion_length;
            if (guided)
                sample_sigma_t *= guide_backward ? backward_stretching : forward_stretching;
        }
        float t = -logf(1.0f - randt) / sample_sigma_t;
        ray.tmax = bounce == 0 ? fmaxf(t, 10.0f / fminf(sigma_t.x, fminf(sigma_t.y, sigma_t.z))) : t;
        WalkExit e;
        hit = cast(ray, e);
        if (hit) {
            ray.tmax = e.t;
            exit = e;
        }
        if (bounce == 0) {
            if (hit) {
                have_opposite = true;
                opposite_distance = dot(ray.o + ray.tmax * ray.d - P, -N);
            }
            hit = ray.tmax < t;
        }
        if (hit)
            t = ray.tmax;
        ray.o = ray.o + t * ray.d;
        // subsurface_random_walk_pdf (subsurface.cpp:139-146) and the MIS of subsurface.cpp:455-482
        const f3 transmittance = f3_exp(-t * s_t);
        f3 pdf = hit ? transmittance : mk(s_t.x * transmittance.x, s_t.y * transmittance.y, s_t.z * transmittance.z);
        if (bounce > 0) {
            const f3 tf = f3_exp(-t * (forward_stretching * s_t));
            f3 guided_pdf = hit ? tf : (forward_stretching * s_t) * tf;
            if (have_opposite) {
                const f3 tb = f3_exp(-t * (backward_stretching * s_t));
                const f3 back_pdf = hit ? tb : (backward_stretching * s_t) * tb;
                guided_pdf = f3_lerp(guided_pdf * forward_pdf_factor, back_pdf * backward_pdf_factor, backward_fraction);
            } else {
                guided_pdf = guided_pdf * forward_pdf_factor;
            }
            pdf = f3_lerp(pdf, guided_pdf, guided_fraction);
        }
        const f3 num = hit ? transmittance : s_s * transmittance;
        const float den = f3_sum(channel_pdf * pdf);
        throughput = throughput * (num / den);
        if (hit)
            break;
        if (fmaxf(throughput.x, fmaxf(throughput.y, throughput.z)) < 1e-6f)
            break;
    }
    wi = ray.d;
    return hit;
}

} // namespace ksb
