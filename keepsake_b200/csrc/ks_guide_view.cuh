// Guided rendering, device side: the per-vertex vMF mixtures written by the guide's path-inference
// kernel, sampling and pdf evaluation from them, and the training records a render captures.
//
// Mixture of path slot i (cap = path capacity, structure of arrays):
//   lobes[j * cap + i]       j < 8: mean direction xyz, concentration kappa of lobe j
//   lobes[(8 + k) * cap + i] k < 2: mixture weights of lobes 4k .. 4k+3, scaled by the selection
//                            probability alpha of the vertex (they sum to alpha)
// Training record r (one vertex of one path):
//   rec_pos[r]   hit position, bounce of the vertex (bits)
//   rec_wo[r]    outgoing direction, BSDF pdf of the sampled direction;
//   rec_wi[r]    sampled incident direction
//   rec_n[r]     geometric normal on the side of wo (guide::facing_normal)
//   rec_ibeta[r] 1 / path throughput before the vertex, per channel (0 where the throughput is 0)
//   rec_t[r]     luminance of the radiance gathered after the vertex, times rec_ibeta: the
//                one-sample estimate f cos L_i / pdf that the guide learns to be proportional to.
//                Emitter hits count with their MIS weight, as in the pixel estimate: light that
//                NEE already collects is not what the directional proposal should chase.
#pragma once
#include "ks_guide.cuh"
#include "ks_math.cuh"

namespace ksb
{

constexpr uint32_t kNoRecord = 0xffffffffu;
constexpr int kGuideLobeVecs = 10; // float4 per path slot

struct GuideView
{
    const float4 *lobes;
    uint32_t cap;
    int active; // directions are drawn from the guide (else: BSDF sampling only)
    float4 *rec_pos, *rec_wo, *rec_wi, *rec_ibeta, *rec_n;
    float *rec_t;
    uint32_t *rec_count;
    uint32_t rec_cap;       // 0 = no capture
    uint32_t rec_threshold; // a path records when the low 16 bits of its hash are below this
    uint32_t rec_bounces;   // the recorded bounce is drawn from [0, rec_bounces)
    float min_roughness;    // vertices below this roughness are not guided (alpha 0) and not recorded
};

// Selection probability alpha of the guide at path slot i.
KS_D float guide_alpha(const GuideView &g, uint32_t i)
{
    float4 wa = g.lobes[(size_t)8 * g.cap + i], wb = g.lobes[(size_t)9 * g.cap + i];
    return ((wa.x + wa.y) + (wa.z + wa.w)) + ((wb.x + wb.y) + (wb.z + wb.w));
}

// alpha times the mixture density at unit direction w (VMF::eval, vmf.h:32-39, summed with the
// stored lobe weights).
KS_D float guide_pdf(const GuideView &g, uint32_t i, f3 w)
{
    float4 wa = g.lobes[(size_t)8 * g.cap + i], wb = g.lobes[(size_t)9 * g.cap + i];
    float wt[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
    float p = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float4 m = g.lobes[(size_t)j * g.cap + i];
        p += wt[j] * guide::vmf_eval(mk(m.x, m.y, m.z), m.w, w);
    }
    return p;
}

// sample_vmm (vmf.h:123-127): lobe by sample_small_distrib (rng.h:399-432) on u0, remapped u0 and
// u1 then drive VMF::sample (vmf.h:41-56).
KS_D f3 guide_sample(const GuideView &g, uint32_t i, float u0, float u1)
{
    float4 wa = g.lobes[(size_t)8 * g.cap + i], wb = g.lobes[(size_t)9 * g.cap + i];
    float wt[8] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
    float sum_w = 0.0f;
    int last_positive = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        sum_w += wt[j];
        if (wt[j] > 0.0f)
            last_positive = j;
    }
    float inv = 1.0f / sum_w, cdf = 0.0f;
    int sel = -1;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float nx = cdf + wt[j] * inv;
        if (sel < 0 && u0 < nx) {
            sel = j;
            u0 = (u0 - cdf) / (nx - cdf);
        }
        cdf = nx;
    }
    if (sel < 0)
        sel = last_positive;
    float4 m = g.lobes[(size_t)sel * g.cap + i];
    const float kappa = m.w;
    float cos_theta = 1.0f + logf(u0 + expf(-2.0f * kappa) * (1.0f - u0)) / kappa;
    // u0 = 0 with a concentration whose exp(-2 kappa) underflows gives log(0): the pole opposite mu
    cos_theta = fminf(fmaxf(cos_theta, -1.0f), 1.0f);
    float sin_theta = sqrtf(fmaxf(0.0f, 1.0f - cos_theta * cos_theta));
    float phi = kTwoPi * u1;
    f3 w = mk(cosf(phi) * sin_theta, sinf(phi) * sin_theta, cos_theta);
    f3 N = mk(m.x, m.y, m.z);
    // orthonormal_basis (maths.h:814-821)
    float sign = copysignf(1.0f, N.z);
    const float a = -1.0f / (sign + N.z);
    const float b = N.x * N.y * a;
    f3 X = mk(1.0f + sign * N.x * N.x * a, sign * b, -sign * N.x);
    f3 Y = mk(b, sign + N.y * N.y * a, -N.y);
    return normalize(w.x * X + w.y * Y + w.z * N);
}

// Adds radiance gathered along the recorded direction (already multiplied by the current path
// throughput) to record r.
KS_D void record_add(const GuideView &g, uint32_t r, f3 c)
{
    float4 ib = g.rec_ibeta[r];
    g.rec_t[r] += luminance(mk(c.x * ib.x, c.y * ib.y, c.z * ib.z));
}

KS_D uint32_t path_hash(uint32_t pix, uint32_t smp)
{
    uint32_t h = pix * 0x9E3779B1u ^ (smp + 0x7F4A7C15u) * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    h *= 0x297A2D39u;
    h ^= h >> 15;
    return h;
}

} // namespace ksb
