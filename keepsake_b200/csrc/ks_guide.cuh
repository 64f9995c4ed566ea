// Learned path guiding: input encodings, the vMF mixture head and its loss gradient.
//
// The network maps a shading point (position, outgoing direction, surface normal) to an 8-lobe
// von Mises-Fisher mixture over incident directions:
//   input  = multiresolution hash-grid encoding of the position (16 levels x 2 features) +
//            real spherical harmonics up to degree 3 of the outgoing direction (16 values) and of
//            the geometric normal turned towards it (16 values)
//   MLP    = 64 -> 64 -> 64 -> 64 -> 64 -> 41 (4 hidden ReLU layers, no biases)
//   output = per lobe: mean direction (3, normalised), log concentration, mixture logit; then one
//            logit of the selection probability alpha = alpha_max * sigmoid(logit) with which a
//            renderer draws from the mixture instead of the BSDF (one-sample MIS).
// vMF evaluation and sampling follow the reference's VMF (vmf.h:10-56, max_kappa 1e4) and
// sample_vmm (vmf.h:123-127); lobe selection is sample_small_distrib (rng.h:399-434).
#pragma once
#include "ks_math.cuh"

namespace ksb
{
namespace guide
{

constexpr int kLevels = 16;
constexpr int kFeatPerLevel = 2;
constexpr int kLog2T = 19;
constexpr uint32_t kTableSize = 1u << kLog2T;
constexpr int kGridFeatures = kLevels * kFeatPerLevel; // 32
constexpr int kShCoeffs = 16;
constexpr int kIn = kGridFeatures + 2 * kShCoeffs; // 64
constexpr int kHidden = 64;
constexpr int kLobes = 8;
constexpr int kSel = kLobes * 5;     // index of the selection logit
constexpr int kOut = kLobes * 5 + 1; // 41
constexpr int kOutPad = 48;      // output layer rows padded to a multiple of 16
constexpr int kLayers = 5;
constexpr float kMaxKappa = 1e4f; // VMF::max_kappa (vmf.h:111)
constexpr float kMinLogKappa = -6.0f;

// layer l: W_l is [out_l][in_l], row-major, fp32 master copy, concatenated
__host__ __device__ constexpr int layer_in(int l) { return l == 0 ? kIn : kHidden; }
__host__ __device__ constexpr int layer_out(int l) { return l == kLayers - 1 ? kOutPad : kHidden; }
__host__ __device__ constexpr int weight_offset(int l)
{
    int o = 0;
    for (int i = 0; i < l; ++i)
        o += layer_in(i) * layer_out(i);
    return o;
}
constexpr int kWeights = weight_offset(kLayers); // 19456

struct GridParams
{
    uint32_t res[kLevels]; // cells per axis of each level (geometric from base to max resolution)
    float bmin[3];         // scene bound used to normalise positions
    float inv_ext[3];
};

__host__ __device__ inline uint32_t level_res(const GridParams &g, int l) { return g.res[l]; }

// Grid cell corner -> table entry.  While a level's corners fit the table they are stored in
// 2 x 2 x 2 blocks of 8 consecutive entries (a block of 4-byte FP16 feature pairs is one 32-byte L2
// sector, so a cell's 8 corners fall into 3.4 blocks on average instead of 8 sectors); finer levels
// hash each corner with the spatial hash of Teschner et al. and the primes of instant-ngp (corners
// collide independently, which keeps the trilinear blend of a cell from taking all 8 corners from one
// colliding block).
__host__ __device__ __forceinline__ uint32_t grid_index(uint32_t res, uint32_t x, uint32_t y, uint32_t z)
{
    const uint64_t side = ((uint64_t)res + 2) >> 1; // blocks per axis over corners 0..res
    if (side * side * side * 8 <= kTableSize) {
        const uint32_t inner = (x & 1u) | ((y & 1u) << 1) | ((z & 1u) << 2);
        return (uint32_t)((x >> 1) + side * ((y >> 1) + side * (z >> 1))) * 8u + inner;
    }
    return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & (kTableSize - 1u);
}

struct Corner
{
    uint32_t idx[8];
    float w[8];
};

__device__ __forceinline__ void level_corners(const GridParams &g, int l, f3 pn, Corner &c)
{
    uint32_t res = level_res(g, l);
    float px = pn.x * (float)res, py = pn.y * (float)res, pz = pn.z * (float)res;
    // pn is in [0, 1]; the cell index is clamped to res - 1 so that corners stay in [0, res]
    float fx0 = fminf(floorf(px), (float)(res - 1)), fy0 = fminf(floorf(py), (float)(res - 1)),
          fz0 = fminf(floorf(pz), (float)(res - 1));
    uint32_t ix = (uint32_t)fx0, iy = (uint32_t)fy0, iz = (uint32_t)fz0;
    float tx = px - fx0, ty = py - fy0, tz = pz - fz0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        uint32_t dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        c.idx[k] = grid_index(res, ix + dx, iy + dy, iz + dz);
        c.w[k] = (dx ? tx : 1.0f - tx) * (dy ? ty : 1.0f - ty) * (dz ? tz : 1.0f - tz);
    }
}

// Geometric normal of triangle (p0, p1, p2) on the side of the unit direction wo: the normal input
// of the network (the same arithmetic wherever a vertex is encoded).
__device__ __forceinline__ f3 facing_normal(f3 p0, f3 p1, f3 p2, f3 wo)
{
    f3 n = normalize(cross(p1 - p0, p2 - p0));
    return dot(n, wo) < 0.0f ? -n : n;
}

__device__ __forceinline__ f3 normalise_position(const GridParams &g, f3 p)
{
    f3 q = mk((p.x - g.bmin[0]) * g.inv_ext[0], (p.y - g.bmin[1]) * g.inv_ext[1], (p.z - g.bmin[2]) * g.inv_ext[2]);
    q.x = fminf(fmaxf(q.x, 0.0f), 1.0f);
    q.y = fminf(fmaxf(q.y, 0.0f), 1.0f);
    q.z = fminf(fmaxf(q.z, 0.0f), 1.0f);
    return q;
}

// Real spherical harmonics Y_lm of a unit direction, l = 0..3 (16 values).
__host__ __device__ inline void sh16(f3 d, float out[16])
{
    float x = d.x, y = d.y, z = d.z;
    float xx = x * x, yy = y * y, zz = z * z;
    out[0] = 0.28209479177387814f;
    out[1] = -0.48860251190291987f * y;
    out[2] = 0.48860251190291987f * z;
    out[3] = -0.48860251190291987f * x;
    out[4] = 1.0925484305920792f * x * y;
    out[5] = -1.0925484305920792f * y * z;
    out[6] = 0.94617469575755997f * zz - 0.31539156525251999f;
    out[7] = -1.0925484305920792f * x * z;
    out[8] = 0.54627421529603959f * (xx - yy);
    out[9] = 0.59004358992664352f * y * (-3.0f * xx + yy);
    out[10] = 2.8906114426405538f * x * y * z;
    out[11] = 0.45704579946446572f * y * (1.0f - 5.0f * zz);
    out[12] = 0.3731763325901154f * z * (5.0f * zz - 3.0f);
    out[13] = 0.45704579946446572f * x * (1.0f - 5.0f * zz);
    out[14] = 1.4453057213202769f * z * (xx - yy);
    out[15] = 0.59004358992664352f * x * (-xx + 3.0f * yy);
}

// ---- vMF mixture -------------------------------------------------------------------------------
struct Lobe
{
    f3 mu;
    float kappa;
    float w;
};

__host__ __device__ inline float sigmoid(float x) { return 1.0f / (1.0f + expf(-x)); }
__host__ __device__ inline float softplus(float x) { return x > 20.0f ? x : log1pf(expf(x)); }

// log concentration from its raw output: a smooth clamp into (kMinLogKappa, log kMaxKappa) whose
// derivative (sigmoid(z - lo) - sigmoid(z - hi)) stays positive, so no lobe is ever cut off from
// the gradient by a bound.
__host__ __device__ inline float log_kappa(float z)
{
    const float lo = kMinLogKappa, hi = 9.210340372f; // log(1e4)
    return lo + softplus(z - lo) - softplus(z - hi);
}
__host__ __device__ inline float log_kappa_grad(float z)
{
    const float lo = kMinLogKappa, hi = 9.210340372f;
    return sigmoid(z - lo) - sigmoid(z - hi);
}

// Decodes the raw outputs of one sample into the mixture.
__device__ __forceinline__ void decode_mixture(const float o[kOut], Lobe lobes[kLobes])
{
    float mx = -kInf;
    for (int j = 0; j < kLobes; ++j)
        mx = fmaxf(mx, o[5 * j + 4]);
    float sum = 0.0f;
    for (int j = 0; j < kLobes; ++j) {
        f3 r = mk(o[5 * j], o[5 * j + 1], o[5 * j + 2]);
        float n = sqrtf(sqnorm(r));
        lobes[j].mu = n > 1e-20f ? r / n : mk(0.0f, 0.0f, 1.0f);
        lobes[j].kappa = fminf(expf(log_kappa(o[5 * j + 3])), kMaxKappa);
        lobes[j].w = expf(o[5 * j + 4] - mx);
        sum += lobes[j].w;
    }
    for (int j = 0; j < kLobes; ++j)
        lobes[j].w /= sum;
}

// VMF::eval (vmf.h:34-41)
__host__ __device__ inline float vmf_eval(f3 mu, float kappa, f3 w)
{
    if (kappa == 0.0f)
        return kInvPi * 0.25f;
    float scale = kappa / (kTwoPi * (1.0f - expf(-2.0f * kappa)));
    float c = dot(mu, w) - 1.0f;
    return scale * expf(kappa * fminf(0.0f, c));
}

__device__ __forceinline__ float mixture_pdf(const Lobe lobes[kLobes], f3 w)
{
    float p = 0.0f;
    for (int j = 0; j < kLobes; ++j)
        p += lobes[j].w * vmf_eval(lobes[j].mu, lobes[j].kappa, w);
    return p;
}

// sample_vmm (vmf.h:123-127): lobe by sample_small_distrib with u0 remapped, then VMF::sample.
__device__ __forceinline__ f3 mixture_sample(const Lobe lobes[kLobes], float u0, float u1)
{
    float sum_w = 0.0f;
    int last_positive = 0;
    for (int j = 0; j < kLobes; ++j) {
        sum_w += lobes[j].w;
        if (lobes[j].w > 0.0f)
            last_positive = j;
    }
    float inv = 1.0f / sum_w, cdf = 0.0f;
    int sel = -1;
    for (int j = 0; j < kLobes; ++j) {
        float nx = cdf + lobes[j].w * inv;
        if (u0 < nx) {
            sel = j;
            u0 = (u0 - cdf) / (nx - cdf);
            break;
        }
        cdf = nx;
    }
    if (sel < 0)
        sel = last_positive;
    const Lobe &L = lobes[sel];
    // VMF::sample (vmf.h:43-56)
    float kappa = L.kappa;
    float cos_theta = 1.0f + logf(u0 + expf(-2.0f * kappa) * (1.0f - u0)) / kappa;
    float sin_theta = sqrtf(fmaxf(0.0f, 1.0f - cos_theta * cos_theta));
    float phi = kTwoPi * u1;
    f3 w = mk(cosf(phi) * sin_theta, sinf(phi) * sin_theta, cos_theta);
    f3 N = L.mu;
    float sign = copysignf(1.0f, N.z);
    const float a = -1.0f / (sign + N.z);
    const float b = N.x * N.y * a;
    f3 X = mk(1.0f + sign * N.x * N.x * a, sign * b, -sign * N.x);
    f3 Y = mk(b, sign + N.y * N.y * a, -N.y);
    return w.x * X + w.y * Y + w.z * N;
}

// Loss of one training sample and its gradient with respect to the raw outputs (exact derivatives
// of decode_mixture + mixture_pdf + the selection sigmoid).  Two objectives over samples with
// t = f cos L / p (the estimate of the integrand over the density the direction was drawn from):
//   mixture:   -t log q(wi)    fits q to the integrand f cos L (its KL divergence);
//   selection: -t log m(wi)    m = alpha q + (1 - alpha) p_bsdf, the combined proposal of one-
//                              sample MIS, minimised over alpha alone (q held fixed), so that
//                              alpha learns how far to trust q without starving q of gradient.
// `loss` returns -t log m.  Returns false for an unusable sample (m == 0 or q == 0); the gradient
// is then zero.
__device__ __forceinline__ bool mixture_loss_grad(const float o[kOut], f3 wi, float t, float p_bsdf, float alpha_max,
                                                  float &loss, float g[kOut])
{
    for (int i = 0; i < kOut; ++i)
        g[i] = 0.0f;
    loss = 0.0f;
    if (!(t > 0.0f))
        return true;
    Lobe lobes[kLobes];
    decode_mixture(o, lobes);
    float v[kLobes], q = 0.0f;
    for (int j = 0; j < kLobes; ++j) {
        v[j] = vmf_eval(lobes[j].mu, lobes[j].kappa, wi);
        q += lobes[j].w * v[j];
    }
    const float sg = sigmoid(o[kSel]), alpha = alpha_max * sg;
    const float m = alpha * q + (1.0f - alpha) * p_bsdf;
    if (!(m > 1e-30f) || !(q > 1e-30f))
        return false;
    loss = -t * logf(m);
    // d(-t log m)/d alpha = -t (q - p_bsdf) / m, alpha = alpha_max sigmoid(z)
    g[kSel] = -t * (q - p_bsdf) / m * alpha_max * sg * (1.0f - sg);
    for (int j = 0; j < kLobes; ++j) {
        float r = lobes[j].w * v[j] / q; // responsibility
        // mixture logit: d(-t log q)/dz_j = -t (r_j - pi_j)
        g[5 * j + 4] = -t * (r - lobes[j].w);
        float kappa = lobes[j].kappa;
        // d log v / d kappa = 1/kappa - 2 / (e^{2 kappa} - 1) + (mu.w - 1); kappa = exp(log_kappa(z))
        float dlog = 1.0f / kappa - 2.0f / expm1f(2.0f * kappa) + (dot(lobes[j].mu, wi) - 1.0f);
        g[5 * j + 3] = -t * r * dlog * kappa * log_kappa_grad(o[5 * j + 3]);
        // mean direction: mu = raw / |raw|, d log v / d mu = kappa * wi
        f3 raw = mk(o[5 * j], o[5 * j + 1], o[5 * j + 2]);
        float n = sqrtf(sqnorm(raw));
        if (n > 1e-20f) {
            f3 mu = lobes[j].mu;
            f3 gm = kappa * wi;
            f3 proj = (gm - dot(gm, mu) * mu) / n;
            g[5 * j + 0] = -t * r * proj.x;
            g[5 * j + 1] = -t * r * proj.y;
            g[5 * j + 2] = -t * r * proj.z;
        }
    }
    return true;
}

} // namespace guide
} // namespace ksb
