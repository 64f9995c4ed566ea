// Owen-scrambled Sobol (0,2) sampler with permuted Morton indices, per pixel and per sample.
//
// Follows the reference CPU sampler `OwenScrambledSobol02Morton` + `PTRenderSampler`
// (sobol.h:131-248) integer for integer, including its quirks:
//   * the Morton index is formed in 32 bits before widening (sobol.h:145),
//   * `0x55555555u * dimension` is a 32-bit product (sobol.h:209,218),
//   * next()/next2d() permute with the dimension *before* the increment and hash the dimension
//     *after* it (sobol.h:148-166).
// Only generator matrices 0 and 1 are ever read by this sampler (sobol.h:44, :160-166).  Their
// closed forms (checked against the reference table sobol.cpp:154+ by the golden fixture):
//   dim 0 column k = 0x80000000 >> k for k < 32, else 0
//   dim 1 column k = P[k mod 32], P[0] = 0x80000000, P[k] = P[k-1] ^ (P[k-1] >> 1).
#pragma once
#include "ks_math.cuh"

namespace ksb
{

KS_HD uint64_t mix_bits64(uint64_t v)
{
    // hash.h:206-214
    v ^= (v >> 31);
    v *= 0x7fb5d329728ea185ull;
    v ^= (v >> 27);
    v *= 0x81dadef4bc2dd44dull;
    v ^= (v >> 33);
    return v;
}

// MurmurHash64A of exactly 8 bytes (two little-endian int32s), seed 0: hash(int, int) in hash.h:243-252.
KS_HD uint64_t murmur64a_2x32(uint32_t lo, uint32_t hi)
{
    const uint64_t m = 0xc6a4a7935bd1e995ull;
    const int r = 47;
    uint64_t h = 0ull ^ (8ull * m);
    uint64_t k = (uint64_t)lo | ((uint64_t)hi << 32);
    k *= m;
    k ^= k >> r;
    k *= m;
    h ^= k;
    h *= m;
    h ^= h >> r;
    h *= m;
    h ^= h >> r;
    return h;
}

KS_HD uint32_t reverse_bits32(uint32_t v)
{
#ifdef __CUDA_ARCH__
    return __brev(v);
#else
    v = (v << 16u) | (v >> 16u);
    v = ((v & 0x55555555u) << 1u) | ((v & 0xAAAAAAAAu) >> 1u);
    v = ((v & 0x33333333u) << 2u) | ((v & 0xCCCCCCCCu) >> 2u);
    v = ((v & 0x0F0F0F0Fu) << 4u) | ((v & 0xF0F0F0F0u) >> 4u);
    v = ((v & 0x00FF00FFu) << 8u) | ((v & 0xFF00FF00u) >> 8u);
    return v;
#endif
}

KS_HD uint32_t owen_scramble(uint32_t v, uint32_t seed)
{
    // FastOwenScrambler (sobol.h:17-33)
    v = reverse_bits32(v);
    v ^= v * 0x3d20adeau;
    v += seed;
    v *= (seed >> 16) | 1u;
    v ^= v * 0x05526c56u;
    v ^= v * 0x53a22864u;
    return reverse_bits32(v);
}

// FastOwenScrambler applied to a value given in bit-reversed form: owen_scramble(reverse(x)).
KS_HD uint32_t owen_scramble_reversed(uint32_t x, uint32_t seed)
{
    x ^= x * 0x3d20adeau;
    x += seed;
    x *= (seed >> 16) | 1u;
    x ^= x * 0x05526c56u;
    x ^= x * 0x53a22864u;
    return reverse_bits32(x);
}

// sobol_sample(a, dim, FastOwenScrambler(seed)) for dim in {0, 1} (sobol.h:35-49).
//   dim 0: v = reverse(a mod 2^32)                         (columns 0x80000000 >> k, zero for k >= 32)
//   dim 1: v = XOR of P[k mod 32] over the set bits k of a. Bit 31-j of P[k] is C(k, j) mod 2, i.e.
//          set iff j is a bit-subset of k (Lucas), so reverse(v) is the GF(2) superset-sum transform
//          of the folded index: five masked shift-xor steps instead of a 52-column loop.
// The scrambler reverses its input first, so both cases hand it the reversed form directly.
KS_HD float sobol_sample_01(uint64_t a, int dim, uint32_t seed)
{
    uint32_t x = (uint32_t)a;
    if (dim != 0) {
        x ^= (uint32_t)(a >> 32); // columns repeat with period 32
        x ^= (x >> 1) & 0x55555555u;
        x ^= (x >> 2) & 0x33333333u;
        x ^= (x >> 4) & 0x0f0f0f0fu;
        x ^= (x >> 8) & 0x00ff00ffu;
        x ^= (x >> 16) & 0x0000ffffu;
    }
    uint32_t v = owen_scramble_reversed(x, seed);
    float f = (float)v * 0x1p-32f;
    return f < kOneMinusEps ? f : kOneMinusEps;
}

// mix_bits (hash.h:206-214) of a value below 2^32, then (>> 24) % 24 as in sobol.h:209.
KS_HD int digit_perm_index(uint32_t x)
{
    uint64_t v = mix_bits64((uint64_t)x);
    uint64_t y = v >> 24; // < 2^40
    // y % 24 without a 64-bit division: 2^32 = 16 (mod 24)
    uint32_t hi = (uint32_t)(y >> 32), lo = (uint32_t)y;
    return (int)((hi * 16u + lo % 24u) % 24u);
}

KS_HD uint32_t part1by1(uint32_t x)
{
    x &= 0x0000ffffu;
    x = (x ^ (x << 8)) & 0x00ff00ffu;
    x = (x ^ (x << 4)) & 0x0f0f0f0fu;
    x = (x ^ (x << 2)) & 0x33333333u;
    x = (x ^ (x << 1)) & 0x55555555u;
    return x;
}

// All 24 orderings of {0,1,2,3}, in the order the reference enumerates them (sobol.h:169-199).
KS_HD int digit_permutation(int p, int digit)
{
    // Packed: 2 bits per entry (entry 0 in the low bits), one byte per permutation, 8 bytes per
    // 64-bit word, so the lookup stays in registers.  Bytes, permutation 0 first:
    //   E4 B4 D8 78 6C 9C E1 B1 | C9 39 2D 8D C6 36 D2 72 | 4E 1E 27 87 1B 4B 63 93
    constexpr uint64_t w0 = 0xB1E19C6C78D8B4E4ull, w1 = 0x72D236C68D2D39C9ull, w2 = 0x93634B1B87271E4Eull;
    const uint64_t w = p < 8 ? w0 : (p < 16 ? w1 : w2);
#ifdef __CUDA_ARCH__
    // byte p & 7 of the word in the low byte (one byte-permute instead of a 64-bit shift)
    const uint32_t byte = __byte_perm((uint32_t)w, (uint32_t)(w >> 32), (uint32_t)(p & 7));
#else
    const uint32_t byte = (uint32_t)(w >> (8 * (p & 7))) & 0xffu;
#endif
    return (int)((byte >> (2 * digit)) & 3u);
}

struct SobolSampler
{
    uint64_t morton_index;
    int dimension;
    uint32_t seed;
    int log2_spp;
    int n_base4_digits;

    // PTRenderSampler constructor + start_pixel(pixel, index, 0) (sobol.h:139-147, 237-241)
    KS_HD static SobolSampler start(uint32_t px, uint32_t py, uint32_t sample_index, int log2_spp,
                                    int n_base4_digits, uint32_t seed, int dim = 0)
    {
        SobolSampler s;
        s.dimension = dim;
        s.seed = seed;
        s.log2_spp = log2_spp;
        s.n_base4_digits = n_base4_digits;
        uint32_t morton = (part1by1(py) << 1) + part1by1(px);
        s.morton_index = (uint64_t)((morton << log2_spp) | sample_index);
        return s;
    }

    // get_sample_index (sobol.h:168-222).  The Morton index is built in 32 bits (sobol.h:145), so
    // every `higher digits` value is below 2^32 and the loop runs in 32-bit integers; only the
    // permuted index itself can exceed 32 bits (up to 2 * n_base4_digits).
    // For N dimensions at once (dim_mix[k] = 0x55555555 * dimension, a 32-bit product): one pass
    // over the digits, whose values and higher digits do not depend on the dimension.  The digits
    // are visited from the top, each one lands 2 bits below the previous one, so the index is
    // built by shifting in 2 bits at a time (and the final bit of an odd log2 spp by one more).
    template <int N>
    KS_HD void sample_indices(const uint32_t (&dim_mix)[N], uint64_t (&out)[N]) const
    {
        const uint32_t m = (uint32_t)morton_index;
        const bool pow2 = (log2_spp & 1) != 0;
        const int last_digit = pow2 ? 1 : 0;
#pragma unroll
        for (int k = 0; k < N; ++k)
            out[k] = 0;
        for (int i = n_base4_digits - 1; i >= last_digit; --i) {
            int shift = 2 * i - (pow2 ? 1 : 0);
            uint32_t digit = shift >= 32 ? 0u : ((m >> shift) & 3u);
            uint32_t higher = shift + 2 >= 32 ? 0u : (m >> (shift + 2));
#pragma unroll
            for (int k = 0; k < N; ++k)
                out[k] = (out[k] << 2) |
                         (uint64_t)digit_permutation(digit_perm_index(higher ^ dim_mix[k]), (int)digit);
        }
        if (pow2) {
            uint32_t digit = m & 1u;
#pragma unroll
            for (int k = 0; k < N; ++k)
                out[k] = (out[k] << 1) |
                         (uint64_t)(digit ^ (uint32_t)(mix_bits64((uint64_t)((m >> 1) ^ dim_mix[k])) & 1u));
        }
    }

    KS_HD uint64_t sample_index() const
    {
        const uint32_t dim_mix[1] = {0x55555555u * (uint32_t)dimension};
        uint64_t out[1];
        sample_indices<1>(dim_mix, out);
        return out[0];
    }

    KS_HD float next()
    {
        uint64_t a = sample_index();
        ++dimension;
        uint32_t h = (uint32_t)murmur64a_2x32((uint32_t)dimension, seed);
        return sobol_sample_01(a, 0, h);
    }

    KS_HD void next2d(float &u0, float &u1)
    {
        uint64_t a = sample_index();
        dimension += 2;
        uint64_t bits = murmur64a_2x32((uint32_t)dimension, seed);
        u0 = sobol_sample_01(a, 0, (uint32_t)bits);
        u1 = sobol_sample_01(a, 1, (uint32_t)(bits >> 32));
    }

    // The seven values of one bounce, equal to next(), next2d(), next(), next2d(), next() in turn
    // (light selection, light uv, BSDF lobe, BSDF direction, roulette: nee.cpp:28-34,
    // material.cpp:157-158, small_pt.cpp:168-174), with the five permuted indices from one pass.
    KS_HD void bounce_values(float (&u)[7])
    {
        const uint32_t d = (uint32_t)dimension;
        const uint32_t mix[5] = {0x55555555u * d, 0x55555555u * (d + 1), 0x55555555u * (d + 3),
                                 0x55555555u * (d + 4), 0x55555555u * (d + 6)};
        uint64_t a[5];
        sample_indices<5>(mix, a);
        u[0] = sobol_sample_01(a[0], 0, (uint32_t)murmur64a_2x32(d + 1, seed));
        uint64_t h = murmur64a_2x32(d + 3, seed);
        u[1] = sobol_sample_01(a[1], 0, (uint32_t)h);
        u[2] = sobol_sample_01(a[1], 1, (uint32_t)(h >> 32));
        u[3] = sobol_sample_01(a[2], 0, (uint32_t)murmur64a_2x32(d + 4, seed));
        h = murmur64a_2x32(d + 6, seed);
        u[4] = sobol_sample_01(a[3], 0, (uint32_t)h);
        u[5] = sobol_sample_01(a[3], 1, (uint32_t)(h >> 32));
        u[6] = sobol_sample_01(a[4], 0, (uint32_t)murmur64a_2x32(d + 7, seed));
        dimension += 7;
    }
};

// Host-side setup of the per-render constants (sobol.h:131-138).
inline void sobol_setup(int spp, int full_w, int full_h, int &log2_spp, int &n_base4_digits)
{
    auto log2i = [](uint32_t v) { return 31 - __builtin_clz(v); };
    log2_spp = log2i((uint32_t)spp);
    int32_t m = full_w > full_h ? full_w : full_h;
    int32_t v = m - 1;
    v |= v >> 1;
    v |= v >> 2;
    v |= v >> 4;
    v |= v >> 8;
    v |= v >> 16;
    int res = v + 1;
    int log4 = (log2_spp + 1) / 2;
    n_base4_digits = log2i((uint32_t)res) + log4;
}

} // namespace ksb
