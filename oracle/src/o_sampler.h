// ORACLE (test infrastructure only; never linked into the product).
// CPU restatement of keepsake's Owen-scrambled Sobol sampler with permuted Morton indices.
//
// Follows: sobol.h:17-49 (FastOwenScrambler, sobol_sample), sobol.h:131-228
// (OwenScrambledSobol02Morton), sobol.h:235-248 (PTRenderSampler), hash.h:140-185
// (murmur_hash_64A), hash.h:206-214 (mix_bits), hash.h:243-252 (hash(args...)),
// maths.h:194-205 (round_up_pow2, log2_int), maths.h:267 (reverse_bits_32), maths.h:382-425
// (part_1_by_1, encode_morton_2).
//
// Generator matrices: the reference table sobol.cpp:154+ is rebuilt here for dimensions 0 and 1
// (the only ones this sampler reads) by the recurrence that tests/golden/sobol_matrices.json
// pins against the reference table.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle
{

inline const float fp32_before_one = std::nextafter(1.0f, -INFINITY);

inline uint64_t murmur_hash_64A(const unsigned char *key, size_t len, uint64_t seed)
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
    switch (len & 7) {
    case 7:
        h ^= uint64_t(key[6]) << 48;
        [[fallthrough]];
    case 6:
        h ^= uint64_t(key[5]) << 40;
        [[fallthrough]];
    case 5:
        h ^= uint64_t(key[4]) << 32;
        [[fallthrough]];
    case 4:
        h ^= uint64_t(key[3]) << 24;
        [[fallthrough]];
    case 3:
        h ^= uint64_t(key[2]) << 16;
        [[fallthrough]];
    case 2:
        h ^= uint64_t(key[1]) << 8;
        [[fallthrough]];
    case 1:
        h ^= uint64_t(key[0]);
        h *= m;
    }
    h ^= h >> r;
    h *= m;
    h ^= h >> r;
    return h;
}

// hash(int a, int b): the two values are laid out back to back and hashed with seed 0.
inline uint64_t hash2i(int a, int b)
{
    unsigned char buf[8];
    std::memcpy(buf, &a, 4);
    std::memcpy(buf + 4, &b, 4);
    return murmur_hash_64A(buf, 8, 0);
}

inline uint64_t mix_bits(uint64_t v)
{
    v ^= (v >> 31);
    v *= 0x7fb5d329728ea185;
    v ^= (v >> 27);
    v *= 0x81dadef4bc2dd44d;
    v ^= (v >> 33);
    return v;
}

inline uint32_t reverse_bits_32(uint32_t bits)
{
    bits = (bits << 16u) | (bits >> 16u);
    bits = ((bits & 0x55555555u) << 1u) | ((bits & 0xAAAAAAAAu) >> 1u);
    bits = ((bits & 0x33333333u) << 2u) | ((bits & 0xCCCCCCCCu) >> 2u);
    bits = ((bits & 0x0F0F0F0Fu) << 4u) | ((bits & 0xF0F0F0F0u) >> 4u);
    bits = ((bits & 0x00FF00FFu) << 8u) | ((bits & 0xFF00FF00u) >> 8u);
    return bits;
}

inline int log2_int(uint32_t v) { return 31 - __builtin_clz(v); }

inline int32_t round_up_pow2(int32_t v)
{
    v--;
    v |= v >> 1;
    v |= v >> 2;
    v |= v >> 4;
    v |= v >> 8;
    v |= v >> 16;
    return v + 1;
}

inline uint32_t part_1_by_1(uint32_t x)
{
    x &= 0x0000ffff;
    x = (x ^ (x << 8)) & 0x00ff00ff;
    x = (x ^ (x << 4)) & 0x0f0f0f0f;
    x = (x ^ (x << 2)) & 0x33333333;
    x = (x ^ (x << 1)) & 0x55555555;
    return x;
}

inline uint32_t encode_morton_2(uint32_t x, uint32_t y) { return (part_1_by_1(y) << 1) + part_1_by_1(x); }

constexpr int sobol_matrix_size = 52;

// Columns of the generator matrices of dimensions 0 and 1.
struct SobolMatrices01
{
    uint32_t m[2 * sobol_matrix_size];
    SobolMatrices01()
    {
        uint32_t p = 0x80000000u;
        for (int k = 0; k < sobol_matrix_size; ++k) {
            m[k] = k < 32 ? (0x80000000u >> k) : 0u;
            if (k % 32 == 0)
                p = 0x80000000u;
            m[sobol_matrix_size + k] = p;
            p ^= p >> 1;
        }
    }
};
inline const SobolMatrices01 &sobol_matrices()
{
    static SobolMatrices01 s;
    return s;
}

struct FastOwenScrambler
{
    explicit FastOwenScrambler(uint32_t seed) : seed(seed) {}
    uint32_t operator()(uint32_t v) const
    {
        v = reverse_bits_32(v);
        v ^= v * 0x3d20adea;
        v += seed;
        v *= (seed >> 16) | 1;
        v ^= v * 0x05526c56;
        v ^= v * 0x53a22864;
        return reverse_bits_32(v);
    }
    uint32_t seed;
};

inline float sobol_sample(int64_t a, int dimension, FastOwenScrambler randomizer)
{
    uint32_t v = 0;
    for (int i = dimension * sobol_matrix_size; a != 0; a >>= 1, i++)
        if (a & 1)
            v ^= sobol_matrices().m[i];
    v = randomizer(v);
    return std::min(v * 0x1p-32f, fp32_before_one);
}

struct OwenScrambledSobol02Morton
{
    OwenScrambledSobol02Morton(int samples_per_pixel, int full_w, int full_h, int seed) : seed(seed)
    {
        log2_samples_per_pixel = log2_int((uint32_t)samples_per_pixel);
        int res = round_up_pow2(std::max(full_w, full_h));
        int log4_samples_per_pixel = (log2_samples_per_pixel + 1) / 2;
        n_base4_digits = log2_int((uint32_t)res) + log4_samples_per_pixel;
    }

    void start_pixel(int px, int py, int index, int dim)
    {
        dimension = dim;
        morton_index = (encode_morton_2(px, py) << log2_samples_per_pixel) | index;
    }

    float next()
    {
        uint64_t sample_index = get_sample_index();
        ++dimension;
        uint32_t sample_hash = hash2i(dimension, seed);
        return sobol_sample(sample_index, 0, FastOwenScrambler(sample_hash));
    }

    void next2d(float &u0, float &u1)
    {
        uint64_t sample_index = get_sample_index();
        dimension += 2;
        uint64_t bits = hash2i(dimension, seed);
        uint32_t sample_hash[2] = {uint32_t(bits), uint32_t(bits >> 32)};
        u0 = sobol_sample(sample_index, 0, FastOwenScrambler(sample_hash[0]));
        u1 = sobol_sample(sample_index, 1, FastOwenScrambler(sample_hash[1]));
    }

    uint64_t get_sample_index() const
    {
        static constexpr uint8_t permutations[24][4] = {
            {0, 1, 2, 3}, {0, 1, 3, 2}, {0, 2, 1, 3}, {0, 2, 3, 1}, {0, 3, 2, 1}, {0, 3, 1, 2},
            {1, 0, 2, 3}, {1, 0, 3, 2}, {1, 2, 0, 3}, {1, 2, 3, 0}, {1, 3, 2, 0}, {1, 3, 0, 2},
            {2, 1, 0, 3}, {2, 1, 3, 0}, {2, 0, 1, 3}, {2, 0, 3, 1}, {2, 3, 0, 1}, {2, 3, 1, 0},
            {3, 1, 2, 0}, {3, 1, 0, 2}, {3, 2, 1, 0}, {3, 2, 0, 1}, {3, 0, 2, 1}, {3, 0, 1, 2}};
        uint64_t sample_index = 0;
        bool pow_2_samples = log2_samples_per_pixel & 1;
        int last_digit = pow_2_samples ? 1 : 0;
        for (int i = n_base4_digits - 1; i >= last_digit; --i) {
            int digit_shift = 2 * i - (pow_2_samples ? 1 : 0);
            int digit = (morton_index >> digit_shift) & 3;
            uint64_t higher_digits = morton_index >> (digit_shift + 2);
            int p = (mix_bits(higher_digits ^ (0x55555555u * dimension)) >> 24) % 24;
            digit = permutations[p][digit];
            sample_index |= uint64_t(digit) << digit_shift;
        }
        if (pow_2_samples) {
            int digit = morton_index & 1;
            sample_index |= digit ^ (mix_bits((morton_index >> 1) ^ (0x55555555u * dimension)) & 1);
        }
        return sample_index;
    }

    int dimension = 0;
    int seed, log2_samples_per_pixel, n_base4_digits;
    uint64_t morton_index = 0;
};

// PTRenderSampler (sobol.h:235-248).  The PCG32 member is not used by small_pt without subsurface
// scattering, so only the Sobol part is kept.
struct PTRenderSampler
{
    PTRenderSampler(uint32_t full_w, uint32_t full_h, uint32_t px, uint32_t py, uint32_t spp, uint32_t sample_index,
                    uint32_t seed)
        : sobol((int)spp, (int)full_w, (int)full_h, (int)seed)
    {
        sobol.start_pixel((int)px, (int)py, (int)sample_index, 0);
    }
    OwenScrambledSobol02Morton sobol;
};

} // namespace oracle
