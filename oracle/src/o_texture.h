// ORACLE (test infrastructure only).  Restatement of keepsake's textures as the small_pt path reads
// them: Texture::fetch_as_float (texture.cpp:403-460) of u8 / u16 / f32 texels in linear or sRGB
// encoding (srgb_to_linear, maths.h:631-638; the 8-bit table texture.cpp:369-401 is that curve in
// double precision), wrap (texture.cpp:520-531), NearestSampler (:575-585), TextureSampler::bilinear
// (:541-573), CubicSampler::bicubic and spline (:629-677) on textures of one level, TextureField
// (shader_field.h:38-86), NormalMap::sample / apply (normal_map.cpp:9-40) and OpacityMap::eval /
// stochastic_test (opacity_map.cpp:6-30) with hash_float of the ray (hash.h:140-258).
#pragma once
#include "../../include/ks_b200.h"
#include "o_math.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace oracle
{

struct Texture
{
    int w = 0, h = 0, ch = 0;
    std::vector<float> texels; // ch floats per texel, as fetch_as_float returns them

    explicit Texture(const ks_texture_desc &t) : w((int)t.width), h((int)t.height), ch((int)t.channels)
    {
        const size_t n = (size_t)w * h * ch;
        texels.resize(n);
        for (size_t k = 0; k < n; ++k) {
            float f;
            if (t.format == 0) {
                const uint8_t u = ((const uint8_t *)t.texels)[k];
                if (t.srgb) {
                    const double c = u / 255.0;
                    f = (float)(c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4));
                } else {
                    f = (float)u / 255.0f;
                }
            } else if (t.format == 1) {
                f = (float)((const uint16_t *)t.texels)[k] / 65535.0f;
                if (t.srgb)
                    f = srgb_to_linear(f);
            } else {
                f = ((const float *)t.texels)[k];
                if (t.srgb)
                    f = srgb_to_linear(f);
            }
            texels[k] = f;
        }
    }
    static float srgb_to_linear(float x)
    {
        if (x < 0.04045f)
            return x / 12.92f;
        return std::pow((x + 0.055f) / 1.055f, 2.4f);
    }
    void fetch(int x, int y, float out[4]) const
    {
        for (int c = 0; c < 4; ++c)
            out[c] = c < ch ? texels[((size_t)y * w + x) * ch + c] : 0.0f;
    }
};

inline int tex_mod(int a, int b)
{
    int r = a % b;
    return r < 0 ? r + b : r;
}

inline int tex_wrap(int x, int dim, int clamp) { return clamp ? std::clamp(x, 0, dim - 1) : tex_mod(x, dim); }

struct Binding
{
    ks_texture_binding b;
    float ca[4], cb[4];

    explicit Binding(const ks_texture_binding &in) : b(in)
    {
        // CubicSampler::CubicSampler (texture.h:91-121)
        static const double ca_[3][4] = {{21.0, -36.0, 0.0, 16.0}, {3.0, -6.0, 0.0, 4.0}, {3.0, -5.0, 0.0, 2.0}};
        static const double cb_[3][4] = {{-7.0, 36.0, -60.0, 32.0}, {-1.0, 6.0, -12.0, 8.0}, {-1.0, 5.0, -8.0, 4.0}};
        static const double div[3] = {18.0, 6.0, 2.0};
        for (int k = 0; k < 4; ++k) {
            ca[k] = (float)(ca_[b.cubic_kernel][k] / div[b.cubic_kernel]);
            cb[k] = (float)(cb_[b.cubic_kernel][k] / div[b.cubic_kernel]);
        }
    }

    void nearest(const Texture &t, float ux, float uy, float out[4]) const
    {
        float u = ux * t.w - 0.5f, v = uy * t.h - 0.5f;
        t.fetch(tex_wrap((int)std::floor(u), t.w, b.wrap_u), tex_wrap((int)std::floor(v), t.h, b.wrap_v), out);
    }
    void bilinear(const Texture &t, float ux, float uy, float out[4]) const
    {
        float u = ux * t.w - 0.5f, v = uy * t.h - 0.5f;
        int u0 = (int)std::floor(u), v0 = (int)std::floor(v);
        float du = u - u0, dv = v - v0;
        u0 = tex_wrap(u0, t.w, b.wrap_u);
        v0 = tex_wrap(v0, t.h, b.wrap_v);
        int u1 = tex_wrap(u0 + 1, t.w, b.wrap_u), v1 = tex_wrap(v0 + 1, t.h, b.wrap_v);
        float w00 = (1 - du) * (1 - dv), w10 = du * (1 - dv), w01 = (1 - du) * dv, w11 = du * dv;
        float a[4], c[4], d[4], e[4];
        t.fetch(u0, v0, a);
        t.fetch(u1, v0, c);
        t.fetch(u0, v1, d);
        t.fetch(u1, v1, e);
        for (int i = 0; i < 4; ++i)
            out[i] = w00 * a[i] + w10 * c[i] + w01 * d[i] + w11 * e[i];
    }
    static float weight(const float c[4], float x) { return c[0] * (x * x * x) + c[1] * (x * x) + c[2] * x + c[3]; }
    void bicubic(const Texture &t, float ux, float uy, float out[4]) const
    {
        float u = ux * t.w - 0.5f, v = uy * t.h - 0.5f;
        int u0 = (int)std::floor(u), v0 = (int)std::floor(v);
        float du = u - u0, dv = v - v0;
        const float ax[4] = {weight(cb, du + 1.0f), weight(ca, du), weight(ca, 1.0f - du), weight(cb, 2.0f - du)};
        const float ay[4] = {weight(cb, dv + 1.0f), weight(ca, dv), weight(ca, 1.0f - dv), weight(cb, 2.0f - dv)};
        float rows[4][4];
        for (int y = 0; y < 4; ++y) {
            float cols[4][4];
            for (int x = 0; x < 4; ++x)
                t.fetch(tex_wrap(u0 + x - 1, t.w, b.wrap_u), tex_wrap(v0 + y - 1, t.h, b.wrap_v), cols[x]);
            for (int i = 0; i < 4; ++i)
                rows[y][i] = cols[0][i] * ax[0] + cols[1][i] * ax[1] + cols[2][i] * ax[2] + cols[3][i] * ax[3];
        }
        for (int i = 0; i < 4; ++i)
            out[i] = rows[0][i] * ay[0] + rows[1][i] * ay[1] + rows[2][i] * ay[2] + rows[3][i] * ay[3];
    }
    // TextureField::operator() (shader_field.h:61-80)
    void eval(const Texture &t, float u, float v, float out[4]) const
    {
        float fu = u, fv = b.flip_v ? 1.0f - v : v;
        fu = fu * b.uv_scale[0] + b.uv_offset[0];
        fv = fv * b.uv_scale[1] + b.uv_offset[1];
        float s[4];
        if (b.filter == 0)
            nearest(t, fu, fv, s);
        else if (b.filter == 1)
            bilinear(t, fu, fv, s);
        else
            bicubic(t, fu, fv, s);
        for (int c = 0; c < 4; ++c)
            out[c] = (b.swizzle[c] >= 0 && b.swizzle[c] < t.ch ? s[b.swizzle[c]] : 0.0f) * b.scale[c];
    }
};

// hash_float(ro, rd) (hash.h:140-258): murmur_hash_64A of the 24 bytes of the two vectors, seed 0,
// its low 32 bits times 2^-32
inline float hash_float_ray(V3 ro, V3 rd)
{
    const float f[6] = {ro.x, ro.y, ro.z, rd.x, rd.y, rd.z};
    uint64_t k[3];
    std::memcpy(k, f, 24);
    const uint64_t m = 0xc6a4a7935bd1e995ull;
    const int r = 47;
    uint64_t h = 0 ^ (24 * m);
    for (int i = 0; i < 3; ++i) {
        uint64_t x = k[i];
        x *= m;
        x ^= x >> r;
        x *= m;
        h ^= x;
        h *= m;
    }
    h ^= h >> r;
    h *= m;
    h ^= h >> r;
    return uint32_t(h) * 0x1p-32f;
}

} // namespace oracle
