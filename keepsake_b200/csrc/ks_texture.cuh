// Textured shader fields, normal maps and opacity maps on the device.
//
// Textures (Texture, texture.h:43-65) are uploaded converted to linear float texels (4 per texel,
// Texture::fetch_as_float, texture.cpp:403-460: u8 / u16 / f32 in linear or sRGB encoding), so a
// lookup reads the values the reference's fetch returns.  A binding is one TextureField
// (shader_field.h:38-86): flip_v, uv_scale / uv_offset, a sampler (texture.cpp:520-677: nearest,
// bilinear or bicubic at level 0, repeat or clamp per axis), swizzle and scale; the textures have one
// level, so the samplers' level selection (texture.cpp:587-627) always picks level 0.  The lookups
// run on the device (shading) and on the host (the importance of textured emitters).
#pragma once
#include "ks_math.cuh"

namespace ksb
{

struct TexInfo
{
    uint32_t offset; // first texel in the scene's texel array
    int w, h, ch;
};

// One texture bound to one material (ks_texture_binding), with the cubic kernel's coefficients.
struct BindingGPU
{
    int tex, field, filter, wrap_u, wrap_v, flip_v;
    int swz[4];
    float uv_scale[2], uv_offset[2], scale[4];
    float ca[4], cb[4]; // CubicSampler kernel (texture.h:91-121)
    int space, range01; // NormalMap
    float strength;
    float nrm[9]; // world-space normal maps: the 3x3 inverse transpose of to_world
};

// wrap (texture.cpp:520-531)
KS_HD int tex_wrap(int x, int dim, int clamp)
{
    if (clamp)
        return x < 0 ? 0 : (x > dim - 1 ? dim - 1 : x);
    const int r = x % dim;
    return r < 0 ? r + dim : r;
}

KS_HD float4 texel(const float4 *texels, const TexInfo &t, int x, int y)
{
#ifdef __CUDA_ARCH__
    return __ldg(&texels[t.offset + (size_t)y * t.w + x]);
#else
    return texels[t.offset + (size_t)y * t.w + x];
#endif
}

KS_HD float4 f4_axpy(float a, float4 x, float4 y) { return make_float4(a * x.x + y.x, a * x.y + y.y, a * x.z + y.z, a * x.w + y.w); }

// TextureSampler::bilinear (texture.cpp:541-573) at level 0
KS_HD float4 tex_bilinear(const float4 *texels, const TexInfo &t, const BindingGPU &b, float ux, float uy)
{
    float u = ux * t.w - 0.5f, v = uy * t.h - 0.5f;
    int u0 = (int)floorf(u), v0 = (int)floorf(v);
    float du = u - u0, dv = v - v0;
    u0 = tex_wrap(u0, t.w, b.wrap_u);
    v0 = tex_wrap(v0, t.h, b.wrap_v);
    int u1 = tex_wrap(u0 + 1, t.w, b.wrap_u), v1 = tex_wrap(v0 + 1, t.h, b.wrap_v);
    float w00 = (1 - du) * (1 - dv), w10 = du * (1 - dv), w01 = (1 - du) * dv, w11 = du * dv;
    const float4 a = texel(texels, t, u0, v0), c = texel(texels, t, u1, v0), d = texel(texels, t, u0, v1),
                 e = texel(texels, t, u1, v1);
    return make_float4(w00 * a.x + w10 * c.x + w01 * d.x + w11 * e.x, w00 * a.y + w10 * c.y + w01 * d.y + w11 * e.y,
                       w00 * a.z + w10 * c.z + w01 * d.z + w11 * e.z, w00 * a.w + w10 * c.w + w01 * d.w + w11 * e.w);
}

// NearestSampler (texture.cpp:575-585)
KS_HD float4 tex_nearest(const float4 *texels, const TexInfo &t, const BindingGPU &b, float ux, float uy)
{
    int u0 = (int)floorf(ux * t.w - 0.5f), v0 = (int)floorf(uy * t.h - 0.5f);
    return texel(texels, t, tex_wrap(u0, t.w, b.wrap_u), tex_wrap(v0, t.h, b.wrap_v));
}

// spline / CubicSampler::bicubic (texture.cpp:629-677) at level 0
KS_HD float cubic_weight(const float c[4], float x) { return c[0] * (x * x * x) + c[1] * (x * x) + c[2] * x + c[3]; }

KS_HD float4 tex_bicubic(const float4 *texels, const TexInfo &t, const BindingGPU &b, float ux, float uy)
{
    float u = ux * t.w - 0.5f, v = uy * t.h - 0.5f;
    int u0 = (int)floorf(u), v0 = (int)floorf(v);
    float du = u - u0, dv = v - v0;
    const float ax[4] = {cubic_weight(b.cb, du + 1.0f), cubic_weight(b.ca, du), cubic_weight(b.ca, 1.0f - du),
                         cubic_weight(b.cb, 2.0f - du)};
    const float ay[4] = {cubic_weight(b.cb, dv + 1.0f), cubic_weight(b.ca, dv), cubic_weight(b.ca, 1.0f - dv),
                         cubic_weight(b.cb, 2.0f - dv)};
    float4 out = make_float4(0, 0, 0, 0);
    for (int y = 0; y < 4; ++y) {
        const int vy = tex_wrap(v0 + y - 1, t.h, b.wrap_v);
        float4 row = make_float4(0, 0, 0, 0);
        for (int x = 0; x < 4; ++x)
            row = f4_axpy(ax[x], texel(texels, t, tex_wrap(u0 + x - 1, t.w, b.wrap_u), vy), row);
        out = f4_axpy(ay[y], row, out);
    }
    return out;
}

// TextureField::operator() (shader_field.h:61-80): the field's value (4 channels, unused ones 0)
KS_HD float4 field_eval(const float4 *texels, const TexInfo *infos, const BindingGPU &b, float u, float v)
{
    float fu = u, fv = b.flip_v ? 1.0f - v : v;
    fu = fu * b.uv_scale[0] + b.uv_offset[0];
    fv = fv * b.uv_scale[1] + b.uv_offset[1];
    const TexInfo t = infos[b.tex];
    float4 s = b.filter == 0 ? tex_nearest(texels, t, b, fu, fv)
                             : (b.filter == 1 ? tex_bilinear(texels, t, b, fu, fv) : tex_bicubic(texels, t, b, fu, fv));
    const float sv[4] = {s.x, t.ch > 1 ? s.y : 0.0f, t.ch > 2 ? s.z : 0.0f, t.ch > 3 ? s.w : 0.0f};
    float o[4];
#pragma unroll
    for (int c = 0; c < 4; ++c)
        o[c] = (b.swz[c] >= 0 && b.swz[c] < t.ch ? sv[b.swz[c]] : 0.0f) * b.scale[c];
    return make_float4(o[0], o[1], o[2], o[3]);
}

} // namespace ksb
