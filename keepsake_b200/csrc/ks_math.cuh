// Device-side scalar/vector helpers for the B200 small_pt path.
//
// The translation units of the bit-exact parts (sampler, camera rays, SBVH build and traversal) are
// compiled with -fmad=false and IEEE division/sqrt, so a float expression there rounds exactly like
// the same expression in the reference's x86-64 SSE host build; the shading unit (ks_shade.cu) uses
// fast math and is checked statistically.  Where the reference relies on a fused multiply-add (ksc::difference_of_products,
// cuda/math.cuh:189-195) it is written out with fmaf() explicitly.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define KS_HD __host__ __device__ __forceinline__
#define KS_D __device__ __forceinline__
// Large shading functions called from several places: kept out of line so that the shading
// kernel's code fits the instruction cache (KS_SHADE_INLINE=1 inlines them).
#if defined(KS_SHADE_INLINE) && KS_SHADE_INLINE
#define KS_BIG __device__ __forceinline__
#else
#define KS_BIG __device__ __noinline__
#endif

namespace ksb
{

// Constants as spelled in maths.h:58-64 (rounded to float by the compiler exactly the same way).
constexpr float kPi = 3.14159265359f;
constexpr float kTwoPi = 6.28318530718f;
constexpr float kHalfPi = kPi / 2.0f;
constexpr float kInvPi = 1.0f / kPi;
constexpr float kInf = __builtin_huge_valf();
// std::nextafter(1.0f, -inf) (maths.h:65)
constexpr float kOneMinusEps = 0x1.fffffep-1f;

struct f3
{
    float x, y, z;
};

KS_HD f3 mk(float x, float y, float z) { return f3{x, y, z}; }
KS_HD f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
KS_HD f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
KS_HD f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
KS_HD f3 operator*(f3 a, f3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
KS_HD f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
KS_HD f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
KS_HD f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
KS_HD f3 operator/(f3 a, f3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
KS_HD f3 &operator+=(f3 &a, f3 b)
{
    a = a + b;
    return a;
}
KS_HD f3 &operator*=(f3 &a, f3 b)
{
    a = a * b;
    return a;
}
KS_HD f3 &operator*=(f3 &a, float s)
{
    a = a * s;
    return a;
}
KS_HD f3 &operator/=(f3 &a, float s)
{
    a = a / s;
    return a;
}
KS_HD float get(f3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
KS_HD void set(f3 &v, int i, float s)
{
    if (i == 0)
        v.x = s;
    else if (i == 1)
        v.y = s;
    else
        v.z = s;
}
// Eigen-style dot: left-to-right sum of products.
KS_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
KS_HD float sqnorm(f3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
// Plain cross product as Eigen computes it (a.y*b.z - a.z*b.y, ...).
KS_HD f3 cross(f3 a, f3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
KS_HD f3 normalize(f3 a)
{
    float n2 = sqnorm(a);
    if (n2 > 0.0f) {
        float n = sqrtf(n2);
        return {a.x / n, a.y / n, a.z / n};
    }
    return a;
}
KS_HD float max3(f3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
KS_HD bool is_zero(f3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
KS_HD f3 cwise_min(f3 a, float c) { return {a.x < c ? a.x : c, a.y < c ? a.y : c, a.z < c ? a.z : c}; }
KS_HD float sqr(float x) { return x * x; }
KS_HD float clampf(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); }
KS_HD float saturate(float v) { return clampf(v, 0.0f, 1.0f); }
// std::lerp(a, b, t) for finite a, b (libstdc++ algorithm, P0811): exact at t=0 and t=1, monotonic.
KS_HD float std_lerp(float a, float b, float t)
{
    if ((a <= 0 && b >= 0) || (a >= 0 && b <= 0))
        return t * b + (1 - t) * a;
    if (t == 1)
        return b;
    const float x = a + t * (b - a);
    return (t > 1) == (b > a) ? (b < x ? x : b) : (x < b ? x : b);
}
// Affine transform of a point / direction by a row-major 3x4 matrix, the same float arithmetic on
// host and device.
KS_HD f3 xf_point(const float *m, f3 p)
{
    return mk(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
              m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
}
KS_HD f3 xf_dir(const float *m, f3 d)
{
    return mk(m[0] * d.x + m[1] * d.y + m[2] * d.z, m[4] * d.x + m[5] * d.y + m[6] * d.z,
              m[8] * d.x + m[9] * d.y + m[10] * d.z);
}

// luminance() weights (maths.h:675-679)
KS_HD float luminance(f3 c) { return 0.212671f * c.x + 0.715160f * c.y + 0.072169f * c.z; }
KS_HD float fsign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

} // namespace ksb
