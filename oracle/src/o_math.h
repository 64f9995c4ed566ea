// ORACLE (test infrastructure only).  Float vector helpers with the evaluation order of the
// reference's Eigen expressions (left-to-right sums, plain cross products, normalized() =
// v / sqrt(squaredNorm) when the norm is positive), plus the scalar helpers of maths.h.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace oracle
{

inline constexpr float pi = 3.14159265359f;     // maths.h:58
inline constexpr float two_pi = 6.28318530718f; // maths.h:59
inline constexpr float half_pi = pi / 2.0f;
inline constexpr float inv_pi = 1.0f / pi;
inline constexpr float inf = std::numeric_limits<float>::infinity();

struct V3
{
    float x = 0, y = 0, z = 0;
    V3() = default;
    V3(float x, float y, float z) : x(x), y(y), z(z) {}
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3 &operator+=(V3 &a, V3 b) { return a = a + b; }
inline V3 &operator-=(V3 &a, V3 b) { return a = a - b; }
inline V3 &operator*=(V3 &a, V3 b) { return a = a * b; }
inline V3 &operator*=(V3 &a, float s) { return a = a * s; }
inline V3 &operator/=(V3 &a, float s) { return a = a / s; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float sqnorm(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3 normalized(V3 a)
{
    float n2 = sqnorm(a);
    if (n2 > 0.0f) {
        float n = std::sqrt(n2);
        return {a.x / n, a.y / n, a.z / n};
    }
    return a;
}
inline float norm(V3 a) { return std::sqrt(sqnorm(a)); }
inline float max_coeff(V3 a) { return std::max(std::max(a.x, a.y), a.z); }
inline bool is_zero(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
inline bool all_finite(V3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
inline V3 cwise_min(V3 a, float c) { return {std::min(a.x, c), std::min(a.y, c), std::min(a.z, c)}; }
inline float sqr(float x) { return x * x; }
inline float saturate(float x) { return std::clamp(x, 0.0f, 1.0f); }
inline float luminance(V3 c) { return 0.212671f * c.x + 0.715160f * c.y + 0.072169f * c.z; }
inline float sgn(float x) { return float((0.0f < x) - (x < 0.0f)); }
inline float safe_sqrt(float x) { return std::sqrt(std::max(0.0f, x)); }
inline float safe_pow(float a, float b)
{
    if (a == 0.0 && b == 0.0f)
        return 0.0f;
    return std::pow(a, b);
}
// Eigen lerp(a, b, t) = (1 - t) * a + t * b (maths.h:681-697)
inline V3 lerp3(V3 a, V3 b, float t) { return (1.0f - t) * a + t * b; }
inline float power_heur(float pf, float pg)
{
    float f2 = pf * pf, g2 = pg * pg;
    return f2 / (f2 + g2);
}
inline float int_as_float(int i)
{
    float f;
    std::memcpy(&f, &i, 4);
    return f;
}
inline int float_as_int(float f)
{
    int i;
    std::memcpy(&i, &f, 4);
    return i;
}

// offset_ray (ray.h:66-81)
inline V3 offset_ray(V3 p, V3 n)
{
    constexpr float origin = 1.0f / 32.0f;
    constexpr float float_scale = 1.0f / 65536.0f;
    constexpr float int_scale = 256.0f;
    int ox = (int)(int_scale * n.x), oy = (int)(int_scale * n.y), oz = (int)(int_scale * n.z);
    V3 pi_(int_as_float(float_as_int(p.x) + ((p.x < 0) ? -ox : ox)),
           int_as_float(float_as_int(p.y) + ((p.y < 0) ? -oy : oy)),
           int_as_float(float_as_int(p.z) + ((p.z < 0) ? -oz : oz)));
    return V3(std::fabs(p.x) < origin ? p.x + float_scale * n.x : pi_.x,
              std::fabs(p.y) < origin ? p.y + float_scale * n.y : pi_.y,
              std::fabs(p.z) < origin ? p.z + float_scale * n.z : pi_.z);
}

struct Frame
{
    V3 t{1, 0, 0}, b{0, 1, 0}, n{0, 0, 1};
    V3 to_local(V3 w) const { return {dot(t, w), dot(b, w), dot(n, w)}; }
    V3 to_world(V3 w) const { return t * w.x + b * w.y + n * w.z; }
};

// 4x4 row-major matrix applied to a point (w = 1), Eigen mat * vec4 order.
inline void mat_vec4(const float *m, V3 p, float out[4])
{
    for (int r = 0; r < 4; ++r)
        out[r] = m[4 * r + 0] * p.x + m[4 * r + 1] * p.y + m[4 * r + 2] * p.z + m[4 * r + 3] * 1.0f;
}
inline V3 point_hdiv(const float *m, V3 p)
{
    float o[4];
    mat_vec4(m, p, o);
    return {o[0] / o[3], o[1] / o[3], o[2] / o[3]};
}
inline V3 transform_dir(const float *m, V3 v)
{
    return {m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z,
            m[8] * v.x + m[9] * v.y + m[10] * v.z};
}

} // namespace oracle
