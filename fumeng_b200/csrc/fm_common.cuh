// Shared device/host helpers for the fumeng_b200 CUDA kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#define FM_HD __host__ __device__ __forceinline__
#define FM_D __device__ __forceinline__

namespace fm {

// Constants of the reference (src/engine/include/engine/common.h:53-56).  PI is the
// reference's own truncated value 3.14159265354, rounded to float.
constexpr float kPi = 3.14159265354f;
constexpr float kInvPi = float(1.0 / 3.14159265354);
constexpr float kEps = 1e-4f;
constexpr float kEpsPdf = 1e-20f;
constexpr float kRealMax = 3.402823466e+38f;

struct f3 {
    float x, y, z;
};

FM_HD f3 mk(float x, float y, float z) { return f3{x, y, z}; }
FM_HD f3 mk(float s) { return f3{s, s, s}; }
FM_HD f3 operator+(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
FM_HD f3 operator-(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
FM_HD f3 operator*(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }
FM_HD f3 operator/(f3 a, f3 b) { return f3{a.x / b.x, a.y / b.y, a.z / b.z}; }
FM_HD f3 operator*(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
FM_HD f3 operator*(float s, f3 a) { return f3{a.x * s, a.y * s, a.z * s}; }
FM_HD f3 operator/(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }
FM_HD f3 operator+(f3 a, float s) { return f3{a.x + s, a.y + s, a.z + s}; }
FM_HD f3 operator-(f3 a, float s) { return f3{a.x - s, a.y - s, a.z - s}; }
FM_HD f3 operator-(float s, f3 a) { return f3{s - a.x, s - a.y, s - a.z}; }
FM_HD f3 operator-(f3 a) { return f3{-a.x, -a.y, -a.z}; }
FM_HD f3& operator+=(f3& a, f3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
FM_HD f3& operator*=(f3& a, f3 b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; return a; }
FM_HD f3& operator*=(f3& a, float s) { a.x *= s; a.y *= s; a.z *= s; return a; }
FM_HD f3& operator/=(f3& a, float s) { a.x /= s; a.y /= s; a.z /= s; return a; }
FM_HD float comp(f3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

FM_HD float dot(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
FM_HD f3 cross(f3 a, f3 b)
{
    return f3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
FM_HD float length(f3 a) { return sqrtf(dot(a, a)); }
FM_HD f3 normalize(f3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
FM_HD float absdot(f3 a, f3 b) { return fabsf(dot(a, b)); }
FM_HD f3 fmin3(f3 a, f3 b) { return f3{fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
FM_HD f3 fmax3(f3 a, f3 b) { return f3{fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
FM_HD float clampf(float v, float lo, float hi) { return v > hi ? hi : (v < lo ? lo : v); }
FM_HD float luminance(f3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
FM_HD bool is_black(f3 c)
{
    // IsBlack (core/utils.h:85-97): zero or any negative component.
    if (c.x == 0.0f && c.y == 0.0f && c.z == 0.0f) return true;
    return c.x < 0.0f || c.y < 0.0f || c.z < 0.0f;
}

FM_HD f3 ld3(const float* p) { return f3{p[0], p[1], p[2]}; }
FM_HD void st3(float* p, f3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

// 3x4 affine transform, row-major: y = M[:, :3] x + M[:, 3].
struct Xf {
    float m[12];
};
FM_HD f3 xf_point(const Xf& t, f3 p)
{
    return f3{t.m[0] * p.x + t.m[1] * p.y + t.m[2] * p.z + t.m[3],
              t.m[4] * p.x + t.m[5] * p.y + t.m[6] * p.z + t.m[7],
              t.m[8] * p.x + t.m[9] * p.y + t.m[10] * p.z + t.m[11]};
}
FM_HD f3 xf_vec(const Xf& t, f3 v)
{
    return f3{t.m[0] * v.x + t.m[1] * v.y + t.m[2] * v.z, t.m[4] * v.x + t.m[5] * v.y + t.m[6] * v.z,
              t.m[8] * v.x + t.m[9] * v.y + t.m[10] * v.z};
}
// Normal transform with the transpose of the inverse linear part, given the inverse.
FM_HD f3 xf_normal_from_inv(const Xf& inv, f3 n)
{
    return f3{inv.m[0] * n.x + inv.m[4] * n.y + inv.m[8] * n.z, inv.m[1] * n.x + inv.m[5] * n.y + inv.m[9] * n.z,
              inv.m[2] * n.x + inv.m[6] * n.y + inv.m[10] * n.z};
}

// Monotonic float <-> uint encoding for atomicMin/atomicMax on floats.
FM_HD uint32_t f2ord(float f)
{
#ifdef __CUDA_ARCH__
    uint32_t u = __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
#endif
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
FM_HD float ord2f(uint32_t u)
{
    uint32_t v = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
#ifdef __CUDA_ARCH__
    return __uint_as_float(v);
#else
    float f;
    memcpy(&f, &v, 4);
    return f;
#endif
}

}  // namespace fm
