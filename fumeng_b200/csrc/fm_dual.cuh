// Forward-mode dual numbers for the adjoint renderer: a value with its partial
// derivatives with respect to the N material parameters of one shading point.
//
// The adjoint kernels differentiate BSDF values with respect to basecolor (r, g, b),
// metallic and roughness; every other quantity in a BSDF evaluation (directions,
// Fresnel terms of fixed IOR, the other material parameters) enters as a plain float.
#pragma once
#include "fm_common.cuh"

namespace fm {

template <int N>
struct Dual {
    float v;
    float d[N];
};

constexpr int kGradParams = 5;   // basecolor r, g, b, metallic, roughness
using D5 = Dual<kGradParams>;

template <int N>
FM_D Dual<N> dconst(float v)
{
    Dual<N> r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = 0.0f;
    return r;
}

template <int N>
FM_D Dual<N> dvar(float v, int which)
{
    Dual<N> r = dconst<N>(v);
    r.d[which] = 1.0f;
    return r;
}

FM_D float val(float x) { return x; }
template <int N>
FM_D float val(const Dual<N>& x)
{
    return x.v;
}

template <int N>
FM_D Dual<N> operator+(const Dual<N>& a, const Dual<N>& b)
{
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N>
FM_D Dual<N> operator+(const Dual<N>& a, float b)
{
    Dual<N> r = a;
    r.v += b;
    return r;
}
template <int N>
FM_D Dual<N> operator+(float a, const Dual<N>& b)
{
    return b + a;
}
template <int N>
FM_D Dual<N> operator-(const Dual<N>& a)
{
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N>
FM_D Dual<N> operator-(const Dual<N>& a, const Dual<N>& b)
{
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N>
FM_D Dual<N> operator-(const Dual<N>& a, float b)
{
    Dual<N> r = a;
    r.v -= b;
    return r;
}
template <int N>
FM_D Dual<N> operator-(float a, const Dual<N>& b)
{
    Dual<N> r;
    r.v = a - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -b.d[i];
    return r;
}
template <int N>
FM_D Dual<N> operator*(const Dual<N>& a, const Dual<N>& b)
{
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N>
FM_D Dual<N> operator*(const Dual<N>& a, float b)
{
    Dual<N> r;
    r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
    return r;
}
template <int N>
FM_D Dual<N> operator*(float a, const Dual<N>& b)
{
    return b * a;
}
template <int N>
FM_D Dual<N> operator/(const Dual<N>& a, const Dual<N>& b)
{
    Dual<N> r;
    const float inv = 1.0f / b.v;
    r.v = a.v * inv;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
}
template <int N>
FM_D Dual<N> operator/(const Dual<N>& a, float b)
{
    Dual<N> r;
    r.v = a.v / b;
    const float inv = 1.0f / b;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * inv;
    return r;
}
template <int N>
FM_D Dual<N> operator/(float a, const Dual<N>& b)
{
    Dual<N> r;
    r.v = a / b.v;
    const float k = -r.v / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = k * b.d[i];
    return r;
}
template <int N>
FM_D Dual<N> dsqrt(const Dual<N>& a)
{
    Dual<N> r;
    r.v = sqrtf(a.v);
    const float k = r.v > 0.0f ? 0.5f / r.v : 0.0f;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = k * a.d[i];
    return r;
}
FM_D float dsqrt(float a) { return sqrtf(a); }
// max(a, b) with b a constant floor (the derivative is zero where the floor applies)
template <int N>
FM_D Dual<N> dmax(const Dual<N>& a, float b)
{
    return a.v >= b ? a : dconst<N>(b);
}
FM_D float dmax(float a, float b) { return fmaxf(a, b); }

// Three-channel colour of duals.
struct DV3 {
    D5 x, y, z;
};

FM_D DV3 dv3(const D5& a) { return DV3{a, a, a}; }
FM_D DV3 dv3(f3 a) { return DV3{dconst<kGradParams>(a.x), dconst<kGradParams>(a.y), dconst<kGradParams>(a.z)}; }
FM_D f3 val(const DV3& a) { return f3{a.x.v, a.y.v, a.z.v}; }
FM_D DV3 operator+(const DV3& a, const DV3& b) { return DV3{a.x + b.x, a.y + b.y, a.z + b.z}; }
FM_D DV3 operator+(const DV3& a, f3 b) { return DV3{a.x + b.x, a.y + b.y, a.z + b.z}; }
FM_D DV3 operator-(const DV3& a, const DV3& b) { return DV3{a.x - b.x, a.y - b.y, a.z - b.z}; }
FM_D DV3 operator-(f3 a, const DV3& b) { return DV3{a.x - b.x, a.y - b.y, a.z - b.z}; }
FM_D DV3 operator*(const DV3& a, const D5& s) { return DV3{a.x * s, a.y * s, a.z * s}; }
FM_D DV3 operator*(const D5& s, const DV3& a) { return a * s; }
FM_D DV3 operator*(const DV3& a, float s) { return DV3{a.x * s, a.y * s, a.z * s}; }
FM_D DV3 operator*(float s, const DV3& a) { return a * s; }
FM_D DV3 operator*(const DV3& a, f3 b) { return DV3{a.x * b.x, a.y * b.y, a.z * b.z}; }
FM_D DV3 operator/(const DV3& a, const D5& s) { return DV3{a.x / s, a.y / s, a.z / s}; }
FM_D DV3 operator/(const DV3& a, float s) { return DV3{a.x / s, a.y / s, a.z / s}; }
FM_D D5 luminance(const DV3& c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
// (1 - t) a + t b
FM_D DV3 lerp3(const DV3& a, const DV3& b, const D5& t) { return (1.0f - t) * a + t * b; }
FM_D DV3 lerp3(f3 a, const DV3& b, float t) { return dv3(a * (1.0f - t)) + t * b; }
FM_D DV3 lerp3(const DV3& a, const DV3& b, float t) { return (1.0f - t) * a + t * b; }
FM_D D5 lerpf(float a, float b, const D5& t) { return (1.0f - t) * a + t * b; }

}  // namespace fm
