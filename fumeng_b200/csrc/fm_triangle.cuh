// Ray/primitive intersection with the reference's exact float arithmetic.
//
// Closest-hit primitive IDs must match the reference's built-in BVH bit for bit, so the
// triangle test performs the same IEEE float operations in the same order as
// triangle_func::IntersectTriangle (src/engine/src/geometry/triangle.cpp:25-94), with
// every multiply and add written as an explicitly rounded intrinsic so that the compiler
// cannot contract them into FMAs.  The double-precision fallback of triangle.cpp:61-66
// is reproduced with explicitly rounded double operations.
//
// The main-axis choice reproduces triangle.cpp:13-18 as the reference compiles: the
// unqualified `abs` there binds to the C library's int abs(int), so each direction
// component is truncated toward zero before the comparison (so the test almost always
// permutes z to the main axis).  The oracle's known-answer test pins this binding.
#pragma once
#include "fm_common.cuh"

namespace fm {

// Per-ray constants of the watertight test (permutation and shear).
struct RayPre {
    f3 o;            // origin
    int kx, ky, kz;  // permutation: (dir[kx], dir[ky], dir[kz])
    float sx, sy, sz;
};

FM_D int trunc_abs(float v)
{
    // (int)v then abs(): float -> int conversion truncates toward zero.
    const int i = __float2int_rz(v);
    return i < 0 ? -i : i;
}

FM_D RayPre ray_pre(f3 o, f3 d)
{
    RayPre p;
    p.o = o;
    const int a0 = trunc_abs(d.x), a1 = trunc_abs(d.y), a2 = trunc_abs(d.z);
    int az;
    if (a0 > a1 && a0 > a2)
        az = 0;
    else
        az = a1 > a2 ? 1 : 2;
    // A main-axis component of zero (or so small that 1/dz overflows) makes the shear
    // infinite and every edge function NaN; the reference then reports NaN hits.  Its
    // double build practically never draws such a ray, but float sampling does (a
    // cosine-hemisphere sample at an axis-aligned wall has d.z == 0 exactly about once
    // in 2^24 draws), so those rays use the axis of largest magnitude instead.  Rays
    // with |dz| >= 1e-30 keep the reference's choice and its results bit for bit.
    if (!(fabsf(comp(d, az)) >= 1e-30f)) {
        const float m0 = fabsf(d.x), m1 = fabsf(d.y), m2 = fabsf(d.z);
        az = (m0 >= m1 && m0 >= m2) ? 0 : (m1 >= m2 ? 1 : 2);
    }
    const int ax = (az + 1) % 3;
    const int ay = (ax + 1) % 3;
    p.kx = ax;
    p.ky = ay;
    p.kz = az;
    const float dx = comp(d, ax), dy = comp(d, ay), dz = comp(d, az);
    p.sx = __fdiv_rn(-dx, dz);
    p.sy = __fdiv_rn(-dy, dz);
    p.sz = __fdiv_rn(1.0f, dz);
    return p;
}

FM_D float edge_double(float ax, float ay, float bx, float by)
{
    // (real)((double)ax * (double)by - (double)ay * (double)bx)
    return __double2float_rn(__dsub_rn(__dmul_rn((double)ax, (double)by), __dmul_rn((double)ay, (double)bx)));
}

// triangle_func::IntersectTriangle.  Returns true on a hit with t in (tmin, tmax).  The
// reference's rejection test (t <= tmin || t >= tmax) lets a NaN t through; here a NaN
// t is rejected as well (it arises only from degenerate input, never on a ray the
// reference handles with finite arithmetic).
template <bool IDENTITY>
FM_D bool intersect_triangle_p(const RayPre& r, f3 v0, f3 v1, f3 v2, float tmin, float tmax, float& t_out,
                               float& b0, float& b1, float& b2)
{
    // translate
    v0 = f3{__fsub_rn(v0.x, r.o.x), __fsub_rn(v0.y, r.o.y), __fsub_rn(v0.z, r.o.z)};
    v1 = f3{__fsub_rn(v1.x, r.o.x), __fsub_rn(v1.y, r.o.y), __fsub_rn(v1.z, r.o.z)};
    v2 = f3{__fsub_rn(v2.x, r.o.x), __fsub_rn(v2.y, r.o.y), __fsub_rn(v2.z, r.o.z)};
    // permute
    float p0x = IDENTITY ? v0.x : comp(v0, r.kx), p0y = IDENTITY ? v0.y : comp(v0, r.ky);
    float p0z = IDENTITY ? v0.z : comp(v0, r.kz);
    float p1x = IDENTITY ? v1.x : comp(v1, r.kx), p1y = IDENTITY ? v1.y : comp(v1, r.ky);
    float p1z = IDENTITY ? v1.z : comp(v1, r.kz);
    float p2x = IDENTITY ? v2.x : comp(v2, r.kx), p2y = IDENTITY ? v2.y : comp(v2, r.ky);
    float p2z = IDENTITY ? v2.z : comp(v2, r.kz);
    // shear
    p0x = __fadd_rn(p0x, __fmul_rn(r.sx, p0z));
    p0y = __fadd_rn(p0y, __fmul_rn(r.sy, p0z));
    p1x = __fadd_rn(p1x, __fmul_rn(r.sx, p1z));
    p1y = __fadd_rn(p1y, __fmul_rn(r.sy, p1z));
    p2x = __fadd_rn(p2x, __fmul_rn(r.sx, p2z));
    p2y = __fadd_rn(p2y, __fmul_rn(r.sy, p2z));
    // edge functions
    float e0 = __fsub_rn(__fmul_rn(p1x, p2y), __fmul_rn(p1y, p2x));
    float e1 = __fsub_rn(__fmul_rn(p2x, p0y), __fmul_rn(p2y, p0x));
    float e2 = __fsub_rn(__fmul_rn(p0x, p1y), __fmul_rn(p0y, p1x));
    if (e0 == 0.0f || e1 == 0.0f || e2 == 0.0f) {
        e0 = edge_double(p1x, p1y, p2x, p2y);
        e1 = edge_double(p2x, p2y, p0x, p0y);
        e2 = edge_double(p0x, p0y, p1x, p1y);
    }
    if ((e0 < 0 || e1 < 0 || e2 < 0) && (e0 > 0 || e1 > 0 || e2 > 0)) return false;
    const float det = __fadd_rn(__fadd_rn(e0, e1), e2);
    if (det == 0) return false;
    p0z = __fmul_rn(p0z, r.sz);
    p1z = __fmul_rn(p1z, r.sz);
    p2z = __fmul_rn(p2z, r.sz);
    const float inv_det = __fdiv_rn(1.0f, det);
    const float t = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(e0, p0z), __fmul_rn(e1, p1z)), __fmul_rn(e2, p2z)), inv_det);
    if (t <= tmin || t >= tmax || t != t) return false;
    t_out = t;
    b0 = __fmul_rn(e0, inv_det);
    b1 = __fmul_rn(e1, inv_det);
    b2 = __fmul_rn(e2, inv_det);
    return true;
}

// The permutation is the identity (x, y, z) whenever z is the main axis, which the
// truncating main-axis choice makes it for almost every ray; that case skips the
// per-component selects.
FM_D bool intersect_triangle(const RayPre& r, f3 v0, f3 v1, f3 v2, float tmin, float tmax, float& t_out,
                             float& b0, float& b1, float& b2)
{
    if (r.kz == 2) return intersect_triangle_p<true>(r, v0, v1, v2, tmin, tmax, t_out, b0, b1, b2);
    return intersect_triangle_p<false>(r, v0, v1, v2, tmin, tmax, t_out, b0, b1, b2);
}

// Sphere::IntersectSphere (geometry/sphere.cpp:91-129, GetCoef :206-212): the ray is
// taken to object space (not renormalized, so t is shared), the quadratic is solved
// without the robust form, and the nearer root inside the inclusive range [tmin, tmax]
// is returned.  Every operation is explicitly rounded in the reference's order
// (SquareSum and glm::dot left to right, b*b - (4a)*c, 0.5/a), so no multiply-add is
// contracted and the result equals the reference's float build bit for bit whenever the
// object-space ray does (always for translation-only transforms, whose world-to-object
// step is one rounded subtraction per origin component and exact for the direction).
FM_D bool intersect_sphere(const Xf& world_to_object, float radius, f3 o, f3 d, float tmin, float tmax,
                           float& t_out)
{
    const f3 ol = xf_point(world_to_object, o);
    const f3 dl = xf_vec(world_to_object, d);
    const float a = __fadd_rn(__fadd_rn(__fmul_rn(dl.x, dl.x), __fmul_rn(dl.y, dl.y)), __fmul_rn(dl.z, dl.z));
    const float b =
        __fmul_rn(2.0f, __fadd_rn(__fadd_rn(__fmul_rn(dl.x, ol.x), __fmul_rn(dl.y, ol.y)), __fmul_rn(dl.z, ol.z)));
    const float c = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(ol.x, ol.x), __fmul_rn(ol.y, ol.y)), __fmul_rn(ol.z, ol.z)),
                              __fmul_rn(radius, radius));
    float delta = __fsub_rn(__fmul_rn(b, b), __fmul_rn(__fmul_rn(4.0f, a), c));
    if (delta < 0) return false;
    delta = __fsqrt_rn(delta);
    const float inv2a = __fdiv_rn(0.5f, a);
    const float t0 = __fmul_rn(__fsub_rn(-b, delta), inv2a);
    const float t1 = __fmul_rn(__fadd_rn(-b, delta), inv2a);
    if (t0 >= tmin && t0 <= tmax) {
        t_out = t0;
        return true;
    }
    if (t1 >= tmin && t1 <= tmax) {
        t_out = t1;
        return true;
    }
    return false;
}

}  // namespace fm
