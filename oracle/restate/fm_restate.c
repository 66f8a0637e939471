/*
 * CPU restatement of the reference's ray-query arithmetic in plain C.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; never linked into the product).  Needs no
 * reference sources, so it also builds on machines without them.  Validated against the
 * compiled reference (oracle/_ref/libfmref_f.so) by tests/test_oracle.py.
 *
 * Compile with -ffp-contract=off (oracle/Makefile) so that no multiply-add is fused,
 * matching a stock x86-64 build of the reference.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

/* triangle_func::GetMaxAxis (src/engine/src/geometry/triangle.cpp:13-18) as the
 * reference compiles it: the unqualified abs is the C library's int abs(int), so each
 * component is truncated toward zero first. */
int fmo_get_max_axis(float x, float y, float z)
{
    const int ax = abs((int)x), ay = abs((int)y), az = abs((int)z);
    if (ax > ay && ax > az) return 0;
    return ay > az ? 1 : 2;
}

static float comp3(const float* v, int i) { return v[i]; }

/* triangle_func::IntersectTriangle (triangle.cpp:25-94).
 * ray: ox oy oz tmin dx dy dz tmax; v: v0 v1 v2.  Returns 1 on a hit. */
int fmo_intersect_triangle(const float* ray, const float* v, float* t_out, float* bc)
{
    const float o[3] = {ray[0], ray[1], ray[2]};
    const float d[3] = {ray[4], ray[5], ray[6]};
    const float tmin = ray[3], tmax = ray[7];
    float p0[3], p1[3], p2[3];
    for (int k = 0; k < 3; ++k) {
        p0[k] = v[k] - o[k];
        p1[k] = v[3 + k] - o[k];
        p2[k] = v[6 + k] - o[k];
    }
    const int kz = fmo_get_max_axis(d[0], d[1], d[2]);
    const int kx = (kz + 1) % 3;
    const int ky = (kx + 1) % 3;
    const float dx = comp3(d, kx), dy = comp3(d, ky), dz = comp3(d, kz);
    float a0x = p0[kx], a0y = p0[ky], a0z = p0[kz];
    float a1x = p1[kx], a1y = p1[ky], a1z = p1[kz];
    float a2x = p2[kx], a2y = p2[ky], a2z = p2[kz];
    const float sx = -dx / dz, sy = -dy / dz, sz = 1.0f / dz;
    a0x += sx * a0z;
    a0y += sy * a0z;
    a1x += sx * a1z;
    a1y += sy * a1z;
    a2x += sx * a2z;
    a2y += sy * a2z;
    float e0 = a1x * a2y - a1y * a2x;
    float e1 = a2x * a0y - a2y * a0x;
    float e2 = a0x * a1y - a0y * a1x;
    if (e0 == 0.0f || e1 == 0.0f || e2 == 0.0f) {
        e0 = (float)((double)a1x * (double)a2y - (double)a1y * (double)a2x);
        e1 = (float)((double)a2x * (double)a0y - (double)a2y * (double)a0x);
        e2 = (float)((double)a0x * (double)a1y - (double)a0y * (double)a1x);
    }
    if ((e0 < 0 || e1 < 0 || e2 < 0) && (e0 > 0 || e1 > 0 || e2 > 0)) return 0;
    const float det = e0 + e1 + e2;
    if (det == 0) return 0;
    a0z *= sz;
    a1z *= sz;
    a2z *= sz;
    const float inv_det = 1.0f / det;
    const float t = (e0 * a0z + e1 * a1z + e2 * a2z) * inv_det;
    if (t <= tmin || t >= tmax) return 0;
    if (t_out) *t_out = t;
    if (bc) {
        bc[0] = e0 * inv_det;
        bc[1] = e1 * inv_det;
        bc[2] = e2 * inv_det;
    }
    return 1;
}

/* Closest hit over a triangle soup by exhaustive testing, with the acceptance rule of
 * Triangle::GetIntersect (triangle.cpp:211-225) against the shrinking t_max of
 * BVHAggregate::GetIntersectImpl (bvh_aggregate.cpp:108-115): accept when the test
 * succeeds within (t_min, t_best) and not (t > t_best || t <= 0).  Ties keep the
 * lower index.  prim[i] = -1 on a miss. */
void fmo_closest_bruteforce(const float* tri, int64_t ntri, const float* rays, int64_t nrays, int32_t* prim,
                            float* t_out)
{
    for (int64_t i = 0; i < nrays; ++i) {
        float r[8];
        for (int k = 0; k < 8; ++k) r[k] = rays[8 * i + k];
        float best = r[7];
        int32_t bp = -1;
        for (int64_t j = 0; j < ntri; ++j) {
            float t;
            r[7] = best;
            if (!fmo_intersect_triangle(r, tri + 9 * j, &t, 0)) continue;
            if (t > best || t <= 0.0f) continue;
            best = t;
            bp = (int32_t)j;
        }
        prim[i] = bp;
        t_out[i] = bp >= 0 ? best : INFINITY;
    }
}

/* Sphere::IntersectSphere (src/engine/src/geometry/sphere.cpp:91-129, GetCoef :206-212)
 * for a sphere whose object-to-world transform is the translation `center`: the
 * object-space origin is o - center (Transform::ApplyToPoint of a translation is one
 * rounded subtraction per component whatever the matrix-product order), the direction
 * is unchanged; a = SquareSum(d), b = 2 dot(d, o), c = SquareSum(o) - r^2 (sums left to
 * right), delta = b*b - 4*a*c, roots (-b -+ sqrt(delta)) * (0.5 / a); the nearer root in
 * the inclusive range [tmin, tmax] (Ray::Contains) is returned.  Returns 1 on a hit. */
int fmo_intersect_sphere(const float* ray, const float* center, float radius, float* t_out)
{
    const float o0 = ray[0] - center[0], o1 = ray[1] - center[1], o2 = ray[2] - center[2];
    const float d0 = ray[4], d1 = ray[5], d2 = ray[6];
    const float tmin = ray[3], tmax = ray[7];
    const float a = d0 * d0 + d1 * d1 + d2 * d2;
    const float b = 2.0f * (d0 * o0 + d1 * o1 + d2 * o2);
    const float c = o0 * o0 + o1 * o1 + o2 * o2 - radius * radius;
    float delta = b * b - 4.0f * a * c;
    if (delta < 0) return 0;
    delta = sqrtf(delta);
    const float inv2a = 0.5f / a;
    const float t0 = (-b - delta) * inv2a;
    const float t1 = (-b + delta) * inv2a;
    if (t0 >= tmin && t0 <= tmax) {
        *t_out = t0;
        return 1;
    }
    if (t1 >= tmin && t1 <= tmax) {
        *t_out = t1;
        return 1;
    }
    return 0;
}

/* Closest hit over triangles and translated spheres by exhaustive testing: triangles as
 * fmo_closest_bruteforce; a sphere (Sphere::GetIntersect, sphere.cpp:40-55) is accepted
 * when its root lies in [t_min, t_best] (BVHAggregate::GetIntersectImpl then shrinks
 * t_max to it, bvh_aggregate.cpp:108-115).  Spheres are numbered after the triangles:
 * prim[i] = ntri + sphere index for a sphere hit, -1 on a miss. */
void fmo_closest_bruteforce_spheres(const float* tri, int64_t ntri, const float* centers, const float* radii,
                                    int64_t nsph, const float* rays, int64_t nrays, int32_t* prim, float* t_out)
{
    for (int64_t i = 0; i < nrays; ++i) {
        float r[8];
        for (int k = 0; k < 8; ++k) r[k] = rays[8 * i + k];
        float best = r[7];
        int32_t bp = -1;
        for (int64_t j = 0; j < ntri; ++j) {
            float t;
            r[7] = best;
            if (!fmo_intersect_triangle(r, tri + 9 * j, &t, 0)) continue;
            if (t > best || t <= 0.0f) continue;
            best = t;
            bp = (int32_t)j;
        }
        for (int64_t j = 0; j < nsph; ++j) {
            float t;
            r[7] = best;
            if (!fmo_intersect_sphere(r, centers + 3 * j, radii[j], &t)) continue;
            best = t;
            bp = (int32_t)(ntri + j);
        }
        prim[i] = bp;
        t_out[i] = bp >= 0 ? best : INFINITY;
    }
}
