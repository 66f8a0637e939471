// Hit points, lights, camera and the per-vertex integrator logic shared by the
// megakernel and the wavefront kernels.
#pragma once
#include "fm_bsdf.cuh"
#include "fm_bvh.cuh"
#include "fm_rng.cuh"
#include "fm_texture.cuh"

namespace fm {

// ---- camera (camera/pin_hole_camera.cpp:5-56, camera/thin_lens_camera.cpp:23-30) ----
struct DevCamera {
    f3 pos;
    f3 s, u, f;   // camera-to-world basis (x right, y up, z forward; left-handed lookAt)
    float film_w, film_h, focal, lens_radius;
    int type;     // 0 pinhole, 1 thin lens
};

// ndc (px, py) in [0,1)^2 with py = 0 at the bottom row; lens sample in [0,1)^2.
FM_D void camera_ray(const DevCamera& c, float px, float py, float lx, float ly, f3& o, f3& d)
{
    const f3 film = f3{(px - 0.5f) * c.film_w, (py - 0.5f) * c.film_h, c.focal};
    if (c.type == 0) {
        const f3 fw = c.pos + c.s * film.x + c.u * film.y + c.f * film.z;
        o = c.pos;
        d = normalize(fw - c.pos);
    } else {
        // square aperture [0, r)^2, off-centre, as the reference samples it
        const f3 ol = f3{c.lens_radius * lx, c.lens_radius * ly, 0.0f};
        const f3 dl = normalize(film - ol);
        o = c.pos + c.s * ol.x + c.u * ol.y + c.f * ol.z;
        d = c.s * dl.x + c.u * dl.y + c.f * dl.z;
    }
}

// ---- hit points ------------------------------------------------------------------

FM_D f3 sphere_normal_world(const SphereDev& sp, f3 n_local)
{
    return normalize(xf_normal_from_inv(sp.w2o, n_local));
}

// Sphere::CalHitPoint (sphere.cpp:61-88) for an object-space position.
FM_D void sphere_point(const SphereDev& sp, f3 pl, HitInfo& h)
{
    float phi = (pl.x == 0.0f && !(pl.y != 0.0f)) ? 0.0f : atan2f(pl.y, pl.x);
    if (phi < 0) phi += 2.0f * kPi;
    const float ct = clampf(pl.z / sp.radius, -1.0f, 1.0f);
    const float theta = acosf(ct);
    const f3 gn = normalize(pl);
    f3 aux = f3{0.0f, 0.0f, 1.0f};
    if (fabsf(gn.z - 1.0f) < kEps || fabsf(gn.z + 1.0f) < kEps) aux = f3{1.0f, 0.0f, 0.0f};
    h.u = phi * 0.5f * kInvPi;
    h.v = theta * kInvPi;
    h.pos = xf_point(sp.o2w, pl);
    h.ng = sphere_normal_world(sp, gn);
    h.ns = h.ng;
    h.ss = xf_vec(sp.o2w, cross(gn, aux));
}

// Triangle::GetIntersect hit fill (triangle.cpp:225-245), Rectangle::CalHitPoint
// (rectangle.cpp:58-85), Sphere::GetIntersect (sphere.cpp:41-55).
FM_D HitInfo make_hit(const DevScene& S, f3 o, f3 d, const Hit& hit)
{
    HitInfo h;
    h.prim = hit.prim;
    h.obj = __ldg(S.prim_obj + hit.prim);
    h.mat = __ldg(S.obj_material + h.obj);
    h.wo = -d;
    h.b1 = hit.b1;
    h.b2 = hit.b2;
    h.b0 = 1.0f - hit.b1 - hit.b2;
    const int p = hit.prim;
    if (p < S.num_tris) {
        const float* v = S.tri_pos + 9 * (size_t)p;
        const f3 v0 = ld3(v), v1 = ld3(v + 3), v2 = ld3(v + 6);
        h.pos = o + d * hit.t;
        if (S.tri_uv) {
            const float* q = S.tri_uv + 6 * (size_t)p;
            h.u = h.b0 * q[0] + h.b1 * q[2] + h.b2 * q[4];
            h.v = h.b0 * q[1] + h.b1 * q[3] + h.b2 * q[5];
        } else {
            h.u = h.v = 0.0f;
        }
        if (S.tri_normal && S.tri_has_normal[p]) {
            const float* n = S.tri_normal + 9 * (size_t)p;
            h.ng = h.b0 * ld3(n) + h.b1 * ld3(n + 3) + h.b2 * ld3(n + 6);
        } else {
            h.ng = normalize(cross(v0 - v2, v1 - v2));
        }
        h.ns = h.ng;
        h.ss = normalize(v1 - v0);
    } else if (p < S.num_tris + 2 * S.num_rects) {
        const int r = (p - S.num_tris) >> 1, half = (p - S.num_tris) & 1;
        const RectDev& R = S.rects[r];
        h.pos = o + d * hit.t;
        h.ng = ld3(R.normal);
        h.ns = h.ng;
        h.ss = ld3(R.ss);
        if (half == 0) {   // bc.x*(0,0) + bc.y*(0,1) + bc.z*(1,1)
            h.u = h.b2;
            h.v = h.b1 + h.b2;
        } else {           // bc.x*(1,1) + bc.y*(0,1) + bc.z*(0,0)
            h.u = h.b0;
            h.v = h.b0 + h.b1;
        }
    } else {
        const SphereDev& sp = S.spheres[p - S.num_tris - 2 * S.num_rects];
        const f3 ol = xf_point(sp.w2o, o), dl = xf_vec(sp.w2o, d);
        sphere_point(sp, ol + dl * hit.t, h);
    }
    return h;
}

// HitPoint::GenRay (hit_point.h:26-37)
FM_D f3 spawn_origin(const HitInfo& h, f3 dir) { return dot(dir, h.ng) > 0 ? h.pos + h.ng * kEps : h.pos - h.ng * kEps; }

// ---- lights (light/*.cpp, geometry Sample/Pdf) -------------------------------------

struct LightSample {
    f3 wi, radiance;
    float pdf, dist;
    bool delta;
};

FM_D float tri_area(f3 v0, f3 v1, f3 v2) { return length(cross(v1 - v0, v2 - v0)) * 0.5f; }

// Geometry::Sample(ref, ...) of an area light's shape: position, normal, area pdf.
FM_D void area_geom_sample(const DevScene& S, const DevLight& L, f3 ref, f3 u, f3& pos, f3& n, float& pdf_area)
{
    if (L.kind == LK_AREA_SPHERE) {
        const SphereDev& sp = S.spheres[L.index];
        const f3 spl = xf_point(sp.w2o, ref);
        const float dis = length(spl);
        HitInfo hh;
        if (dis < sp.radius) {
            // UniformSphere (utils.h:36-42)
            const float z = 1.0f - 2.0f * u.x;
            const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
            const float phi = 2.0f * kPi * u.y;
            sphere_point(sp, f3{r * cosf(phi), r * sinf(phi), z} * sp.radius, hh);
            pdf_area = 1.0f / sp.area;
        } else {
            // UniformCone about the direction to the shading point (sphere.cpp:143-179)
            const float cmin = fminf(sp.radius / dis, 1.0f);
            const float ct = cmin + u.x * (1.0f - cmin);
            const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
            const float phi = 2.0f * kPi * u.y;
            const f3 ds = f3{cosf(phi) * st, sinf(phi) * st, ct};
            const float pa = 1.0f / (2.0f * kPi * (1.0f - cmin));
            const f3 az = normalize(spl);
            f3 ax;
            if (fabsf(az.x) > fabsf(az.y))
                ax = normalize(f3{-az.z, 0.0f, az.x});
            else
                ax = normalize(f3{0.0f, az.z, -az.y});
            const f3 ay = cross(az, ax);
            sphere_point(sp, sp.radius * (ax * ds.x + ay * ds.y + az * ds.z), hh);
            pdf_area = pa / sp.rw2;
        }
        pos = hh.pos;
        n = hh.ng;
        return;
    }
    const float su = sqrtf(u.x);
    const float b0 = 1.0f - su;
    const float b1 = u.y * su;
    const float b2 = 1.0f - b0 - b1;
    if (L.kind == LK_AREA_RECT) {
        const RectDev& R = S.rects[L.index];
        n = ld3(R.normal);
        if (u.z < 0.5f)
            pos = b0 * ld3(R.pa) + b1 * ld3(R.pb) + b2 * ld3(R.pc);
        else
            pos = b0 * ld3(R.pc) + b1 * ld3(R.pd) + b2 * ld3(R.pa);
        pdf_area = 1.0f / R.area;
        return;
    }
    int t = L.index;
    if (L.kind == LK_AREA_MESH) {
        // TriangleEmbree::Sample (geometry/triangle_embree.cpp:253-260): a triangle by area
        // with sample.z (alias table instead of the CDF search), a point on it with
        // sample.xy, area pdf 1 / (total area)
        const float x = u.z * (float)L.count;
        int k = min((int)x, L.count - 1);
        if (x - (float)k >= __ldg(S.mlight_prob + L.index + k)) k = __ldg(S.mlight_alias + L.index + k);
        t = __ldg(S.mlight_tri + L.index + k);
    }
    const float* v = S.tri_pos + 9 * (size_t)t;
    const f3 v0 = ld3(v), v1 = ld3(v + 3), v2 = ld3(v + 6);
    pos = b0 * v0 + b1 * v1 + b2 * v2;
    if (S.tri_normal && S.tri_has_normal[t]) {
        const float* q = S.tri_normal + 9 * (size_t)t;
        n = b0 * ld3(q) + b1 * ld3(q + 3) + b2 * ld3(q + 6);
    } else {
        n = normalize(cross(v0 - v2, v1 - v2));
    }
    pdf_area = L.kind == LK_AREA_MESH ? L.inv_area : 1.0f / tri_area(v0, v1, v2);
}

// Light::Sample at a shading position (area_light.cpp:16-26, directional_light.cpp:15-18,
// env_light.cpp:38-44).  Returns false when the sample is invalid (pdf 0).
FM_D bool light_sample(const DevScene& S, const DevLight& L, f3 ref, f3 u, LightSample& ls)
{
    if (L.kind == LK_DIR) {
        ls.wi = -ld3(L.direction);
        ls.radiance = ld3(L.radiance);
        ls.pdf = 1.0f;
        ls.dist = kRealMax;
        ls.delta = true;
        return true;
    }
    if (L.kind == LK_ENV) {
        ls.delta = false;
        ls.dist = kRealMax;
        if (!env_sample(S, u, ls.wi, ls.pdf, ls.radiance)) {
            ls.pdf = 0.0f;
            return false;
        }
        return true;
    }
    f3 pos, n;
    float pa;
    area_geom_sample(S, L, ref, u, pos, n, pa);
    const f3 rl = pos - ref;
    const float dist = length(rl);
    ls.delta = false;
    if (dist < kEps) {
        ls.pdf = 0.0f;
        return false;
    }
    ls.wi = normalize(rl);
    ls.pdf = pa * dist * dist / absdot(n, -ls.wi);
    ls.radiance = ld3(L.radiance);   // two-sided: radiance regardless of facing
    ls.dist = dist;
    return true;
}

// AreaLight::Pdf (area_light.cpp:40-50) with Geometry::Pdf of the shape.
FM_D float area_light_pdf(const DevScene& S, const DevLight& L, f3 shd, f3 lpos, f3 lnor, f3 l2s)
{
    if (dot(lnor, l2s) < 0) return 0.0f;
    float pa;
    if (L.kind == LK_AREA_RECT) {
        pa = 1.0f / S.rects[L.index].area;
    } else if (L.kind == LK_AREA_TRI) {
        const float* v = S.tri_pos + 9 * (size_t)L.index;
        pa = 1.0f / tri_area(ld3(v), ld3(v + 3), ld3(v + 6));
    } else if (L.kind == LK_AREA_MESH) {
        pa = L.inv_area;   // TriangleEmbree::Pdf (triangle_embree.cpp:267-270)
    } else {
        const SphereDev& sp = S.spheres[L.index];
        const float dis = length(xf_point(sp.w2o, shd));
        if (dis < sp.radius) {
            pa = 1.0f / sp.area;
        } else {
            const float ct = fminf(sp.radius / dis, 1.0f);
            pa = 1.0f / (2.0f * kPi * (1.0f - ct)) / sp.rw2;
        }
    }
    const float dist = length(shd - lpos);
    return pa * dist * dist / absdot(lnor, l2s);
}

// PowerHeuristic (core/utils.h:108-111), f^2 / (f^2 + g^2), evaluated as 1 / (1 + (g/f)^2)
// so that float does not overflow where the reference's double build does not (a light
// pdf near 1e20 at grazing angles squares to inf in float and the ratio becomes NaN).
// Callers guarantee f >= eps_pdf > 0.
FM_D float power_heuristic(float f, float g)
{
    const float r = g / f;
    return 1.0f / (1.0f + r * r);
}

// ---- render configuration ----------------------------------------------------------
struct RenderCfg {
    // width x height: the rendered pixels (the region, or the whole image); the camera
    // sees the img_w x img_h image, and rendered pixel (i, row) is image pixel
    // (x0 + i, y0 + row)
    int width, height, spp, depth, direct_loop, rr_depth;
    int img_w, img_h, x0, y0;
    float rr_coef;
    uint64_t seed;
    int sample_offset;
    int rr_enabled;   // depth > rr_depth (path_tracing.cpp:107)
    float clamp;      // > 0: per-channel limit of a sample's radiance (extension), 0: off
};

// Camera-film coordinates and random-stream key of rendered pixel p: film position
// (i, j) with j counted from the bottom row (renderer.h:98,106) and the image pixel index.
struct PixelRef {
    int i, j;
    uint64_t key;
};
FM_HD PixelRef pixel_ref(const RenderCfg& cfg, int p)
{
    const int row = cfg.y0 + p / cfg.width;
    const int i = cfg.x0 + p % cfg.width;
    return PixelRef{i, cfg.img_h - 1 - row, (uint64_t)row * (uint64_t)cfg.img_w + (uint64_t)i};
}

// A camera sample's radiance as it enters the pixel sum: each channel limited to
// cfg.clamp when the clamp is on (a NaN channel stays NaN, so it is still counted).
FM_HD f3 clamp_sample(const RenderCfg& cfg, f3 c)
{
    if (cfg.clamp > 0.0f) {
        c.x = c.x > cfg.clamp ? cfg.clamp : c.x;
        c.y = c.y > cfg.clamp ? cfg.clamp : c.y;
        c.z = c.z > cfg.clamp ? cfg.clamp : c.z;
    }
    return c;
}

struct Counters {
    unsigned long long paths, closest, shadow, bounces, nans;
};

}  // namespace fm
