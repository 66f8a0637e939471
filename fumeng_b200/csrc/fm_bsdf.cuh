// BSDFs: Lambert, conductor mirror, dielectric, Disney.
//
// Device restatement of the reference's shading models, in the reference's float
// semantics and evaluation order (including its quirks, which change the converged
// image):
//   core/bsdf.h:30-125                 frame, default cosine sampling / pdf
//   material/lambert_diffuse.cpp       f = basecolor / pi in both hemispheres
//   material/specular_reflection.cpp   conductor Fresnel (core/fresnel.h:70-110)
//   material/specular_transmission.cpp dielectric Fresnel (core/fresnel.h:16-68)
//   material/disney.cpp                lobes :11-356, mixture :359-579, params :627-662
//   material/material_common.cpp       GTR1/GTR2, Smith, refraction
#pragma once
#include "fm_common.cuh"
#include "fm_dual.cuh"
#include "fm_scene.cuh"
#include "fm_texture.cuh"

namespace fm {

struct HitInfo {
    f3 pos, ng, ns, ss, wo;   // world space; wo = -ray direction
    float u, v;               // surface uv
    int obj, mat, prim;
    float b0, b1, b2;         // barycentrics (triangles)
};

struct BsdfSample {
    f3 f;
    f3 wi;      // world space
    float pdf;
    bool delta;
};

FM_D float p5(float x)
{
    const float x2 = x * x;
    return x2 * x2 * x;
}

// DielectricFresnel::CalFr (fresnel.h:16-55)
FM_D float fresnel_dielectric(float cos_i, float eta_i, float eta_t)
{
    float ein = eta_i, eout = eta_t;
    if (cos_i < 0) {
        const float t = ein;
        ein = eout;
        eout = t;
        cos_i = -cos_i;
    }
    const float sin_i = sqrtf(fmaxf(0.0f, 1.0f - cos_i * cos_i));
    const float sin_t = ein / eout * sin_i;
    if (sin_t >= 1.0f) return 1.0f;
    const float cos_t = sqrtf(fmaxf(0.0f, 1.0f - sin_t * sin_t));
    const float perp = (ein * cos_i - eout * cos_t) / (ein * cos_i + eout * cos_t);
    const float para = (eout * cos_i - ein * cos_t) / (eout * cos_i + ein * cos_t);
    return (para * para + perp * perp) * 0.5f;
}

// ConductorFresnel::CalFr (fresnel.h:86-107), per channel
FM_D float fresnel_conductor1(float cos_i, float eta2, float etak2)
{
    if (cos_i <= 0.0f) return 0.0f;
    const float cos2 = cos_i * cos_i;
    const float sin2 = fmaxf(0.0f, 1.0f - cos2);
    const float t0 = eta2 - etak2 - sin2;
    const float a2b2 = sqrtf(t0 * t0 + 4.0f * eta2 * etak2);
    const float t1 = a2b2 + cos2;
    const float a = sqrtf(0.5f * (a2b2 + t0));
    const float t2 = 2.0f * cos_i * a;
    const float rs = (t1 - t2) / (t1 + t2);
    const float t3 = cos2 * a2b2 + sin2 * sin2;
    const float t4 = t2 * sin2;
    const float rp = rs * (t3 - t4) / (t3 + t4);
    return (rp + rs) * 0.5f;
}

// RefractDir (material_common.cpp:112-125); returns false on total internal reflection.
FM_D bool refract_dir(f3 wi, f3 n, float eta, f3& out)
{
    const float cos_i = dot(n, wi);
    const float sin2i = fmaxf(0.0f, 1.0f - cos_i * cos_i);
    const float sin2t = eta * eta * sin2i;
    if (sin2t >= 1.0f) return false;
    const float cos_t = sqrtf(1.0f - sin2t);
    out = normalize(eta * (-wi) + (eta * cos_i - cos_t) * n);
    return true;
}

// The microfacet helpers below evaluate the reference's formulas
// (material_common.cpp:7-103), which are written with the spherical angles of a unit
// vector w (phi = atan2(y, x), theta = acos(z)), with those angles eliminated:
// sin(theta)cos(phi) = x, sin(theta)sin(phi) = y, cos(theta) = z,
// tan^2(theta) = (1 - z^2) / z^2.  The functions are the same; only rounding differs,
// and the code avoids acos/atan2/tan and their large inline expansions.

// GTR2Anisotropic: 1 / (pi ax ay (sin^2(th)(cos^2(ph)/ax^2 + sin^2(ph)/ay^2) + cos^2(th))^2)
// (T is float, or a dual number when the adjoint differentiates with respect to the
// roughness that the alphas come from.)
template <class T>
FM_D T gtr2_aniso(f3 wh, T ax, T ay)
{
    const float z = clampf(wh.z, -1.0f, 1.0f);
    const T a = wh.x / ax, b = wh.y / ay;
    const T den = a * a + b * b + z * z;
    return 1.0f / (kPi * ax * ay * den * den);
}

FM_D f3 sample_gtr2(float ax, float ay, float u0, float u1)
{
    float s2, c2;
    sincosf(2.0f * kPi * u0, &s2, &c2);
    float sin_phi = ay * s2;
    float cos_phi = ax * c2;
    const float norm = 1.0f / sqrtf(sin_phi * sin_phi + cos_phi * cos_phi);
    sin_phi *= norm;
    cos_phi *= norm;
    const float a = cos_phi / ax;
    const float b = sin_phi / ay;
    const float psi = a * a + b * b;
    const float ct = sqrtf(psi * (1.0f - u1) / ((1.0f - psi) * u1 + psi));
    const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    return normalize(f3{st * cos_phi, st * sin_phi, ct});
}

// GTR1GGX: (a^2 - 1) / (2 pi log(a) (a^2 cos^2(th) + sin^2(th)))
FM_D float gtr1(f3 wh, float alpha)
{
    const float z = clampf(wh.z, -1.0f, 1.0f);
    const float c2 = z * z;
    const float a2 = alpha * alpha;
    const float den = 2.0f * kPi * logf(alpha) * (a2 * c2 + (1.0f - c2));
    return (a2 - 1.0f) / den;
}

FM_D f3 sample_gtr1(float alpha, float u0, float u1)
{
    const float phi = 2.0f * kPi * u0;
    const float ct = sqrtf((powf(alpha, 2.0f - 2.0f * u1) - 1.0f) / (alpha * alpha - 1.0f));
    const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    float sp, cp;
    sincosf(phi, &sp, &cp);
    return normalize(f3{st * cp, st * sp, ct});
}

// SmithLambda: -1/2 + 1/2 sqrt(1 + (cos^2(ph) ax^2 + sin^2(ph) ay^2) tan^2(th))
template <class T>
FM_D T smith_lambda(f3 w, T ax, T ay)
{
    const float z = clampf(w.z, -1.0f, 1.0f);
    const T a = w.x * ax, b = w.y * ay;
    const T t = (a * a + b * b) / (z * z);
    return -0.5f + 0.5f * dsqrt(1.0f + t);
}

// SmithGGXAnisotropic uses alpha_y for both axes (material_common.cpp:85-90).
template <class T>
FM_D T smith_ggx_aniso(f3 wo, f3 wi, T ax, T ay)
{
    (void)ax;
    const T li = smith_lambda(wi, ay, ay) + 1.0f;
    const T lo = smith_lambda(wo, ay, ay) + 1.0f;
    return 1.0f / li / lo;
}

// SmithGGXSeprate: 2 / (1 + sqrt(1 + (alpha tan(th))^2)), 1 when tan(th) < eps_pdf
FM_D float smith_ggx_sep(f3 w, float alpha)
{
    const float z = clampf(w.z, -1.0f, 1.0f);
    const float s2 = fmaxf(0.0f, 1.0f - z * z);
    const float tt = sqrtf(s2) / fabsf(z);
    if (tt < kEpsPdf) return 1.0f;
    const float den = tt * alpha;
    return 2.0f / (1.0f + sqrtf(1.0f + den * den));
}

FM_D f3 cosine_hemisphere(float u0, float u1)
{
    const float r = sqrtf(u0);
    const float th = 2.0f * kPi * u1;
    float sn, cs;
    sincosf(th, &sn, &cs);
    const float px = r * cs, py = r * sn;
    float zz = 1.0f - px * px - py * py;
    if (zz < 0.0f) zz = 0.0f;
    return normalize(f3{px, py, sqrtf(zz)});
}

FM_D float cos_dir(f3 w) { return normalize(w).z; }
FM_D bool same_hemi(f3 a, f3 b) { return a.z * b.z > 0; }
FM_D bool opposite_hemi(f3 a, f3 b) { return a.z * b.z < 0; }
FM_D f3 flipz(f3 w) { return f3{w.x, w.y, -w.z}; }
FM_D f3 lerp3(f3 a, f3 b, float t) { return (1.0f - t) * a + t * b; }
FM_D float lerpf(float a, float b, float t) { return (1.0f - t) * a + t * b; }

// ---- material parameter fetch ---------------------------------------------------

FM_D f3 fetch(const DevScene& S, const TexRef& r, const HitInfo& h)
{
    if (r.tex < 0) return f3{r.v[0], r.v[1], r.v[2]};
    return tex_sample(S.textures[r.tex], h.u, h.v);
}

struct Disney {
    f3 basecolor;
    float metallic, specular, specular_tint, roughness, anisotropic, sheen, sheen_tint, clearcoat, clearcoat_gloss,
        spec_trans, spec_trans_roughness, diff_trans, flatness, ior;
    bool thin;
    // derived (disney.cpp:395-456)
    float ax, ay, trans_ax, trans_ay, rough_ax, rough_ay, cc_rough, ior_r, diffuse_weight;
    f3 ctint, cspec0;
    float w_dr, w_sr, w_cc, w_st, w_dt;
    float c_dr, c_cc, c_dt, c_sr, c_st;
};

struct Bsdf {
    int type;
    f3 ng, xs, ys, zs;
    // Lambert / conductor / dielectric parameters
    f3 color;
    f3 color2;   // dielectric refract colour
    f3 eta2, etak2;
    float eta_i, eta_t;
    Disney d;
};

FM_D f3 to_local(const Bsdf& b, f3 v) { return normalize(f3{dot(v, b.xs), dot(v, b.ys), dot(v, b.zs)}); }
FM_D f3 to_world(const Bsdf& b, f3 v)
{
    return normalize(f3{b.xs.x * v.x + b.ys.x * v.y + b.zs.x * v.z, b.xs.y * v.x + b.ys.y * v.y + b.zs.y * v.z,
                        b.xs.z * v.x + b.ys.z * v.y + b.zs.z * v.z});
}

FM_D void disney_setup(Disney& d, float wo_z)
{
    const f3 white = mk(1.0f);
    const float lum = luminance(d.basecolor);
    d.ctint = lum > 0.0f ? d.basecolor * (1.0f / lum) : white;
    float cc = lerpf(0.1f, 0.0f, d.clearcoat_gloss);
    cc *= cc;
    d.cc_rough = cc > 0.0001f ? cc : 0.0001f;
    d.ior_r = 1.0f / d.ior;
    d.cspec0 = lerp3(white, d.ctint, d.specular_tint);
    d.cspec0 = lerp3(d.cspec0, d.basecolor, d.metallic);
    d.diffuse_weight = (1.0f - d.metallic) * (1.0f - d.spec_trans);
    const float aspect = d.anisotropic > 0 ? sqrtf(1.0f - 0.9f * d.anisotropic) : 1.0f;
    const float r2 = d.roughness * d.roughness;
    d.ax = fmaxf(0.001f, r2 / aspect);
    d.ay = fmaxf(0.001f, r2 * aspect);
    const float t2 = d.spec_trans_roughness * d.spec_trans_roughness;
    d.trans_ax = fmaxf(0.001f, t2 / aspect);
    d.trans_ay = fmaxf(0.001f, t2 * aspect);
    const float fr_approx = fresnel_dielectric(wo_z, 1.0f, d.ior);
    const float cspec0_lum = luminance(d.cspec0);
    d.w_dr = lum * d.diffuse_weight * (d.thin ? (1.0f - d.diff_trans) : 1.0f);
    d.w_cc = d.clearcoat * 0.25f;
    d.w_sr = lerpf(cspec0_lum, luminance(white), fr_approx);
    d.w_st = (float)((double)(lum * (1.0f - d.metallic) * d.spec_trans) * (1.0 - (double)fr_approx));
    d.w_dt = d.thin ? lum * d.diffuse_weight * d.diff_trans : 0.0f;
    const float inv = 1.0f / (d.w_dr + d.w_sr + d.w_cc + d.w_st + d.w_dt);
    d.w_dr *= inv;
    d.w_sr *= inv;
    d.w_cc *= inv;
    d.w_st *= inv;
    d.w_dt *= inv;
    d.c_dr = d.w_dr;
    d.c_cc = d.w_cc + d.c_dr;
    d.c_dt = d.w_dt + d.c_cc;
    d.c_sr = d.w_sr + d.c_dt;
    d.c_st = d.w_st + d.c_sr;
    if (d.thin) {
        const float rs = (0.65f * d.ior - 0.35f) * d.spec_trans_roughness;
        d.rough_ax = fmaxf(0.001f, rs * rs / aspect);
        d.rough_ay = fmaxf(0.001f, rs * rs * aspect);
    } else {
        d.rough_ax = d.trans_ax;
        d.rough_ay = d.trans_ay;
    }
}


template <int CLS = kClsAny>
FM_D Bsdf make_bsdf(const DevScene& S, const HitInfo& h)
{
    Bsdf b;
    const DevMaterial& M = S.materials[h.mat];
    b.type = CLS == kClsDisney ? 3 : M.type;
    b.ng = h.ng;
    b.zs = h.ns;
    b.xs = normalize(h.ss);
    b.ys = cross(b.zs, b.xs);
    if (CLS == kClsDisney) {
        // fall through to the Disney branch below
    } else if (M.type == 0) {
        b.color = fetch(S, M.p[MP_BASECOLOR], h);
    } else if (M.type == 1) {
        b.color = ld3(M.color);
        b.eta2 = ld3(M.cond_eta2);
        b.etak2 = ld3(M.cond_etak2);
    } else if (M.type == 2) {
        b.color = ld3(M.reflect_color);
        b.color2 = ld3(M.refract_color);
        b.eta_i = M.eta_i;
        b.eta_t = M.eta_t;
    }
    if (CLS != kClsSimple && b.type == 3) {
        Disney& d = b.d;
        d.basecolor = fetch(S, M.p[MP_BASECOLOR], h);
        d.metallic = fetch(S, M.p[MP_METALLIC], h).z;
        d.specular = fetch(S, M.p[MP_SPECULAR], h).x;
        d.specular_tint = fetch(S, M.p[MP_SPECULAR_TINT], h).x;
        d.roughness = fetch(S, M.p[MP_ROUGHNESS], h).y;
        d.anisotropic = fetch(S, M.p[MP_ANISOTROPIC], h).x;
        d.sheen = fetch(S, M.p[MP_SHEEN], h).x;
        d.sheen_tint = fetch(S, M.p[MP_SHEEN_TINT], h).x;
        d.clearcoat = fetch(S, M.p[MP_CLEARCOAT], h).x;
        d.clearcoat_gloss = fetch(S, M.p[MP_CLEARCOAT_GLOSS], h).x;
        d.spec_trans = fetch(S, M.p[MP_SPEC_TRANS], h).x;
        d.spec_trans_roughness = fetch(S, M.p[MP_SPEC_TRANS_ROUGHNESS], h).x;
        d.diff_trans = fetch(S, M.p[MP_DIFF_TRANS], h).x;
        d.flatness = fetch(S, M.p[MP_FLATNESS], h).x;
        d.ior = fetch(S, M.p[MP_IOR], h).x;
        d.thin = M.thin != 0;
        if (M.vattr_offset >= 0 && h.prim < S.num_tris && S.tri_vattr) {
            // per-vertex attributes: basecolor.rgb, roughness, metallic, clearcoat
            const float* a = S.tri_vattr + (size_t)h.prim * 3 * S.vattr_dim + M.vattr_offset;
            const int k = S.vattr_dim;
            float v[6];
            for (int q = 0; q < 6; ++q) v[q] = h.b0 * a[q] + h.b1 * a[k + q] + h.b2 * a[2 * k + q];
            d.basecolor = f3{v[0], v[1], v[2]};
            d.roughness = v[3];
            d.metallic = v[4];
            d.clearcoat = v[5];
        }
        disney_setup(d, to_local(b, h.wo).z);
    }
    return b;
}

FM_D f3 bsdf_albedo(const Bsdf& b)
{
    return b.type == 3 ? b.d.basecolor : b.color;
}

// ---- Disney lobes (disney.cpp:11-356) ---------------------------------------------

FM_D f3 ds_spec_eval(const Disney& d, f3 wo, f3 wi)
{
    if (!same_hemi(wo, wi)) return mk(0.0f);
    const f3 wh = normalize(wo + wi);
    const float cos_o = cos_dir(wo), cos_i = cos_dir(wi);
    const float cos_d = dot(wi, wh.z > 0 ? wh : -wh);
    const f3 f_diel = d.cspec0 * fresnel_dielectric(cos_d, 1.0f, d.ior);
    const f3 white = mk(1.0f);
    const float pf = p5(clampf(1.0f - fabsf(cos_d), 0.0f, 1.0f));
    const f3 f_cond = d.cspec0 + (white - d.cspec0) * pf;
    const f3 f = lerp3(d.specular * f_diel, f_cond, d.metallic);
    const float D = gtr2_aniso(wh, d.ax, d.ay);
    const float G = smith_ggx_aniso(wo, wi, d.ax, d.ay);
    // Exactly grazing directions give 0/0 here; the value is set to zero (a set of
    // measure zero) so that float does not emit NaN where the double build does not.
    const float den = fabsf(4.0f * cos_i * cos_o);
    if (den == 0.0f) return mk(0.0f);
    return f * D * G / den;
}

FM_D f3 ds_spec_sample(const Disney& d, f3 wo, float u0, float u1)
{
    f3 wh = sample_gtr2(d.ax, d.ay, u0, u1);
    if (same_hemi(wo, wh)) wh = flipz(wh);
    const f3 wi = normalize(2.0f * dot(wo, wh) * wh - wo);
    return same_hemi(wo, wi) ? wi : flipz(wi);
}

FM_D float ds_spec_pdf(const Disney& d, f3 wo, f3 wi)
{
    if (!same_hemi(wo, wi)) return 0.0f;
    const f3 wh = normalize(wo + wi);
    const float cos_d = dot(wi, wh.z > 0 ? wh : -wh);
    const float D = gtr2_aniso(wh, d.ax, d.ay);
    return fabsf(fabsf(cos_dir(wh)) * D / (4.0f * cos_d));
}

FM_D f3 ds_diffuse_eval(const Disney& d, f3 wo, f3 wi)
{
    const f3 wh = normalize(wo + wi);
    const float cos_o = fabsf(cos_dir(wo));
    const float cos_i = fabsf(cos_dir(wi));
    const float cos_d = fabsf(dot(wi, wh));
    const f3 f_lambert = d.basecolor / kPi;
    const float fl = p5(1.0f - cos_i);
    const float fv = p5(1.0f - cos_o);
    const float rr = 2.0f * d.roughness * cos_d * cos_d;
    const f3 f_retro = f_lambert * rr * (fl + fv + fl * fv * (rr - 1.0f));
    const f3 c_sheen = lerp3(mk(1.0f), d.ctint, d.sheen_tint);
    const f3 f_sheen = 4.0f * d.sheen * c_sheen * p5(1.0f - cos_d);
    float wt = d.diffuse_weight;
    if (d.thin) wt *= (1.0f - d.flatness) * (1.0f - d.diff_trans);
    return wt * f_lambert * (1.0f - 0.5f * fl) * (1.0f - 0.5f * fv) + f_retro + f_sheen;
}

FM_D f3 ds_diffuse_sample(f3 wo, float u0, float u1)
{
    const f3 wi = cosine_hemisphere(u0, u1);
    return same_hemi(wo, wi) ? wi : flipz(wi);
}

FM_D float ds_diffuse_pdf(f3 wo, f3 wi)
{
    if (!same_hemi(wo, wi)) return 0.0f;
    return fabsf(wi.z) * kInvPi;
}

FM_D f3 ds_cc_eval(const Disney& d, f3 wo, f3 wi)
{
    if (!same_hemi(wo, wi)) return mk(0.0f);
    const f3 wh = normalize(wo + wi);
    const float cos_o = fabsf(cos_dir(wo));
    const float cos_i = fabsf(cos_dir(wi));
    const float cos_d = fabsf(dot(wi, wh));
    const float f = 0.04f + (1.0f - 0.04f) * p5(clampf(1.0f - cos_d, 0.0f, 1.0f));
    const float D = gtr1(wh, d.cc_rough);
    const float G = smith_ggx_sep(wi, 0.25f) * smith_ggx_sep(wo, 0.25f);
    const float den = fabsf(4.0f * cos_i * cos_o);
    if (den == 0.0f) return mk(0.0f);
    return mk(d.clearcoat * f * D * G / den);
}

FM_D f3 ds_cc_sample(const Disney& d, f3 wo, float u0, float u1)
{
    f3 wh = sample_gtr1(d.cc_rough, u0, u1);
    if (same_hemi(wo, wh)) wh = flipz(wh);
    const f3 wi = normalize(2.0f * dot(wo, wh) * wh - wo);
    return same_hemi(wo, wi) ? wi : flipz(wi);
}

FM_D float ds_cc_pdf(const Disney& d, f3 wo, f3 wi)
{
    if (!same_hemi(wo, wi)) return 0.0f;
    const f3 wh = normalize(wo + wi);
    const float cos_d = dot(wi, wh);
    const float D = gtr1(wh, d.cc_rough);
    return fabsf(fabsf(cos_dir(wh)) * D / (4.0f * cos_d));
}

// DisneyMicrofacetTransmission with lobe alphas (ax, ay) and colour `c`.  Sampling and
// pdf use the BSDF's trans_alpha (disney.cpp:238-273) whatever the lobe's own alphas.
// |ft| of the transmission lobe: everything but spec_trans (1 - metallic) c; wo, wi in
// opposite hemispheres.
FM_D float ds_trans_ft(const Disney& d, f3 wo, f3 wi, float ax, float ay)
{
    const float eta = wo.z > 0 ? d.ior : d.ior_r;
    f3 wh = normalize(wo + eta * wi);
    if (wh.z < 0) wh = -wh;
    const float cos_o = cos_dir(wo), cos_i = cos_dir(wi);
    const float cdo = dot(wo, wh), cdi = dot(wi, wh);
    const float f = fresnel_dielectric(cdo, 1.0f, d.ior);
    const float D = gtr2_aniso(wh, ax, ay);
    const float G = smith_ggx_aniso(wo, wi, ax, ay);
    const float den = eta * cdi + cdo;
    const float q = cos_i * cos_o * den * den;
    if (q == 0.0f) return 0.0f;
    return fabsf((1.0f - f) * D * G * cdo * cdi / q);
}

FM_D f3 ds_trans_eval(const Disney& d, f3 wo, f3 wi, float ax, float ay, f3 c)
{
    if (!opposite_hemi(wo, wi)) return mk(0.0f);
    return d.spec_trans * (1.0f - d.metallic) * c * ds_trans_ft(d, wo, wi, ax, ay);
}

FM_D f3 ds_trans_sample(const Disney& d, f3 wo, float u0, float u1)
{
    f3 wh = sample_gtr2(d.trans_ax, d.trans_ay, u0, u1);
    const float eta_r = wo.z > 0 ? d.ior_r : d.ior;
    const f3 n = same_hemi(wo, wh) ? wh : flipz(wh);
    f3 wt;
    if (!refract_dir(wo, n, eta_r, wt)) return mk(0.0f);
    return wt;
}

FM_D float ds_trans_pdf(const Disney& d, f3 wo, f3 wi)
{
    if (!opposite_hemi(wo, wi)) return 0.0f;
    const float eta = wo.z > 0 ? d.ior : d.ior_r;
    f3 wh = normalize(wo + eta * wi);
    if (wh.z < 0) wh = -wh;
    const float cdo = dot(wo, wh), cdi = dot(wi, wh);
    const float D = gtr2_aniso(wh, d.trans_ax, d.trans_ay);
    const float den = eta * cdi + cdo;
    const float dwh_dwi = eta * eta * cdi / den / den;
    return fabsf(cdi * D * dwh_dwi);
}

FM_D f3 ds_fakess_eval(const Disney& d, f3 wo, f3 wi)
{
    if (!same_hemi(wo, wi)) return mk(0.0f);
    const f3 wh = normalize(wo + wi);
    const float cos_o = fabsf(cos_dir(wo));
    const float cos_i = fabsf(cos_dir(wi));
    const float cos_d = fabsf(dot(wi, wh));
    const float fss90 = cos_d * cos_d * d.roughness;
    const float fo = p5(1.0f - cos_o), fi = p5(1.0f - cos_i);
    const float fss = lerpf(fo, 1.0f, fss90) * lerpf(fi, 1.0f, fss90);
    const float ss = 1.25f * (fss * (1.0f / (cos_o + cos_i) - 0.5f) + 0.5f);
    const float weight = d.diffuse_weight * d.flatness * (1.0f - d.diff_trans);
    return weight * d.basecolor * kInvPi * ss;
}

FM_D f3 ds_ltrans_eval(const Disney& d, f3 wo, f3 wi)
{
    if (!opposite_hemi(wo, wi)) return mk(0.0f);
    return d.diff_trans * d.basecolor;
}

FM_D f3 ds_ltrans_sample(f3 wo, float u0, float u1)
{
    const f3 wi = cosine_hemisphere(u0, u1);
    return same_hemi(wo, wi) ? flipz(wi) : wi;
}

FM_D float ds_ltrans_pdf(f3 wo, f3 wi)
{
    if (!opposite_hemi(wo, wi)) return 0.0f;
    return fabsf(wi.z) * kInvPi;
}

FM_D f3 disney_f(const Disney& d, f3 wo, f3 wi)
{
    f3 r = mk(0.0f);
    if (wo.z * wi.z < 0) {
        if (d.thin) {
            r += ds_trans_eval(d, wo, wi, d.rough_ax, d.rough_ay, f3{sqrtf(d.basecolor.x), sqrtf(d.basecolor.y), sqrtf(d.basecolor.z)});
            r += ds_ltrans_eval(d, wo, wi);
        } else {
            r += ds_trans_eval(d, wo, wi, d.trans_ax, d.trans_ay, d.basecolor);
        }
        return r;
    }
    if (d.metallic < 1.0f && d.spec_trans < 1.0f) {
        if (d.thin && d.flatness > 0.0f) r += ds_fakess_eval(d, wo, wi);
        r += ds_diffuse_eval(d, wo, wi);
    }
    r += ds_spec_eval(d, wo, wi);
    if (d.clearcoat > 0.0f) r += ds_cc_eval(d, wo, wi);
    return r;
}

FM_D float disney_pdf_refl_trans(const Disney& d, f3 wo, f3 wi)
{
    float fr = fresnel_dielectric(wo.z, 1.0f, d.ior);
    fr = 1.0f - ((1.0f - fr) * d.spec_trans * (1.0f - d.metallic));
    if (wo.z * wi.z > 0.0f) return (d.w_st + d.w_sr) * fr * ds_spec_pdf(d, wo, wi);
    return (d.w_st + d.w_sr) * (1.0f - fr) * ds_trans_pdf(d, wo, wi);
}

FM_D float disney_pdf(const Disney& d, f3 wo, f3 wi)
{
    float p = 0.0f;
    if (d.w_dr > 0.0f) p += d.w_dr * ds_diffuse_pdf(wo, wi);
    if (d.w_cc > 0.0f) p += d.w_cc * ds_cc_pdf(d, wo, wi);
    if (d.w_st + d.w_sr > 0.0f) p += disney_pdf_refl_trans(d, wo, wi);
    if (d.w_dt > 0.0f) p += d.w_dt * ds_ltrans_pdf(wo, wi);
    return p;
}

// DisneyBSDF::RouletteSample / SampleReflOrTrans (disney.cpp:489-531): the lobe choice
// and the reflect/transmit choice both read samples.z.
FM_D f3 disney_sample_dir(const Disney& d, f3 wo, f3 u)
{
    const float r = u.z;
    if (r <= d.c_dr) return ds_diffuse_sample(wo, u.x, u.y);
    if (r <= d.c_cc) return ds_cc_sample(d, wo, u.x, u.y);
    if (r <= d.c_dt) return ds_ltrans_sample(wo, u.x, u.y);
    float fr = fresnel_dielectric(wo.z, 1.0f, d.ior);
    fr = 1.0f - ((1.0f - fr) * d.spec_trans * (1.0f - d.metallic));
    if (u.z <= fr) return ds_spec_sample(d, wo, u.x, u.y);
    return ds_trans_sample(d, wo, u.x, u.y);
}

// ---- BSDF interface (bsdf.h:136-182 and the overrides) ------------------------------

// CalFunc(wo_w, wi_w)
template <int CLS = kClsAny>
FM_D f3 bsdf_f(const Bsdf& b, f3 wo_w, f3 wi_w)
{
    if (CLS != kClsDisney) {
        if (b.type == 0) return b.color * kInvPi;
        if (b.type == 1 || b.type == 2 || CLS == kClsSimple) return mk(0.0f);
    }
    return disney_f(b.d, to_local(b, wo_w), to_local(b, wi_w));
}

// Pdf(wo_w, wi_w)
template <int CLS = kClsAny>
FM_D float bsdf_pdf(const Bsdf& b, f3 wo_w, f3 wi_w)
{
    if (CLS != kClsDisney && (b.type == 1 || b.type == 2)) return 0.0f;
    const f3 wo = to_local(b, wo_w), wi = to_local(b, wi_w);
    if (CLS != kClsDisney) {
        if (b.type == 0 || CLS == kClsSimple) {
            if (wo.z * wi.z < 0.0f) return 0.0f;
            return fabsf(wi.z) * kInvPi;
        }
    }
    return disney_pdf(b.d, wo, wi);
}

template <int CLS = kClsAny>
FM_D BsdfSample bsdf_sample(const Bsdf& b, f3 wo_w, f3 u)
{
    BsdfSample s;
    const f3 wo = to_local(b, wo_w);
    if (CLS == kClsDisney) goto disney;
    if (b.type == 0) {
        f3 wi = cosine_hemisphere(u.x, u.y);
        if (wo.z * wi.z < 0.0f) wi.z *= -1.0f;
        s.pdf = (wo.z * wi.z < 0.0f) ? 0.0f : fabsf(wi.z) * kInvPi;
        s.f = b.color * kInvPi;
        s.wi = to_world(b, wi);
        s.delta = false;
        return s;
    }
    // Delta samples at an exactly grazing angle (cos = 0) give 0/0 or x/0; they are
    // returned as failed samples (a set of measure zero) instead of NaN.
    if (b.type == 1) {
        const f3 wi = f3{-wo.x, -wo.y, wo.z};
        const float ci = cos_dir(wi);
        if (ci == 0.0f) {
            s.f = mk(0.0f);
            s.wi = mk(0.0f);
            s.pdf = 0.0f;
            s.delta = true;
            return s;
        }
        const f3 fr = f3{fresnel_conductor1(ci, b.eta2.x, b.etak2.x), fresnel_conductor1(ci, b.eta2.y, b.etak2.y),
                         fresnel_conductor1(ci, b.eta2.z, b.etak2.z)};
        s.f = fr * b.color / fabsf(ci);
        s.wi = to_world(b, wi);
        s.pdf = 1.0f;
        s.delta = true;
        return s;
    }
    if (b.type == 2) {
        const float fr = fresnel_dielectric(cos_dir(wo), b.eta_i, b.eta_t);
        s.delta = true;
        if (cos_dir(wo) == 0.0f) {
            s.f = mk(0.0f);
            s.wi = mk(0.0f);
            s.pdf = 0.0f;
            return s;
        }
        if (u.x < fr) {
            const f3 wi = f3{-wo.x, -wo.y, wo.z};
            const float ci = cos_dir(wi);
            s.pdf = fr;
            s.f = fresnel_dielectric(ci, b.eta_i, b.eta_t) * b.color / fabsf(ci);
            s.wi = to_world(b, wi);
            return s;
        }
        float ei = b.eta_i, et = b.eta_t;
        f3 n = f3{0.0f, 0.0f, 1.0f};
        if (cos_dir(wo) < 0) {
            const float t = ei;
            ei = et;
            et = t;
            n = -n;
        }
        const float eta = ei / et;
        f3 wt;
        if (!refract_dir(wo, n, eta, wt)) {
            s.f = mk(0.0f);
            s.wi = mk(0.0f);
            s.pdf = 0.0f;
            return s;
        }
        s.pdf = 1.0f - fr;
        const float ct = cos_dir(wt);
        if (ct == 0.0f) {
            s.f = mk(0.0f);
            s.wi = mk(0.0f);
            s.pdf = 0.0f;
            return s;
        }
        s.f = eta * eta * b.color2 * (1.0f - fr) / fabsf(ct);
        s.wi = to_world(b, wt);
        return s;
    }
    if (CLS == kClsSimple) {
        s.f = mk(0.0f);
        s.wi = mk(0.0f);
        s.pdf = 0.0f;
        s.delta = false;
        return s;
    }
disney:
    // Disney: SampleBSDF -> SampleInfoFromWoWi (disney.cpp:481-548)
    const f3 wi = disney_sample_dir(b.d, wo, u);
    s.delta = false;
    if (length(wi) < kEpsPdf) {
        s.f = mk(0.0f);
        s.wi = mk(0.0f);
        s.pdf = 0.0f;
        return s;
    }
    s.pdf = disney_pdf(b.d, wo, wi);
    s.f = disney_f(b.d, wo, wi);
    s.wi = to_world(b, wi);
    return s;
}

}  // namespace fm
