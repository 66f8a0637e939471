// BSDF values with their derivatives with respect to the shading point's basecolor
// (r, g, b), metallic and roughness, for the adjoint renderer.
//
// Each lobe is the float lobe of fm_bsdf.cuh (same formulas, same branches) evaluated
// on dual numbers where a quantity depends on those five parameters; directions stay
// plain floats (sampled directions are held fixed).  The densities that weight a
// sampled direction are differentiated too (disney_pdfs_grad below).
#pragma once
#include "fm_bsdf.cuh"
#include "fm_dual.cuh"

namespace fm {

// Parameter indices of a D5's partials.
enum GradParam : int { GP_BASE_R = 0, GP_BASE_G = 1, GP_BASE_B = 2, GP_METALLIC = 3, GP_ROUGHNESS = 4 };

// The Disney quantities that depend on the differentiated parameters
// (disney_setup's derived values ctint, cspec0, diffuse weight and the alphas).
struct DisneyG {
    DV3 basecolor, ctint, cspec0;
    D5 metallic, roughness, diffuse_weight, ax, ay;
};

FM_D DisneyG disney_grad_setup(const Disney& d)
{
    DisneyG g;
    g.basecolor = DV3{dvar<kGradParams>(d.basecolor.x, GP_BASE_R), dvar<kGradParams>(d.basecolor.y, GP_BASE_G),
                      dvar<kGradParams>(d.basecolor.z, GP_BASE_B)};
    g.metallic = dvar<kGradParams>(d.metallic, GP_METALLIC);
    g.roughness = dvar<kGradParams>(d.roughness, GP_ROUGHNESS);
    const D5 lum = luminance(g.basecolor);
    g.ctint = lum.v > 0.0f ? g.basecolor / lum : dv3(mk(1.0f));
    g.cspec0 = lerp3(mk(1.0f), g.ctint, d.specular_tint);
    g.cspec0 = lerp3(g.cspec0, g.basecolor, g.metallic);
    g.diffuse_weight = (1.0f - g.metallic) * (1.0f - d.spec_trans);
    const float aspect = d.anisotropic > 0 ? sqrtf(1.0f - 0.9f * d.anisotropic) : 1.0f;
    const D5 r2 = g.roughness * g.roughness;
    g.ax = dmax(r2 / aspect, 0.001f);
    g.ay = dmax(r2 * aspect, 0.001f);
    return g;
}

FM_D DV3 dv3_zero() { return dv3(mk(0.0f)); }

// ds_spec_eval
FM_D DV3 dsg_spec(const Disney& d, const DisneyG& g, f3 wo, f3 wi)
{
    if (!same_hemi(wo, wi)) return dv3_zero();
    const f3 wh = normalize(wo + wi);
    const float cos_o = cos_dir(wo), cos_i = cos_dir(wi);
    const float cos_d = dot(wi, wh.z > 0 ? wh : -wh);
    const DV3 f_diel = g.cspec0 * fresnel_dielectric(cos_d, 1.0f, d.ior);
    const float pf = p5(clampf(1.0f - fabsf(cos_d), 0.0f, 1.0f));
    const DV3 f_cond = g.cspec0 + (mk(1.0f) - g.cspec0) * pf;
    const DV3 f = lerp3(d.specular * f_diel, f_cond, g.metallic);
    const D5 D = gtr2_aniso(wh, g.ax, g.ay);
    const D5 G = smith_ggx_aniso(wo, wi, g.ax, g.ay);
    const float den = fabsf(4.0f * cos_i * cos_o);
    if (den == 0.0f) return dv3_zero();
    return f * (D * G / den);
}

// ds_diffuse_eval
FM_D DV3 dsg_diffuse(const Disney& d, const DisneyG& g, f3 wo, f3 wi)
{
    const f3 wh = normalize(wo + wi);
    const float cos_o = fabsf(cos_dir(wo));
    const float cos_i = fabsf(cos_dir(wi));
    const float cos_d = fabsf(dot(wi, wh));
    const DV3 f_lambert = g.basecolor / kPi;
    const float fl = p5(1.0f - cos_i);
    const float fv = p5(1.0f - cos_o);
    const D5 rr = 2.0f * g.roughness * (cos_d * cos_d);
    const DV3 f_retro = f_lambert * (rr * (fl + fv + fl * fv * (rr - 1.0f)));
    const DV3 c_sheen = lerp3(mk(1.0f), g.ctint, d.sheen_tint);
    const DV3 f_sheen = c_sheen * (4.0f * d.sheen * p5(1.0f - cos_d));
    D5 wt = g.diffuse_weight;
    if (d.thin) wt = wt * ((1.0f - d.flatness) * (1.0f - d.diff_trans));
    return f_lambert * (wt * ((1.0f - 0.5f * fl) * (1.0f - 0.5f * fv))) + f_retro + f_sheen;
}

// ds_trans_eval (the lobe's alphas come from spec_trans_roughness, not roughness)
FM_D DV3 dsg_trans(const Disney& d, const DisneyG& g, f3 wo, f3 wi, float ax, float ay, const DV3& c)
{
    if (!opposite_hemi(wo, wi)) return dv3_zero();
    return c * ((1.0f - g.metallic) * (d.spec_trans * ds_trans_ft(d, wo, wi, ax, ay)));
}

// ds_fakess_eval
FM_D DV3 dsg_fakess(const Disney& d, const DisneyG& g, f3 wo, f3 wi)
{
    if (!same_hemi(wo, wi)) return dv3_zero();
    const f3 wh = normalize(wo + wi);
    const float cos_o = fabsf(cos_dir(wo));
    const float cos_i = fabsf(cos_dir(wi));
    const float cos_d = fabsf(dot(wi, wh));
    const D5 fss90 = g.roughness * (cos_d * cos_d);
    const float fo = p5(1.0f - cos_o), fi = p5(1.0f - cos_i);
    const D5 fss = lerpf(fo, 1.0f, fss90) * lerpf(fi, 1.0f, fss90);
    const D5 ss = 1.25f * (fss * (1.0f / (cos_o + cos_i) - 0.5f) + 0.5f);
    const D5 weight = g.diffuse_weight * (d.flatness * (1.0f - d.diff_trans));
    return g.basecolor * (weight * kInvPi * ss);
}

// disney_f on dual numbers; wo, wi in the shading frame
FM_D DV3 disney_f_grad(const Disney& d, const DisneyG& g, f3 wo, f3 wi)
{
    DV3 r = dv3_zero();
    if (wo.z * wi.z < 0) {
        if (d.thin) {
            const DV3 sc = DV3{dsqrt(g.basecolor.x), dsqrt(g.basecolor.y), dsqrt(g.basecolor.z)};
            r = r + dsg_trans(d, g, wo, wi, d.rough_ax, d.rough_ay, sc);
            if (opposite_hemi(wo, wi)) r = r + g.basecolor * d.diff_trans;
        } else {
            r = r + dsg_trans(d, g, wo, wi, d.trans_ax, d.trans_ay, g.basecolor);
        }
        return r;
    }
    if (d.metallic < 1.0f && d.spec_trans < 1.0f) {
        if (d.thin && d.flatness > 0.0f) r = r + dsg_fakess(d, g, wo, wi);
        r = r + dsg_diffuse(d, g, wo, wi);
    }
    r = r + dsg_spec(d, g, wo, wi);
    if (d.clearcoat > 0.0f) r = r + ds_cc_eval(d, wo, wi);
    return r;
}

// ---- sampling densities ---------------------------------------------------------------
//
// A BSDF-sampled direction enters the estimator as f / p, with p the density the
// reference's Pdf reports, while the direction is drawn with the sampler's true density
// q.  For the Disney specular and clearcoat lobes the two differ: the sampler reflects
// wo about a sampled half vector and, when the reflection points below the surface,
// flips it back up (ds_spec_sample / ds_cc_sample), so q(wi) also holds the density of
// the reflection that landed at flipz(wi); Pdf reports only the direct part.  The
// renderer's expected image therefore depends on the parameters through q / p, and its
// exact derivative needs d log q and d log p (and the MIS weights built from p) along
// with df.  Diffuse and Lambert sampling have q = p; the transmission lobes are taken
// to have q = p.

// Lobe weights of disney_setup on duals (the float selection thresholds stay in d).
struct DisneyWG {
    D5 w_dr, w_sr, w_cc, w_st, w_dt;
};

FM_D DisneyWG disney_weights_grad(const Disney& d, const DisneyG& g, float wo_z)
{
    DisneyWG w;
    const D5 lum = luminance(g.basecolor);
    const float fr_approx = fresnel_dielectric(wo_z, 1.0f, d.ior);
    const D5 cspec0_lum = luminance(g.cspec0);
    w.w_dr = lum * g.diffuse_weight * (d.thin ? (1.0f - d.diff_trans) : 1.0f);
    w.w_cc = dconst<kGradParams>(d.clearcoat * 0.25f);
    w.w_sr = (1.0f - fr_approx) * cspec0_lum + fr_approx;   // lerp(cspec0_lum, 1, fr_approx)
    w.w_st = lum * (1.0f - g.metallic) * (d.spec_trans * (1.0f - fr_approx));
    w.w_dt = d.thin ? lum * g.diffuse_weight * d.diff_trans : dconst<kGradParams>(0.0f);
    const D5 inv = 1.0f / (w.w_dr + w.w_sr + w.w_cc + w.w_st + w.w_dt);
    w.w_dr = w.w_dr * inv;
    w.w_sr = w.w_sr * inv;
    w.w_cc = w.w_cc * inv;
    w.w_st = w.w_st * inv;
    w.w_dt = w.w_dt * inv;
    return w;
}

// Density of the reflection sampler at w for half-vector density D(h)|h.z| (either
// hemisphere of w): D |h.z| / (4 |wo.h|), h = normalize(wo + w).
template <class DFN>
FM_D auto reflect_density(f3 wo, f3 w, DFN Dfn) -> decltype(Dfn(w))
{
    const f3 sum = wo + w;
    const float len2 = dot(sum, sum);
    f3 h = len2 > 0.0f ? normalize(sum) : f3{0.0f, 0.0f, 1.0f};
    if (h.z < 0) h = -h;
    const float cd = fabsf(dot(wo, h));
    const float k = (len2 > 0.0f && cd > 0.0f) ? fabsf(h.z) / (4.0f * cd) : 0.0f;
    return Dfn(h) * k;
}

struct PdfQ {
    D5 p;   // density reported by the reference's Pdf (disney_pdf)
    D5 q;   // density the sampler draws with
};

// disney_pdf and the sampler's density at wi, with derivatives (wo, wi local).
FM_D PdfQ disney_pdfs_grad(const Disney& d, const DisneyG& g, f3 wo, f3 wi)
{
    const DisneyWG w = disney_weights_grad(d, g, wo.z);
    const D5 zero = dconst<kGradParams>(0.0f);
    PdfQ r;
    r.p = zero;
    r.q = zero;
    auto spec_D = [&](f3 h) { return gtr2_aniso(h, g.ax, g.ay); };
    auto cc_D = [&](f3 h) { return gtr1(h, d.cc_rough); };
    // reported (disney_pdf / disney_pdf_refl_trans)
    const float fr0 = fresnel_dielectric(wo.z, 1.0f, d.ior);
    const D5 fr = 1.0f - ((1.0f - fr0) * d.spec_trans) * (1.0f - g.metallic);
    const bool same = wo.z * wi.z > 0.0f;
    if (d.w_dr > 0.0f && same) r.p = r.p + w.w_dr * (fabsf(wi.z) * kInvPi);
    if (d.w_cc > 0.0f && same) r.p = r.p + w.w_cc * ds_cc_pdf(d, wo, wi);
    if (d.w_st + d.w_sr > 0.0f) {
        if (same) {
            // ds_spec_pdf with dual alphas
            const f3 wh = normalize(wo + wi);
            const float cos_d = dot(wi, wh.z > 0 ? wh : -wh);
            const D5 D = gtr2_aniso(wh, g.ax, g.ay);
            const D5 ps = D * fabsf(fabsf(cos_dir(wh)) / (4.0f * cos_d));
            r.p = r.p + (w.w_st + w.w_sr) * fr * ps;
        } else if (wo.z * wi.z < 0.0f) {
            r.p = r.p + (w.w_st + w.w_sr) * (1.0f - fr) * ds_trans_pdf(d, wo, wi);
        }
    }
    if (d.w_dt > 0.0f && wo.z * wi.z < 0.0f) r.p = r.p + w.w_dt * (fabsf(wi.z) * kInvPi);
    // sampler: lobe choice by the thresholds of disney_sample_dir (diffuse, clearcoat,
    // diffuse transmission, then specular reflection while u.z <= fr, else transmission)
    const D5 c_dt = w.w_dr + w.w_cc + w.w_dt;
    D5 p_spec = fr - c_dt;
    if (fr.v > 1.0f) p_spec = 1.0f - c_dt;
    if (p_spec.v < 0.0f) p_spec = zero;
    const D5 p_trans = (1.0f - c_dt) - p_spec;
    if (same) {
        r.q = r.q + w.w_dr * (fabsf(wi.z) * kInvPi);
        const f3 wf = flipz(wi);
        r.q = r.q + w.w_cc * (reflect_density(wo, wi, cc_D) + reflect_density(wo, wf, cc_D));
        r.q = r.q + p_spec * (reflect_density(wo, wi, spec_D) + reflect_density(wo, wf, spec_D));
    } else if (wo.z * wi.z < 0.0f) {
        r.q = r.q + w.w_dt * (fabsf(wi.z) * kInvPi);
        if (d.w_st + d.w_sr > 0.0f) r.q = r.q + p_trans * ds_trans_pdf(d, wo, wi);
    }
    return r;
}

// Everything the adjoint needs at one sampled direction, from one parameter set-up:
// df/dp per channel, d log pdf_b/dp (pdf_b the density the reference's Pdf reports)
// and d log q/dp - d log pdf_b/dp (q the sampler's density).
struct BsdfGrads {
    DV3 f;
    float dlogp[kGradParams];
    float dscore[kGradParams];
};

// Not inlined: the replay shading kernel calls it for every NEE, MIS and continuation
// direction, and one copy keeps its code and register use down.
FM_D void disney_grads(const Disney& d, f3 wo, f3 wi, BsdfGrads* out)
{
    const DisneyG g = disney_grad_setup(d);
    out->f = disney_f_grad(d, g, wo, wi);
    const PdfQ pq = disney_pdfs_grad(d, g, wo, wi);
    const bool ok = pq.p.v > 0.0f && pq.q.v > 0.0f;
    for (int i = 0; i < kGradParams; ++i) {
        out->dlogp[i] = ok ? pq.p.d[i] / pq.p.v : 0.0f;
        out->dscore[i] = ok ? pq.q.d[i] / pq.q.v - out->dlogp[i] : 0.0f;
    }
}

// bsdf_f with derivatives, and the density terms (zero where the sampler draws the
// reported density).  Lambert: f = basecolor / pi; conductor and dielectric have no
// differentiated parameters (and a zero non-delta value).
template <int CLS = kClsAny>
FM_D void bsdf_grads(const Bsdf& b, f3 wo_w, f3 wi_w, BsdfGrads& out)
{
    if (CLS != kClsDisney && (b.type != 3 || CLS == kClsSimple)) {
        out.f = b.type == 0 ? dv3(b.color * kInvPi) : dv3_zero();
        if (b.type == 0) {
            out.f.x.d[GP_BASE_R] = kInvPi;
            out.f.y.d[GP_BASE_G] = kInvPi;
            out.f.z.d[GP_BASE_B] = kInvPi;
        }
        for (int i = 0; i < kGradParams; ++i) out.dlogp[i] = out.dscore[i] = 0.0f;
        return;
    }
    disney_grads(b.d, to_local(b, wo_w), to_local(b, wi_w), &out);
}

// sum_c w_c * dF_c / dp_i for the five parameters
FM_D void contract(const DV3& F, f3 w, float g[kGradParams])
{
#pragma unroll
    for (int i = 0; i < kGradParams; ++i) g[i] = w.x * F.x.d[i] + w.y * F.y.d[i] + w.z * F.z.d[i];
}

}  // namespace fm
