// Texture fetch and environment-map lookup.
#pragma once
#include "fm_common.cuh"
#include "fm_scene.cuh"

namespace fm {

// Texture::WrapClamp / WrapRepeat (core/texture.h:88-96).
FM_D float wrap_coord(float x, int mode)
{
    if (mode == 1) return clampf(x, 0.0f, 1.0f);
    return clampf(x - floorf(x), 0.0f, 1.0f);
}

FM_D f3 texel(const DevTexture& t, int x, int y)
{
    const float4 v = __ldg(t.texels + (size_t)y * t.w + x);
    return f3{v.x, v.y, v.z};
}

// Texture::Sample -> ImageTexture::LinearSample / NearestSample
// (texture/image_texture.cpp:13-44): bilinear taps are clamped at the border, never
// wrapped.
FM_D f3 tex_sample(const DevTexture& t, float uu, float vv)
{
    const float u = wrap_coord(uu, t.wrap_u);
    const float v = wrap_coord(vv, t.wrap_v);
    const float ru = u * (float)t.w;
    const float rv = v * (float)t.h;
    if (t.filter == 1) {
        int x = (int)ru, y = (int)rv;
        x = x < 0 ? 0 : (x > t.w - 1 ? t.w - 1 : x);
        y = y < 0 ? 0 : (y > t.h - 1 ? t.h - 1 : y);
        return texel(t, x, y);
    }
    const int u0 = (int)clampf(ru - 0.5f, 0.0f, (float)(t.w - 1));
    const int u1 = min(u0 + 1, t.w - 1);
    const float pu = clampf(ru - 0.5f - (float)u0, 0.0f, 1.0f);
    const int v0 = (int)clampf(rv - 0.5f, 0.0f, (float)(t.h - 1));
    const int v1 = min(v0 + 1, t.h - 1);
    const float pv = clampf(rv - 0.5f - (float)v0, 0.0f, 1.0f);
    const f3 a = texel(t, u0, v0), b = texel(t, u1, v0), c = texel(t, u0, v1), d = texel(t, u1, v1);
    return (a * (1.0f - pu) + b * pu) * (1.0f - pv) + (c * (1.0f - pu) + d * pu) * pv;
}

// The texels tex_sample reads at (uu, vv) and their weights (the same taps; the
// weights are the bilinear products), for scattering derivatives back onto texels.
struct TexTaps {
    int x[4], y[4];
    float w[4];
    int n;
};

FM_D TexTaps tex_taps(const DevTexture& t, float uu, float vv)
{
    TexTaps r;
    const float u = wrap_coord(uu, t.wrap_u);
    const float v = wrap_coord(vv, t.wrap_v);
    const float ru = u * (float)t.w;
    const float rv = v * (float)t.h;
    if (t.filter == 1) {
        int x = (int)ru, y = (int)rv;
        r.x[0] = x < 0 ? 0 : (x > t.w - 1 ? t.w - 1 : x);
        r.y[0] = y < 0 ? 0 : (y > t.h - 1 ? t.h - 1 : y);
        r.w[0] = 1.0f;
        r.n = 1;
        return r;
    }
    const int u0 = (int)clampf(ru - 0.5f, 0.0f, (float)(t.w - 1));
    const int u1 = min(u0 + 1, t.w - 1);
    const float pu = clampf(ru - 0.5f - (float)u0, 0.0f, 1.0f);
    const int v0 = (int)clampf(rv - 0.5f, 0.0f, (float)(t.h - 1));
    const int v1 = min(v0 + 1, t.h - 1);
    const float pv = clampf(rv - 0.5f - (float)v0, 0.0f, 1.0f);
    r.x[0] = u0, r.y[0] = v0, r.w[0] = (1.0f - pu) * (1.0f - pv);
    r.x[1] = u1, r.y[1] = v0, r.w[1] = pu * (1.0f - pv);
    r.x[2] = u0, r.y[2] = v1, r.w[2] = (1.0f - pu) * pv;
    r.x[3] = u1, r.y[3] = v1, r.w[3] = pu * pv;
    r.n = 4;
    return r;
}

// GetSphericalUV (core/utils.h:149-173): z-up, u = phi / 2pi, v = theta / pi.
FM_D void spherical_uv(f3 d, float& u, float& v, float& theta)
{
    theta = acosf(clampf(d.z, -1.0f, 1.0f));
    float phi = atan2f(d.y, d.x);
    if (phi < 0) phi += 2.0f * kPi;
    u = phi * kInvPi * 0.5f;
    v = theta * kInvPi;
}

// EnvLight::GetRadiance for a world direction `dir` pointing from the scene toward the
// sky (env_light.cpp:51-55 with light_to_shd = -dir).
FM_D f3 env_radiance(const DevScene& S, f3 dir)
{
    const DevEnv& E = S.env;
    float u, v, th;
    spherical_uv(xf_vec(E.w2l, dir), u, v, th);
    return E.factor * tex_sample(S.textures[E.tex], u, v);
}

// EnvLight::Pdf(dir) (env_light.cpp:58-61 -> env_importance_sampler.h:84-94 ->
// distribution_2d.cpp:42-58), reproducing its normalisation: the density it reports is
// the conditional density of u given v divided by the marginal's sum, without the
// marginal density of v.  The table pdf_eval holds exactly that per texel.
FM_D float env_pdf(const DevScene& S, f3 dir)
{
    const DevEnv& E = S.env;
    float u, v, th;
    spherical_uv(xf_vec(E.w2l, dir), u, v, th);
    const float st = sinf(th);
    if (st == 0.0f) return 0.0f;
    int iu = (int)(u * (float)E.w);
    int iv = (int)(v * (float)E.h);
    iu = iu < 0 ? 0 : (iu > E.w - 1 ? E.w - 1 : iu);
    iv = iv < 0 ? 0 : (iv > E.h - 1 ? E.h - 1 : iv);
    return __ldg(E.pdf_eval + (size_t)iv * E.w + iu) / (2.0f * kPi * kPi * st);
}

// Alias-table draw: index in [0, n) from a uniform x; `rem` returns a fresh uniform in
// [0, 1) recovered from the unused part of x.
FM_D int alias_draw(const float* prob, const int32_t* alias, int n, float x, float& rem)
{
    const float s = x * (float)n;
    int i = (int)s;
    if (i > n - 1) i = n - 1;
    float f = s - (float)i;
    const float p = __ldg(prob + i);
    if (f < p) {
        rem = p > 0.0f ? f / p : 0.0f;
        return i;
    }
    rem = p < 1.0f ? (f - p) / (1.0f - p) : 0.0f;
    return __ldg(alias + i);
}

// EnvLight::Sample (env_light.cpp:38-44): the texel is chosen from the 2-D
// piecewise-constant distribution (marginal over rows, conditional within the row) with
// alias tables instead of the reference's CDF binary search, which changes only the
// mapping from random numbers to directions; the density per texel is the reference's.
FM_D bool env_sample(const DevScene& S, f3 smp, f3& wi, float& pdf, f3& radiance)
{
    const DevEnv& E = S.env;
    float rv, ru;
    const int j = alias_draw(E.marg_prob, E.marg_alias, E.h, smp.x, rv);
    const int i = alias_draw(E.row_prob + (size_t)j * E.w, E.row_alias + (size_t)j * E.w, E.w, smp.y, ru);
    const float u = ((float)i + ru) / (float)E.w;
    const float v = ((float)j + rv) / (float)E.h;
    const float phi = u * 2.0f * kPi;
    const float theta = v * kPi;
    float sp, cp, st, ct;
    sincosf(phi, &sp, &cp);
    sincosf(theta, &st, &ct);
    if (st == 0.0f) return false;
    pdf = __ldg(E.pdf_sample + (size_t)j * E.w + i) / (2.0f * kPi * kPi * st);
    wi = xf_vec(E.l2w, f3{st * cp, st * sp, ct});
    radiance = env_radiance(S, wi);
    return true;
}

}  // namespace fm
