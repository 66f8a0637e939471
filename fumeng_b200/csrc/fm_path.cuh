// One camera path, written as the reference's PathTracer::RenderPixel
// (renderer/path_tracing.cpp:34-117) with MisLight (:122-161) and MisBSDF (:166-229).
// Used by the plain per-pixel megakernel; the wavefront kernels split the same steps
// across launches.
#pragma once
#include "fm_integrator.cuh"

namespace fm {

struct PathOut {
    f3 color, albedo, normal;
    int closest, shadow, bounces;
};

// The path's large steps are called, not inlined: a lane of a warp may be sampling a
// Disney lobe while its neighbour evaluates a dielectric or traverses the BVH, and with
// every call site inlined the kernel's code outgrows the instruction caches (most issue
// slots then wait for instruction fetch).  One copy each of BSDF sampling, hit
// construction, next-event estimation and the MIS-BSDF step keeps the loop compact.
static __device__ __noinline__ BsdfSample path_bsdf_sample(const Bsdf& b, f3 wo, f3 u) { return bsdf_sample(b, wo, u); }
static __device__ __noinline__ HitInfo path_make_hit(const DevScene& S, f3 o, f3 d, const Hit& hit)
{
    return make_hit(S, o, d, hit);
}

// MisLight: NEE for one light.  The BSDF value and pdf are evaluated before the shadow
// ray (the reference traces first), which skips rays whose contribution is zero without
// changing any result.
static __device__ __noinline__ f3 mis_light(const DevScene& S, const DevLight& L, const HitInfo& h, const Bsdf& b,
                                            f3 u, int& nshadow, uint32_t* status)
{
    LightSample ls;
    if (!light_sample(S, L, h.pos, u, ls)) return mk(0.0f);
    if (ls.pdf < kEpsPdf || length(ls.radiance) < kEpsPdf) return mk(0.0f);
    const f3 f = bsdf_f(b, h.wo, ls.wi);
    if (length(f) < kEpsPdf) return mk(0.0f);
    const float pb = bsdf_pdf(b, h.wo, ls.wi);
    if (pb < kEpsPdf) return mk(0.0f);
    Hit sh;
    ++nshadow;
    if (trace_ray<true>(S, h.pos, ls.wi, kEps, ls.dist - kEps, sh, status)) return mk(0.0f);
    const f3 c = f * ls.radiance * absdot(ls.wi, h.ng);
    if (ls.delta) return c / ls.pdf;
    return c / ls.pdf * power_heuristic(ls.pdf, pb);
}

// MisBSDF: a separate BSDF sample, traced to an emitter or the environment.
static __device__ __noinline__ f3 mis_bsdf(const DevScene& S, const HitInfo& h, const Bsdf& b, f3 u, int& nclosest,
                                           uint32_t* status)
{
    const BsdfSample s = path_bsdf_sample(b, h.wo, u);
    if (length(s.f) < kEpsPdf || s.pdf < kEpsPdf) return mk(0.0f);
    const f3 wi = normalize(s.wi);
    const f3 ro = spawn_origin(h, wi);
    Hit lh;
    ++nclosest;
    if (!trace_ray<false>(S, ro, wi, 0.0f, kRealMax, lh, status)) {
        if (S.env_light < 0) return mk(0.0f);
        const f3 rad = env_radiance(S, wi);
        const f3 f = s.f * rad * absdot(wi, h.ng);
        if (s.delta) return f / s.pdf;
        return f / s.pdf * power_heuristic(s.pdf, env_pdf(S, wi));
    }
    const int obj = __ldg(S.prim_obj + lh.prim);
    const int li = __ldg(S.obj_light + obj);
    if (li < 0) return mk(0.0f);
    const HitInfo lhit = path_make_hit(S, ro, wi, lh);
    const f3 l2s = normalize(ro - lhit.pos);
    const DevLight& L = S.lights[li];
    const f3 rad = dot(lhit.ng, l2s) > 0 ? ld3(L.radiance) : mk(0.0f);
    if (length(rad) < kEpsPdf) return mk(0.0f);
    const f3 f = s.f * rad * absdot(h.ng, wi);
    if (s.delta) return f / s.pdf;
    return f / s.pdf * power_heuristic(s.pdf, area_light_pdf(S, L, ro, lhit.pos, lhit.ng, l2s));
}

FM_D PathOut trace_path(const DevScene& S, const RenderCfg& cfg, f3 o, f3 d, Rng& rng, uint32_t* status)
{
    PathOut out;
    out.color = out.albedo = out.normal = mk(0.0f);
    out.closest = out.shadow = out.bounces = 0;
    f3 beta = mk(1.0f);
    const f3 cam_dir = d;
    for (int depth = 1; depth <= cfg.depth; ++depth) {
        Hit hit;
        ++out.closest;
        if (!trace_ray<false>(S, o, d, 0.0f, kRealMax, hit, status)) {
            if (depth == 1 && S.env_light >= 0) out.color = env_radiance(S, cam_dir);
            break;
        }
        const HitInfo h = path_make_hit(S, o, d, hit);
        if (depth == 1) {
            const int li = __ldg(S.obj_light + h.obj);
            if (li >= 0) {
                const f3 rad = dot(h.ng, h.wo) > 0 ? ld3(S.lights[li].radiance) : mk(0.0f);
                out.color += beta * rad;
                break;
            }
        }
        ++out.bounces;
        const Bsdf b = make_bsdf(S, h);
        if (depth == 1) {
            out.albedo = bsdf_albedo(b);
            out.normal = h.ng;
        }
        f3 direct = mk(0.0f);
        for (int k = 0; k < cfg.direct_loop; ++k) {
            for (int l = 0; l < S.num_lights; ++l)
                direct += beta * mis_light(S, S.lights[l], h, b, rng_3d(rng), out.shadow, status);
            direct += beta * mis_bsdf(S, h, b, rng_3d(rng), out.closest, status);
        }
        out.color += direct / (float)cfg.direct_loop;
        const BsdfSample s = path_bsdf_sample(b, h.wo, rng_3d(rng));
        if (length(s.f) < kEpsPdf || s.pdf < kEpsPdf) break;
        beta *= s.f * absdot(h.ng, s.wi) / s.pdf;
        o = spawn_origin(h, s.wi);
        d = s.wi;
        if (cfg.rr_enabled) {
            if (rng_1d(rng) > cfg.rr_coef) break;
            beta /= cfg.rr_coef;
        }
    }
    return out;
}

}  // namespace fm
