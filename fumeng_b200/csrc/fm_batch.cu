// Batched rendering (many views / scenes in one persistent wavefront) and the autotuner.
#include <algorithm>
#include <cmath>
#include <vector>

#include "fm_render.h"
#include "fm_staging.h"

namespace fm {

namespace {

std::tuple<int, int, int> shape_class(int n, const fm_render_params* params, const fm_scene* const* scenes)
{
    double samples = 0.0;
    int lights = 0;
    for (int i = 0; i < n; ++i) {
        samples += (double)out_width(params[i]) * out_height(params[i]) * params[i].spp;
        lights = std::max(lights, scenes[i]->dev.num_lights);
    }
    return {n, (int)std::floor(std::log2(std::max(1.0, samples))), lights};
}

WfTuning to_wf(const fm_tuning& t)
{
    WfTuning w;
    w.pool = t.pool;
    w.trace_block = t.trace_block;
    w.shade_block = t.shade_block;
    w.iters_per_graph = t.iters_per_graph;
    w.max_iterations = t.max_iterations;
    w.queue_limit = t.queue_limit;
    return w;
}

fm_status check_tuning(fm_ctx* ctx, const fm_tuning& t)
{
    auto okb = [](int b) { return b == 32 || b == 64 || b == 128 || b == 256; };
    if (t.pool < 1024 || t.pool > ((int64_t)1 << 26) || !okb(t.trace_block) || !okb(t.shade_block) ||
        t.iters_per_graph < 1 || t.iters_per_graph > 64 || t.max_iterations < 0 || t.queue_limit < 0)
        return set_error(ctx, FM_ERR_INVALID, "tuning out of range");
    return FM_OK;
}

// Views rendering into the given device images (spp overridden when spp_override > 0).
std::vector<WfView> make_views(int n, const fm_scene* const* scenes, const fm_camera* cams, const fm_render_params* params,
                               float* const* rgb, float* const* alb, float* const* nrm, int spp_override)
{
    std::vector<WfView> v((size_t)n);
    for (int i = 0; i < n; ++i) {
        WfView& w = v[i];
        w = WfView{};
        w.scene = scenes[i]->d_dev;
        w.num_lights = scenes[i]->dev.num_lights;
        w.cam = make_camera(cams[i]);
        fm_render_params p = params[i];
        if (spp_override > 0) p.spp = std::min(p.spp, spp_override);
        w.cfg = make_cfg(p);
        w.rgb = rgb[i];
        w.alb = alb ? alb[i] : nullptr;
        w.nrm = nrm ? nrm[i] : nullptr;
    }
    return v;
}

fm_status validate_batch(fm_ctx* ctx, int32_t n, const fm_scene* const* scenes, const fm_camera* cams,
                         const fm_render_params* params)
{
    if (n <= 0 || !scenes || !cams || !params) return set_error(ctx, FM_ERR_INVALID, "batch: bad arguments");
    for (int i = 0; i < n; ++i) {
        fm_status st = validate_render(ctx, scenes[i], &cams[i], &params[i]);
        if (st != FM_OK) return st;
        if (params[i].mode != params[0].mode) return set_error(ctx, FM_ERR_INVALID, "batch: all views must use one mode");
    }
    return FM_OK;
}

fm_status autotune(fm_ctx* ctx, int32_t n, const fm_scene* const* scenes, const fm_camera* cams,
                   const fm_render_params* params, fm_tuning* out)
{
    // scratch images for the trial renders
    std::vector<float*> imgs((size_t)n, nullptr);
    size_t total = 0;
    for (int i = 0; i < n; ++i) total += (size_t)out_width(params[i]) * out_height(params[i]) * 3;
    float* buf = nullptr;
    FM_CUDA_TRY(ctx, cudaMalloc(&buf, total * sizeof(float)), "autotune alloc");
    Counters* cnt = nullptr;
    if (cudaMalloc(&cnt, sizeof(Counters)) != cudaSuccess) {
        cudaFree(buf);
        return set_error(ctx, FM_ERR_OOM, "autotune alloc");
    }
    size_t off = 0;
    for (int i = 0; i < n; ++i) {
        imgs[i] = buf + off;
        off += (size_t)out_width(params[i]) * out_height(params[i]) * 3;
    }
    // Trial renders of the batch itself when it has at most 2^28 samples (a trial then
    // takes well under a second), else at up to 8 spp per view.  The best pool depends
    // on the samples a render has: at 8 spp the 64-scene batch favoured 2^23 slots, its
    // full render 2^25 (302 against 349 ms); at 2 spp it favoured smaller pools still.
    double full_samples = 0.0;
    for (int i = 0; i < n; ++i) full_samples += (double)out_width(params[i]) * out_height(params[i]) * params[i].spp;
    const int trial_spp = full_samples <= (double)(1 << 28) ? 0 : 8;
    const std::vector<WfView> views = make_views(n, scenes, cams, params, imgs.data(), nullptr, nullptr, trial_spp);
    double samples = 0.0;
    for (const auto& v : views) samples += (double)v.cfg.width * v.cfg.height * v.cfg.spp;
    fm_tuning best{(int64_t)1 << 21, 128, 128, 8, 0, 0};
    double best_rate = -1.0;
    fm_status st = FM_OK;
    // each candidate's faster of two renders, so that one slow render does not decide
    auto trial = [&](fm_tuning t) -> fm_status {
        double ms = 1e30;
        for (int rep = 0; rep < 2; ++rep) {
            WfTimes tm;
            cudaMemsetAsync(cnt, 0, sizeof(Counters), ctx->stream);
            fm_status s = wavefront_views(ctx, views, to_wf(t), cnt, &tm);
            if (s != FM_OK) return s;
            ms = std::min(ms, tm.total_ms);
        }
        const double rate = samples / std::max(ms, 1e-3);
        if (rate > best_rate) {
            best_rate = rate;
            best = t;
        }
        return FM_OK;
    };
    // Pools up to 2^25 slots: on the 64-scene batch (250 M paths) a render ran 368 /
    // 333 / 302 / 307 ms at 2^22 / 2^24 / 2^25 / 2^26 slots -- a larger pool means fewer
    // wavefront iterations, so fewer launches and fewer kernel tails.  A candidate's
    // workspace (about 284 B plus 52 B per light and direct-lighting round per slot) must
    // fit in half of the device memory free now.
    int max_rays = 1;
    for (const auto& v : views) max_rays = std::max(max_rays, v.num_lights * v.cfg.direct_loop);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        free_b = 0;
    }
    const double slot_bytes = 284.0 + 52.0 * max_rays + 64.0;
    const double pool_cap = 0.5 * (double)free_b / slot_bytes;
    // warm-up, then coordinate descent over pool size, trace block, shade block, graph depth
    st = trial(best);
    best_rate = -1.0;
    const int64_t pools[] = {(int64_t)1 << 19, (int64_t)1 << 20, (int64_t)1 << 21, (int64_t)1 << 22,
                             (int64_t)1 << 23, (int64_t)1 << 24, (int64_t)1 << 25};
    for (int64_t p : pools) {
        if (st != FM_OK) break;
        if (((double)p > samples * 2.0 || (double)p > pool_cap) && p != pools[0]) continue;
        fm_tuning t = best;
        t.pool = p;
        st = trial(t);
    }
    for (int b : {64, 128, 256}) {
        if (st != FM_OK) break;
        fm_tuning t = best;
        t.trace_block = b;
        st = trial(t);
    }
    for (int b : {64, 128, 256}) {
        if (st != FM_OK) break;
        fm_tuning t = best;
        t.shade_block = b;
        st = trial(t);
    }
    for (int k : {4, 8, 16}) {
        if (st != FM_OK) break;
        fm_tuning t = best;
        t.iters_per_graph = k;
        st = trial(t);
    }
    cudaFree(buf);
    cudaFree(cnt);
    if (st != FM_OK) return st;
    *out = best;
    return FM_OK;
}

}  // namespace

}  // namespace fm

using namespace fm;

extern "C" fm_status fm_autotune_batch(fm_ctx* ctx, int32_t n, const fm_scene* const* scenes, const fm_camera* cameras,
                                       const fm_render_params* params, fm_tuning* out)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!out) return set_error(ctx, FM_ERR_INVALID, "autotune: null output");
    fm_status st = validate_batch(ctx, n, scenes, cameras, params);
    if (st != FM_OK) return st;
    FM_CUDA_TRY(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    st = autotune(ctx, n, scenes, cameras, params, out);
    if (st == FM_OK) ctx->tune_cache[shape_class(n, params, scenes)] = *out;
    return st;
}

extern "C" fm_status fm_render_batch(fm_ctx* ctx, int32_t n, const fm_scene* const* scenes, const fm_camera* cameras,
                                     const fm_render_params* params, float* const* rgb, float* const* albedo,
                                     float* const* normal, int32_t flags, const fm_tuning* tuning,
                                     fm_render_stats* stats)
{
    if (!ctx) return FM_ERR_INVALID;
    fm_status st = validate_batch(ctx, n, scenes, cameras, params);
    if (st != FM_OK) return st;
    if (!rgb) return set_error(ctx, FM_ERR_INVALID, "batch: rgb is null");
    for (int i = 0; i < n; ++i)
        if (!rgb[i]) return set_error(ctx, FM_ERR_INVALID, "batch: rgb entry is null");
    FM_CUDA_TRY(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    const bool dev = (flags & FM_FLAG_DEVICE_PTRS) != 0;
    const bool wave = params[0].mode == FM_MODE_WAVEFRONT;
    fm_tuning tune{(int64_t)1 << 21, 128, 128, 8, 0, 0};
    if (wave) {
        if (tuning) {
            st = check_tuning(ctx, *tuning);
            if (st != FM_OK) return st;
            tune = *tuning;
        } else {
            const auto key = shape_class(n, params, scenes);
            auto it = ctx->tune_cache.find(key);
            if (it == ctx->tune_cache.end()) {
                st = autotune(ctx, n, scenes, cameras, params, &tune);
                if (st != FM_OK) return st;
                ctx->tune_cache[key] = tune;
            } else {
                tune = it->second;
            }
        }
    }
    // device images (staging when the caller passed host buffers)
    std::vector<float*> d_rgb((size_t)n), d_alb((size_t)n, nullptr), d_nrm((size_t)n, nullptr);
    std::vector<size_t> bytes((size_t)n);
    char* staging = nullptr;
    size_t total = 0;
    for (int i = 0; i < n; ++i) {
        bytes[i] = (size_t)out_width(params[i]) * out_height(params[i]) * 3 * sizeof(float);
        if (!dev) total += bytes[i] * (1 + (albedo && albedo[i] ? 1 : 0) + (normal && normal[i] ? 1 : 0));
    }
    Counters* d_cnt = nullptr;
    FM_CUDA_TRY(ctx, cudaMallocAsync((void**)&staging, total + 256, ctx->stream), "batch alloc");
    d_cnt = reinterpret_cast<Counters*>(staging);
    {
        char* q = staging + 256;
        for (int i = 0; i < n; ++i) {
            if (dev) {
                d_rgb[i] = rgb[i];
                d_alb[i] = albedo ? albedo[i] : nullptr;
                d_nrm[i] = normal ? normal[i] : nullptr;
                continue;
            }
            d_rgb[i] = reinterpret_cast<float*>(q);
            q += bytes[i];
            if (albedo && albedo[i]) {
                d_alb[i] = reinterpret_cast<float*>(q);
                q += bytes[i];
            }
            if (normal && normal[i]) {
                d_nrm[i] = reinterpret_cast<float*>(q);
                q += bytes[i];
            }
        }
    }
    FM_CUDA_TRY(ctx, cudaMemsetAsync(d_cnt, 0, sizeof(Counters), ctx->stream), "batch");
    FM_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream), "batch");
    double ms = 0.0;
    WfTimes tm;
    if (wave) {
        const std::vector<WfView> views = make_views(n, scenes, cameras, params, d_rgb.data(), d_alb.data(), d_nrm.data(), 0);
        WfTuning wt = to_wf(tune);
        wt.profile = (flags & FM_FLAG_PROFILE) != 0;
        st = wavefront_views(ctx, views, wt, d_cnt, &tm);
        ms = tm.total_ms;
    } else {
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, ctx->stream);
        st = megakernel_views(ctx, make_views(n, scenes, cameras, params, d_rgb.data(), d_alb.data(), d_nrm.data(), 0),
                              d_cnt);
        cudaEventRecord(e1, ctx->stream);
        cudaEventSynchronize(e1);
        float f = 0.0f;
        cudaEventElapsedTime(&f, e0, e1);
        ms = f;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    cudaError_t ecopy = cudaSuccess;
    if (st == FM_OK && !dev) {
        std::vector<OutCopy> out;
        for (int i = 0; i < n; ++i) {
            out.push_back(OutCopy{rgb[i], d_rgb[i], bytes[i]});
            if (d_alb[i]) out.push_back(OutCopy{albedo[i], d_alb[i], bytes[i]});
            if (d_nrm[i]) out.push_back(OutCopy{normal[i], d_nrm[i], bytes[i]});
        }
        ecopy = copy_out(ctx, ctx->stream, out);
    }
    Counters hc{};
    uint32_t hs = 0;
    cudaMemcpyAsync(&hc, d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream);
    cudaMemcpyAsync(&hs, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream);
    cudaFreeAsync(staging, ctx->stream);
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (st != FM_OK) return st;
    if (ecopy != cudaSuccess) return cuda_error(ctx, ecopy, "batch: image copy");
    if (e != cudaSuccess) return cuda_error(ctx, e, "batch");
    if (stats) {
        stats->paths = (int64_t)hc.paths;
        stats->closest_rays = (int64_t)hc.closest;
        stats->shadow_rays = (int64_t)hc.shadow;
        stats->bounces = (int64_t)hc.bounces;
        stats->nan_samples = (int64_t)hc.nans;
        stats->kernel_ms = ms;
        stats->trace_ms = tm.trace_ms;
        stats->shade_ms = tm.shade_ms;
        stats->launches = wave ? tm.launches : 1 + (int64_t)n;
    }
    if (hs & 1u) return set_error(ctx, FM_ERR_QUEUE_OVERFLOW, "batch: traversal stack overflow");
    if (hs & 2u) return set_error(ctx, FM_ERR_QUEUE_OVERFLOW, "batch: wavefront queue overflow");
    return FM_OK;
}
