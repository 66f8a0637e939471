// Rendering: the plain per-pixel megakernel and the fm_render entry point.
#include <algorithm>
#include <array>
#include <cmath>
#include <vector>

#include "fm_internal.h"
#include "fm_path.cuh"
#include "fm_render.h"
#include "fm_staging.h"

namespace fm {

namespace {

FM_D void kahan_add(f3& sum, f3& c, f3 x)
{
    f3 y = x - c;
    f3 t = sum + y;
    c = (t - sum) - y;
    sum = t;
}

// Called once per thread after its loop, by all 32 lanes of the warp.
FM_D void add_counters(Counters* cnt, unsigned long long paths, unsigned long long closest, unsigned long long shadow,
                       unsigned long long bounces, unsigned long long nans)
{
    for (int off = 16; off > 0; off >>= 1) {
        paths += __shfl_xor_sync(0xffffffffu, paths, off);
        closest += __shfl_xor_sync(0xffffffffu, closest, off);
        shadow += __shfl_xor_sync(0xffffffffu, shadow, off);
        bounces += __shfl_xor_sync(0xffffffffu, bounces, off);
        nans += __shfl_xor_sync(0xffffffffu, nans, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&cnt->paths, paths);
        atomicAdd(&cnt->closest, closest);
        atomicAdd(&cnt->shadow, shadow);
        atomicAdd(&cnt->bounces, bounces);
        atomicAdd(&cnt->nans, nans);
    }
}

// Plain megakernel: each thread runs whole camera paths (the reference's per-sample
// RenderPixel inside DrawFrame's pixel task, renderer.h:97-116), one sample after
// another, with no queues.  Work items are (view, pixel, chunk of consecutive samples)
// over every view of the call, numbered and laid out like the wavefront's items (chunk
// index major, then pixel, so a warp's lanes take neighbouring pixels); threads are
// persistent and each takes its next item from a global counter as soon as it finishes
// one, so one launch covers a whole batch and no SM idles while others have work.  Each
// item writes its Kahan-compensated colour sum and its albedo / normal sums once; the
// per-pixel reduction (reduce_views) adds the chunks in order, so the image does not
// depend on which thread ran which item.
__global__ void __launch_bounds__(128, 4) k_megakernel(const WfView* __restrict__ views, int nviews, int64_t total_items,
                                                    unsigned long long* next, Counters* cnt, uint32_t* status)
{
    unsigned long long np = 0, nc = 0, ns = 0, nb = 0, nn = 0;
    for (;;) {
        const int64_t it = (int64_t)atomicAdd(next, 1ull);
        if (it >= total_items) break;
        int lo = 0, hi = nviews - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (views[mid].item_base <= it)
                lo = mid;
            else
                hi = mid - 1;
        }
        const WfView& V = views[lo];
        const RenderCfg cfg = V.cfg;
        const int npix = cfg.width * cfg.height;
        const int64_t local = it - V.item_base;
        const int c = (int)(local / npix);
        const PixelRef pr = pixel_ref(cfg, (int)(local % npix));
        const int first = c * V.chunk;
        const int n = min(V.chunk, cfg.spp - first);
        f3 sum = mk(0.0f), comp = mk(0.0f), asum = mk(0.0f), nsum = mk(0.0f);
        for (int k = 0; k < n; ++k) {
            Rng rng = rng_for(cfg.seed, pr.key, (uint64_t)(cfg.sample_offset + first + k));
            const float fx = rng_1d(rng), fy = rng_1d(rng);
            const float lx = rng_1d(rng), ly = rng_1d(rng);
            const float px = ((float)pr.i + fx) / (float)cfg.img_w;
            const float py = ((float)pr.j + fy) / (float)cfg.img_h;
            f3 o, d;
            camera_ray(V.cam, px, py, lx, ly, o, d);
            const PathOut po = trace_path(*V.scene, cfg, o, d, rng, status);
            if (!isfinite(po.color.x) || !isfinite(po.color.y) || !isfinite(po.color.z)) ++nn;
            kahan_add(sum, comp, clamp_sample(cfg, po.color));
            asum += po.albedo;
            nsum += po.normal;
            nc += po.closest;
            ns += po.shadow;
            nb += po.bounces;
        }
        float4* P = V.partial + 3 * (size_t)local;
        P[0] = make_float4(sum.x, sum.y, sum.z, 0.0f);
        P[1] = make_float4(asum.x, asum.y, asum.z, 0.0f);
        P[2] = make_float4(nsum.x, nsum.y, nsum.z, 0.0f);
        np += (unsigned long long)n;
    }
    add_counters(cnt, np, nc, ns, nb, nn);
}

}  // namespace

DevCamera make_camera(const fm_camera& c)
{
    // camera_to_world = inverse(lookAt_LH(pos, look_at, normalize(up)))
    // (pin_hole_camera.cpp:5-16): columns s, u, f and translation pos.
    auto v = [](const float* a) { return std::array<double, 3>{a[0], a[1], a[2]}; };
    auto sub = [](std::array<double, 3> a, std::array<double, 3> b) {
        return std::array<double, 3>{a[0] - b[0], a[1] - b[1], a[2] - b[2]};
    };
    auto nrm = [](std::array<double, 3> a) {
        const double l = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        return std::array<double, 3>{a[0] / l, a[1] / l, a[2] / l};
    };
    auto crs = [](std::array<double, 3> a, std::array<double, 3> b) {
        return std::array<double, 3>{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    };
    const auto pos = v(c.pos), at = v(c.look_at), up = nrm(v(c.up));
    const auto f = nrm(sub(at, pos));
    const auto s = nrm(crs(up, f));
    const auto u = crs(f, s);
    DevCamera d;
    d.pos = f3{c.pos[0], c.pos[1], c.pos[2]};
    d.s = f3{(float)s[0], (float)s[1], (float)s[2]};
    d.u = f3{(float)u[0], (float)u[1], (float)u[2]};
    d.f = f3{(float)f[0], (float)f[1], (float)f[2]};
    const float fov_rad = c.fov / 180.0f * kPi;
    d.film_h = 2.0f * c.focal_distance * std::tan(fov_rad / 2.0f);
    d.film_w = c.aspect * d.film_h;
    d.focal = c.focal_distance;
    d.lens_radius = c.lens_radius;
    d.type = c.type;
    return d;
}

RenderCfg make_cfg(const fm_render_params& p)
{
    RenderCfg r;
    r.img_w = p.width;
    r.img_h = p.height;
    r.width = out_width(p);
    r.height = out_height(p);
    r.x0 = p.region_w > 0 ? p.region_x : 0;
    r.y0 = p.region_w > 0 ? p.region_y : 0;
    r.spp = p.spp;
    r.depth = p.depth;
    r.direct_loop = p.direct_loop;
    r.rr_depth = p.rr_depth;
    r.rr_coef = p.rr_coef;
    r.seed = p.seed;
    r.sample_offset = p.sample_offset;
    r.rr_enabled = p.depth > p.rr_depth ? 1 : 0;
    r.clamp = p.max_sample_value;
    return r;
}

fm_status validate_render(fm_ctx* ctx, const fm_scene* scene, const fm_camera* camera, const fm_render_params* p)
{
    if (!scene || !camera || !p) return set_error(ctx, FM_ERR_INVALID, "render: null argument");
    if (p->width <= 0 || p->height <= 0 || p->spp <= 0 || p->depth <= 0 || p->direct_loop <= 0)
        return set_error(ctx, FM_ERR_INVALID, "render: width, height, spp, depth and direct_loop must be positive");
    if ((int64_t)p->width * p->height > (int64_t)1 << 30) return set_error(ctx, FM_ERR_INVALID, "render: image too large");
    if (camera->type != FM_CAMERA_PINHOLE && camera->type != FM_CAMERA_THIN_LENS)
        return set_error(ctx, FM_ERR_INVALID, "render: bad camera type");
    if (p->mode != FM_MODE_MEGAKERNEL && p->mode != FM_MODE_WAVEFRONT)
        return set_error(ctx, FM_ERR_INVALID, "render: bad mode");
    if (p->sample_offset < 0) return set_error(ctx, FM_ERR_INVALID, "render: negative sample_offset");
    if (!(p->max_sample_value >= 0.0f)) return set_error(ctx, FM_ERR_INVALID, "render: max_sample_value must be >= 0");
    if (p->region_w != 0 || p->region_h != 0) {
        if (p->region_w <= 0 || p->region_h <= 0 || p->region_x < 0 || p->region_y < 0 ||
            (int64_t)p->region_x + p->region_w > p->width || (int64_t)p->region_y + p->region_h > p->height)
            return set_error(ctx, FM_ERR_INVALID, "render: region outside the image");
    }
    return FM_OK;
}

fm_status megakernel_views(fm_ctx* ctx, std::vector<WfView> views, Counters* cnt)
{
    cudaStream_t s = ctx->stream;
    const int block = 128;
    int per_sm = 0;
    FM_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_megakernel, block, 0), "megakernel occupancy");
    per_sm = std::max(per_sm, 1);
    const int grid = ctx->num_sms * per_sm;
    const double resident = (double)grid * block;
    // samples per item: enough items (about 32 per resident thread) that the threads
    // finishing last hold little work, and no more (each item writes 48 B of sums)
    double total_samples = 0.0;
    for (const auto& v : views) total_samples += (double)v.cfg.width * v.cfg.height * v.cfg.spp;
    const int target = (int)std::max(1.0, std::floor(total_samples / (32.0 * resident)));
    int64_t item_base = 0;
    for (auto& v : views) {
        v.chunk = std::max(1, std::min(target, v.cfg.spp));
        v.nchunks = (v.cfg.spp + v.chunk - 1) / v.chunk;
        v.item_base = item_base;
        item_base += (int64_t)v.cfg.width * v.cfg.height * v.nchunks;
    }
    const size_t head = 256;
    const size_t views_bytes = (sizeof(WfView) * views.size() + 255) / 256 * 256;
    const size_t partial_bytes = (size_t)item_base * 3 * sizeof(float4);
    char* buf = nullptr;
    FM_CUDA_TRY(ctx, cudaMallocAsync((void**)&buf, head + views_bytes + partial_bytes, s), "megakernel alloc");
    auto* next = reinterpret_cast<unsigned long long*>(buf);
    auto* d_views = reinterpret_cast<WfView*>(buf + head);
    float4* partial = reinterpret_cast<float4*>(buf + head + views_bytes);
    for (auto& v : views) {
        v.partial = partial;
        partial += 3 * (size_t)v.cfg.width * v.cfg.height * v.nchunks;
    }
    fm_status st = FM_OK;
    cudaError_t e = cudaMemsetAsync(next, 0, sizeof(unsigned long long), s);
    // pageable source: the driver stages it before this call returns
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_views, views.data(), sizeof(WfView) * views.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        k_megakernel<<<grid, block, 0, s>>>(d_views, (int)views.size(), item_base, next, cnt, ctx->d_status);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        st = cuda_error(ctx, e, "megakernel");
    else
        st = reduce_views(ctx, views);
    cudaFreeAsync(buf, s);
    return st;
}

fm_status launch_megakernel(fm_ctx* ctx, const fm_scene* scene, const DevCamera& cam, const RenderCfg& cfg, float* rgb,
                            float* alb, float* nrm, Counters* cnt)
{
    WfView v{};
    v.scene = scene->d_dev;
    v.num_lights = scene->dev.num_lights;
    v.cam = cam;
    v.cfg = cfg;
    v.rgb = rgb;
    v.alb = alb;
    v.nrm = nrm;
    return megakernel_views(ctx, {v}, cnt);
}

}  // namespace fm

using namespace fm;

extern "C" fm_status fm_render(fm_ctx* ctx, const fm_scene* scene, const fm_camera* camera,
                               const fm_render_params* params, float* rgb, float* albedo, float* normal,
                               int32_t flags, fm_render_stats* stats)
{
    if (!ctx) return FM_ERR_INVALID;
    fm_status st = validate_render(ctx, scene, camera, params);
    if (st != FM_OK) return st;
    if (!rgb) return set_error(ctx, FM_ERR_INVALID, "render: rgb output is null");
    FM_CUDA_TRY(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    const DevCamera cam = make_camera(*camera);
    const RenderCfg cfg = make_cfg(*params);
    const size_t npix = (size_t)cfg.width * cfg.height;
    const size_t img_bytes = npix * 3 * sizeof(float);
    const bool dev = (flags & FM_FLAG_DEVICE_PTRS) != 0;
    char* tmp = nullptr;
    float *d_rgb = rgb, *d_alb = albedo, *d_nrm = normal;
    Counters* d_cnt = nullptr;
    const size_t nimg = dev ? 0 : 1 + (albedo ? 1 : 0) + (normal ? 1 : 0);
    FM_CUDA_TRY(ctx, cudaMallocAsync((void**)&tmp, nimg * img_bytes + 256, ctx->stream), "render alloc");
    d_cnt = reinterpret_cast<Counters*>(tmp);
    if (!dev) {
        char* q = tmp + 256;
        d_rgb = reinterpret_cast<float*>(q);
        q += img_bytes;
        d_alb = albedo ? reinterpret_cast<float*>(q) : nullptr;
        q += albedo ? img_bytes : 0;
        d_nrm = normal ? reinterpret_cast<float*>(q) : nullptr;
    }
    FM_CUDA_TRY(ctx, cudaMemsetAsync(d_cnt, 0, sizeof(Counters), ctx->stream), "render");
    FM_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream), "render");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ctx->stream);
    if (cfg.spp > 0 && params->mode == FM_MODE_WAVEFRONT)
        st = launch_wavefront(ctx, scene, cam, cfg, d_rgb, d_alb, d_nrm, d_cnt);
    else
        st = launch_megakernel(ctx, scene, cam, cfg, d_rgb, d_alb, d_nrm, d_cnt);
    cudaEventRecord(e1, ctx->stream);
    cudaError_t ecopy = cudaSuccess;
    if (st == FM_OK && !dev) {
        std::vector<OutCopy> out{OutCopy{rgb, d_rgb, img_bytes}};
        if (albedo) out.push_back(OutCopy{albedo, d_alb, img_bytes});
        if (normal) out.push_back(OutCopy{normal, d_nrm, img_bytes});
        ecopy = copy_out(ctx, ctx->stream, out);
    }
    Counters hc{};
    uint32_t hs = 0;
    cudaMemcpyAsync(&hc, d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream);
    cudaMemcpyAsync(&hs, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream);
    cudaFreeAsync(tmp, ctx->stream);
    const cudaError_t e = cudaStreamSynchronize(ctx->stream);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != FM_OK) return st;
    if (ecopy != cudaSuccess) return cuda_error(ctx, ecopy, "render: image copy");
    if (e != cudaSuccess) return cuda_error(ctx, e, "render");
    if (stats) {
        stats->paths = (int64_t)hc.paths;
        stats->closest_rays = (int64_t)hc.closest;
        stats->shadow_rays = (int64_t)hc.shadow;
        stats->bounces = (int64_t)hc.bounces;
        stats->nan_samples = (int64_t)hc.nans;
        stats->kernel_ms = ms;
        stats->trace_ms = 0.0;
        stats->shade_ms = 0.0;
        stats->launches = params->mode == FM_MODE_WAVEFRONT ? -1 : 2;
    }
    if (hs & 1u) return set_error(ctx, FM_ERR_QUEUE_OVERFLOW, "render: traversal stack overflow");
    if (hs & 2u) return set_error(ctx, FM_ERR_QUEUE_OVERFLOW, "render: wavefront queue overflow");
    return FM_OK;
}
