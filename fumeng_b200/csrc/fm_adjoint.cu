// Differentiable rendering entry points: in-place texture updates (for an optimisation
// loop over texels) and the path-replay adjoint render.  The reference renders forward
// only; nothing here replaces a reference interface.
#include <vector>

#include "fm_render.h"

namespace fm {

namespace {

// out[i] += sum over the copies of acc (FP64 sums of the FP32 accumulators).
__global__ void k_grad_reduce(const float* __restrict__ acc, int copies, size_t n, double* __restrict__ out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double sum = 0.0;
        for (int k = 0; k < copies; ++k) sum += (double)acc[(size_t)k * n + i];
        out[i] += sum;
    }
}

// Device allocations of one call, released on every exit path.
struct Allocs {
    cudaStream_t s;
    std::vector<void*> ptrs;
    template <class T>
    T* get(size_t count)
    {
        void* p = nullptr;
        if (cudaMallocAsync(&p, sizeof(T) * count, s) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    ~Allocs()
    {
        for (void* p : ptrs) cudaFreeAsync(p, s);
        cudaStreamSynchronize(s);
    }
};

}  // namespace

}  // namespace fm

using namespace fm;

extern "C" fm_status fm_scene_info(fm_ctx* ctx, const fm_scene* scene, int64_t* objects, int32_t* materials,
                                   int32_t* textures, int32_t* lights)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!scene) return set_error(ctx, FM_ERR_INVALID, "scene_info: scene is null");
    if (objects) *objects = scene->num_objects;
    if (materials) *materials = scene->dev.num_materials;
    if (textures) *textures = scene->dev.num_textures;
    if (lights) *lights = scene->dev.num_lights;
    return FM_OK;
}

extern "C" fm_status fm_scene_update_texture(fm_ctx* ctx, fm_scene* scene, int32_t texture, const float* texels,
                                             int32_t flags)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!scene || !texels || texture < 0 || texture >= (int32_t)scene->textures.size())
        return set_error(ctx, FM_ERR_INVALID, "update_texture: bad arguments");
    FM_CUDA_TRY(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    const DevTexture& t = scene->textures[(size_t)texture];
    const size_t n = (size_t)t.w * t.h;
    cudaStream_t s = ctx->stream;
    {
        Allocs a{s, {}};
        const float* src = texels;
        if (!(flags & FM_FLAG_DEVICE_PTRS)) {
            float* staged = a.get<float>(3 * n);
            if (!staged) return set_error(ctx, FM_ERR_OOM, "update_texture: staging allocation failed");
            FM_CUDA_TRY(ctx, cudaMemcpyAsync(staged, texels, 3 * n * sizeof(float), cudaMemcpyHostToDevice, s),
                        "update_texture h2d");
            src = staged;
        }
        launch_rgb_to_texels(s, src, const_cast<float4*>(t.texels), n, ctx->num_sms);
        FM_CUDA_TRY(ctx, cudaGetLastError(), "update_texture");
    }
    if (scene->dev.env_light >= 0 && scene->dev.env.tex == texture) {
        // the environment's importance tables follow its texels (rebuilt in place)
        const fm_status st = env_build_tables(ctx, s, scene, t, scene->dev.env);
        if (st != FM_OK) return st;
    }
    FM_CUDA_TRY(ctx, cudaStreamSynchronize(s), "update_texture");
    return FM_OK;
}

extern "C" fm_status fm_render_adjoint(fm_ctx* ctx, const fm_scene* scene, int32_t n, const fm_camera* cams,
                                       const fm_render_params* params, const float* const* d_rgb, float* const* rgb,
                                       const fm_grad_desc* grads, int32_t flags, fm_render_stats* stats)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!scene || n <= 0 || !cams || !params || !d_rgb || !grads)
        return set_error(ctx, FM_ERR_INVALID, "render_adjoint: bad arguments");
    for (int32_t i = 0; i < n; ++i) {
        const fm_status st = validate_render(ctx, scene, &cams[i], &params[i]);
        if (st != FM_OK) return st;
        if (params[i].mode != FM_MODE_WAVEFRONT)
            return set_error(ctx, FM_ERR_INVALID, "render_adjoint: views must use FM_MODE_WAVEFRONT");
        if (params[i].max_sample_value != 0.0f)
            return set_error(ctx, FM_ERR_INVALID, "render_adjoint: max_sample_value must be 0 (no clamp)");
        if (!d_rgb[i]) return set_error(ctx, FM_ERR_INVALID, "render_adjoint: d_rgb entry is null");
    }
    FM_CUDA_TRY(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    const bool dev = (flags & FM_FLAG_DEVICE_PTRS) != 0;
    cudaStream_t s = ctx->stream;
    const int nt = scene->dev.num_textures, nm = scene->dev.num_materials;
    fm_status result = FM_OK;
    std::vector<double*> dtex((size_t)nt, nullptr);
    double* dmat = nullptr;
    std::vector<float*> drgb_in((size_t)n), rgb_out((size_t)n);
    std::vector<size_t> img_floats((size_t)n);
    Counters hc{};
    uint32_t hs = 0;
    WfTimes tm;
    {
        Allocs a{s, {}};
        auto oom = [&]() { return set_error(ctx, FM_ERR_OOM, "render_adjoint: allocation failed"); };
        // gradient buffers
        for (int t = 0; t < nt; ++t) {
            double* user = grads->texture_grads ? grads->texture_grads[t] : nullptr;
            if (!user) continue;
            if (dev) {
                dtex[t] = user;
            } else {
                const size_t cnt = (size_t)scene->textures[t].w * scene->textures[t].h * 3;
                dtex[t] = a.get<double>(cnt);
                if (!dtex[t]) return oom();
                FM_CUDA_TRY(ctx, cudaMemsetAsync(dtex[t], 0, cnt * sizeof(double), s), "render_adjoint");
            }
        }
        if (grads->material_grads) {
            if (dev) {
                dmat = grads->material_grads;
            } else {
                dmat = a.get<double>((size_t)nm * kGradParams);
                if (!dmat) return oom();
                FM_CUDA_TRY(ctx, cudaMemsetAsync(dmat, 0, (size_t)nm * kGradParams * sizeof(double), s),
                            "render_adjoint");
            }
        }
        // FP32 accumulators the kernels add to: 8 copies of a texture, more for small
        // ones (up to about 8M floats, at most 256 copies)
        std::vector<float*> facc((size_t)nt, nullptr);
        std::vector<size_t> tex_n((size_t)nt, 0);
        std::vector<int32_t> copies((size_t)(nt > 0 ? nt : 1), 1);
        for (int t = 0; t < nt; ++t) {
            if (!dtex[t]) continue;
            tex_n[t] = (size_t)scene->textures[t].w * scene->textures[t].h * 3;
            int k = 8;
            while (k < 256 && (size_t)(2 * k) * tex_n[t] <= ((size_t)8 << 20)) k *= 2;
            copies[t] = k;
            facc[t] = a.get<float>(tex_n[t] * k);
            if (!facc[t]) return oom();
            FM_CUDA_TRY(ctx, cudaMemsetAsync(facc[t], 0, tex_n[t] * k * sizeof(float), s), "render_adjoint");
        }
        int32_t* d_copies = a.get<int32_t>(copies.size());
        if (!d_copies) return oom();
        FM_CUDA_TRY(ctx, cudaMemcpyAsync(d_copies, copies.data(), sizeof(int32_t) * copies.size(), cudaMemcpyHostToDevice, s),
                    "render_adjoint");
        float* macc = nullptr;
        if (dmat) {
            macc = a.get<float>((size_t)nm * kGradParams);
            if (!macc) return oom();
            FM_CUDA_TRY(ctx, cudaMemsetAsync(macc, 0, (size_t)nm * kGradParams * sizeof(float), s), "render_adjoint");
        }
        float** d_tex_arr = a.get<float*>((size_t)(nt > 0 ? nt : 1));
        Counters* d_cnt = a.get<Counters>(1);
        if (!d_tex_arr || !d_cnt) return oom();
        if (nt > 0)
            FM_CUDA_TRY(ctx, cudaMemcpyAsync(d_tex_arr, facc.data(), sizeof(float*) * nt, cudaMemcpyHostToDevice, s),
                        "render_adjoint");
        FM_CUDA_TRY(ctx, cudaMemsetAsync(d_cnt, 0, sizeof(Counters), s), "render_adjoint");
        FM_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), s), "render_adjoint");
        // per-view dLoss/dI inputs and image outputs
        std::vector<WfView> views((size_t)n);
        for (int32_t i = 0; i < n; ++i) {
            img_floats[i] = (size_t)out_width(params[i]) * out_height(params[i]) * 3;
            const size_t bytes = img_floats[i] * sizeof(float);
            if (dev) {
                drgb_in[i] = const_cast<float*>(d_rgb[i]);
            } else {
                drgb_in[i] = a.get<float>(img_floats[i]);
                if (!drgb_in[i]) return oom();
                FM_CUDA_TRY(ctx, cudaMemcpyAsync(drgb_in[i], d_rgb[i], bytes, cudaMemcpyHostToDevice, s),
                            "render_adjoint h2d");
            }
            // the wavefront always writes a primal image; scratch when none is wanted
            if (dev && rgb && rgb[i]) {
                rgb_out[i] = rgb[i];
            } else {
                rgb_out[i] = a.get<float>(img_floats[i]);
                if (!rgb_out[i]) return oom();
            }
            WfView& v = views[i];
            v = WfView{};
            v.scene = scene->d_dev;
            v.num_lights = scene->dev.num_lights;
            v.cam = make_camera(cams[i]);
            v.cfg = make_cfg(params[i]);
            v.rgb = rgb_out[i];
            v.drgb = drgb_in[i];
        }
        // the env light's importance densities depend on every texel through their row
        // and map sums: score sums per row and in total, spread after the render
        const int env_tex = scene->dev.env_light >= 0 ? scene->dev.env.tex : -1;
        double *env_row = nullptr, *env_total = nullptr;
        if (env_tex >= 0 && dtex[env_tex]) {
            const int eh = scene->textures[env_tex].h;
            env_row = a.get<double>((size_t)eh + 1);
            if (!env_row) return oom();
            env_total = env_row + eh;
            FM_CUDA_TRY(ctx, cudaMemsetAsync(env_row, 0, sizeof(double) * (eh + 1), s), "render_adjoint");
        }
        WfAdjoint adj{d_tex_arr, d_copies, macc, env_row, env_total};
        WfTuning wt;
        wt.profile = (flags & FM_FLAG_PROFILE) != 0;
        result = wavefront_adjoint(ctx, views, wt, adj, d_cnt, &tm);
        if (result == FM_OK) {
            const int grid = ctx->num_sms * 8;
            for (int t = 0; t < nt; ++t)
                if (facc[t]) k_grad_reduce<<<grid, 256, 0, s>>>(facc[t], copies[t], tex_n[t], dtex[t]);
            if (macc) k_grad_reduce<<<grid, 256, 0, s>>>(macc, 1, (size_t)nm * kGradParams, dmat);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) result = cuda_error(ctx, e, "render_adjoint reduce");
        }
        if (result == FM_OK && env_row)
            result = env_grad_finalize(ctx, scene->textures[env_tex], env_row, env_total, dtex[env_tex]);
        if (result == FM_OK && !dev) {
            // results back to the host: images, then gradients added into the caller's buffers
            for (int32_t i = 0; i < n; ++i)
                if (rgb && rgb[i])
                    cudaMemcpyAsync(rgb[i], rgb_out[i], img_floats[i] * sizeof(float), cudaMemcpyDeviceToHost, s);
            for (int t = 0; t < nt; ++t) {
                if (!dtex[t]) continue;
                const size_t cnt = (size_t)scene->textures[t].w * scene->textures[t].h * 3;
                std::vector<double> h(cnt);
                FM_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), dtex[t], cnt * sizeof(double), cudaMemcpyDeviceToHost, s),
                            "render_adjoint d2h");
                FM_CUDA_TRY(ctx, cudaStreamSynchronize(s), "render_adjoint");
                double* user = grads->texture_grads[t];
                for (size_t q = 0; q < cnt; ++q) user[q] += h[q];
            }
            if (dmat) {
                std::vector<double> h((size_t)nm * kGradParams);
                FM_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), dmat, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s),
                            "render_adjoint d2h");
                FM_CUDA_TRY(ctx, cudaStreamSynchronize(s), "render_adjoint");
                for (size_t q = 0; q < h.size(); ++q) grads->material_grads[q] += h[q];
            }
        }
        cudaMemcpyAsync(&hc, d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(&hs, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
        const cudaError_t e = cudaStreamSynchronize(s);
        if (result == FM_OK && e != cudaSuccess) result = cuda_error(ctx, e, "render_adjoint");
    }
    if (result != FM_OK) return result;
    if (stats) {
        stats->paths = (int64_t)hc.paths;
        stats->closest_rays = (int64_t)hc.closest;
        stats->shadow_rays = (int64_t)hc.shadow;
        stats->bounces = (int64_t)hc.bounces;
        stats->nan_samples = (int64_t)hc.nans;
        stats->kernel_ms = tm.total_ms;
        stats->trace_ms = tm.trace_ms;
        stats->shade_ms = tm.shade_ms;
        stats->launches = tm.launches;
    }
    if (hs & 1u) return set_error(ctx, FM_ERR_QUEUE_OVERFLOW, "render_adjoint: traversal stack overflow");
    if (hs & 2u) return set_error(ctx, FM_ERR_QUEUE_OVERFLOW, "render_adjoint: wavefront queue overflow");
    return FM_OK;
}
