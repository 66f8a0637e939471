// Rendering internals shared by fm_render.cu, fm_wavefront.cu and fm_batch.cu.
#pragma once
#include "fm_integrator.cuh"
#include "fm_internal.h"

namespace fm {

DevCamera make_camera(const fm_camera& c);
// Output image size of a render: the region's when one is set, else the whole image's.
inline int out_width(const fm_render_params& p) { return p.region_w > 0 ? p.region_w : p.width; }
inline int out_height(const fm_render_params& p) { return p.region_w > 0 ? p.region_h : p.height; }
RenderCfg make_cfg(const fm_render_params& p);
fm_status validate_render(fm_ctx* ctx, const fm_scene* scene, const fm_camera* camera, const fm_render_params* p);

// Device-side description of one view in a wavefront launch.
struct WfView {
    const DevScene* scene;   // device pointer
    DevCamera cam;
    RenderCfg cfg;
    int64_t item_base;       // first work item of this view
    int32_t chunk;           // samples per work item
    int32_t nchunks;         // work items per pixel
    float4* partial;         // [nchunks * npix * 3] (color Kahan sum, albedo sum, normal sum)
    float* rgb;              // outputs (device)
    float* alb;
    float* nrm;
    const float* drgb;       // adjoint renders: dLoss/dI per pixel (device, w*h*3)
    int32_t num_lights;      // the scene's light count (host copy, sizes the shadow queue)
};

// Gradient accumulators of an adjoint render (device buffers, zeroed by the caller).
struct WfAdjoint {
    float* const* tex_acc;     // device array over the scene's textures: NULL or tex_copies[t] x w*h*3
    const int32_t* tex_copies; // device array: FP32 copies per texture
    float* mat_acc;            // num_materials * 5 (basecolor rgb, metallic, roughness) or NULL
    double* env_row;           // env map height doubles, zeroed (score sums per row)
    double* env_total;         // one double, zeroed
};

// Spreads the env importance-table normalisation terms collected during an adjoint
// render (row and total score sums) over the env texels' gradient.
fm_status env_grad_finalize(fm_ctx* ctx, const DevTexture& tex, const double* env_row, const double* env_total,
                            double* grad);

// Wavefront tuning knobs (pool size, block sizes, graph depth).
struct WfTuning {
    int64_t pool = 1 << 21;   // path slots
    int trace_block = 128;
    int shade_block = 128;
    int iters_per_graph = 8;
    bool profile = false;     // record CUDA events around each trace / shade launch
    int max_iterations = 0;   // > 0: iteration cap below the automatic bound (then FM_ERR_TIMEOUT)
    int queue_limit = 0;      // > 0: ray-queue capacity cap (then FM_ERR_QUEUE_OVERFLOW)
};

struct WfTimes {
    double total_ms = 0.0, trace_ms = 0.0, shade_ms = 0.0;
    int64_t launches = 0;
};

fm_status launch_wavefront(fm_ctx* ctx, const fm_scene* scene, const DevCamera& cam, const RenderCfg& cfg, float* rgb,
                           float* alb, float* nrm, Counters* cnt);
fm_status launch_megakernel(fm_ctx* ctx, const fm_scene* scene, const DevCamera& cam, const RenderCfg& cfg, float* rgb,
                            float* alb, float* nrm, Counters* cnt);
// The plain megakernel over several views (possibly of different scenes) in one launch.
fm_status megakernel_views(fm_ctx* ctx, std::vector<WfView> views, Counters* cnt);
// Per pixel of each view: sums the view's partial sums in chunk order and writes the
// mean colour, albedo and normal images.
fm_status reduce_views(fm_ctx* ctx, const std::vector<WfView>& views);
// Renders several views (possibly of different scenes) in one wavefront.
fm_status wavefront_views(fm_ctx* ctx, const std::vector<WfView>& views, const WfTuning& tune, Counters* cnt,
                          WfTimes* times);
// Path-replay adjoint over views of one scene: gradients of sum(drgb * image) with
// respect to texture texels and material constants.  rgb (if set) receives the primal
// image of the same samples.
fm_status wavefront_adjoint(fm_ctx* ctx, const std::vector<WfView>& views, const WfTuning& tune, const WfAdjoint& adj,
                            Counters* cnt, WfTimes* times);

}  // namespace fm
