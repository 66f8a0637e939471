// Rendering entry point (integrator kernels are added in this file).
#include "fm_internal.h"

extern "C" fm_status fm_render(fm_ctx* ctx, const fm_scene* scene, const fm_camera* camera,
                               const fm_render_params* params, float* rgb, float* albedo, float* normal,
                               int32_t flags, fm_render_stats* stats)
{
    (void)scene; (void)camera; (void)params; (void)rgb; (void)albedo; (void)normal; (void)flags; (void)stats;
    return fm::set_error(ctx, FM_ERR_INVALID, "fm_render: integrator not built yet");
}
