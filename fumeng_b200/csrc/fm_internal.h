// Host-side definitions shared by the C-ABI translation units.
#pragma once
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/fumeng_b200.h"
#include "fm_bvh_build.h"
#include "fm_scene.cuh"

namespace fm {
struct WfCache;    // wavefront workspace (fm_wavefront.cu)
class CopyPool;    // host copy threads (fm_staging.cu)
void wf_cache_release(fm_ctx* ctx);
}  // namespace fm

struct fm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string error;
    uint32_t* d_status = nullptr;   // device status word: bit 0 stack overflow, bit 1 queue overflow
    int num_sms = 148;
    // autotuned wavefront settings per batch shape class (views, log2 samples, max lights)
    std::map<std::tuple<int, int, int>, fm_tuning> tune_cache;
    // wavefront workspaces (forward, adjoint): state buffers, pinned staging and the
    // instantiated graph, kept between renders
    fm::WfCache* wf_cache[2] = {nullptr, nullptr};
    // scene creation: streams that build scenes side by side
    std::vector<cudaStream_t> build_streams;
    std::vector<cudaEvent_t> build_events;
    cudaStream_t capture_stream = nullptr;   // BVH build graphs are captured here, never run
    char* build_pinned = nullptr;            // BVH builds' scene tables and counters (pinned)
    size_t build_pinned_bytes = 0;
    // pinned staging ring for host <-> device transfers (fm_staging.h): kStageChunks
    // chunks, an event per chunk, and the host copy threads
    char* stage = nullptr;
    std::vector<cudaEvent_t> stage_events;
    fm::CopyPool* copy_pool = nullptr;
};

struct fm_scene {
    fm::DevScene dev{};               // device pointers filled in
    fm::DevScene* d_dev = nullptr;    // device copy of `dev` (for batched kernels)
    std::vector<void*> allocations;   // everything to cudaFree on destroy
    std::shared_ptr<void> shared_bvh;  // BVH arrays shared with the scenes built alongside
    fm::BvhResult bvh;
    int64_t num_objects = 0;
    // host copies kept for validation and light sampling set-up
    std::vector<fm::DevLight> lights;
    std::vector<fm::DevTexture> textures;   // device texel pointers, for in-place updates
};

namespace fm {

inline fm_status set_error(fm_ctx* ctx, fm_status st, const std::string& msg)
{
    if (ctx) ctx->error = msg;
    return st;
}

inline fm_status cuda_error(fm_ctx* ctx, cudaError_t e, const char* where)
{
    return set_error(ctx, FM_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define FM_CUDA_TRY(ctx, expr, where)                                   \
    do {                                                                \
        cudaError_t e__ = (expr);                                       \
        if (e__ != cudaSuccess) return ::fm::cuda_error(ctx, e__, where); \
    } while (0)

// Environment-map importance tables (fm_env.cu), enqueued on `stream` (no host wait; the
// tables are ready in stream order).
fm_status env_build_tables(fm_ctx* ctx, cudaStream_t stream, fm_scene* scene, const DevTexture& tex, DevEnv& env);

// RGB float texels (3 per texel) -> the float4 texels the device samples (fm_adjoint.cu).
void launch_rgb_to_texels(cudaStream_t stream, const float* src, float4* dst, size_t n, int num_sms);

// Releases the scene builder's streams (fm_scene_build.cu).
void scene_builder_release(fm_ctx* ctx);

}  // namespace fm
