// C-ABI: contexts, scene release and ray queries (scene creation: fm_scene_build.cu).
#include <cmath>
#include <cstring>
#include <new>
#include <unordered_map>

#include "fm_bvh.cuh"
#include "fm_internal.h"
#include "fm_staging.h"

using namespace fm;

namespace {

__global__ void k_trace(const __grid_constant__ DevScene S, const float* __restrict__ rays, int64_t n,
                        int32_t* obj_out, float* t_out, uint8_t* occ_out, uint32_t* status)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(rays) + 2 * i);
        const float4 b = __ldg(reinterpret_cast<const float4*>(rays) + 2 * i + 1);
        Hit h;
        if (occ_out) {
            occ_out[i] = trace_ray<true>(S, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, a.w, b.w, h, status) ? 1 : 0;
        } else {
            const bool hit = trace_ray<false>(S, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, a.w, b.w, h, status);
            obj_out[i] = hit ? __ldg(S.prim_obj + h.prim) : -1;
            t_out[i] = hit ? h.t : __int_as_float(0x7f800000);
        }
    }
}

fm_status trace_common(fm_ctx* ctx, const fm_scene* sc, const float* rays, int64_t n, int32_t* obj, float* t,
                       uint8_t* occ, int32_t flags)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!sc || n < 0 || (n > 0 && !rays)) return set_error(ctx, FM_ERR_INVALID, "trace: bad arguments");
    if (n == 0) return FM_OK;
    if (!occ && (!obj || !t)) return set_error(ctx, FM_ERR_INVALID, "trace: null output");
    FM_CUDA_TRY(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    const bool dev = (flags & FM_FLAG_DEVICE_PTRS) != 0;
    const float* d_rays = rays;
    int32_t* d_obj = obj;
    float* d_t = t;
    uint8_t* d_occ = occ;
    void* tmp = nullptr;
    if (!dev) {
        const size_t bytes = 32 * (size_t)n + (occ ? (size_t)n : 8 * (size_t)n);
        FM_CUDA_TRY(ctx, cudaMallocAsync(&tmp, bytes, ctx->stream), "trace alloc");
        char* p = static_cast<char*>(tmp);
        d_rays = reinterpret_cast<float*>(p);
        FM_CUDA_TRY(ctx, cudaMemcpyAsync(p, rays, 32 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream), "trace h2d");
        p += 32 * (size_t)n;
        if (occ) {
            d_occ = reinterpret_cast<uint8_t*>(p);
        } else {
            d_obj = reinterpret_cast<int32_t*>(p);
            d_t = reinterpret_cast<float*>(p + 4 * (size_t)n);
        }
    }
    FM_CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), ctx->stream), "trace");
    const int block = 128;
    int64_t grid = (n + block - 1) / block;
    if (grid > (int64_t)ctx->num_sms * 64) grid = (int64_t)ctx->num_sms * 64;
    k_trace<<<(int)grid, block, 0, ctx->stream>>>(sc->dev, d_rays, n, d_obj, d_t, d_occ, ctx->d_status);
    FM_CUDA_TRY(ctx, cudaGetLastError(), "trace launch");
    if (!dev) {
        if (occ) {
            FM_CUDA_TRY(ctx, cudaMemcpyAsync(occ, d_occ, n, cudaMemcpyDeviceToHost, ctx->stream), "trace d2h");
        } else {
            FM_CUDA_TRY(ctx, cudaMemcpyAsync(obj, d_obj, 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
            FM_CUDA_TRY(ctx, cudaMemcpyAsync(t, d_t, 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
        }
        FM_CUDA_TRY(ctx, cudaFreeAsync(tmp, ctx->stream), "trace free");
    }
    uint32_t status = 0;
    FM_CUDA_TRY(ctx, cudaMemcpyAsync(&status, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream),
                "status");
    FM_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "trace sync");
    if (status & 1u) return set_error(ctx, FM_ERR_QUEUE_OVERFLOW, "trace: traversal stack overflow");
    return FM_OK;
}

}  // namespace

extern "C" {

fm_status fm_ctx_create(int device, fm_ctx** out)
{
    if (!out) return FM_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return FM_ERR_NO_DEVICE;
    if (device < 0 || device >= count) return FM_ERR_INVALID;
    fm_ctx* ctx = new (std::nothrow) fm_ctx();
    if (!ctx) return FM_ERR_OOM;
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->d_status, 64) != cudaSuccess) {
        delete ctx;
        return FM_ERR_CUDA;
    }
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    // Scenes, BVH builds and renders allocate from the device's default memory pool with
    // stream-ordered calls; keeping freed blocks in the pool makes creating and
    // destroying scenes cheap (no release to the driver at every synchronisation).
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    *out = ctx;
    return FM_OK;
}

void fm_ctx_destroy(fm_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    fm::scene_builder_release(ctx);
    fm::staging_release(ctx);
    fm::wf_cache_release(ctx);
    cudaFree(ctx->d_status);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* fm_last_error(const fm_ctx* ctx) { return ctx ? ctx->error.c_str() : "null context"; }

// Used by the host-side scene loader (compiled by the C++ compiler) to report errors.
void fm_internal_set_error(fm_ctx* ctx, const char* msg)
{
    if (ctx) ctx->error = msg ? msg : "";
}

fm_status fm_scene_destroy(fm_ctx* ctx, fm_scene* sc)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!sc) return FM_OK;
    cudaSetDevice(ctx->device);
    for (void* p : sc->allocations) cudaFreeAsync(p, ctx->stream);
    sc->shared_bvh.reset();   // frees the BVH arrays when no other scene of its group holds them
    cudaStreamSynchronize(ctx->stream);
    delete sc;
    return FM_OK;
}

fm_status fm_scene_bvh_stats(fm_ctx* ctx, const fm_scene* sc, int64_t* nodes, int64_t* prims, int32_t* depth,
                             double* build_ms)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!sc) return set_error(ctx, FM_ERR_INVALID, "bvh_stats: null scene");
    if (nodes) *nodes = sc->bvh.num_nodes;
    if (prims) *prims = sc->bvh.num_leaf;
    if (depth) *depth = sc->bvh.depth;
    if (build_ms) *build_ms = sc->bvh.build_ms;
    return FM_OK;
}

fm_status fm_trace_closest(fm_ctx* ctx, const fm_scene* scene, const float* rays, int64_t n, int32_t* obj_id, float* t,
                           int32_t flags)
{
    return trace_common(ctx, scene, rays, n, obj_id, t, nullptr, flags);
}

fm_status fm_trace_any(fm_ctx* ctx, const fm_scene* scene, const float* rays, int64_t n, uint8_t* occluded,
                       int32_t flags)
{
    if (!occluded && n > 0) return ctx ? set_error(ctx, FM_ERR_INVALID, "trace_any: null output") : FM_ERR_INVALID;
    return trace_common(ctx, scene, rays, n, nullptr, nullptr, occluded, flags);
}

}  // extern "C"
