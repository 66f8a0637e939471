// Closest-hit queries that allocate no device memory.
//
// fm_trace_closest stages host rays and results in device memory it allocates per call.
// Some callers cannot let the library allocate once they are running: a real-time loop
// with a fixed device-memory budget and a frame deadline (cudaMalloc / cudaFree can fail
// at an arbitrary point or stall on device synchronisation), or an application that
// hands all device memory to its own pool.  fm_trace_closest_noalloc does the same
// query through a staging area that is part of the library image instead: a file-scope
// __device__ array of fixed size, which every GPU that loads the library holds until
// the process exits.
#include <mutex>

#include "fm_bvh.cuh"
#include "fm_internal.h"

namespace fm {

namespace {

// At most this many rays per call (32 B per ray in, 8 B per ray out: 10 MiB in all).
constexpr int64_t kNoallocMaxRays = int64_t(1) << 18;
constexpr size_t kStatusBytes = 256;
constexpr size_t kScratchBytes = kStatusBytes + (size_t)kNoallocMaxRays * (32 + 4 + 4);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device.  The array's name in host
// code is only a host-side handle, so its address on each device is looked up once, with
// that device current.
fm_status scratch_for_device(fm_ctx* ctx, unsigned char** out)
{
    if (ctx->device < 0 || ctx->device >= kMaxDevices) return set_error(ctx, FM_ERR_INVALID, "noalloc: device index too large");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[ctx->device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_error(ctx, e, "noalloc: cudaGetSymbolAddress");
        g_scratch_ptr[ctx->device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[ctx->device];
    return FM_OK;
}

__global__ void k_trace_closest_staged(const __grid_constant__ DevScene S, const float4* __restrict__ rays, int64_t n,
                                       int32_t* obj_out, float* t_out, uint32_t* status)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 a = rays[2 * i], b = rays[2 * i + 1];
        Hit h;
        const bool hit = trace_ray<false>(S, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, a.w, b.w, h, status);
        obj_out[i] = hit ? __ldg(S.prim_obj + h.prim) : -1;
        t_out[i] = hit ? h.t : __int_as_float(0x7f800000);
    }
}

}  // namespace

}  // namespace fm

using namespace fm;

extern "C" fm_status fm_trace_closest_noalloc(fm_ctx* ctx, const fm_scene* scene, const float* rays, int64_t n,
                                              int32_t* obj_id, float* t)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!scene || n < 0 || (n > 0 && (!rays || !obj_id || !t)))
        return set_error(ctx, FM_ERR_INVALID, "trace_closest_noalloc: bad arguments");
    if (n > kNoallocMaxRays)
        return set_error(ctx, FM_ERR_INVALID,
                         "trace_closest_noalloc: at most 262144 rays per call (the fixed staging area); split the batch");
    if (n == 0) return FM_OK;
    FM_CUDA_TRY(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    unsigned char* base = nullptr;
    fm_status st = scratch_for_device(ctx, &base);
    if (st != FM_OK) return st;
    uint32_t* status = reinterpret_cast<uint32_t*>(base);
    float4* d_rays = reinterpret_cast<float4*>(base + kStatusBytes);
    int32_t* d_obj = reinterpret_cast<int32_t*>(base + kStatusBytes + 32 * (size_t)kNoallocMaxRays);
    float* d_t = reinterpret_cast<float*>(base + kStatusBytes + 36 * (size_t)kNoallocMaxRays);
    cudaStream_t s = ctx->stream;
    // the staging area keeps the previous call's contents: the status word must start at 0
    FM_CUDA_TRY(ctx, cudaMemsetAsync(status, 0, sizeof(uint32_t), s), "noalloc status");
    FM_CUDA_TRY(ctx, cudaMemcpyAsync(d_rays, rays, 32 * (size_t)n, cudaMemcpyHostToDevice, s), "noalloc h2d");
    const int block = 128;
    int64_t grid = (n + block - 1) / block;
    if (grid > (int64_t)ctx->num_sms * 64) grid = (int64_t)ctx->num_sms * 64;
    k_trace_closest_staged<<<(int)grid, block, 0, s>>>(scene->dev, d_rays, n, d_obj, d_t, status);
    FM_CUDA_TRY(ctx, cudaGetLastError(), "noalloc launch");
    FM_CUDA_TRY(ctx, cudaMemcpyAsync(obj_id, d_obj, 4 * (size_t)n, cudaMemcpyDeviceToHost, s), "noalloc d2h");
    FM_CUDA_TRY(ctx, cudaMemcpyAsync(t, d_t, 4 * (size_t)n, cudaMemcpyDeviceToHost, s), "noalloc d2h");
    uint32_t hs = 0;
    FM_CUDA_TRY(ctx, cudaMemcpyAsync(&hs, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "noalloc status");
    FM_CUDA_TRY(ctx, cudaStreamSynchronize(s), "noalloc sync");
    if (hs & 1u) return set_error(ctx, FM_ERR_QUEUE_OVERFLOW, "trace_closest_noalloc: traversal stack overflow");
    return FM_OK;
}
