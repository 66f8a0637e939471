// Device BVH construction (fm_bvh_build.cu): interface used by scene creation.
#pragma once
#include <string>

#include "fm_bvh.cuh"
#include "fm_scene.cuh"

namespace fm {

// Device pointers to the primitive data the builder reads.
struct PrimSource {
    int32_t num_tris, num_rects, num_spheres;
    const float* tri_pos;       // [num_tris*9]
    const RectDev* rects;       // [num_rects]
    const SphereDev* spheres;   // [num_spheres]
};

struct BvhResult {
    uint4* nodes = nullptr;    // 5 x uint4 per wide node (cudaMalloc'd, owned by the caller)
    float4* leaf = nullptr;    // 3 x float4 per leaf slot (cudaMalloc'd, owned by the caller)
    int32_t num_nodes = 0, num_leaf = 0, depth = 0;
    double build_ms = 0.0;
};

struct BvhJob;   // a build in flight

// Enqueues the wide-BVH build on `stream`: allocations (stream-ordered, from the device's
// pool), one graph launch, and the copy of the build's 16 counters into `h_counters`
// (pinned host memory that stays valid until bvh_build_end).  The graph is captured on
// `capture`, a stream that nothing else uses (work another thread puts on `stream`
// meanwhile must not join the capture).  `out.nodes` / `out.leaf` are allocated here.  No
// host wait.  Returns 0 with `job` set (null for an empty scene), or -1 with `err` set and
// nothing left allocated.
int bvh_build_begin(cudaStream_t stream, cudaStream_t capture, const PrimSource& src, int32_t* h_counters, int sms,
                    BvhJob*& job, BvhResult& out, std::string& err);

// Waits for the build, checks its counters (overflows, leaf count, depth), fills
// out.num_nodes / num_leaf / depth / build_ms and releases the temporaries.  Returns 0, or
// -1 with `err` set and `out` freed.  Consumes `job`.
int bvh_build_end(BvhJob* job, BvhResult& out, std::string& err);

// Drops a job that will not be finished (another scene of its batch failed); frees `out`.
void bvh_build_abort(BvhJob* job, BvhResult& out);

}  // namespace fm
