// Device BVH construction (fm_bvh_build.cu): interface used by scene creation.
#pragma once
#include <string>
#include <vector>

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

// Per-scene figures of a built scene (fm_scene_bvh_stats).
struct BvhResult {
    int32_t num_nodes = 0, num_leaf = 0, depth = 0;
    double build_ms = 0.0;
};

// A BVH build over a batch of scenes: one wide-node array and one leaf array shared by
// the batch (allocated by the build, owned by the caller afterwards).  Scene i's nodes
// start at nodes + 5 * root[i] (child bases in its nodes are relative to that start);
// its leaf slots index the shared leaf array directly; root[i] is -1 for a scene
// without primitives.
struct BvhBatch {
    uint4* nodes = nullptr;    // 5 x uint4 per wide node
    float4* leaf = nullptr;    // 3 x float4 per leaf slot (primitive ids local to their scene)
    std::vector<int32_t> root, num_nodes, num_leaf, depth;
    double build_ms = 0.0;
};

struct BvhJob;   // a build in flight

// Pinned host bytes a build over `nscenes` scenes needs (bvh_build_batch_begin).
size_t bvh_batch_pinned_bytes(int nscenes);

// Enqueues one build over the scenes' primitives on `stream` (after the work already on
// it, which must have uploaded them): allocations (stream-ordered, from the device's
// pool), one graph launch (captured on `capture`, a stream that nothing else uses), and
// the copies of its scene table from and its counters to `h_pinned` (pinned, of
// bvh_batch_pinned_bytes, valid until bvh_build_batch_end).  Every level of the build
// serves all scenes at once.  No host wait.  Returns 0 with `job` set (null when no
// scene has primitives), or -1 with `err` set and nothing left allocated.
int bvh_build_batch_begin(cudaStream_t stream, cudaStream_t capture, const PrimSource* srcs, int nscenes,
                          void* h_pinned, int sms, BvhJob*& job, BvhBatch& out, std::string& err);

// Waits for the build, checks its counters (overflows, leaf count, depth), fills the
// per-scene figures and releases the temporaries.  Returns 0, or -1 with `err` set and
// `out`'s arrays freed.  Consumes `job`.
int bvh_build_batch_end(BvhJob* job, BvhBatch& out, std::string& err);

// Drops a job that will not be finished; frees `out`'s arrays.
void bvh_build_abort(BvhJob* job, BvhBatch& out);

}  // namespace fm
