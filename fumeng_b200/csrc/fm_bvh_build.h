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

// Builds the wide BVH on `stream`.  Returns 0 on success, -1 with `err` set otherwise.
int bvh_build(cudaStream_t stream, const PrimSource& src, BvhResult& out, std::string& err);

}  // namespace fm
