// 8-wide compressed BVH: node format and traversal.
//
// Node (80 bytes = 5 x uint4), one per internal node of the wide tree:
//   w0: origin p.xyz (float), byte-packed [ex, ey, ez, imask]
//   w1: child_base, prim_base, meta[0..3], meta[4..7]
//   w2: qlo_x[0..7], qlo_y[0..7]      w3: qlo_z[0..7], qhi_x[0..7]
//   w4: qhi_y[0..7], qhi_z[0..7]
// Child i's box is p + q * 2^(e-127) per axis; the quantized box is rounded outward, so
// it always contains the exact box.  imask bit i marks child i as an internal node; the
// internal children are stored contiguously from child_base in slot order.  A leaf child
// holds 1-3 primitives at prim_base + (meta & 31); meta >> 5 is the unary count
// (1 -> 0b001, 2 -> 0b011, 3 -> 0b111).  Empty slots have meta 0.
//
// Slots are assigned by octant of the child's centroid relative to the node centre at
// build time, so that visiting slots in the order key = slot ^ ray_octant (highest
// first) is approximately front to back.
//
// Traversal keeps a short stack of node groups (child_base, hit bits << 24 | imask),
// one entry per tree level at most, and tests each node's leaf primitives as soon as
// the node is intersected.  The stack is an accessor type: a plain per-thread array
// (LocalStack), or one whose top entries live in shared memory (SharedTopStack), which
// keeps the traversal's most frequent stack traffic out of the L1 cache that holds the
// nodes.
#pragma once
#include "fm_common.cuh"
#include "fm_scene.cuh"
#include "fm_triangle.cuh"

namespace fm {

constexpr int kTraversalStack = 32;   // the builder rejects trees deeper than this
constexpr uint32_t kSphereFlag = 0x80000000u;

// The fields of a DevScene the traversal reads, kept in registers.
struct TraceScene {
    const uint4* nodes;
    const float4* leaf;
    const SphereDev* spheres;
    int32_t num_nodes, num_tris;
};

FM_HD TraceScene trace_scene(const DevScene& S) { return TraceScene{S.nodes, S.leaf, S.spheres, S.num_nodes, S.num_tris}; }

struct Hit {
    float t;
    int32_t prim;   // -1 on a miss
    float b1, b2;   // barycentrics of v1 and v2 (triangles)
};

FM_D float byte_f(uint32_t w, int k) { return (float)((w >> (8 * k)) & 0xffu); }

// Intersect the 8 children of `node`; returns the internal hit bits (<< 24, keyed by
// slot ^ oct) | imask in node_bits, and the primitive hit bits in prim_bits.
FM_D void intersect_node(const uint4* __restrict__ nodes, int node, f3 o, f3 idir, uint32_t oct, float tmin,
                         float tmax, uint32_t& child_base, uint32_t& node_bits, uint32_t& prim_base,
                         uint32_t& prim_bits)
{
    const uint4* np = nodes + 5 * (size_t)node;
    const uint4 w0 = __ldg(np + 0);
    const uint4 w1 = __ldg(np + 1);
    const uint4 w2 = __ldg(np + 2);
    const uint4 w3 = __ldg(np + 3);
    const uint4 w4 = __ldg(np + 4);
    const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
    const uint32_t ex = w0.w & 0xffu, ey = (w0.w >> 8) & 0xffu, ez = (w0.w >> 16) & 0xffu;
    const uint32_t imask = w0.w >> 24;
    const float ax = __uint_as_float(ex << 23) * idir.x;
    const float ay = __uint_as_float(ey << 23) * idir.y;
    const float az = __uint_as_float(ez << 23) * idir.z;
    const float bx = (px - o.x) * idir.x;
    const float by = (py - o.y) * idir.y;
    const float bz = (pz - o.z) * idir.z;
    uint32_t nbits = 0, pbits = 0, hmask = 0;
    const float tfar_limit = tmax;
    // Near and far planes per axis chosen once per node from the ray's direction signs
    // (t = q a + b grows with q when a = 2^e / d >= 0), so the per-child slab test needs
    // no min / max to order the two planes.  Equal to min / max of the two plane
    // distances, so the results do not change.
    const bool sx = idir.x >= 0.0f, sy = idir.y >= 0.0f, sz = idir.z >= 0.0f;
    const uint32_t nx0 = sx ? w2.x : w3.z, nx1 = sx ? w2.y : w3.w, fx0 = sx ? w3.z : w2.x, fx1 = sx ? w3.w : w2.y;
    const uint32_t ny0 = sy ? w2.z : w4.x, ny1 = sy ? w2.w : w4.y, fy0 = sy ? w4.x : w2.z, fy1 = sy ? w4.y : w2.w;
    const uint32_t nz0 = sz ? w3.x : w4.z, nz1 = sz ? w3.y : w4.w, fz0 = sz ? w4.z : w3.x, fz1 = sz ? w4.w : w3.y;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t wm = i < 4 ? w1.z : w1.w;
        const uint32_t meta = (wm >> (8 * (i & 3))) & 0xffu;
        const int k = i & 3;
        const float txn = fmaf(byte_f(i < 4 ? nx0 : nx1, k), ax, bx), txf = fmaf(byte_f(i < 4 ? fx0 : fx1, k), ax, bx);
        const float tyn = fmaf(byte_f(i < 4 ? ny0 : ny1, k), ay, by), tyf = fmaf(byte_f(i < 4 ? fy0 : fy1, k), ay, by);
        const float tzn = fmaf(byte_f(i < 4 ? nz0 : nz1, k), az, bz), tzf = fmaf(byte_f(i < 4 ? fz0 : fz1, k), az, bz);
        // The slab interval with three-input integer min / max on the float bits (one
        // instruction each instead of two float ones).  Signed-integer order is float
        // order among non-negative floats and puts every negative float below them, so
        // tn, a maximum that includes tmin >= 0, is the float maximum exactly; tf is the
        // float minimum when it is non-negative and otherwise some negative candidate,
        // which rejects the box just as the float minimum does (tn >= 0) except within
        // 1e-30 of zero, where it can only accept a box more -- never reject one.
        // An empty slot (meta 0) needs no branch: its bits below are zero.
        const float tn = __int_as_float(__vimax3_s32(__float_as_int(txn), __float_as_int(tyn),
                                                     max(__float_as_int(tzn), __float_as_int(tmin))));
        const float tf = __int_as_float(__vimin3_s32(__float_as_int(txf), __float_as_int(tyf),
                                                     min(__float_as_int(tzf), __float_as_int(tfar_limit))));
        // Widen the interval by a few ulps so that rounding in the slab arithmetic can
        // never reject a box that the exact box test accepts.
        const bool hit = tn <= tf * 1.0000010f + 1e-30f;
        hmask |= hit ? 1u << i : 0u;
        pbits |= hit && !((imask >> i) & 1u) ? (meta >> 5) << (meta & 31u) : 0u;
    }
    // internal children hit, re-keyed slot -> slot ^ oct (three conditional swaps of
    // bit groups instead of a shift per child)
    uint32_t m = hmask & imask;
    if (oct & 1u) m = ((m & 0x55u) << 1) | ((m >> 1) & 0x55u);
    if (oct & 2u) m = ((m & 0x33u) << 2) | ((m >> 2) & 0x33u);
    if (oct & 4u) m = ((m & 0x0fu) << 4) | ((m >> 4) & 0x0fu);
    nbits = m << 24;
    child_base = w1.x;
    prim_base = w1.y;
    node_bits = nbits | imask;
    prim_bits = pbits;
}

// Leaf primitive test.  Closest-hit acceptance follows the reference: a triangle of a
// mesh is accepted when IntersectTriangle(t_min, t_best) succeeds and not
// (t > t_best || t <= 0) (triangle.cpp:211-225, bvh_aggregate.cpp:108-115); rectangle
// halves skip the second check (rectangle.cpp:42-56); spheres use the inclusive range
// (sphere.cpp:116-127).
FM_D bool test_prim(const TraceScene& S, const RayPre& rp, f3 o, f3 d, int slot, float tmin, float& tbest,
                    Hit& hit, bool any)
{
    // all three records at once (a sphere's slot has them too), so the loads overlap
    const float4 a = __ldg(S.leaf + 3 * (size_t)slot);
    const float4 b = __ldg(S.leaf + 3 * (size_t)slot + 1);
    const float4 c = __ldg(S.leaf + 3 * (size_t)slot + 2);
    const uint32_t tag = __float_as_uint(a.w);
    if (tag & kSphereFlag) {
        const int sidx = (int)__float_as_uint(a.x);
        const SphereDev& sp = S.spheres[sidx];
        float t;
        if (!intersect_sphere(sp.w2o, sp.radius, o, d, tmin, tbest, t)) return false;
        hit.prim = (int)(tag & ~kSphereFlag);
        if (!any) {
            tbest = t;
            hit.t = t;
            hit.b1 = hit.b2 = 0.0f;
        }
        return true;
    }
    float t, b0, b1, b2;
    if (!intersect_triangle(rp, f3{a.x, a.y, a.z}, f3{b.x, b.y, b.z}, f3{c.x, c.y, c.z}, tmin, tbest, t, b0, b1, b2))
        return false;
    const int prim = (int)tag;
    if (any) {
        hit.prim = prim;
        return true;
    }
    if (prim < S.num_tris && (t > tbest || t <= 0.0f)) return false;
    tbest = t;
    hit.t = t;
    hit.prim = prim;
    hit.b1 = b1;
    hit.b2 = b2;
    return true;
}

// A per-thread traversal stack in local memory.
struct LocalStack {
    uint2 e[kTraversalStack];
    FM_D void put(int i, uint2 v) { e[i] = v; }
    FM_D uint2 get(int i) const { return e[i]; }
};

// A traversal stack whose K top entries are in shared memory (entry i of thread tid at
// top[i * stride], stride = the block size, so a warp's accesses are consecutive 8-byte
// words) and whose deeper entries are in local memory.
template <int K>
struct SharedTopStack {
    uint2* top;
    int stride;
    uint2 e[kTraversalStack - K];
    FM_D void put(int i, uint2 v)
    {
        if (i < K)
            top[i * stride] = v;
        else
            e[i - K] = v;
    }
    FM_D uint2 get(int i) const { return i < K ? top[i * stride] : e[i - K]; }
};

// Resumable traversal: the state of one query, advanced one node at a time by
// trav_step.  Kernels that keep a warp busy with a stream of rays (fetching a new ray
// into a lane as soon as its query completes) drive it directly; trace_ray_any runs it
// to completion.
struct Traversal {
    RayPre rp;        // rp.o is the ray origin
    f3 d, idir;
    uint32_t oct;
    float tmin, tbest;
    bool any;
    int sp;
    uint2 ngrp, pgrp;
    Hit hit;
};

FM_D void trav_begin(Traversal& t, const TraceScene& S, f3 o, f3 d, float tmin, float tmax, bool any)
{
    t.hit.t = tmax;
    t.hit.prim = -1;
    t.hit.b1 = t.hit.b2 = 0.0f;
    t.rp = ray_pre(o, d);
    t.d = d;
    const float sdx = fabsf(d.x) < 1e-20f ? copysignf(1e-20f, d.x) : d.x;
    const float sdy = fabsf(d.y) < 1e-20f ? copysignf(1e-20f, d.y) : d.y;
    const float sdz = fabsf(d.z) < 1e-20f ? copysignf(1e-20f, d.z) : d.z;
    t.idir = f3{1.0f / sdx, 1.0f / sdy, 1.0f / sdz};
    t.oct = (d.x >= 0.0f ? 1u : 0u) | (d.y >= 0.0f ? 2u : 0u) | (d.z >= 0.0f ? 4u : 0u);
    t.tmin = tmin;
    t.tbest = tmax;
    t.any = any;
    t.sp = 0;
    // virtual parent of the root: one internal child in slot 0 (none for an empty tree)
    t.ngrp = S.num_nodes == 0 ? make_uint2(0u, 0u) : make_uint2(0u, (1u << (24 + (0u ^ t.oct))) | 1u);
    t.pgrp = make_uint2(0u, 0u);
}

// Visits the nearest pending child node, tests the primitives it exposes and pops the
// stack when the current group is exhausted.  Returns true when the query is complete
// (t.hit.prim >= 0 on a hit).  *overflow is set when the traversal stack would overflow
// (the builder bounds the tree depth so that this cannot happen for trees it accepted).
template <class Stack>
FM_D bool trav_step(Traversal& t, const TraceScene& S, Stack& stack, uint32_t* overflow)
{
    if (t.ngrp.y > 0x00ffffffu) {
        const uint32_t key = 31u - __clz(t.ngrp.y) - 24u;
        t.ngrp.y &= ~(1u << (24u + key));
        const uint32_t slot = key ^ t.oct;
        const uint32_t imask = t.ngrp.y & 0xffu;
        const int child = (int)(t.ngrp.x + __popc(imask & ((1u << slot) - 1u)));
        if (t.ngrp.y > 0x00ffffffu) {
            if (t.sp < kTraversalStack)
                stack.put(t.sp++, t.ngrp);
            else if (overflow)
                atomicOr(overflow, 1u);
        }
        uint32_t cb, nb, pb, pbits;
        intersect_node(S.nodes, child, t.rp.o, t.idir, t.oct, t.tmin, t.tbest, cb, nb, pb, pbits);
        t.ngrp = make_uint2(cb, nb);
        t.pgrp = make_uint2(pb, pbits);
    }
    while (t.pgrp.y != 0u) {
        const int bit = __ffs(t.pgrp.y) - 1;
        t.pgrp.y &= t.pgrp.y - 1u;
        if (test_prim(S, t.rp, t.rp.o, t.d, (int)t.pgrp.x + bit, t.tmin, t.tbest, t.hit, t.any) && t.any) return true;
    }
    if (t.ngrp.y <= 0x00ffffffu) {
        if (t.sp == 0) return true;
        t.ngrp = stack.get(--t.sp);
    }
    return false;
}

// Closest hit (any = false) or occlusion (any = true) query; hit.prim >= 0 on a hit.
// Not inlined: a kernel that traces several kinds of rays holds one copy of the
// traversal loop, which keeps its code within the instruction caches.
static __device__ __noinline__ Hit trace_ray_any(TraceScene S, f3 o, f3 d, float tmin, float tmax, bool any,
                                                 uint32_t* overflow)
{
    Traversal t;
    LocalStack stack;
    trav_begin(t, S, o, d, tmin, tmax, any);
    while (!trav_step(t, S, stack, overflow)) {
    }
    return t.hit;
}

template <bool ANY>
FM_D bool trace_ray(const TraceScene& S, f3 o, f3 d, float tmin, float tmax, Hit& hit, uint32_t* overflow)
{
    hit = trace_ray_any(S, o, d, tmin, tmax, ANY, overflow);
    return hit.prim >= 0;
}

template <bool ANY>
FM_D bool trace_ray(const DevScene& S, f3 o, f3 d, float tmin, float tmax, Hit& hit, uint32_t* overflow)
{
    return trace_ray<ANY>(trace_scene(S), o, d, tmin, tmax, hit, overflow);
}

}  // namespace fm
