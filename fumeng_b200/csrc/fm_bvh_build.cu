// Device BVH construction: binned SAH (top-down, breadth first) into a binary tree, an
// exact-SAH sweep for clusters of <= 32 primitives, then collapse into the 8-wide
// compressed node format of fm_bvh.cuh.
//
// The reference builds a median-split binary BVH on the CPU (accelerator/
// bvh_aggregate.cpp:38-79, leaf <= 5).  The tree shape does not change closest-hit
// results (every primitive whose exact box the ray enters is tested, and the
// primitive test is the reference's), so the device builder is free to optimise for
// traversal cost.
//
// Determinism: bins are accumulated with integer and order-preserving float atomics,
// whose results do not depend on scheduling; the partition is a stable scatter driven by
// a device-wide exclusive scan.  Node numbering uses atomic counters and therefore
// varies between builds, which changes no query result.
#include "fm_bvh_build.h"

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

namespace fm {

namespace {

// 8 bins: on the batched workload (64 scenes of displaced meshes) the trees traced
// faster than with 4, 16 or 32 (trace kernel 248 ms per step against 255 ms at 16).
constexpr int kBins = 8;
constexpr int kSmall = 32;     // clusters of <= kSmall primitives are built by one thread
constexpr int kLeafMax = 3;    // primitives per leaf (a wide-node leaf slot holds <= 3)
constexpr int kScanBlock = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanBlock * kScanItems;

struct BNode {
    float lo[3], hi[3];
    int32_t a, b;   // internal: children; leaf: a = ~begin (< 0), b = count
};

struct Task {
    int32_t node, begin, count, pad;
    float cmin[3], cmax[3];
};

// Per-task bins: for each axis and bin, count, box (lo/hi) and centroid box, as ordered
// uints for atomic min/max.
struct Bins {
    uint32_t cnt[3][kBins];
    uint32_t lo[3][kBins][3], hi[3][kBins][3];
    uint32_t clo[3][kBins][3], chi[3][kBins][3];
};

struct Split {
    int32_t axis;   // -1: median split by position
    int32_t bin;    // left = bins [0, bin]
    int32_t nl;
    int32_t child_task[2];   // -1 when the child is a small cluster
};

// A scene of a batched build: its primitives are positions [begin, begin + count) of the
// batch, its root is binary and wide node `root` (-1 for an empty scene).
struct BatchScene {
    PrimSource src;
    int32_t begin, count, root, pad;
};

// The scene of batch position g: the last scene that begins at or before g (empty scenes
// share their begin with the next one and are skipped by taking the last).
FM_D int scene_of(const BatchScene* __restrict__ scenes, int nscenes, int g)
{
    int lo = 0, hi = nscenes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (scenes[mid].begin <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

FM_D int bin_of(float c, float cmin, float scale)
{
    int b = (int)((c - cmin) * scale);
    return b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
}

FM_HD float half_area(const float* lo, const float* hi)
{
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (!(dx >= 0.0f) || !(dy >= 0.0f) || !(dz >= 0.0f)) return 0.0f;
    return dx * dy + dy * dz + dz * dx;
}

// The level loops run on the device (see bvh_build): kernels whose work depends on a
// level's task or frontier count read that count from device memory and stride over
// it with a fixed grid.
__global__ void k_init_bins(Bins* bins, const int32_t* ntasks_p)
{
    const int ntasks = *ntasks_p;
    const int nw = sizeof(Bins) / 4;
    const int ncnt = 3 * kBins;
    const int nlo = ncnt + 3 * kBins * 3;
    const int nhi = nlo + 3 * kBins * 3;
    const int nclo = nhi + 3 * kBins * 3;
    for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
        uint32_t* w = reinterpret_cast<uint32_t*>(bins + t);
        for (int i = threadIdx.x; i < nw; i += blockDim.x) {
            uint32_t v;
            if (i < ncnt) v = 0u;
            else if (i < nlo) v = 0xffffffffu;   // min slots start at +max
            else if (i < nhi) v = 0u;            // max slots start at -max
            else if (i < nclo) v = 0xffffffffu;
            else v = 0u;
            w[i] = v;
        }
    }
}

// Root-bounds accumulators (12 per scene) before k_root_bounds: minima at +inf bits,
// maxima at 0 (orderable-uint encoding of the bounds).
__global__ void k_init_root_bounds(uint32_t* rb, int nscenes)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 12 * nscenes; i += gridDim.x * blockDim.x)
        rb[i] = (i % 6) < 3 ? 0xffffffffu : 0u;
}

// Per-scene bounds: [0..2] centroid min, [3..5] centroid max, [6..8] box min, [9..11]
// box max, 12 words per scene.  A warp whose primitives all belong to one scene reduces
// them first and updates once (the usual case: scenes are contiguous ranges); a warp
// that straddles a scene boundary updates per lane.
__global__ void k_root_bounds(const float4* __restrict__ plo, const float4* __restrict__ phi,
                              const int32_t* __restrict__ prim_scene, int n, uint32_t* rb)
{
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const int i = base + threadIdx.x;
        const bool valid = i < n;
        float cmn[3] = {kRealMax, kRealMax, kRealMax}, cmx[3] = {-kRealMax, -kRealMax, -kRealMax};
        float bmn[3] = {kRealMax, kRealMax, kRealMax}, bmx[3] = {-kRealMax, -kRealMax, -kRealMax};
        // lanes past the end take the last primitive's scene with empty bounds
        const int s = prim_scene[valid ? i : n - 1];
        if (valid) {
            const float4 l = plo[i], h = phi[i];
            const float lv[3] = {l.x, l.y, l.z}, hv[3] = {h.x, h.y, h.z};
            for (int a = 0; a < 3; ++a) {
                const float c = 0.5f * (lv[a] + hv[a]);
                cmn[a] = cmx[a] = c;
                bmn[a] = lv[a];
                bmx[a] = hv[a];
            }
        }
        const int s0 = __shfl_sync(0xffffffffu, s, 0);
        if (__all_sync(0xffffffffu, s == s0)) {
            for (int a = 0; a < 3; ++a) {
                for (int off = 16; off > 0; off >>= 1) {
                    cmn[a] = fminf(cmn[a], __shfl_xor_sync(0xffffffffu, cmn[a], off));
                    cmx[a] = fmaxf(cmx[a], __shfl_xor_sync(0xffffffffu, cmx[a], off));
                    bmn[a] = fminf(bmn[a], __shfl_xor_sync(0xffffffffu, bmn[a], off));
                    bmx[a] = fmaxf(bmx[a], __shfl_xor_sync(0xffffffffu, bmx[a], off));
                }
            }
            if ((threadIdx.x & 31) != 0) continue;
        } else if (!valid) {
            continue;
        }
        uint32_t* out = rb + 12 * s;
        for (int a = 0; a < 3; ++a) {
            atomicMin(out + a, f2ord(cmn[a]));
            atomicMax(out + 3 + a, f2ord(cmx[a]));
            atomicMin(out + 6 + a, f2ord(bmn[a]));
            atomicMax(out + 9 + a, f2ord(bmx[a]));
        }
    }
}

// One thread per scene: the scene's root binary node (node index = the scene's root
// index) and either a root task or, for <= kSmall primitives, a small cluster.
__global__ void k_make_roots(const BatchScene* __restrict__ scenes, int nscenes, const uint32_t* rb, BNode* nodes,
                             Task* tasks, int32_t* small_list, int32_t* counters, int32_t* scene_task, int nroots)
{
    // counters: [0] node count, [1] next-level task count, [2] small-cluster count
    if (blockIdx.x == 0 && threadIdx.x == 0) counters[0] = nroots;
    for (int si = blockIdx.x * blockDim.x + threadIdx.x; si < nscenes; si += gridDim.x * blockDim.x) {
        const BatchScene sc = scenes[si];
        scene_task[si] = -1;
        if (sc.count == 0) continue;
        const uint32_t* r = rb + 12 * si;
        BNode root;
        for (int a = 0; a < 3; ++a) {
            root.lo[a] = ord2f(r[6 + a]);
            root.hi[a] = ord2f(r[9 + a]);
        }
        root.a = 0;
        root.b = 0;
        nodes[sc.root] = root;
        if (sc.count <= kSmall) {
            const int q = atomicAdd(&counters[2], 1);
            small_list[3 * q + 0] = sc.root;    // node
            small_list[3 * q + 1] = sc.begin;   // begin
            small_list[3 * q + 2] = sc.count;   // count
        } else {
            const int q = atomicAdd(&counters[1], 1);
            Task t;
            t.node = sc.root;
            t.begin = sc.begin;
            t.count = sc.count;
            t.pad = 0;
            for (int a = 0; a < 3; ++a) {
                t.cmin[a] = ord2f(r[a]);
                t.cmax[a] = ord2f(r[3 + a]);
            }
            tasks[q] = t;
            scene_task[si] = q;
        }
    }
}

__global__ void k_fill_pos_task(int32_t* pos_task, int32_t* pidx, const int32_t* __restrict__ prim_scene,
                                const int32_t* __restrict__ scene_task, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        pos_task[i] = scene_task[prim_scene[i]];
        pidx[i] = i;
    }
}

// Binning.  Each block covers a contiguous range of positions; when the whole range
// belongs to one task (the common case in the upper levels) the block accumulates in
// shared memory and merges once, otherwise it falls back to global atomics.
__global__ void k_bin(const float4* __restrict__ plo, const float4* __restrict__ phi, const int32_t* __restrict__ pidx,
                      const int32_t* __restrict__ pos_task, const Task* __restrict__ tasks, Bins* bins, int n)
{
    __shared__ Bins sb;
    __shared__ int s_task;
    const int begin = blockIdx.x * blockDim.x * 4;
    if (begin >= n) return;
    const int end = min(n, begin + (int)blockDim.x * 4);
    if (threadIdx.x == 0) {
        const int t0 = pos_task[begin], t1 = pos_task[end - 1];
        // A run of positions between two of the same task belongs to that task (task
        // ranges are contiguous); finished positions (-1) can surround active ones.
        s_task = (t0 == t1 && t0 >= 0) ? t0 : -2;
    }
    __syncthreads();
    const int shared_task = s_task;
    const bool use_smem = shared_task >= 0;
    if (use_smem) {
        uint32_t* w = reinterpret_cast<uint32_t*>(&sb);
        const int nw = sizeof(Bins) / 4;
        const int ncnt = 3 * kBins;
        const int nlo = ncnt + 3 * kBins * 3;
        const int nhi = nlo + 3 * kBins * 3;
        const int nclo = nhi + 3 * kBins * 3;
        for (int i = threadIdx.x; i < nw; i += blockDim.x)
            w[i] = (i < ncnt) ? 0u : (i < nlo ? 0xffffffffu : (i < nhi ? 0u : (i < nclo ? 0xffffffffu : 0u)));
        __syncthreads();
    }
    for (int i = begin + threadIdx.x; i < end; i += blockDim.x) {
        const int t = pos_task[i];
        if (t < 0) continue;
        const Task& tk = tasks[t];
        const int p = pidx[i];
        const float4 l = plo[p], h = phi[p];
        const float lv[3] = {l.x, l.y, l.z}, hv[3] = {h.x, h.y, h.z};
        Bins* B = use_smem ? &sb : bins + t;
        for (int a = 0; a < 3; ++a) {
            const float ext = tk.cmax[a] - tk.cmin[a];
            if (!(ext > 0.0f)) continue;
            const float c = 0.5f * (lv[a] + hv[a]);
            const float scale = (float)kBins * (1.0f - 1e-6f) / ext;
            const int b = bin_of(c, tk.cmin[a], scale);
            atomicAdd(&B->cnt[a][b], 1u);
            for (int k = 0; k < 3; ++k) {
                const float ck = 0.5f * (lv[k] + hv[k]);
                atomicMin(&B->lo[a][b][k], f2ord(lv[k]));
                atomicMax(&B->hi[a][b][k], f2ord(hv[k]));
                atomicMin(&B->clo[a][b][k], f2ord(ck));
                atomicMax(&B->chi[a][b][k], f2ord(ck));
            }
        }
    }
    if (use_smem) {
        __syncthreads();
        Bins* G = bins + shared_task;
        for (int a = 0; a < 3; ++a)
            for (int b = threadIdx.x; b < kBins; b += blockDim.x) {
                if (sb.cnt[a][b] == 0u) continue;
                atomicAdd(&G->cnt[a][b], sb.cnt[a][b]);
                for (int k = 0; k < 3; ++k) {
                    atomicMin(&G->lo[a][b][k], sb.lo[a][b][k]);
                    atomicMax(&G->hi[a][b][k], sb.hi[a][b][k]);
                    atomicMin(&G->clo[a][b][k], sb.clo[a][b][k]);
                    atomicMax(&G->chi[a][b][k], sb.chi[a][b][k]);
                }
            }
    }
}

// SAH split of task ti: choose the split from the bins, create the two child nodes
// (exact boxes from the bins) and either a next-level task or a small cluster for each.
FM_D void sah_split(const Task* __restrict__ tasks, int ti, const Bins* __restrict__ bins, Split* splits,
                    BNode* nodes, Task* next_tasks, int32_t* small_list, int32_t* counters, int32_t* pending_bounds,
                    int max_tasks)
{
    const Task tk = tasks[ti];
    const Bins& B = bins[ti];
    float best = kRealMax;
    int best_axis = -1, best_bin = -1, best_nl = 0;
    for (int a = 0; a < 3; ++a) {
        if (!(tk.cmax[a] - tk.cmin[a] > 0.0f)) continue;
        // suffix areas
        float rlo[3] = {kRealMax, kRealMax, kRealMax}, rhi[3] = {-kRealMax, -kRealMax, -kRealMax};
        float rarea[kBins];
        int rcnt[kBins];
        int acc = 0;
        for (int b = kBins - 1; b >= 0; --b) {
            if (B.cnt[a][b]) {
                for (int k = 0; k < 3; ++k) {
                    rlo[k] = fminf(rlo[k], ord2f(B.lo[a][b][k]));
                    rhi[k] = fmaxf(rhi[k], ord2f(B.hi[a][b][k]));
                }
            }
            acc += (int)B.cnt[a][b];
            rarea[b] = half_area(rlo, rhi);
            rcnt[b] = acc;
        }
        float llo[3] = {kRealMax, kRealMax, kRealMax}, lhi[3] = {-kRealMax, -kRealMax, -kRealMax};
        int lacc = 0;
        for (int b = 0; b < kBins - 1; ++b) {
            if (B.cnt[a][b]) {
                for (int k = 0; k < 3; ++k) {
                    llo[k] = fminf(llo[k], ord2f(B.lo[a][b][k]));
                    lhi[k] = fmaxf(lhi[k], ord2f(B.hi[a][b][k]));
                }
            }
            lacc += (int)B.cnt[a][b];
            const int nr = rcnt[b + 1];
            if (lacc == 0 || nr == 0) continue;
            const float cost = half_area(llo, lhi) * (float)lacc + rarea[b + 1] * (float)nr;
            if (cost < best) {
                best = cost;
                best_axis = a;
                best_bin = b;
                best_nl = lacc;
            }
        }
    }
    Split sp;
    int nl, nr;
    float clo[2][3], chi[2][3], ccl[2][3], cch[2][3];
    bool child_bounds_known = true;
    if (best_axis < 0) {
        // Every centroid falls in one bin on every axis: split the range in half.
        sp.axis = -1;
        sp.bin = 0;
        nl = tk.count / 2;
        child_bounds_known = false;
    } else {
        sp.axis = best_axis;
        sp.bin = best_bin;
        nl = best_nl;
        for (int s = 0; s < 2; ++s)
            for (int k = 0; k < 3; ++k) {
                clo[s][k] = kRealMax;
                chi[s][k] = -kRealMax;
                ccl[s][k] = kRealMax;
                cch[s][k] = -kRealMax;
            }
        for (int b = 0; b < kBins; ++b) {
            if (!B.cnt[best_axis][b]) continue;
            const int s = b <= best_bin ? 0 : 1;
            for (int k = 0; k < 3; ++k) {
                clo[s][k] = fminf(clo[s][k], ord2f(B.lo[best_axis][b][k]));
                chi[s][k] = fmaxf(chi[s][k], ord2f(B.hi[best_axis][b][k]));
                ccl[s][k] = fminf(ccl[s][k], ord2f(B.clo[best_axis][b][k]));
                cch[s][k] = fmaxf(cch[s][k], ord2f(B.chi[best_axis][b][k]));
            }
        }
    }
    nr = tk.count - nl;
    sp.nl = nl;
    const int c0 = atomicAdd(&counters[0], 2);
    nodes[tk.node].a = c0;
    nodes[tk.node].b = c0 + 1;
    const int cnt[2] = {nl, nr};
    const int beg[2] = {tk.begin, tk.begin + nl};
    for (int s = 0; s < 2; ++s) {
        BNode cn;
        for (int k = 0; k < 3; ++k) {
            cn.lo[k] = child_bounds_known ? clo[s][k] : kRealMax;
            cn.hi[k] = child_bounds_known ? chi[s][k] : -kRealMax;
        }
        cn.a = 0;
        cn.b = 0;
        nodes[c0 + s] = cn;
        if (cnt[s] <= kSmall) {
            const int q = atomicAdd(&counters[2], 1);
            small_list[3 * q + 0] = c0 + s;
            small_list[3 * q + 1] = beg[s];
            small_list[3 * q + 2] = cnt[s];
            sp.child_task[s] = -1;
        } else {
            const int q = atomicAdd(&counters[1], 1);
            if (q >= max_tasks) {
                // cannot happen (tasks hold > kSmall primitives each); recorded, and the
                // primitives are left out so that the build reports a leaf-count error
                atomicOr(&counters[5], 1);
                sp.child_task[s] = -1;
                continue;
            }
            Task nt;
            nt.node = c0 + s;
            nt.begin = beg[s];
            nt.count = cnt[s];
            nt.pad = child_bounds_known ? 0 : 1;
            for (int k = 0; k < 3; ++k) {
                nt.cmin[k] = child_bounds_known ? ccl[s][k] : kRealMax;
                nt.cmax[k] = child_bounds_known ? cch[s][k] : -kRealMax;
            }
            next_tasks[q] = nt;
            sp.child_task[s] = q;
        }
    }
    if (!child_bounds_known) atomicAdd(pending_bounds, 1);
    splits[ti] = sp;
}

// One thread per task of the level.
__global__ void k_sah(const Task* __restrict__ tasks, const int32_t* ntasks_p, const Bins* __restrict__ bins,
                      Split* splits, BNode* nodes, Task* next_tasks, int32_t* small_list, int32_t* counters,
                      int32_t* pending_bounds, int max_tasks)
{
    const int ntasks = *ntasks_p;
    for (int ti = blockIdx.x * blockDim.x + threadIdx.x; ti < ntasks; ti += gridDim.x * blockDim.x)
        sah_split(tasks, ti, bins, splits, nodes, next_tasks, small_list, counters, pending_bounds, max_tasks);
}

__global__ void k_flags(const float4* __restrict__ plo, const float4* __restrict__ phi, const int32_t* __restrict__ pidx,
                        const int32_t* __restrict__ pos_task, const Task* __restrict__ tasks,
                        const Split* __restrict__ splits, int32_t* flags, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int t = pos_task[i];
        int f = 0;
        if (t >= 0) {
            const Split sp = splits[t];
            const Task& tk = tasks[t];
            if (sp.axis < 0) {
                f = (i - tk.begin) < sp.nl ? 1 : 0;
            } else {
                const int a = sp.axis;
                const int p = pidx[i];
                const float c = 0.5f * ((&plo[p].x)[a] + (&phi[p].x)[a]);
                const float ext = tk.cmax[a] - tk.cmin[a];
                const float scale = (float)kBins * (1.0f - 1e-6f) / ext;
                f = bin_of(c, tk.cmin[a], scale) <= sp.bin ? 1 : 0;
            }
        }
        flags[i] = f;
    }
}

// Exclusive scan, three phases.
__global__ void k_scan_tiles(const int32_t* in, int32_t* out, int32_t* tile_sums, int n)
{
    __shared__ int32_t s[kScanBlock];
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int v[kScanItems];
    int sum = 0;
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        sum += v[k];
    }
    s[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < kScanBlock; off <<= 1) {
        const int x = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
        __syncthreads();
        s[threadIdx.x] += x;
        __syncthreads();
    }
    int run = s[threadIdx.x] - sum;
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == kScanBlock - 1) tile_sums[blockIdx.x] = s[threadIdx.x];
}

__global__ void k_scan_sums(int32_t* sums, int ntiles, int32_t* total)
{
    __shared__ int32_t s[kScanBlock];
    int carry = 0;
    for (int base = 0; base < ntiles; base += kScanBlock) {
        const int i = base + threadIdx.x;
        const int v = i < ntiles ? sums[i] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int off = 1; off < kScanBlock; off <<= 1) {
            const int x = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
            __syncthreads();
            s[threadIdx.x] += x;
            __syncthreads();
        }
        if (i < ntiles) sums[i] = carry + s[threadIdx.x] - v;
        const int tot = s[kScanBlock - 1];
        __syncthreads();
        carry += tot;
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(int32_t* out, const int32_t* sums, int n)
{
    const int base = blockIdx.x * kScanTile;
    const int add = sums[blockIdx.x];
    for (int k = threadIdx.x; k < kScanTile; k += blockDim.x) {
        const int i = base + k;
        if (i < n) out[i] += add;
    }
}

__global__ void k_scatter(const int32_t* __restrict__ pidx, const int32_t* __restrict__ pos_task,
                          const Task* __restrict__ tasks, const Split* __restrict__ splits,
                          const int32_t* __restrict__ flags, const int32_t* __restrict__ scan,
                          int32_t* pidx_out, int32_t* pos_task_out, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int t = pos_task[i];
        if (t < 0) {
            pidx_out[i] = pidx[i];
            pos_task_out[i] = -1;
            continue;
        }
        const Task& tk = tasks[t];
        const Split& sp = splits[t];
        const int lbefore = scan[i] - scan[tk.begin];
        int np, child;
        if (flags[i]) {
            np = tk.begin + lbefore;
            child = sp.child_task[0];
        } else {
            np = tk.begin + sp.nl + (i - tk.begin - lbefore);
            child = sp.child_task[1];
        }
        pidx_out[np] = pidx[i];
        pos_task_out[np] = child;
    }
}

// Boxes of children created by a median split are accumulated here after the scatter.
__global__ void k_pending_bounds(const float4* __restrict__ plo, const float4* __restrict__ phi,
                                 const int32_t* __restrict__ pidx, const Task* __restrict__ tasks, const Split* splits,
                                 const int32_t* ntasks_p, const int32_t* pending_p, BNode* nodes, Task* next_tasks)
{
    // One block per task of the previous level whose split was a median split.
    if (*pending_p == 0) return;
    const int ntasks = *ntasks_p;
    for (int ti = blockIdx.x; ti < ntasks; ti += gridDim.x) {
        const Split sp = splits[ti];
        if (sp.axis >= 0) continue;
        const Task tk = tasks[ti];
        for (int s = 0; s < 2; ++s) {
            const int beg = s == 0 ? tk.begin : tk.begin + sp.nl;
            const int cnt = s == 0 ? sp.nl : tk.count - sp.nl;
            const int node = nodes[tk.node].a + s;
            for (int i = beg + threadIdx.x; i < beg + cnt; i += blockDim.x) {
                const int p = pidx[i];
                const float4 l = plo[p], h = phi[p];
                const float lv[3] = {l.x, l.y, l.z}, hv[3] = {h.x, h.y, h.z};
                for (int k = 0; k < 3; ++k) {
                    // nodes hold floats; use a CAS loop through the ordered encoding
                    float* lo = &nodes[node].lo[k];
                    float* hi = &nodes[node].hi[k];
                    int* li = reinterpret_cast<int*>(lo);
                    int* hiI = reinterpret_cast<int*>(hi);
                    int old = *li;
                    while (lv[k] < __int_as_float(old)) {
                        const int prev = atomicCAS(li, old, __float_as_int(lv[k]));
                        if (prev == old) break;
                        old = prev;
                    }
                    old = *hiI;
                    while (hv[k] > __int_as_float(old)) {
                        const int prev = atomicCAS(hiI, old, __float_as_int(hv[k]));
                        if (prev == old) break;
                        old = prev;
                    }
                    if (sp.child_task[s] >= 0) {
                        const float c = 0.5f * (lv[k] + hv[k]);
                        Task& nt = next_tasks[sp.child_task[s]];
                        int* cl = reinterpret_cast<int*>(&nt.cmin[k]);
                        int* ch = reinterpret_cast<int*>(&nt.cmax[k]);
                        old = *cl;
                        while (c < __int_as_float(old)) {
                            const int prev = atomicCAS(cl, old, __float_as_int(c));
                            if (prev == old) break;
                            old = prev;
                        }
                        old = *ch;
                        while (c > __int_as_float(old)) {
                            const int prev = atomicCAS(ch, old, __float_as_int(c));
                            if (prev == old) break;
                            old = prev;
                        }
                    }
                }
            }
        }
    }
}

// Sequential exact-SAH build of cluster ci (<= kSmall primitives) by one thread.
FM_D void small_build(const float4* __restrict__ plo, const float4* __restrict__ phi, int32_t* pidx,
                      const int32_t* __restrict__ small_list, int ci, BNode* nodes, int32_t* counters)
{
    const int root = small_list[3 * ci], begin = small_list[3 * ci + 1], count = small_list[3 * ci + 2];
    int ids[kSmall];
    for (int k = 0; k < count; ++k) ids[k] = pidx[begin + k];
    // explicit stack of (node, lo, n) ranges within ids[]
    int st_node[kSmall], st_lo[kSmall], st_n[kSmall];
    int sp = 0;
    st_node[0] = root;
    st_lo[0] = 0;
    st_n[0] = count;
    sp = 1;
    {
        // the cluster root's box (may be unset after a median split higher up)
        float lo[3] = {kRealMax, kRealMax, kRealMax}, hi[3] = {-kRealMax, -kRealMax, -kRealMax};
        for (int k = 0; k < count; ++k) {
            const float4 l = plo[ids[k]], h = phi[ids[k]];
            lo[0] = fminf(lo[0], l.x); lo[1] = fminf(lo[1], l.y); lo[2] = fminf(lo[2], l.z);
            hi[0] = fmaxf(hi[0], h.x); hi[1] = fmaxf(hi[1], h.y); hi[2] = fmaxf(hi[2], h.z);
        }
        for (int a = 0; a < 3; ++a) {
            nodes[root].lo[a] = lo[a];
            nodes[root].hi[a] = hi[a];
        }
    }
    float racc[kSmall];
    while (sp > 0) {
        --sp;
        const int node = st_node[sp], lo0 = st_lo[sp], n = st_n[sp];
        float nlo[3], nhi[3];
        for (int a = 0; a < 3; ++a) {
            nlo[a] = nodes[node].lo[a];
            nhi[a] = nodes[node].hi[a];
        }
        const float parent_area = half_area(nlo, nhi);
        float best = kRealMax;
        int best_axis = -1, best_k = 0;
        if (n > 1) {
            for (int a = 0; a < 3; ++a) {
                // insertion sort of ids[lo0 .. lo0+n) by centroid along a
                for (int i = lo0 + 1; i < lo0 + n; ++i) {
                    const int v = ids[i];
                    const float cv = (&plo[v].x)[a] + (&phi[v].x)[a];
                    int j = i - 1;
                    while (j >= lo0) {
                        const int u = ids[j];
                        if ((&plo[u].x)[a] + (&phi[u].x)[a] <= cv) break;
                        ids[j + 1] = u;
                        --j;
                    }
                    ids[j + 1] = v;
                }
                float rlo[3] = {kRealMax, kRealMax, kRealMax}, rhi[3] = {-kRealMax, -kRealMax, -kRealMax};
                for (int i = n - 1; i >= 1; --i) {
                    const float4 l = plo[ids[lo0 + i]], h = phi[ids[lo0 + i]];
                    rlo[0] = fminf(rlo[0], l.x); rlo[1] = fminf(rlo[1], l.y); rlo[2] = fminf(rlo[2], l.z);
                    rhi[0] = fmaxf(rhi[0], h.x); rhi[1] = fmaxf(rhi[1], h.y); rhi[2] = fmaxf(rhi[2], h.z);
                    racc[i] = half_area(rlo, rhi);
                }
                float llo[3] = {kRealMax, kRealMax, kRealMax}, lhi[3] = {-kRealMax, -kRealMax, -kRealMax};
                for (int i = 0; i < n - 1; ++i) {
                    const float4 l = plo[ids[lo0 + i]], h = phi[ids[lo0 + i]];
                    llo[0] = fminf(llo[0], l.x); llo[1] = fminf(llo[1], l.y); llo[2] = fminf(llo[2], l.z);
                    lhi[0] = fmaxf(lhi[0], h.x); lhi[1] = fmaxf(lhi[1], h.y); lhi[2] = fmaxf(lhi[2], h.z);
                    const float cost = half_area(llo, lhi) * (float)(i + 1) + racc[i + 1] * (float)(n - i - 1);
                    if (cost < best) {
                        best = cost;
                        best_axis = a;
                        best_k = i + 1;
                    }
                }
            }
        }
        // SAH termination: a binary node costs half a primitive test.  The collapse into
        // 8-wide nodes removes most binary levels, so splitting down to single-primitive
        // leaves pays (trace kernel 270 -> 248 ms per step on the batched workload
        // against unit costs; costs of 0.25 and 0 give the same trees).
        const float split_cost = parent_area > 0.0f ? 0.5f + best / parent_area : kRealMax;
        const bool make_leaf = n <= 1 || (n <= kLeafMax && (float)n <= split_cost);
        if (make_leaf) {
            for (int k = 0; k < n; ++k) pidx[begin + lo0 + k] = ids[lo0 + k];
            nodes[node].a = ~(begin + lo0);
            nodes[node].b = n;
            continue;
        }
        if (best_axis < 0) {
            best_axis = 0;
            best_k = n / 2;
        }
        // re-sort along the chosen axis (the loop above left ids sorted along z)
        if (best_axis != 2) {
            const int a = best_axis;
            for (int i = lo0 + 1; i < lo0 + n; ++i) {
                const int v = ids[i];
                const float cv = (&plo[v].x)[a] + (&phi[v].x)[a];
                int j = i - 1;
                while (j >= lo0) {
                    const int u = ids[j];
                    if ((&plo[u].x)[a] + (&phi[u].x)[a] <= cv) break;
                    ids[j + 1] = u;
                    --j;
                }
                ids[j + 1] = v;
            }
        }
        const int c0 = atomicAdd(&counters[0], 2);
        nodes[node].a = c0;
        nodes[node].b = c0 + 1;
        const int rng_lo[2] = {lo0, lo0 + best_k};
        const int rng_n[2] = {best_k, n - best_k};
        for (int s = 0; s < 2; ++s) {
            float lo[3] = {kRealMax, kRealMax, kRealMax}, hi[3] = {-kRealMax, -kRealMax, -kRealMax};
            for (int k = 0; k < rng_n[s]; ++k) {
                const float4 l = plo[ids[rng_lo[s] + k]], h = phi[ids[rng_lo[s] + k]];
                lo[0] = fminf(lo[0], l.x); lo[1] = fminf(lo[1], l.y); lo[2] = fminf(lo[2], l.z);
                hi[0] = fmaxf(hi[0], h.x); hi[1] = fmaxf(hi[1], h.y); hi[2] = fmaxf(hi[2], h.z);
            }
            BNode cn;
            for (int a = 0; a < 3; ++a) {
                cn.lo[a] = lo[a];
                cn.hi[a] = hi[a];
            }
            cn.a = 0;
            cn.b = 0;
            nodes[c0 + s] = cn;
            st_node[sp] = c0 + s;
            st_lo[sp] = rng_lo[s];
            st_n[sp] = rng_n[s];
            ++sp;
        }
    }
}

// Sequential exact-SAH builder for one cluster of <= kSmall primitives per thread.
__global__ void k_small(const float4* __restrict__ plo, const float4* __restrict__ phi, int32_t* pidx,
                        const int32_t* __restrict__ small_list, const int32_t* nsmall_p, BNode* nodes, int32_t* counters)
{
    const int nsmall = *nsmall_p;
    for (int ci = blockIdx.x * blockDim.x + threadIdx.x; ci < nsmall; ci += gridDim.x * blockDim.x)
        small_build(plo, phi, pidx, small_list, ci, nodes, counters);
}

// ---- collapse to 8-wide nodes --------------------------------------------------

FM_D float node_area(const BNode& b) { return half_area(b.lo, b.hi); }

// SAH-optimal collapse (after Ylitie, Karras and Laine 2017, "Efficient Incoherent Ray
// Traversal on GPUs Through Compressed Wide BVHs"): for every binary node n and slot
// budget i = 1..8, c[i-1] is the least SAH cost of n's subtree when its wide parent
// gives it at most i slots.  One slot holds n as a leaf (at most kMergeMax primitives,
// cost kPrimCost * A(n) * count) or as a wide node of its own (kWideNodeCost * A(n) plus
// the best distribution of 8 slots over n's two children); i > 1 slots either leave one
// unused or split i between the two children.  The costs are computed bottom-up once per
// build (k_collapse_dp) and the choices read top-down by the collapse.  Costs: a wide
// node test 1, a primitive test 1 (measured on the batched workload against the greedy
// collapse that opens the largest child until 8 slots are used: trace 164.2 -> 161.0 ms
// per step; the same DP without merged leaves 160.7 ms; a primitive cost of 0.3, 166.2
// ms).
struct __align__(16) DpNode {
    float c[8];
    // bit 0: the one-slot choice is a leaf; bits 1-3: the left child's share of the
    // 8-slot distribution; nibble i-1 (i = 2..8): the left child's share of i slots, 0
    // when i-1 slots cost no more
    uint32_t dec;
    int32_t begin, count;   // the subtree's primitives are pidx[begin, begin + count)
    int32_t pad;
};

constexpr float kWideNodeCost = 1.0f;
constexpr float kPrimCost = 1.0f;
constexpr int kMergeMax = kLeafMax;   // a merged leaf slot holds at most 3 primitives

__global__ void k_parents(const BNode* __restrict__ bnodes, const int32_t* nnodes_p, int32_t* parent)
{
    const int nn = *nnodes_p;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const BNode& b = bnodes[i];
        if (b.a >= 0) {
            parent[b.a] = i;
            parent[b.b] = i;
        }
    }
}

FM_D void dp_leaf(const BNode& bn, DpNode& out)
{
    const float cost = kPrimCost * node_area(bn) * (float)bn.b;
#pragma unroll
    for (int i = 0; i < 8; ++i) out.c[i] = cost;
    out.dec = 1u;
    out.begin = ~bn.a;
    out.count = bn.b;
    out.pad = 0;
}

FM_D void dp_internal(const BNode& bn, const DpNode& L, const DpNode& R, DpNode& out)
{
    out.count = L.count + R.count;
    out.begin = min(L.begin, R.begin);
    out.pad = 0;
    float dist[9];
    uint32_t darg[9];
#pragma unroll
    for (int j = 2; j <= 8; ++j) {
        float best = kRealMax;
        uint32_t arg = 1u;
#pragma unroll
        for (int k = 1; k < j; ++k) {
            const float v = L.c[k - 1] + R.c[j - k - 1];
            if (v < best) {
                best = v;
                arg = (uint32_t)k;
            }
        }
        dist[j] = best;
        darg[j] = arg;
    }
    const float area = node_area(bn);
    const float c_wide = kWideNodeCost * area + dist[8];
    const float c_leaf = out.count <= kMergeMax ? kPrimCost * area * (float)out.count : kRealMax;
    uint32_t dec = darg[8] << 1;
    if (c_leaf < c_wide) {
        out.c[0] = c_leaf;
        dec |= 1u;
    } else {
        out.c[0] = c_wide;
    }
#pragma unroll
    for (int i = 2; i <= 8; ++i) {
        if (dist[i] < out.c[i - 2]) {
            out.c[i - 1] = dist[i];
            dec |= darg[i] << (4 * (i - 1));
        } else {
            out.c[i - 1] = out.c[i - 2];
        }
    }
    out.dec = dec;
}

FM_D DpNode load_dp(const DpNode* p)
{
    // through L2: the node was written by another thread of this launch
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a = __ldcg(q), b = __ldcg(q + 1), c = __ldcg(q + 2);
    DpNode d;
    d.c[0] = a.x; d.c[1] = a.y; d.c[2] = a.z; d.c[3] = a.w;
    d.c[4] = b.x; d.c[5] = b.y; d.c[6] = b.z; d.c[7] = b.w;
    d.dec = __float_as_uint(c.x);
    d.begin = __float_as_int(c.y);
    d.count = __float_as_int(c.z);
    d.pad = 0;
    return d;
}

// Bottom-up pass: a thread starts at each binary leaf and climbs while it is the second
// of a node's two children to arrive (the first stops), so every node is computed once,
// after both children.  No thread waits on another.
__global__ void k_collapse_dp(const BNode* __restrict__ bnodes, const int32_t* nnodes_p,
                              const int32_t* __restrict__ parent, int32_t* arrive, DpNode* dp)
{
    const int nn = *nnodes_p;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        const BNode leaf = bnodes[i];
        if (leaf.a >= 0) continue;
        DpNode cur;
        dp_leaf(leaf, cur);
        dp[i] = cur;
        int node = i;
        for (int level = 0; level < 4096; ++level) {
            const int p = parent[node];
            if (p < 0) break;
            __threadfence();
            if (atomicAdd(&arrive[p], 1) == 0) break;
            __threadfence();
            const BNode pn = bnodes[p];
            const DpNode L = load_dp(dp + pn.a), R = load_dp(dp + pn.b);
            DpNode out;
            dp_internal(pn, L, R, out);
            dp[p] = out;
            node = p;
        }
    }
}

// Collapses the binary subtree under frontier entry fi (binary node, wide slot, scene
// root) into one 8-wide node whose children are the slots of the root's least-cost
// 8-slot distribution (the choices of k_collapse_dp): binary leaves, subtrees of at most
// three primitives merged into one leaf slot, and wide nodes of their own.  Child bases are stored relative to the scene's root slot
// (the scene's node array starts there); leaf slots are batch-wide.  Per scene root:
// wide nodes, leaf slots and depth (the collapse level) go to stats[3 * root + 0..2].
FM_D void collapse_node(const BNode* __restrict__ bnodes, const DpNode* __restrict__ dp,
                        const int32_t* __restrict__ pidx, const int4* __restrict__ frontier, int fi,
                        int4* next_frontier, int32_t* counters, uint4* wnodes, int32_t* leaf_prim, int32_t* stats,
                        int level)
{
    const int bn = frontier[fi].x, wslot = frontier[fi].y, sroot = frontier[fi].z;
    const BNode root = bnodes[bn];
    int ch[8];
    int nch = 0;
    if (root.a < 0) {
        ch[nch++] = bn;
    } else {
        // the slots of the root's 8-slot distribution, read from the costs' choices
        int st_n[8], st_b[8];
        int sp = 0;
        const uint32_t k8 = (dp[bn].dec >> 1) & 7u;
        st_n[sp] = root.b;
        st_b[sp++] = 8 - (int)k8;
        st_n[sp] = root.a;
        st_b[sp++] = (int)k8;
        while (sp > 0 && nch < 8) {
            --sp;
            const int n = st_n[sp];
            int i = st_b[sp];
            const uint32_t d = dp[n].dec;
            while (i > 1 && ((d >> (4 * (i - 1))) & 15u) == 0u) --i;
            const BNode nd = bnodes[n];
            if (i <= 1 || nd.a < 0 || sp > 6) {
                ch[nch++] = n;
                continue;
            }
            int kl = (int)((d >> (4 * (i - 1))) & 15u);
            kl = kl < 1 ? 1 : (kl > i - 1 ? i - 1 : kl);
            st_n[sp] = nd.b;
            st_b[sp++] = i - kl;
            st_n[sp] = nd.a;
            st_b[sp++] = kl;
        }
    }
    // what each child becomes: a leaf slot (its subtree's primitives) or a wide node
    bool is_leaf[8];
    int leaf_beg[8], leaf_cnt[8];
    for (int k = 0; k < nch; ++k) {
        const BNode& c = bnodes[ch[k]];
        if (c.a < 0) {
            is_leaf[k] = true;
            leaf_beg[k] = ~c.a;
            leaf_cnt[k] = c.b;
        } else if (dp[ch[k]].dec & 1u) {
            is_leaf[k] = true;
            leaf_beg[k] = dp[ch[k]].begin;
            leaf_cnt[k] = dp[ch[k]].count;
        } else {
            is_leaf[k] = false;
            leaf_beg[k] = 0;
            leaf_cnt[k] = 0;
        }
    }
    // node box and centre
    float lo[3] = {kRealMax, kRealMax, kRealMax}, hi[3] = {-kRealMax, -kRealMax, -kRealMax};
    for (int k = 0; k < nch; ++k) {
        const BNode& c = bnodes[ch[k]];
        for (int a = 0; a < 3; ++a) {
            lo[a] = fminf(lo[a], c.lo[a]);
            hi[a] = fmaxf(hi[a], c.hi[a]);
        }
    }
    const float ctr[3] = {0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]), 0.5f * (lo[2] + hi[2])};
    // greedy octant slot assignment: farthest children first pick their best free slot
    int slot_of[8];
    bool used[8] = {false, false, false, false, false, false, false, false};
    bool done[8] = {false, false, false, false, false, false, false, false};
    for (int it = 0; it < nch; ++it) {
        int pick = -1;
        float pd = -1.0f;
        for (int k = 0; k < nch; ++k) {
            if (done[k]) continue;
            const BNode& c = bnodes[ch[k]];
            float d2 = 0.0f;
            for (int a = 0; a < 3; ++a) {
                const float dv = 0.5f * (c.lo[a] + c.hi[a]) - ctr[a];
                d2 += dv * dv;
            }
            if (d2 > pd) {
                pd = d2;
                pick = k;
            }
        }
        const BNode& c = bnodes[ch[pick]];
        float best = -kRealMax;
        int bs = 0;
        for (int s = 0; s < 8; ++s) {
            if (used[s]) continue;
            float score = 0.0f;
            for (int a = 0; a < 3; ++a) {
                const float dv = 0.5f * (c.lo[a] + c.hi[a]) - ctr[a];
                score += ((s >> a) & 1) ? dv : -dv;
            }
            if (score > best) {
                best = score;
                bs = s;
            }
        }
        used[bs] = true;
        done[pick] = true;
        slot_of[pick] = bs;
    }
    int at_slot[8];   // index into ch[], -1 for an empty slot
    for (int s = 0; s < 8; ++s) at_slot[s] = -1;
    for (int k = 0; k < nch; ++k) at_slot[slot_of[k]] = k;
    int n_int = 0, n_prim = 0;
    for (int k = 0; k < nch; ++k) {
        if (is_leaf[k]) n_prim += leaf_cnt[k];
        else ++n_int;
    }
    const int child_base = n_int ? atomicAdd(&counters[0], n_int) : 0;
    const int prim_base = n_prim ? atomicAdd(&counters[1], n_prim) : 0;
    atomicAdd(&stats[3 * sroot + 0], 1);
    if (n_prim) atomicAdd(&stats[3 * sroot + 1], n_prim);
    atomicMax(&stats[3 * sroot + 2], level);
    // quantization
    uint32_t e[3];
    float scale[3];
    for (int a = 0; a < 3; ++a) {
        const float ext = hi[a] - lo[a];
        float s = ext > 0.0f ? ext * (1.0f / 255.0f) * 1.0000005f : 0.0f;
        uint32_t bits = __float_as_uint(s);
        uint32_t ex = (bits >> 23) & 0xffu;
        if (bits & 0x7fffffu) ++ex;   // round up to a power of two
        if (ex < 1u) ex = 1u;
        if (ex > 254u) ex = 254u;
        e[a] = ex;
        scale[a] = __uint_as_float(ex << 23);
    }
    uint32_t meta[8], ql[3][8], qh[3][8];
    uint32_t imask = 0;
    int int_rank = 0, prim_off = 0;
    for (int s = 0; s < 8; ++s) {
        meta[s] = 0;
        for (int a = 0; a < 3; ++a) {
            ql[a][s] = 0;
            qh[a][s] = 0;
        }
        if (at_slot[s] < 0) continue;
        const int k = at_slot[s];
        const BNode& c = bnodes[ch[k]];
        for (int a = 0; a < 3; ++a) {
            float qlo = floorf(__fdiv_rd(__fsub_rd(c.lo[a], lo[a]), scale[a]));
            float qhi = ceilf(__fdiv_ru(__fsub_ru(c.hi[a], lo[a]), scale[a]));
            qlo = fminf(fmaxf(qlo, 0.0f), 255.0f);
            qhi = fminf(fmaxf(qhi, 0.0f), 255.0f);
            ql[a][s] = (uint32_t)qlo;
            qh[a][s] = (uint32_t)qhi;
        }
        if (!is_leaf[k]) {
            imask |= 1u << s;
            meta[s] = 0x20u | (uint32_t)(24 + s);   // nonzero marker; traversal uses imask
            const int q = atomicAdd(&counters[2], 1);
            next_frontier[q] = make_int4(ch[k], child_base + int_rank, sroot, 0);
            ++int_rank;
        } else {
            const int cnt = leaf_cnt[k], beg = leaf_beg[k];
            meta[s] = (((1u << cnt) - 1u) << 5) | (uint32_t)prim_off;
            for (int j = 0; j < cnt; ++j) leaf_prim[prim_base + prim_off + j] = pidx[beg + j];
            prim_off += cnt;
        }
    }
    auto pack4 = [](const uint32_t* v) { return v[0] | (v[1] << 8) | (v[2] << 16) | (v[3] << 24); };
    uint4* np = wnodes + 5 * (size_t)wslot;
    np[0] = make_uint4(__float_as_uint(lo[0]), __float_as_uint(lo[1]), __float_as_uint(lo[2]),
                       e[0] | (e[1] << 8) | (e[2] << 16) | (imask << 24));
    np[1] = make_uint4(n_int ? (uint32_t)(child_base - sroot) : 0u, (uint32_t)prim_base, pack4(meta), pack4(meta + 4));
    np[2] = make_uint4(pack4(ql[0]), pack4(ql[0] + 4), pack4(ql[1]), pack4(ql[1] + 4));
    np[3] = make_uint4(pack4(ql[2]), pack4(ql[2] + 4), pack4(qh[0]), pack4(qh[0] + 4));
    np[4] = make_uint4(pack4(qh[1]), pack4(qh[1] + 4), pack4(qh[2]), pack4(qh[2] + 4));
}

__global__ void k_collapse(const BNode* __restrict__ bnodes, const DpNode* __restrict__ dp,
                           const int32_t* __restrict__ pidx, const int4* __restrict__ frontier,
                           const int32_t* nfront_p, int4* next_frontier, int32_t* counters, uint4* wnodes,
                           int32_t* leaf_prim, int32_t* stats)
{
    // counters: [0] wide node count, [1] leaf slot count, [2] next frontier count, [4] level
    const int nfront = *nfront_p;
    const int level = counters[4];
    for (int fi = blockIdx.x * blockDim.x + threadIdx.x; fi < nfront; fi += gridDim.x * blockDim.x)
        collapse_node(bnodes, dp, pidx, frontier, fi, next_frontier, counters, wnodes, leaf_prim, stats, level);
}

// Leaf records: the primitive's corners (or sphere index) and its id within its scene.
__global__ void k_fill_leaf(const int32_t* __restrict__ leaf_prim, int nleaf, const BatchScene* __restrict__ scenes,
                            const int32_t* __restrict__ prim_scene, int n, float4* leaf)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nleaf; i += gridDim.x * blockDim.x) {
        const int g = leaf_prim[i];
        float4 a, b, c;
        if (g < 0 || g >= n) {
            // a slot the collapse did not fill (the build then reports a leaf-count error)
            a = b = c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else {
            const BatchScene& sc = scenes[prim_scene[g]];
            const PrimSource& src = sc.src;
            const int p = g - sc.begin;
            if (p < src.num_tris) {
                const float* v = src.tri_pos + 9 * (size_t)p;
                a = make_float4(v[0], v[1], v[2], __uint_as_float((uint32_t)p));
                b = make_float4(v[3], v[4], v[5], 0.0f);
                c = make_float4(v[6], v[7], v[8], 0.0f);
            } else if (p < src.num_tris + 2 * src.num_rects) {
                const int r = (p - src.num_tris) >> 1, h = (p - src.num_tris) & 1;
                const RectDev& R = src.rects[r];
                const float* q0 = h ? R.pc : R.pa;
                const float* q1 = h ? R.pd : R.pb;
                const float* q2 = h ? R.pa : R.pc;
                a = make_float4(q0[0], q0[1], q0[2], __uint_as_float((uint32_t)p));
                b = make_float4(q1[0], q1[1], q1[2], 0.0f);
                c = make_float4(q2[0], q2[1], q2[2], 0.0f);
            } else {
                const int sp = p - src.num_tris - 2 * src.num_rects;
                a = make_float4(__uint_as_float((uint32_t)sp), 0.0f, 0.0f, __uint_as_float((uint32_t)p | kSphereFlag));
                b = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
        }
        leaf[3 * (size_t)i] = a;
        leaf[3 * (size_t)i + 1] = b;
        leaf[3 * (size_t)i + 2] = c;
    }
}

// Primitive boxes, and each batch position's scene.
__global__ void k_prim_bounds(const BatchScene* __restrict__ scenes, int nscenes, int n, float4* plo, float4* phi,
                              int32_t* prim_scene)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const int si = scene_of(scenes, nscenes, g);
        prim_scene[g] = si;
        const PrimSource& src = scenes[si].src;
        const int p = g - scenes[si].begin;
        float lo[3], hi[3];
        if (p < src.num_tris + 2 * src.num_rects) {
            f3 v[3];
            if (p < src.num_tris) {
                const float* q = src.tri_pos + 9 * (size_t)p;
                v[0] = ld3(q);
                v[1] = ld3(q + 3);
                v[2] = ld3(q + 6);
            } else {
                const int r = (p - src.num_tris) >> 1, h = (p - src.num_tris) & 1;
                const RectDev& R = src.rects[r];
                v[0] = ld3(h ? R.pc : R.pa);
                v[1] = ld3(h ? R.pd : R.pb);
                v[2] = ld3(h ? R.pa : R.pc);
            }
            for (int a = 0; a < 3; ++a) {
                lo[a] = fminf(fminf(comp(v[0], a), comp(v[1], a)), comp(v[2], a));
                hi[a] = fmaxf(fmaxf(comp(v[0], a), comp(v[1], a)), comp(v[2], a));
            }
        } else {
            const SphereDev& S = src.spheres[p - src.num_tris - 2 * src.num_rects];
            const f3 c = f3{S.o2w.m[3], S.o2w.m[7], S.o2w.m[11]};
            for (int a = 0; a < 3; ++a) {
                lo[a] = comp(c, a) - S.radius_world;
                hi[a] = comp(c, a) + S.radius_world;
            }
        }
        plo[g] = make_float4(lo[0], lo[1], lo[2], 0.0f);
        phi[g] = make_float4(hi[0], hi[1], hi[2], 0.0f);
    }
}

// Level-loop control.  Split phase counters: [0] binary nodes, [1] tasks of the next
// level, [2] small clusters, [3] median splits awaiting child bounds, [4] tasks of the
// current level, [5] error bits, [6] loop bodies run.
__global__ void k_level_begin(int32_t* counters)
{
    counters[4] = counters[1];
    counters[1] = 0;
    counters[3] = 0;
}

__global__ void k_split_continue(int32_t* counters, cudaGraphConditionalHandle handle, int max_bodies)
{
    const int bodies = ++counters[6];
    bool more = counters[1] > 0;
    if (more && bodies >= max_bodies) {
        counters[5] |= 2;
        more = false;
    }
    cudaGraphSetConditional(handle, more ? 1u : 0u);
}

// Collapse phase counters: [0] wide nodes, [1] leaf slots, [2] next frontier, [3]
// current frontier, [4] levels, [5] loop bodies run, [6] error bits.  The first frontier
// holds every scene's root (binary node = wide slot = the root index).
__global__ void k_collapse_init(const BatchScene* __restrict__ scenes, int nscenes, int nroots, int4* front,
                                int32_t* ccnt)
{
    for (int si = blockIdx.x * blockDim.x + threadIdx.x; si < nscenes; si += gridDim.x * blockDim.x) {
        const int r = scenes[si].root;
        if (r >= 0) front[r] = make_int4(r, r, r, 0);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ccnt[0] = nroots;
        ccnt[1] = 0;
        ccnt[2] = nroots;
        ccnt[3] = 0;
        ccnt[4] = 0;
        ccnt[5] = 0;
        ccnt[6] = 0;
    }
}

__global__ void k_collapse_begin(int32_t* ccnt)
{
    const int cur = ccnt[2];
    ccnt[2] = 0;
    ccnt[3] = cur;
    if (cur > 0) ++ccnt[4];
}

__global__ void k_collapse_continue(int32_t* ccnt, cudaGraphConditionalHandle handle, int max_bodies)
{
    const int bodies = ++ccnt[5];
    bool more = ccnt[2] > 0;
    if (more && bodies >= max_bodies) {
        ccnt[6] |= 1;
        more = false;
    }
    cudaGraphSetConditional(handle, more ? 1u : 0u);
}

inline int grid_for(int64_t n, int block)
{
    int64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

}  // namespace

#define FM_BUILD_CHECK(x)                                                        \
    do {                                                                         \
        cudaError_t e__ = (x);                                                   \
        if (e__ != cudaSuccess) {                                                \
            err = std::string("bvh build: ") + cudaGetErrorString(e__);          \
            goto fail;                                                           \
        }                                                                        \
    } while (0)

namespace {

// Buffers of one build over a batch of scenes (n primitives in all).
struct BuildBufs {
    int n, max_tasks, ntiles, sms, nscenes, nroots;
    BatchScene* scenes;
    float4 *plo, *phi;
    int32_t *pidx, *pidx2, *pos_task, *pos_task2, *flags, *scan, *tile_sums, *small_list, *leaf_prim;
    int32_t *prim_scene, *scene_task;
    int32_t *parent, *arrive;   // binary node -> parent (-1 at roots); bottom-up arrival counts
    DpNode* dp;                 // per binary node: collapse costs and choices
    int64_t max_nodes;
    int32_t* meta;   // [0..15] split counters ([8..15] collapse), then 3 stats per scene root
    int32_t *counters, *ccnt, *stats;
    uint32_t* rb;
    BNode* bnodes;
    Task *tasks, *tasks2;
    Split* splits;
    Bins* bins;
    int4 *front, *front2;
    uint4* wnodes;
    float4* leaf;
};

// One split level: bins, SAH splits, stable partition of the level's primitives (in ->
// out), and the bounds of children made by median splits.  Tasks never span two scenes,
// so the level serves every scene of the batch at once.
void split_level(cudaStream_t s, const BuildBufs& b, const int32_t* pidx_in, const int32_t* pos_in,
                 const Task* tasks_in, int32_t* pidx_out, int32_t* pos_out, Task* tasks_out)
{
    const int n = b.n;
    const int task_blocks = std::min(b.max_tasks, b.sms * 16);
    k_level_begin<<<1, 1, 0, s>>>(b.counters);
    k_init_bins<<<task_blocks, 256, 0, s>>>(b.bins, b.counters + 4);
    k_bin<<<(n + 1023) / 1024, 256, 0, s>>>(b.plo, b.phi, pidx_in, pos_in, tasks_in, b.bins, n);
    k_sah<<<grid_for(b.max_tasks, 128), 128, 0, s>>>(tasks_in, b.counters + 4, b.bins, b.splits, b.bnodes, tasks_out,
                                                    b.small_list, b.counters, b.counters + 3, b.max_tasks);
    k_flags<<<grid_for(n, 256), 256, 0, s>>>(b.plo, b.phi, pidx_in, pos_in, tasks_in, b.splits, b.flags, n);
    k_scan_tiles<<<b.ntiles, kScanBlock, 0, s>>>(b.flags, b.scan, b.tile_sums, n);
    k_scan_sums<<<1, kScanBlock, 0, s>>>(b.tile_sums, b.ntiles, b.scan + n);
    k_scan_add<<<b.ntiles, 256, 0, s>>>(b.scan, b.tile_sums, n);
    k_scatter<<<grid_for(n, 256), 256, 0, s>>>(pidx_in, pos_in, tasks_in, b.splits, b.flags, b.scan, pidx_out, pos_out,
                                               n);
    k_pending_bounds<<<task_blocks, 256, 0, s>>>(b.plo, b.phi, pidx_out, tasks_in, b.splits, b.counters + 4,
                                                 b.counters + 3, b.bnodes, tasks_out);
}

void collapse_level(cudaStream_t s, const BuildBufs& b, const int4* front_in, int4* front_out)
{
    k_collapse_begin<<<1, 1, 0, s>>>(b.ccnt);
    k_collapse<<<grid_for((int64_t)b.n + b.nroots, 128), 128, 0, s>>>(b.bnodes, b.dp, b.pidx, front_in, b.ccnt + 3,
                                                                      front_out, b.ccnt, b.wnodes, b.leaf_prim,
                                                                      b.stats);
}

// Adds a WHILE node after `dep` whose body is what `body_fn` launches on `s`.
template <class F>
cudaError_t add_while(cudaGraph_t graph, cudaGraphNode_t dep, cudaStream_t s, cudaGraphConditionalHandle& handle,
                      cudaGraphNode_t& node, F&& body_fn)
{
    cudaError_t e = cudaGraphConditionalHandleCreate(&handle, graph, 1u, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&node, graph, &dep, 1, &cp);
    if (e != cudaSuccess) return e;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    body_fn(handle);
    return cudaStreamEndCapture(s, &body);
}

// Adds a child-graph node after `dep` (none when dep is null) holding what `fn` launches.
template <class F>
cudaError_t add_captured(cudaGraph_t graph, const cudaGraphNode_t* dep, cudaStream_t s, cudaGraphNode_t& node, F&& fn)
{
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    fn();
    e = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess) return e;
    e = cudaGraphAddChildGraphNode(&node, graph, dep, dep ? 1 : 0, g);
    cudaGraphDestroy(g);
    return e;
}

// The whole build as one graph: root set-up for every scene, a WHILE loop of split
// levels (two per body, so that the ping-pong buffers are fixed: after every body the
// partition is back in pidx — a level without tasks copies it through), the small
// clusters, a WHILE loop of collapse levels, and the leaf records.  The host waits once,
// at the end.
cudaError_t build_graph(cudaStream_t s, const BuildBufs& b, cudaGraph_t& graph)
{
    cudaError_t e = cudaGraphCreate(&graph, 0);
    if (e != cudaSuccess) return e;
    const int n = b.n, ns = b.nscenes;
    cudaGraphNode_t n_pre = nullptr, n_split = nullptr, n_mid = nullptr, n_collapse = nullptr, n_post = nullptr;
    cudaGraphConditionalHandle h_split{}, h_collapse{};
    e = add_captured(graph, nullptr, s, n_pre, [&]() {
        k_init_root_bounds<<<grid_for(12 * ns, 256), 256, 0, s>>>(b.rb, ns);
        cudaMemsetAsync(b.meta, 0, sizeof(int32_t) * (16 + 3 * (size_t)b.nroots), s);
        cudaMemsetAsync(b.leaf_prim, 0xff, sizeof(int32_t) * n, s);
        k_prim_bounds<<<grid_for(n, 256), 256, 0, s>>>(b.scenes, ns, n, b.plo, b.phi, b.prim_scene);
        k_root_bounds<<<grid_for(n, 256), 256, 0, s>>>(b.plo, b.phi, b.prim_scene, n, b.rb);
        k_make_roots<<<grid_for(ns, 128), 128, 0, s>>>(b.scenes, ns, b.rb, b.bnodes, b.tasks, b.small_list,
                                                        b.counters, b.scene_task, b.nroots);
        k_fill_pos_task<<<grid_for(n, 256), 256, 0, s>>>(b.pos_task, b.pidx, b.prim_scene, b.scene_task, n);
    });
    if (e != cudaSuccess) return e;
    e = add_while(graph, n_pre, s, h_split, n_split, [&](cudaGraphConditionalHandle h) {
        split_level(s, b, b.pidx, b.pos_task, b.tasks, b.pidx2, b.pos_task2, b.tasks2);
        split_level(s, b, b.pidx2, b.pos_task2, b.tasks2, b.pidx, b.pos_task, b.tasks);
        k_split_continue<<<1, 1, 0, s>>>(b.counters, h, 1024);
    });
    if (e != cudaSuccess) return e;
    e = add_captured(graph, &n_split, s, n_mid, [&]() {
        k_small<<<grid_for(n, 64), 64, 0, s>>>(b.plo, b.phi, b.pidx, b.small_list, b.counters + 2, b.bnodes,
                                               b.counters);
        cudaMemsetAsync(b.parent, 0xff, sizeof(int32_t) * b.max_nodes, s);
        cudaMemsetAsync(b.arrive, 0, sizeof(int32_t) * b.max_nodes, s);
        k_parents<<<grid_for(b.max_nodes, 256), 256, 0, s>>>(b.bnodes, b.counters, b.parent);
        k_collapse_dp<<<grid_for(b.max_nodes, 128), 128, 0, s>>>(b.bnodes, b.counters, b.parent, b.arrive, b.dp);
        k_collapse_init<<<grid_for(ns, 128), 128, 0, s>>>(b.scenes, ns, b.nroots, b.front, b.ccnt);
    });
    if (e != cudaSuccess) return e;
    e = add_while(graph, n_mid, s, h_collapse, n_collapse, [&](cudaGraphConditionalHandle h) {
        collapse_level(s, b, b.front, b.front2);
        collapse_level(s, b, b.front2, b.front);
        k_collapse_continue<<<1, 1, 0, s>>>(b.ccnt, h, 64);
    });
    if (e != cudaSuccess) return e;
    return add_captured(graph, &n_collapse, s, n_post, [&]() {
        k_fill_leaf<<<grid_for(n, 256), 256, 0, s>>>(b.leaf_prim, n, b.scenes, b.prim_scene, n, b.leaf);
    });
}

// Releases the build's temporaries (stream-ordered).
void free_temporaries(cudaStream_t s, BuildBufs& b)
{
    void* bufs[] = {b.plo,    b.phi,       b.pidx,       b.pidx2,      b.pos_task, b.pos_task2, b.flags,
                    b.scan,   b.tile_sums, b.small_list, b.meta,       b.rb,       b.bnodes,    b.tasks,
                    b.tasks2, b.splits,    b.bins,       b.front,      b.front2,   b.leaf_prim, b.prim_scene,
                    b.scene_task, b.scenes, b.parent,   b.arrive,     b.dp};
    for (void* p : bufs)
        if (p) cudaFreeAsync(p, s);
}

}  // namespace

// A build in flight: its buffers, graph and the events around it.
struct BvhJob {
    BuildBufs b{};
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    const int32_t* h_meta = nullptr;   // pinned: counters and per-root stats after the build
    std::vector<int32_t> scene_root, scene_count;
};

namespace {

// Drops a job: waits for its stream (on failure paths only), then frees everything,
// including the result arrays.
void drop_job(BvhJob* job, BvhBatch& out)
{
    cudaGetLastError();
    cudaStreamSynchronize(job->stream);
    if (job->exec) cudaGraphExecDestroy(job->exec);
    if (job->graph) cudaGraphDestroy(job->graph);
    free_temporaries(job->stream, job->b);
    if (out.nodes) cudaFreeAsync(out.nodes, job->stream);
    if (out.leaf) cudaFreeAsync(out.leaf, job->stream);
    cudaStreamSynchronize(job->stream);
    out = BvhBatch{};
    if (job->ev0) cudaEventDestroy(job->ev0);
    if (job->ev1) cudaEventDestroy(job->ev1);
    delete job;
}

size_t align64(size_t x) { return (x + 63) & ~size_t(63); }

}  // namespace

size_t bvh_batch_pinned_bytes(int nscenes)
{
    return align64(sizeof(BatchScene) * (size_t)nscenes) + sizeof(int32_t) * (16 + 3 * (size_t)nscenes);
}

int bvh_build_batch_begin(cudaStream_t stream, cudaStream_t capture, const PrimSource* srcs, int nscenes,
                          void* h_pinned, int sms, BvhJob*& job_out, BvhBatch& out, std::string& err)
{
    job_out = nullptr;
    out = BvhBatch{};
    out.root.assign((size_t)nscenes, -1);
    // layout of the batch: scenes' primitives back to back, roots numbered in scene order
    std::vector<BatchScene> table((size_t)nscenes);
    int64_t total = 0;
    int nroots = 0;
    for (int i = 0; i < nscenes; ++i) {
        const PrimSource& p = srcs[i];
        const int64_t cnt = (int64_t)p.num_tris + 2 * (int64_t)p.num_rects + p.num_spheres;
        BatchScene& t = table[(size_t)i];
        t.src = p;
        t.begin = (int32_t)total;
        t.count = (int32_t)cnt;
        t.root = cnt > 0 ? nroots++ : -1;
        t.pad = 0;
        out.root[(size_t)i] = t.root;
        total += cnt;
    }
    if (total > (int64_t)0x3fffffff) {
        err = "bvh build: too many primitives in one batch";
        return -1;
    }
    if (nroots == 0) return 0;
    const int n = (int)total;
    BvhJob* job = new (std::nothrow) BvhJob();
    if (!job) {
        err = "bvh build: host allocation failed";
        return -1;
    }
    job->stream = stream;
    job->scene_root = out.root;
    job->scene_count.resize((size_t)nscenes);
    for (int i = 0; i < nscenes; ++i) job->scene_count[(size_t)i] = table[(size_t)i].count;
    char* hp = static_cast<char*>(h_pinned);
    std::memcpy(hp, table.data(), sizeof(BatchScene) * (size_t)nscenes);
    job->h_meta = reinterpret_cast<const int32_t*>(hp + align64(sizeof(BatchScene) * (size_t)nscenes));
    BuildBufs& b = job->b;
    b.n = n;
    b.nscenes = nscenes;
    b.nroots = nroots;
    b.max_tasks = n / (kSmall + 1) + 2 + nroots;
    b.ntiles = (n + kScanTile - 1) / kScanTile;
    b.sms = sms;
    const size_t max_nodes = 2 * (size_t)n + 2;
    const size_t max_wide = (size_t)n + nroots + 1;
    FM_BUILD_CHECK(cudaEventCreate(&job->ev0));
    FM_BUILD_CHECK(cudaEventCreate(&job->ev1));
    FM_BUILD_CHECK(cudaEventRecord(job->ev0, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.scenes, sizeof(BatchScene) * (size_t)nscenes, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.plo, sizeof(float4) * n, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.phi, sizeof(float4) * n, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.pidx, sizeof(int32_t) * n, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.pidx2, sizeof(int32_t) * n, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.pos_task, sizeof(int32_t) * n, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.pos_task2, sizeof(int32_t) * n, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.flags, sizeof(int32_t) * n, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.scan, sizeof(int32_t) * (n + 1), stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.tile_sums, sizeof(int32_t) * (b.ntiles + 1), stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.small_list, sizeof(int32_t) * 3 * max_wide, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.prim_scene, sizeof(int32_t) * n, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.scene_task, sizeof(int32_t) * nscenes, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.meta, sizeof(int32_t) * (16 + 3 * (size_t)nroots), stream));
    b.counters = b.meta;
    b.ccnt = b.meta + 8;
    b.stats = b.meta + 16;
    FM_BUILD_CHECK(cudaMallocAsync(&b.rb, sizeof(uint32_t) * 12 * (size_t)nscenes, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.bnodes, sizeof(BNode) * max_nodes, stream));
    b.max_nodes = (int64_t)max_nodes;
    FM_BUILD_CHECK(cudaMallocAsync(&b.parent, sizeof(int32_t) * max_nodes, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.arrive, sizeof(int32_t) * max_nodes, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.dp, sizeof(DpNode) * max_nodes, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.tasks, sizeof(Task) * b.max_tasks, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.tasks2, sizeof(Task) * b.max_tasks, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.splits, sizeof(Split) * b.max_tasks, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.bins, sizeof(Bins) * b.max_tasks, stream));
    // wide nodes <= binary internal nodes + one root per scene; leaf slots == n
    FM_BUILD_CHECK(cudaMallocAsync(&out.nodes, sizeof(uint4) * 5 * max_wide, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.leaf_prim, sizeof(int32_t) * n, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.front, sizeof(int4) * max_wide, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&b.front2, sizeof(int4) * max_wide, stream));
    FM_BUILD_CHECK(cudaMallocAsync(&out.leaf, sizeof(float4) * 3 * (size_t)n, stream));
    b.wnodes = out.nodes;
    b.leaf = out.leaf;
    FM_BUILD_CHECK(cudaMemcpyAsync(b.scenes, hp, sizeof(BatchScene) * (size_t)nscenes, cudaMemcpyHostToDevice, stream));
    FM_BUILD_CHECK(build_graph(capture, b, job->graph));
    FM_BUILD_CHECK(cudaGraphInstantiate(&job->exec, job->graph, 0));
    FM_BUILD_CHECK(cudaGraphLaunch(job->exec, stream));
    FM_BUILD_CHECK(cudaMemcpyAsync(const_cast<int32_t*>(job->h_meta), b.meta, sizeof(int32_t) * (16 + 3 * (size_t)nroots),
                                   cudaMemcpyDeviceToHost, stream));
    FM_BUILD_CHECK(cudaEventRecord(job->ev1, stream));
    job_out = job;
    return 0;
fail:
    drop_job(job, out);
    return -1;
}

int bvh_build_batch_end(BvhJob* job, BvhBatch& out, std::string& err)
{
    if (!job) return 0;
    const int32_t* h_cnt = job->h_meta;
    const int32_t* stats = job->h_meta + 16;
    const int nscenes = (int)job->scene_root.size();
    FM_BUILD_CHECK(cudaEventSynchronize(job->ev1));
    if (h_cnt[5] & 1) {
        err = "bvh build: task list overflow";
        goto fail;
    }
    if (h_cnt[5] & 2) {
        err = "bvh build: too many split levels";
        goto fail;
    }
    if (h_cnt[8 + 6] & 1) {
        err = "bvh build: too many collapse levels";
        goto fail;
    }
    if (h_cnt[8 + 1] != job->b.n) {
        err = "bvh build: leaf count mismatch";
        goto fail;
    }
    out.num_nodes.assign((size_t)nscenes, 0);
    out.num_leaf.assign((size_t)nscenes, 0);
    out.depth.assign((size_t)nscenes, 0);
    for (int i = 0; i < nscenes; ++i) {
        const int r = job->scene_root[(size_t)i];
        if (r < 0) continue;
        out.num_nodes[(size_t)i] = stats[3 * r];
        out.num_leaf[(size_t)i] = stats[3 * r + 1];
        out.depth[(size_t)i] = stats[3 * r + 2];
        if (out.num_leaf[(size_t)i] != job->scene_count[(size_t)i]) {
            err = "bvh build: leaf count mismatch";
            goto fail;
        }
        if (out.depth[(size_t)i] >= kTraversalStack) {
            err = "bvh build: tree deeper than the traversal stack";
            goto fail;
        }
    }
    {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, job->ev0, job->ev1);
        out.build_ms = ms;
    }
    cudaGraphExecDestroy(job->exec);
    cudaGraphDestroy(job->graph);
    free_temporaries(job->stream, job->b);
    cudaEventDestroy(job->ev0);
    cudaEventDestroy(job->ev1);
    delete job;
    return 0;
fail:
    drop_job(job, out);
    return -1;
}

void bvh_build_abort(BvhJob* job, BvhBatch& out)
{
    if (job) drop_job(job, out);
}

}  // namespace fm
