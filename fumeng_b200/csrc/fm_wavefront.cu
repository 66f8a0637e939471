// Wavefront path tracer: a pool of path slots advanced one bounce per iteration by
// three kernels (prep, trace, shade), replayed from a CUDA graph until every work item
// is done.  Works on any number of views (one view = one camera over one scene), which
// is how a batch of scenes renders in one launch.
//
// Queues (rebuilt every iteration by the shade kernel, consumed by the trace kernel):
//   cont    slot ids whose continuation ray is in the slot's ray registers
//   mis     MIS-BSDF rays (origin|slot, direction|pdf, weight|view)
//   shadow  NEE shadow rays (origin|t_max, direction|slot, contribution|view)
// Entries are appended with warp-aggregated atomics (one atomic per warp and queue:
// ballot, popcount, prefix), so each queue is dense and its float4 records are read
// coalesced.  The trace kernel resolves MIS and shadow rays itself and adds their
// contribution to the slot's accumulator; the next shade folds it into the path.
//
// Work items are (view, pixel, chunk of `chunk` consecutive samples).  A slot runs its
// item's samples one after another with Kahan-compensated sums and writes the item's
// partial sums once; a final kernel sums the chunks of each pixel in chunk order.  When
// a path ends, its slot immediately starts the next sample (path regeneration).
#include <cmath>
#include <vector>

#include "fm_path.cuh"
#include "fm_render.h"

namespace fm {

namespace {

constexpr int kNeedItem = -2;
constexpr int kDone = -1;
constexpr int kHasCont = 1;

struct WfState {
    int64_t pool;
    const WfView* views;
    int32_t nviews;
    int64_t total_items;
    unsigned long long* next_item;
    // per slot
    int64_t* item;        // global work item, or kNeedItem / kDone
    int32_t* k;           // sample within the item
    int32_t* view;
    int32_t* flags;       // bit 0: continuation ray pending; bits 8..: depth
    uint64_t* rng;
    float4* beta;
    float4* col;
    float4* ro;
    float4* rd;
    float4* hit;
    float4* acc;          // MIS + shadow contributions (atomic adds from the trace kernel)
    float4* isum;
    float4* icomp;
    float4* asum;
    float4* nsum;
    // queues
    int32_t* cont_q;
    float4* mis_o;
    float4* mis_d;
    float4* mis_a;
    float4* sh_o;
    float4* sh_d;
    float4* sh_c;
    int64_t cap_cont, cap_mis, cap_sh;
    // counters: [0..2] queue sizes being written, [3..5] sizes being traced, [6] active slots
    unsigned* qc;
    Counters* cnt;
    uint32_t* status;
};

FM_D unsigned lanemask_lt() { return (1u << (threadIdx.x & 31)) - 1u; }

// Warp-aggregated append: returns this lane's index (or -1 when !want).
FM_D int64_t wagg_append(unsigned* counter, bool want)
{
    const unsigned mask = __activemask();
    const unsigned b = __ballot_sync(mask, want);
    if (!want) return -1;
    const int leader = __ffs(b) - 1;
    unsigned base = 0;
    if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(counter, (unsigned)__popc(b));
    base = __shfl_sync(b, base, leader);
    return (int64_t)base + __popc(b & lanemask_lt());
}

FM_D void acc_add(float4* a, f3 c)
{
    atomicAdd(&a->x, c.x);
    atomicAdd(&a->y, c.y);
    atomicAdd(&a->z, c.z);
}

FM_D int find_view(const WfState& st, int64_t item)
{
    int lo = 0, hi = st.nviews - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (st.views[mid].item_base <= item)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__global__ void k_wf_prep(WfState st)
{
    st.qc[3] = st.qc[0];
    st.qc[4] = st.qc[1];
    st.qc[5] = st.qc[2];
    st.qc[0] = 0;
    st.qc[1] = 0;
    st.qc[2] = 0;
    st.qc[6] = 0;
}

__global__ void __launch_bounds__(256) k_wf_trace(WfState st)
{
    const int64_t nc = st.qc[3], nm = st.qc[4], ns = st.qc[5];
    const int64_t total = nc + nm + ns;
    unsigned long long n_closest = 0, n_shadow = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < nc) {
            const int slot = st.cont_q[i];
            const DevScene& S = *st.views[st.view[slot]].scene;
            const float4 o = st.ro[slot], d = st.rd[slot];
            Hit h;
            trace_ray<false>(S, f3{o.x, o.y, o.z}, f3{d.x, d.y, d.z}, 0.0f, kRealMax, h, st.status);
            st.hit[slot] = make_float4(h.t, __int_as_float(h.prim), h.b1, h.b2);
            ++n_closest;
        } else if (i < nc + nm) {
            const int64_t q = i - nc;
            const float4 o4 = st.mis_o[q], d4 = st.mis_d[q], a4 = st.mis_a[q];
            const int slot = __float_as_int(o4.w);
            const DevScene& S = *st.views[__float_as_int(a4.w)].scene;
            const f3 o = f3{o4.x, o4.y, o4.z}, d = f3{d4.x, d4.y, d4.z}, A = f3{a4.x, a4.y, a4.z};
            const float pdf = d4.w;   // < 0: delta BSDF sample (no MIS weight)
            Hit h;
            ++n_closest;
            f3 c = mk(0.0f);
            if (!trace_ray<false>(S, o, d, 0.0f, kRealMax, h, st.status)) {
                if (S.env_light >= 0) {
                    c = A * env_radiance(S, d);
                    if (pdf >= 0.0f) c *= power_heuristic(pdf, env_pdf(S, d));
                }
            } else {
                const int obj = __ldg(S.prim_obj + h.prim);
                const int li = __ldg(S.obj_light + obj);
                if (li >= 0) {
                    const HitInfo lh = make_hit(S, o, d, h);
                    const f3 l2s = normalize(o - lh.pos);
                    const DevLight& L = S.lights[li];
                    const f3 rad = dot(lh.ng, l2s) > 0 ? ld3(L.radiance) : mk(0.0f);
                    if (length(rad) >= kEpsPdf) {
                        c = A * rad;
                        if (pdf >= 0.0f) c *= power_heuristic(pdf, area_light_pdf(S, L, o, lh.pos, lh.ng, l2s));
                    }
                }
            }
            if (c.x != 0.0f || c.y != 0.0f || c.z != 0.0f) acc_add(&st.acc[slot], c);
        } else {
            const int64_t q = i - nc - nm;
            const float4 o4 = st.sh_o[q], d4 = st.sh_d[q], c4 = st.sh_c[q];
            const int slot = __float_as_int(d4.w);
            const DevScene& S = *st.views[__float_as_int(c4.w)].scene;
            Hit h;
            ++n_shadow;
            if (!trace_ray<true>(S, f3{o4.x, o4.y, o4.z}, f3{d4.x, d4.y, d4.z}, kEps, o4.w, h, st.status))
                acc_add(&st.acc[slot], f3{c4.x, c4.y, c4.z});
        }
    }
    // per-warp counter aggregation
    for (int off = 16; off > 0; off >>= 1) {
        n_closest += __shfl_xor_sync(0xffffffffu, n_closest, off);
        n_shadow += __shfl_xor_sync(0xffffffffu, n_shadow, off);
    }
    if ((threadIdx.x & 31) == 0 && (n_closest | n_shadow)) {
        atomicAdd(&st.cnt->closest, n_closest);
        atomicAdd(&st.cnt->shadow, n_shadow);
    }
}

FM_D void kahan_add4(float4& sum, float4& c, f3 x)
{
    const float yx = x.x - c.x, yy = x.y - c.y, yz = x.z - c.z;
    const float tx = sum.x + yx, ty = sum.y + yy, tz = sum.z + yz;
    c.x = (tx - sum.x) - yx;
    c.y = (ty - sum.y) - yy;
    c.z = (tz - sum.z) - yz;
    sum.x = tx;
    sum.y = ty;
    sum.z = tz;
}

FM_D int item_samples(const WfView& V, int chunk_index)
{
    const int first = chunk_index * V.chunk;
    return min(V.chunk, V.cfg.spp - first);
}

// Start sample `k` of the slot's item: camera ray into the slot registers, enqueue it.
FM_D void start_sample(const WfState& st, int slot, const WfView& V, int64_t item_local, int k)
{
    const int npix = V.cfg.width * V.cfg.height;
    const int c = (int)(item_local / npix);
    const int p = (int)(item_local % npix);
    const int row = p / V.cfg.width, i = p % V.cfg.width;
    const int j = V.cfg.height - 1 - row;
    const int sample = c * V.chunk + k;
    Rng rng = rng_for(V.cfg.seed, (uint64_t)p, (uint64_t)(V.cfg.sample_offset + sample));
    const float fx = rng_1d(rng), fy = rng_1d(rng);
    const float lx = rng_1d(rng), ly = rng_1d(rng);
    const float px = ((float)i + fx) / (float)V.cfg.width;
    const float py = ((float)j + fy) / (float)V.cfg.height;
    f3 o, d;
    camera_ray(V.cam, px, py, lx, ly, o, d);
    st.ro[slot] = make_float4(o.x, o.y, o.z, 0.0f);
    st.rd[slot] = make_float4(d.x, d.y, d.z, 0.0f);
    st.rng[slot] = rng.state;
    st.beta[slot] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    st.col[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    st.flags[slot] = kHasCont | (1 << 8);
}

__global__ void __launch_bounds__(256) k_wf_shade(WfState st)
{
    unsigned long long n_paths = 0, n_bounces = 0, n_nans = 0;
    unsigned n_active = 0;
    for (int64_t s0 = blockIdx.x * (int64_t)blockDim.x; s0 < st.pool; s0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s64 = s0 + threadIdx.x;
        const int slot = (int)s64;
        const bool in_range = s64 < st.pool;
        int64_t item = in_range ? st.item[slot] : (int64_t)kDone;
        bool need_new = item == kNeedItem;
        bool enqueue_cont = false;
        if (item >= 0) {
            const int vid = st.view[slot];
            const WfView& V = st.views[vid];
            const DevScene& S = *V.scene;
            const float4 a4 = st.acc[slot];
            const float4 c4 = st.col[slot];
            f3 col = f3{c4.x + a4.x, c4.y + a4.y, c4.z + a4.z};
            st.acc[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            int flags = st.flags[slot];
            bool pending = false;
            if (flags & kHasCont) {
                const int depth = flags >> 8;
                flags = 0;
                const float4 h4 = st.hit[slot];
                const float4 o4 = st.ro[slot], d4 = st.rd[slot];
                const f3 o = f3{o4.x, o4.y, o4.z}, d = f3{d4.x, d4.y, d4.z};
                const float4 b4 = st.beta[slot];
                f3 beta = f3{b4.x, b4.y, b4.z};
                Hit hit;
                hit.t = h4.x;
                hit.prim = __float_as_int(h4.y);
                hit.b1 = h4.z;
                hit.b2 = h4.w;
                if (hit.prim < 0) {
                    if (depth == 1 && S.env_light >= 0) col = env_radiance(S, d);
                } else {
                    const HitInfo h = make_hit(S, o, d, hit);
                    const int li = depth == 1 ? __ldg(S.obj_light + h.obj) : -1;
                    if (li >= 0) {
                        const f3 rad = dot(h.ng, h.wo) > 0 ? ld3(S.lights[li].radiance) : mk(0.0f);
                        col += beta * rad;
                    } else {
                        ++n_bounces;
                        Rng rng;
                        rng.state = st.rng[slot];
                        const Bsdf b = make_bsdf(S, h);
                        if (depth == 1) {
                            const f3 al = bsdf_albedo(b);
                            float4 as = st.asum[slot], ns = st.nsum[slot];
                            as.x += al.x; as.y += al.y; as.z += al.z;
                            ns.x += h.ng.x; ns.y += h.ng.y; ns.z += h.ng.z;
                            st.asum[slot] = as;
                            st.nsum[slot] = ns;
                        }
                        const float inv_dl = 1.0f / (float)V.cfg.direct_loop;
                        for (int kk = 0; kk < V.cfg.direct_loop; ++kk) {
                            for (int l = 0; l < S.num_lights; ++l) {
                                const DevLight& L = S.lights[l];
                                LightSample ls;
                                bool ok = light_sample(S, L, h.pos, rng_3d(rng), ls);
                                ok = ok && ls.pdf >= kEpsPdf && length(ls.radiance) >= kEpsPdf;
                                f3 f = mk(0.0f);
                                float pb = 0.0f;
                                if (ok) {
                                    f = bsdf_f(b, h.wo, ls.wi);
                                    ok = length(f) >= kEpsPdf;
                                }
                                if (ok) {
                                    pb = bsdf_pdf(b, h.wo, ls.wi);
                                    ok = pb >= kEpsPdf;
                                }
                                const int64_t q = wagg_append(&st.qc[2], ok);
                                if (ok) {
                                    f3 c = beta * (f * ls.radiance * absdot(ls.wi, h.ng)) / ls.pdf;
                                    if (!ls.delta) c *= power_heuristic(ls.pdf, pb);
                                    c *= inv_dl;
                                    if (q < st.cap_sh) {
                                        st.sh_o[q] = make_float4(h.pos.x, h.pos.y, h.pos.z, ls.dist - kEps);
                                        st.sh_d[q] = make_float4(ls.wi.x, ls.wi.y, ls.wi.z, __int_as_float(slot));
                                        st.sh_c[q] = make_float4(c.x, c.y, c.z, __int_as_float(vid));
                                        pending = true;
                                    } else {
                                        atomicOr(st.status, 2u);
                                    }
                                }
                            }
                            const BsdfSample ms = bsdf_sample(b, h.wo, rng_3d(rng));
                            const bool ok = length(ms.f) >= kEpsPdf && ms.pdf >= kEpsPdf;
                            const int64_t q = wagg_append(&st.qc[1], ok);
                            if (ok) {
                                const f3 wi = normalize(ms.wi);
                                const f3 ro = spawn_origin(h, wi);
                                const f3 A = beta * ms.f * absdot(h.ng, wi) / ms.pdf * inv_dl;
                                if (q < st.cap_mis) {
                                    st.mis_o[q] = make_float4(ro.x, ro.y, ro.z, __int_as_float(slot));
                                    st.mis_d[q] = make_float4(wi.x, wi.y, wi.z, ms.delta ? -1.0f : ms.pdf);
                                    st.mis_a[q] = make_float4(A.x, A.y, A.z, __int_as_float(vid));
                                    pending = true;
                                } else {
                                    atomicOr(st.status, 2u);
                                }
                            }
                        }
                        const BsdfSample sc = bsdf_sample(b, h.wo, rng_3d(rng));
                        if (length(sc.f) >= kEpsPdf && sc.pdf >= kEpsPdf) {
                            beta *= sc.f * absdot(h.ng, sc.wi) / sc.pdf;
                            if (depth < V.cfg.depth) {
                                bool go = true;
                                if (V.cfg.rr_enabled) {
                                    if (rng_1d(rng) > V.cfg.rr_coef)
                                        go = false;
                                    else
                                        beta /= V.cfg.rr_coef;
                                }
                                if (go) {
                                    const f3 no = spawn_origin(h, sc.wi);
                                    st.ro[slot] = make_float4(no.x, no.y, no.z, 0.0f);
                                    st.rd[slot] = make_float4(sc.wi.x, sc.wi.y, sc.wi.z, 0.0f);
                                    st.beta[slot] = make_float4(beta.x, beta.y, beta.z, 0.0f);
                                    flags = kHasCont | ((depth + 1) << 8);
                                    enqueue_cont = true;
                                }
                            }
                        }
                        st.rng[slot] = rng.state;
                    }
                }
            }
            if (!enqueue_cont && !pending) {
                // sample finished
                ++n_paths;
                if (!isfinite(col.x) || !isfinite(col.y) || !isfinite(col.z)) ++n_nans;
                float4 sum = st.isum[slot], cmp = st.icomp[slot];
                kahan_add4(sum, cmp, col);
                const int kdone = st.k[slot] + 1;
                const int64_t local = item - V.item_base;
                const int npix = V.cfg.width * V.cfg.height;
                const int chunk_index = (int)(local / npix);
                if (kdone >= item_samples(V, chunk_index)) {
                    float4* P = V.partial + 3 * (size_t)local;
                    P[0] = sum;
                    P[1] = st.asum[slot];
                    P[2] = st.nsum[slot];
                    need_new = true;
                } else {
                    st.isum[slot] = sum;
                    st.icomp[slot] = cmp;
                    st.k[slot] = kdone;
                    start_sample(st, slot, V, local, kdone);
                    enqueue_cont = true;
                }
            } else {
                st.col[slot] = make_float4(col.x, col.y, col.z, 0.0f);
                st.flags[slot] = flags;
            }
        }
        // new work items for slots that finished theirs (one atomic per warp)
        {
            const unsigned mask = __activemask();
            const unsigned b = __ballot_sync(mask, need_new);
            if (need_new) {
                const int leader = __ffs(b) - 1;
                unsigned long long base = 0;
                if ((int)(threadIdx.x & 31) == leader) base = atomicAdd(st.next_item, (unsigned long long)__popc(b));
                base = __shfl_sync(b, base, leader);
                const int64_t it = (int64_t)(base + __popc(b & lanemask_lt()));
                if (it >= st.total_items) {
                    st.item[slot] = kDone;
                } else {
                    const int vid = find_view(st, it);
                    const WfView& V = st.views[vid];
                    st.item[slot] = it;
                    st.view[slot] = vid;
                    st.k[slot] = 0;
                    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    st.isum[slot] = z;
                    st.icomp[slot] = z;
                    st.asum[slot] = z;
                    st.nsum[slot] = z;
                    st.acc[slot] = z;
                    start_sample(st, slot, V, it - V.item_base, 0);
                    enqueue_cont = true;
                }
            }
        }
        const int64_t q = wagg_append(&st.qc[0], enqueue_cont);
        if (enqueue_cont) {
            if (q < st.cap_cont)
                st.cont_q[q] = slot;
            else
                atomicOr(st.status, 2u);
            ++n_active;
        }
        if (in_range && !enqueue_cont && st.item[slot] >= 0) ++n_active;
    }
    for (int off = 16; off > 0; off >>= 1) {
        n_paths += __shfl_xor_sync(0xffffffffu, n_paths, off);
        n_bounces += __shfl_xor_sync(0xffffffffu, n_bounces, off);
        n_nans += __shfl_xor_sync(0xffffffffu, n_nans, off);
        n_active += __shfl_xor_sync(0xffffffffu, n_active, off);
    }
    if ((threadIdx.x & 31) == 0) {
        if (n_paths | n_bounces | n_nans) {
            atomicAdd(&st.cnt->paths, n_paths);
            atomicAdd(&st.cnt->bounces, n_bounces);
            atomicAdd(&st.cnt->nans, n_nans);
        }
        if (n_active) atomicAdd(&st.qc[6], n_active);
    }
}

__global__ void k_wf_init(WfState st)
{
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < st.pool; s += (int64_t)gridDim.x * blockDim.x) {
        st.item[s] = kNeedItem;
        st.flags[s] = 0;
        st.acc[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

// Per pixel: sum the chunks in order (Kahan) and divide by spp.
__global__ void k_wf_reduce(WfView V)
{
    const int npix = V.cfg.width * V.cfg.height;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        float4 s = make_float4(0.0f, 0.0f, 0.0f, 0.0f), c = s;
        f3 a = mk(0.0f), n = mk(0.0f);
        for (int ch = 0; ch < V.nchunks; ++ch) {
            const float4* P = V.partial + 3 * ((size_t)ch * npix + p);
            const float4 x = P[0], y = P[1], z = P[2];
            kahan_add4(s, c, f3{x.x, x.y, x.z});
            a += f3{y.x, y.y, y.z};
            n += f3{z.x, z.y, z.z};
        }
        const float inv = 1.0f / (float)V.cfg.spp;
        st3(V.rgb + 3 * (size_t)p, f3{s.x, s.y, s.z} * inv);
        if (V.alb) st3(V.alb + 3 * (size_t)p, a * inv);
        if (V.nrm) st3(V.nrm + 3 * (size_t)p, n * inv);
    }
}

}  // namespace

fm_status wavefront_views(fm_ctx* ctx, const std::vector<WfView>& views_in, const WfTuning& tune, Counters* cnt,
                          WfTimes* times)
{
    cudaStream_t s = ctx->stream;
    std::vector<WfView> views = views_in;
    // samples per work item: aim for ~4 items per path slot over the whole job
    double total_samples = 0.0;
    int max_lights = 1, max_dl = 1;
    for (const auto& v : views) {
        total_samples += (double)v.cfg.width * v.cfg.height * v.cfg.spp;
        max_dl = std::max(max_dl, v.cfg.direct_loop);
    }
    for (const auto& v : views) {
        DevScene hs;
        FM_CUDA_TRY(ctx, cudaMemcpy(&hs, v.scene, sizeof(DevScene), cudaMemcpyDeviceToHost), "wavefront scene");
        max_lights = std::max(max_lights, hs.num_lights);
    }
    const int64_t pool = std::max<int64_t>(1024, std::min<int64_t>(tune.pool, (int64_t)total_samples));
    const double per_item = total_samples / (4.0 * (double)pool);
    int64_t item_base = 0;
    std::vector<void*> allocs;
    auto alloc = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMallocAsync(&p, bytes, s) != cudaSuccess) return nullptr;
        allocs.push_back(p);
        return p;
    };
    auto free_all = [&]() {
        for (void* p : allocs) cudaFreeAsync(p, s);
        allocs.clear();
    };
    for (auto& v : views) {
        int chunk = (int)std::floor(per_item);
        chunk = std::max(1, std::min(chunk, v.cfg.spp));
        v.chunk = chunk;
        v.nchunks = (v.cfg.spp + chunk - 1) / chunk;
        v.item_base = item_base;
        const int64_t npix = (int64_t)v.cfg.width * v.cfg.height;
        item_base += npix * v.nchunks;
        v.partial = static_cast<float4*>(alloc(sizeof(float4) * 3 * (size_t)(npix * v.nchunks)));
        if (!v.partial) {
            free_all();
            return set_error(ctx, FM_ERR_OOM, "wavefront: partial buffer allocation failed");
        }
    }
    WfState st{};
    st.pool = pool;
    st.nviews = (int32_t)views.size();
    st.total_items = item_base;
    st.cap_cont = pool;
    st.cap_mis = pool * max_dl;
    st.cap_sh = pool * max_dl * (int64_t)max_lights;
    bool ok = true;
    auto A = [&](auto*& p, size_t count) {
        p = static_cast<std::remove_reference_t<decltype(p)>>(alloc(sizeof(*p) * count));
        ok = ok && p != nullptr;
    };
    WfView* d_views = nullptr;
    A(d_views, views.size());
    A(st.next_item, 1);
    A(st.item, pool);
    A(st.k, pool);
    A(st.view, pool);
    A(st.flags, pool);
    A(st.rng, pool);
    A(st.beta, pool);
    A(st.col, pool);
    A(st.ro, pool);
    A(st.rd, pool);
    A(st.hit, pool);
    A(st.acc, pool);
    A(st.isum, pool);
    A(st.icomp, pool);
    A(st.asum, pool);
    A(st.nsum, pool);
    A(st.cont_q, st.cap_cont);
    A(st.mis_o, st.cap_mis);
    A(st.mis_d, st.cap_mis);
    A(st.mis_a, st.cap_mis);
    A(st.sh_o, st.cap_sh);
    A(st.sh_d, st.cap_sh);
    A(st.sh_c, st.cap_sh);
    A(st.qc, 8);
    if (!ok) {
        free_all();
        return set_error(ctx, FM_ERR_OOM, "wavefront: state allocation failed");
    }
    st.views = d_views;
    st.cnt = cnt;
    st.status = ctx->d_status;
    FM_CUDA_TRY(ctx, cudaMemcpyAsync(d_views, views.data(), sizeof(WfView) * views.size(), cudaMemcpyHostToDevice, s),
                "wavefront views");
    FM_CUDA_TRY(ctx, cudaMemsetAsync(st.next_item, 0, sizeof(unsigned long long), s), "wavefront");
    FM_CUDA_TRY(ctx, cudaMemsetAsync(st.qc, 0, sizeof(unsigned) * 8, s), "wavefront");
    const int sms = ctx->num_sms;
    k_wf_init<<<sms * 8, 256, 0, s>>>(st);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    // one graph = `iters_per_graph` iterations of prep -> trace -> shade
    const int trace_grid = sms * 16;
    const int shade_grid = (int)std::min<int64_t>((pool + tune.shade_block - 1) / tune.shade_block, (int64_t)sms * 32);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    fm_status result = FM_OK;
    // optional per-kernel timing: event-record nodes around every trace and shade launch
    std::vector<cudaEvent_t> pev;
    if (tune.profile) {
        pev.resize(3 * (size_t)tune.iters_per_graph);
        for (auto& ev : pev) cudaEventCreate(&ev);
    }
    double trace_ms = 0.0, shade_ms = 0.0;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        for (int it = 0; it < tune.iters_per_graph; ++it) {
            k_wf_prep<<<1, 1, 0, s>>>(st);
            if (tune.profile) cudaEventRecordWithFlags(pev[3 * it], s, cudaEventRecordExternal);
            k_wf_trace<<<trace_grid, tune.trace_block, 0, s>>>(st);
            if (tune.profile) cudaEventRecordWithFlags(pev[3 * it + 1], s, cudaEventRecordExternal);
            k_wf_shade<<<shade_grid, tune.shade_block, 0, s>>>(st);
            if (tune.profile) cudaEventRecordWithFlags(pev[3 * it + 2], s, cudaEventRecordExternal);
        }
        e = cudaStreamEndCapture(s, &graph);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        free_all();
        return cuda_error(ctx, e, "wavefront graph");
    }
    unsigned* h_qc = nullptr;
    cudaMallocHost(&h_qc, sizeof(unsigned) * 8);
    // Bound on graph launches: every sample takes at most depth + 1 iterations and a slot
    // runs its samples one after another.
    int max_depth = 1, max_chunk = 1;
    for (const auto& v : views) {
        max_depth = std::max(max_depth, v.cfg.depth);
        max_chunk = std::max(max_chunk, v.chunk);
    }
    const double iter_bound = (total_samples / (double)pool + 4.0 * max_chunk + 8.0) * (max_depth + 2) * 4.0 + 1000.0;
    const int64_t max_launches = (int64_t)(iter_bound / tune.iters_per_graph) + 16;
    int64_t guard = 0, graph_launches = 0;
    for (;;) {
        e = cudaGraphLaunch(exec, s);
        if (e != cudaSuccess) break;
        ++graph_launches;
        e = cudaMemcpyAsync(h_qc, st.qc, sizeof(unsigned) * 8, cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) break;
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) break;
        for (int it = 0; it < (int)pev.size() / 3; ++it) {
            float a = 0.0f, b = 0.0f;
            cudaEventElapsedTime(&a, pev[3 * it], pev[3 * it + 1]);
            cudaEventElapsedTime(&b, pev[3 * it + 1], pev[3 * it + 2]);
            trace_ms += a;
            shade_ms += b;
        }
        // done when no slot holds work after the last shade
        if (h_qc[6] == 0u) break;
        if (++guard > max_launches) {
            result = set_error(ctx, FM_ERR_TIMEOUT, "wavefront: iteration limit reached");
            break;
        }
    }
    if (e != cudaSuccess) result = cuda_error(ctx, e, "wavefront loop");
    if (result == FM_OK) {
        for (const auto& v : views) {
            const int npix = v.cfg.width * v.cfg.height;
            k_wf_reduce<<<std::min((npix + 255) / 256, sms * 16), 256, 0, s>>>(v);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) result = cuda_error(ctx, e, "wavefront reduce");
    }
    cudaEventRecord(e1, s);
    cudaStreamSynchronize(s);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (times) {
        times->launches = 1 + graph_launches * 3 * tune.iters_per_graph + (int64_t)views.size();
        times->total_ms = ms;
        times->trace_ms = trace_ms;
        times->shade_ms = shade_ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (auto& ev : pev) cudaEventDestroy(ev);
    cudaFreeHost(h_qc);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    free_all();
    cudaStreamSynchronize(s);
    return result;
}

fm_status launch_wavefront(fm_ctx* ctx, const fm_scene* scene, const DevCamera& cam, const RenderCfg& cfg, float* rgb,
                           float* alb, float* nrm, Counters* cnt)
{
    WfView v{};
    v.scene = scene->d_dev;
    v.cam = cam;
    v.cfg = cfg;
    v.rgb = rgb;
    v.alb = alb;
    v.nrm = nrm;
    WfTuning t;
    return wavefront_views(ctx, {v}, t, cnt, nullptr);
}

}  // namespace fm
