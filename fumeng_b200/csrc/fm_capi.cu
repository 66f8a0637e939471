// C-ABI: contexts, scenes and ray queries.
#include <cmath>
#include <cstring>
#include <new>
#include <unordered_map>

#include "fm_bvh.cuh"
#include "fm_internal.h"

using namespace fm;

namespace {

template <typename T>
fm_status upload(fm_ctx* ctx, fm_scene* sc, const T* host, size_t count, const T** dev_out)
{
    *dev_out = nullptr;
    if (!host || count == 0) return FM_OK;
    void* p = nullptr;
    // stream-ordered allocation from the device's memory pool: no device-wide sync
    cudaError_t e = cudaMallocAsync(&p, sizeof(T) * count, ctx->stream);
    if (e != cudaSuccess) return set_error(ctx, FM_ERR_OOM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    sc->allocations.push_back(p);
    e = cudaMemcpyAsync(p, host, sizeof(T) * count, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_error(ctx, e, "upload");
    *dev_out = static_cast<const T*>(p);
    return FM_OK;
}

// 3x3 rotation about a unit axis by `deg` degrees (right-handed), row-major.
void axis_rotation(double deg, int axis, double R[9])
{
    const double a = deg / 180.0 * 3.14159265354;
    const double c = std::cos(a), s = std::sin(a);
    for (int i = 0; i < 9; ++i) R[i] = 0.0;
    if (axis == 0) {
        R[0] = 1; R[4] = c; R[5] = -s; R[7] = s; R[8] = c;
    } else if (axis == 1) {
        R[0] = c; R[2] = s; R[4] = 1; R[6] = -s; R[8] = c;
    } else {
        R[0] = c; R[1] = -s; R[3] = s; R[4] = c; R[8] = 1;
    }
}

void mat3_mul(const double A[9], const double B[9], double C[9])
{
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) C[3 * r + c] = A[3 * r] * B[c] + A[3 * r + 1] * B[3 + c] + A[3 * r + 2] * B[6 + c];
}

// Transform(translation, rotation (deg, applied Z*Y*X), scale) (math/transform.cpp:17-25)
// for the env light: rotation only.
void rotation_zyx(const float rot[3], Xf& l2w, Xf& w2l)
{
    double Rz[9], Ry[9], Rx[9], T[9], R[9];
    axis_rotation(rot[2], 2, Rz);
    axis_rotation(rot[1], 1, Ry);
    axis_rotation(rot[0], 0, Rx);
    mat3_mul(Rz, Ry, T);
    mat3_mul(T, Rx, R);
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            l2w.m[4 * r + c] = (float)R[3 * r + c];
            w2l.m[4 * r + c] = (float)R[3 * c + r];
        }
        l2w.m[4 * r + 3] = 0.0f;
        w2l.m[4 * r + 3] = 0.0f;
    }
}

// Vose's alias method (M. D. Vose, "A linear algorithm for generating random numbers with
// a given distribution", IEEE TSE 1991) over non-negative weights: slot i keeps itself
// with probability prob[i], else its alias.
void vose_alias(const std::vector<double>& w, std::vector<float>& prob, std::vector<int32_t>& alias)
{
    const size_t n = w.size();
    double sum = 0.0;
    for (double x : w) sum += x;
    std::vector<double> p(n);
    std::vector<size_t> small, large;
    for (size_t i = 0; i < n; ++i) {
        p[i] = w[i] * (double)n / sum;
        (p[i] < 1.0 ? small : large).push_back(i);
    }
    prob.assign(n, 1.0f);
    alias.resize(n);
    for (size_t i = 0; i < n; ++i) alias[i] = (int32_t)i;
    while (!small.empty() && !large.empty()) {
        const size_t s = small.back(), l = large.back();
        small.pop_back();
        prob[s] = (float)p[s];
        alias[s] = (int32_t)l;
        p[l] = (p[l] + p[s]) - 1.0;
        if (p[l] < 1.0) {
            large.pop_back();
            small.push_back(l);
        }
    }
}

bool affine_inverse(const float m16[16], Xf& fwd, Xf& inv)
{
    double A[9], t[3];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) A[3 * r + c] = m16[4 * r + c];
        t[r] = m16[4 * r + 3];
    }
    const double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
                       A[2] * (A[3] * A[7] - A[4] * A[6]);
    if (!(std::fabs(det) > 0.0)) return false;
    double I[9];
    I[0] = (A[4] * A[8] - A[5] * A[7]) / det;
    I[1] = (A[2] * A[7] - A[1] * A[8]) / det;
    I[2] = (A[1] * A[5] - A[2] * A[4]) / det;
    I[3] = (A[5] * A[6] - A[3] * A[8]) / det;
    I[4] = (A[0] * A[8] - A[2] * A[6]) / det;
    I[5] = (A[2] * A[3] - A[0] * A[5]) / det;
    I[6] = (A[3] * A[7] - A[4] * A[6]) / det;
    I[7] = (A[1] * A[6] - A[0] * A[7]) / det;
    I[8] = (A[0] * A[4] - A[1] * A[3]) / det;
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            fwd.m[4 * r + c] = (float)A[3 * r + c];
            inv.m[4 * r + c] = (float)I[3 * r + c];
        }
        fwd.m[4 * r + 3] = (float)t[r];
        inv.m[4 * r + 3] = (float)(-(I[3 * r] * t[0] + I[3 * r + 1] * t[1] + I[3 * r + 2] * t[2]));
    }
    return true;
}

void to_texref(const fm_tex_ref& in, TexRef& out)
{
    out.tex = in.texture;
    out.v[0] = in.value[0];
    out.v[1] = in.value[1];
    out.v[2] = in.value[2];
}

bool is_black_h(const float* c)
{
    if (c[0] == 0.0f && c[1] == 0.0f && c[2] == 0.0f) return true;
    return c[0] < 0.0f || c[1] < 0.0f || c[2] < 0.0f;
}

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

fm_status fm_scene_create(fm_ctx* ctx, const fm_scene_desc* d, fm_scene** out)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!d || !out) return set_error(ctx, FM_ERR_INVALID, "scene_create: null argument");
    *out = nullptr;
    // ---- validation -----------------------------------------------------------
    if (d->num_objects < 0 || d->num_triangles < 0 || d->num_rects < 0 || d->num_spheres < 0 ||
        d->num_materials < 0 || d->num_textures < 0 || d->num_lights < 0)
        return set_error(ctx, FM_ERR_INVALID, "scene_create: negative count");
    const int64_t nprim = d->num_triangles + 2 * d->num_rects + d->num_spheres;
    if (nprim > (int64_t)0x3fffffff) return set_error(ctx, FM_ERR_INVALID, "scene_create: too many primitives");
    if (d->num_objects > 0 && !d->obj_material) return set_error(ctx, FM_ERR_INVALID, "scene_create: obj_material is null");
    if (d->num_triangles > 0 && (!d->tri_pos || !d->tri_object))
        return set_error(ctx, FM_ERR_INVALID, "scene_create: triangle arrays are null");
    if (d->num_rects > 0 && (!d->rect_pts || !d->rect_object))
        return set_error(ctx, FM_ERR_INVALID, "scene_create: rectangle arrays are null");
    if (d->num_spheres > 0 && (!d->sphere_radius || !d->sphere_xform || !d->sphere_object))
        return set_error(ctx, FM_ERR_INVALID, "scene_create: sphere arrays are null");
    if (d->num_materials > 0 && !d->materials) return set_error(ctx, FM_ERR_INVALID, "scene_create: materials is null");
    if (d->num_textures > 0 && !d->textures) return set_error(ctx, FM_ERR_INVALID, "scene_create: textures is null");
    if (d->num_lights > 0 && !d->lights) return set_error(ctx, FM_ERR_INVALID, "scene_create: lights is null");
    if (d->tri_vattr && d->vattr_dim < 6) return set_error(ctx, FM_ERR_INVALID, "scene_create: vattr_dim < 6");
    for (int64_t o = 0; o < d->num_objects; ++o)
        if (d->obj_material[o] < 0 || d->obj_material[o] >= d->num_materials)
            return set_error(ctx, FM_ERR_INVALID, "scene_create: object material index out of range");
    // object -> geometry (needed for area lights), and range checks
    std::vector<int32_t> geo_kind(d->num_objects, -1), geo_index(d->num_objects, -1), geo_count(d->num_objects, 0);
    auto note = [&](int32_t obj, int kind, int64_t idx) -> bool {
        if (obj < 0 || obj >= d->num_objects) return false;
        geo_kind[obj] = kind;
        geo_index[obj] = (int32_t)idx;
        ++geo_count[obj];
        return true;
    };
    for (int64_t i = 0; i < d->num_triangles; ++i)
        if (!note(d->tri_object[i], LK_AREA_TRI, i)) return set_error(ctx, FM_ERR_INVALID, "scene_create: triangle object out of range");
    for (int64_t i = 0; i < d->num_rects; ++i)
        if (!note(d->rect_object[i], LK_AREA_RECT, i)) return set_error(ctx, FM_ERR_INVALID, "scene_create: rectangle object out of range");
    for (int64_t i = 0; i < d->num_spheres; ++i)
        if (!note(d->sphere_object[i], LK_AREA_SPHERE, i)) return set_error(ctx, FM_ERR_INVALID, "scene_create: sphere object out of range");
    for (int32_t i = 0; i < d->num_textures; ++i) {
        const fm_texture_desc& t = d->textures[i];
        if (t.width <= 0 || t.height <= 0 || !t.texels) return set_error(ctx, FM_ERR_INVALID, "scene_create: bad texture");
    }
    auto tex_ok = [&](const fm_tex_ref& r) { return r.texture < d->num_textures; };
    for (int32_t i = 0; i < d->num_materials; ++i) {
        const fm_material_desc& m = d->materials[i];
        if (m.type < FM_MAT_LAMBERT || m.type > FM_MAT_DISNEY) return set_error(ctx, FM_ERR_INVALID, "scene_create: bad material type");
        const fm_tex_ref* refs = &m.basecolor;
        for (int k = 0; k < MP_COUNT; ++k)
            if (!tex_ok(refs[k])) return set_error(ctx, FM_ERR_INVALID, "scene_create: material texture out of range");
        if (m.vattr_offset >= 0 && (!d->tri_vattr || m.vattr_offset + 6 > d->vattr_dim))
            return set_error(ctx, FM_ERR_INVALID, "scene_create: material vertex attributes out of range");
    }
    int env_light_desc = -1;
    for (int32_t i = 0; i < d->num_lights; ++i) {
        const fm_light_desc& l = d->lights[i];
        if (l.type == FM_LIGHT_ENV) {
            if (l.texture < 0 || l.texture >= d->num_textures) return set_error(ctx, FM_ERR_INVALID, "scene_create: env texture out of range");
            if (env_light_desc < 0) env_light_desc = i;
        } else if (l.type != FM_LIGHT_DIRECTIONAL) {
            return set_error(ctx, FM_ERR_INVALID, "scene_create: bad light type");
        }
    }
    FM_CUDA_TRY(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");

    fm_scene* sc = new (std::nothrow) fm_scene();
    if (!sc) return set_error(ctx, FM_ERR_OOM, "scene_create: host allocation");
    sc->num_objects = d->num_objects;
    DevScene& S = sc->dev;
    fm_status st = FM_OK;
#define FM_TRY(expr)            \
    do {                        \
        st = (expr);            \
        if (st != FM_OK) goto fail; \
    } while (0)
    {
        S.num_tris = (int32_t)d->num_triangles;
        S.num_rects = (int32_t)d->num_rects;
        S.num_spheres = (int32_t)d->num_spheres;
        S.num_prims = (int32_t)nprim;
        S.num_objects = (int32_t)d->num_objects;
        S.vattr_dim = d->tri_vattr ? d->vattr_dim : 0;
        // primitive -> object
        std::vector<int32_t> prim_obj((size_t)nprim);
        for (int64_t i = 0; i < d->num_triangles; ++i) prim_obj[i] = d->tri_object[i];
        for (int64_t i = 0; i < d->num_rects; ++i)
            prim_obj[d->num_triangles + 2 * i] = prim_obj[d->num_triangles + 2 * i + 1] = d->rect_object[i];
        for (int64_t i = 0; i < d->num_spheres; ++i) prim_obj[d->num_triangles + 2 * d->num_rects + i] = d->sphere_object[i];
        FM_TRY(upload(ctx, sc, prim_obj.data(), prim_obj.size(), &S.prim_obj));
        FM_TRY(upload(ctx, sc, d->tri_pos, 9 * (size_t)d->num_triangles, &S.tri_pos));
        FM_TRY(upload(ctx, sc, d->tri_normal, 9 * (size_t)d->num_triangles, &S.tri_normal));
        if (d->tri_normal) {
            std::vector<uint8_t> hn((size_t)d->num_triangles, 1);
            if (d->tri_has_normal) std::memcpy(hn.data(), d->tri_has_normal, hn.size());
            FM_TRY(upload(ctx, sc, hn.data(), hn.size(), &S.tri_has_normal));
        }
        FM_TRY(upload(ctx, sc, d->tri_uv, 6 * (size_t)d->num_triangles, &S.tri_uv));
        FM_TRY(upload(ctx, sc, d->tri_vattr, 3 * (size_t)d->num_triangles * (size_t)S.vattr_dim, &S.tri_vattr));
        // rectangles (rectangle.cpp:20-32, 58-74)
        std::vector<RectDev> rects((size_t)d->num_rects);
        for (int64_t i = 0; i < d->num_rects; ++i) {
            RectDev& R = rects[i];
            const float* q = d->rect_pts + 12 * i;
            for (int k = 0; k < 3; ++k) {
                R.pa[k] = q[k];
                R.pb[k] = q[3 + k];
                R.pc[k] = q[6 + k];
                R.pd[k] = q[9 + k];
            }
            const f3 e0 = ld3(R.pb) - ld3(R.pa), e1 = ld3(R.pc) - ld3(R.pa);
            f3 nrm = cross(e0, e1);
            R.area = length(nrm);
            nrm = normalize(nrm);
            f3 aux = f3{0.0f, 0.0f, 1.0f};
            if (std::fabs(nrm.z - 1.0f) < kEps || std::fabs(nrm.z + 1.0f) < kEps) aux = f3{1.0f, 0.0f, 0.0f};
            st3(R.normal, nrm);
            st3(R.ss, cross(nrm, aux));
            R.pad = 0.0f;
        }
        FM_TRY(upload(ctx, sc, rects.data(), rects.size(), &S.rects));
        // spheres (sphere.cpp:19-32)
        std::vector<SphereDev> sph((size_t)d->num_spheres);
        for (int64_t i = 0; i < d->num_spheres; ++i) {
            SphereDev& P = sph[i];
            if (!affine_inverse(d->sphere_xform + 16 * i, P.o2w, P.w2o)) {
                st = set_error(ctx, FM_ERR_INVALID, "scene_create: singular sphere transform");
                goto fail;
            }
            P.radius = d->sphere_radius[i];
            const f3 ax = f3{P.o2w.m[0], P.o2w.m[4], P.o2w.m[8]};
            P.radius_world = P.radius * length(ax);
            P.rw2 = P.radius_world * P.radius_world;
            P.area = 4.0f * kPi * P.rw2;
        }
        FM_TRY(upload(ctx, sc, sph.data(), sph.size(), &S.spheres));
        // materials
        std::vector<DevMaterial> mats((size_t)d->num_materials);
        for (int32_t i = 0; i < d->num_materials; ++i) {
            const fm_material_desc& m = d->materials[i];
            DevMaterial& M = mats[i];
            std::memset(&M, 0, sizeof(M));
            M.type = m.type;
            M.thin = m.thin;
            M.vattr_offset = m.vattr_offset;
            const fm_tex_ref* refs = &m.basecolor;
            for (int k = 0; k < MP_COUNT; ++k) to_texref(refs[k], M.p[k]);
            for (int k = 0; k < 3; ++k) {
                M.reflect_color[k] = m.reflect_color[k];
                M.refract_color[k] = m.refract_color[k];
                M.color[k] = m.color[k];
                // ConductorFresnel (fresnel.h:77-84)
                const float eta2 = m.cond_eta_t[k] / m.cond_eta_i[k];
                const float etak2 = m.cond_k[k] / m.cond_eta_i[k];
                M.cond_eta2[k] = eta2 * eta2;
                M.cond_etak2[k] = etak2 * etak2;
            }
            M.eta_i = m.eta_i;
            M.eta_t = m.eta_t;
        }
        FM_TRY(upload(ctx, sc, mats.data(), mats.size(), &S.materials));
        S.num_materials = d->num_materials;
        // textures (float4 texels)
        std::vector<DevTexture> texs((size_t)d->num_textures);
        for (int32_t i = 0; i < d->num_textures; ++i) {
            const fm_texture_desc& t = d->textures[i];
            const size_t nt = (size_t)t.width * t.height;
            std::vector<float4> px(nt);
            for (size_t q = 0; q < nt; ++q) px[q] = make_float4(t.texels[3 * q], t.texels[3 * q + 1], t.texels[3 * q + 2], 0.0f);
            const float4* dp = nullptr;
            FM_TRY(upload(ctx, sc, px.data(), nt, &dp));
            texs[i] = DevTexture{dp, t.width, t.height, t.wrap_u, t.wrap_v, t.filter, 0};
            FM_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "texture upload");
        }
        FM_TRY(upload(ctx, sc, texs.data(), texs.size(), &S.textures));
        S.num_textures = d->num_textures;
        sc->textures = texs;
        // lights: area lights in object order (Scene::Scene via
        // Aggregate::ConstructAreaLight, core/scene.h:21-25), then the given lights
        std::vector<DevLight> lights;
        std::vector<int32_t> obj_light((size_t)d->num_objects, -1);
        // mesh lights: group id -> light index, and each mesh light's triangles
        std::map<int32_t, int32_t> group_light;
        std::vector<std::vector<int32_t>> mesh_tris;
        if (d->obj_emission) {
            for (int64_t o = 0; o < d->num_objects; ++o) {
                const float* em = d->obj_emission + 3 * o;
                if (is_black_h(em)) continue;
                if (geo_count[o] != 1) {
                    st = set_error(ctx, FM_ERR_INVALID, "scene_create: an emissive object must have exactly one shape");
                    goto fail;
                }
                const int32_t group =
                    geo_kind[o] == LK_AREA_TRI && d->tri_light_group ? d->tri_light_group[geo_index[o]] : -1;
                if (group >= 0) {
                    auto it = group_light.find(group);
                    if (it != group_light.end()) {
                        const DevLight& G = lights[it->second];
                        if (G.radiance[0] != em[0] || G.radiance[1] != em[1] || G.radiance[2] != em[2]) {
                            st = set_error(ctx, FM_ERR_INVALID, "scene_create: a mesh light's triangles differ in emission");
                            goto fail;
                        }
                        mesh_tris[G.index].push_back(geo_index[o]);
                        obj_light[o] = it->second;
                        continue;
                    }
                }
                DevLight L{};
                L.kind = group >= 0 ? LK_AREA_MESH : geo_kind[o];
                L.obj = (int32_t)o;
                L.index = geo_index[o];
                for (int k = 0; k < 3; ++k) L.radiance[k] = em[k];
                if (group >= 0) {
                    // index: the light's slot in mesh_tris until the tables are laid out
                    L.index = (int32_t)mesh_tris.size();
                    mesh_tris.push_back({geo_index[o]});
                    group_light[group] = (int32_t)lights.size();
                }
                obj_light[o] = (int32_t)lights.size();
                lights.push_back(L);
            }
        }
        if (!mesh_tris.empty()) {
            // each mesh light's triangles, contiguous, with an alias table over their areas
            std::vector<int32_t> mtri, malias;
            std::vector<float> mprob;
            for (auto& L : lights) {
                if (L.kind != LK_AREA_MESH) continue;
                const std::vector<int32_t>& tris = mesh_tris[L.index];
                std::vector<double> area(tris.size());
                double total = 0.0;
                for (size_t k = 0; k < tris.size(); ++k) {
                    const float* v = d->tri_pos + 9 * (size_t)tris[k];
                    const double e1[3] = {(double)v[3] - v[0], (double)v[4] - v[1], (double)v[5] - v[2]};
                    const double e2[3] = {(double)v[6] - v[0], (double)v[7] - v[1], (double)v[8] - v[2]};
                    const double c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                                         e1[0] * e2[1] - e1[1] * e2[0]};
                    area[k] = 0.5 * std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
                    total += area[k];
                }
                if (!(total > 0.0)) {
                    st = set_error(ctx, FM_ERR_INVALID, "scene_create: a mesh light has zero area");
                    goto fail;
                }
                std::vector<float> prob;
                std::vector<int32_t> alias;
                vose_alias(area, prob, alias);
                L.index = (int32_t)mtri.size();
                L.count = (int32_t)tris.size();
                L.inv_area = (float)(1.0 / total);
                mtri.insert(mtri.end(), tris.begin(), tris.end());
                mprob.insert(mprob.end(), prob.begin(), prob.end());
                malias.insert(malias.end(), alias.begin(), alias.end());
            }
            FM_TRY(upload(ctx, sc, mtri.data(), mtri.size(), &S.mlight_tri));
            FM_TRY(upload(ctx, sc, mprob.data(), mprob.size(), &S.mlight_prob));
            FM_TRY(upload(ctx, sc, malias.data(), malias.size(), &S.mlight_alias));
        }
        S.env_light = -1;
        for (int32_t i = 0; i < d->num_lights; ++i) {
            const fm_light_desc& l = d->lights[i];
            DevLight L{};
            if (l.type == FM_LIGHT_ENV) {
                L.kind = LK_ENV;
                if (i == env_light_desc) S.env_light = (int32_t)lights.size();
            } else {
                L.kind = LK_DIR;
                for (int k = 0; k < 3; ++k) {
                    L.radiance[k] = l.radiance[k];
                    L.direction[k] = l.direction[k];
                }
            }
            L.obj = -1;
            L.index = i;
            lights.push_back(L);
        }
        sc->lights = lights;
        {
            // what the wavefront's hit resolution needs of a primitive, in one load
            std::vector<int32_t> prim_info((size_t)nprim);
            for (int64_t p = 0; p < nprim; ++p) {
                const int32_t o = prim_obj[p];
                prim_info[p] = ((obj_light[o] + 1) << 2) | (material_class(mats[d->obj_material[o]].type) + 1);
            }
            FM_TRY(upload(ctx, sc, prim_info.data(), prim_info.size(), &S.prim_info));
        }
        FM_TRY(upload(ctx, sc, obj_light.data(), obj_light.size(), &S.obj_light));
        FM_TRY(upload(ctx, sc, d->obj_material, (size_t)d->num_objects, &S.obj_material));
        FM_TRY(upload(ctx, sc, lights.data(), lights.size(), &S.lights));
        S.num_lights = (int32_t)lights.size();
        FM_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "scene upload");
        // environment light
        std::memset(&S.env, 0, sizeof(S.env));
        if (env_light_desc >= 0) {
            const fm_light_desc& l = d->lights[env_light_desc];
            S.env.present = 1;
            S.env.tex = l.texture;
            S.env.factor = l.factor;
            rotation_zyx(l.rotation, S.env.l2w, S.env.w2l);
            FM_TRY(env_build_tables(ctx, sc, texs[l.texture], S.env));
        }
        // BVH
        PrimSource src;
        src.num_tris = S.num_tris;
        src.num_rects = S.num_rects;
        src.num_spheres = S.num_spheres;
        src.tri_pos = S.tri_pos;
        src.rects = S.rects;
        src.spheres = S.spheres;
        std::string err;
        if (bvh_build(ctx->stream, src, sc->bvh, err) != 0) {
            st = set_error(ctx, FM_ERR_CUDA, err);
            goto fail;
        }
        sc->allocations.push_back(sc->bvh.nodes);
        sc->allocations.push_back(sc->bvh.leaf);
        S.nodes = sc->bvh.nodes;
        S.leaf = sc->bvh.leaf;
        S.num_nodes = sc->bvh.num_nodes;
        S.num_leaf = sc->bvh.num_leaf;
        void* dd = nullptr;
        FM_CUDA_TRY(ctx, cudaMallocAsync(&dd, sizeof(DevScene), ctx->stream), "scene alloc");
        sc->allocations.push_back(dd);
        sc->d_dev = static_cast<DevScene*>(dd);
        FM_CUDA_TRY(ctx, cudaMemcpyAsync(dd, &S, sizeof(DevScene), cudaMemcpyHostToDevice, ctx->stream), "scene copy");
        FM_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream), "scene sync");
    }
#undef FM_TRY
    *out = sc;
    return FM_OK;
fail:
    for (void* p : sc->allocations) cudaFreeAsync(p, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    delete sc;
    return st;
}

fm_status fm_scene_destroy(fm_ctx* ctx, fm_scene* sc)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!sc) return FM_OK;
    cudaSetDevice(ctx->device);
    for (void* p : sc->allocations) cudaFreeAsync(p, ctx->stream);
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
