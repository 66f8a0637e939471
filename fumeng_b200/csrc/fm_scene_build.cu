// Scene creation: a scene description flattened into one device block per scene, its
// environment tables and its BVH built on the device.
//
// Many scenes are created in one call (fm_scene_create_batch).  The host prepares every
// scene first, in parallel (validation, derived arrays, light tables, the block's
// layout); then each scene's arrays stream through a pinned staging ring into the scene's
// device block on the context's stream, its texel expansion and environment tables run on
// one of a few builder streams, and every kGroupScenes scenes one BVH build serves the
// whole group (one chain of level launches instead of one per scene; a build alone is
// latency-bound), overlapping the next groups' uploads.  The host waits once for all
// builds, writes each scene's DevScene record, and waits once more.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <new>

#include "fm_bvh.cuh"
#include "fm_internal.h"
#include "fm_staging.h"

using namespace fm;

namespace fm {

namespace {

__global__ void k_rgb_to_texels(const float* __restrict__ src, float4* __restrict__ dst, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.0f);
}

}  // namespace

void launch_rgb_to_texels(cudaStream_t stream, const float* src, float4* dst, size_t n, int num_sms)
{
    const int grid = (int)std::min<size_t>((n + 255) / 256, (size_t)num_sms * 16);
    if (grid > 0) k_rgb_to_texels<<<grid, 256, 0, stream>>>(src, dst, n);
}

}  // namespace fm

namespace {

constexpr int kBuildStreams = 16;   // scenes whose device work runs side by side
constexpr size_t kAlign = 256;     // sub-array alignment inside a scene's block

size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

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

// One host array bound for a scene's device block.
struct Piece {
    const void* src;
    size_t bytes;
    size_t off;     // offset in the block
    void* field;    // address of the device-pointer member to point at it
};

// One texture: RGB texels copied to a staging allocation, expanded to float4 in the block.
struct TexPiece {
    const float* src;
    size_t texels;
    size_t rgb_off;   // offset in the RGB staging allocation
    size_t off;       // offset of the float4 texels in the block
};

// A scene under construction.
struct SceneBuild {
    fm_scene* sc = nullptr;
    int env_light_desc = -1;
    std::vector<Piece> pieces;
    std::vector<TexPiece> tex_pieces;
    size_t block_bytes = 0;   // DevScene record, the arrays, the float4 texels
    size_t rgb_bytes = 0;
    char* d_block = nullptr;
    char* d_rgb = nullptr;
    // host arrays the pieces point into
    std::vector<int32_t> prim_obj, prim_info, obj_light, mtri, malias;
    std::vector<uint8_t> has_normal;
    std::vector<float> mprob;
    std::vector<RectDev> rects;
    std::vector<SphereDev> sph;
    std::vector<DevMaterial> mats;

    std::string error;

    fm_status fail(fm_status st, const char* msg)
    {
        error = msg;
        return st;
    }

    template <typename T>
    void add(const T* host, size_t count, const T** field)
    {
        *field = nullptr;
        if (!host || count == 0) return;
        block_bytes = align_up(block_bytes);
        pieces.push_back(Piece{host, sizeof(T) * count, block_bytes, static_cast<void*>(field)});
        block_bytes += sizeof(T) * count;
    }
};

// Validates a description and prepares everything host-side: derived arrays, lights and
// their tables, and the layout of the scene's device block.  No device work and no
// context state (scenes are prepared on several threads); errors go to B.error.
fm_status prepare_scene(const fm_scene_desc* d, SceneBuild& B)
{
    if (!d) return B.fail(FM_ERR_INVALID, "scene_create: null argument");
    if (d->num_objects < 0 || d->num_triangles < 0 || d->num_rects < 0 || d->num_spheres < 0 ||
        d->num_materials < 0 || d->num_textures < 0 || d->num_lights < 0)
        return B.fail(FM_ERR_INVALID, "scene_create: negative count");
    const int64_t nprim = d->num_triangles + 2 * d->num_rects + d->num_spheres;
    if (nprim > (int64_t)0x3fffffff) return B.fail(FM_ERR_INVALID, "scene_create: too many primitives");
    if (d->num_objects > 0 && !d->obj_material) return B.fail(FM_ERR_INVALID, "scene_create: obj_material is null");
    if (d->num_triangles > 0 && (!d->tri_pos || !d->tri_object))
        return B.fail(FM_ERR_INVALID, "scene_create: triangle arrays are null");
    if (d->num_rects > 0 && (!d->rect_pts || !d->rect_object))
        return B.fail(FM_ERR_INVALID, "scene_create: rectangle arrays are null");
    if (d->num_spheres > 0 && (!d->sphere_radius || !d->sphere_xform || !d->sphere_object))
        return B.fail(FM_ERR_INVALID, "scene_create: sphere arrays are null");
    if (d->num_materials > 0 && !d->materials) return B.fail(FM_ERR_INVALID, "scene_create: materials is null");
    if (d->num_textures > 0 && !d->textures) return B.fail(FM_ERR_INVALID, "scene_create: textures is null");
    if (d->num_lights > 0 && !d->lights) return B.fail(FM_ERR_INVALID, "scene_create: lights is null");
    if (d->tri_vattr && d->vattr_dim < 6) return B.fail(FM_ERR_INVALID, "scene_create: vattr_dim < 6");
    for (int64_t o = 0; o < d->num_objects; ++o)
        if (d->obj_material[o] < 0 || d->obj_material[o] >= d->num_materials)
            return B.fail(FM_ERR_INVALID, "scene_create: object material index out of range");
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
        if (!note(d->tri_object[i], LK_AREA_TRI, i)) return B.fail(FM_ERR_INVALID, "scene_create: triangle object out of range");
    for (int64_t i = 0; i < d->num_rects; ++i)
        if (!note(d->rect_object[i], LK_AREA_RECT, i)) return B.fail(FM_ERR_INVALID, "scene_create: rectangle object out of range");
    for (int64_t i = 0; i < d->num_spheres; ++i)
        if (!note(d->sphere_object[i], LK_AREA_SPHERE, i)) return B.fail(FM_ERR_INVALID, "scene_create: sphere object out of range");
    for (int32_t i = 0; i < d->num_textures; ++i) {
        const fm_texture_desc& t = d->textures[i];
        if (t.width <= 0 || t.height <= 0 || !t.texels) return B.fail(FM_ERR_INVALID, "scene_create: bad texture");
    }
    auto tex_ok = [&](const fm_tex_ref& r) { return r.texture < d->num_textures; };
    for (int32_t i = 0; i < d->num_materials; ++i) {
        const fm_material_desc& m = d->materials[i];
        if (m.type < FM_MAT_LAMBERT || m.type > FM_MAT_DISNEY) return B.fail(FM_ERR_INVALID, "scene_create: bad material type");
        const fm_tex_ref* refs = &m.basecolor;
        for (int k = 0; k < MP_COUNT; ++k)
            if (!tex_ok(refs[k])) return B.fail(FM_ERR_INVALID, "scene_create: material texture out of range");
        if (m.vattr_offset >= 0 && (!d->tri_vattr || m.vattr_offset + 6 > d->vattr_dim))
            return B.fail(FM_ERR_INVALID, "scene_create: material vertex attributes out of range");
    }
    int env_light_desc = -1;
    for (int32_t i = 0; i < d->num_lights; ++i) {
        const fm_light_desc& l = d->lights[i];
        if (l.type == FM_LIGHT_ENV) {
            if (l.texture < 0 || l.texture >= d->num_textures) return B.fail(FM_ERR_INVALID, "scene_create: env texture out of range");
            if (env_light_desc < 0) env_light_desc = i;
        } else if (l.type != FM_LIGHT_DIRECTIONAL) {
            return B.fail(FM_ERR_INVALID, "scene_create: bad light type");
        }
    }
    B.env_light_desc = env_light_desc;

    fm_scene* sc = new (std::nothrow) fm_scene();
    if (!sc) return B.fail(FM_ERR_OOM, "scene_create: host allocation");
    B.sc = sc;
    sc->num_objects = d->num_objects;
    DevScene& S = sc->dev;
    B.block_bytes = sizeof(DevScene);   // the record itself, written last
    S.num_tris = (int32_t)d->num_triangles;
    S.num_rects = (int32_t)d->num_rects;
    S.num_spheres = (int32_t)d->num_spheres;
    S.num_prims = (int32_t)nprim;
    S.num_objects = (int32_t)d->num_objects;
    S.vattr_dim = d->tri_vattr ? d->vattr_dim : 0;
    // primitive -> object
    B.prim_obj.resize((size_t)nprim);
    for (int64_t i = 0; i < d->num_triangles; ++i) B.prim_obj[i] = d->tri_object[i];
    for (int64_t i = 0; i < d->num_rects; ++i)
        B.prim_obj[d->num_triangles + 2 * i] = B.prim_obj[d->num_triangles + 2 * i + 1] = d->rect_object[i];
    for (int64_t i = 0; i < d->num_spheres; ++i) B.prim_obj[d->num_triangles + 2 * d->num_rects + i] = d->sphere_object[i];
    B.add(B.prim_obj.data(), B.prim_obj.size(), &S.prim_obj);
    B.add(d->tri_pos, 9 * (size_t)d->num_triangles, &S.tri_pos);
    B.add(d->tri_normal, 9 * (size_t)d->num_triangles, &S.tri_normal);
    S.tri_has_normal = nullptr;
    if (d->tri_normal) {
        if (d->tri_has_normal) {
            B.add(d->tri_has_normal, (size_t)d->num_triangles, &S.tri_has_normal);
        } else {
            B.has_normal.assign((size_t)d->num_triangles, 1);
            B.add(B.has_normal.data(), B.has_normal.size(), &S.tri_has_normal);
        }
    }
    B.add(d->tri_uv, 6 * (size_t)d->num_triangles, &S.tri_uv);
    B.add(d->tri_vattr, 3 * (size_t)d->num_triangles * (size_t)S.vattr_dim, &S.tri_vattr);
    // rectangles (rectangle.cpp:20-32, 58-74)
    B.rects.resize((size_t)d->num_rects);
    for (int64_t i = 0; i < d->num_rects; ++i) {
        RectDev& R = B.rects[i];
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
    B.add(B.rects.data(), B.rects.size(), &S.rects);
    // spheres (sphere.cpp:19-32)
    B.sph.resize((size_t)d->num_spheres);
    for (int64_t i = 0; i < d->num_spheres; ++i) {
        SphereDev& P = B.sph[i];
        if (!affine_inverse(d->sphere_xform + 16 * i, P.o2w, P.w2o))
            return B.fail(FM_ERR_INVALID, "scene_create: singular sphere transform");
        P.radius = d->sphere_radius[i];
        const f3 ax = f3{P.o2w.m[0], P.o2w.m[4], P.o2w.m[8]};
        P.radius_world = P.radius * length(ax);
        P.rw2 = P.radius_world * P.radius_world;
        P.area = 4.0f * kPi * P.rw2;
    }
    B.add(B.sph.data(), B.sph.size(), &S.spheres);
    // materials
    B.mats.resize((size_t)d->num_materials);
    for (int32_t i = 0; i < d->num_materials; ++i) {
        const fm_material_desc& m = d->materials[i];
        DevMaterial& M = B.mats[i];
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
    B.add(B.mats.data(), B.mats.size(), &S.materials);
    S.num_materials = d->num_materials;
    // textures: float4 texels in the block, expanded on the device from RGB
    sc->textures.resize((size_t)d->num_textures);
    for (int32_t i = 0; i < d->num_textures; ++i) {
        const fm_texture_desc& t = d->textures[i];
        const size_t nt = (size_t)t.width * t.height;
        B.block_bytes = align_up(B.block_bytes);
        B.rgb_bytes = align_up(B.rgb_bytes);
        B.tex_pieces.push_back(TexPiece{t.texels, nt, B.rgb_bytes, B.block_bytes});
        B.block_bytes += nt * sizeof(float4);
        B.rgb_bytes += nt * 3 * sizeof(float);
        sc->textures[i] = DevTexture{nullptr, t.width, t.height, t.wrap_u, t.wrap_v, t.filter, 0};
    }
    B.add(sc->textures.data(), sc->textures.size(), &S.textures);
    S.num_textures = d->num_textures;
    // lights: area lights in object order (Scene::Scene via
    // Aggregate::ConstructAreaLight, core/scene.h:21-25), then the given lights
    std::vector<DevLight>& lights = sc->lights;
    B.obj_light.assign((size_t)d->num_objects, -1);
    // mesh lights: group id -> light index, and each mesh light's triangles
    std::map<int32_t, int32_t> group_light;
    std::vector<std::vector<int32_t>> mesh_tris;
    if (d->obj_emission) {
        for (int64_t o = 0; o < d->num_objects; ++o) {
            const float* em = d->obj_emission + 3 * o;
            if (is_black_h(em)) continue;
            if (geo_count[o] != 1)
                return B.fail(FM_ERR_INVALID, "scene_create: an emissive object must have exactly one shape");
            const int32_t group =
                geo_kind[o] == LK_AREA_TRI && d->tri_light_group ? d->tri_light_group[geo_index[o]] : -1;
            if (group >= 0) {
                auto it = group_light.find(group);
                if (it != group_light.end()) {
                    const DevLight& G = lights[it->second];
                    if (G.radiance[0] != em[0] || G.radiance[1] != em[1] || G.radiance[2] != em[2])
                        return B.fail(FM_ERR_INVALID, "scene_create: a mesh light's triangles differ in emission");
                    mesh_tris[G.index].push_back(geo_index[o]);
                    B.obj_light[o] = it->second;
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
            B.obj_light[o] = (int32_t)lights.size();
            lights.push_back(L);
        }
    }
    if (!mesh_tris.empty()) {
        // each mesh light's triangles, contiguous, with an alias table over their areas
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
            if (!(total > 0.0)) return B.fail(FM_ERR_INVALID, "scene_create: a mesh light has zero area");
            std::vector<float> prob;
            std::vector<int32_t> alias;
            vose_alias(area, prob, alias);
            L.index = (int32_t)B.mtri.size();
            L.count = (int32_t)tris.size();
            L.inv_area = (float)(1.0 / total);
            B.mtri.insert(B.mtri.end(), tris.begin(), tris.end());
            B.mprob.insert(B.mprob.end(), prob.begin(), prob.end());
            B.malias.insert(B.malias.end(), alias.begin(), alias.end());
        }
    }
    B.add(B.mtri.data(), B.mtri.size(), &S.mlight_tri);
    B.add(B.mprob.data(), B.mprob.size(), &S.mlight_prob);
    B.add(B.malias.data(), B.malias.size(), &S.mlight_alias);
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
    // what the wavefront's hit resolution needs of a primitive, in one load
    B.prim_info.resize((size_t)nprim);
    for (int64_t p = 0; p < nprim; ++p) {
        const int32_t o = B.prim_obj[p];
        B.prim_info[p] = ((B.obj_light[o] + 1) << 2) | (material_class(B.mats[d->obj_material[o]].type) + 1);
    }
    B.add(B.prim_info.data(), B.prim_info.size(), &S.prim_info);
    B.add(B.obj_light.data(), B.obj_light.size(), &S.obj_light);
    B.add(d->obj_material, (size_t)d->num_objects, &S.obj_material);
    B.add(lights.data(), lights.size(), &S.lights);
    S.num_lights = (int32_t)lights.size();
    // environment light (tables built on the device)
    std::memset(&S.env, 0, sizeof(S.env));
    if (env_light_desc >= 0) {
        const fm_light_desc& l = d->lights[env_light_desc];
        S.env.present = 1;
        S.env.tex = l.texture;
        S.env.factor = l.factor;
        rotation_zyx(l.rotation, S.env.l2w, S.env.w2l);
    }
    return FM_OK;
}

fm_status ensure_builder(fm_ctx* ctx)
{
    if (ctx->build_streams.empty()) {
        // streams: kBuildStreams run device work, one more only captures the BVH build
        // graphs; events: [0] a scene's arrays are on the device, [1 + k] builder stream k
        // is done
        std::vector<cudaStream_t> streams;
        std::vector<cudaEvent_t> events;
        cudaError_t e = cudaSuccess;
        for (int k = 0; k <= kBuildStreams && e == cudaSuccess; ++k) {
            cudaStream_t s = nullptr;
            e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
            if (e == cudaSuccess) streams.push_back(s);
        }
        for (int k = 0; k <= kBuildStreams && e == cudaSuccess; ++k) {
            cudaEvent_t ev = nullptr;
            e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (e == cudaSuccess) events.push_back(ev);
        }
        if (e != cudaSuccess) {
            for (cudaStream_t s : streams) cudaStreamDestroy(s);
            for (cudaEvent_t ev : events) cudaEventDestroy(ev);
            return cuda_error(ctx, e, "scene builder streams");
        }
        ctx->capture_stream = streams.back();
        streams.pop_back();
        ctx->build_streams = streams;
        ctx->build_events = events;
    }
    FM_CUDA_TRY(ctx, staging_ensure(ctx), "scene staging");
    return FM_OK;
}

// A group of consecutive scenes whose BVHs are built together.
struct Group {
    int first = 0, count = 0;
    BvhJob* job = nullptr;
    BvhBatch bvh;
    char* h_pinned = nullptr;
};

// Frees every scene of a failed batch, and the group builds (after the device work has
// drained).
void discard(fm_ctx* ctx, std::vector<SceneBuild>& builds, std::vector<Group>& groups)
{
    for (cudaStream_t s : ctx->build_streams) cudaStreamSynchronize(s);
    cudaStreamSynchronize(ctx->stream);
    for (Group& g : groups) {
        if (g.job) bvh_build_abort(g.job, g.bvh);
        g.job = nullptr;
    }
    for (SceneBuild& B : builds) {
        if (!B.sc) continue;
        if (B.d_rgb) cudaFreeAsync(B.d_rgb, ctx->stream);
        for (void* p : B.sc->allocations) cudaFreeAsync(p, ctx->stream);
        B.sc->shared_bvh.reset();
        delete B.sc;
        B.sc = nullptr;
    }
    cudaStreamSynchronize(ctx->stream);
    cudaGetLastError();
}

// Scenes per BVH build: the builds of a batch's groups overlap the uploads of the later
// groups, and each build serves all scenes of its group with one chain of launches.
// Creating the 64-scene batch with 8 / 16 / 32 / 64 scenes per build: 29-31 / 26-28 /
// 23-24.5 / 28-29 ms.
constexpr int kGroupScenes = 32;

fm_status create_scenes(fm_ctx* ctx, int32_t n, const fm_scene_desc* const* descs, fm_scene** out)
{
    FM_CUDA_TRY(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    {
        const fm_status st = ensure_builder(ctx);
        if (st != FM_OK) return st;
    }
    std::vector<SceneBuild> builds((size_t)n);
    // host preparation, scenes side by side
    {
        std::vector<fm_status> sts((size_t)n, FM_OK);
        host_parallel(ctx, n, [&](int i) {
            try {
                sts[i] = prepare_scene(descs[i], builds[i]);
            } catch (const std::bad_alloc&) {
                sts[i] = builds[i].fail(FM_ERR_OOM, "scene_create: host allocation failed");
            }
        });
        for (int32_t i = 0; i < n; ++i) {
            if (sts[i] != FM_OK) {
                const std::string msg = builds[i].error;
                for (SceneBuild& B : builds) delete B.sc;
                return set_error(ctx, sts[i], msg);
            }
        }
    }
    // groups and their pinned space (scene table and counters of each build)
    std::vector<Group> groups;
    size_t pinned = 0;
    for (int32_t i = 0; i < n; i += kGroupScenes) {
        Group g;
        g.first = i;
        g.count = std::min<int32_t>(kGroupScenes, n - i);
        pinned += (bvh_batch_pinned_bytes(g.count) + 255) & ~size_t(255);
        groups.push_back(g);
    }
    if (ctx->build_pinned_bytes < pinned) {
        if (ctx->build_pinned) cudaFreeHost(ctx->build_pinned);
        ctx->build_pinned = nullptr;
        ctx->build_pinned_bytes = 0;
        void* p = nullptr;
        const cudaError_t e = cudaHostAlloc(&p, pinned, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            for (SceneBuild& B : builds) delete B.sc;
            return cuda_error(ctx, e, "scene build staging");
        }
        ctx->build_pinned = static_cast<char*>(p);
        ctx->build_pinned_bytes = pinned;
    }
    {
        size_t off = 0;
        for (Group& g : groups) {
            g.h_pinned = ctx->build_pinned + off;
            off += (bvh_batch_pinned_bytes(g.count) + 255) & ~size_t(255);
        }
    }
    cudaStream_t cs = ctx->stream;
    Stager stager(ctx, cs);
    fm_status st = FM_OK;
    auto fail = [&](fm_status code, const std::string& msg) {
        discard(ctx, builds, groups);
        return set_error(ctx, code, msg);
    };
    auto fail_cuda = [&](cudaError_t e, const char* where) {
        return fail(FM_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
    };
    size_t next_group = 0;
    for (int32_t i = 0; i < n; ++i) {
        SceneBuild& B = builds[i];
        fm_scene* sc = B.sc;
        DevScene& S = sc->dev;
        cudaStream_t bs = ctx->build_streams[(size_t)i % ctx->build_streams.size()];
        cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&B.d_block), B.block_bytes, cs);
        if (e != cudaSuccess) return fail_cuda(e, "scene allocation");
        sc->allocations.push_back(B.d_block);
        sc->d_dev = reinterpret_cast<DevScene*>(B.d_block);
        if (B.rgb_bytes) {
            e = cudaMallocAsync(reinterpret_cast<void**>(&B.d_rgb), B.rgb_bytes, cs);
            if (e != cudaSuccess) return fail_cuda(e, "scene allocation");
        }
        for (const Piece& p : B.pieces) {
            const void* dp = B.d_block + p.off;
            std::memcpy(p.field, &dp, sizeof(dp));
        }
        for (size_t t = 0; t < B.tex_pieces.size(); ++t)
            sc->textures[t].texels = reinterpret_cast<const float4*>(B.d_block + B.tex_pieces[t].off);
        // pieces of a block (and of the RGB staging) that only alignment padding separates
        // go to the device as one copy; the float4 texel regions in between are not copied
        auto padding = [](size_t end, size_t off) { return off - end < kAlign ? off - end : 0; };
        size_t end = sizeof(DevScene);
        for (const Piece& p : B.pieces) {
            stager.put(B.d_block + p.off, p.src, p.bytes, padding(end, p.off));
            end = p.off + p.bytes;
        }
        end = 0;
        for (const TexPiece& t : B.tex_pieces) {
            stager.put(B.d_rgb + t.rgb_off, t.src, t.texels * 3 * sizeof(float), padding(end, t.rgb_off));
            end = t.rgb_off + t.texels * 3 * sizeof(float);
        }
        stager.flush();
        if (stager.err != cudaSuccess) return fail_cuda(stager.err, "scene upload");
        // the scene's device work follows its copies, on its builder stream
        e = cudaEventRecord(ctx->build_events[0], cs);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(bs, ctx->build_events[0], 0);
        if (e != cudaSuccess) return fail_cuda(e, "scene upload");
        for (const TexPiece& t : B.tex_pieces)
            launch_rgb_to_texels(bs, reinterpret_cast<const float*>(B.d_rgb + t.rgb_off),
                                 reinterpret_cast<float4*>(B.d_block + t.off), t.texels, ctx->num_sms);
        if (B.d_rgb) {
            cudaFreeAsync(B.d_rgb, bs);
            B.d_rgb = nullptr;
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return fail_cuda(e, "texel expansion");
        if (B.env_light_desc >= 0) {
            st = env_build_tables(ctx, bs, sc, sc->textures[S.env.tex], S.env);
            if (st != FM_OK) return fail(st, ctx->error);
        }
        // the group's last scene is on the device: build the group's BVHs on a builder
        // stream while the next groups upload
        Group& g = groups[next_group];
        if (i == g.first + g.count - 1) {
            ++next_group;
            std::vector<PrimSource> srcs((size_t)g.count);
            for (int k = 0; k < g.count; ++k) {
                const DevScene& D = builds[(size_t)(g.first + k)].sc->dev;
                PrimSource& p = srcs[(size_t)k];
                p.num_tris = D.num_tris;
                p.num_rects = D.num_rects;
                p.num_spheres = D.num_spheres;
                p.tri_pos = D.tri_pos;
                p.rects = D.rects;
                p.spheres = D.spheres;
            }
            cudaStream_t gs = ctx->build_streams[(next_group - 1) % ctx->build_streams.size()];
            e = cudaStreamWaitEvent(gs, ctx->build_events[0], 0);
            if (e != cudaSuccess) return fail_cuda(e, "scene build");
            std::string err;
            if (bvh_build_batch_begin(gs, ctx->capture_stream, srcs.data(), g.count, g.h_pinned, ctx->num_sms, g.job,
                                      g.bvh, err) != 0)
                return fail(FM_ERR_CUDA, err);
        }
    }
    // wait for the builds; then every scene's record
    for (Group& g : groups) {
        BvhJob* job = g.job;
        g.job = nullptr;
        std::string err;
        if (bvh_build_batch_end(job, g.bvh, err) != 0) return fail(FM_ERR_CUDA, err);
        // the group's arrays live until the last of its scenes is destroyed
        std::shared_ptr<void> shared;
        uint4* gnodes = g.bvh.nodes;
        float4* gleaf = g.bvh.leaf;
        if (gnodes) {
            cudaStream_t fs = ctx->stream;
            shared = std::shared_ptr<void>(gnodes, [gleaf, fs](void* p) {
                cudaFreeAsync(p, fs);
                cudaFreeAsync(gleaf, fs);
            });
            g.bvh.nodes = nullptr;
            g.bvh.leaf = nullptr;
        }
        for (int k = 0; k < g.count; ++k) {
            fm_scene* sc = builds[(size_t)(g.first + k)].sc;
            DevScene& S = sc->dev;
            const int r = g.bvh.root.empty() ? -1 : g.bvh.root[(size_t)k];
            sc->bvh = BvhResult{};
            sc->bvh.build_ms = g.bvh.build_ms;
            if (r >= 0) {
                sc->shared_bvh = shared;
                S.nodes = gnodes + 5 * (size_t)r;
                S.leaf = gleaf;
                sc->bvh.num_nodes = g.bvh.num_nodes[(size_t)k];
                sc->bvh.num_leaf = g.bvh.num_leaf[(size_t)k];
                sc->bvh.depth = g.bvh.depth[(size_t)k];
            } else {
                S.nodes = nullptr;
                S.leaf = nullptr;
            }
            S.num_nodes = sc->bvh.num_nodes;
            S.num_leaf = sc->bvh.num_leaf;
        }
    }
    for (size_t k = 0; k < ctx->build_streams.size(); ++k) {
        cudaError_t e = cudaEventRecord(ctx->build_events[1 + k], ctx->build_streams[k]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, ctx->build_events[1 + k], 0);
        if (e != cudaSuccess) return fail_cuda(e, "scene build join");
    }
    for (int32_t i = 0; i < n; ++i) stager.put(builds[i].sc->d_dev, &builds[i].sc->dev, sizeof(DevScene));
    stager.close();
    if (stager.err != cudaSuccess) return fail_cuda(stager.err, "scene record upload");
    {
        const cudaError_t e = cudaStreamSynchronize(cs);
        if (e != cudaSuccess) return fail_cuda(e, "scene sync");
    }
    for (int32_t i = 0; i < n; ++i) out[i] = builds[i].sc;
    return FM_OK;
}

}  // namespace

namespace fm {

void scene_builder_release(fm_ctx* ctx)
{
    for (cudaStream_t s : ctx->build_streams) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    for (cudaEvent_t e : ctx->build_events) cudaEventDestroy(e);
    if (ctx->capture_stream) cudaStreamDestroy(ctx->capture_stream);
    ctx->capture_stream = nullptr;
    ctx->build_streams.clear();
    ctx->build_events.clear();
    if (ctx->build_pinned) cudaFreeHost(ctx->build_pinned);
    ctx->build_pinned = nullptr;
    ctx->build_pinned_bytes = 0;
}

}  // namespace fm

extern "C" {

fm_status fm_scene_create(fm_ctx* ctx, const fm_scene_desc* d, fm_scene** out)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!d || !out) return set_error(ctx, FM_ERR_INVALID, "scene_create: null argument");
    *out = nullptr;
    return create_scenes(ctx, 1, &d, out);
}

fm_status fm_scene_create_batch(fm_ctx* ctx, int32_t n, const fm_scene_desc* const* descs, fm_scene** out)
{
    if (!ctx) return FM_ERR_INVALID;
    if (n < 0 || (n > 0 && (!descs || !out))) return set_error(ctx, FM_ERR_INVALID, "scene_create_batch: bad arguments");
    for (int32_t i = 0; i < n; ++i) out[i] = nullptr;
    if (n == 0) return FM_OK;
    return create_scenes(ctx, n, descs, out);
}

}  // extern "C"
