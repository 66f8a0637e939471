// Oracle harness: a C API over the UNMODIFIED reference engine (hietwll/Fumeng),
// compiled from the reference sources where they lie by oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product (the fumeng_b200 package, its
// shared library, bench.py's measured arm) links, loads or calls this code.  Only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm use it,
// as the checker and the CPU baseline.
//
// Built twice: with USE_FLOAT (the reference's float build: hit-ID oracle and timed CPU
// baseline) and without it (the reference's default double build: image oracle).
//
// How the harness reaches the reference:
//  * scene loading goes through the reference's own SceneLoader (scene_loader.h:293-302)
//    step by step, so that one schema extension can be injected: materials of type
//    "specular_reflection" (reachable in the reference only through
//    CreateSpecularReflection, create/material.h:11) are inserted into the loader's
//    material table before ParseScene runs; ParseMaterial's later emplace of the
//    unknown type is then a no-op (scene_loader.h:199).
//  * private/protected members are opened with a preprocessor define for this
//    translation unit only, so that the harness can read the loader's object list and
//    reseed each PathTracer's sampler (sampler.h:16) per pixel; the reference files
//    themselves are not edited.
//  * path_tracing.cpp is compiled inside this translation unit (it defines class
//    PathTracer in a .cpp file), and the reference's RenderPixel (path_tracing.cpp:34)
//    is called per camera sample exactly as Renderer::DrawFrame does
//    (renderer.h:97-116), but with one sampler per thread seeded per pixel, which makes
//    the oracle deterministic and removes the reference's shared-sampler data race.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <exception>
#include <filesystem>
#include <fstream>
#include <functional>
#include <future>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <optional>
#include <queue>
#include <random>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <type_traits>
#include <typeinfo>
#include <unordered_map>
#include <utility>
#include <vector>

#include <glm/vec2.hpp>
#include <glm/vec3.hpp>
#include <glm/vec4.hpp>
#include <glm/mat4x4.hpp>
#include <glm/gtx/transform.hpp>
#include <glm/gtc/matrix_transform.hpp>
#include <spdlog/spdlog.h>
#include <nlohmann/json.hpp>
#include <thread_pool.hpp>
#include <tiny_obj_loader.h>

#define private public
#define protected public
#include <engine/create/scene_loader.h>
#include <engine/create/post_process.h>
#include <renderer/path_tracing.cpp>
#include <geometry/triangle.h>
#include <engine/core/fresnel.h>
#include <material/disney.h>
#include <material/disney.cpp>
#undef private
#undef protected

namespace fe = fumeng::engine;
using fe::real;
using fe::vec2;
using fe::vec3;

// The reference's link-time gap: SceneLoader::ParsePostProcess calls CreateOidnDenoise
// unconditionally (scene_loader.h:269-270) but its only definition is compiled under
// USE_EMBREE (src/post/oidn_denoise.cpp:1).  OIDN is not installed here, so the stub
// returns a post-process that leaves the image unchanged.
namespace fumeng::engine {
class FmrefNoDenoise : public PostProcess {
public:
    void Process(RenderTarget&) override {}
};
SP<PostProcess> CreateOidnDenoise() { return MakeSP<FmrefNoDenoise>(); }
}  // namespace fumeng::engine

namespace {

thread_local std::string g_error;

// ---- per-vertex Disney parameters ---------------------------------------------------
//
// A scene-file extension the reference's loader cannot express: a triangle-mesh entry
// may carry "fm_vertex_attributes": {"path": <raw float32 V x dim file>, "dim": dim},
// giving each vertex basecolor r, g, b, roughness, metallic, clearcoat (at the offset
// its Disney material's "vertex_attributes" names).  The harness registers, under that
// material's name, a Material that interpolates the hit triangle's vertex values with
// barycentrics recovered from the hit position and builds the reference's own
// DisneyBSDF from them; the material's other parameters come from its JSON entry,
// parsed and sampled by the reference's DisneyConfig and textures.
struct VertexTri {
    fe::vec3 p[3];
    double a[3][6];
};

class VertexDisneyMaterial : public fe::Material {
public:
    const std::unordered_map<const fe::RenderObject*, VertexTri>* tris = nullptr;
    fe::SP<fe::Texture> specular, specularTint, anisotropic, sheen, sheenTint, clearcoatGloss, specTrans,
        specTransRoughness, diffTrans, flatness, ior;
    bool thin = false;

    explicit VertexDisneyMaterial(const fe::DisneyConfig& c)
    {
        specular = fe::CreateTexture(c.specular);
        specularTint = fe::CreateTexture(c.specularTint);
        anisotropic = fe::CreateTexture(c.anisotropic);
        sheen = fe::CreateTexture(c.sheen);
        sheenTint = fe::CreateTexture(c.sheenTint);
        clearcoatGloss = fe::CreateTexture(c.clearcoatGloss);
        specTrans = fe::CreateTexture(c.specTrans);
        specTransRoughness = fe::CreateTexture(c.specTransRoughness);
        diffTrans = fe::CreateTexture(c.diffTrans);
        flatness = fe::CreateTexture(c.flatness);
        ior = fe::CreateTexture(c.ior);
        thin = c.thin;
    }

    void CreateBSDF(fe::HitPoint& hp) const override
    {
        const VertexTri& t = tris->at(hp.object);
        // barycentrics of hp.pos in the triangle (least squares in the triangle's plane)
        const fe::vec3 e1 = t.p[1] - t.p[0], e2 = t.p[2] - t.p[0], q = hp.pos - t.p[0];
        const double d11 = glm::dot(e1, e1), d12 = glm::dot(e1, e2), d22 = glm::dot(e2, e2);
        const double q1 = glm::dot(q, e1), q2 = glm::dot(q, e2);
        const double den = d11 * d22 - d12 * d12;
        const double b1 = den != 0.0 ? (d22 * q1 - d12 * q2) / den : 0.0;
        const double b2 = den != 0.0 ? (d11 * q2 - d12 * q1) / den : 0.0;
        const double b0 = 1.0 - b1 - b2;
        double v[6];
        for (int k = 0; k < 6; ++k) v[k] = b0 * t.a[0][k] + b1 * t.a[1][k] + b2 * t.a[2][k];
        const vec2 uv = hp.uv;
        hp.bsdf = fe::MakeSP<fe::DisneyBSDF>(hp, vec3(real(v[0]), real(v[1]), real(v[2])), real(v[4]),
                                             specular->Sample(uv).x, specularTint->Sample(uv).x, real(v[3]),
                                             anisotropic->Sample(uv).x, sheen->Sample(uv).x, sheenTint->Sample(uv).x,
                                             real(v[5]), clearcoatGloss->Sample(uv).x, specTrans->Sample(uv).x,
                                             specTransRoughness->Sample(uv).x, diffTrans->Sample(uv).x,
                                             flatness->Sample(uv).x, ior->Sample(uv).x, thin);
    }
};

// Triangles of an OBJ written by the scene generator ("v x y z" lines and triangular
// "f" lines whose first index of each corner is the vertex): positions and indices.
// Parsed with C stdio (the Python process that loads this library may carry an older
// C++ runtime than the one this file was compiled against).
void read_obj_triangles(const std::string& path, std::vector<fe::vec3>& verts, std::vector<std::array<int, 3>>& faces)
{
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) throw std::runtime_error("cannot open " + path);
    char line[512];
    while (std::fgets(line, sizeof(line), f)) {
        if (line[0] == 'v' && line[1] == ' ') {
            double x = 0, y = 0, z = 0;
            if (std::sscanf(line + 2, "%lf %lf %lf", &x, &y, &z) == 3) verts.emplace_back(real(x), real(y), real(z));
        } else if (line[0] == 'f' && line[1] == ' ') {
            std::array<int, 3> tri{};
            char* p = line + 2;
            for (int k = 0; k < 3; ++k) {
                char* end = nullptr;
                tri[k] = int(std::strtol(p, &end, 10)) - 1;
                p = end;
                while (*p && *p != ' ' && *p != '\t' && *p != '\n') ++p;   // skip "/vt/vn"
            }
            faces.push_back(tri);
        }
    }
    std::fclose(f);
}

struct RefScene {
    fe::SceneLoader loader;
    std::unordered_map<const fe::RenderObject*, int> obj_index;
    std::unordered_map<const fe::RenderObject*, VertexTri> vertex_tris;
    fe::PathTracerConfig pt_config;
    int width = 1, height = 1, spp = 1;
};

vec3 json_vec3(const nlohmann::json& j, const char* key, vec3 dflt)
{
    if (!j.contains(key)) return dflt;
    auto v = j.at(key).get<std::vector<double>>();
    if (v.empty()) return dflt;
    if (v.size() < 3) return vec3(real(v[0]));
    return vec3(real(v[0]), real(v[1]), real(v[2]));
}

uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

template <typename F>
void parallel_for(int64_t n, int nthreads, F&& fn)
{
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::atomic<int64_t> next{0};
    const int64_t chunk = std::max<int64_t>(1, n / (int64_t(nthreads) * 16));
    auto worker = [&]() {
        for (;;) {
            const int64_t b = next.fetch_add(chunk);
            if (b >= n) break;
            const int64_t e = std::min(n, b + chunk);
            for (int64_t i = b; i < e; ++i) fn(i);
        }
    };
    std::vector<std::thread> ts;
    for (int t = 1; t < nthreads; ++t) ts.emplace_back(worker);
    worker();
    for (auto& t : ts) t.join();
}

fe::Ray make_ray(const double* r8)
{
    return fe::Ray(vec3(real(r8[0]), real(r8[1]), real(r8[2])),
                   vec3(real(r8[4]), real(r8[5]), real(r8[6])), real(r8[3]), real(r8[7]));
}

}  // namespace

extern "C" {

const char* fmref_last_error() { return g_error.c_str(); }

int fmref_precision() { return int(sizeof(real)); }

// triangle_func::GetMaxAxis (triangle.cpp:13-18) as compiled here; its unqualified
// `abs` decides which direction component the watertight test treats as the main axis.
int fmref_get_max_axis(double x, double y, double z)
{
    return fe::triangle_func::GetMaxAxis(vec3(real(x), real(y), real(z)));
}

// triangle_func::IntersectTriangle (triangle.cpp:25-94) on one ray and one triangle.
// ray8 = ox,oy,oz,tmin, dx,dy,dz,tmax ; v9 = v0,v1,v2.  Returns 1 on hit.
int fmref_intersect_triangle(const double* ray8, const double* v9, double* t_out, double* bc_out)
{
    const fe::Ray r = make_ray(ray8);
    vec3 bc;
    real t = 0;
    const bool hit = fe::triangle_func::IntersectTriangle(
        r, vec3(real(v9[0]), real(v9[1]), real(v9[2])), vec3(real(v9[3]), real(v9[4]), real(v9[5])),
        vec3(real(v9[6]), real(v9[7]), real(v9[8])), bc, t);
    if (t_out) *t_out = double(t);
    if (bc_out && hit) {
        bc_out[0] = bc.x;
        bc_out[1] = bc.y;
        bc_out[2] = bc.z;
    }
    return hit ? 1 : 0;
}

void* fmref_load(const char* json_path)
{
    try {
        auto s = std::make_unique<RefScene>();
        auto& L = s->loader;
        const std::filesystem::path p = std::filesystem::absolute(json_path);
        // SceneLoader::Load (scene_loader.h:293-302), with the material pre-insertion.
        L.m_scene_root = p.parent_path().string() + '/';
        std::ifstream ifs(p.string());
        if (!ifs) throw std::runtime_error("cannot open scene file");
        L.m_config = nlohmann::json::parse(ifs);
        L.ParseCamera();
        L.ParseRender();
        if (L.m_config.contains("scene") && L.m_config["scene"].contains("materials")) {
            for (auto& m : L.m_config["scene"]["materials"]) {
                if (m.value("type", std::string()) != "specular_reflection") continue;
                const std::string name = m.value("name", std::string());
                const vec3 color = json_vec3(m, "color", fe::white);
                const vec3 eta_i = json_vec3(m, "eta_i", fe::white);
                const vec3 eta_t = json_vec3(m, "eta_t", fe::white);
                const vec3 k = json_vec3(m, "k", fe::black);
                L.m_materials.emplace(name, fe::CreateSpecularReflection(color, eta_i, eta_t, k));
            }
        }
        // per-vertex Disney materials, registered before the loader builds its own
        std::map<std::string, std::pair<fe::SP<VertexDisneyMaterial>, int>> vmats;   // name -> (material, offset)
        if (L.m_config.contains("scene") && L.m_config["scene"].contains("materials")) {
            for (auto& m : L.m_config["scene"]["materials"]) {
                if (m.value("type", std::string()) != "disney" || !m.contains("vertex_attributes")) continue;
                fe::DisneyConfig dc;
                dc.Load(m);
                auto vm = std::make_shared<VertexDisneyMaterial>(dc);
                vm->tris = &s->vertex_tris;
                const std::string name = m.value("name", std::string());
                vmats[name] = {vm, m["vertex_attributes"].value("offset", 0)};
                L.m_materials.emplace(name, vm);
            }
        }
        L.ParseScene();
        L.ParsePostProcess();
        for (size_t i = 0; i < L.m_render_objects.size(); ++i)
            s->obj_index[L.m_render_objects[i].get()] = int(i);
        // vertex attributes of the triangles of meshes that carry them: render objects
        // follow the scene file's entries in order, one per triangle of a mesh
        if (!vmats.empty()) {
            size_t obj = 0;
            for (auto& e : L.m_config["scene"]["render_objects"]) {
                const auto& shape = e["shape"];
                const std::string type = shape.value("type", std::string());
                if (type != "triangle_mesh") {
                    ++obj;
                    continue;
                }
                std::vector<fe::vec3> verts;
                std::vector<std::array<int, 3>> faces;
                read_obj_triangles(L.m_scene_root + shape.value("path", std::string()), verts, faces);
                if (e.contains("fm_vertex_attributes") && vmats.count(e.value("material", std::string()))) {
                    const auto& va = e["fm_vertex_attributes"];
                    const int dim = va.value("dim", 6);
                    const int off = vmats[e.value("material", std::string())].second;
                    std::vector<float> attr(verts.size() * size_t(dim));
                    FILE* af = std::fopen((L.m_scene_root + va.value("path", std::string())).c_str(), "rb");
                    const size_t got = af ? std::fread(attr.data(), sizeof(float), attr.size(), af) : 0;
                    if (af) std::fclose(af);
                    if (got != attr.size()) throw std::runtime_error("short vertex attribute file");
                    for (size_t f = 0; f < faces.size(); ++f) {
                        VertexTri t;
                        for (int k = 0; k < 3; ++k) {
                            t.p[k] = verts[size_t(faces[f][k])];
                            for (int q = 0; q < 6; ++q) t.a[k][q] = attr[size_t(faces[f][k]) * dim + off + q];
                        }
                        s->vertex_tris[L.m_render_objects.at(obj + f).get()] = t;
                    }
                }
                obj += faces.size();
            }
            if (obj != L.m_render_objects.size()) throw std::runtime_error("vertex attributes: object count mismatch");
        }
        fe::RendererConfig::SetRootPath(L.m_scene_root);
        s->pt_config.Load(L.m_config["renderer"]);
        s->width = s->pt_config.width;
        s->height = s->pt_config.height;
        s->spp = s->pt_config.spp;
        return s.release();
    } catch (const std::exception& e) {
        g_error = e.what();
        return nullptr;
    } catch (...) {
        g_error = "unknown error";
        return nullptr;
    }
}

void fmref_free(void* h) { delete static_cast<RefScene*>(h); }

int64_t fmref_num_objects(void* h) { return int64_t(static_cast<RefScene*>(h)->loader.m_render_objects.size()); }

void fmref_image_size(void* h, int* w, int* hh, int* spp)
{
    auto* s = static_cast<RefScene*>(h);
    *w = s->width;
    *hh = s->height;
    *spp = s->spp;
}

// Scene::GetIntersect -> BVHAggregate::GetIntersect (bvh_aggregate.cpp:167-176) per ray.
// rays: n x 8 (ox,oy,oz,tmin,dx,dy,dz,tmax).  obj: load-order object index or -1.
int fmref_trace_closest(void* h, const double* rays, int64_t n, int32_t* obj, double* t, int nthreads)
{
    auto* s = static_cast<RefScene*>(h);
    fe::Scene& scene = *s->loader.m_scene;
    parallel_for(n, nthreads, [&](int64_t i) {
        const fe::Ray r = make_ray(rays + 8 * i);
        fe::HitPoint hp;
        const bool hit = scene.GetIntersect(r, &hp);
        obj[i] = hit ? s->obj_index.at(hp.object) : -1;
        t[i] = hit ? double(hp.t) : std::numeric_limits<double>::infinity();
    });
    return 0;
}

// Scene::IsIntersect (bvh_aggregate.cpp:157-165) per ray; out[i] = 1 when occluded.
int fmref_trace_any(void* h, const double* rays, int64_t n, uint8_t* out, int nthreads)
{
    auto* s = static_cast<RefScene*>(h);
    fe::Scene& scene = *s->loader.m_scene;
    parallel_for(n, nthreads, [&](int64_t i) {
        out[i] = scene.IsIntersect(make_ray(rays + 8 * i)) ? 1 : 0;
    });
    return 0;
}

// Brute force over every render object (RenderObject::GetIntersect with a fresh hit
// record), returning the nearest and second-nearest hit distances of distinct objects.
// Used to exclude near-tie rays from the bit-exact hit-ID comparison.
int fmref_two_nearest(void* h, const double* rays, int64_t n, double* t1, double* t2, int nthreads)
{
    auto* s = static_cast<RefScene*>(h);
    const auto& objs = s->loader.m_render_objects;
    parallel_for(n, nthreads, [&](int64_t i) {
        const fe::Ray r = make_ray(rays + 8 * i);
        double a = std::numeric_limits<double>::infinity(), b = a;
        for (const auto& o : objs) {
            fe::HitPoint hp;
            if (!o->GetIntersect(r, &hp)) continue;
            const double tt = double(hp.t);
            if (tt < a) {
                b = a;
                a = tt;
            } else if (tt < b) {
                b = tt;
            }
        }
        t1[i] = a;
        t2[i] = b;
    });
    return 0;
}

// Camera::SampleRay (pin_hole_camera.cpp:50-56, thin_lens_camera.cpp:23-30).
// ndc, lens: n x 2 ; out: n x 6 (ori, dir).
int fmref_camera_rays(void* h, const double* ndc, const double* lens, int64_t n, double* out)
{
    auto* s = static_cast<RefScene*>(h);
    auto cam = s->loader.m_camera;
    for (int64_t i = 0; i < n; ++i) {
        const fe::Ray r = cam->SampleRay(vec2(real(ndc[2 * i]), real(ndc[2 * i + 1])),
                                         vec2(real(lens[2 * i]), real(lens[2 * i + 1])));
        out[6 * i + 0] = r.ori.x;
        out[6 * i + 1] = r.ori.y;
        out[6 * i + 2] = r.ori.z;
        out[6 * i + 3] = r.dir.x;
        out[6 * i + 4] = r.dir.y;
        out[6 * i + 5] = r.dir.z;
    }
    return 0;
}

// Per-pixel Monte-Carlo estimate with the reference's own sample loop
// (renderer.h:98-115) and integrator (path_tracing.cpp:34-117), over the image rows
// [y0, y0+h) and columns [x0, x0+w) (row 0 = top, as Image stores it).  Each pixel's
// mt19937_64 is seeded with splitmix64(seed ^ pixel); each thread owns a PathTracer.
// With stride > 1 only every stride-th pixel of the tile (in row-major tile order) is
// rendered.  Outputs (one row of 3 doubles per rendered pixel): per-pixel sums of color,
// color^2, albedo and normal over `spp` samples; when clamp > 0 also the sums of the
// sample colours limited per channel to clamp (min(c, clamp)) and of their squares.
int fmref_render(void* hnd, uint64_t seed, int x0, int y0, int w, int h, int spp, double* sum,
                 double* sumsq, double* albedo, double* normal, int nthreads, int stride, double clamp,
                 double* csum, double* csumsq)
{
    if (stride < 1) stride = 1;
    auto* s = static_cast<RefScene*>(hnd);
    fe::Scene& scene = *s->loader.m_scene;
    const int W = s->width, H = s->height;
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::shared_ptr<fe::PathTracer>> tracers(nthreads);
    for (auto& t : tracers) t = std::static_pointer_cast<fe::PathTracer>(fe::CreatePathTracer(s->pt_config));
    std::atomic<int64_t> next{0};
    const int64_t npix = (int64_t(w) * h + stride - 1) / stride;
    auto worker = [&](int tid) {
        fe::PathTracer& pt = *tracers[tid];
        const real res_x = real(W), res_y = real(H);
        for (;;) {
            const int64_t q = next.fetch_add(1);
            if (q >= npix) break;
            const int64_t tq = q * stride;
            const int row = y0 + int(tq / w), i = x0 + int(tq % w);
            const int j = H - 1 - row;
            pt.m_sampler.rng.seed(splitmix64(seed ^ (uint64_t(row) * uint64_t(W) + uint64_t(i))));
            pt.m_sampler.udis.reset();
            double c[3] = {0, 0, 0}, c2[3] = {0, 0, 0}, a[3] = {0, 0, 0}, nn[3] = {0, 0, 0};
            double cc[3] = {0, 0, 0}, cc2[3] = {0, 0, 0};
            for (int k = 0; k < spp; ++k) {
                const vec2 film_sample = pt.m_sampler.Get2D();
                const vec2 lens_sample = pt.m_sampler.Get2D();
                const real px = (i + film_sample.x) / res_x;
                const real py = (j + film_sample.y) / res_y;
                fe::Ray camera_ray = scene.GetCamera()->SampleRay({px, py}, lens_sample);
                const auto res = pt.RenderPixel(scene, camera_ray);
                for (int ch = 0; ch < 3; ++ch) {
                    const double v = double(res.color[ch]);
                    c[ch] += v;
                    c2[ch] += v * v;
                    if (clamp > 0.0) {
                        const double vc = v > clamp ? clamp : v;
                        cc[ch] += vc;
                        cc2[ch] += vc * vc;
                    }
                    a[ch] += double(res.albedo[ch]);
                    nn[ch] += double(res.normal[ch]);
                }
            }
            for (int ch = 0; ch < 3; ++ch) {
                sum[3 * q + ch] = c[ch];
                if (sumsq) sumsq[3 * q + ch] = c2[ch];
                if (albedo) albedo[3 * q + ch] = a[ch];
                if (normal) normal[3 * q + ch] = nn[ch];
                if (csum) csum[3 * q + ch] = cc[ch];
                if (csumsq) csumsq[3 * q + ch] = cc2[ch];
            }
        }
    };
    std::vector<std::thread> ts;
    for (int t = 1; t < nthreads; ++t) ts.emplace_back(worker, t);
    worker(0);
    for (auto& t : ts) t.join();
    return 0;
}

// The reference's own Renderer::DrawFrame (renderer.h:84-144) with its thread pool,
// shared sampler, 1 s progress polling, post-process chain and PNG writes.  Returns
// wall-clock seconds around the call.
double fmref_draw_frame(void* h)
{
    auto* s = static_cast<RefScene*>(h);
    const auto t0 = std::chrono::steady_clock::now();
    s->loader.DrawFrame();
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// The reference's PostProcess chain (create/post_process.h: ToneMapping with its lum,
// LinearToSrgb, SrgbToLinear) over a frame held in a RenderTarget, then the 8-bit values
// RenderTarget::save_to_file writes (Image::save_to_file -> RealToUInt8 per channel, of
// the colour, albedo and normal images; only the colour is post-processed).
// types: 0 tonemapping, 1 linear_to_srgb, 2 srgb_to_linear.  Images: h x w x 3.
int fmref_postprocess(const int* types, const double* lums, int nsteps, int w, int h, const double* rgb,
                      const double* alb, const double* nrm, uint8_t* rgb8, uint8_t* alb8, uint8_t* nrm8)
{
    try {
        fe::RenderTarget target;
        target.resize(size_t(w), size_t(h));
        const size_t npix = size_t(w) * size_t(h);
        for (size_t i = 0; i < npix; ++i) {
            target.m_color(i) = vec3(real(rgb[3 * i]), real(rgb[3 * i + 1]), real(rgb[3 * i + 2]));
            target.m_albedo(i) = vec3(real(alb[3 * i]), real(alb[3 * i + 1]), real(alb[3 * i + 2]));
            target.m_normal(i) = vec3(real(nrm[3 * i]), real(nrm[3 * i + 1]), real(nrm[3 * i + 2]));
        }
        for (int k = 0; k < nsteps; ++k) {
            fe::SP<fe::PostProcess> step;
            if (types[k] == 0) {
                fe::ToneMappingConfig cfg;
                cfg.lum = real(lums[k]);
                step = fe::CreateToneMapping(cfg);
            } else if (types[k] == 1) {
                step = fe::CreateLinearToSrgb();
            } else if (types[k] == 2) {
                step = fe::CreateSrgbToLinear();
            } else {
                return 1;
            }
            step->Process(target);
        }
        for (size_t i = 0; i < npix; ++i)
            for (int c = 0; c < 3; ++c) {
                rgb8[3 * i + c] = fe::RealToUInt8(target.m_color(i)[c]);
                alb8[3 * i + c] = fe::RealToUInt8(target.m_albedo(i)[c]);
                nrm8[3 * i + c] = fe::RealToUInt8(target.m_normal(i)[c]);
            }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

// Image::load_from_file (image.cpp:81-96) as the reference decodes textures and env maps.
// out (nullable): h x w x 3 doubles, row 0 = top.
int fmref_load_image(const char* path, int is_hdr, int* w, int* h, double* out)
{
    fe::Image img;
    img.load_from_file(path, is_hdr != 0);
    *w = int(img.width());
    *h = int(img.height());
    if (out) {
        for (size_t y = 0; y < img.height(); ++y)
            for (size_t x = 0; x < img.width(); ++x) {
                const vec3 v = static_cast<const fe::Image&>(img)(x, y);
                const size_t q = y * img.width() + x;
                out[3 * q] = v.x;
                out[3 * q + 1] = v.y;
                out[3 * q + 2] = v.z;
            }
    }
    return 0;
}

// Texture::Sample of an image texture (texture.h:109-115, image_texture.cpp:13-44).
int fmref_texture_sample(const char* path, const char* sampler, const char* wrap_u, const char* wrap_v,
                         const double* uv, int64_t n, double* out)
{
    try {
        fe::TextureDesc desc;
        desc.type = fe::TextureDesc::TextureType::IMAGE;
        auto cfg = fe::MakeUP<fe::ImageTextureConfig>(std::string(path));
        cfg->sampler = sampler;
        cfg->wrap_u = wrap_u;
        cfg->wrap_v = wrap_v;
        desc.config = std::move(cfg);
        auto tex = fe::CreateTexture(desc);
        for (int64_t i = 0; i < n; ++i) {
            const vec3 v = tex->Sample(vec2(real(uv[2 * i]), real(uv[2 * i + 1])));
            out[3 * i] = v.x;
            out[3 * i + 1] = v.y;
            out[3 * i + 2] = v.z;
        }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

// EnvLight of the loaded scene (env_light.cpp:38-61): pdf of directions (shading point
// to light, world space) as used by MisBSDF, and the light's own sampling.
int fmref_env_pdf(void* h, const double* dirs, int64_t n, double* pdf)
{
    auto* s = static_cast<RefScene*>(h);
    const fe::EnvLight* env = s->loader.m_scene->GetEnvLight();
    if (!env) {
        g_error = "scene has no env light";
        return -1;
    }
    for (int64_t i = 0; i < n; ++i)
        pdf[i] = env->Pdf(vec3(real(dirs[3 * i]), real(dirs[3 * i + 1]), real(dirs[3 * i + 2])));
    return 0;
}

// Env radiance seen along world directions `dirs` (what a miss along dir returns,
// path_tracing.cpp:48-52).
int fmref_env_radiance(void* h, const double* dirs, int64_t n, double* out)
{
    auto* s = static_cast<RefScene*>(h);
    const fe::EnvLight* env = s->loader.m_scene->GetEnvLight();
    if (!env) {
        g_error = "scene has no env light";
        return -1;
    }
    for (int64_t i = 0; i < n; ++i) {
        const vec3 d(real(dirs[3 * i]), real(dirs[3 * i + 1]), real(dirs[3 * i + 2]));
        const vec3 v = env->GetRadiance({}, {}, {}, -d);
        out[3 * i] = v.x;
        out[3 * i + 1] = v.y;
        out[3 * i + 2] = v.z;
    }
    return 0;
}

// EnvLight::Sample (env_light.cpp:38-44): out n x 4 (dir xyz, pdf).
int fmref_env_sample(void* h, const double* samples, int64_t n, double* out)
{
    auto* s = static_cast<RefScene*>(h);
    const fe::EnvLight* env = s->loader.m_scene->GetEnvLight();
    if (!env) {
        g_error = "scene has no env light";
        return -1;
    }
    fe::HitPoint hp;
    hp.pos = vec3(real(0));
    for (int64_t i = 0; i < n; ++i) {
        const auto info = env->Sample(hp, vec3(real(samples[3 * i]), real(samples[3 * i + 1]), real(samples[3 * i + 2])));
        out[4 * i] = info.wi_w.x;
        out[4 * i + 1] = info.wi_w.y;
        out[4 * i + 2] = info.wi_w.z;
        out[4 * i + 3] = info.pdf;
    }
    return 0;
}

// BSDF of a named material of the loaded scene at a synthetic hit point
// (material->CreateBSDF, bsdf.h:136-182, disney.cpp:359-579 ...).
// frame: ng(3) ns(3) ss(3) uv(2) wo_w(3) = 14 doubles.
// For each i: f(wo, wi[i]) -> f_out[3i..], pdf(wo, wi[i]) -> pdf_out[i],
// SampleBSDF(wo, samples[i]) -> smp_out[8i..] = f(3), wi_w(3), pdf, is_delta.
int fmref_bsdf(void* h, const char* material, const double* frame, int64_t n, const double* wi,
               const double* samples, double* f_out, double* pdf_out, double* smp_out)
{
    auto* s = static_cast<RefScene*>(h);
    auto it = s->loader.m_materials.find(material);
    if (it == s->loader.m_materials.end() || !it->second) {
        g_error = "unknown material";
        return -1;
    }
    fe::HitPoint hp;
    hp.ng = vec3(real(frame[0]), real(frame[1]), real(frame[2]));
    hp.ns = vec3(real(frame[3]), real(frame[4]), real(frame[5]));
    hp.ss = vec3(real(frame[6]), real(frame[7]), real(frame[8]));
    hp.uv = vec2(real(frame[9]), real(frame[10]));
    hp.wo_r_w = vec3(real(frame[11]), real(frame[12]), real(frame[13]));
    hp.pos = vec3(real(0));
    it->second->CreateBSDF(hp);
    for (int64_t i = 0; i < n; ++i) {
        if (wi) {
            const vec3 w(real(wi[3 * i]), real(wi[3 * i + 1]), real(wi[3 * i + 2]));
            const vec3 f = hp.bsdf->CalFunc(hp.wo_r_w, w);
            f_out[3 * i] = f.x;
            f_out[3 * i + 1] = f.y;
            f_out[3 * i + 2] = f.z;
            pdf_out[i] = hp.bsdf->Pdf(hp.wo_r_w, w);
        }
        if (samples) {
            const auto sm = hp.bsdf->SampleBSDF(
                hp.wo_r_w, vec3(real(samples[3 * i]), real(samples[3 * i + 1]), real(samples[3 * i + 2])));
            double* o = smp_out + 8 * i;
            o[0] = sm.f.x;
            o[1] = sm.f.y;
            o[2] = sm.f.z;
            o[3] = sm.wi_w.x;
            o[4] = sm.wi_w.y;
            o[5] = sm.wi_w.z;
            o[6] = sm.pdf;
            o[7] = sm.is_delta ? 1.0 : 0.0;
        }
    }
    return 0;
}

}  // extern "C"
