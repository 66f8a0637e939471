#include "fm_scene_loader.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <system_error>
#include <thread>

#include "fm_image_io.h"

extern "C" void fm_internal_set_error(fm_ctx* ctx, const char* msg);

namespace fmhost {

namespace {

void warn(const std::string& m) { std::fprintf(stderr, "[fumeng_b200] %s\n", m.c_str()); }

// Transform(translation, rotation, scale) (math/transform.cpp:17-25): T * Rz*Ry*Rx * S,
// rotation angles in degrees, as a row-major 4x4 in double.
struct Mat4 {
    double m[16];
};

Mat4 mul(const Mat4& a, const Mat4& b)
{
    Mat4 r;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s += a.m[4 * i + k] * b.m[4 * k + j];
            r.m[4 * i + j] = s;
        }
    return r;
}

Mat4 identity()
{
    Mat4 r{};
    r.m[0] = r.m[5] = r.m[10] = r.m[15] = 1.0;
    return r;
}

Mat4 rot(int axis, double deg)
{
    const double a = deg / 180.0 * 3.14159265354;
    const double c = std::cos(a), s = std::sin(a);
    Mat4 r = identity();
    const int i = (axis + 1) % 3, j = (axis + 2) % 3;
    r.m[4 * i + i] = c;
    r.m[4 * i + j] = -s;
    r.m[4 * j + i] = s;
    r.m[4 * j + j] = c;
    return r;
}

Mat4 trs(const float t[3], const float r[3], const float s[3])
{
    Mat4 T = identity();
    T.m[3] = t[0];
    T.m[7] = t[1];
    T.m[11] = t[2];
    Mat4 S = identity();
    S.m[0] = s[0];
    S.m[5] = s[1];
    S.m[10] = s[2];
    return mul(mul(mul(mul(T, rot(2, r[2])), rot(1, r[1])), rot(0, r[0])), S);
}

bool is_identity(const Mat4& a)
{
    const Mat4 i = identity();
    for (int k = 0; k < 16; ++k)
        if (a.m[k] != i.m[k]) return false;
    return true;
}

// Inverse-transpose of the upper 3x3 (for normals), row-major.
void normal_matrix(const Mat4& a, double n[9])
{
    const double* m = a.m;
    const double A = m[5] * m[10] - m[6] * m[9], B = m[6] * m[8] - m[4] * m[10], C = m[4] * m[9] - m[5] * m[8];
    const double det = m[0] * A + m[1] * B + m[2] * C;
    // cofactor matrix / det = inverse transpose
    n[0] = A / det;
    n[1] = B / det;
    n[2] = C / det;
    n[3] = (m[2] * m[9] - m[1] * m[10]) / det;
    n[4] = (m[0] * m[10] - m[2] * m[8]) / det;
    n[5] = (m[1] * m[8] - m[0] * m[9]) / det;
    n[6] = (m[1] * m[6] - m[2] * m[5]) / det;
    n[7] = (m[2] * m[4] - m[0] * m[6]) / det;
    n[8] = (m[0] * m[5] - m[1] * m[4]) / det;
}

void normalize_f(float* v)
{
    const float d = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2];
    const float inv = 1.0f / std::sqrt(d);
    v[0] *= inv;
    v[1] *= inv;
    v[2] *= inv;
}

// strtol(s, nullptr, 10) for the token characters [s, e): decimal digits with an
// optional sign are converted here, anything else by strtol itself.
long obj_long(const char* s, const char* e)
{
    const char* q = s;
    bool neg = false;
    if (q < e && (*q == '-' || *q == '+')) neg = *q++ == '-';
    long v = 0;
    int nd = 0;
    while (q < e && *q >= '0' && *q <= '9' && nd < 18) {
        v = 10 * v + (*q++ - '0');
        ++nd;
    }
    if (nd == 18 && q < e && *q >= '0' && *q <= '9') return std::strtol(s, nullptr, 10);
    return neg ? -v : v;
}

int obj_index(const char* s, const char* e, size_t count)
{
    if (s == e) return -1;
    const long i = obj_long(s, e);
    if (i > 0) return (int)(i - 1);
    if (i < 0) return (int)((long)count + i);
    return -1;
}

bool obj_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// Next whitespace-separated token of [p, e): returns its start and sets `end`; p is
// advanced past it (start == e when the line has no more tokens).
const char* obj_token(const char*& p, const char* e, const char*& end)
{
    while (p < e && obj_space(*p)) ++p;
    const char* t = p;
    while (p < e && !obj_space(*p)) ++p;
    end = p;
    return t;
}

// A token as a float: the value strtof gives for its characters (0 for a missing
// token).  std::from_chars converts plain decimal tokens (correctly rounded, as strtof);
// a token it does not take whole without error (a leading '+', hexadecimal, out of
// range, trailing characters) goes to strtof.  Lines are NUL-terminated in the buffer,
// so strtof cannot read past the line.
float obj_float(const char*& p, const char* e)
{
    const char* end;
    const char* t = obj_token(p, e, end);
    if (t == end) return 0.0f;
    float v = 0.0f;
    const auto r = std::from_chars(t, end, v, std::chars_format::general);
    if (r.ec == std::errc() && r.ptr == end) return v;
    return std::strtof(t, nullptr);
}

}  // namespace

// Wavefront OBJ (v / vt / vn / f); polygons are split into fans (0, k, k+1) in file order,
// one object per triangle (triangle.cpp:312-329).  The file is read whole and scanned in
// place (no per-line or per-token strings); numbers are converted with strtof / strtol
// on each whitespace-separated token, as a token-by-token reader would.
ObjData load_obj(const std::string& path)
{
    std::FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) throw std::runtime_error("Loading model failed: " + path);
    std::string buf;
    if (std::fseek(fp, 0, SEEK_END) == 0) {
        const long size = std::ftell(fp);
        if (size > 0) {
            buf.resize((size_t)size);
            std::rewind(fp);
            buf.resize(std::fread(&buf[0], 1, (size_t)size, fp));
        }
    }
    std::fclose(fp);
    ObjData o;
    // rough capacity from the file size (a vertex or face line is >= 20 bytes)
    o.v.reserve(buf.size() / 40 * 3);
    o.faces.reserve(buf.size() / 40);
    std::vector<ObjData::Corner> poly;
    char* p = buf.empty() ? nullptr : &buf[0];
    char* const end_all = p + buf.size();
    while (p && p < end_all) {
        char* nl = static_cast<char*>(std::memchr(p, '\n', (size_t)(end_all - p)));
        char* line_end = nl ? nl : end_all;
        const size_t len = (size_t)(line_end - p);
        if (nl) *nl = '\0';
        const char* q = p;
        p = nl ? nl + 1 : end_all;
        if (len < 2) continue;
        const char* e = q + len;
        const char* tag_end;
        const char* tag = obj_token(q, e, tag_end);
        const size_t tl = (size_t)(tag_end - tag);
        if (tl == 1 && tag[0] == 'v') {
            const float x = obj_float(q, e), y = obj_float(q, e), z = obj_float(q, e);
            o.v.push_back(x);
            o.v.push_back(y);
            o.v.push_back(z);
        } else if (tl == 2 && tag[0] == 'v' && tag[1] == 't') {
            const float u = obj_float(q, e), v = obj_float(q, e);
            o.vt.push_back(u);
            o.vt.push_back(v);
        } else if (tl == 2 && tag[0] == 'v' && tag[1] == 'n') {
            const float x = obj_float(q, e), y = obj_float(q, e), z = obj_float(q, e);
            o.vn.push_back(x);
            o.vn.push_back(y);
            o.vn.push_back(z);
        } else if (tl == 1 && tag[0] == 'f') {
            poly.clear();
            for (;;) {
                const char* te;
                const char* t = obj_token(q, e, te);
                if (t == te) break;
                ObjData::Corner c{-1, -1, -1};
                const char* s1 = static_cast<const char*>(std::memchr(t, '/', (size_t)(te - t)));
                if (!s1) {
                    c.v = obj_index(t, te, o.v.size() / 3);
                } else {
                    c.v = obj_index(t, s1, o.v.size() / 3);
                    const char* s2 = static_cast<const char*>(std::memchr(s1 + 1, '/', (size_t)(te - s1 - 1)));
                    if (!s2) {
                        c.vt = obj_index(s1 + 1, te, o.vt.size() / 2);
                    } else {
                        c.vt = obj_index(s1 + 1, s2, o.vt.size() / 2);
                        c.vn = obj_index(s2 + 1, te, o.vn.size() / 3);
                    }
                }
                if (c.v < 0 || (size_t)c.v >= o.v.size() / 3) throw std::runtime_error("bad OBJ vertex index: " + path);
                poly.push_back(c);
            }
            for (size_t k = 1; k + 1 < poly.size(); ++k) o.faces.push_back({poly[0], poly[k], poly[k + 1]});
        }
    }
    return o;
}

fm_scene_desc FlatScene::desc() const
{
    for (size_t i = 0; i < textures.size(); ++i) textures[i].texels = texels[i].data();
    fm_scene_desc d{};
    d.num_objects = (int64_t)obj_material.size();
    d.obj_material = obj_material.data();
    d.obj_emission = obj_emission.data();
    d.num_triangles = (int64_t)tri_object.size();
    d.tri_pos = tri_pos.data();
    d.tri_normal = any_normal ? tri_normal.data() : nullptr;
    d.tri_has_normal = any_normal ? tri_has_normal.data() : nullptr;
    d.tri_uv = any_uv ? tri_uv.data() : nullptr;
    d.tri_object = tri_object.data();
    d.tri_vattr = nullptr;
    d.vattr_dim = 0;
    d.num_rects = (int64_t)rect_object.size();
    d.rect_pts = rect_pts.data();
    d.rect_object = rect_object.data();
    d.num_spheres = (int64_t)sphere_object.size();
    d.sphere_radius = sphere_radius.data();
    d.sphere_xform = sphere_xform.data();
    d.sphere_object = sphere_object.data();
    d.num_materials = (int32_t)materials.size();
    d.materials = materials.data();
    d.num_textures = (int32_t)textures.size();
    d.textures = textures.data();
    d.num_lights = (int32_t)lights.size();
    d.lights = lights.data();
    d.tri_light_group = mesh_lights ? tri_light_group.data() : nullptr;
    return d;
}

int32_t SceneLoader::LoadTexture(const std::string& path, const std::string& sampler, const std::string& wrap_u,
                                 const std::string& wrap_v)
{
    const std::string key = path + "|" + sampler + "|" + wrap_u + "|" + wrap_v;
    auto it = m_texture_cache.find(key);
    if (it != m_texture_cache.end()) return it->second;
    // ImageTexture: ".hdr" anywhere in the path selects the HDR reader (image_texture.cpp:64)
    const bool is_hdr = path.find(".hdr") != std::string::npos;
    ImageF img = read_image(path, is_hdr);
    fm_texture_desc t{};
    t.width = img.width;
    t.height = img.height;
    t.wrap_u = wrap_u == "clamp" ? FM_WRAP_CLAMP : FM_WRAP_REPEAT;
    t.wrap_v = wrap_v == "clamp" ? FM_WRAP_CLAMP : FM_WRAP_REPEAT;
    if (wrap_u != "clamp" && wrap_u != "repeat") warn("invalid wrap type");
    if (wrap_v != "clamp" && wrap_v != "repeat") warn("invalid wrap type");
    t.filter = sampler == "nearest" ? FM_FILTER_NEAREST : FM_FILTER_LINEAR;
    if (sampler != "nearest" && sampler != "linear") warn("invalid sample type");
    m_flat.texels.push_back(std::move(img.rgb));
    m_flat.textures.push_back(t);
    const int32_t idx = (int32_t)m_flat.textures.size() - 1;
    m_texture_cache[key] = idx;
    return idx;
}

// TextureDesc::Load (core/config.cpp:6-23)
fm_tex_ref SceneLoader::ParseTexture(const Json& j, float dflt[3])
{
    fm_tex_ref r{};
    r.texture = -1;
    r.value[0] = dflt[0];
    r.value[1] = dflt[1];
    r.value[2] = dflt[2];
    std::string type = "constant";
    load(j, "type", type);
    std::string wrap_u = "repeat", wrap_v = "repeat";
    load(j, "wrap_u", wrap_u);
    load(j, "wrap_v", wrap_v);
    if (type == "constant") {
        r.value[0] = r.value[1] = r.value[2] = 0.0f;   // ConstantTextureConfig default: black
        load_vec3(j, "value", r.value);
    } else if (type == "image") {
        std::string path, sampler = "linear";
        load(j, "path", path);
        load(j, "sampler", sampler);
        r.texture = LoadTexture(m_root + path, sampler, wrap_u, wrap_v);
    } else {
        throw std::runtime_error("texture type not support.");
    }
    return r;
}

void SceneLoader::ParseCamera(const Json& root)
{
    const Json* c = root.find("camera");
    if (!c) throw std::runtime_error("Camera is not specified.");
    std::string type = "pin_hole";
    load(*c, "type", type);
    if (type != "pin_hole" && type != "thin_lens") throw std::runtime_error("Camera is not specified.");
    fm_camera& cam = m_camera;
    cam.type = type == "thin_lens" ? FM_CAMERA_THIN_LENS : FM_CAMERA_PINHOLE;
    for (int k = 0; k < 3; ++k) {
        cam.pos[k] = 0.0f;
        cam.look_at[k] = 0.0f;
        cam.up[k] = k == 2 ? 1.0f : 0.0f;
    }
    cam.fov = 60.0f;
    cam.aspect = 1.0f;
    cam.focal_distance = 1.0f;
    cam.lens_radius = 0.0f;
    load_vec3(*c, "pos", cam.pos);
    load_vec3(*c, "look_at", cam.look_at);
    load_vec3(*c, "up", cam.up);
    load(*c, "fov", cam.fov);
    load(*c, "aspect", cam.aspect);
    load(*c, "focal_distance", cam.focal_distance);
    if (cam.type == FM_CAMERA_THIN_LENS) {
        if (!c->has("lens_radius")) warn("thin_lens camera without lens_radius: using 0");
        load(*c, "lens_radius", cam.lens_radius);
    }
}

void SceneLoader::ParseRender(const Json& root)
{
    const Json* c = root.find("renderer");
    std::string type = "path_tracer";
    if (c) load(*c, "type", type);
    if (!c || type != "path_tracer") throw std::runtime_error("Renderer is not specified.");
    fm_render_params& p = m_params;
    p.width = 1;
    p.height = 1;
    p.spp = 10;
    p.depth = 10;
    p.direct_loop = 1;
    p.rr_depth = 10;
    p.rr_coef = 0.85f;
    p.seed = 0;
    p.mode = FM_MODE_WAVEFRONT;
    p.sample_offset = 0;
    int thread_count = 8;
    load(*c, "width", p.width);
    load(*c, "height", p.height);
    load(*c, "spp", p.spp);
    load(*c, "thread_count", thread_count);
    m_output = "result";
    load(*c, "output", m_output);
    m_output = m_root + m_output;
    load(*c, "depth", p.depth);
    load(*c, "direct_loop", p.direct_loop);
    load(*c, "rr_depth", p.rr_depth);
    load(*c, "rr_coef", p.rr_coef);
    std::string mode = "wavefront";
    load(*c, "mode", mode);
    p.mode = mode == "megakernel" ? FM_MODE_MEGAKERNEL : FM_MODE_WAVEFRONT;
    double seed = 0.0;
    load(*c, "seed", seed);
    p.seed = (uint64_t)seed;
}

void SceneLoader::ParseMaterial(const Json& j)
{
    std::string type, name;
    load(j, "type", type);
    load(j, "name", name);
    if (m_material_index.count(name)) return;   // the first definition wins (map::emplace)
    fm_material_desc m{};
    m.vattr_offset = -1;
    fm_tex_ref* refs = &m.basecolor;
    float zero[3] = {0, 0, 0};
    for (int k = 0; k < 15; ++k) {
        refs[k].texture = -1;
        refs[k].value[0] = refs[k].value[1] = refs[k].value[2] = 0.0f;
    }
    auto tex = [&](const char* key, fm_tex_ref& r, float d0) {
        float d[3] = {d0, d0, d0};
        r.texture = -1;
        r.value[0] = r.value[1] = r.value[2] = d0;
        if (const Json* f = j.find(key)) r = ParseTexture(*f, d);
    };
    if (type == "lambert_diffuse") {
        m.type = FM_MAT_LAMBERT;
        tex("basecolor", m.basecolor, 1.0f);
    } else if (type == "disney") {
        m.type = FM_MAT_DISNEY;
        tex("basecolor", m.basecolor, 0.0f);
        tex("metallic", m.metallic, 0.0f);
        tex("specular", m.specular, 0.5f);
        tex("specularTint", m.specular_tint, 0.0f);
        tex("roughness", m.roughness, 0.0f);
        tex("anisotropic", m.anisotropic, 0.0f);
        tex("sheen", m.sheen, 0.0f);
        tex("sheenTint", m.sheen_tint, 0.0f);
        tex("clearcoat", m.clearcoat, 0.0f);
        tex("clearcoatGloss", m.clearcoat_gloss, 0.0f);
        tex("specTrans", m.spec_trans, 0.0f);
        tex("specTransRoughness", m.spec_trans_roughness, 0.0f);
        tex("diffTrans", m.diff_trans, 0.0f);
        tex("flatness", m.flatness, 0.0f);
        tex("ior", m.ior, 1.5f);
        bool thin = false;
        load(j, "thin", thin);
        m.thin = thin ? 1 : 0;
    } else if (type == "specular_transmission") {
        m.type = FM_MAT_SPEC_TRANS;
        for (int k = 0; k < 3; ++k) m.reflect_color[k] = m.refract_color[k] = 1.0f;
        load_vec3(j, "reflect_color", m.reflect_color);
        load_vec3(j, "refract_color", m.refract_color);
        m.eta_i = 1.0f;
        m.eta_t = 1.5f;
        if (!j.has("eta_i") || !j.has("eta_t")) warn("specular_transmission without eta_i/eta_t: using 1 / 1.5");
        load(j, "eta_i", m.eta_i);
        load(j, "eta_t", m.eta_t);
    } else if (type == "specular_reflection") {
        m.type = FM_MAT_SPEC_REFL;
        for (int k = 0; k < 3; ++k) {
            m.color[k] = 1.0f;
            m.cond_eta_i[k] = 1.0f;
            m.cond_eta_t[k] = 1.0f;
            m.cond_k[k] = 0.0f;
        }
        load_vec3(j, "color", m.color);
        load_vec3(j, "eta_i", m.cond_eta_i);
        load_vec3(j, "eta_t", m.cond_eta_t);
        load_vec3(j, "k", m.cond_k);
    } else {
        throw std::runtime_error("Material type not supported: " + type);
    }
    (void)zero;
    m_material_index[name] = (int32_t)m_flat.materials.size();
    m_flat.materials.push_back(m);
}

void SceneLoader::PreloadMeshes(const Json& objs)
{
    // the paths as ParseRenderObject reads them; an object whose fields do not parse is
    // left to ParseRenderObject, which reports it in order
    std::vector<std::string> paths;
    for (const auto& o : objs.arr) {
        try {
            const Json* sh = o.find("shape");
            if (!sh) continue;
            std::string type, path;
            load(*sh, "type", type);
            if (type != "triangle_mesh") continue;
            load(*sh, "path", path);
            auto ins = m_meshes.emplace(m_root + path, PreloadedMesh{});
            if (ins.second) paths.push_back(m_root + path);
            ++ins.first->second.uses;
        } catch (const std::exception&) {
        }
    }
    if (paths.empty()) return;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nthreads = std::min<size_t>(std::min<size_t>(paths.size(), hw), 16);
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t i = next++; i < paths.size(); i = next++) {
            PreloadedMesh& m = m_meshes.at(paths[i]);
            try {
                m.data = load_obj(paths[i]);
            } catch (...) {
                m.error = std::current_exception();
            }
        }
    };
    std::vector<std::thread> pool;
    try {
        for (size_t t = 1; t < nthreads; ++t) pool.emplace_back(work);
    } catch (const std::system_error&) {
        // no more threads: the ones started and this thread share the files
    }
    work();
    for (auto& t : pool) t.join();
}

void SceneLoader::release_mesh(const std::string& path)
{
    // a mesh's parsed file is dropped once the last object that names it is flattened,
    // so that peak host memory stays near one copy of the scene's geometry
    auto it = m_meshes.find(path);
    if (it != m_meshes.end() && --it->second.uses <= 0) m_meshes.erase(it);
}

const ObjData& SceneLoader::mesh_data(const std::string& path)
{
    auto it = m_meshes.find(path);
    if (it == m_meshes.end()) {
        PreloadedMesh m;
        m.data = load_obj(path);
        it = m_meshes.emplace(path, std::move(m)).first;
    }
    if (it->second.error) std::rethrow_exception(it->second.error);
    return it->second.data;
}

void SceneLoader::ParseRenderObject(const Json& j)
{
    float em[3] = {0, 0, 0};
    load_vec3(j, "emittance", em);
    std::string mat = "default_material";
    load(j, "material", mat);
    auto it = m_material_index.find(mat);
    if (it == m_material_index.end()) {
        warn("Fail to find material " + mat + ", use default lambert.");
        it = m_material_index.find("default_material");
    }
    const int32_t mi = it->second;
    FlatScene& F = m_flat;
    auto add_object = [&]() {
        const int32_t o = (int32_t)F.obj_material.size();
        F.obj_material.push_back(mi);
        F.obj_emission.insert(F.obj_emission.end(), em, em + 3);
        return o;
    };
    const Json* sh = j.find("shape");
    if (!sh) return;
    std::string type;
    load(*sh, "type", type);
    float t[3] = {0, 0, 0}, r[3] = {0, 0, 0}, s[3] = {1, 1, 1};
    if (type == "triangle_mesh") {
        std::string path;
        load(*sh, "path", path);
        load_vec3(*sh, "translation", t);
        load_vec3(*sh, "rotation", r);
        load_vec3(*sh, "scale", s);
        const Mat4 M = trs(t, r, s);
        const bool ident = is_identity(M);
        double N[9];
        normal_matrix(M, N);
        const ObjData& obj = mesh_data(m_root + path);
        // room for this mesh, growing geometrically across the scene's meshes
        auto grow = [](auto& vec, size_t add) {
            if (vec.capacity() < vec.size() + add) vec.reserve(std::max(vec.size() + add, 2 * vec.capacity()));
        };
        const size_t nf = obj.faces.size();
        grow(F.tri_object, nf);
        grow(F.tri_pos, 9 * nf);
        grow(F.tri_has_normal, nf);
        grow(F.tri_normal, 9 * nf);
        grow(F.tri_uv, 6 * nf);
        if (F.mesh_lights) F.tri_light_group.insert(F.tri_light_group.end(), nf, F.num_meshes);
        ++F.num_meshes;
        for (const auto& f : obj.faces) {
            const int32_t o = add_object();
            F.tri_object.push_back(o);
            bool hn = true, huv = false;
            for (int c = 0; c < 3; ++c) {
                const float* v = &obj.v[3 * (size_t)f[c].v];
                if (ident) {
                    F.tri_pos.insert(F.tri_pos.end(), v, v + 3);
                } else {
                    for (int row = 0; row < 3; ++row)
                        F.tri_pos.push_back((float)(M.m[4 * row] * v[0] + M.m[4 * row + 1] * v[1] +
                                                    M.m[4 * row + 2] * v[2] + M.m[4 * row + 3]));
                }
                hn = hn && f[c].vn >= 0 && (size_t)f[c].vn < obj.vn.size() / 3;
                huv = huv || f[c].vt >= 0;
            }
            F.tri_has_normal.push_back(hn ? 1 : 0);
            for (int c = 0; c < 3; ++c) {
                float n[3] = {0, 0, 0};
                if (hn) {
                    const float* q = &obj.vn[3 * (size_t)f[c].vn];
                    for (int row = 0; row < 3; ++row)
                        n[row] = (float)(N[3 * row] * q[0] + N[3 * row + 1] * q[1] + N[3 * row + 2] * q[2]);
                    normalize_f(n);
                    F.any_normal = true;
                }
                F.tri_normal.insert(F.tri_normal.end(), n, n + 3);
                // GetUVFromMesh (triangle.cpp:148-156): (u, 1 - v), or (0, 0) without texcoords
                float uv[2] = {0.0f, 0.0f};
                if (f[c].vt >= 0 && (size_t)f[c].vt < obj.vt.size() / 2) {
                    uv[0] = obj.vt[2 * (size_t)f[c].vt];
                    uv[1] = 1.0f - obj.vt[2 * (size_t)f[c].vt + 1];
                    F.any_uv = true;
                }
                F.tri_uv.insert(F.tri_uv.end(), uv, uv + 2);
            }
            (void)huv;
        }
        release_mesh(m_root + path);
    } else if (type == "sphere") {
        float radius = 1.0f;
        load(*sh, "radius", radius);
        load_vec3(*sh, "translation", t);
        load_vec3(*sh, "rotation", r);
        load_vec3(*sh, "scale", s);
        const Mat4 M = trs(t, r, s);
        const int32_t o = add_object();
        F.sphere_object.push_back(o);
        F.sphere_radius.push_back(radius);
        for (int k = 0; k < 16; ++k) F.sphere_xform.push_back((float)M.m[k]);
    } else if (type == "rectangle") {
        float pts[12] = {0};
        load_vec3(*sh, "pa", pts);
        load_vec3(*sh, "pb", pts + 3);
        load_vec3(*sh, "pc", pts + 6);
        load_vec3(*sh, "pd", pts + 9);
        const int32_t o = add_object();
        F.rect_object.push_back(o);
        F.rect_pts.insert(F.rect_pts.end(), pts, pts + 12);
    } else {
        warn("Shape type not supported: " + type + ".");
    }
}

void SceneLoader::ParseLight(const Json& j)
{
    std::string type;
    load(j, "type", type);
    fm_light_desc l{};
    if (type == "env") {
        std::string path;
        load(j, "path", path);
        if (path.empty()) return;
        l.type = FM_LIGHT_ENV;
        l.texture = LoadTexture(m_root + path, "linear", "repeat", "repeat");
        load_vec3(j, "rotation", l.rotation);
        l.factor = 1.0f;
        load(j, "factor", l.factor);
        m_flat.lights.push_back(l);
    } else if (type == "directional") {
        l.type = FM_LIGHT_DIRECTIONAL;
        float dir[3] = {1.0f, 0.0f, 0.0f};
        load_vec3(j, "radiance", l.radiance);
        load_vec3(j, "direction", dir);
        normalize_f(dir);
        std::memcpy(l.direction, dir, sizeof(dir));
        m_flat.lights.push_back(l);
    } else {
        warn("Light type not supported: " + type + ".");
    }
}

void SceneLoader::ParseScene(const Json& root)
{
    const Json* c = root.find("scene");
    if (!c) throw std::runtime_error("Scene is not specified.");
    if (const Json* acc = c->find("accelerator")) {
        std::string t = "bvh";
        load(*acc, "type", t);
        if (t == "embree") {
            warn("accelerator 'embree': the device BVH is used; each emissive mesh is one light sampled by area, "
                 "as the reference's Embree meshes are");
            m_flat.mesh_lights = true;
        }
    }
    if (const Json* mats = c->find("materials"))
        for (const auto& m : mats->arr) ParseMaterial(m);
    if (!m_material_index.count("default_material")) {
        fm_material_desc m{};
        m.type = FM_MAT_LAMBERT;
        m.vattr_offset = -1;
        fm_tex_ref* refs = &m.basecolor;
        for (int k = 0; k < 15; ++k) refs[k].texture = -1;
        m.basecolor.value[0] = m.basecolor.value[1] = m.basecolor.value[2] = 1.0f;
        m_material_index["default_material"] = (int32_t)m_flat.materials.size();
        m_flat.materials.push_back(m);
    }
    if (const Json* objs = c->find("render_objects")) {
        PreloadMeshes(*objs);
        for (const auto& o : objs->arr) ParseRenderObject(o);
        m_meshes.clear();
    }
    if (const Json* ls = c->find("lights"))
        for (const auto& l : ls->arr) ParseLight(l);
}

void SceneLoader::ParsePostProcess(const Json& root)
{
    const Json* c = root.find("post_process");
    if (!c) return;
    for (const auto& p : c->arr) {
        PostStep s;
        load(p, "type", s.type);
        if (s.type == "tonemapping") {
            load(p, "lum", s.lum);
        } else if (s.type == "oidn_denoise") {
            warn("oidn_denoise: OIDN is not available; an edge-avoiding a-trous filter guided by the albedo and "
                 "normal images runs instead");
        } else if (s.type != "linear_to_srgb" && s.type != "srgb_to_linear") {
            warn("Post process type not supported: " + s.type + ".");
            continue;
        }
        m_post.push_back(s);
    }
}

void SceneLoader::Load(const std::string& path)
{
    const std::filesystem::path p = std::filesystem::absolute(path);
    m_root = p.parent_path().string() + '/';
    std::ifstream f(p);
    if (!f) throw std::runtime_error("cannot open scene file: " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    const Json root = Json::parse(ss.str());
    *this = SceneLoader{};
    m_root = p.parent_path().string() + '/';
    ParseCamera(root);
    ParseRender(root);
    ParseScene(root);
    ParsePostProcess(root);
}

fm_status SceneLoader::CreateScene(fm_ctx* ctx, fm_scene** out) const
{
    const fm_scene_desc d = m_flat.desc();
    return fm_scene_create(ctx, &d, out);
}

std::vector<fm_post_step> post_steps(const std::vector<PostStep>& steps)
{
    std::vector<fm_post_step> out;
    for (const auto& s : steps) {
        fm_post_step p{};
        p.lum = s.lum;
        if (s.type == "tonemapping")
            p.type = FM_POST_TONEMAP;
        else if (s.type == "linear_to_srgb")
            p.type = FM_POST_LINEAR_TO_SRGB;
        else if (s.type == "srgb_to_linear")
            p.type = FM_POST_SRGB_TO_LINEAR;
        else if (s.type == "oidn_denoise")
            p.type = FM_POST_DENOISE;
        else
            continue;
        out.push_back(p);
    }
    return out;
}

fm_status SceneLoader::DrawFrame(fm_ctx* ctx)
{
    fm_scene* scene = nullptr;
    fm_status st = CreateScene(ctx, &scene);
    if (st != FM_OK) return st;
    const size_t n = (size_t)m_params.width * m_params.height * 3;
    std::vector<float> rgb(n), alb(n), nrm(n);
    fm_render_stats stats{};
    st = fm_render(ctx, scene, &m_camera, &m_params, rgb.data(), alb.data(), nrm.data(), 0, &stats);
    fm_scene_destroy(ctx, scene);
    if (st != FM_OK) return st;
    std::fprintf(stderr, "[fumeng_b200] Current progress is : 1.00 (%lld paths in %.1f ms)\n", (long long)stats.paths,
                 stats.kernel_ms);
    // the post-process chain and the 8-bit conversion on the device (fm_postprocess),
    // then RenderTarget::save_to_file's three PNG files
    const std::vector<fm_post_step> steps = post_steps(m_post);
    std::vector<uint8_t> c8(n), a8(n), n8(n);
    st = fm_postprocess(ctx, m_params.width, m_params.height, steps.data(), (int32_t)steps.size(), rgb.data(),
                        alb.data(), nrm.data(), c8.data(), a8.data(), n8.data(), 0);
    if (st != FM_OK) return st;
    write_png_u8(m_output + ".png", m_params.width, m_params.height, c8.data());
    write_png_u8(m_output + "_albedo.png", m_params.width, m_params.height, a8.data());
    write_png_u8(m_output + "_normal.png", m_params.width, m_params.height, n8.data());
    return FM_OK;
}

}  // namespace fmhost

extern "C" {

fm_status fm_scene_load(fm_ctx* ctx, const char* json_path, fm_scene** out, fm_camera* camera,
                        fm_render_params* params)
{
    if (!json_path || (out && !ctx)) {
        fm_internal_set_error(ctx, "scene_load: null argument");
        return FM_ERR_INVALID;
    }
    try {
        fmhost::SceneLoader loader;
        loader.Load(json_path);
        if (camera) *camera = loader.camera();
        if (params) *params = loader.params();
        if (!out) return FM_OK;   // parse only
        return loader.CreateScene(ctx, out);
    } catch (const std::exception& e) {
        fm_internal_set_error(ctx, e.what());
        return FM_ERR_INVALID;
    }
}

fm_status fm_draw_frame(fm_ctx* ctx, const char* json_path)
{
    if (!ctx) return FM_ERR_INVALID;
    if (!json_path) {
        fm_internal_set_error(ctx, "draw_frame: null path");
        return FM_ERR_INVALID;
    }
    try {
        fmhost::SceneLoader loader;
        loader.Load(json_path);
        return loader.DrawFrame(ctx);
    } catch (const std::exception& e) {
        fm_internal_set_error(ctx, e.what());
        return FM_ERR_INVALID;
    }
}

}  // extern "C"
