// Scene loading and the drop-in integrator, with the reference's interface.
//
// SceneLoader mirrors fumeng::engine::SceneLoader (create/scene_loader.h:22-308): Load()
// reads the same JSON schema (camera, renderer, scene{accelerator, materials,
// render_objects, lights}, post_process) with the same defaults and field rules, and
// DrawFrame() renders through the CUDA library, runs the post-process chain and writes
// <output>.png, <output>_albedo.png and <output>_normal.png as RenderTarget::save_to_file
// does (core/render_target.h:26-31).
//
// Schema extensions (ignored by the reference, read here): material type
// "specular_reflection" {color, eta_i, eta_t, k}, and "renderer": {"mode":
// "wavefront"|"megakernel", "seed"}.
#pragma once
#include <array>
#include <exception>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fumeng_b200.h"
#include "fm_json.h"

namespace fmhost {

// Everything fm_scene_create needs, owned by host vectors.
struct FlatScene {
    std::vector<int32_t> obj_material;
    std::vector<float> obj_emission;
    std::vector<float> tri_pos, tri_normal, tri_uv;
    std::vector<uint8_t> tri_has_normal;
    std::vector<int32_t> tri_object;
    bool any_normal = false, any_uv = false;
    std::vector<float> rect_pts;
    std::vector<int32_t> rect_object;
    std::vector<float> sphere_radius, sphere_xform;
    std::vector<int32_t> sphere_object;
    std::vector<fm_material_desc> materials;
    std::vector<std::vector<float>> texels;
    mutable std::vector<fm_texture_desc> textures;   // texel pointers are set by desc()
    std::vector<fm_light_desc> lights;
    // "accelerator": "embree" -- each emissive mesh is one light sampled by area, as the
    // reference's Embree meshes are; tri_light_group holds each triangle's mesh ordinal
    bool mesh_lights = false;
    std::vector<int32_t> tri_light_group;
    int32_t num_meshes = 0;

    fm_scene_desc desc() const;
};

// The triangles of a Wavefront OBJ file: positions, texture coordinates and normals as
// read, and each face's corners (0-based indices, -1 where absent).
struct ObjData {
    std::vector<float> v, vt, vn;
    struct Corner {
        int v, vt, vn;
    };
    std::vector<std::array<Corner, 3>> faces;
};

// Reads an OBJ file (v, vt, vn, f; other lines ignored; polygons split into fans in file
// order).  Throws std::runtime_error on an unreadable file or a face whose vertex index
// is out of range.
ObjData load_obj(const std::string& path);

struct PostStep {
    std::string type;   // tonemapping | linear_to_srgb | srgb_to_linear | oidn_denoise
    float lum = 1.0f;
};

class SceneLoader {
public:
    // Parses the JSON file and everything it references.  Throws std::runtime_error
    // with the reference's messages where it throws ("Camera is not specified.", ...).
    void Load(const std::string& path);
    // Creates the device scene (requires Load).
    fm_status CreateScene(fm_ctx* ctx, fm_scene** out) const;
    // Renders, post-processes and writes the PNG outputs (requires Load).
    fm_status DrawFrame(fm_ctx* ctx);

    const FlatScene& flat() const { return m_flat; }
    const fm_camera& camera() const { return m_camera; }
    const fm_render_params& params() const { return m_params; }
    const std::string& output() const { return m_output; }

private:
    void ParseCamera(const Json& j);
    void ParseRender(const Json& j);
    void ParseScene(const Json& j);
    void ParseMaterial(const Json& j);
    void ParseRenderObject(const Json& j);
    void ParseLight(const Json& j);
    void ParsePostProcess(const Json& j);
    // Reads every OBJ file the render objects name, on several host threads, before the
    // objects are flattened in order (mesh_data hands the results out).
    void PreloadMeshes(const Json& objs);
    const ObjData& mesh_data(const std::string& path);
    void release_mesh(const std::string& path);
    fm_tex_ref ParseTexture(const Json& j, float dflt[3]);
    int32_t LoadTexture(const std::string& path, const std::string& sampler, const std::string& wrap_u,
                        const std::string& wrap_v);

    std::string m_root;
    fm_camera m_camera{};
    fm_render_params m_params{};
    std::string m_output = "result";
    FlatScene m_flat;
    std::map<std::string, int32_t> m_material_index;
    std::vector<PostStep> m_post;
    std::map<std::string, int32_t> m_texture_cache;
    struct PreloadedMesh {
        ObjData data;
        std::exception_ptr error;   // rethrown when the object that names the file is reached
        int uses = 0;               // render objects still to flatten that name this file
    };
    std::map<std::string, PreloadedMesh> m_meshes;
};

// Post-process chain on a float RGB image (post/tonemapping.cpp, post/*_srgb.cpp).
// The post-process chain as the C-ABI's steps (unknown types were dropped when parsed).
std::vector<fm_post_step> post_steps(const std::vector<PostStep>& steps);

}  // namespace fmhost
