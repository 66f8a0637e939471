// Device-side scene layout (one DevScene per scene; batches index an array of them).
//
// Primitive id space (used by the BVH leaves and hit records):
//   [0, T)            mesh triangles, in fm_scene_desc order
//   [T, T + 2R)       rectangle halves: prim T + 2r + h, h = 0 for (pa,pb,pc), 1 for
//                     (pc,pd,pa) (geometry/rectangle.cpp:38-56)
//   [T + 2R, +S)      spheres
#pragma once
#include "fm_common.cuh"

namespace fm {

enum PrimKind : int32_t { PK_TRI = 0, PK_RECT = 1, PK_SPHERE = 2 };

struct SphereDev {
    Xf o2w;   // object_to_world
    Xf w2o;   // world_to_object
    float radius, radius_world, rw2, area;
};

struct RectDev {
    float pa[3], pb[3], pc[3], pd[3];
    float normal[3];   // normalize(cross(pb - pa, pc - pa))
    float ss[3];       // cross(normal, aux) (rectangle.cpp:66-74)
    float area;        // |cross(pb - pa, pc - pa)|
    float pad;
};

struct TexRef {
    int32_t tex;   // < 0: constant
    float v[3];
};

struct DevTexture {
    const float4* texels;   // row 0 = top
    int32_t w, h, wrap_u, wrap_v, filter, pad;
};

enum MatParam : int32_t {
    MP_BASECOLOR = 0, MP_METALLIC, MP_SPECULAR, MP_SPECULAR_TINT, MP_ROUGHNESS, MP_ANISOTROPIC, MP_SHEEN,
    MP_SHEEN_TINT, MP_CLEARCOAT, MP_CLEARCOAT_GLOSS, MP_SPEC_TRANS, MP_SPEC_TRANS_ROUGHNESS, MP_DIFF_TRANS,
    MP_FLATNESS, MP_IOR, MP_COUNT
};

struct DevMaterial {
    int32_t type, thin, vattr_offset, pad;
    TexRef p[MP_COUNT];
    float reflect_color[3], refract_color[3];
    float eta_i, eta_t;
    float color[3];
    float cond_eta2[3], cond_etak2[3];   // ConductorFresnel members (fresnel.h:77-84)
};

enum LightKind : int32_t { LK_AREA_TRI = 0, LK_AREA_RECT = 1, LK_AREA_SPHERE = 2, LK_DIR = 3, LK_ENV = 4, LK_AREA_MESH = 5 };

struct DevLight {
    int32_t kind;
    int32_t obj;     // emissive object (area lights; mesh lights: the first triangle's object)
    int32_t index;   // triangle / rect / sphere index (area lights); mesh lights: first entry
                     // of the light's triangles in DevScene::mlight_tri
    int32_t count;   // mesh lights: number of triangles
    float radiance[3];
    float direction[3];   // directional: light-to-scene direction
    float inv_area;       // mesh lights: 1 / total area
};

struct DevEnv {
    int32_t present;
    int32_t tex;
    int32_t w, h;
    float factor;
    float pad[3];
    Xf l2w, w2l;
    // piecewise-constant tables (built on the device)
    const float* pdf_sample;      // [h*w] density of the sampling routine w.r.t. (u,v)
    const float* pdf_eval;        // [h*w] density EnvLight::Pdf reports (see fm_env.cu)
    const float* row_prob;        // [h*w] alias acceptance per texel within its row
    const int32_t* row_alias;     // [h*w]
    const float* marg_prob;       // [h]
    const int32_t* marg_alias;    // [h]
};

// Material classes for specialised shading kernels: kClsDisney holds only Disney,
// kClsSimple holds Lambert / conductor / dielectric, kClsAny holds every type.  A kernel
// instantiated for one class contains only that class's code.
constexpr int kClsAny = -1, kClsDisney = 0, kClsSimple = 1;
FM_HD int material_class(int type) { return type == 3 ? kClsDisney : kClsSimple; }

struct DevScene {
    // BVH: 5 x uint4 (80 B) per wide node; 3 x float4 per leaf primitive slot
    const uint4* nodes;
    const float4* leaf;
    int32_t num_nodes, num_leaf;
    int32_t num_tris, num_rects, num_spheres, num_prims;

    const int32_t* prim_obj;      // [num_prims] object of each primitive
    const int32_t* prim_info;     // [num_prims] (object's area light + 1) << 2 | (material class + 1)
    // shading data in original order
    const float* tri_pos;         // [T*9]
    const float* tri_normal;      // [T*9] or null
    const uint8_t* tri_has_normal;
    const float* tri_uv;          // [T*6] or null
    const float* tri_vattr;       // [T*3*vattr_dim] or null
    int32_t vattr_dim;
    int32_t num_objects;
    const RectDev* rects;
    const SphereDev* spheres;

    const int32_t* obj_material;  // [num_objects]
    const int32_t* obj_light;     // [num_objects] area light index or -1
    const DevMaterial* materials;
    const DevTexture* textures;
    const DevLight* lights;
    int32_t num_materials, num_textures, num_lights, env_light;   // env_light: index in lights or -1
    // mesh lights: triangle indices of every mesh light (grouped, in object order) and an
    // alias table over each light's triangle areas (acceptance, alias as a local index)
    const int32_t* mlight_tri;
    const float* mlight_prob;
    const int32_t* mlight_alias;
    DevEnv env;
};

}  // namespace fm
