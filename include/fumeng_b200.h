/*
 * fumeng_b200 — C-ABI of the B200 path-tracing core.
 *
 * This library replaces the reference engine's integrator hot path
 * (hietwll/Fumeng: Renderer::DrawFrame -> PathTracer::RenderPixel -> Scene /
 * Aggregate / Geometry / Material / Light) with CUDA kernels for sm_100a.  Callers
 * flatten a scene into the plain arrays below (the package's C++ SceneLoader does it
 * from the reference's JSON schema), create it once, and render it.
 *
 * Conventions
 *  - Every entry point returns an fm_status; FM_OK is 0.  On failure the message is
 *    available from fm_last_error(ctx).  No C++ exception crosses this boundary.
 *  - A context owns one CUDA stream and all device memory of its scenes.  A context is
 *    not thread-safe: use one context per host thread.
 *  - Images are row-major float32 RGB, row 0 = top row, like the reference's Image
 *    (src/engine/src/image/image.cpp:58-61).
 *  - Rays are 8 floats: origin xyz, t_min, direction xyz, t_max.
 *  - Buffers are host memory unless FM_FLAG_DEVICE_PTRS is passed, in which case they
 *    are device pointers of the context's device.
 */
#ifndef FUMENG_B200_H
#define FUMENG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FM_OK = 0,
    FM_ERR_INVALID = 1,        /* bad argument or scene description */
    FM_ERR_OOM = 2,            /* device allocation failed */
    FM_ERR_CUDA = 3,           /* CUDA runtime error */
    FM_ERR_QUEUE_OVERFLOW = 4, /* a device queue or traversal stack overflowed */
    FM_ERR_TIMEOUT = 5,        /* a bounded device wait ran out */
    FM_ERR_NO_DEVICE = 6       /* no CUDA device / extension not usable */
} fm_status;

typedef struct fm_ctx fm_ctx;
typedef struct fm_scene fm_scene;

enum {
    FM_FLAG_DEVICE_PTRS = 1, /* buffers are device pointers */
    FM_FLAG_PROFILE = 2      /* time the wavefront's kernels with CUDA events: the render then runs
                                as a host loop over graphs of iters_per_graph iterations instead of
                                one conditional graph launch (slower; profilers see its kernels) */
};

/* ---- textures ------------------------------------------------------------------ */
enum { FM_WRAP_REPEAT = 0, FM_WRAP_CLAMP = 1 };
enum { FM_FILTER_LINEAR = 0, FM_FILTER_NEAREST = 1 };

/* Texture::Sample / ImageTexture (core/texture.h:70-120, texture/image_texture.cpp:13-44).
 * texels: width*height*3 linear floats, row 0 = top (as decoded by Image). */
typedef struct {
    int32_t width, height;
    const float* texels;
    int32_t wrap_u, wrap_v;
    int32_t filter;
} fm_texture_desc;

/* A material parameter: a constant (texture < 0) or an image texture index. */
typedef struct {
    int32_t texture;
    float value[3];
} fm_tex_ref;

/* ---- materials ----------------------------------------------------------------- */
enum {
    FM_MAT_LAMBERT = 0,     /* material/lambert_diffuse.cpp */
    FM_MAT_SPEC_REFL = 1,   /* material/specular_reflection.cpp (conductor Fresnel) */
    FM_MAT_SPEC_TRANS = 2,  /* material/specular_transmission.cpp (dielectric) */
    FM_MAT_DISNEY = 3       /* material/disney.cpp */
};

/* Per-vertex Disney attributes (extension): when vattr_offset >= 0, the Disney
 * parameters basecolor.rgb, roughness, metallic, clearcoat are interpolated with the
 * hit's barycentrics from fm_scene_desc.tri_vattr at [offset .. offset+6) of each
 * triangle corner; the fm_tex_ref values of those six parameters are then ignored. */
typedef struct {
    int32_t type;
    int32_t thin;
    /* Lambert uses basecolor.  Disney (disney.cpp:627-662 channel rules: metallic reads
     * channel z, roughness channel y, the others channel x). */
    fm_tex_ref basecolor, metallic, specular, specular_tint, roughness, anisotropic, sheen,
        sheen_tint, clearcoat, clearcoat_gloss, spec_trans, spec_trans_roughness, diff_trans,
        flatness, ior;
    /* specular transmission (SpecularTransmissionConfig, core/material.h:20-34) */
    float reflect_color[3], refract_color[3];
    float eta_i, eta_t;
    /* specular reflection (CreateSpecularReflection, create/material.h:11) */
    float color[3], cond_eta_i[3], cond_eta_t[3], cond_k[3];
    int32_t vattr_offset;
} fm_material_desc;

/* ---- lights given explicitly (area lights come from emissive objects) ---------- */
enum { FM_LIGHT_ENV = 0, FM_LIGHT_DIRECTIONAL = 1 };

typedef struct {
    int32_t type;
    /* env (light/env_light.cpp): texture index, rotation in degrees (Z*Y*X), factor */
    int32_t texture;
    float rotation[3];
    float factor;
    /* directional (light/directional_light.cpp): radiance and normalized direction */
    float radiance[3];
    float direction[3];
} fm_light_desc;

/* ---- scene ----------------------------------------------------------------------
 * Objects are the reference's RenderObjects in load order (scene_loader.h:202-252):
 * one per mesh triangle, rectangle or sphere.  Object index = hit ID. */
typedef struct {
    int64_t num_objects;
    const int32_t* obj_material;   /* [num_objects] index into materials */
    const float* obj_emission;     /* [num_objects*3] emittance, or NULL for none */

    /* mesh triangles, world space, corner order as in the OBJ face */
    int64_t num_triangles;
    const float* tri_pos;          /* [n*9]  v0, v1, v2 */
    const float* tri_normal;       /* [n*9]  or NULL */
    const uint8_t* tri_has_normal; /* [n]    or NULL (all have normals iff tri_normal) */
    const float* tri_uv;           /* [n*6]  (u, 1-v) per corner as triangle.cpp:152, or NULL */
    const int32_t* tri_object;     /* [n]    object index */
    const float* tri_vattr;        /* [n*3*vattr_dim] per-corner attributes, or NULL */
    int32_t vattr_dim;

    /* rectangles (geometry/rectangle.cpp): pa, pb, pc, pd */
    int64_t num_rects;
    const float* rect_pts;         /* [n*12] */
    const int32_t* rect_object;    /* [n] */

    /* spheres (geometry/sphere.cpp): object-space radius and the object-to-world
     * transform as a row-major 4x4 */
    int64_t num_spheres;
    const float* sphere_radius;    /* [n] */
    const float* sphere_xform;     /* [n*16] */
    const int32_t* sphere_object;  /* [n] */

    int32_t num_materials;
    const fm_material_desc* materials;
    int32_t num_textures;
    const fm_texture_desc* textures;
    int32_t num_lights;            /* JSON lights, appended after area lights */
    const fm_light_desc* lights;

    /* Extension: mesh lights.  NULL, or [num_triangles] group ids: the emissive triangles
     * that share a group id >= 0 form ONE area light, sampled by picking a triangle in
     * proportion to its area and a point on it (area pdf 1 / total area), as the
     * reference's Embree meshes do (geometry/triangle_embree.cpp:119-130, 253-270) --
     * one light sample per mesh per bounce instead of one per triangle.  The light takes
     * the place of the group's first triangle in the light list; every triangle of a
     * group must have the same emission.  Object indices (hit IDs) are unchanged.
     * Triangles with group -1 stay one light each (the built-in BVH path,
     * core/render_object.h:29-32). */
    const int32_t* tri_light_group;
} fm_scene_desc;

/* ---- camera and render parameters ---------------------------------------------- */
enum { FM_CAMERA_PINHOLE = 0, FM_CAMERA_THIN_LENS = 1 };

/* PinHoleCameraConfig / ThinLensCameraConfig (core/camera.h:9-41) */
typedef struct {
    int32_t type;
    float pos[3], look_at[3], up[3];
    float fov;            /* degrees */
    float aspect;
    float focal_distance;
    float lens_radius;
} fm_camera;

enum { FM_MODE_MEGAKERNEL = 0, FM_MODE_WAVEFRONT = 1 };

/* PathTracerConfig (core/renderer.h:17-60) plus the seed of the counter-based RNG. */
typedef struct {
    int32_t width, height, spp;
    int32_t depth, direct_loop, rr_depth;
    float rr_coef;
    uint64_t seed;
    int32_t mode;
    int32_t sample_offset;   /* first sample index (for split / decorrelated renders) */
    /* Extension (the reference has no clamp): when > 0, each colour channel of every
     * camera sample's radiance is limited to this value before it enters the pixel's
     * sum (min(L, max_sample_value); NaN stays NaN).  0 renders the reference's
     * estimator unchanged.  The clamped estimator is biased low; it exists for
     * firefly-free previews and for comparisons whose variance must stay bounded.
     * fm_render_adjoint requires 0. */
    float max_sample_value;
    /* Extension: render region.  With region_w > 0 only the pixels [region_x, region_x +
     * region_w) x [region_y, region_y + region_h) of the width x height image (row 0 =
     * top) are rendered, and the outputs are region_w x region_h images of exactly those
     * pixels' values in a full render with the same seed (random streams are keyed by
     * the full image's pixel index).  region_w = region_h = 0: the whole image. */
    int32_t region_x, region_y, region_w, region_h;
} fm_render_params;

/* Counters of one render, read back after it completes. */
typedef struct {
    int64_t paths;            /* camera samples completed */
    int64_t closest_rays;     /* closest-hit queries traced */
    int64_t shadow_rays;      /* any-hit queries traced */
    int64_t bounces;          /* shading events */
    int64_t nan_samples;      /* samples whose radiance was not finite */
    double kernel_ms;         /* device time of the render kernels */
    double trace_ms;          /* wavefront trace kernels: CUDA events with FM_FLAG_PROFILE, else the
                                 GPU global timer (first block start to last block end per launch) */
    double shade_ms;          /* wavefront kernels after the trace (resolve, shading, logic): CUDA
                                 events with FM_FLAG_PROFILE, else kernel_ms minus trace_ms */
    int64_t launches;         /* kernels launched (graph nodes included) */
} fm_render_stats;

/* ---- entry points ---------------------------------------------------------------- */

/* Replaces: nothing in the reference (it has no device); creates the CUDA context
 * holder used by every other call.  A context keeps its wavefront workspace between
 * renders (path-state and queue buffers sized to the largest pool and queues seen: for
 * forward renders about 284 B plus 52 B per light per path slot, 1.6 GB at 2^22 slots
 * and two lights; more for adjoint renders; pinned staging; the instantiated render
 * graph) and releases it in fm_ctx_destroy. */
fm_status fm_ctx_create(int device, fm_ctx** out);
void fm_ctx_destroy(fm_ctx* ctx);
const char* fm_last_error(const fm_ctx* ctx);

/* Replaces: SceneLoader::ParseScene's aggregate construction
 * (scene_loader.h:86-146 -> CreateBVHAggregate, accelerator/bvh_aggregate.cpp:126-155)
 * and the area-light collection of Scene::Scene (core/scene.h:21-25).  Copies the
 * description to the device and builds the BVH there (binned SAH, 8-wide nodes). */
fm_status fm_scene_create(fm_ctx* ctx, const fm_scene_desc* desc, fm_scene** out);

/* Creates n scenes in one call (out[i] from descs[i]; all or none: on an error every
 * out[i] is null).  The same work as n fm_scene_create calls -- the reference loads one
 * scene per run (SceneLoader::Load, create/scene_loader.h:293-302) -- with the uploads
 * of all scenes streamed through one pinned staging ring and the BVH builds of different
 * scenes running side by side on the device; the host waits twice per call instead of
 * several times per scene.  The context keeps the ring (32 MiB pinned) and its builder
 * streams until fm_ctx_destroy. */
fm_status fm_scene_create_batch(fm_ctx* ctx, int32_t n, const fm_scene_desc* const* descs, fm_scene** out);
fm_status fm_scene_destroy(fm_ctx* ctx, fm_scene* scene);
/* BVH statistics: wide nodes, leaf primitive slots, max depth, build milliseconds. */
fm_status fm_scene_bvh_stats(fm_ctx* ctx, const fm_scene* scene, int64_t* nodes, int64_t* prims,
                             int32_t* depth, double* build_ms);

/* Sizes of a created scene: objects, materials, textures, lights (area lights first).
 * Any output may be NULL. */
fm_status fm_scene_info(fm_ctx* ctx, const fm_scene* scene, int64_t* objects, int32_t* materials,
                        int32_t* textures, int32_t* lights);

/* Replaces: Aggregate::GetIntersect (core/aggregate.h:30, accelerator/bvh_aggregate.cpp:
 * 167-176).  rays: n x 8 floats.  obj_id[i] = object index of the closest hit or -1;
 * t[i] = its distance (+inf on a miss). */
fm_status fm_trace_closest(fm_ctx* ctx, const fm_scene* scene, const float* rays, int64_t n,
                           int32_t* obj_id, float* t, int32_t flags);

/* Replaces: Aggregate::IsIntersect (core/aggregate.h:24, bvh_aggregate.cpp:157-165).
 * occluded[i] = 1 if any object is hit with t in (t_min, t_max). */
fm_status fm_trace_any(fm_ctx* ctx, const fm_scene* scene, const float* rays, int64_t n,
                       uint8_t* occluded, int32_t flags);

/* Replaces: Renderer::DrawFrame's sample loop and PathTracer::RenderPixel
 * (core/renderer.h:84-117, renderer/path_tracing.cpp:34-229).  Writes width*height*3
 * floats to each non-NULL output: mean color, mean albedo, mean normal over spp
 * samples.  stats may be NULL. */
fm_status fm_render(fm_ctx* ctx, const fm_scene* scene, const fm_camera* camera,
                    const fm_render_params* params, float* rgb, float* albedo, float* normal,
                    int32_t flags, fm_render_stats* stats);

/* Wavefront tuning: path-slot pool size (queue capacities scale with it), block sizes of
 * the trace and shade kernels, and iterations per captured CUDA graph.  The last two
 * fields bound a render below its automatic limits (0 = automatic): max_iterations caps
 * the wavefront iterations (a render that still has work then stops and returns
 * FM_ERR_TIMEOUT), queue_limit caps the entries of each ray queue (a render that needs
 * more stops and returns FM_ERR_QUEUE_OVERFLOW).  Both leave the context usable; they
 * exist to bound a render's time and to exercise those error paths. */
typedef struct {
    int64_t pool;
    int32_t trace_block, shade_block, iters_per_graph;
    int32_t max_iterations;
    int32_t queue_limit;
} fm_tuning;

/* Replaces: running the reference once per scene (main.cpp:5-11, one SceneLoader and one
 * Renderer::DrawFrame per process).  Renders n views -- view i is scenes[i] seen by
 * cameras[i] with params[i] -- in one persistent wavefront whose kernel sequence is
 * captured as a CUDA graph.  rgb[i] / albedo[i] / normal[i] receive view i's images
 * (albedo and normal arrays, or their entries, may be NULL).  All params must use
 * FM_MODE_WAVEFRONT, or all FM_MODE_MEGAKERNEL (then all views are rendered by one launch
 * of the plain megakernel, the baseline: persistent threads that each run whole camera
 * paths, taking (view, pixel, sample chunk) items from a shared counter).  tuning == NULL selects the tuning
 * cached for this batch's shape class, running the autotuner on first use. */
fm_status fm_render_batch(fm_ctx* ctx, int32_t n, const fm_scene* const* scenes, const fm_camera* cameras,
                          const fm_render_params* params, float* const* rgb, float* const* albedo,
                          float* const* normal, int32_t flags, const fm_tuning* tuning, fm_render_stats* stats);

/* Replaces: nothing in the reference (its thread pool has no knobs beyond thread_count).
 * Times candidate tunings by coordinate descent -- path-slot pools of 2^19 to 2^25 slots
 * (those whose workspace fits in half of the free device memory), trace and shade block
 * sizes, iterations per graph -- on trial renders of the batch itself when it has at most
 * 2^28 samples, else of a copy at up to 8 spp per view, and returns the fastest; the
 * result is cached in the context for the batch's shape class. */
fm_status fm_autotune_batch(fm_ctx* ctx, int32_t n, const fm_scene* const* scenes, const fm_camera* cameras,
                            const fm_render_params* params, fm_tuning* out);

/* Replaces: SceneLoader::Load (create/scene_loader.h:293-302).  Reads a scene file in
 * the reference's JSON schema (plus the extensions documented in
 * fumeng_b200/host/fm_scene_loader.h), loads its OBJ meshes and .hdr / PNG textures,
 * creates the device scene and returns the camera and renderer settings it names.
 * With out == NULL the file is only parsed and checked (no device is needed and ctx
 * may be NULL). */
fm_status fm_scene_load(fm_ctx* ctx, const char* json_path, fm_scene** out, fm_camera* camera,
                        fm_render_params* params);

/* Replaces: SceneLoader::DrawFrame -> Renderer::DrawFrame (scene_loader.h:304-307,
 * core/renderer.h:84-144), as called by the command line (src/cmd/src/main.cpp:5-11):
 * renders the scene file, applies its post-process chain and writes <output>.png,
 * <output>_albedo.png and <output>_normal.png. */
fm_status fm_draw_frame(fm_ctx* ctx, const char* json_path);

/* No counterpart in the reference (its queries never leave host memory).  Same query and
 * results as fm_trace_closest with host buffers, for callers that cannot have the
 * library allocate device memory while they run -- a real-time loop with a fixed
 * device-memory budget and a frame deadline, or an application whose own pool owns the
 * device memory.  Instead of per-call allocations it stages rays and results in a fixed
 * 10 MiB array that is part of the library image; every GPU that loads the library holds
 * that array until the process exits.
 *   - n may be at most 262144 rays; larger batches are rejected with FM_ERR_INVALID.
 *   - The first call on a device looks up the array's device address (with that device
 *     current); make that first call before any stream capture.
 *   - All calls on a device share the array: calls that run at the same time on that
 *     device (from different contexts or threads) race with each other. */
fm_status fm_trace_closest_noalloc(fm_ctx* ctx, const fm_scene* scene, const float* rays, int64_t n,
                                   int32_t* obj_id, float* t);

/* ---- post-processing ----------------------------------------------------------------- */
enum {
    FM_POST_TONEMAP = 0,         /* "tonemapping" (post/tonemapping.cpp), parameter lum */
    FM_POST_LINEAR_TO_SRGB = 1,  /* "linear_to_srgb" (post/linear_to_srgb.cpp) */
    FM_POST_SRGB_TO_LINEAR = 2,  /* "srgb_to_linear" (post/srgb_to_linear.cpp) */
    FM_POST_DENOISE = 3          /* "oidn_denoise" (post/oidn_denoise.cpp): see fm_postprocess */
};

typedef struct {
    int32_t type;
    float lum;                   /* FM_POST_TONEMAP only */
} fm_post_step;

/* Replaces: the PostProcess chain Renderer::DrawFrame runs on the finished frame
 * (core/renderer.h:131-135) and the 8-bit conversion of RenderTarget::save_to_file
 * (render_target.h:26-31 -> Image::save_to_file, image/image.cpp:98-109, RealToUInt8
 * core/utils.h:134-137).  Applies steps[0..num_steps) in order to rgb (width*height*3
 * floats, updated in place) and writes round(255 * clamp(x, 0, 1)) of rgb, albedo and
 * normal to the non-NULL 8-bit outputs (albedo and normal are not post-processed, as in
 * the reference).  The per-pixel steps use the reference's float arithmetic, so the bytes
 * equal the reference's float build's for the same input (the sRGB steps' pow may differ
 * in its last bit, which can move a value sitting on a rounding boundary by one code).
 * FM_POST_DENOISE needs albedo and normal: the reference calls Intel Open Image Denoise
 * there, which is not available; this library runs an edge-avoiding a-trous wavelet
 * filter guided by the same albedo and normal images instead (its output is not
 * OIDN's).  At most 16 steps.  Host buffers unless FM_FLAG_DEVICE_PTRS. */
fm_status fm_postprocess(fm_ctx* ctx, int32_t width, int32_t height, const fm_post_step* steps, int32_t num_steps,
                         float* rgb, const float* albedo, const float* normal, uint8_t* rgb8, uint8_t* albedo8,
                         uint8_t* normal8, int32_t flags);

/* ---- differentiable rendering ------------------------------------------------------
 * The reference renders forward only; the two entry points below have no counterpart
 * in it. */

/* Replaces texture contents in place (texels: width*height*3 floats in the texture's
 * own size, row 0 = top; device pointer with FM_FLAG_DEVICE_PTRS).  If the texture is
 * the environment light's, its importance-sampling tables are rebuilt. */
fm_status fm_scene_update_texture(fm_ctx* ctx, fm_scene* scene, int32_t texture, const float* texels,
                                  int32_t flags);

/* Number of differentiated parameters per material: basecolor r, g, b, metallic,
 * roughness (in this order). */
enum { FM_GRAD_PARAMS = 5 };

/* Gradient outputs of fm_render_adjoint.  Values are ADDED to what the buffers hold.
 * texture_grads[t] (t a scene texture index) is NULL or width*height*3 doubles, the
 * derivative with respect to each texel channel; a material parameter read from a
 * texture sends its derivative there (basecolor: rgb, metallic: the third channel,
 * roughness: the second), as does the environment light's texture.  material_grads is
 * NULL or num_materials * FM_GRAD_PARAMS doubles: derivatives with respect to the
 * constant (untextured) parameters of Lambert and Disney materials. */
typedef struct {
    double* const* texture_grads;   /* array of num_textures pointers, or NULL */
    double* material_grads;
} fm_grad_desc;

/* Path-replay adjoint.  For views v of one scene (cameras[v], params[v]; wavefront mode),
 * computes the gradient of  sum_v sum_pixels d_rgb[v] . image_v  with respect to the
 * texels and material constants above, where image_v is the mean over params[v].spp
 * samples (use a seed different from the forward render's for a decorrelated
 * estimate).  Each sample's path is traced once for its radiance and replayed with the
 * same random numbers to accumulate derivatives, so memory does not grow with depth or
 * spp.  The sampled directions are held fixed (the derivative of the estimator for its
 * random numbers, which is unbiased for the gradient of the image's expectation);
 * everything that depends on the parameters along the fixed path is differentiated: the
 * BSDF values, the sampling pdfs in f / pdf, the MIS weights built from them and, for
 * env-map texels, the env map's sampling and reported densities (their normalisation
 * over all texels included).  rgb (NULL, or an
 * array of per-view NULL or width*height*3 buffers -- region size when a region is set)
 * receives the primal image of the samples used.  params[v].max_sample_value must be 0.
 * Host buffers unless FM_FLAG_DEVICE_PTRS. */
fm_status fm_render_adjoint(fm_ctx* ctx, const fm_scene* scene, int32_t num_views, const fm_camera* cameras,
                            const fm_render_params* params, const float* const* d_rgb, float* const* rgb,
                            const fm_grad_desc* grads, int32_t flags, fm_render_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* FUMENG_B200_H */
