"""fumeng_b200: B200 path-tracing core behind a C-ABI (ctypes binding).

The product is the shared library ``libfumeng_b200.so`` (CUDA kernels for sm_100a plus
the C++ host layer); this module only binds its C entry points (include/fumeng_b200.h)
for Python callers such as the tests and bench.py.  Every call goes to the CUDA
library; there is no CPU fallback, and loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libfumeng_b200.so"

FM_OK, FM_ERR_INVALID, FM_ERR_OOM, FM_ERR_CUDA, FM_ERR_QUEUE_OVERFLOW, FM_ERR_TIMEOUT, FM_ERR_NO_DEVICE = range(7)
FM_FLAG_DEVICE_PTRS = 1
FM_FLAG_PROFILE = 2
FM_WRAP_REPEAT, FM_WRAP_CLAMP = 0, 1
FM_FILTER_LINEAR, FM_FILTER_NEAREST = 0, 1
FM_MAT_LAMBERT, FM_MAT_SPEC_REFL, FM_MAT_SPEC_TRANS, FM_MAT_DISNEY = 0, 1, 2, 3
FM_LIGHT_ENV, FM_LIGHT_DIRECTIONAL = 0, 1
FM_CAMERA_PINHOLE, FM_CAMERA_THIN_LENS = 0, 1
FM_MODE_MEGAKERNEL, FM_MODE_WAVEFRONT = 0, 1

_f3 = C.c_float * 3
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)


class TexRef(C.Structure):
    _fields_ = [("texture", C.c_int32), ("value", _f3)]


class TextureDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("texels", _fp), ("wrap_u", C.c_int32),
                ("wrap_v", C.c_int32), ("filter", C.c_int32)]


MAT_PARAMS = ["basecolor", "metallic", "specular", "specular_tint", "roughness", "anisotropic", "sheen",
              "sheen_tint", "clearcoat", "clearcoat_gloss", "spec_trans", "spec_trans_roughness", "diff_trans",
              "flatness", "ior"]


class MaterialDesc(C.Structure):
    _fields_ = ([("type", C.c_int32), ("thin", C.c_int32)] + [(p, TexRef) for p in MAT_PARAMS] +
                [("reflect_color", _f3), ("refract_color", _f3), ("eta_i", C.c_float), ("eta_t", C.c_float),
                 ("color", _f3), ("cond_eta_i", _f3), ("cond_eta_t", _f3), ("cond_k", _f3),
                 ("vattr_offset", C.c_int32)])


class LightDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("texture", C.c_int32), ("rotation", _f3), ("factor", C.c_float),
                ("radiance", _f3), ("direction", _f3)]


class SceneDesc(C.Structure):
    _fields_ = [("num_objects", C.c_int64), ("obj_material", _ip), ("obj_emission", _fp),
                ("num_triangles", C.c_int64), ("tri_pos", _fp), ("tri_normal", _fp), ("tri_has_normal", _u8p),
                ("tri_uv", _fp), ("tri_object", _ip), ("tri_vattr", _fp), ("vattr_dim", C.c_int32),
                ("num_rects", C.c_int64), ("rect_pts", _fp), ("rect_object", _ip),
                ("num_spheres", C.c_int64), ("sphere_radius", _fp), ("sphere_xform", _fp), ("sphere_object", _ip),
                ("num_materials", C.c_int32), ("materials", C.POINTER(MaterialDesc)),
                ("num_textures", C.c_int32), ("textures", C.POINTER(TextureDesc)),
                ("num_lights", C.c_int32), ("lights", C.POINTER(LightDesc)), ("tri_light_group", _ip)]


class Camera(C.Structure):
    _fields_ = [("type", C.c_int32), ("pos", _f3), ("look_at", _f3), ("up", _f3), ("fov", C.c_float),
                ("aspect", C.c_float), ("focal_distance", C.c_float), ("lens_radius", C.c_float)]


class RenderParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("depth", C.c_int32),
                ("direct_loop", C.c_int32), ("rr_depth", C.c_int32), ("rr_coef", C.c_float), ("seed", C.c_uint64),
                ("mode", C.c_int32), ("sample_offset", C.c_int32), ("max_sample_value", C.c_float),
                ("region_x", C.c_int32), ("region_y", C.c_int32), ("region_w", C.c_int32), ("region_h", C.c_int32)]

    def out_shape(self) -> tuple:
        """(rows, columns) of the rendered images: the region's, or the whole image's."""
        return (self.region_h, self.region_w) if self.region_w > 0 else (self.height, self.width)

    def out_pixels(self) -> int:
        h, w = self.out_shape()
        return h * w


class RenderStats(C.Structure):
    _fields_ = [("paths", C.c_int64), ("closest_rays", C.c_int64), ("shadow_rays", C.c_int64),
                ("bounces", C.c_int64), ("nan_samples", C.c_int64), ("kernel_ms", C.c_double),
                ("trace_ms", C.c_double), ("shade_ms", C.c_double), ("launches", C.c_int64)]


class Tuning(C.Structure):
    _fields_ = [("pool", C.c_int64), ("trace_block", C.c_int32), ("shade_block", C.c_int32),
                ("iters_per_graph", C.c_int32), ("max_iterations", C.c_int32), ("queue_limit", C.c_int32)]

    def as_dict(self) -> dict:
        return {"pool": self.pool, "trace_block": self.trace_block, "shade_block": self.shade_block,
                "iters_per_graph": self.iters_per_graph}


FM_POST_TONEMAP, FM_POST_LINEAR_TO_SRGB, FM_POST_SRGB_TO_LINEAR, FM_POST_DENOISE = range(4)


class PostStep(C.Structure):
    _fields_ = [("type", C.c_int32), ("lum", C.c_float)]


class FumengError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"fumeng_b200 error {status}: {message}")
        self.status = status


class GradDesc(C.Structure):
    """fm_grad_desc: gradient outputs of fm_render_adjoint (added to)."""
    _fields_ = [("texture_grads", C.POINTER(C.c_void_p)), ("material_grads", C.c_void_p)]


GRAD_PARAMS = 5   # basecolor r, g, b, metallic, roughness

_lib = None


def load_library() -> C.CDLL:
    """Load libfumeng_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("FUMENG_B200_LIB", LIB_PATH))
    if not path.exists():
        raise FileNotFoundError(f"{path} is missing: build it with `python -m fumeng_b200.build`")
    lib = C.CDLL(str(path))
    vp = C.c_void_p
    sig = {
        "fm_ctx_create": ([C.c_int, C.POINTER(vp)], C.c_int),
        "fm_ctx_destroy": ([vp], None),
        "fm_last_error": ([vp], C.c_char_p),
        "fm_scene_create": ([vp, C.POINTER(SceneDesc), C.POINTER(vp)], C.c_int),
        "fm_scene_create_batch": ([vp, C.c_int32, C.POINTER(C.POINTER(SceneDesc)), C.POINTER(vp)], C.c_int),
        "fm_scene_destroy": ([vp, vp], C.c_int),
        "fm_scene_bvh_stats": ([vp, vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                C.POINTER(C.c_double)], C.c_int),
        "fm_trace_closest": ([vp, vp, vp, C.c_int64, vp, vp, C.c_int32], C.c_int),
        "fm_trace_any": ([vp, vp, vp, C.c_int64, vp, C.c_int32], C.c_int),
        "fm_render": ([vp, vp, C.POINTER(Camera), C.POINTER(RenderParams), vp, vp, vp, C.c_int32,
                       C.POINTER(RenderStats)], C.c_int),
        "fm_render_batch": ([vp, C.c_int32, C.POINTER(vp), C.POINTER(Camera), C.POINTER(RenderParams),
                             C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.c_int32, C.POINTER(Tuning),
                             C.POINTER(RenderStats)], C.c_int),
        "fm_autotune_batch": ([vp, C.c_int32, C.POINTER(vp), C.POINTER(Camera), C.POINTER(RenderParams),
                               C.POINTER(Tuning)], C.c_int),
        "fm_scene_load": ([vp, C.c_char_p, C.POINTER(vp), C.POINTER(Camera), C.POINTER(RenderParams)], C.c_int),
        "fm_draw_frame": ([vp, C.c_char_p], C.c_int),
        "fm_trace_closest_noalloc": ([vp, vp, vp, C.c_int64, vp, vp], C.c_int),
        "fm_scene_update_texture": ([vp, vp, C.c_int32, vp, C.c_int32], C.c_int),
        "fm_scene_info": ([vp, vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                           C.POINTER(C.c_int32)], C.c_int),
        "fm_postprocess": ([vp, C.c_int32, C.c_int32, C.POINTER(PostStep), C.c_int32, vp, vp, vp, vp, vp, vp,
                            C.c_int32], C.c_int),
        "fm_render_adjoint": ([vp, vp, C.c_int32, C.POINTER(Camera), C.POINTER(RenderParams), C.POINTER(vp),
                               C.POINTER(vp), C.POINTER(GradDesc), C.c_int32, C.POINTER(RenderStats)], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


EXPORTED_SYMBOLS = ["fm_ctx_create", "fm_ctx_destroy", "fm_last_error", "fm_scene_create", "fm_scene_create_batch",
                    "fm_scene_destroy",
                    "fm_scene_bvh_stats", "fm_trace_closest", "fm_trace_any", "fm_render", "fm_render_batch",
                    "fm_autotune_batch", "fm_scene_load", "fm_draw_frame", "fm_trace_closest_noalloc",
                    "fm_scene_update_texture", "fm_render_adjoint", "fm_scene_info", "fm_postprocess"]


def _ptr(a, ctype=C.c_void_p):
    if a is None:
        return None
    return a.ctypes.data_as(ctype)


class Context:
    """One CUDA device context (owns a stream); not thread-safe."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        st = self.lib.fm_ctx_create(device, C.byref(h))
        if st != FM_OK:
            raise FumengError(st, "fm_ctx_create failed (no usable CUDA device?)")
        self.h = h

    def check(self, st: int) -> None:
        if st != FM_OK:
            raise FumengError(st, self.lib.fm_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.fm_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _batch_args(self, scenes, cams, params):
        n = len(scenes)
        sc = (C.c_void_p * n)(*[s.h.value if hasattr(s.h, "value") else s.h for s in scenes])
        ca = (Camera * n)(*cams)
        pa = (RenderParams * n)(*params)
        return n, sc, ca, pa

    def render_batch(self, scenes, cams, params, want_aov: bool = False, tuning: Tuning | None = None,
                     device_outputs=None, profile: bool = False, out=None):
        """Render view i = (scenes[i], cams[i], params[i]) for all i in one call.

        device_outputs: optional list of device pointers (ints) for the rgb images, which
        makes the call skip the device-to-host copies (FM_FLAG_DEVICE_PTRS).
        out: optional list of host arrays for the rgb images (float32, C-contiguous, of
        shape params[i].out_shape() + (3,)), written in place and returned; a caller that
        renders repeatedly passes the same arrays each time instead of having new ones
        allocated (and their pages faulted in by the copies) on every call."""
        n, sc, ca, pa = self._batch_args(scenes, cams, params)
        stats = RenderStats()
        tp = C.byref(tuning) if tuning is not None else None
        if device_outputs is not None:
            rgb_p = (C.c_void_p * n)(*device_outputs)
            flags = FM_FLAG_DEVICE_PTRS | (FM_FLAG_PROFILE if profile else 0)
            self.check(self.lib.fm_render_batch(self.h, n, sc, ca, pa, rgb_p, None, None, flags, tp, C.byref(stats)))
            return None, None, None, stats
        if out is not None:
            if len(out) != n:
                raise ValueError(f"out holds {len(out)} arrays for {n} views")
            for a, p in zip(out, params):
                if (not isinstance(a, np.ndarray) or a.dtype != np.float32 or not a.flags.c_contiguous
                        or not a.flags.writeable or a.shape != p.out_shape() + (3,)):
                    raise ValueError("out arrays must be writeable C-contiguous float32 arrays of shape "
                                     "out_shape() + (3,)")
            rgb = list(out)
        else:
            rgb = [np.empty(p.out_shape() + (3,), np.float32) for p in params]
        alb = [np.empty(p.out_shape() + (3,), np.float32) for p in params] if want_aov else None
        nrm = [np.empty(p.out_shape() + (3,), np.float32) for p in params] if want_aov else None
        rgb_p = (C.c_void_p * n)(*[a.ctypes.data for a in rgb])
        alb_p = (C.c_void_p * n)(*[a.ctypes.data for a in alb]) if want_aov else None
        nrm_p = (C.c_void_p * n)(*[a.ctypes.data for a in nrm]) if want_aov else None
        flags = FM_FLAG_PROFILE if profile else 0
        self.check(self.lib.fm_render_batch(self.h, n, sc, ca, pa, rgb_p, alb_p, nrm_p, flags, tp, C.byref(stats)))
        return rgb, alb, nrm, stats

    def autotune_batch(self, scenes, cams, params) -> Tuning:
        n, sc, ca, pa = self._batch_args(scenes, cams, params)
        t = Tuning()
        self.check(self.lib.fm_autotune_batch(self.h, n, sc, ca, pa, C.byref(t)))
        return t

    def load_scene(self, json_path):
        """SceneLoader::Load through the C++ loader: returns (Scene, Camera, RenderParams)."""
        h = C.c_void_p()
        cam = Camera()
        params = RenderParams()
        self.check(self.lib.fm_scene_load(self.h, str(json_path).encode(), C.byref(h), C.byref(cam), C.byref(params)))
        return Scene(self, h, None), cam, params

    def postprocess(self, steps, rgb, albedo=None, normal=None):
        """The post-process chain and 8-bit conversion (fm_postprocess) of HxWx3 float32
        images; steps: [(type, lum)].  Returns (rgb after the chain, rgb8, albedo8,
        normal8), the 8-bit arrays None where the input was None."""
        rgb = np.array(rgb, np.float32, copy=True, order="C")
        h, w, _ = rgb.shape
        st = (PostStep * max(1, len(steps)))(*[PostStep(int(t), float(l)) for t, l in steps])
        a = None if albedo is None else np.ascontiguousarray(albedo, np.float32)
        n = None if normal is None else np.ascontiguousarray(normal, np.float32)
        c8 = np.empty((h, w, 3), np.uint8)
        a8 = np.empty((h, w, 3), np.uint8) if a is not None else None
        n8 = np.empty((h, w, 3), np.uint8) if n is not None else None
        self.check(self.lib.fm_postprocess(self.h, w, h, st, len(steps), _ptr(rgb), _ptr(a), _ptr(n), _ptr(c8),
                                           _ptr(a8), _ptr(n8), 0))
        return rgb, c8, a8, n8

    def draw_frame(self, json_path) -> None:
        """SceneLoader::DrawFrame: render the scene file and write its PNG outputs."""
        self.check(self.lib.fm_draw_frame(self.h, str(json_path).encode()))

    def create_scene(self, desc_holder) -> "Scene":
        h = C.c_void_p()
        self.check(self.lib.fm_scene_create(self.h, C.byref(desc_holder.desc), C.byref(h)))
        return Scene(self, h, desc_holder)

    def create_scenes(self, desc_holders) -> list:
        """All scenes in one fm_scene_create_batch call (uploads and BVH builds overlapped)."""
        n = len(desc_holders)
        descs = (C.POINTER(SceneDesc) * n)(*[C.pointer(h.desc) for h in desc_holders])
        hs = (C.c_void_p * n)()
        self.check(self.lib.fm_scene_create_batch(self.h, n, descs, hs))
        return [Scene(self, C.c_void_p(hs[i]), desc_holders[i]) for i in range(n)]


class Scene:
    def __init__(self, ctx: Context, h, holder):
        self.ctx, self.h, self._holder = ctx, h, holder

    def destroy(self) -> None:
        if self.h:
            self.ctx.check(self.ctx.lib.fm_scene_destroy(self.ctx.h, self.h))
            self.h = None

    def bvh_stats(self) -> dict:
        n, p, d, ms = C.c_int64(), C.c_int64(), C.c_int32(), C.c_double()
        self.ctx.check(self.ctx.lib.fm_scene_bvh_stats(self.ctx.h, self.h, C.byref(n), C.byref(p), C.byref(d),
                                                       C.byref(ms)))
        return {"nodes": n.value, "prims": p.value, "depth": d.value, "build_ms": ms.value}

    def trace_closest(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        obj = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        self.ctx.check(self.ctx.lib.fm_trace_closest(self.ctx.h, self.h, _ptr(rays), n, _ptr(obj), _ptr(t), 0))
        return obj, t

    def trace_closest_noalloc(self, rays: np.ndarray):
        """fm_trace_closest through the library's fixed staging area (no device allocation)."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        obj = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        self.ctx.check(self.ctx.lib.fm_trace_closest_noalloc(self.ctx.h, self.h, _ptr(rays), n, _ptr(obj), _ptr(t)))
        return obj, t

    def trace_any(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        n = rays.shape[0]
        occ = np.empty(n, np.uint8)
        self.ctx.check(self.ctx.lib.fm_trace_any(self.ctx.h, self.h, _ptr(rays), n, _ptr(occ), 0))
        return occ

    def info(self) -> dict:
        o, m, t, l = C.c_int64(), C.c_int32(), C.c_int32(), C.c_int32()
        self.ctx.check(self.ctx.lib.fm_scene_info(self.ctx.h, self.h, C.byref(o), C.byref(m), C.byref(t), C.byref(l)))
        return {"objects": o.value, "materials": m.value, "textures": t.value, "lights": l.value}

    def update_texture(self, index: int, texels: np.ndarray) -> None:
        """Replace texture `index`'s texels (HxWx3 float32, row 0 = top) in place."""
        texels = np.ascontiguousarray(texels, dtype=np.float32)
        self.ctx.check(self.ctx.lib.fm_scene_update_texture(self.ctx.h, self.h, int(index), _ptr(texels), 0))

    def render_adjoint(self, cams, params, d_rgb, texture_shapes: dict, material_grads: bool = False,
                       want_image: bool = False, profile: bool = False):
        """Path-replay adjoint over views (cams[i], params[i]) with dLoss/dI images d_rgb[i].

        texture_shapes: {texture index: (height, width)} of the textures whose texel
        gradients are wanted.  Returns (texture grads {index: HxWx3 float64},
        material grads (num_materials x 5 float64) or None, images or None, stats)."""
        n = len(cams)
        ca = (Camera * n)(*cams)
        pa = (RenderParams * n)(*params)
        d_rgb = [np.ascontiguousarray(d, dtype=np.float32) for d in d_rgb]
        dp = (C.c_void_p * n)(*[d.ctypes.data for d in d_rgb])
        imgs = [np.empty(p.out_shape() + (3,), np.float32) for p in params] if want_image else None
        ip = (C.c_void_p * n)(*[a.ctypes.data for a in imgs]) if want_image else None
        info = self.info()
        nt = info["textures"]
        if any(k < 0 or k >= nt for k in texture_shapes):
            raise ValueError("texture index out of range")
        tg = {k: np.zeros((h, w, 3), np.float64) for k, (h, w) in texture_shapes.items()}
        tarr = (C.c_void_p * max(nt, 1))(*[tg[k].ctypes.data if k in tg else None for k in range(nt)])
        mg = None
        if material_grads:
            mg = np.zeros((info["materials"], GRAD_PARAMS), np.float64)
        gd = GradDesc(tarr if nt else None, mg.ctypes.data if mg is not None else None)
        stats = RenderStats()
        flags = FM_FLAG_PROFILE if profile else 0
        self.ctx.check(self.ctx.lib.fm_render_adjoint(self.ctx.h, self.h, n, ca, pa, dp, ip, C.byref(gd), flags,
                                                      C.byref(stats)))
        return tg, mg, imgs, stats

    def render(self, camera: Camera, params: RenderParams, want_aov: bool = True):
        """Returns (rgb, albedo, normal, stats) as HxWx3 float32 arrays (row 0 = top)."""
        h, w = params.out_shape()
        rgb = np.empty((h, w, 3), np.float32)
        alb = np.empty((h, w, 3), np.float32) if want_aov else None
        nrm = np.empty((h, w, 3), np.float32) if want_aov else None
        stats = RenderStats()
        self.ctx.check(self.ctx.lib.fm_render(self.ctx.h, self.h, C.byref(camera), C.byref(params), _ptr(rgb),
                                              _ptr(alb), _ptr(nrm), 0, C.byref(stats)))
        return rgb, alb, nrm, stats


def parse_scene_file(json_path):
    """Parse-only SceneLoader::Load (no device): returns (status, Camera, RenderParams)."""
    lib = load_library()
    cam = Camera()
    params = RenderParams()
    st = lib.fm_scene_load(None, str(json_path).encode(), None, C.byref(cam), C.byref(params))
    return st, cam, params
