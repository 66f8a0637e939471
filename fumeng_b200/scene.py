"""Scene specification in the reference's JSON schema, plus its flattened C-ABI form.

A SceneSpec describes one scene the way the reference's SceneLoader reads it
(src/engine/include/engine/create/scene_loader.h:42-276): camera, renderer, materials,
render objects (triangle meshes, rectangles, spheres) and lights.  It can

* write itself as ``scene.json`` + OBJ meshes + Radiance ``.hdr`` textures that the
  reference loads unchanged (``write``), and
* flatten itself into an ``fm_scene_desc`` for ``fm_scene_create`` (``to_desc``),
  with the same object order (render_objects order, one object per mesh face) and the
  same float values the reference sees after parsing those files.

Two schema extensions are written to JSON as well: ``specular_reflection`` materials
(reachable in the reference only via CreateSpecularReflection, create/material.h:11)
and per-vertex Disney attributes.

Float texture data are stored as the values a Radiance RGBE file decodes to
(byte * 2^(e-136), image/stb_image.h hdr reader), so that file and array agree exactly.
"""
from __future__ import annotations

import ctypes as C
import json
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import (FM_CAMERA_PINHOLE, FM_CAMERA_THIN_LENS, FM_FILTER_LINEAR, FM_FILTER_NEAREST, FM_LIGHT_DIRECTIONAL,
               FM_LIGHT_ENV, FM_MAT_DISNEY, FM_MAT_LAMBERT, FM_MAT_SPEC_REFL, FM_MAT_SPEC_TRANS, FM_MODE_WAVEFRONT,
               FM_WRAP_CLAMP, FM_WRAP_REPEAT, MAT_PARAMS, Camera, LightDesc, MaterialDesc, RenderParams, SceneDesc,
               TextureDesc)

# JSON names of the Disney parameters (DisneyConfig, core/material.h:36-76) in MAT_PARAMS order
DISNEY_JSON = ["basecolor", "metallic", "specular", "specularTint", "roughness", "anisotropic", "sheen", "sheenTint",
               "clearcoat", "clearcoatGloss", "specTrans", "specTransRoughness", "diffTrans", "flatness", "ior"]
DISNEY_DEFAULTS = {"specular": 0.5, "ior": 1.5}


# ---- Radiance RGBE ----------------------------------------------------------------

def rgbe_encode(rgb: np.ndarray) -> np.ndarray:
    """float HxWx3 -> uint8 HxWx4 (the encoding of stb_image_write's hdr writer)."""
    rgb = np.asarray(rgb, np.float32)
    m = rgb.max(axis=-1)
    mant, ex = np.frexp(m)
    norm = np.where(m < 1e-32, 0.0, mant.astype(np.float32) * np.float32(256.0) / np.where(m < 1e-32, 1.0, m))
    norm = norm.astype(np.float32)
    out = np.zeros(rgb.shape[:-1] + (4,), np.uint8)
    out[..., :3] = np.clip((rgb * norm[..., None]).astype(np.float32), 0, 255).astype(np.uint8)
    out[..., 3] = np.where(m < 1e-32, 0, ex + 128).astype(np.uint8)
    return out


def rgbe_decode(rgbe: np.ndarray) -> np.ndarray:
    """uint8 HxWx4 -> float32 HxWx3 exactly as stb_image's hdr reader decodes."""
    e = rgbe[..., 3].astype(np.int32)
    f = np.where(e != 0, np.ldexp(np.float32(1.0), e - 136), 0.0).astype(np.float32)
    return (rgbe[..., :3].astype(np.float32) * f[..., None]).astype(np.float32)


def rgbe_quantize(rgb: np.ndarray) -> np.ndarray:
    """Round float radiance to the nearest-below values an .hdr file can hold."""
    return rgbe_decode(rgbe_encode(rgb))


def write_hdr(path: Path, rgb: np.ndarray) -> None:
    """Radiance file with new-style run-length scanlines made of literal runs only (flat
    RGBE pixels when the width is outside [8, 32768), where run-length coding is not
    defined)."""
    h, w, _ = rgb.shape
    enc = rgbe_encode(rgb)
    parts = [b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n", f"-Y {h} +X {w}\n".encode()]
    if not (8 <= w < 32768):
        parts.append(np.ascontiguousarray(enc, np.uint8).tobytes())
        Path(path).write_bytes(b"".join(parts))
        return
    for y in range(h):
        row = [bytes([2, 2, w >> 8, w & 255])]
        for c in range(4):
            data = enc[y, :, c].tobytes()
            for s in range(0, w, 128):
                chunk = data[s:s + 128]
                row.append(bytes([len(chunk)]) + chunk)
        parts.append(b"".join(row))
    Path(path).write_bytes(b"".join(parts))


def write_png8(path: Path, codes01: np.ndarray) -> None:
    """8-bit RGB PNG of values that are multiples of 1/255 (stored as round(255 x))."""
    import struct
    import zlib
    a = np.clip(np.round(np.asarray(codes01, np.float64) * 255.0), 0, 255).astype(np.uint8)
    h, w, _ = a.shape
    raw = b"".join(b"\x00" + a[y].tobytes() for y in range(h))

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xffffffff)
    Path(path).write_bytes(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)) +
                           chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))


def srgb_to_linear(c: np.ndarray) -> np.ndarray:
    """Image::to_linear of a decoded LDR image (utils.h SrgbToLinear), in float32."""
    c = np.asarray(c, np.float32)
    lo = c * np.float32(1.0 / 12.92)
    hi = np.power((c + np.float32(0.055)) * np.float32(1.0 / 1.055), np.float32(2.4)).astype(np.float32)
    return np.where(c <= np.float32(0.04045), lo, hi).astype(np.float32)


# ---- transforms ---------------------------------------------------------------------

def trs_matrix(translation, rotation_deg, scale) -> np.ndarray:
    """Transform(translation, rotation, scale) (math/transform.cpp:17-25): T * Rz*Ry*Rx * S,
    row-major 4x4 in double."""
    def rot(axis, deg):
        a = deg / 180.0 * 3.14159265354
        c, s = math.cos(a), math.sin(a)
        R = np.eye(4)
        i, j = [(1, 2), (2, 0), (0, 1)][axis]
        R[i, i] = c
        R[i, j] = -s
        R[j, i] = s
        R[j, j] = c
        return R
    T = np.eye(4)
    T[:3, 3] = translation
    S = np.diag([scale[0], scale[1], scale[2], 1.0])
    return T @ rot(2, rotation_deg[2]) @ rot(1, rotation_deg[1]) @ rot(0, rotation_deg[0]) @ S


def f32(x) -> float:
    return float(np.float32(x))


def fmt(x) -> str:
    return "%.9g" % float(np.float32(x))


# ---- spec -------------------------------------------------------------------------

@dataclass
class Mesh:
    vertices: np.ndarray            # V x 3 float32 (world space; written with no transform)
    faces: np.ndarray               # F x 3 int (0-based)
    material: str = "default_material"
    emittance: tuple | None = None
    uvs: np.ndarray | None = None   # V x 2 (OBJ vt); the reference flips v
    normals: np.ndarray | None = None   # V x 3 (OBJ vn)
    vattr: np.ndarray | None = None     # V x K per-vertex attributes (extension)


@dataclass
class Rect:
    pa: tuple
    pb: tuple
    pc: tuple
    pd: tuple
    material: str = "default_material"
    emittance: tuple | None = None


@dataclass
class Sphere:
    radius: float
    translation: tuple = (0.0, 0.0, 0.0)
    rotation: tuple = (0.0, 0.0, 0.0)
    scale: tuple = (1.0, 1.0, 1.0)
    material: str = "default_material"
    emittance: tuple | None = None


def camera_struct(c: dict) -> Camera:
    """fm_camera from a camera dict in the reference's JSON schema."""
    cam = Camera()
    cam.type = FM_CAMERA_THIN_LENS if c.get("type", "pin_hole") == "thin_lens" else FM_CAMERA_PINHOLE
    cam.pos = _f3(c.get("pos", [0, 0, 0]))
    cam.look_at = _f3(c.get("look_at", [0, 0, 0]))
    cam.up = _f3(c.get("up", [0, 0, 1]))
    cam.fov = f32(c.get("fov", 60.0))
    cam.aspect = f32(c.get("aspect", 1.0))
    cam.focal_distance = f32(c.get("focal_distance", 1.0))
    cam.lens_radius = f32(c.get("lens_radius", 0.0))
    return cam


@dataclass
class SceneSpec:
    camera: dict
    renderer: dict
    materials: list = field(default_factory=list)   # dicts in the reference's material schema
    objects: list = field(default_factory=list)     # Mesh | Rect | Sphere
    lights: list = field(default_factory=list)      # dicts: env {texture, rotation, factor} | directional
    textures: dict = field(default_factory=dict)    # name -> HxWx3 float32 (RGBE-representable)
    # textures stored as 8-bit sRGB PNG files: their arrays hold the sRGB codes / 255, and
    # the scene decodes them to linear values as the reference's Image loader does
    ldr_textures: set = field(default_factory=set)
    # "bvh" (the reference's built-in BVH: every emissive triangle is its own light) or
    # "embree" (each emissive mesh is one light sampled by area, as the reference's Embree
    # meshes; the device BVH serves both)
    accelerator: str = "bvh"

    # -- derived ---------------------------------------------------------------------
    def material_index(self) -> dict:
        names = {}
        for m in self.materials:
            names.setdefault(m["name"], len(names))
        return names

    def num_objects(self) -> int:
        return sum(len(o.faces) if isinstance(o, Mesh) else 1 for o in self.objects)

    # -- JSON + files ------------------------------------------------------------------
    def write(self, root: Path, output: str = "out") -> Path:
        root = Path(root)
        root.mkdir(parents=True, exist_ok=True)
        tex_files = {}
        for name, arr in self.textures.items():
            if name in self.ldr_textures:
                fn = f"tex_{name}.png"
                write_png8(root / fn, arr)
            else:
                fn = f"tex_{name}.hdr"
                write_hdr(root / fn, arr)
            tex_files[name] = fn

        def tex_json(v):
            if isinstance(v, dict) and "image" in v:
                return {"type": "image", "path": tex_files[v["image"]], "sampler": v.get("sampler", "linear"),
                        "wrap_u": v.get("wrap_u", "repeat"), "wrap_v": v.get("wrap_v", "repeat")}
            vals = [v] if np.isscalar(v) else list(v)
            return {"type": "constant", "value": [float(fmt(x)) for x in vals]}

        mats = []
        for m in self.materials:
            t = m["type"]
            j = {"name": m["name"], "type": t}
            if t == "lambert_diffuse":
                j["basecolor"] = tex_json(m.get("basecolor", [1, 1, 1]))
            elif t == "disney":
                for k in DISNEY_JSON:
                    if k in m:
                        j[k] = tex_json(m[k])
                j["thin"] = bool(m.get("thin", False))
                if "vattr_offset" in m:
                    j["vertex_attributes"] = {"offset": m["vattr_offset"]}
            elif t == "specular_transmission":
                for k in ("reflect_color", "refract_color"):
                    j[k] = [float(fmt(x)) for x in m.get(k, [1, 1, 1])]
                j["eta_i"] = float(fmt(m["eta_i"]))
                j["eta_t"] = float(fmt(m["eta_t"]))
            elif t == "specular_reflection":
                for k, d in (("color", [1, 1, 1]), ("eta_i", [1, 1, 1]), ("eta_t", [1, 1, 1]), ("k", [0, 0, 0])):
                    j[k] = [float(fmt(x)) for x in m.get(k, d)]
            mats.append(j)
        objs = []
        for i, o in enumerate(self.objects):
            extra = {}
            if isinstance(o, Mesh):
                fn = f"mesh_{i}.obj"
                self._write_obj(root / fn, o)
                shape = {"type": "triangle_mesh", "path": fn}
                if o.vattr is not None:
                    # per-vertex attributes (extension): raw float32, V x dim
                    va = np.ascontiguousarray(o.vattr, np.float32)
                    (root / f"mesh_{i}.vattr").write_bytes(va.tobytes())
                    extra["fm_vertex_attributes"] = {"path": f"mesh_{i}.vattr", "dim": int(va.shape[1])}
            elif isinstance(o, Rect):
                shape = {"type": "rectangle", **{k: [float(fmt(x)) for x in getattr(o, k)] for k in ("pa", "pb", "pc", "pd")}}
            else:
                shape = {"type": "sphere", "radius": float(fmt(o.radius)), "translation": [float(fmt(x)) for x in o.translation],
                         "rotation": [float(fmt(x)) for x in o.rotation], "scale": [float(fmt(x)) for x in o.scale]}
            e = {"shape": shape, "material": o.material, **extra}
            if o.emittance is not None:
                e["emittance"] = [float(fmt(x)) for x in o.emittance]
            objs.append(e)
        lights = []
        for l in self.lights:
            if l["type"] == "env":
                lights.append({"type": "env", "path": tex_files[l["texture"]], "rotation": list(l.get("rotation", [0, 0, 0])),
                               "factor": float(fmt(l.get("factor", 1.0)))})
            else:
                lights.append({"type": "directional", "radiance": list(l["radiance"]), "direction": list(l["direction"])})
        cam = {k: v for k, v in self.camera.items()}
        ren = {"type": "path_tracer", "thread_count": 8, "output": output, **self.renderer}
        doc = {"camera": cam, "renderer": ren,
               "scene": {"accelerator": {"type": self.accelerator}, "materials": mats, "render_objects": objs,
                         "lights": lights}}
        p = root / "scene.json"
        p.write_text(json.dumps(doc, indent=1))
        return p

    @staticmethod
    def _write_obj(path: Path, m: Mesh) -> None:
        v = np.asarray(m.vertices, np.float32)
        lines = ["v %s %s %s" % (fmt(a), fmt(b), fmt(c)) for a, b, c in v]
        if m.uvs is not None:
            lines += ["vt %s %s" % (fmt(a), fmt(b)) for a, b in np.asarray(m.uvs, np.float32)]
        if m.normals is not None:
            lines += ["vn %s %s %s" % (fmt(a), fmt(b), fmt(c)) for a, b, c in np.asarray(m.normals, np.float32)]
        f = np.asarray(m.faces, np.int64) + 1
        if m.uvs is not None and m.normals is not None:
            lines += ["f %d/%d/%d %d/%d/%d %d/%d/%d" % (a, a, a, b, b, b, c, c, c) for a, b, c in f]
        elif m.uvs is not None:
            lines += ["f %d/%d %d/%d %d/%d" % (a, a, b, b, c, c) for a, b, c in f]
        elif m.normals is not None:
            lines += ["f %d//%d %d//%d %d//%d" % (a, a, b, b, c, c) for a, b, c in f]
        else:
            lines += ["f %d %d %d" % (a, b, c) for a, b, c in f]
        Path(path).write_text("\n".join(lines) + "\n")

    # -- C-ABI form ----------------------------------------------------------------------
    def to_desc(self) -> "DescHolder":
        return DescHolder(self)

    def camera_struct(self) -> Camera:
        return camera_struct(self.camera)

    def render_params(self, spp: int | None = None, seed: int = 0, mode: int = FM_MODE_WAVEFRONT,
                      sample_offset: int = 0, clamp: float = 0.0, region=None) -> RenderParams:
        r = self.renderer
        p = RenderParams()
        p.width = int(r.get("width", 1))
        p.height = int(r.get("height", 1))
        p.spp = int(spp if spp is not None else r.get("spp", 10))
        p.depth = int(r.get("depth", 10))
        p.direct_loop = int(r.get("direct_loop", 1))
        p.rr_depth = int(r.get("rr_depth", 10))
        p.rr_coef = f32(r.get("rr_coef", 0.85))
        p.seed = seed
        p.mode = mode
        p.sample_offset = sample_offset
        p.max_sample_value = clamp
        if region is not None:
            p.region_x, p.region_y, p.region_w, p.region_h = (int(v) for v in region)
        return p


def _f3(v) -> C.Array:
    v = list(v)
    if len(v) < 3:
        v = [v[0]] * 3
    return (C.c_float * 3)(*[f32(x) for x in v[:3]])


def _normalize_f32(n: np.ndarray) -> np.ndarray:
    n = n.astype(np.float32)
    d = (n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1]).astype(np.float32) + n[:, 2] * n[:, 2]
    inv = (np.float32(1.0) / np.sqrt(d.astype(np.float32))).astype(np.float32)
    return (n * inv[:, None]).astype(np.float32)


class DescHolder:
    """Owns the numpy arrays behind an fm_scene_desc built from a SceneSpec."""

    def __init__(self, spec: SceneSpec):
        self.spec = spec
        mat_idx = spec.material_index()
        if "default_material" not in mat_idx:
            mat_idx["default_material"] = len(mat_idx)
        tex_names = list(spec.textures)
        tex_idx = {n: i for i, n in enumerate(tex_names)}
        self.texture_index = tex_idx            # texture name -> scene texture index
        self.material_index = mat_idx           # material name -> scene material index
        self.num_materials = len(mat_idx)
        keep = []
        # objects
        obj_mat, obj_em = [], []
        tri_pos, tri_uv, tri_nrm, tri_obj, tri_vattr = [], [], [], [], []
        rect_pts, rect_obj = [], []
        sph_r, sph_x, sph_obj = [], [], []
        any_uv = any(isinstance(o, Mesh) and o.uvs is not None for o in spec.objects)
        any_nrm = any(isinstance(o, Mesh) and o.normals is not None for o in spec.objects)
        vdim = max([o.vattr.shape[1] for o in spec.objects if isinstance(o, Mesh) and o.vattr is not None] or [0])
        has_nrm = []
        light_group = []
        n_mesh = 0
        obj = 0
        for o in spec.objects:
            em = list(o.emittance) if o.emittance is not None else [0.0, 0.0, 0.0]
            m = mat_idx.get(o.material, mat_idx["default_material"])
            if isinstance(o, Mesh):
                v = np.asarray(o.vertices, np.float32)
                f = np.asarray(o.faces, np.int64)
                nf = len(f)
                tri_pos.append(v[f].reshape(nf, 9))
                light_group.append(np.full(nf, n_mesh, np.int32))
                n_mesh += 1
                if any_uv:
                    if o.uvs is not None:
                        uv = np.asarray(o.uvs, np.float32).copy()
                        uv[:, 1] = (np.float32(1.0) - uv[:, 1]).astype(np.float32)
                        tri_uv.append(uv[f].reshape(nf, 6))
                    else:
                        tri_uv.append(np.zeros((nf, 6), np.float32))
                if any_nrm:
                    if o.normals is not None:
                        tri_nrm.append(_normalize_f32(np.asarray(o.normals, np.float32))[f].reshape(nf, 9))
                        has_nrm.append(np.ones(nf, np.uint8))
                    else:
                        tri_nrm.append(np.zeros((nf, 9), np.float32))
                        has_nrm.append(np.zeros(nf, np.uint8))
                if vdim:
                    va = np.zeros((len(v), vdim), np.float32)
                    if o.vattr is not None:
                        va[:, :o.vattr.shape[1]] = o.vattr
                    tri_vattr.append(va[f].reshape(nf, 3 * vdim))
                tri_obj.append(np.arange(obj, obj + nf, dtype=np.int32))
                obj_mat += [m] * nf
                obj_em += [em] * nf
                obj += nf
            elif isinstance(o, Rect):
                rect_pts.append(np.array([o.pa, o.pb, o.pc, o.pd], np.float32).reshape(12))
                rect_obj.append(obj)
                obj_mat.append(m)
                obj_em.append(em)
                obj += 1
            else:
                sph_r.append(f32(o.radius))
                sph_x.append(trs_matrix(o.translation, o.rotation, o.scale).astype(np.float32).reshape(16))
                sph_obj.append(obj)
                obj_mat.append(m)
                obj_em.append(em)
                obj += 1

        def arr(lst, dtype, width):
            return np.ascontiguousarray(np.concatenate(lst) if lst else np.zeros((0, width)), dtype=dtype)

        self.obj_material = np.asarray(obj_mat, np.int32)
        self.obj_emission = np.asarray(obj_em, np.float32).reshape(-1, 3)
        self.tri_pos = arr(tri_pos, np.float32, 9)
        self.tri_uv = arr(tri_uv, np.float32, 6) if any_uv else None
        self.tri_normal = arr(tri_nrm, np.float32, 9) if any_nrm else None
        self.tri_has_normal = np.ascontiguousarray(np.concatenate(has_nrm)) if any_nrm else None
        self.tri_vattr = arr(tri_vattr, np.float32, 3 * vdim) if vdim else None
        self.tri_object = np.ascontiguousarray(np.concatenate(tri_obj) if tri_obj else np.zeros(0), np.int32)
        self.rect_pts = np.asarray(rect_pts, np.float32).reshape(-1, 12)
        self.rect_object = np.asarray(rect_obj, np.int32)
        self.sphere_radius = np.asarray(sph_r, np.float32)
        self.sphere_xform = np.asarray(sph_x, np.float32).reshape(-1, 16)
        self.sphere_object = np.asarray(sph_obj, np.int32)

        # textures
        self.tex_arrays = [np.ascontiguousarray(srgb_to_linear(spec.textures[n]) if n in spec.ldr_textures
                                                else spec.textures[n], np.float32) for n in tex_names]
        self.textures = (TextureDesc * max(1, len(tex_names)))()
        for i, a in enumerate(self.tex_arrays):
            self.textures[i].width = a.shape[1]
            self.textures[i].height = a.shape[0]
            self.textures[i].texels = a.ctypes.data_as(C.POINTER(C.c_float))
            self.textures[i].wrap_u = FM_WRAP_REPEAT
            self.textures[i].wrap_v = FM_WRAP_REPEAT
            self.textures[i].filter = FM_FILTER_LINEAR
        image_sampler = {}

        def texref(v, channel_default=None):
            r = TexRef_()
            if isinstance(v, dict) and "image" in v:
                r.texture = tex_idx[v["image"]]
                r.value = _f3([0, 0, 0])
                image_sampler[r.texture] = v
            else:
                r.texture = -1
                r.value = _f3([v] if np.isscalar(v) else v)
            return r

        from . import TexRef as TexRef_
        n_mat = len(mat_idx)
        self.materials = (MaterialDesc * n_mat)()
        by_name = {m["name"]: m for m in spec.materials}
        for name, i in mat_idx.items():
            m = by_name.get(name, {"type": "lambert_diffuse", "basecolor": [1, 1, 1]})
            M = self.materials[i]
            M.vattr_offset = -1
            for p in MAT_PARAMS:
                setattr(M, p, texref(0.0))
            t = m["type"]
            if t == "lambert_diffuse":
                M.type = FM_MAT_LAMBERT
                M.basecolor = texref(m.get("basecolor", [1, 1, 1]))
            elif t == "disney":
                M.type = FM_MAT_DISNEY
                M.thin = 1 if m.get("thin", False) else 0
                for p, jn in zip(MAT_PARAMS, DISNEY_JSON):
                    setattr(M, p, texref(m.get(jn, DISNEY_DEFAULTS.get(jn, 0.0))))
                M.vattr_offset = int(m.get("vattr_offset", -1))
            elif t == "specular_transmission":
                M.type = FM_MAT_SPEC_TRANS
                M.reflect_color = _f3(m.get("reflect_color", [1, 1, 1]))
                M.refract_color = _f3(m.get("refract_color", [1, 1, 1]))
                M.eta_i = f32(m["eta_i"])
                M.eta_t = f32(m["eta_t"])
            elif t == "specular_reflection":
                M.type = FM_MAT_SPEC_REFL
                M.color = _f3(m.get("color", [1, 1, 1]))
                M.cond_eta_i = _f3(m.get("eta_i", [1, 1, 1]))
                M.cond_eta_t = _f3(m.get("eta_t", [1, 1, 1]))
                M.cond_k = _f3(m.get("k", [0, 0, 0]))
            else:
                raise ValueError(f"material type {t}")
        for ti, v in image_sampler.items():
            self.textures[ti].filter = FM_FILTER_NEAREST if v.get("sampler", "linear") == "nearest" else FM_FILTER_LINEAR
            self.textures[ti].wrap_u = FM_WRAP_CLAMP if v.get("wrap_u", "repeat") == "clamp" else FM_WRAP_REPEAT
            self.textures[ti].wrap_v = FM_WRAP_CLAMP if v.get("wrap_v", "repeat") == "clamp" else FM_WRAP_REPEAT
        # lights
        self.lights = (LightDesc * max(1, len(spec.lights)))()
        for i, l in enumerate(spec.lights):
            L = self.lights[i]
            if l["type"] == "env":
                L.type = FM_LIGHT_ENV
                L.texture = tex_idx[l["texture"]]
                L.rotation = _f3(l.get("rotation", [0, 0, 0]))
                L.factor = f32(l.get("factor", 1.0))
            else:
                L.type = FM_LIGHT_DIRECTIONAL
                L.radiance = _f3(l["radiance"])
                d = np.asarray(l["direction"], np.float32)
                d = _normalize_f32(d[None])[0]
                L.direction = _f3(d)
        d = SceneDesc()
        fp = C.POINTER(C.c_float)
        ip = C.POINTER(C.c_int32)
        d.num_objects = obj
        d.obj_material = self.obj_material.ctypes.data_as(ip)
        d.obj_emission = self.obj_emission.ctypes.data_as(fp)
        d.num_triangles = len(self.tri_object)
        d.tri_pos = self.tri_pos.ctypes.data_as(fp)
        d.tri_normal = self.tri_normal.ctypes.data_as(fp) if self.tri_normal is not None else None
        d.tri_has_normal = (self.tri_has_normal.ctypes.data_as(C.POINTER(C.c_uint8))
                            if self.tri_has_normal is not None else None)
        d.tri_uv = self.tri_uv.ctypes.data_as(fp) if self.tri_uv is not None else None
        d.tri_object = self.tri_object.ctypes.data_as(ip)
        d.tri_vattr = self.tri_vattr.ctypes.data_as(fp) if self.tri_vattr is not None else None
        d.vattr_dim = vdim
        d.num_rects = len(self.rect_object)
        d.rect_pts = self.rect_pts.ctypes.data_as(fp)
        d.rect_object = self.rect_object.ctypes.data_as(ip)
        d.num_spheres = len(self.sphere_object)
        d.sphere_radius = self.sphere_radius.ctypes.data_as(fp)
        d.sphere_xform = self.sphere_xform.ctypes.data_as(fp)
        d.sphere_object = self.sphere_object.ctypes.data_as(ip)
        d.num_materials = n_mat
        d.materials = self.materials
        d.num_textures = len(tex_names)
        d.textures = self.textures
        d.num_lights = len(spec.lights)
        d.lights = self.lights
        # "embree": one light per emissive mesh (its triangles share the mesh's ordinal)
        self.tri_light_group = (np.ascontiguousarray(np.concatenate(light_group), np.int32)
                                if spec.accelerator == "embree" and light_group else None)
        d.tri_light_group = self.tri_light_group.ctypes.data_as(ip) if self.tri_light_group is not None else None
        self.desc = d
        self._keep = keep
