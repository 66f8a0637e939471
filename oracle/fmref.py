"""ctypes wrapper over the oracle libraries (the unmodified reference engine).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / reference arm, as the checker and the CPU baseline; never by the product.

    libfmref_f.so : the reference's float build (USE_FLOAT)
    libfmref_d.so : the reference's double build
Both are compiled by oracle/Makefile from the reference sources (see fmref_harness.cpp).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
LIBS = {"float": REF_DIR / "libfmref_f.so", "double": REF_DIR / "libfmref_d.so"}

_D = C.POINTER(C.c_double)
_cache: dict = {}


def available(precision: str = "float") -> bool:
    return LIBS[precision].exists()


def build(reference_root: str) -> bool:
    """Compile the oracle libraries from the reference checkout at reference_root when
    its sources are present."""
    if not Path(reference_root, "src/engine").exists():
        return available("float") and available("double")
    subprocess.run(["make", "-C", str(HERE), "-j8", "ref", f"REF={reference_root}"], check=True,
                   capture_output=True)
    return True


def lib(precision: str = "float") -> C.CDLL:
    if precision in _cache:
        return _cache[precision]
    path = LIBS[precision]
    if not path.exists():
        raise FileNotFoundError(f"oracle library {path} is missing (run make -C oracle)")
    L = C.CDLL(str(path))
    vp = C.c_void_p
    L.fmref_last_error.restype = C.c_char_p
    L.fmref_precision.restype = C.c_int
    L.fmref_get_max_axis.argtypes = [C.c_double] * 3
    L.fmref_intersect_triangle.argtypes = [_D, _D, _D, _D]
    L.fmref_load.argtypes = [C.c_char_p]
    L.fmref_load.restype = vp
    L.fmref_free.argtypes = [vp]
    L.fmref_num_objects.argtypes = [vp]
    L.fmref_num_objects.restype = C.c_int64
    L.fmref_image_size.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.fmref_trace_closest.argtypes = [vp, _D, C.c_int64, C.POINTER(C.c_int32), _D, C.c_int]
    L.fmref_trace_any.argtypes = [vp, _D, C.c_int64, C.POINTER(C.c_uint8), C.c_int]
    L.fmref_two_nearest.argtypes = [vp, _D, C.c_int64, _D, _D, C.c_int]
    L.fmref_camera_rays.argtypes = [vp, _D, _D, C.c_int64, _D]
    L.fmref_render.argtypes = [vp, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _D, _D, _D, _D, C.c_int,
                               C.c_int, C.c_double, _D, _D]
    L.fmref_draw_frame.argtypes = [vp]
    L.fmref_draw_frame.restype = C.c_double
    L.fmref_load_image.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), _D]
    L.fmref_texture_sample.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, _D, C.c_int64, _D]
    L.fmref_env_pdf.argtypes = [vp, _D, C.c_int64, _D]
    L.fmref_env_radiance.argtypes = [vp, _D, C.c_int64, _D]
    L.fmref_env_sample.argtypes = [vp, _D, C.c_int64, _D]
    L.fmref_bsdf.argtypes = [vp, C.c_char_p, _D, C.c_int64, _D, _D, _D, _D, _D]
    U8 = C.POINTER(C.c_uint8)
    L.fmref_postprocess.argtypes = [C.POINTER(C.c_int), _D, C.c_int, C.c_int, C.c_int, _D, _D, _D, U8, U8, U8]
    _cache[precision] = L
    return L


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


class RefScene:
    """A scene loaded by the reference's SceneLoader."""

    def __init__(self, json_path, precision: str = "float"):
        self.L = lib(precision)
        self.h = self.L.fmref_load(str(json_path).encode())
        if not self.h:
            raise RuntimeError("oracle load failed: " + self.L.fmref_last_error().decode())

    def close(self):
        if self.h:
            self.L.fmref_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def num_objects(self) -> int:
        return int(self.L.fmref_num_objects(self.h))

    def image_size(self):
        w, h, s = C.c_int(), C.c_int(), C.c_int()
        self.L.fmref_image_size(self.h, C.byref(w), C.byref(h), C.byref(s))
        return w.value, h.value, s.value

    def trace_closest(self, rays: np.ndarray, threads: int = 0):
        rays = np.ascontiguousarray(rays, np.float64).reshape(-1, 8)
        n = len(rays)
        obj = np.empty(n, np.int32)
        t = np.empty(n, np.float64)
        self.L.fmref_trace_closest(self.h, _dp(rays), n, obj.ctypes.data_as(C.POINTER(C.c_int32)), _dp(t), threads)
        return obj, t

    def trace_any(self, rays: np.ndarray, threads: int = 0):
        rays = np.ascontiguousarray(rays, np.float64).reshape(-1, 8)
        out = np.empty(len(rays), np.uint8)
        self.L.fmref_trace_any(self.h, _dp(rays), len(rays), out.ctypes.data_as(C.POINTER(C.c_uint8)), threads)
        return out

    def two_nearest(self, rays: np.ndarray, threads: int = 0):
        rays = np.ascontiguousarray(rays, np.float64).reshape(-1, 8)
        t1 = np.empty(len(rays))
        t2 = np.empty(len(rays))
        self.L.fmref_two_nearest(self.h, _dp(rays), len(rays), _dp(t1), _dp(t2), threads)
        return t1, t2

    def camera_rays(self, ndc: np.ndarray, lens: np.ndarray) -> np.ndarray:
        ndc = np.ascontiguousarray(ndc, np.float64)
        lens = np.ascontiguousarray(lens, np.float64)
        out = np.empty((len(ndc), 6))
        self.L.fmref_camera_rays(self.h, _dp(ndc), _dp(lens), len(ndc), _dp(out))
        return out

    def render(self, spp: int, seed: int = 0, tile=None, threads: int = 0, aov: bool = False, clamp: float = 0.0,
               stride: int = 1):
        """Per-pixel sums over `spp` samples: returns dict of (h, w, 3) float64 arrays
        ("csum" / "csumsq": sums of the per-channel clamped sample colours when clamp > 0).
        With stride > 1 only every stride-th pixel of the tile is rendered and the arrays
        are (n, 3) over those pixels."""
        W, H, _ = self.image_size()
        x0, y0, w, h = tile if tile is not None else (0, 0, W, H)
        shape = (h, w, 3) if stride == 1 else ((w * h + stride - 1) // stride, 3)
        s = np.zeros(shape)
        s2 = np.zeros(shape)
        a = np.zeros(shape) if aov else None
        nrm = np.zeros(shape) if aov else None
        cs = np.zeros(shape) if clamp > 0 else None
        cs2 = np.zeros(shape) if clamp > 0 else None
        self.L.fmref_render(self.h, seed, x0, y0, w, h, spp, _dp(s), _dp(s2), _dp(a), _dp(nrm), threads, stride,
                            float(clamp), _dp(cs), _dp(cs2))
        return {"sum": s, "sumsq": s2, "albedo": a, "normal": nrm, "csum": cs, "csumsq": cs2, "spp": spp}

    def draw_frame(self) -> float:
        return float(self.L.fmref_draw_frame(self.h))

    def env_pdf(self, dirs: np.ndarray) -> np.ndarray:
        dirs = np.ascontiguousarray(dirs, np.float64)
        out = np.empty(len(dirs))
        if self.L.fmref_env_pdf(self.h, _dp(dirs), len(dirs), _dp(out)) != 0:
            raise RuntimeError(self.L.fmref_last_error().decode())
        return out

    def env_radiance(self, dirs: np.ndarray) -> np.ndarray:
        dirs = np.ascontiguousarray(dirs, np.float64)
        out = np.empty((len(dirs), 3))
        if self.L.fmref_env_radiance(self.h, _dp(dirs), len(dirs), _dp(out)) != 0:
            raise RuntimeError(self.L.fmref_last_error().decode())
        return out

    def env_sample(self, samples: np.ndarray) -> np.ndarray:
        samples = np.ascontiguousarray(samples, np.float64)
        out = np.empty((len(samples), 4))
        if self.L.fmref_env_sample(self.h, _dp(samples), len(samples), _dp(out)) != 0:
            raise RuntimeError(self.L.fmref_last_error().decode())
        return out

    def bsdf(self, material: str, frame, wi=None, samples=None):
        frame = np.ascontiguousarray(frame, np.float64)
        n = len(wi) if wi is not None else len(samples)
        wi = None if wi is None else np.ascontiguousarray(wi, np.float64)
        samples = None if samples is None else np.ascontiguousarray(samples, np.float64)
        f = np.zeros((n, 3))
        pdf = np.zeros(n)
        sm = np.zeros((n, 8))
        if self.L.fmref_bsdf(self.h, material.encode(), _dp(frame), n, _dp(wi), _dp(samples), _dp(f), _dp(pdf),
                             _dp(sm)) != 0:
            raise RuntimeError(self.L.fmref_last_error().decode())
        return f, pdf, sm


def load_image(path, is_hdr: bool, precision: str = "float") -> np.ndarray:
    L = lib(precision)
    w, h = C.c_int(), C.c_int()
    L.fmref_load_image(str(path).encode(), int(is_hdr), C.byref(w), C.byref(h), None)
    out = np.empty((h.value, w.value, 3))
    L.fmref_load_image(str(path).encode(), int(is_hdr), C.byref(w), C.byref(h), _dp(out))
    return out


def get_max_axis(d, precision: str = "float") -> int:
    return int(lib(precision).fmref_get_max_axis(*map(float, d)))


def intersect_triangle(ray8, v9, precision: str = "float"):
    r = np.ascontiguousarray(ray8, np.float64)
    v = np.ascontiguousarray(v9, np.float64)
    t = C.c_double()
    bc = np.zeros(3)
    hit = lib(precision).fmref_intersect_triangle(_dp(r), _dp(v), C.byref(t), _dp(bc))
    return bool(hit), t.value, bc


# ---- C restatement (oracle/restate/*.c; builds without the reference sources) -------

RESTATE_LIB = REF_DIR / "libfmoracle.so"


def restate() -> C.CDLL:
    """The C restatement library, compiled on first use."""
    if "restate" in _cache:
        return _cache["restate"]
    srcs = list((HERE / "restate").glob("*.c"))
    if not RESTATE_LIB.exists() or any(s.stat().st_mtime > RESTATE_LIB.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(HERE), "restate"], check=True, capture_output=True)
    L = C.CDLL(str(RESTATE_LIB))
    F = C.POINTER(C.c_float)
    L.fmo_get_max_axis.argtypes = [C.c_float] * 3
    L.fmo_intersect_triangle.argtypes = [F, F, F, F]
    L.fmo_closest_bruteforce.argtypes = [F, C.c_int64, F, C.c_int64, C.POINTER(C.c_int32), F]
    L.fmo_closest_bruteforce.restype = None
    L.fmo_intersect_sphere.argtypes = [F, F, C.c_float, F]
    L.fmo_closest_bruteforce_spheres.argtypes = [F, C.c_int64, F, F, C.c_int64, F, C.c_int64, C.POINTER(C.c_int32), F]
    L.fmo_closest_bruteforce_spheres.restype = None
    _cache["restate"] = L
    return L


def restate_closest(tri_pos: np.ndarray, rays: np.ndarray):
    L = restate()
    tri = np.ascontiguousarray(tri_pos, np.float32).reshape(-1, 9)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    prim = np.empty(len(r), np.int32)
    t = np.empty(len(r), np.float32)
    F = C.POINTER(C.c_float)
    L.fmo_closest_bruteforce(tri.ctypes.data_as(F), len(tri), r.ctypes.data_as(F), len(r),
                             prim.ctypes.data_as(C.POINTER(C.c_int32)), t.ctypes.data_as(F))
    return prim, t


def restate_closest_spheres(tri_pos: np.ndarray, centers: np.ndarray, radii: np.ndarray, rays: np.ndarray):
    """Exhaustive closest hit over triangles and translated spheres (prim >= n_tri: sphere
    prim - n_tri)."""
    L = restate()
    tri = np.ascontiguousarray(tri_pos, np.float32).reshape(-1, 9)
    cen = np.ascontiguousarray(centers, np.float32).reshape(-1, 3)
    rad = np.ascontiguousarray(radii, np.float32).reshape(-1)
    r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    prim = np.empty(len(r), np.int32)
    t = np.empty(len(r), np.float32)
    F = C.POINTER(C.c_float)
    L.fmo_closest_bruteforce_spheres(tri.ctypes.data_as(F), len(tri), cen.ctypes.data_as(F), rad.ctypes.data_as(F),
                                     len(rad), r.ctypes.data_as(F), len(r), prim.ctypes.data_as(C.POINTER(C.c_int32)),
                                     t.ctypes.data_as(F))
    return prim, t


def postprocess_u8(steps, rgb, albedo, normal, precision: str = "float"):
    """The reference's post-process chain and 8-bit conversion (fmref_postprocess).
    steps: [(type, lum)] with type 0 tonemapping, 1 linear_to_srgb, 2 srgb_to_linear.
    Returns (rgb8, albedo8, normal8) as h x w x 3 uint8."""
    L = lib(precision)
    h, w, _ = rgb.shape
    types = (C.c_int * max(1, len(steps)))(*[int(t) for t, _ in steps])
    lums = np.asarray([float(l) for _, l in steps] or [0.0], np.float64)
    a = [np.ascontiguousarray(x, np.float64) for x in (rgb, albedo, normal)]
    outs = [np.empty((h, w, 3), np.uint8) for _ in range(3)]
    U8 = C.POINTER(C.c_uint8)
    if L.fmref_postprocess(types, _dp(lums), len(steps), w, h, _dp(a[0]), _dp(a[1]), _dp(a[2]),
                           *[o.ctypes.data_as(U8) for o in outs]) != 0:
        raise RuntimeError(L.fmref_last_error().decode())
    return tuple(outs)
