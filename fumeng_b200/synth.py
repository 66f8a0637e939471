"""Seeded synthetic workloads (the reference ships no scenes; its scene submodule is empty).

Generators for the benchmark configurations:
  cornell()        Cornell box, 5 walls + 2 spheres + area light (256x256, 16 spp, depth 5)
  icosphere_mesh() icosphere subdivided `level` times, displaced by 0.05 * fBm of
                   Perlin's improved noise (Perlin 2002), 6 octaves
  sky_env()        HDR sky gradient x lognormal(0, 0.3) noise + a Gaussian sun lobe
  single_mesh()    1.31M-triangle icosphere with per-vertex Disney parameters, thin lens
  batch_scenes()   64 scenes of 1-40 displaced icospheres / subdivided boxes
  hit_scene()      meshes + rectangles for hit-ID parity tests, with random rays
All randomness comes from numpy Generators seeded by the caller.
"""
from __future__ import annotations

import math

import numpy as np

from .scene import Mesh, Rect, SceneSpec, Sphere, rgbe_quantize

# ---- geometry -------------------------------------------------------------------------


def icosahedron():
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], np.int64)
    return v, f


def subdivide(v: np.ndarray, f: np.ndarray):
    """One loop of midpoint subdivision projected to the unit sphere (20*4^L faces)."""
    e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
    es = np.sort(e, axis=1)
    uniq, inv = np.unique(es, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    mid = v[uniq[:, 0]] + v[uniq[:, 1]]
    mid /= np.linalg.norm(mid, axis=1, keepdims=True)
    base = len(v)
    nf = len(f)
    m01 = base + inv[:nf]
    m12 = base + inv[nf:2 * nf]
    m20 = base + inv[2 * nf:]
    a, b, c = f[:, 0], f[:, 1], f[:, 2]
    nf_ = np.concatenate([np.stack([a, m01, m20], 1), np.stack([b, m12, m01], 1), np.stack([c, m20, m12], 1),
                          np.stack([m01, m12, m20], 1)])
    return np.concatenate([v, mid]), nf_


def icosphere(level: int):
    v, f = icosahedron()
    for _ in range(level):
        v, f = subdivide(v, f)
    return v, f


class PerlinNoise:
    """Perlin's improved noise (K. Perlin, "Improving Noise", SIGGRAPH 2002): quintic fade,
    12 edge gradients selected by a hashed permutation table (seeded here)."""

    GRAD = np.array([[1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1], [-1, 0, -1],
                     [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1], [1, 1, 0], [0, -1, 1], [-1, 1, 0], [0, -1, -1]],
                    np.float64)

    def __init__(self, seed: int):
        p = np.random.default_rng(seed).permutation(256)
        self.p = np.concatenate([p, p]).astype(np.int64)

    @staticmethod
    def _fade(t):
        return t * t * t * (t * (t * 6 - 15) + 10)

    def __call__(self, x, y, z):
        X, Y, Z = np.floor(x).astype(np.int64) & 255, np.floor(y).astype(np.int64) & 255, np.floor(z).astype(np.int64) & 255
        x, y, z = x - np.floor(x), y - np.floor(y), z - np.floor(z)
        u, v, w = self._fade(x), self._fade(y), self._fade(z)
        p = self.p
        A, B = p[X] + Y, p[X + 1] + Y
        AA, AB, BA, BB = p[A] + Z, p[A + 1] + Z, p[B] + Z, p[B + 1] + Z

        def g(h, dx, dy, dz):
            G = self.GRAD[h & 15]
            return G[..., 0] * dx + G[..., 1] * dy + G[..., 2] * dz

        def lerp(t, a, b):
            return a + t * (b - a)
        return lerp(w, lerp(v, lerp(u, g(p[AA], x, y, z), g(p[BA], x - 1, y, z)),
                            lerp(u, g(p[AB], x, y - 1, z), g(p[BB], x - 1, y - 1, z))),
                    lerp(v, lerp(u, g(p[AA + 1], x, y, z - 1), g(p[BA + 1], x - 1, y, z - 1)),
                         lerp(u, g(p[AB + 1], x, y - 1, z - 1), g(p[BB + 1], x - 1, y - 1, z - 1))))

    def fbm(self, P: np.ndarray, octaves=6, lacunarity=2.0, gain=0.5, freq=2.0):
        out = np.zeros(len(P))
        amp = 1.0
        for _ in range(octaves):
            out += amp * self(P[:, 0] * freq, P[:, 1] * freq, P[:, 2] * freq)
            freq *= lacunarity
            amp *= gain
        return out


def displaced_icosphere(level: int, seed: int, amp: float = 0.05):
    v, f = icosphere(level)
    n = PerlinNoise(seed).fbm(v)
    return v * (1.0 + amp * n)[:, None], f


def subdivided_box(n: int):
    """Unit cube [-1,1]^3 with each face split into n x n quads (12 n^2 triangles)."""
    verts, faces = [], []
    g = np.linspace(-1.0, 1.0, n + 1)
    for axis in range(3):
        for sign in (-1.0, 1.0):
            uu, vv = np.meshgrid(g, g, indexing="ij")
            P = np.zeros((n + 1, n + 1, 3))
            a1, a2 = (axis + 1) % 3, (axis + 2) % 3
            P[..., axis] = sign
            P[..., a1] = uu
            P[..., a2] = vv
            base = sum(len(x) for x in verts)
            verts.append(P.reshape(-1, 3))
            idx = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1) + base
            q0, q1, q2, q3 = idx[:-1, :-1], idx[1:, :-1], idx[1:, 1:], idx[:-1, 1:]
            if sign > 0:
                t1 = np.stack([q0, q1, q2], -1)
                t2 = np.stack([q0, q2, q3], -1)
            else:
                t1 = np.stack([q0, q2, q1], -1)
                t2 = np.stack([q0, q3, q2], -1)
            faces.append(np.concatenate([t1.reshape(-1, 3), t2.reshape(-1, 3)]))
    return np.concatenate(verts), np.concatenate(faces)


# ---- environment maps ---------------------------------------------------------------


def sky_env(w: int, h: int, seed: int, sun_dir=(0.4, 0.3, 0.866), sun_peak=5e4, sun_sigma_deg=0.5) -> np.ndarray:
    """z-up lat-long HDR (row 0 = zenith): sky gradient x lognormal(0, 0.3) + sun lobe."""
    rng = np.random.default_rng(seed)
    j = (np.arange(h) + 0.5) / h
    i = (np.arange(w) + 0.5) / w
    theta = j * math.pi
    phi = i * 2 * math.pi
    TH, PH = np.meshgrid(theta, phi, indexing="ij")
    d = np.stack([np.sin(TH) * np.cos(PH), np.sin(TH) * np.sin(PH), np.cos(TH)], -1)
    up = np.clip(d[..., 2], -1, 1)
    zen = np.array([0.25, 0.45, 1.0])
    hor = np.array([0.9, 0.85, 0.8])
    gnd = np.array([0.25, 0.22, 0.2])
    t = np.clip(up, 0, 1)[..., None]
    sky = np.where(up[..., None] >= 0, hor * (1 - t) + zen * t, gnd * (0.6 + 0.4 * (1 + up[..., None])))
    noise = rng.lognormal(0.0, 0.3, size=(h, w, 1))
    s = np.asarray(sun_dir, np.float64)
    s /= np.linalg.norm(s)
    ang = np.arccos(np.clip((d * s).sum(-1), -1, 1))
    sig = math.radians(sun_sigma_deg)
    sun = sun_peak * np.exp(-0.5 * (ang / sig) ** 2)
    img = sky * noise + sun[..., None] * np.array([1.0, 0.95, 0.85])
    return rgbe_quantize(img.astype(np.float32))


# ---- scenes -------------------------------------------------------------------------


def cornell(res: int = 256, spp: int = 16, depth: int = 5, rr_depth: int = 3) -> SceneSpec:
    """Cornell box in [0,1]^3, camera at (0.5,0.5,-1.4) looking at the centre."""
    cam = {"type": "pin_hole", "pos": [0.5, 0.5, -1.4], "look_at": [0.5, 0.5, 0.5], "up": [0, 1, 0], "fov": 40.0,
           "aspect": 1.0}
    ren = {"width": res, "height": res, "spp": spp, "depth": depth, "rr_depth": rr_depth, "rr_coef": 0.85}
    mats = [
        {"name": "white", "type": "lambert_diffuse", "basecolor": [0.73, 0.73, 0.73]},
        {"name": "red", "type": "lambert_diffuse", "basecolor": [0.65, 0.05, 0.05]},
        {"name": "green", "type": "lambert_diffuse", "basecolor": [0.12, 0.45, 0.15]},
        {"name": "ball", "type": "lambert_diffuse", "basecolor": [0.8, 0.8, 0.8]},
        # aluminium-like conductor
        {"name": "mirror", "type": "specular_reflection", "color": [1, 1, 1], "eta_i": [1, 1, 1],
         "eta_t": [1.66, 0.88, 0.52], "k": [9.2, 6.3, 4.8]},
        {"name": "light", "type": "lambert_diffuse", "basecolor": [0.78, 0.78, 0.78]},
    ]
    objs = [
        Rect((0, 0, 0), (0, 0, 1), (1, 0, 1), (1, 0, 0), "white"),            # floor  (normal +y)
        Rect((0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1), "white"),            # ceiling (normal -y)
        Rect((0, 0, 1), (0, 1, 1), (1, 1, 1), (1, 0, 1), "white"),            # back (normal -z)
        Rect((0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1), "red"),              # left x=0 (normal +x)
        Rect((1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0), "green"),            # right x=1 (normal -x)
        Sphere(0.15, translation=(0.3, 0.15, 0.4), material="ball"),
        Sphere(0.15, translation=(0.7, 0.15, 0.6), material="mirror"),
        Rect((0.375, 0.999, 0.375), (0.625, 0.999, 0.375), (0.625, 0.999, 0.625), (0.375, 0.999, 0.625), "light",
             emittance=(17.0, 12.0, 4.0)),                                     # normal -y
    ]
    return SceneSpec(cam, ren, mats, objs)


def random_rays(rng: np.random.Generator, n: int, lo, hi, min_component: float = 1e-3) -> np.ndarray:
    """Rays with origins uniform in the box [lo, hi] and isotropic directions whose
    components are all at least `min_component` in magnitude.  Layout n x 8:
    ox oy oz tmin dx dy dz tmax (tmin 0, tmax FLT_MAX)."""
    o = rng.uniform(lo, hi, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    small = np.abs(d) < min_component
    d[small] = np.sign(d[small] + 1e-30) * min_component
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = o
    r[:, 4:7] = d
    r[:, 3] = 0.0
    r[:, 7] = np.finfo(np.float32).max
    return r


def hit_scene(seed: int, level: int = 4, boxes: int = 3, spheres: int = 0) -> SceneSpec:
    """Displaced icosphere + subdivided boxes + a few rectangles, identity transforms,
    and `spheres` analytic spheres with translation-only transforms (drawn after
    everything else, so spheres=0 reproduces the earlier scenes exactly)."""
    rng = np.random.default_rng(seed)
    objs = []
    v, f = displaced_icosphere(level, seed)
    objs.append(Mesh((v * 0.8).astype(np.float32), f, "m0"))
    for b in range(boxes):
        bv, bf = subdivided_box(4 + b)
        s = rng.uniform(0.15, 0.35)
        c = rng.uniform(-1.2, 1.2, size=3)
        objs.append(Mesh((bv * s + c).astype(np.float32), bf, "m0"))
    objs.append(Rect((-2, -1.5, -2), (-2, -1.5, 2), (2, -1.5, 2), (2, -1.5, -2), "m0"))
    objs.append(Rect((-2, -2, 1.9), (2, -2, 1.9), (2, 2, 1.9), (-2, 2, 1.9), "m0"))
    for _ in range(spheres):
        r = float(np.float32(rng.uniform(0.1, 0.45)))
        c = tuple(float(x) for x in rng.uniform(-1.4, 1.4, size=3).astype(np.float32))
        objs.append(Sphere(r, translation=c, material="m0"))
    cam = {"type": "pin_hole", "pos": [0, 0, -4], "look_at": [0, 0, 0], "up": [0, 1, 0], "fov": 45.0, "aspect": 1.0}
    ren = {"width": 64, "height": 64, "spp": 1, "depth": 4}
    mats = [{"name": "m0", "type": "lambert_diffuse", "basecolor": [0.5, 0.5, 0.5]}]
    return SceneSpec(cam, ren, mats, objs)


def single_mesh_hit_scene(level: int = 8) -> SceneSpec:
    """The single-mesh configuration's geometry alone (the displaced icosphere of
    single_mesh_scene, 1,310,720 triangles at level 8, mesh seed 1) with a Lambert
    material, for closest-hit queries."""
    v, f = displaced_icosphere(level, 1, amp=0.05)
    cam = {"type": "pin_hole", "pos": [0.0, -4.0, 0.6], "look_at": [0.0, 0.0, 0.0], "up": [0, 0, 1], "fov": 40.0,
           "aspect": 16 / 9}
    ren = {"width": 64, "height": 36, "spp": 1, "depth": 4}
    mats = [{"name": "m0", "type": "lambert_diffuse", "basecolor": [0.5, 0.5, 0.5]}]
    return SceneSpec(cam, ren, mats, [Mesh(v.astype(np.float32), f, "m0")])


def pinhole_rays(rng: np.random.Generator, camera: dict, nx: int, ny: int) -> np.ndarray:
    """Primary rays of a pinhole camera: one jittered ray per cell of an nx x ny film
    grid, direction = normalize(f + (2x-1) tan(fov/2) aspect s + (2y-1) tan(fov/2) u)
    with the camera's forward f, side s and up u; computed in float64 and stored as
    float32 (n x 8, tmin 0, tmax FLT_MAX).  Coherent rays for the closest-hit tests."""
    pos = np.asarray(camera["pos"], np.float64)
    f = np.asarray(camera["look_at"], np.float64) - pos
    f /= np.linalg.norm(f)
    up = np.asarray(camera.get("up", [0, 0, 1]), np.float64)
    s = np.cross(up, f)
    s /= np.linalg.norm(s)
    u = np.cross(f, s)
    th = np.tan(np.radians(float(camera.get("fov", 60.0))) / 2.0)
    asp = float(camera.get("aspect", 1.0))
    gx, gy = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    x = (gx.ravel() + rng.random(nx * ny)) / nx
    y = (gy.ravel() + rng.random(nx * ny)) / ny
    d = f[None] + ((2 * x - 1) * th * asp)[:, None] * s[None] + ((2 * y - 1) * th)[:, None] * u[None]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((nx * ny, 8), np.float32)
    r[:, 0:3] = pos
    r[:, 4:7] = d
    r[:, 7] = np.finfo(np.float32).max
    return r


def textured_scene(res: int = 48, spp: int = 16, depth: int = 5) -> SceneSpec:
    """Image textures in every form the reference's ImageTexture has: a ground quad whose
    uv run over [0, 3]^2 (repeat wrap) with a nearest-filtered 8-bit sRGB PNG checker; a
    UV sphere whose Disney basecolor is a bilinear HDR texture sampled with clamp wrap
    (uv over [-0.5, 1.5]) and whose roughness / metallic come from a nearest-filtered PNG
    (decoded from sRGB like every LDR texture); a box with a bilinear, repeat-wrapped PNG
    basecolor; a rectangle light and a small sky."""
    rng = np.random.default_rng(31)
    # ground quad, uv 0..3
    g = np.array([[-2, -2, 0], [2, -2, 0], [2, 2, 0], [-2, 2, 0]], np.float32)
    guv = np.array([[0, 0], [3, 0], [3, 3], [0, 3]], np.float32)
    gf = np.array([[0, 1, 2], [0, 2, 3]])
    chk = np.zeros((8, 8, 3), np.float32)
    ii, jj = np.meshgrid(np.arange(8), np.arange(8), indexing="ij")
    on = ((ii + jj) % 2 == 0)
    chk[on] = np.array([200, 180, 60]) / 255.0
    chk[~on] = np.array([40, 90, 160]) / 255.0
    # sphere, uv mapped to [-0.5, 1.5]
    sv, sf, suv = uv_sphere(48, 24, 0.6, (-0.5, 0.3, 0.6))
    suv = (suv * 2.0 - 0.5).astype(np.float32)
    hdr_base = rgbe_quantize(smooth_texture(32, 41, 0.1, 0.9))
    rm = np.round(rng.uniform(0, 255, (16, 16, 3))) / 255.0
    rm[..., 0] = 0.0
    # box with repeat-wrapped bilinear PNG
    bv, bf = subdivided_box(2)
    bv = (bv * 0.35 + np.array([0.8, -0.4, 0.35])).astype(np.float32)
    buv = np.stack([bv[:, 0] * 2.0 + bv[:, 2], bv[:, 1] * 2.0 - bv[:, 2]], 1).astype(np.float32)
    stripes = np.round(rng.uniform(20, 235, (4, 8, 3))) / 255.0
    objs = [Mesh(g, gf, "ground", uvs=guv), Mesh(sv, sf, "ball", uvs=suv), Mesh(bv, bf, "box", uvs=buv),
            Rect((-0.5, -0.5, 3.0), (-0.5, 0.5, 3.0), (0.5, 0.5, 3.0), (0.5, -0.5, 3.0), "ground",
                 emittance=(10.0, 10.0, 9.0))]
    mats = [{"name": "ground", "type": "lambert_diffuse",
             "basecolor": {"image": "checker", "sampler": "nearest", "wrap_u": "repeat", "wrap_v": "repeat"}},
            {"name": "ball", "type": "disney", "specular": 0.5, "clearcoat": 0.3,
             "basecolor": {"image": "hdrbase", "sampler": "linear", "wrap_u": "clamp", "wrap_v": "clamp"},
             "roughness": {"image": "rm", "sampler": "nearest", "wrap_u": "repeat", "wrap_v": "repeat"},
             "metallic": {"image": "rm", "sampler": "nearest", "wrap_u": "repeat", "wrap_v": "repeat"}},
            {"name": "box", "type": "lambert_diffuse",
             "basecolor": {"image": "stripes", "sampler": "linear", "wrap_u": "repeat", "wrap_v": "repeat"}}]
    env = sky_env(64, 32, 33, sun_peak=30.0, sun_sigma_deg=6.0)
    cam = {"type": "pin_hole", "pos": [0.4, -3.6, 2.0], "look_at": [0.0, 0.0, 0.4], "up": [0, 0, 1], "fov": 45.0,
           "aspect": 1.0}
    ren = {"width": res, "height": res, "spp": spp, "depth": depth, "rr_depth": 3, "rr_coef": 0.85}
    lights = [{"type": "env", "texture": "sky", "rotation": [0, 0, 30.0], "factor": 1.0}]
    tex = {"checker": chk, "hdrbase": hdr_base, "rm": rm.astype(np.float32), "stripes": stripes.astype(np.float32),
           "sky": env}
    return SceneSpec(cam, ren, mats, objs, lights, tex, ldr_textures={"checker", "rm", "stripes"})


def emitters_scene(res: int = 32, spp: int = 16, depth: int = 5, accelerator: str = "bvh") -> SceneSpec:
    """Emissive meshes and an emissive sphere as the only lights: a displaced icosphere of
    20 triangles and a box of 12 triangles, each emitting as a whole, and an analytic
    sphere light (cone sampling from outside, sphere.cpp:143-193), over a Lambert floor
    and back wall with a Disney icosphere and a Lambert box.  accelerator "bvh" makes every
    emissive triangle its own light (the reference's built-in path), "embree" one light
    per emissive mesh sampled by area (the reference's Embree meshes)."""
    v0, f0 = displaced_icosphere(0, 51, amp=0.05)
    lamp = (v0 * 0.25 + np.array([-0.9, 0.4, 1.6])).astype(np.float32)
    bv, bf = subdivided_box(1)
    box_lamp = (bv * np.array([0.3, 0.15, 0.05]) + np.array([0.7, 0.6, 1.9])).astype(np.float32)
    dv, df = displaced_icosphere(2, 52)
    disney = (dv * 0.45 + np.array([0.1, -0.1, 0.45])).astype(np.float32)
    cv, cf = subdivided_box(2)
    cube = (cv * 0.25 + np.array([-0.7, -0.6, 0.25])).astype(np.float32)
    objs = [Rect((-2, -2, 0), (2, -2, 0), (2, 2, 0), (-2, 2, 0), "floor"),
            Rect((-2, 1.5, 0), (-2, 1.5, 3), (2, 1.5, 3), (2, 1.5, 0), "floor"),
            Mesh(disney, df, "disney"), Mesh(cube, cf, "floor"),
            Mesh(lamp, f0, "floor", emittance=(6.0, 5.0, 3.0)),
            Mesh(box_lamp, bf, "floor", emittance=(9.0, 9.0, 12.0)),
            Sphere(0.12, translation=(0.9, -0.8, 1.3), material="floor", emittance=(20.0, 14.0, 10.0))]
    mats = [{"name": "floor", "type": "lambert_diffuse", "basecolor": [0.6, 0.55, 0.5]},
            {"name": "disney", "type": "disney", "basecolor": [0.7, 0.3, 0.2], "roughness": 0.35, "metallic": 0.4,
             "specular": 0.5, "clearcoat": 0.5}]
    cam = {"type": "pin_hole", "pos": [0.2, -3.8, 1.6], "look_at": [0.0, 0.2, 0.6], "up": [0, 0, 1], "fov": 50.0,
           "aspect": 1.0}
    ren = {"width": res, "height": res, "spp": spp, "depth": depth, "rr_depth": 3, "rr_coef": 0.85}
    return SceneSpec(cam, ren, mats, objs, [], {}, accelerator=accelerator)


def material_scene(seed: int, res: int = 64, env_w: int = 128, env_h: int = 64, spp: int = 16, depth: int = 6) -> SceneSpec:
    """Small scene exercising every BSDF and light kind: Disney icosphere (specTrans 0),
    Disney clearcoat sphere, dielectric sphere, conductor sphere, Lambert floor, a
    rectangle area light, a directional light and an HDR environment (z-up)."""
    rng = np.random.default_rng(seed)
    v, f = displaced_icosphere(3, seed)
    objs = [Mesh((v * 0.45 + np.array([-0.5, 0.0, 0.45])).astype(np.float32), f, "disney_a"),
            Sphere(0.3, translation=(0.45, -0.35, 0.3), material="glass"),
            Sphere(0.25, translation=(0.55, 0.45, 0.25), material="coat"),
            Sphere(0.2, translation=(-0.1, -0.75, 0.2), material="metal"),
            Rect((-2, -2, 0), (2, -2, 0), (2, 2, 0), (-2, 2, 0), "floor"),
            Rect((-0.4, -0.4, 1.8), (-0.4, 0.4, 1.8), (0.4, 0.4, 1.8), (0.4, -0.4, 1.8), "floor", emittance=(6.0, 6.0, 5.0))]
    mats = [
        {"name": "disney_a", "type": "disney", "basecolor": [0.8, 0.3, 0.2], "metallic": 0.0, "roughness": 0.4,
         "specular": 0.5, "clearcoat": 0.3, "clearcoatGloss": 0.7, "sheen": 0.2, "anisotropic": 0.3},
        {"name": "coat", "type": "disney", "basecolor": [0.2, 0.5, 0.8], "metallic": 1.0, "roughness": 0.25,
         "clearcoat": 1.0, "clearcoatGloss": 0.9},
        {"name": "glass", "type": "specular_transmission", "reflect_color": [1, 1, 1], "refract_color": [1, 1, 1],
         "eta_i": 1.0, "eta_t": float(rng.uniform(1.3, 1.7))},
        {"name": "metal", "type": "specular_reflection", "color": [0.95, 0.9, 0.8], "eta_i": [1, 1, 1],
         "eta_t": [0.2, 0.92, 1.1], "k": [3.9, 2.45, 2.14]},
        {"name": "floor", "type": "lambert_diffuse", "basecolor": [0.6, 0.6, 0.55]},
    ]
    env = sky_env(env_w, env_h, seed + 1, sun_peak=200.0, sun_sigma_deg=4.0)
    cam = {"type": "pin_hole", "pos": [0.0, -3.2, 1.4], "look_at": [0.0, 0.0, 0.35], "up": [0, 0, 1], "fov": 45.0,
           "aspect": 1.0}
    ren = {"width": res, "height": res, "spp": spp, "depth": depth, "rr_depth": 3, "rr_coef": 0.85}
    lights = [{"type": "env", "texture": "sky", "rotation": [0, 0, 30], "factor": 1.0},
              {"type": "directional", "radiance": [1.5, 1.4, 1.2], "direction": [0.3, 0.5, -0.8]}]
    return SceneSpec(cam, ren, mats, objs, lights, {"sky": env})


def _random_disney(rng):
    return {"type": "disney", "basecolor": list(rng.uniform(0.1, 0.9, 3)), "roughness": float(rng.uniform(0.05, 1.0)),
            "metallic": float(rng.random() < 0.3), "specular": 0.5, "clearcoat": float(rng.uniform(0, 1)),
            "clearcoatGloss": float(rng.uniform(0, 1)), "specTrans": 0.0}


def batch_scene(s: int, env_w: int = 512, env_h: int = 256, res: int | None = None, spp: int | None = None,
                depth: int = 8) -> SceneSpec:
    """Scene `s` of the batched workload (seed 100 + s): 1-40 meshes (displaced
    icospheres or subdivided boxes) totalling a log-uniform 1k-200k triangles, materials
    drawn from {Disney (specTrans 0), Lambert, dielectric IOR U[1.3, 1.7]}, a ground
    plane, one rectangle area light and a 512x256 sky; resolution in {128, 256, 384, 512}^2,
    spp in {4, 16, 64}, depth 8."""
    rng = np.random.default_rng(100 + s)
    k = int(rng.integers(1, 41))
    total = float(np.exp(rng.uniform(np.log(1e3), np.log(2e5))))
    w = rng.dirichlet(np.ones(k))
    objs, mats = [], []
    for m in range(k):
        budget = max(20.0, total * w[m])
        name = f"m{m}"
        kind = rng.random()
        if kind < 0.45:
            mats.append({"name": name, **_random_disney(rng)})
        elif kind < 0.8:
            mats.append({"name": name, "type": "lambert_diffuse", "basecolor": list(rng.uniform(0.1, 0.9, 3))})
        else:
            mats.append({"name": name, "type": "specular_transmission", "reflect_color": [1, 1, 1],
                         "refract_color": list(rng.uniform(0.7, 1.0, 3)), "eta_i": 1.0,
                         "eta_t": float(rng.uniform(1.3, 1.7))})
        r = float(rng.uniform(0.12, 0.45))
        c = np.array([rng.uniform(-1.6, 1.6), rng.uniform(-1.6, 1.6), 0.0])
        if rng.random() < 0.6:
            level = int(np.clip(np.round(np.log(budget / 20.0) / np.log(4.0)), 0, 7))
            v, f = displaced_icosphere(level, 1000 * s + m)
            c[2] = r
        else:
            n = max(1, int(round(np.sqrt(budget / 12.0))))
            v, f = subdivided_box(n)
            v = v * np.array([1.0, rng.uniform(0.5, 1.5), rng.uniform(0.5, 1.5)])
            c[2] = r * abs(v[:, 2]).max()
        objs.append(Mesh((v * r + c).astype(np.float32), f, name))
    mats.append({"name": "ground", "type": "lambert_diffuse", "basecolor": [0.5, 0.5, 0.5]})
    objs.append(Rect((-4, -4, 0), (4, -4, 0), (4, 4, 0), (-4, 4, 0), "ground"))
    objs.append(Rect((-0.6, -0.6, 3.5), (-0.6, 0.6, 3.5), (0.6, 0.6, 3.5), (0.6, -0.6, 3.5), "ground",
                     emittance=(10.0, 10.0, 9.0)))
    if res is None:
        res = int(rng.choice([128, 256, 384, 512]))
    if spp is None:
        spp = int(rng.choice([4, 16, 64]))
    az = rng.uniform(0, 2 * np.pi)
    cam = {"type": "pin_hole", "pos": [4.5 * np.cos(az), 4.5 * np.sin(az), 2.2], "look_at": [0.0, 0.0, 0.4],
           "up": [0, 0, 1], "fov": 45.0, "aspect": 1.0}
    ren = {"width": res, "height": res, "spp": spp, "depth": depth, "rr_depth": 3, "rr_coef": 0.85}
    env = sky_env(env_w, env_h, 100 + s, sun_peak=5e4, sun_sigma_deg=0.5)
    lights = [{"type": "env", "texture": "sky", "rotation": [0, 0, float(rng.uniform(0, 360))], "factor": 1.0}]
    return SceneSpec(cam, ren, mats, objs, lights, {"sky": env})


def batch_scenes(n: int = 64, **kw) -> list:
    return [batch_scene(s, **kw) for s in range(n)]


# ---- inverse rendering workload ------------------------------------------------------


def uv_plane(n: int, size: float, seed: int, amp: float):
    """n x n quads over [-size, size]^2 in z = 0, displaced along z by amp * fBm, with
    uv in [0, 1]^2 (2 n^2 triangles)."""
    g = np.linspace(-size, size, n + 1)
    X, Y = np.meshgrid(g, g, indexing="xy")
    P = np.stack([X, Y, np.zeros_like(X)], -1).reshape(-1, 3)
    P[:, 2] = amp * PerlinNoise(seed).fbm(P * (1.5 / size))
    t = np.linspace(0.0, 1.0, n + 1)
    U, V = np.meshgrid(t, t, indexing="xy")
    uv = np.stack([U, V], -1).reshape(-1, 2)
    idx = np.arange((n + 1) * (n + 1)).reshape(n + 1, n + 1)
    q0, q1, q2, q3 = idx[:-1, :-1], idx[:-1, 1:], idx[1:, 1:], idx[1:, :-1]
    f = np.concatenate([np.stack([q0, q1, q2], -1).reshape(-1, 3), np.stack([q0, q2, q3], -1).reshape(-1, 3)])
    return P.astype(np.float32), f, uv.astype(np.float32)


def uv_sphere(nu: int, nv: int, radius: float, center):
    """Latitude-longitude sphere (z-up) with u = phi / 2pi, v = theta / pi; a fan of
    nu triangles at each pole (2 nu (nv - 1) triangles)."""
    verts, uvs = [], []
    for j in range(nv + 1):
        th = math.pi * j / nv
        for i in range(nu + 1):
            ph = 2 * math.pi * i / nu
            verts.append([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
            uvs.append([i / nu, j / nv])
    idx = np.arange((nv + 1) * (nu + 1)).reshape(nv + 1, nu + 1)
    faces = []
    for j in range(nv):
        for i in range(nu):
            a, b, c, d = idx[j, i], idx[j, i + 1], idx[j + 1, i + 1], idx[j + 1, i]
            if j > 0:
                faces.append([a, d, b])
            if j < nv - 1:
                faces.append([b, d, c])
    v = np.asarray(verts) * radius + np.asarray(center, np.float64)
    return v.astype(np.float32), np.asarray(faces, np.int64), np.asarray(uvs, np.float32)


def smooth_texture(res: int, seed: int, lo: float, hi: float, channels: int = 3) -> np.ndarray:
    """res x res x channels smoothed noise (fBm) mapped to [lo, hi]."""
    g = (np.arange(res) + 0.5) / res * 4.0
    X, Y = np.meshgrid(g, g, indexing="xy")
    out = np.empty((res, res, channels), np.float32)
    for c in range(channels):
        P = np.stack([X + 17.3 * c, Y - 5.1 * c, np.full_like(X, 0.37 + c)], -1).reshape(-1, 3)
        n = PerlinNoise(seed * 31 + c).fbm(P, octaves=4).reshape(res, res)
        n = (n - n.min()) / max(n.max() - n.min(), 1e-9)
        out[..., c] = lo + (hi - lo) * n
    return out


def inverse_scene(seed: int = 4, tex_res: int = 512, plane_n: int = 200, sphere_nu: int = 200, sphere_nv: int = 100,
                  env_w: int = 128, env_h: int = 64, res: int = 256, spp: int = 32, depth: int = 6,
                  target: bool = True) -> SceneSpec:
    """Differentiable-rendering workload: a displaced UV-mapped plane and a UV sphere
    (about 120k triangles at the defaults) sharing one Disney material whose basecolor
    is texture "basecolor" and whose roughness (G) and metallic (B) are texture "rm";
    a rectangle area light and a small sky.  target=True gives the hidden smoothed-noise
    textures, target=False the constant 0.5 initial guess."""
    pv, pf, puv = uv_plane(plane_n, 2.0, seed, 0.08)
    sv, sf, suv = uv_sphere(sphere_nu, sphere_nv, 0.6, (0.0, 0.0, 0.7))
    objs = [Mesh(pv, pf, "surf", uvs=puv), Mesh(sv, sf, "surf", uvs=suv),
            Rect((-0.8, -0.8, 4.0), (-0.8, 0.8, 4.0), (0.8, 0.8, 4.0), (0.8, -0.8, 4.0), "surf",
                 emittance=(12.0, 12.0, 11.0))]
    if target:
        base = smooth_texture(tex_res, seed, 0.1, 0.9)
        rm = smooth_texture(tex_res, seed + 1, 0.1, 0.9)
        rm[..., 0] = 0.0
        rm[..., 2] = np.clip((rm[..., 2] - 0.3) * 1.6, 0.0, 1.0)
    else:
        base = np.full((tex_res, tex_res, 3), 0.5, np.float32)
        rm = np.full((tex_res, tex_res, 3), 0.5, np.float32)
        rm[..., 0] = 0.0
    mats = [{"name": "surf", "type": "disney", "basecolor": {"image": "basecolor"}, "roughness": {"image": "rm"},
             "metallic": {"image": "rm"}, "specular": 0.5}]
    env = sky_env(env_w, env_h, seed + 2, sun_peak=40.0, sun_sigma_deg=5.0)
    cam = inverse_views(1, seed + 1)[0]
    ren = {"width": res, "height": res, "spp": spp, "depth": depth, "rr_depth": 3, "rr_coef": 0.85}
    lights = [{"type": "env", "texture": "sky", "rotation": [0, 0, 0], "factor": 1.0}]
    return SceneSpec(cam, ren, mats, objs, lights, {"basecolor": base, "rm": rm, "sky": env})


def inverse_views(n: int = 16, seed: int = 5) -> list:
    """n pinhole cameras around the inverse-rendering scene (seeded azimuth jitter)."""
    rng = np.random.default_rng(seed)
    cams = []
    for k in range(n):
        az = 2 * math.pi * (k + rng.uniform(-0.2, 0.2)) / n
        el = math.radians(rng.uniform(25.0, 55.0))
        r = 4.2
        pos = [r * math.cos(el) * math.cos(az), r * math.cos(el) * math.sin(az), r * math.sin(el)]
        cams.append({"type": "pin_hole", "pos": pos, "look_at": [0.0, 0.0, 0.3], "up": [0, 0, 1], "fov": 50.0,
                     "aspect": 1.0})
    return cams


def gradient_scene(res: int = 48, tex_res: int = 4, base=None, rm=None, sky=None, probe=None, lam=(0.3, 0.5, 0.7)) -> SceneSpec:
    """Small scene for gradient checks: a textured Disney plane ("surf": basecolor
    texture "base", roughness (G) / metallic (B) texture "rm"), a Disney sphere with
    constant parameters ("probe"), a Lambert sphere ("lam"), a rectangle light and a
    soft 16x8 sky.  Texel values are RGBE-representable, so the reference reads the
    written .hdr files exactly."""
    pv, pf, puv = uv_plane(8, 1.5, 3, 0.05)
    s1v, s1f, s1uv = uv_sphere(24, 12, 0.45, (0.55, 0.1, 0.45))
    s2v, s2f, s2uv = uv_sphere(24, 12, 0.35, (-0.6, -0.2, 0.35))
    objs = [Mesh(pv, pf, "surf", uvs=puv), Mesh(s1v, s1f, "probe", uvs=s1uv), Mesh(s2v, s2f, "lam", uvs=s2uv),
            Rect((-0.5, -0.5, 3.0), (-0.5, 0.5, 3.0), (0.5, 0.5, 3.0), (0.5, -0.5, 3.0), "lam",
                 emittance=(9.0, 9.0, 8.0))]
    if base is None:
        base = rgbe_quantize(smooth_texture(tex_res, 11, 0.2, 0.8))
    if rm is None:
        rm = smooth_texture(tex_res, 12, 0.25, 0.75)
        rm[..., 0] = 0.0
        rm = rgbe_quantize(rm)
    if sky is None:
        sky = sky_env(16, 8, 7, sun_peak=3.0, sun_sigma_deg=20.0)
    p = dict(basecolor=[0.6, 0.35, 0.25], metallic=0.3, roughness=0.45)
    if probe:
        p.update(probe)
    mats = [{"name": "surf", "type": "disney", "basecolor": {"image": "base"}, "roughness": {"image": "rm"},
             "metallic": {"image": "rm"}, "specular": 0.5},
            {"name": "probe", "type": "disney", "specular": 0.5, "clearcoat": 0.2, **p},
            {"name": "lam", "type": "lambert_diffuse", "basecolor": list(lam)}]
    cam = {"type": "pin_hole", "pos": [0.3, -3.0, 2.4], "look_at": [0.0, 0.0, 0.3], "up": [0, 0, 1], "fov": 45.0,
           "aspect": 1.0}
    ren = {"width": res, "height": res, "spp": 16, "depth": 5, "rr_depth": 3, "rr_coef": 0.85}
    return SceneSpec(cam, ren, mats, objs, [{"type": "env", "texture": "sky", "factor": 1.0}],
                     {"base": base, "rm": rm, "sky": sky})


# ---- single-mesh workload ------------------------------------------------------------


def single_mesh_scene(level: int = 8, width: int = 1920, height: int = 1080, spp: int = 64, depth: int = 8,
                      env_w: int = 2048, env_h: int = 1024) -> SceneSpec:
    """One large mesh: an icosphere subdivided `level` times (level 8: 1,310,720
    triangles) displaced by 0.05 fBm (mesh seed 1), with per-vertex Disney parameters
    (seed 2: basecolor U[0.1, 0.9]^3, roughness U[0.05, 1], metallic Bernoulli(0.3),
    clearcoat U[0, 1]; specular 0.5, other parameters 0), lit by a 2048x1024 sky with a
    sharp sun (seed 3: peak 5e4, sigma 0.5 degrees), seen through a thin lens (radius
    0.02, focal distance 3) at 16:9."""
    v, f = displaced_icosphere(level, 1, amp=0.05)
    rng = np.random.default_rng(2)
    n = len(v)
    attr = np.empty((n, 6), np.float32)
    attr[:, 0:3] = rng.uniform(0.1, 0.9, (n, 3))
    attr[:, 3] = rng.uniform(0.05, 1.0, n)
    attr[:, 4] = (rng.random(n) < 0.3).astype(np.float32)
    attr[:, 5] = rng.uniform(0.0, 1.0, n)
    objs = [Mesh(v.astype(np.float32), f, "pv", vattr=attr)]
    mats = [{"name": "pv", "type": "disney", "basecolor": [0.5, 0.5, 0.5], "specular": 0.5, "vattr_offset": 0}]
    env = sky_env(env_w, env_h, 3, sun_peak=5e4, sun_sigma_deg=0.5)
    cam = {"type": "thin_lens", "pos": [0.0, -4.0, 0.6], "look_at": [0.0, 0.0, 0.0], "up": [0, 0, 1], "fov": 40.0,
           "aspect": width / height, "lens_radius": 0.02, "focal_distance": 3.0}
    ren = {"width": width, "height": height, "spp": spp, "depth": depth, "rr_depth": 3, "rr_coef": 0.85}
    lights = [{"type": "env", "texture": "sky", "rotation": [0, 0, 0], "factor": 1.0}]
    return SceneSpec(cam, ren, mats, objs, lights, {"sky": env})


# ---- large combined workload -----------------------------------------------------------


def large_scene(grid: int = 8, box_n: int = 102, width: int = 1920, height: int = 1080, spp: int = 128,
                depth: int = 16, env_w: int = 2048, env_h: int = 1024, seed: int = 7) -> SceneSpec:
    """grid x grid displaced meshes (subdivided cubes pushed onto a sphere and displaced
    by 0.08 fBm; box_n = 102 gives 124,848 triangles each, 8 M in all) on a ground plane,
    each with its own Disney material and roughness (the per-mesh scalars an adjoint
    differentiates): a third glass-like (specTrans 1), a third diffuse (specular 0), a
    third general; a 2048x1024 sky with a sharp sun and four rectangle lights."""
    rng = np.random.default_rng(seed)
    bv, bf = subdivided_box(box_n)
    unit = bv / np.linalg.norm(bv, axis=1, keepdims=True)
    objs, mats = [], []
    half = grid / 2.0
    for gy in range(grid):
        for gx in range(grid):
            k = gy * grid + gx
            disp = unit * (1.0 + 0.08 * PerlinNoise(seed * 1000 + k).fbm(unit, octaves=4))[:, None]
            c = np.array([(gx - half + 0.5) * 2.2, (gy - half + 0.5) * 2.2, 0.85])
            objs.append(Mesh((disp * 0.8 + c).astype(np.float32), bf, f"m{k}"))
            kind = k % 3
            m = {"name": f"m{k}", "type": "disney", "basecolor": list(rng.uniform(0.15, 0.9, 3)),
                 "roughness": float(rng.uniform(0.1, 0.9)), "specular": 0.5}
            if kind == 0:
                m.update(specTrans=1.0, specTransRoughness=0.1, ior=float(rng.uniform(1.3, 1.7)))
            elif kind == 1:
                m.update(specular=0.0)
            else:
                m.update(metallic=float(rng.random() < 0.5), clearcoat=float(rng.uniform(0, 1)))
            mats.append(m)
    mats.append({"name": "ground", "type": "lambert_diffuse", "basecolor": [0.45, 0.45, 0.42]})
    objs.append(Rect((-12, -12, 0), (12, -12, 0), (12, 12, 0), (-12, 12, 0), "ground"))
    for lx, ly in ((-4, -4), (4, -4), (-4, 4), (4, 4)):
        objs.append(Rect((lx - 0.7, ly - 0.7, 6.0), (lx - 0.7, ly + 0.7, 6.0), (lx + 0.7, ly + 0.7, 6.0),
                         (lx + 0.7, ly - 0.7, 6.0), "ground", emittance=(8.0, 8.0, 7.5)))
    env = sky_env(env_w, env_h, seed, sun_peak=5e4, sun_sigma_deg=0.5)
    cams = large_views(1, seed)
    ren = {"width": width, "height": height, "spp": spp, "depth": depth, "rr_depth": 3, "rr_coef": 0.85}
    lights = [{"type": "env", "texture": "sky", "rotation": [0, 0, 0], "factor": 1.0}]
    return SceneSpec(cams[0], ren, mats, objs, lights, {"sky": env})


def large_views(n: int = 8, seed: int = 7, aspect: float = 16 / 9) -> list:
    """n pinhole cameras around the large workload's grid."""
    rng = np.random.default_rng(seed + 1)
    cams = []
    for k in range(n):
        az = 2 * math.pi * (k + rng.uniform(-0.15, 0.15)) / n
        r, z = 17.0, float(rng.uniform(5.0, 9.0))
        cams.append({"type": "pin_hole", "pos": [r * math.cos(az), r * math.sin(az), z], "look_at": [0.0, 0.0, 0.5],
                     "up": [0, 0, 1], "fov": 50.0, "aspect": aspect})
    return cams
