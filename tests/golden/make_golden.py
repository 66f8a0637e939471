"""Generate the golden fixtures in this directory from the compiled reference.

Run on a machine that has the reference sources (the oracle libraries are built from
them by oracle/Makefile):

    python tests/golden/make_golden.py [hit] [images] [adjoint] [batch] [single] [large] [inverse] [textured] [emitters] [post] [adjoint_texels] [digests] [force]

Scenes and rays are regenerated from seeds by fumeng_b200.synth, so each fixture stores
only the reference's answers plus a SHA-256 of the inputs, which the tests recompute to
detect generator drift.
"""
from __future__ import annotations

import hashlib
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import fmref  # noqa: E402

from fumeng_b200 import synth  # noqa: E402

GOLDEN = Path(__file__).resolve().parent

# name, scene builder, ray kind, rays, ray seed, origin box (random rays) or film grid
# (camera rays: nx, ny).  Random rays start uniformly in the box with isotropic
# directions; camera rays are jittered pinhole primary rays of the scene's camera.
HIT_CASES = [
    ("hit_s1_l4", lambda: synth.hit_scene(1, level=4, boxes=3), "random", 20000, 11, (-1.5, 1.5)),
    ("hit_s2_l6", lambda: synth.hit_scene(2, level=6, boxes=2), "random", 6000, 12, (-1.2, 1.2)),
    # analytic spheres (translation-only transforms) among meshes and rectangles
    ("hit_s3_spheres", lambda: synth.hit_scene(3, level=4, boxes=2, spheres=10), "random", 20000, 13, (-1.5, 1.5)),
    # the single-mesh configuration's 1.31 M-triangle displaced icosphere: random rays
    # from around it, and its camera's primary rays
    ("hit_single_random", synth.single_mesh_hit_scene, "random", 20000, 14, (-1.3, 1.3)),
    ("hit_single_camera", synth.single_mesh_hit_scene, "camera", 0, 15, (192, 108)),
]
_SCENE_CACHE: dict = {}


def hit_inputs(case):
    name, builder, kind, nrays, ray_seed, box = case
    key = builder
    if key not in _SCENE_CACHE:
        _SCENE_CACHE.clear()
        _SCENE_CACHE[key] = builder()
    spec = _SCENE_CACHE[key]
    rng = np.random.default_rng(ray_seed)
    if kind == "camera":
        rays = synth.pinhole_rays(rng, spec.camera, box[0], box[1])
        nrays = len(rays)
    else:
        rays = synth.random_rays(rng, nrays, box[0], box[1])
    shadow = rays.copy()
    shadow[:, 3] = 1e-4
    shadow[:, 7] = rng.uniform(0.05, 3.0 if kind == "random" else 6.0, size=nrays).astype(np.float32)
    desc = spec.to_desc()
    h = hashlib.sha256()
    arrays = [desc.tri_pos, desc.rect_pts, rays, shadow]
    if desc.desc.num_spheres:
        arrays += [desc.sphere_radius, desc.sphere_xform]
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return spec, rays, shadow, h.hexdigest()


def local_second_nearest(spec, rays, obj, t):
    """Second-nearest hit distance near the closest hit, for meshes too large for the
    harness's exhaustive fmref_two_nearest: a near tie (|t2 - t1| <= 1e-6 t1) can only
    come from a triangle passing within 1e-6 t1 |d| of the hit point, so only triangles
    whose centroid lies within their largest circumradius (plus that distance) of it are
    tested, with the C restatement of the reference's triangle test (pinned bit for bit
    against the reference by tests/test_oracle_kat.py).  Returns +inf where no other
    object is hit there (mesh-only scenes: object index = triangle index)."""
    from scipy.spatial import cKDTree
    import ctypes as C
    d = spec.to_desc()
    assert d.desc.num_rects == 0 and d.desc.num_spheres == 0
    tri = d.tri_pos.reshape(-1, 3, 3).astype(np.float64)
    cen = tri.mean(axis=1)
    rad = float(np.linalg.norm(tri - cen[:, None, :], axis=2).max())
    tree = cKDTree(cen)
    L = fmref.restate()
    F = C.POINTER(C.c_float)
    t2 = np.full(len(rays), np.inf)
    hit = np.nonzero(obj >= 0)[0]
    P = rays[hit, 0:3].astype(np.float64) + t[hit, None] * rays[hit, 4:7].astype(np.float64)
    cands = tree.query_ball_point(P, rad + 1e-5 * (1.0 + np.abs(t[hit])))
    tri32 = d.tri_pos.reshape(-1, 9).astype(np.float32)
    for k, i in enumerate(hit):
        r = np.ascontiguousarray(rays[i], np.float32)
        best = np.inf
        for j in cands[k]:
            if j == obj[i]:
                continue
            tt = np.zeros(1, np.float32)
            if L.fmo_intersect_triangle(r.ctypes.data_as(F), tri32[j].ctypes.data_as(F), tt.ctypes.data_as(F), None):
                best = min(best, float(tt[0]))
        t2[i] = best
    return t2


def make_hit(case):
    spec, rays, shadow, digest = hit_inputs(case)
    with tempfile.TemporaryDirectory() as d:
        p = spec.write(Path(d))
        rs = fmref.RefScene(p, "float")
        obj, t = rs.trace_closest(rays)
        if rs.num_objects() > 200000:
            t1, t2 = t.copy(), local_second_nearest(spec, rays, obj, t)
        else:
            t1, t2 = rs.two_nearest(rays)
        occ = rs.trace_any(shadow)
        rs.close()
    assert np.array_equal(np.isfinite(t), np.isfinite(t1))
    np.savez_compressed(GOLDEN / f"{case[0]}.npz", obj=obj.astype(np.int32), t=t.astype(np.float32),
                        t2=t2.astype(np.float32), occ=np.packbits(occ), n=len(rays), sha256=digest)
    tie = np.abs(t2 - t) <= 1e-6 * np.abs(t)
    print(case[0], "rays", len(rays), "hits", int((obj >= 0).sum()), "near ties", int(tie.sum()), "occluded",
          int(occ.sum()))


# name, builder, oracle spp, seed; images are stored at every `stride`-th pixel
IMAGE_CASES = [
    ("img_cornell", lambda: synth.cornell(), 4096, 7, 2),
    ("img_materials", lambda: synth.material_scene(3), 4096, 8, 1),
]


def make_image(case):
    name, builder, spp, seed, stride = case
    spec = builder()
    with tempfile.TemporaryDirectory() as d:
        rs = fmref.RefScene(spec.write(Path(d)), "double")
        t0 = time.time()
        r = rs.render(spp, seed=seed, aov=True)
        dt = time.time() - t0
        rs.close()
    mean = r["sum"] / spp
    var = np.maximum(r["sumsq"] / spp - mean * mean, 0.0) * spp / (spp - 1)
    sl = (slice(None, None, stride), slice(None, None, stride))
    np.savez_compressed(GOLDEN / f"{name}.npz", mean=mean[sl].astype(np.float32), var=var[sl].astype(np.float32),
                        albedo=(r["albedo"] / spp)[sl].astype(np.float32), normal=(r["normal"] / spp)[sl].astype(np.float32),
                        spp=spp, stride=stride)
    print(name, "spp", spp, "%.1fs" % dt, "mean", mean.mean(axis=(0, 1)))


# Scenes of the batched workload (synth.batch_scene index), each a 16x16 tile at the
# centre of its image, rendered by the double build at BATCH_SPP.  Every fixture holds
# the per-pixel mean and single-sample variance of the reference's estimator as it is
# ("mean", "var") and of the same samples with each colour channel limited to
# BATCH_CLAMP ("cmean", "cvar"; fm_render_params.max_sample_value on the GPU side).  The
# clamped estimator has bounded variance, so its comparison resolves a bias of 1e-3
# relMSE even on tiles with dielectric caustics and a sharp sun, where the unclamped
# estimator's heavy tail leaves a noise floor far above that.  Scenes: 14 of the 64,
# chosen for dielectric-heavy material mixes (1-10 dielectric meshes each) at every
# resolution of the workload.
BATCH_CASES = [2, 3, 6, 13, 22, 27, 30, 32, 36, 39, 44, 46, 53, 56]
BATCH_SPP, BATCH_SEED, BATCH_TILE, BATCH_CLAMP = 8192, 9, 16, 10.0


def batch_tile(spec):
    w, h = int(spec.renderer["width"]), int(spec.renderer["height"])
    return ((w - BATCH_TILE) // 2, (h - BATCH_TILE) // 2, BATCH_TILE, BATCH_TILE)


def moments(r, key, spp):
    s, s2 = r[key], r[key + "sq"]
    mean = s / spp
    var = np.maximum(s2 / spp - mean * mean, 0.0) * spp / (spp - 1)
    return mean.astype(np.float32), var.astype(np.float32)


def render_clamped_fixture(spec, name, spp, seed, clamp, tile=None, aov=False):
    with tempfile.TemporaryDirectory() as d:
        rs = fmref.RefScene(spec.write(Path(d)), "double")
        t0 = time.time()
        r = rs.render(spp, seed=seed, tile=tile, clamp=clamp, aov=aov)
        dt = time.time() - t0
        rs.close()
    mean, var = moments(r, "sum", spp)
    cmean, cvar = moments(r, "csum", spp)
    extra = {"tile": np.asarray(tile)} if tile is not None else {}
    if aov:
        extra.update(albedo=(r["albedo"] / spp).astype(np.float32), normal=(r["normal"] / spp).astype(np.float32))
    np.savez_compressed(GOLDEN / f"{name}.npz", mean=mean, var=var, cmean=cmean, cvar=cvar, spp=spp, clamp=clamp,
                        stride=1, **extra)
    print(name, "tile", tile, "%.1fs" % dt, "mean", mean.mean(axis=(0, 1)), "clamped", cmean.mean(axis=(0, 1)),
          flush=True)


def make_batch(s):
    if (GOLDEN / f"batch_s{s}.npz").exists():
        return
    spec = synth.batch_scene(s)
    render_clamped_fixture(spec, f"batch_s{s}", BATCH_SPP, BATCH_SEED, BATCH_CLAMP, batch_tile(spec))


# The single-mesh configuration (1.31 M-triangle displaced icosphere with per-vertex
# Disney parameters, thin lens, 2048x1024 sky with a sharp sun) at 480x270: 32x32 tiles
# at the centre of the sphere and across its silhouette, double build, 1024 spp.
SINGLE_RES = (480, 270)
SINGLE_TILES = [(224, 119, 32, 32), (323, 119, 32, 32)]
SINGLE_SPP, SINGLE_SEED = 1024, 11


def single_scene():
    return synth.single_mesh_scene(width=SINGLE_RES[0], height=SINGLE_RES[1])


def make_single():
    spec = single_scene()
    with tempfile.TemporaryDirectory() as d:
        rs = fmref.RefScene(spec.write(Path(d)), "double")
        for k, tile in enumerate(SINGLE_TILES):
            t0 = time.time()
            r = rs.render(SINGLE_SPP, seed=SINGLE_SEED, tile=tile)
            mean = r["sum"] / SINGLE_SPP
            var = np.maximum(r["sumsq"] / SINGLE_SPP - mean * mean, 0.0) * SINGLE_SPP / (SINGLE_SPP - 1)
            np.savez_compressed(GOLDEN / f"single_t{k}.npz", mean=mean.astype(np.float32), var=var.astype(np.float32),
                                spp=SINGLE_SPP, tile=np.asarray(tile), stride=1)
            print(f"single_t{k}", tile, "%.1fs" % (time.time() - t0), "mean", mean.mean(axis=(0, 1)))
        rs.close()


# The large configuration's scene generator at a size the reference renders here in
# minutes: 2x2 displaced meshes (1,728 triangles each) with the configuration's material
# mix (glass-like Disney with specular transmission 1, diffuse Disney, general Disney),
# the Lambert ground, four rectangle lights and a sky with a sharp sun, depth 16; a closer
# camera; full 64x40 frame, double build, 16384 spp, plain and clamped sums.
LARGE_SMALL_SPP, LARGE_SMALL_SEED = 16384, 13


def large_small_scene():
    spec = synth.large_scene(grid=2, box_n=12, width=64, height=40, spp=16, depth=16, env_w=256, env_h=128)
    spec.camera = {"type": "pin_hole", "pos": [4.5, -5.0, 3.5], "look_at": [0.0, 0.0, 0.8], "up": [0, 0, 1],
                   "fov": 50.0, "aspect": 64 / 40}
    return spec


def make_large_small():
    if (GOLDEN / "large_small.npz").exists():
        return
    render_clamped_fixture(large_small_scene(), "large_small", LARGE_SMALL_SPP, LARGE_SMALL_SEED, BATCH_CLAMP)


# The inverse-rendering configuration's scene with its hidden target textures (512^2
# basecolor and roughness / metallic, RGBE-quantized so that the reference's .hdr reader
# and the device see the same texels), first view, a 16x16 tile on the textured surfaces,
# double build, 8192 spp, plain and clamped sums.
INVERSE_TILE, INVERSE_SPP, INVERSE_SEED = (120, 120, 16, 16), 8192, 17


def inverse_target_scene():
    from fumeng_b200.scene import rgbe_quantize
    spec = synth.inverse_scene()
    for k in ("basecolor", "rm"):
        spec.textures[k] = rgbe_quantize(spec.textures[k])
    return spec


def make_inverse_tile():
    if (GOLDEN / "inverse_t0.npz").exists():
        return
    render_clamped_fixture(inverse_target_scene(), "inverse_t0", INVERSE_SPP, INVERSE_SEED, BATCH_CLAMP, INVERSE_TILE)


# Image textures in every form ImageTexture has (synth.textured_scene: nearest and
# bilinear filtering, repeat and clamp wrap, 8-bit sRGB PNG and HDR files, an LDR
# roughness / metallic map decoded from sRGB), full 48x48 frame, double build, 16384 spp,
# plain and clamped sums and the albedo / normal AOVs.
TEXTURED_SPP, TEXTURED_SEED = 16384, 19


def make_textured():
    if (GOLDEN / "textured.npz").exists():
        return
    render_clamped_fixture(synth.textured_scene(), "textured", TEXTURED_SPP, TEXTURED_SEED, BATCH_CLAMP, aov=True)


# Emissive meshes and an emissive sphere as the only lights (synth.emitters_scene), full
# 32x32 frame, double build with the built-in BVH (one light per emissive triangle),
# 16384 spp, plain and clamped sums.
EMITTERS_SPP, EMITTERS_SEED = 16384, 37


def make_emitters():
    """Double build (mean / var, plain and clamped) and the reference's float build
    (f_mean / f_var) of the same scene."""
    if not (GOLDEN / "emitters.npz").exists():
        render_clamped_fixture(synth.emitters_scene(), "emitters", EMITTERS_SPP, EMITTERS_SEED, BATCH_CLAMP)
    g = dict(np.load(GOLDEN / "emitters.npz"))
    if "f_mean" in g:
        return
    with tempfile.TemporaryDirectory() as d:
        rs = fmref.RefScene(synth.emitters_scene().write(Path(d)), "float")
        r = rs.render(EMITTERS_SPP, seed=EMITTERS_SEED + 1)
        rs.close()
    g["f_mean"], g["f_var"] = moments(r, "sum", EMITTERS_SPP)
    g["f_spp"] = EMITTERS_SPP
    np.savez_compressed(GOLDEN / "emitters.npz", **g)
    print("emitters float build", g["f_mean"].mean(axis=(0, 1)), flush=True)


# ---- post-processing and the 8-bit conversion ----------------------------------------
# A seeded 64x64 frame whose values cover what the chain meets: negative and zero,
# [0, 4] uniform, 1e-6 .. 1e4 log-uniform, the sRGB breakpoints, the exact 8-bit codes
# k / 255 and the rounding midpoints (k + 0.5) / 255 with their float neighbours; albedo
# in [0, 1], normals in [-1, 1].  Chains as DrawFrame runs them (core/renderer.h:131-135).
POST_CHAINS = [[(0, 1.0), (1, 0.0)], [(1, 0.0)], [(2, 0.0)], [(0, 0.35)], []]


def post_inputs():
    rng = np.random.default_rng(29)
    n = 64 * 64 * 3
    v = rng.uniform(0.0, 4.0, n)
    k = rng.integers(0, n, n // 2)
    v[k[: n // 8]] = -rng.uniform(0.0, 1.0, n // 8)
    v[k[n // 8: n // 4]] = np.exp(rng.uniform(np.log(1e-6), np.log(1e4), n // 4 - n // 8))
    codes = np.arange(256) / 255.0
    mids = (np.arange(255) + 0.5) / 255.0
    special = np.concatenate([[0.0, 1.0, 0.0031308, 0.04045], codes, mids,
                              np.nextafter(mids.astype(np.float32), np.float32(2)),
                              np.nextafter(mids.astype(np.float32), np.float32(-1))])
    v[: len(special)] = special
    rgb = v.astype(np.float32).reshape(64, 64, 3)
    alb = rng.uniform(0.0, 1.0, (64, 64, 3)).astype(np.float32)
    nrm = rng.uniform(-1.0, 1.0, (64, 64, 3)).astype(np.float32)
    return rgb, alb, nrm


def make_post():
    rgb, alb, nrm = post_inputs()
    out = {}
    for i, chain in enumerate(POST_CHAINS):
        c8, a8, n8 = fmref.postprocess_u8(chain, rgb.astype(np.float64), alb.astype(np.float64),
                                         nrm.astype(np.float64), "float")
        out[f"rgb8_{i}"] = c8
        if i == 0:
            out["albedo8"], out["normal8"] = a8, n8
    h = hashlib.sha256()
    for a in (rgb, alb, nrm):
        h.update(a.tobytes())
    np.savez_compressed(GOLDEN / "post_u8.npz", sha256=h.hexdigest(), **out)
    print("post_u8", len(POST_CHAINS), "chains")


# ---- texel gradients of the inverse-rendering configuration ---------------------------
# 4x4-pixel tiles of the first view (256^2) on a 17x17 grid over the image centre, the
# first 256 that see the mesh through their centre pixel.  For each tile, the texel seen through its centre pixel (the camera ray's nearest hit on the
# mesh, at its interpolated texture coordinate) and one channel of it, in turn: basecolor
# r, g, b, roughness (rm G), metallic (rm B).  The loss of a case is sum(w * I) over its
# tile with seeded weights w in [0.5, 1.5].
C3_TILE, C3_GRID, C3_STEP, C3_CASES = 4, 17, 8, 256
C3_CHANNELS = [("basecolor", 0), ("basecolor", 1), ("basecolor", 2), ("rm", 1), ("rm", 2)]


def _nearest_hit(tri, o, d):
    """Moller-Trumbore over all triangles (float64): (triangle index, b1, b2) or None."""
    v0, v1, v2 = tri[:, 0], tri[:, 1], tri[:, 2]
    e1, e2 = v1 - v0, v2 - v0
    pv = np.cross(d, e2)
    det = np.einsum("ij,ij->i", e1, pv)
    ok = np.abs(det) > 1e-14
    inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
    tv = o - v0
    b1 = np.einsum("ij,ij->i", tv, pv) * inv
    qv = np.cross(tv, e1)
    b2 = (qv @ d) * inv
    t = np.einsum("ij,ij->i", e2, qv) * inv
    hit = ok & (b1 >= 0) & (b2 >= 0) & (b1 + b2 <= 1) & (t > 1e-6)
    if not hit.any():
        return None
    k = int(np.argmin(np.where(hit, t, np.inf)))
    return k, float(b1[k]), float(b2[k])


def c3_gradient_cases(spec=None):
    """[(tile (x0, y0, w, h), texture name, (row, col, channel), weights (4, 4, 3))]"""
    spec = spec or inverse_target_scene()
    desc = spec.to_desc()
    tri = desc.tri_pos.reshape(-1, 3, 3).astype(np.float64)
    uv = desc.tri_uv.reshape(-1, 3, 2).astype(np.float64)
    cam = spec.camera
    W, H = int(spec.renderer["width"]), int(spec.renderer["height"])
    pos = np.asarray(cam["pos"], np.float64)
    f = np.asarray(cam["look_at"], np.float64) - pos
    f /= np.linalg.norm(f)
    up = np.asarray(cam["up"], np.float64)
    up /= np.linalg.norm(up)
    sv = np.cross(up, f)
    sv /= np.linalg.norm(sv)
    uvv = np.cross(f, sv)
    th = np.tan(np.radians(float(cam["fov"])) / 2.0)
    asp = float(cam.get("aspect", 1.0))
    x_start = (W - C3_GRID * C3_STEP) // 2
    y_start = (H - C3_GRID * C3_STEP) // 2
    rng = np.random.default_rng(23)
    cases = []
    for k in range(C3_GRID * C3_GRID):
        x0 = x_start + C3_STEP * (k % C3_GRID)
        y0 = y_start + C3_STEP * (k // C3_GRID)
        col, row = x0 + C3_TILE // 2, y0 + C3_TILE // 2
        px, py = (col + 0.5) / W, (H - 1 - row + 0.5) / H
        d = f + (2 * px - 1) * th * asp * sv + (2 * py - 1) * th * uvv
        d /= np.linalg.norm(d)
        w = rng.uniform(0.5, 1.5, (C3_TILE, C3_TILE, 3)).astype(np.float32)
        h = _nearest_hit(tri, pos, d)
        if h is None or uv is None:
            continue
        ti, b1, b2 = h
        u, v = (1 - b1 - b2) * uv[ti, 0] + b1 * uv[ti, 1] + b2 * uv[ti, 2]
        tex, ch = C3_CHANNELS[len(cases) % len(C3_CHANNELS)]
        th_, tw_ = spec.textures[tex].shape[:2]
        tx = int(np.clip(np.floor((u - np.floor(u)) * tw_), 0, tw_ - 1))
        ty = int(np.clip(np.floor((v - np.floor(v)) * th_), 0, th_ - 1))
        cases.append(((x0, y0, C3_TILE, C3_TILE), tex, (ty, tx, ch), w))
        if len(cases) == C3_CASES:
            break
    return cases


# Central differences of the same tile losses from the reference's double build for a
# few of these cases (basecolor channels, whose finite differences are the least noisy):
# the perturbed channel is its texel's largest (so the .hdr file's shared exponent, and
# with it the other channels, stay unchanged) and the step is two quanta of that
# exponent; per-pixel seeding makes the +-h renders use common random numbers.
C3_REF = {"cases": 4, "spp": 16384, "seeds": [401, 402, 403, 404, 405, 406, 407, 408]}


def rgbe_step(x):
    """Two quanta of the RGBE mantissa at value x (8-bit mantissa, shared exponent)."""
    e = np.floor(np.log2(x)) + 1.0
    return 2.0 * 2.0 ** (e - 8.0)


def c3_reference_cases(spec=None):
    spec = spec or inverse_target_scene()
    out = []
    for k, (tile, tex, (ty, tx, ch), w) in enumerate(c3_gradient_cases(spec)):
        if tex != "basecolor":
            continue
        texel = spec.textures[tex][ty, tx]
        x = float(texel[ch])
        if x < 0.3 or x > 0.9 or x < float(np.max(texel)):
            continue
        h = rgbe_step(x)
        if np.floor(np.log2(x - h)) != np.floor(np.log2(x + h)):
            continue
        out.append((k, tile, tex, (ty, tx, ch), w, h))
        if len(out) == C3_REF["cases"]:
            break
    return out


def make_adjoint_texels():
    from fumeng_b200.scene import rgbe_quantize
    spec = inverse_target_scene()
    cases = c3_reference_cases(spec)
    fd = np.zeros((len(cases), len(C3_REF["seeds"])))
    spp = C3_REF["spp"]
    for ci, (k, tile, tex, (ty, tx, ch), w, h) in enumerate(cases):
        orig = spec.textures[tex]
        for si, seed in enumerate(C3_REF["seeds"]):
            L = []
            for sign in (1.0, -1.0):
                t = orig.copy()
                t[ty, tx, ch] = orig[ty, tx, ch] + sign * h
                assert np.array_equal(rgbe_quantize(t), t), "perturbed texture is not representable in .hdr"
                spec.textures[tex] = t
                with tempfile.TemporaryDirectory() as d:
                    rs = fmref.RefScene(spec.write(Path(d)), "double")
                    r = rs.render(spp, seed=seed, tile=tile)
                    rs.close()
                L.append(float((w.astype(np.float64) * r["sum"] / spp).sum()))
            spec.textures[tex] = orig
            fd[ci, si] = (L[0] - L[1]) / (2 * h)
        print("c3 texel fd", k, tex, (ty, tx, ch), fd[ci].mean(), fd[ci].std(ddof=1) / np.sqrt(fd.shape[1]), flush=True)
    np.savez_compressed(GOLDEN / "adj_fd_texels_ref.npz", fd=fd, spp=spp, seeds=np.asarray(C3_REF["seeds"]),
                        case_index=np.asarray([c[0] for c in cases]), h=np.asarray([c[5] for c in cases]))


# SHA-256 of the scene inputs behind each image fixture (scene_digests.json), so that a
# change of the scene generators that would invalidate a fixture is caught on the CPU.
def scene_digest(spec) -> str:
    import json as _json
    from fumeng_b200.scene import Mesh, Rect, Sphere
    h = hashlib.sha256()
    h.update(_json.dumps([spec.camera, spec.renderer, spec.materials, spec.lights], sort_keys=True,
                         default=float).encode())
    if getattr(spec, "accelerator", "bvh") != "bvh":
        h.update(spec.accelerator.encode())
    for o in spec.objects:
        if isinstance(o, Mesh):
            h.update(np.ascontiguousarray(o.vertices, np.float32).tobytes())
            h.update(np.ascontiguousarray(o.faces, np.int64).tobytes())
            for extra in (o.uvs, o.normals, o.vattr):
                if extra is not None:
                    h.update(np.ascontiguousarray(extra, np.float32).tobytes())
        elif isinstance(o, (Rect, Sphere)):
            h.update(repr(o).encode())
        h.update(str(getattr(o, "material", "")).encode())
    for name in sorted(spec.textures):
        h.update(name.encode())
        if name in getattr(spec, "ldr_textures", ()):
            h.update(b"ldr")
        h.update(np.ascontiguousarray(spec.textures[name], np.float32).tobytes())
    return h.hexdigest()


def image_fixture_scenes():
    """(fixture name, scene builder) of every image fixture."""
    out = [(name, builder) for name, builder, _, _, _ in IMAGE_CASES]
    out += [(f"batch_s{s}", (lambda s=s: synth.batch_scene(s))) for s in BATCH_CASES]
    out += [("single", single_scene), ("large_small", large_small_scene), ("inverse_t0", inverse_target_scene),
            ("textured", synth.textured_scene), ("emitters", synth.emitters_scene)]
    return out


def make_digests():
    import json as _json
    d = {name: scene_digest(builder()) for name, builder in image_fixture_scenes()}
    (GOLDEN / "scene_digests.json").write_text(_json.dumps(d, indent=1, sort_keys=True) + "\n")
    print("scene digests", len(d))


# Central differences of L = sum(w * image) from the reference's double build, for
# constant material parameters of synth.gradient_scene (48x48), with common random
# numbers across +-h: (material, JSON key, channel or None).
ADJ_FD_CASES = [("probe", "basecolor", 0), ("probe", "metallic", None), ("probe", "roughness", None),
                ("lam", "basecolor", 1)]
ADJ_FD = {"spp": 1024, "seeds": [301, 302, 303, 304], "h": 0.02, "wseed": 5}


def adjoint_fd_weights():
    return np.random.default_rng(ADJ_FD["wseed"]).uniform(0.5, 1.5, (48, 48, 3)).astype(np.float32)


def perturbed_gradient_scene(mat, key, ch, delta):
    spec = synth.gradient_scene()
    m = next(x for x in spec.materials if x["name"] == mat)
    if ch is None:
        m[key] = float(m[key]) + delta
    else:
        v = list(m[key])
        v[ch] += delta
        m[key] = v
    return spec


def make_adjoint_fd():
    w = adjoint_fd_weights().astype(np.float64)
    fd = np.zeros((len(ADJ_FD_CASES), len(ADJ_FD["seeds"])))
    h, spp = ADJ_FD["h"], ADJ_FD["spp"]
    for ci, (mat, key, ch) in enumerate(ADJ_FD_CASES):
        for si, seed in enumerate(ADJ_FD["seeds"]):
            L = []
            for sign in (1.0, -1.0):
                spec = perturbed_gradient_scene(mat, key, ch, sign * h)
                with tempfile.TemporaryDirectory() as d:
                    rs = fmref.RefScene(spec.write(Path(d)), "double")
                    r = rs.render(spp, seed=seed)
                    rs.close()
                L.append(float((w * r["sum"] / spp).sum()))
            fd[ci, si] = (L[0] - L[1]) / (2 * h)
        print("adjoint fd", mat, key, ch, fd[ci].mean(), fd[ci].std(ddof=1) / np.sqrt(fd.shape[1]))
    np.savez_compressed(GOLDEN / "adj_fd_ref.npz", fd=fd, spp=spp, h=h, seeds=np.asarray(ADJ_FD["seeds"]),
                        wseed=ADJ_FD["wseed"],
                        cases=np.asarray([f"{m}.{k}.{-1 if c is None else c}" for m, k, c in ADJ_FD_CASES]))


if __name__ == "__main__":
    what = set(sys.argv[1:]) or {"hit"}
    t0 = time.time()
    if "hit" in what:
        for c in HIT_CASES:
            if (GOLDEN / f"{c[0]}.npz").exists() and "force" not in what:
                continue
            make_hit(c)
    if "images" in what:
        for c in IMAGE_CASES:
            make_image(c)
    if "adjoint" in what:
        make_adjoint_fd()
    if "batch" in what:
        for s in BATCH_CASES:
            make_batch(s)
    if "single" in what:
        make_single()
    if "large" in what:
        make_large_small()
    if "inverse" in what:
        make_inverse_tile()
    if "emitters" in what:
        make_emitters()
    if "post" in what:
        make_post()
    if "textured" in what:
        make_textured()
    if "adjoint_texels" in what:
        make_adjoint_texels()
    if "digests" in what:
        make_digests()
    print("done in %.1fs" % (time.time() - t0))
