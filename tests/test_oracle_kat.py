"""Oracle checks (CPU): the C restatement and the compiled reference agree bit for bit,
and the committed golden fixtures are reproduced by both."""
import hashlib

import numpy as np
import pytest

import fmref
from fumeng_b200 import synth

needs_ref = pytest.mark.skipif(not fmref.available("float"), reason="oracle/_ref not built (no reference sources)")


@needs_ref
def test_abs_binding_kat():
    # triangle.cpp:13-18 compiles with the C library's int abs: components are truncated,
    # so unit directions select z unless a component is exactly +-1.
    assert fmref.get_max_axis((0.9, 0.3, 0.1)) == 2
    assert fmref.get_max_axis((0.1, 0.9, 0.3)) == 2
    assert fmref.get_max_axis((1.0, 0.0, 0.0)) == 0
    assert fmref.get_max_axis((0.0, -1.0, 0.5)) == 1
    assert fmref.get_max_axis((2.5, 1.5, 1.0)) == 0


@needs_ref
def test_restatement_max_axis_matches_reference():
    L = fmref.restate()
    rng = np.random.default_rng(0)
    vs = np.concatenate([rng.normal(size=(500, 3)) * s for s in (0.3, 1.0, 3.0)])
    vs = np.concatenate([vs, np.eye(3), -np.eye(3), [[1, 1, 0], [0, 2, 2], [3, 0, 3]]]).astype(np.float32)
    for v in vs:
        assert L.fmo_get_max_axis(*map(float, v)) == fmref.get_max_axis(v)


def _tri_cases(rng, n):
    rays = np.zeros((n, 8), np.float32)
    tris = np.zeros((n, 9), np.float32)
    for i in range(n):
        kind = i % 4
        v = rng.normal(size=(3, 3)).astype(np.float32)
        if kind == 1:   # axis-aligned triangle, ray through a vertex -> zero edge functions
            v[:, 2] = 0.5
            target = v[0]
        elif kind == 2:  # ray through an edge midpoint
            target = ((v[0] + v[1]) * 0.5).astype(np.float32)
        else:
            b = rng.dirichlet([1, 1, 1])
            target = (b @ v).astype(np.float32)
        o = rng.normal(size=3).astype(np.float32) * 2
        if kind == 3:
            o = target + np.float32(1e-3) * rng.normal(size=3).astype(np.float32)
        d = target - o
        d = (d / np.linalg.norm(d)).astype(np.float32)
        rays[i, :3], rays[i, 4:7] = o, d
        rays[i, 3], rays[i, 7] = 0.0, np.finfo(np.float32).max
        tris[i] = v.reshape(9)
    return rays, tris


@needs_ref
def test_restatement_triangle_bit_exact():
    import ctypes as C
    L = fmref.restate()
    F = C.POINTER(C.c_float)
    rays, tris = _tri_cases(np.random.default_rng(1), 2000)
    for r, v in zip(rays, tris):
        hit_ref, t_ref, bc_ref = fmref.intersect_triangle(r.astype(np.float64), v.astype(np.float64))
        t = np.zeros(1, np.float32)
        bc = np.zeros(3, np.float32)
        hit = L.fmo_intersect_triangle(r.ctypes.data_as(F), v.ctypes.data_as(F), t.ctypes.data_as(F), bc.ctypes.data_as(F))
        assert bool(hit) == hit_ref
        if hit:
            assert np.float32(t_ref) == t[0] or (np.isnan(t_ref) and np.isnan(t[0]))
            assert np.array_equal(bc, bc_ref.astype(np.float32))


def _golden(name):
    from golden.make_golden import HIT_CASES, hit_inputs  # noqa: F401
    case = [c for c in HIT_CASES if c[0] == name][0]
    spec, rays, shadow, digest = hit_inputs(case)
    g = np.load(fmref.HERE.parent / "tests" / "golden" / f"{name}.npz")
    return spec, rays, shadow, digest, g


@pytest.mark.parametrize("name", [c[0] for c in __import__("golden.make_golden", fromlist=["HIT_CASES"]).HIT_CASES])
def test_golden_inputs_reproduce(name):
    spec, rays, shadow, digest, g = _golden(name)
    assert str(g["sha256"]) == digest, "synthetic scene/ray generator drifted from the golden fixture"


def test_restatement_matches_golden_closest():
    # Exhaustive C restatement on a subset of rays reproduces the reference's BVH answers.
    spec, rays, shadow, digest, g = _golden("hit_s1_l4")
    d = spec.to_desc()
    sel = np.arange(0, len(rays), 7)[:2000]
    assert d.desc.num_rects == 2 and d.desc.num_spheres == 0
    # rectangles as their two triangles (rectangle.cpp:38-56), objects after the mesh faces
    rp = d.rect_pts.reshape(-1, 4, 3)
    rect_tris = np.concatenate([np.stack([rp[:, 0], rp[:, 1], rp[:, 2]], 1), np.stack([rp[:, 2], rp[:, 3], rp[:, 0]], 1)])
    rect_obj = np.concatenate([d.rect_object, d.rect_object])
    tri = np.concatenate([d.tri_pos.reshape(-1, 3, 3), rect_tris]).reshape(-1, 9)
    tri_obj = np.concatenate([d.tri_object, rect_obj])
    prim, t = fmref.restate_closest(tri, rays[sel])
    obj = np.where(prim >= 0, tri_obj[np.maximum(prim, 0)], -1)
    gt1, gt2 = g["t"][sel], g["t2"][sel]
    keep = ~(np.abs(gt2 - gt1) <= 1e-6 * np.abs(gt1))
    assert np.array_equal(obj[keep], g["obj"][sel][keep])
    assert np.array_equal(t[keep], gt1[keep])


def test_restatement_matches_golden_spheres():
    # The C restatement of Sphere::IntersectSphere, with the triangles and rectangles,
    # reproduces the reference's closest hits on the scene with analytic spheres.
    spec, rays, shadow, digest, g = _golden("hit_s3_spheres")
    d = spec.to_desc()
    assert d.desc.num_spheres == 10
    xf = d.sphere_xform.reshape(-1, 4, 4)
    assert np.array_equal(xf[:, :3, :3], np.broadcast_to(np.eye(3, dtype=np.float32), (10, 3, 3)))
    centers = xf[:, :3, 3]
    rp = d.rect_pts.reshape(-1, 4, 3)
    rect_tris = np.concatenate([np.stack([rp[:, 0], rp[:, 1], rp[:, 2]], 1), np.stack([rp[:, 2], rp[:, 3], rp[:, 0]], 1)])
    tri = np.concatenate([d.tri_pos.reshape(-1, 3, 3), rect_tris]).reshape(-1, 9)
    tri_obj = np.concatenate([d.tri_object, d.rect_object, d.rect_object])
    sel = np.arange(0, len(rays), 5)[:4000]
    prim, t = fmref.restate_closest_spheres(tri, centers, d.sphere_radius, rays[sel])
    obj = np.where(prim < 0, -1, np.where(prim < len(tri), tri_obj[np.minimum(np.maximum(prim, 0), len(tri) - 1)],
                                           d.sphere_object[np.maximum(prim - len(tri), 0)]))
    gt1, gt2 = g["t"][sel], g["t2"][sel]
    keep = ~(np.abs(gt2 - gt1) <= 1e-6 * np.abs(gt1))
    assert np.isin(g["obj"][sel], d.sphere_object).sum() > 200, "too few sphere hits to pin the sphere test"
    assert np.array_equal(obj[keep], g["obj"][sel][keep])
    assert np.array_equal(t[keep], gt1[keep])


@needs_ref
@pytest.mark.parametrize("name", ["hit_s1_l4", "hit_s3_spheres"])
def test_live_oracle_reproduces_golden(name, tmp_path):
    spec, rays, shadow, digest, g = _golden(name)
    rs = fmref.RefScene(spec.write(tmp_path), "float")
    obj, t = rs.trace_closest(rays)
    occ = rs.trace_any(shadow)
    assert np.array_equal(obj, g["obj"])
    assert np.array_equal(t.astype(np.float32), g["t"])
    assert np.array_equal(np.packbits(occ), g["occ"])
