"""Device BVH builder edge cases: meshes below, at and above the small-cluster size (32
primitives), a large grid, identical triangles (every split is a median split whose
child bounds are accumulated after the partition) and a stack of parallel triangles
(splits along one axis only).  Rays aimed at known triangles must report them."""
import numpy as np
import pytest

from fumeng_b200.scene import Mesh, SceneSpec

CAM = {"type": "pin_hole", "pos": [0, 0, 5], "look_at": [0, 0, 0], "up": [0, 1, 0], "fov": 45.0, "aspect": 1.0}
REN = {"width": 8, "height": 8, "spp": 1, "depth": 2}
MATS = [{"name": "m0", "type": "lambert_diffuse", "basecolor": [0.5, 0.5, 0.5]}]


def grid_mesh(ntri: int, seed: int = 0):
    """`ntri` disjoint triangles on a jittered grid in the plane z = h_i (h_i small and
    distinct), and downward rays through their centroids."""
    rng = np.random.default_rng(seed)
    k = int(np.ceil(np.sqrt(ntri)))
    idx = np.arange(ntri)
    cx, cy = (idx % k).astype(np.float64), (idx // k).astype(np.float64)
    h = rng.uniform(-0.25, 0.25, size=ntri)
    v = np.zeros((3 * ntri, 3), np.float32)
    v[0::3] = np.stack([cx + 0.1, cy + 0.1, h], 1)
    v[1::3] = np.stack([cx + 0.8, cy + 0.15, h], 1)
    v[2::3] = np.stack([cx + 0.2, cy + 0.85, h], 1)
    f = np.arange(3 * ntri).reshape(ntri, 3)
    c = v.reshape(ntri, 3, 3).astype(np.float64).mean(1)
    rays = np.zeros((ntri, 8), np.float32)
    rays[:, 0], rays[:, 1], rays[:, 2] = c[:, 0], c[:, 1], 10.0
    rays[:, 6] = -1.0
    rays[:, 7] = np.finfo(np.float32).max
    return Mesh(v, f, "m0"), rays, 10.0 - h


def _scene(ctx, meshes):
    holder = SceneSpec(CAM, REN, MATS, meshes).to_desc()
    return ctx.create_scene(holder), holder


@pytest.mark.gpu
@pytest.mark.parametrize("ntri", [1, 2, 31, 32, 33, 65, 1000, 90000])
def test_grid_rays_hit_their_triangles(ctx, ntri):
    mesh, rays, t_exp = grid_mesh(ntri, seed=ntri)
    scene, holder = _scene(ctx, [mesh])
    try:
        st = scene.bvh_stats()
        assert st["prims"] == ntri and 1 <= st["depth"] < 32
        obj, t = scene.trace_closest(rays)
        occ = scene.trace_any(rays)
    finally:
        scene.destroy()
    assert np.array_equal(obj, np.arange(ntri))
    np.testing.assert_allclose(t, t_exp, rtol=1e-6)
    assert occ.all()


@pytest.mark.gpu
def test_identical_triangles_median_splits(ctx):
    n = 3000
    tri = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]], np.float32)
    mesh = Mesh(np.tile(tri, (n, 1)), np.arange(3 * n).reshape(n, 3), "m0")
    scene, _ = _scene(ctx, [mesh])
    rays = np.zeros((64, 8), np.float32)
    g = np.random.default_rng(1).uniform(0.05, 0.45, size=(64, 2))
    rays[:, 0:2] = g
    rays[:, 2] = 2.0
    rays[:, 6] = -1.0
    rays[:, 7] = np.finfo(np.float32).max
    try:
        st = scene.bvh_stats()
        assert st["prims"] == n and st["depth"] < 32
        obj, t = scene.trace_closest(rays)
    finally:
        scene.destroy()
    assert np.all((obj >= 0) & (obj < n))
    np.testing.assert_allclose(t, 2.0, rtol=1e-6)


@pytest.mark.gpu
def test_stacked_triangles_report_the_nearest(ctx):
    n = 5000
    tri = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]], np.float32)
    v = np.tile(tri, (n, 1))
    v[:, 2] = np.repeat(np.arange(n, dtype=np.float32) * 1e-3, 3)   # triangle i at z = i / 1000
    mesh = Mesh(v, np.arange(3 * n).reshape(n, 3), "m0")
    scene, _ = _scene(ctx, [mesh])
    rays = np.zeros((2, 8), np.float32)
    rays[:, 0:2] = 0.25
    rays[0, 2], rays[0, 6] = 10.0, -1.0     # from above: the top triangle
    rays[1, 2], rays[1, 6] = -10.0, 1.0     # from below: the bottom one
    rays[:, 7] = np.finfo(np.float32).max
    try:
        obj, t = scene.trace_closest(rays)
    finally:
        scene.destroy()
    assert obj.tolist() == [n - 1, 0]
    np.testing.assert_allclose(t, [10.0 - (n - 1) * 1e-3, 10.0], rtol=1e-6)
