"""Generate the golden fixtures in this directory from the compiled reference.

Run on a machine that has the reference sources (the oracle libraries are built from
them by oracle/Makefile):

    python tests/golden/make_golden.py [hit] [images]

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

# name, scene seed, icosphere level, boxes, rays, ray seed, origin box
HIT_CASES = [
    ("hit_s1_l4", 1, 4, 3, 20000, 11, (-1.5, 1.5)),
    ("hit_s2_l6", 2, 6, 2, 6000, 12, (-1.2, 1.2)),
]


def hit_inputs(case):
    name, seed, level, boxes, nrays, ray_seed, (lo, hi) = case
    spec = synth.hit_scene(seed, level=level, boxes=boxes)
    rng = np.random.default_rng(ray_seed)
    rays = synth.random_rays(rng, nrays, lo, hi)
    shadow = rays.copy()
    shadow[:, 3] = 1e-4
    shadow[:, 7] = rng.uniform(0.05, 3.0, size=nrays).astype(np.float32)
    desc = spec.to_desc()
    h = hashlib.sha256()
    for a in (desc.tri_pos, desc.rect_pts, rays, shadow):
        h.update(np.ascontiguousarray(a).tobytes())
    return spec, rays, shadow, h.hexdigest()


def make_hit(case):
    spec, rays, shadow, digest = hit_inputs(case)
    with tempfile.TemporaryDirectory() as d:
        p = spec.write(Path(d))
        rs = fmref.RefScene(p, "float")
        obj, t = rs.trace_closest(rays)
        t1, t2 = rs.two_nearest(rays)
        occ = rs.trace_any(shadow)
        rs.close()
    assert np.array_equal(np.isfinite(t), np.isfinite(t1))
    np.savez_compressed(GOLDEN / f"{case[0]}.npz", obj=obj.astype(np.int32), t=t.astype(np.float32),
                        t2=t2.astype(np.float32), occ=np.packbits(occ), n=len(rays), sha256=digest)
    print(case[0], "hits", int((obj >= 0).sum()), "occluded", int(occ.sum()))


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


if __name__ == "__main__":
    what = set(sys.argv[1:]) or {"hit"}
    t0 = time.time()
    if "hit" in what:
        for c in HIT_CASES:
            make_hit(c)
    if "images" in what:
        for c in IMAGE_CASES:
            make_image(c)
    print("done in %.1fs" % (time.time() - t0))
