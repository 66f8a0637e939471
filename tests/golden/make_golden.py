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


if __name__ == "__main__":
    what = set(sys.argv[1:]) or {"hit"}
    t0 = time.time()
    if "hit" in what:
        for c in HIT_CASES:
            make_hit(c)
    print("done in %.1fs" % (time.time() - t0))
