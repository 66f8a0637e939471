"""Texel gradients of the inverse-rendering configuration against central finite
differences, at 1e-2 relative.

Scene: the configuration's 120k-triangle plane and sphere with its 512^2 basecolor and
roughness (G) / metallic (B) target textures, first view (256^2, depth 6).  256 cases,
each a 4x4-pixel tile with seeded loss weights and the texel seen through the tile's
centre, one channel per case (basecolor r / g / b, roughness, metallic in turn;
tests/golden/make_golden.py: c3_gradient_cases).

* Finite differences: central, step 0.04, on the tile loss, with common random numbers
  (the same seed at +h and -h), 16 seeds of 32,768 spp rendered together as one batch
  per sign.  Central differences are flat in h here (0.005 to 0.04 agree within their
  noise on probed cases), and the larger step lowers their noise.
* Adjoint: fm_render_adjoint on the same tile with other seeds, 16 x 32,768 spp.
* Standard errors from the 16 seeds of each.  Tolerance per case:
  max(1e-2 |FD|, 4 standard errors of the difference); and over all cases the median of
  |adjoint - FD| / |FD| must be below 1e-2.

Also: central differences of the reference's double build on the basecolor cases whose
perturbation survives the .hdr file exactly (tests/golden/adj_fd_texels_ref.npz) against
the adjoint, max(2e-2 |FD|, 4 standard errors) (the reference's CPU time limits its
sample count).
"""
import json
import os
from pathlib import Path

import numpy as np
import pytest

import fumeng_b200 as fb
from golden.make_golden import c3_gradient_cases, inverse_target_scene

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
H = 0.04
SPP, SEEDS_FD, SEEDS_ADJ = 32768, list(range(11, 27)), list(range(101, 117))


def _sem(x):
    x = np.asarray(x, np.float64)
    return x.mean(), x.std(ddof=1) / np.sqrt(len(x))


@pytest.fixture(scope="module")
def c3():
    spec = inverse_target_scene()
    holder = spec.to_desc()
    ctx = fb.Context(0)
    scene = ctx.create_scene(holder)
    cases = c3_gradient_cases(spec)
    ti = holder.texture_index
    cam = spec.camera_struct()
    shapes = {ti["basecolor"]: spec.textures["basecolor"].shape[:2], ti["rm"]: spec.textures["rm"].shape[:2]}
    adj = []
    for tile, tex, (ty, tx, ch), w in cases:
        vals = []
        for seed in SEEDS_ADJ:
            p = spec.render_params(spp=SPP, seed=seed, region=tile)
            tg, _, _, st = scene.render_adjoint([cam], [p], [w], shapes)
            assert st.nan_samples == 0
            vals.append(tg[ti[tex]][ty, tx, ch])
        adj.append(_sem(vals))
    yield spec, ctx, scene, cases, adj, ti, cam
    scene.destroy()
    ctx.close()


def _fd(spec, ctx, scene, ti, cam, tile, tex, texel, w, h):
    """Central difference per seed: every seed's +h (and -h) render in one batch."""
    orig = spec.textures[tex]
    L = []
    for sign in (1.0, -1.0):
        t = orig.copy()
        t[texel] = orig[texel] + sign * h
        scene.update_texture(ti[tex], t)
        params = [spec.render_params(spp=SPP, seed=s, region=tile) for s in SEEDS_FD]
        imgs, _, _, _ = ctx.render_batch([scene] * len(params), [cam] * len(params), params)
        L.append(np.array([float((w.astype(np.float64) * img).sum()) for img in imgs]))
    scene.update_texture(ti[tex], orig)
    return _sem((L[0] - L[1]) / (2 * h))


def test_texel_gradients_match_central_differences_at_one_percent(c3):
    spec, ctx, scene, cases, adj, ti, cam = c3
    assert len(cases) == 256
    fails, powered, rel = [], 0, []
    for k, ((tile, tex, texel, w), (a, sa)) in enumerate(zip(cases, adj)):
        f, sf = _fd(spec, ctx, scene, ti, cam, tile, tex, texel, w, H)
        noise = 4.0 * np.hypot(sa, sf)
        tol = max(1e-2 * abs(f), noise)
        powered += noise <= 1e-2 * abs(f)
        rel.append(abs(a - f) / max(abs(f), 1e-30))
        if abs(a - f) > tol:
            fails.append((k, tex, texel, a, sa, f, sf))
    med = float(np.median(rel))
    if os.environ.get("FUMENG_B200_PARITY_LOG"):
        with open(os.environ["FUMENG_B200_PARITY_LOG"], "a") as fh:
            fh.write(json.dumps({"case": "c3_texel_gradients", "cases": len(cases), "median_rel_err": med,
                                 "p90_rel_err": float(np.percentile(rel, 90)), "bound_1e-2_binds": int(powered),
                                 "outside_tolerance": len(fails)}) + "\n")
    print(f"c3 texels: median |adjoint - FD| / |FD| = {med:.2e}, 90th percentile {np.percentile(rel, 90):.2e}, "
          f"cases where the 1e-2 bound binds: {powered}/{len(cases)}")
    assert not fails, f"{len(fails)} of {len(cases)} cases outside tolerance: {fails[:5]}"
    assert med < 1e-2, med


def test_texel_gradients_match_reference_double_fd(c3):
    path = GOLDEN / "adj_fd_texels_ref.npz"
    if not path.exists():
        pytest.skip("no reference texel FD fixture (tests/golden/make_golden.py adjoint_texels)")
    spec, ctx, scene, cases, adj, ti, cam = c3
    g = np.load(path)
    for ci, k in enumerate(g["case_index"]):
        tile, tex, texel, w = cases[int(k)]
        a, sa = adj[int(k)]
        f, sf = _sem(g["fd"][ci])
        tol = max(2e-2 * abs(f), 4.0 * np.hypot(sa, sf))
        print(f"reference FD case {int(k)} {tex}{texel}: adjoint {a:.5g} +- {sa:.2g}, reference {f:.5g} +- {sf:.2g}")
        if os.environ.get("FUMENG_B200_PARITY_LOG"):
            with open(os.environ["FUMENG_B200_PARITY_LOG"], "a") as fh:
                fh.write(json.dumps({"case": f"c3_reference_fd_{int(k)}", "adjoint": a, "adjoint_se": sa,
                                     "reference_fd": f, "reference_fd_se": sf}) + "\n")
        assert abs(a - f) <= tol, f"case {k} {tex}{texel}: adjoint {a:.6g} +- {sa:.2g} vs reference FD {f:.6g} +- {sf:.2g}"
