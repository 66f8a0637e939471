"""Converged images of the CUDA renderers against the reference's double build.

For each golden scene the GPU renders 16 independent batches of 256 samples (4096 spp;
batch b uses sample indices [256 b, 256 b + 256)), which gives per-pixel means and the
variance of those means.  The golden fixture holds the reference's per-pixel mean and
single-sample variance at 4096 spp (tests/golden/make_golden.py).  Checks:
  * per-pixel 3-sigma agreement: |mu_gpu - mu_ref| <= 3 sqrt(var_gpu/N + var_ref/N);
    about 0.27% of pixel channels fail under pure noise, the bound is 1%;
  * relMSE = mean((mu_gpu - mu_ref)^2 / (mu_ref^2 + 1e-2)); it contains both estimators'
    noise, so the test bounds relMSE minus its expected noise part (the squared bias) by
    1e-3 plus three standard errors of the relMSE estimate itself (the sample standard
    deviation of the per-channel terms over sqrt(n)): on noisy tiles (caustics, a sharp
    sun) the noise term is large and the mean of n heavy-tailed terms scatters around it;
    on converged ones the standard error is small and 1e-3 is the bound;
  * albedo and normal AOVs (first-hit averages) agree to 2e-2 mean absolute difference.
"""
import json
import os
from pathlib import Path

import numpy as np
import pytest

import fumeng_b200 as fb
from fumeng_b200 import synth
from golden.make_golden import BATCH_CASES, IMAGE_CASES, SINGLE_TILES, large_small_scene, single_scene

GOLDEN_DIR = Path(__file__).resolve().parent / "golden"
BATCHES, BATCH_SPP = 16, 256
# Optional log of every comparison (one JSON line each): the file named by this variable.
RESULTS_LOG = os.environ.get("FUMENG_B200_PARITY_LOG")


def log_result(res: dict) -> None:
    print(json.dumps(res))
    if RESULTS_LOG:
        with open(RESULTS_LOG, "a") as f:
            f.write(json.dumps(res) + "\n")


def render_batches(ctx, spec, mode, seed=1234, batches=BATCHES, spp=BATCH_SPP):
    scene = ctx.create_scene(spec.to_desc())
    try:
        cam = spec.camera_struct()
        rgb, alb, nrm = [], [], []
        for b in range(batches):
            p = spec.render_params(spp=spp, seed=seed, mode=mode, sample_offset=b * spp)
            c, a, n, st = scene.render(cam, p)
            assert st.paths == p.width * p.height * spp
            rgb.append(c)
            alb.append(a)
            nrm.append(n)
    finally:
        scene.destroy()
    return np.stack(rgb).astype(np.float64), np.mean(alb, 0), np.mean(nrm, 0)


def compare(rgb_batches, g):
    K = rgb_batches.shape[0]
    s = int(g["stride"])
    mu = rgb_batches.mean(0)[::s, ::s]
    var_mu = rgb_batches.var(0, ddof=1)[::s, ::s] / K
    r = g["mean"].astype(np.float64)
    var_r = g["var"].astype(np.float64) / float(g["spp"])
    den = r * r + 1e-2
    terms = (mu - r) ** 2 / den
    relmse = float(np.mean(terms))
    se = float(np.std(terms, ddof=1) / np.sqrt(terms.size))
    noise = float(np.mean((var_mu + var_r) / den))
    z = np.abs(mu - r) / np.sqrt(var_mu + var_r + 1e-12)
    return {"relmse": relmse, "relmse_noise": noise, "relmse_bias": relmse - noise, "relmse_se": se,
            "frac_3sigma": float(np.mean(z > 3.0)), "pixels": int(np.prod(r.shape[:2]))}


def assert_parity(res):
    assert res["frac_3sigma"] < 0.01, res
    assert res["relmse_bias"] < 1e-3 + 3.0 * res["relmse_se"], res


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [fb.FM_MODE_MEGAKERNEL, fb.FM_MODE_WAVEFRONT], ids=["megakernel", "wavefront"])
@pytest.mark.parametrize("case", IMAGE_CASES, ids=[c[0] for c in IMAGE_CASES])
def test_converged_image_matches_reference(ctx, case, mode):
    name = case[0]
    g = np.load(GOLDEN_DIR / f"{name}.npz")
    spec = case[1]()
    rgb, alb, nrm = render_batches(ctx, spec, mode)
    res = compare(rgb, g)
    s = int(g["stride"])
    res["albedo_mad"] = float(np.mean(np.abs(alb[::s, ::s] - g["albedo"])))
    res["normal_mad"] = float(np.mean(np.abs(nrm[::s, ::s] - g["normal"])))
    res.update(case=name, mode="megakernel" if mode == fb.FM_MODE_MEGAKERNEL else "wavefront")
    log_result(res)
    assert np.all(np.isfinite(rgb))
    assert_parity(res)
    assert res["albedo_mad"] < 2e-2 and res["normal_mad"] < 2e-2, res


@pytest.mark.gpu
def test_megakernel_is_deterministic(ctx):
    from fumeng_b200 import synth
    spec = synth.material_scene(3, res=32)
    a = render_batches(ctx, spec, fb.FM_MODE_MEGAKERNEL, batches=1, spp=8)[0]
    b = render_batches(ctx, spec, fb.FM_MODE_MEGAKERNEL, batches=1, spp=8)[0]
    assert np.array_equal(a, b, equal_nan=True)


@pytest.mark.gpu
def test_wavefront_matches_megakernel_on_same_random_streams(ctx):
    # Both renderers draw the same random numbers in the same order for every sample, so
    # their images agree up to float summation order (and the rare path that a rounding
    # difference sends another way).
    from fumeng_b200 import synth
    spec = synth.material_scene(3, res=48)
    a = render_batches(ctx, spec, fb.FM_MODE_MEGAKERNEL, batches=1, spp=64)[0][0]
    b = render_batches(ctx, spec, fb.FM_MODE_WAVEFRONT, batches=1, spp=64)[0][0]
    rel = np.abs(a - b) / (np.abs(a) + 1e-3)
    assert np.mean(rel < 1e-3) > 0.97, float(np.mean(rel < 1e-3))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [fb.FM_MODE_MEGAKERNEL, fb.FM_MODE_WAVEFRONT], ids=["megakernel", "wavefront"])
def test_batched_scenes_match_reference(ctx, mode):
    """Four scenes of the batched workload rendered together through fm_render_batch
    (one graph-captured wavefront, or the megakernel view after view), 16 x 256 spp, against
    tiles of the reference's double build (tests/golden/batch_s*.npz; each fixture records
    its tile and spp)."""
    cases = [s for s in BATCH_CASES if (GOLDEN_DIR / f"batch_s{s}.npz").exists()]
    if not cases:
        pytest.skip("no batched-scene fixtures (tests/golden/make_golden.py batch)")
    specs = [synth.batch_scene(s) for s in cases]
    scenes = [ctx.create_scene(sp.to_desc()) for sp in specs]
    try:
        cams = [sp.camera_struct() for sp in specs]
        out = [[] for _ in specs]
        for b in range(BATCHES):
            params = [sp.render_params(spp=BATCH_SPP, seed=1234, mode=mode, sample_offset=b * BATCH_SPP) for sp in specs]
            rgb, _, _, st = ctx.render_batch(scenes, cams, params)
            assert st.paths == sum(p.width * p.height * p.spp for p in params)
            for i, img in enumerate(rgb):
                out[i].append(img)
    finally:
        for sc in scenes:
            sc.destroy()
    for i, s in enumerate(cases):
        g = np.load(GOLDEN_DIR / f"batch_s{s}.npz")
        x0, y0, w, h = (int(v) for v in g["tile"])
        tiles = np.stack(out[i]).astype(np.float64)[:, y0:y0 + h, x0:x0 + w]
        assert np.all(np.isfinite(tiles))
        res = compare(tiles, g)
        res.update(case=f"batch_s{s}", mode="megakernel" if mode == fb.FM_MODE_MEGAKERNEL else "wavefront")
        log_result(res)
        assert_parity(res)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [fb.FM_MODE_MEGAKERNEL, fb.FM_MODE_WAVEFRONT], ids=["megakernel", "wavefront"])
def test_single_mesh_scene_matches_reference(ctx, mode):
    """The single-mesh configuration (1.31 M triangles, per-vertex Disney parameters,
    thin lens, 2048x1024 sky with a sharp sun) at 480x270, 16 x 256 spp, against 32x32
    tiles of the reference's double build (tests/golden/single_t*.npz; each fixture
    records its tile and spp)."""
    tiles = [k for k in range(len(SINGLE_TILES)) if (GOLDEN_DIR / f"single_t{k}.npz").exists()]
    if not tiles:
        pytest.skip("no single-mesh fixtures (tests/golden/make_golden.py single)")
    rgb, _, _ = render_batches(ctx, single_scene(), mode)
    for k in tiles:
        g = np.load(GOLDEN_DIR / f"single_t{k}.npz")
        x0, y0, w, h = (int(v) for v in g["tile"])
        t = rgb[:, y0:y0 + h, x0:x0 + w]
        assert np.all(np.isfinite(t))
        res = compare(t, g)
        res.update(case=f"single_t{k}", mode="megakernel" if mode == fb.FM_MODE_MEGAKERNEL else "wavefront")
        log_result(res)
        assert_parity(res)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [fb.FM_MODE_MEGAKERNEL, fb.FM_MODE_WAVEFRONT], ids=["megakernel", "wavefront"])
def test_large_config_generator_matches_reference(ctx, mode):
    """The large configuration's scene generator at 2x2 meshes (glass-like Disney with
    specular transmission 1, diffuse and general Disney, Lambert ground, four rectangle
    lights, a sky with a sharp sun, depth 16), full 64x40 frame, 16 x 256 spp against the
    reference's double build at 4096 spp (tests/golden/large_small.npz).  The only
    fixture with specular transmission in Disney, whose lobe choice and reflect /
    transmit choice share one random number in the reference."""
    path = GOLDEN_DIR / "large_small.npz"
    if not path.exists():
        pytest.skip("no large-configuration fixture (tests/golden/make_golden.py large)")
    g = np.load(path)
    rgb, _, _ = render_batches(ctx, large_small_scene(), mode)
    res = compare(rgb, g)
    res.update(case="large_small", mode="megakernel" if mode == fb.FM_MODE_MEGAKERNEL else "wavefront")
    log_result(res)
    assert np.all(np.isfinite(rgb))
    assert_parity(res)
