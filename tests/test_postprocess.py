"""Post-processing on the device (fm_postprocess) against the reference's own
post-process classes and its 8-bit conversion, byte for byte, on a seeded frame that
covers negative, huge and boundary values (tests/golden/post_u8.npz, made by the
reference's float build through make_golden.py post); and the denoise step, which
stands in for OIDN (not available), checked by what it is for: a noisy render comes
closer to the converged image."""
from pathlib import Path

import numpy as np
import pytest

import fumeng_b200 as fb
from fumeng_b200 import synth
from golden.make_golden import POST_CHAINS, post_inputs

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_post_inputs_unchanged():
    import hashlib
    g = np.load(GOLDEN / "post_u8.npz")
    h = hashlib.sha256()
    for a in post_inputs():
        h.update(a.tobytes())
    assert str(g["sha256"]) == h.hexdigest()


@pytest.mark.gpu
def test_postprocess_bytes_match_reference(ctx):
    g = np.load(GOLDEN / "post_u8.npz")
    rgb, alb, nrm = post_inputs()
    for i, chain in enumerate(POST_CHAINS):
        _, c8, a8, n8 = ctx.postprocess(chain, rgb, alb, nrm)
        ref = g[f"rgb8_{i}"]
        diff = np.abs(c8.astype(np.int32) - ref.astype(np.int32))
        uses_pow = any(t in (fb.FM_POST_LINEAR_TO_SRGB, fb.FM_POST_SRGB_TO_LINEAR) for t, _ in chain)
        # without pow every byte is equal; the sRGB steps' pow may move a value that sits
        # on a rounding boundary by one code
        assert diff.max() <= (1 if uses_pow else 0), (chain, int(diff.max()))
        assert (diff > 0).sum() <= (8 if uses_pow else 0), (chain, int((diff > 0).sum()))
        assert np.array_equal(a8, g["albedo8"]) and np.array_equal(n8, g["normal8"])


@pytest.mark.gpu
def test_denoise_brings_a_noisy_render_closer_to_the_converged_image(ctx):
    spec = synth.material_scene(3, res=64)
    scene = ctx.create_scene(spec.to_desc())
    try:
        cam = spec.camera_struct()
        noisy, alb, nrm, _ = scene.render(cam, spec.render_params(spp=16, seed=3))
        conv = scene.render(cam, spec.render_params(spp=8192, seed=4), want_aov=False)[0]
    finally:
        scene.destroy()
    den = ctx.postprocess([(fb.FM_POST_DENOISE, 0.0)], noisy, alb, nrm)[0]

    def tmse(x):
        # squared error of the displayed (tone-compressed, x / (1 + x)) values, so that a
        # single firefly of a 16-spp image does not decide the comparison
        t = lambda a: a / (1.0 + np.maximum(a, 0.0))
        return float(np.mean((t(x) - t(conv)) ** 2))
    assert np.all(np.isfinite(den))
    print(f"tone-compressed MSE: noisy {tmse(noisy):.4g}, denoised {tmse(den):.4g}")
    assert tmse(den) < 0.75 * tmse(noisy)
    # a flat image stays flat, and the denoise step needs its guides
    flat = np.full((16, 16, 3), 0.25, np.float32)
    out = ctx.postprocess([(fb.FM_POST_DENOISE, 0.0)], flat, flat, np.dstack([np.zeros((16, 16, 2)), np.ones((16, 16, 1))]))[0]
    assert np.allclose(out, 0.25, rtol=1e-6)
    with pytest.raises(fb.FumengError):
        ctx.postprocess([(fb.FM_POST_DENOISE, 0.0)], flat)
