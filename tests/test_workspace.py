"""The context's wavefront workspace: state buffers and the instantiated graph are kept
between renders and reused while the launch state is the same.  Renders through a
context that has already rendered other scenes, tunings and batch sizes must equal
renders through a fresh context (up to the order of float atomics in the wavefront)."""
import numpy as np
import pytest

import fumeng_b200 as fb
from fumeng_b200 import synth


def _close(a, b):
    rel = np.abs(a - b) / (np.abs(a) + 1e-3)
    return float(np.mean(rel < 1e-3))


def _render(ctx, specs, seed, tuning=None):
    scenes = [ctx.create_scene(s.to_desc()) for s in specs]
    try:
        cams = [s.camera_struct() for s in specs]
        params = [s.render_params(spp=16, seed=seed, mode=fb.FM_MODE_WAVEFRONT) for s in specs]
        rgb, _, _, st = ctx.render_batch(scenes, cams, params, tuning=tuning)
        assert st.paths == sum(p.width * p.height * p.spp for p in params)
        return rgb
    finally:
        for sc in scenes:
            sc.destroy()


@pytest.mark.gpu
def test_reused_workspace_matches_fresh_context():
    a = [synth.material_scene(1, res=48), synth.material_scene(2, res=48)]
    b = [synth.material_scene(3, res=48), synth.material_scene(4, res=48)]
    tune = fb.Tuning(1 << 14, 128, 128, 4)
    warm = fb.Context(0)
    try:
        _render(warm, a, seed=5, tuning=tune)                     # same shape class, other scenes
        _render(warm, a[:1], seed=6, tuning=tune)                 # fewer views
        _render(warm, a + b, seed=7, tuning=fb.Tuning(1 << 15, 64, 256, 8))   # more views, larger pool
        got = _render(warm, b, seed=9, tuning=tune)
        again = _render(warm, b, seed=9, tuning=tune)             # the cached graph, launched again
    finally:
        warm.close()
    fresh = fb.Context(0)
    try:
        ref = _render(fresh, b, seed=9, tuning=tune)
    finally:
        fresh.close()
    for g, a2, r in zip(got, again, ref):
        assert np.all(np.isfinite(g))
        assert _close(g, r) > 0.97 and _close(a2, r) > 0.97


@pytest.mark.gpu
def test_caller_owned_host_images_are_written_in_place(ctx):
    """render_batch(out=...) writes the read-back into the caller's arrays (reused across
    calls) and gives the same images as arrays the call allocates itself."""
    specs = [synth.material_scene(1, res=48), synth.material_scene(2, res=32)]
    scenes = [ctx.create_scene(s.to_desc()) for s in specs]
    try:
        cams = [s.camera_struct() for s in specs]
        params = [s.render_params(spp=16, seed=3, mode=fb.FM_MODE_WAVEFRONT) for s in specs]
        ref, _, _, _ = ctx.render_batch(scenes, cams, params)
        out = [np.full(p.out_shape() + (3,), np.nan, np.float32) for p in params]
        for _ in range(2):
            got, _, _, _ = ctx.render_batch(scenes, cams, params, out=out)
            assert all(g is o for g, o in zip(got, out))
            for o, r in zip(out, ref):
                assert np.all(np.isfinite(o)) and _close(o, r) > 0.97
        with pytest.raises(ValueError):
            ctx.render_batch(scenes, cams, params, out=out[:1])
        with pytest.raises(ValueError):
            ctx.render_batch(scenes, cams, params, out=[out[0].astype(np.float64), out[1]])
    finally:
        for sc in scenes:
            sc.destroy()
