"""Bounded device waits and queue capacities fail cleanly: a render stopped by its
iteration cap returns FM_ERR_TIMEOUT, one whose ray queues are capped below what it needs
returns FM_ERR_QUEUE_OVERFLOW, and the context renders correctly afterwards (its cached
graph is dropped and rebuilt).  Nothing faults or hangs: the kernels only stop early
(tuning fields max_iterations / queue_limit of fm_tuning)."""
import numpy as np
import pytest

import fumeng_b200 as fb
from fumeng_b200 import synth


def _close(a, b):
    rel = np.abs(a - b) / (np.abs(a) + 1e-3)
    return float(np.mean(rel < 1e-3))


def _render(ctx, specs, tuning):
    scenes = [ctx.create_scene(s.to_desc()) for s in specs]
    try:
        cams = [s.camera_struct() for s in specs]
        params = [s.render_params(spp=8, seed=3, mode=fb.FM_MODE_WAVEFRONT) for s in specs]
        rgb, _, _, st = ctx.render_batch(scenes, cams, params, tuning=tuning)
        assert st.paths == sum(p.width * p.height * p.spp for p in params)
        return rgb
    finally:
        for sc in scenes:
            sc.destroy()


SPECS = [synth.material_scene(1, res=32), synth.material_scene(2, res=40)]


def _tuning(**kw):
    t = fb.Tuning(1 << 12, 128, 128, 4)
    for k, v in kw.items():
        setattr(t, k, v)
    return t


@pytest.mark.gpu
@pytest.mark.parametrize("field,value,status", [("max_iterations", 3, fb.FM_ERR_TIMEOUT),
                                                ("queue_limit", 1, fb.FM_ERR_QUEUE_OVERFLOW),
                                                ("queue_limit", 700, fb.FM_ERR_QUEUE_OVERFLOW)],
                         ids=["iteration_cap", "queue_cap_1", "queue_cap_700"])
def test_bounded_render_fails_cleanly_and_context_recovers(field, value, status):
    ctx = fb.Context(0)
    try:
        before = _render(ctx, SPECS, _tuning())
        with pytest.raises(fb.FumengError) as e:
            _render(ctx, SPECS, _tuning(**{field: value}))
        assert e.value.status == status, str(e.value)
        after = _render(ctx, SPECS, _tuning())
    finally:
        ctx.close()
    fresh = fb.Context(0)
    try:
        ref = _render(fresh, SPECS, _tuning())
    finally:
        fresh.close()
    for b, a, r in zip(before, after, ref):
        assert np.all(np.isfinite(a))
        assert _close(a, r) > 0.97 and _close(b, r) > 0.97


@pytest.mark.gpu
def test_limits_above_need_change_nothing(ctx):
    # caps that the render never reaches leave it untouched
    ref = _render(ctx, SPECS, _tuning())
    got = _render(ctx, SPECS, _tuning(max_iterations=100000, queue_limit=1 << 20))
    for g, r in zip(got, ref):
        assert _close(g, r) > 0.97

