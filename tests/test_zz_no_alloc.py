"""The allocation-free closest-hit entry point (fm_trace_closest_noalloc) against the
regular one.

Callers that cannot let the library allocate device memory while they run (a real-time
loop with a fixed memory budget and a frame deadline, or an application whose own pool
owns the device memory) use fm_trace_closest_noalloc, which stages rays and results in a
fixed array inside the library instead.  This file is collected last so that a run that
stops at the first failure has already run every other test.
"""
import numpy as np
import pytest

import fumeng_b200 as fb
from fumeng_b200 import synth

MAX_RAYS = 1 << 18


@pytest.mark.gpu
def test_noalloc_matches_regular_entry_point_on_consecutive_calls(ctx):
    spec = synth.hit_scene(5, level=4, boxes=2)
    scene = ctx.create_scene(spec.to_desc())
    try:
        rng = np.random.default_rng(21)
        # two calls in a row with different sizes: the second must not see the first's data
        for n in (MAX_RAYS, 40000):
            rays = synth.random_rays(rng, n, -1.5, 1.5)
            obj_ref, t_ref = scene.trace_closest(rays)
            obj, t = scene.trace_closest_noalloc(rays)
            assert np.array_equal(obj, obj_ref)
            assert np.array_equal(t, t_ref)
            assert (obj >= 0).any() and (obj < 0).any()
    finally:
        scene.destroy()


@pytest.mark.gpu
def test_noalloc_rejects_batches_beyond_its_maximum(ctx):
    spec = synth.hit_scene(5, level=2, boxes=1)
    scene = ctx.create_scene(spec.to_desc())
    try:
        rays = synth.random_rays(np.random.default_rng(3), MAX_RAYS + 1, -1.5, 1.5)
        with pytest.raises(fb.FumengError) as e:
            scene.trace_closest_noalloc(rays)
        assert e.value.status == fb.FM_ERR_INVALID
        assert "262144" in str(e.value)
        obj, t = scene.trace_closest_noalloc(rays[:1000])   # still usable afterwards
        assert np.array_equal(obj, scene.trace_closest(rays[:1000])[0])
    finally:
        scene.destroy()
