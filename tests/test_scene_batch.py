"""fm_scene_create_batch: scenes created together are the scenes fm_scene_create makes one
at a time -- the same BVH statistics, bit-identical closest hits, occlusion and
(deterministic megakernel) renders -- for a batch larger than the builder's stream count,
with textures, an environment map, mesh lights, spheres and an empty scene; a batch with
one invalid description creates nothing and leaves the context usable."""
import types

import numpy as np
import pytest

import fumeng_b200 as fb
from fumeng_b200 import synth


def _specs():
    base = [synth.hit_scene(1, level=3, spheres=4), synth.textured_scene(res=16, spp=4),
            synth.emitters_scene(res=16, spp=4, accelerator="embree"),
            synth.batch_scene(2, env_w=64, env_h=32, res=16, spp=4), synth.cornell(res=16, spp=4)]
    return base + [synth.batch_scene(s, env_w=64, env_h=32, res=16, spp=4) for s in (3, 6, 13, 22, 27, 30)]


def _rays(spec, seed):
    rng = np.random.default_rng(seed)
    return synth.pinhole_rays(rng, spec.camera, 48, 32)


@pytest.mark.gpu
def test_batch_matches_one_at_a_time(ctx):
    specs = _specs()
    holders = [s.to_desc() for s in specs]
    empty = types.SimpleNamespace(desc=fb.SceneDesc())
    batch = ctx.create_scenes(holders + [empty])
    single = [ctx.create_scene(h) for h in holders]
    try:
        assert len(batch) == len(holders) + 1
        for i, (spec, b, s) in enumerate(zip(specs, batch, single)):
            sb, ss = b.bvh_stats(), s.bvh_stats()
            assert (sb["nodes"], sb["prims"], sb["depth"]) == (ss["nodes"], ss["prims"], ss["depth"]), i
            rays = _rays(spec, 100 + i)
            ob, tb = b.trace_closest(rays)
            os_, ts = s.trace_closest(rays)
            assert (ob >= 0).sum() > 100, i
            assert np.array_equal(ob, os_) and np.array_equal(tb, ts), i
            assert np.array_equal(b.trace_any(rays), s.trace_any(rays)), i
            p = spec.render_params(spp=4, mode=fb.FM_MODE_MEGAKERNEL)
            rb = b.render(spec.camera_struct(), p)
            rs = s.render(spec.camera_struct(), p)
            for x, y in zip(rb[:3], rs[:3]):
                assert np.array_equal(x, y), i
        e = batch[-1]
        assert e.bvh_stats()["prims"] == 0
        obj, t = e.trace_closest(_rays(specs[0], 1))
        assert (obj == -1).all() and np.isinf(t).all()
    finally:
        for sc in batch + single:
            sc.destroy()


@pytest.mark.gpu
def test_batch_with_an_invalid_scene_creates_nothing(ctx):
    specs = _specs()[:3]
    holders = [s.to_desc() for s in specs]
    bad = fb.SceneDesc.from_buffer_copy(holders[1].desc)
    bad.num_materials = 0   # every object's material index is now out of range
    with pytest.raises(fb.FumengError, match="material"):
        ctx.create_scenes([holders[0], types.SimpleNamespace(desc=bad), holders[2]])
    scenes = ctx.create_scenes(holders)
    try:
        obj, _ = scenes[0].trace_closest(_rays(specs[0], 7))
        assert (obj >= 0).sum() > 100
    finally:
        for sc in scenes:
            sc.destroy()
