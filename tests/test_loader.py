"""The C++ scene loader (drop-in for SceneLoader::Load / DrawFrame): schema defaults and
error behaviour (CPU), and bit-identical renders of JSON-loaded vs. directly flattened
scenes (GPU)."""
import json

import numpy as np
import pytest

import fumeng_b200 as fb
from fumeng_b200 import synth


def test_parse_only_reads_camera_and_renderer(fm_lib, tmp_path):
    spec = synth.material_scene(3, res=40, spp=7, depth=6)
    p = spec.write(tmp_path)
    st, cam, params = fb.parse_scene_file(p)
    assert st == fb.FM_OK
    assert cam.type == fb.FM_CAMERA_PINHOLE
    assert list(cam.pos) == pytest.approx([0.0, -3.2, 1.4])
    assert cam.fov == pytest.approx(45.0)
    assert (params.width, params.height, params.spp, params.depth) == (40, 40, 7, 6)
    assert params.rr_depth == 3 and params.rr_coef == pytest.approx(0.85)
    assert params.direct_loop == 1   # default (core/renderer.h:48)


def test_defaults_follow_the_reference(fm_lib, tmp_path):
    doc = {"camera": {"type": "thin_lens", "lens_radius": 0.25},
           "renderer": {"type": "path_tracer"},
           "scene": {"render_objects": [{"shape": {"type": "sphere"}}]}}
    (tmp_path / "s.json").write_text(json.dumps(doc))
    st, cam, params = fb.parse_scene_file(tmp_path / "s.json")
    assert st == fb.FM_OK
    # PinHoleCameraConfig defaults (core/camera.h:9-29) and RendererConfig defaults
    assert cam.type == fb.FM_CAMERA_THIN_LENS and cam.lens_radius == pytest.approx(0.25)
    assert list(cam.up) == [0.0, 0.0, 1.0] and cam.fov == pytest.approx(60.0) and cam.focal_distance == 1.0
    assert (params.width, params.height, params.spp, params.depth, params.rr_depth) == (1, 1, 10, 10, 10)


@pytest.mark.parametrize("doc", [
    {"renderer": {"type": "path_tracer"}, "scene": {}},                        # no camera
    {"camera": {"type": "orthographic"}, "renderer": {}, "scene": {}},          # unknown camera
    {"camera": {}, "scene": {}},                                                # no renderer
    {"camera": {}, "renderer": {}},                                             # no scene
    {"camera": {}, "renderer": {}, "scene": {"materials": [{"name": "x", "type": "glossy"}]}},
    {"camera": {}, "renderer": {}, "scene": {"render_objects": [{"shape": {"type": "triangle_mesh", "path": "none.obj"}}]}},
])
def test_invalid_scene_files_are_rejected(fm_lib, tmp_path, doc):
    (tmp_path / "s.json").write_text(json.dumps(doc))
    st, _, _ = fb.parse_scene_file(tmp_path / "s.json")
    assert st == fb.FM_ERR_INVALID


def test_malformed_json_is_rejected(fm_lib, tmp_path):
    (tmp_path / "s.json").write_text('{"camera": {"pos": [1, 2,}')
    st, _, _ = fb.parse_scene_file(tmp_path / "s.json")
    assert st == fb.FM_ERR_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("builder", [lambda: synth.cornell(res=48), lambda: synth.material_scene(3, res=40)],
                         ids=["cornell", "materials"])
def test_json_scene_renders_like_flattened_scene(ctx, tmp_path, builder):
    spec = builder()
    path = spec.write(tmp_path)
    a_scene, cam, params = ctx.load_scene(path)
    b_scene = ctx.create_scene(spec.to_desc())
    try:
        params.spp = 16
        params.seed = 3
        params.mode = fb.FM_MODE_MEGAKERNEL
        a = a_scene.render(cam, params)[0]
        b = b_scene.render(spec.camera_struct(), params)[0]
    finally:
        a_scene.destroy()
        b_scene.destroy()
    assert np.array_equal(a, b)


@pytest.mark.gpu
def test_draw_frame_writes_the_reference_outputs(ctx, tmp_path):
    spec = synth.cornell(res=32, spp=4)
    path = spec.write(tmp_path, output="frame")
    ctx.draw_frame(path)
    for suffix in ("", "_albedo", "_normal"):
        f = tmp_path / f"frame{suffix}.png"
        assert f.exists() and f.stat().st_size > 100
    from PIL import Image
    img = np.asarray(Image.open(tmp_path / "frame.png"))
    assert img.shape == (32, 32, 3) and img.max() > 0
