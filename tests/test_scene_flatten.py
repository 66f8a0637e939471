"""The C++ scene loader's flattening (SceneLoader::Load: the reference's JSON schema, meshes
read from OBJ files on several host threads, objects flattened in file order) against
the Python flattening of the same scene (SceneSpec.to_desc), array for array, on the
CPU through a small C++ program linked against the library; and the loader's handling of
mesh files that fail (reported when their object is reached, in object order) and of one
file named by several objects."""
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from fumeng_b200 import synth

ROOT = Path(__file__).resolve().parents[1]
FIELDS = [("obj_material", np.int32), ("tri_pos", np.float32), ("tri_object", np.int32),
          ("rect_pts", np.float32), ("rect_object", np.int32), ("tri_uv", np.float32)]


@pytest.fixture(scope="module")
def flatten(fm_lib, tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path_factory.mktemp("flatdump") / "scene_flatten_dump"
    pkg = ROOT / "fumeng_b200"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", str(ROOT / "include"), "-I", str(pkg / "host"),
                    str(ROOT / "tests" / "scene_flatten_dump.cpp"), "-o", str(exe), "-L", str(pkg), "-lfumeng_b200",
                    f"-Wl,-rpath,{pkg}"], check=True, capture_output=True)

    def run(scene_json, out):
        msg = subprocess.run([str(exe), str(scene_json), str(out)], check=True, capture_output=True,
                             text=True).stdout.strip()
        if msg != "ok":
            return msg
        b = Path(out).read_bytes()
        recs, i = {}, 0
        while i < len(b):
            name = b[i:i + 16].split(b"\0")[0].decode()
            es, n = (int.from_bytes(b[i + 16 + 8 * k:i + 24 + 8 * k], "little") for k in (0, 1))
            i += 32
            recs[name] = b[i:i + es * n]
            i += es * n
        return {k: np.frombuffer(recs[k], dt) for k, dt in FIELDS}
    return run


@pytest.mark.parametrize("name", ["materials", "batch16", "inverse"])
def test_loader_flattening_matches_python(flatten, tmp_path, name):
    spec = {"materials": lambda: synth.material_scene(3), "batch16": lambda: synth.batch_scene(16),
            "inverse": lambda: synth.inverse_scene(target=True)}[name]()
    got = flatten(spec.write(tmp_path), tmp_path / "flat.bin")
    want = spec.to_desc()
    for k, dt in FIELDS:
        ref = getattr(want, k, None)
        if ref is None:
            continue   # the Python side leaves absent attributes out
        np.testing.assert_array_equal(got[k], np.asarray(ref).reshape(-1).astype(dt), err_msg=k)


def _two_mesh_scene(tmp_path):
    spec = synth.material_scene(3)
    p = spec.write(tmp_path)
    doc = json.loads(p.read_text())
    objs = doc["scene"]["render_objects"]
    mesh = next(o for o in objs if o["shape"]["type"] == "triangle_mesh")
    return p, doc, objs, mesh


def test_shared_mesh_file_flattens_once_per_object(flatten, tmp_path):
    p, doc, objs, mesh = _two_mesh_scene(tmp_path)
    base = flatten(p, tmp_path / "a.bin")
    ntri = len(base["tri_object"])
    objs.append(json.loads(json.dumps(mesh)))   # the same OBJ file again, as the last object
    p.write_text(json.dumps(doc))
    got = flatten(p, tmp_path / "b.bin")
    assert len(got["tri_object"]) == 2 * ntri
    np.testing.assert_array_equal(got["tri_pos"][: 9 * ntri], got["tri_pos"][9 * ntri:])
    # the new object's triangles are numbered after every earlier object
    assert got["tri_object"][ntri:].min() == len(base["obj_material"])


def test_failing_mesh_files_are_reported_in_object_order(flatten, tmp_path):
    p, doc, objs, mesh = _two_mesh_scene(tmp_path)
    bad = tmp_path / "bad.obj"
    bad.write_text("v 0 0 0\nv 1 0 0\nf 1 2 9\n")
    first = json.loads(json.dumps(mesh))
    first["shape"]["path"] = "bad.obj"
    second = json.loads(json.dumps(mesh))
    second["shape"]["path"] = "missing.obj"
    objs[:0] = [first, second]
    p.write_text(json.dumps(doc))
    assert flatten(p, tmp_path / "c.bin") == f"error: bad OBJ vertex index: {bad}"
    objs[:2] = [second, first]
    p.write_text(json.dumps(doc))
    assert flatten(p, tmp_path / "d.bin") == f"error: Loading model failed: {tmp_path / 'missing.obj'}"
