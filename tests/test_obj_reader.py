"""The scene loader's OBJ reader (fmhost::load_obj, used by fm_scene_load and the
command-line renderer), driven on the CPU through a small C++ program linked against the
library: the OBJ forms the reference's scenes use (v / vt / vn / f with v, v/vt, v//vn,
v/vt/vn corners, negative indices, polygons split into fans in file order), the number
forms strtof accepts, lines it must ignore, and its errors; plus an exact round trip of a
generated mesh."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from fumeng_b200.scene import Mesh, SceneSpec

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def dump(fm_lib, tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path_factory.mktemp("objdump") / "obj_reader_dump"
    pkg = ROOT / "fumeng_b200"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", str(ROOT / "include"), "-I", str(pkg / "host"),
                    str(ROOT / "tests" / "obj_reader_dump.cpp"), "-o", str(exe), "-L", str(pkg), "-lfumeng_b200",
                    f"-Wl,-rpath,{pkg}"], check=True, capture_output=True)

    def run(path):
        out = subprocess.run([str(exe), str(path)], check=True, capture_output=True, text=True).stdout
        if out.startswith("error:"):
            return out.strip()
        lines = out.split("\n")
        nv, nvt, nvn, nf = (int(x) for x in lines[0].split())
        # %.9g round-trips every float32 exactly
        v, vt, vn = (np.array([float(x) for x in lines[k].split()], np.float64).astype(np.float32) for k in (1, 2, 3))
        f = np.array([int(x) for x in lines[4].split()], np.int64).reshape(-1, 3, 3) if nf else np.zeros((0, 3, 3))
        assert (len(v), len(vt), len(vn), len(f)) == (nv, nvt, nvn, nf)
        return v, vt, vn, f
    return run


def test_obj_forms(dump, tmp_path):
    p = tmp_path / "forms.obj"
    p.write_text("# comment\n"
                 "v 0 0 0\n"
                 "v 1.5 0 0 1\n"            # w ignored
                 "v\t0 2.25e0 0\r\n"        # tab, CRLF
                 "v 1 1\n"                  # missing z -> 0
                 "v 0x1p1 -0 +3\n"          # hexadecimal, signed zero, leading '+'
                 "v 1.5abc 2 3\n"           # trailing characters after a number
                 "vt 0.5\n"                 # missing v -> 0
                 "vt 0.25 0.75 0\n"
                 "vn 0 0 1\n"
                 "f 1 2 3\n"
                 "f 1/1 2/2 3/1\n"
                 "f 1//1 2//1 3//1\n"
                 "f 1/1/1 2/2/1 3/2/1 4/1/1\n"   # quad -> two triangles (0,1,2), (0,2,3)
                 "f -1 -2 -3\n"
                 "g group\nusemtl m\ns off\no obj\n\nv\nf\nx\n"
                 "f 2 3 4 5 6\n"            # pentagon -> three triangles
                 "v 9 9 9")                 # no final newline
    v, vt, vn, f = dump(p)
    np.testing.assert_array_equal(v, [0, 0, 0, 1.5, 0, 0, 0, 2.25, 0, 1, 1, 0, 2, -0.0, 3, 1.5, 2, 3, 9, 9, 9])
    assert np.signbit(v[13])
    np.testing.assert_array_equal(vt, [0.5, 0, 0.25, 0.75])
    np.testing.assert_array_equal(vn, [0, 0, 1])
    corners = f.tolist()
    assert corners[0] == [[0, -1, -1], [1, -1, -1], [2, -1, -1]]
    assert corners[1] == [[0, 0, -1], [1, 1, -1], [2, 0, -1]]
    assert corners[2] == [[0, -1, 0], [1, -1, 0], [2, -1, 0]]
    assert corners[3] == [[0, 0, 0], [1, 1, 0], [2, 1, 0]] and corners[4] == [[0, 0, 0], [2, 1, 0], [3, 0, 0]]
    assert corners[5] == [[5, -1, -1], [4, -1, -1], [3, -1, -1]]   # -1 is the latest vertex (6th)
    assert [c[0][0] for c in corners[6:9]] == [1, 1, 1] and [c[2][0] for c in corners[6:9]] == [3, 4, 5]
    assert len(corners) == 9


def test_obj_numbers_as_strtof(dump, tmp_path):
    p = tmp_path / "numbers.obj"
    p.write_text("v 1e40 -1e40 1e-50\nv 3.4028235e38 1.17549435e-38 1e-40\nv inf -INF 00012.5\n"
                 "v .5 5. 1e\n")
    v, _, _, _ = dump(p)
    f32 = np.finfo(np.float32)
    assert np.isposinf(v[0]) and np.isneginf(v[1]) and v[2] == 0.0
    assert v[3] == f32.max and v[4] == f32.tiny
    assert v[5] == np.float32(1e-40)   # subnormal, correctly rounded
    assert np.isposinf(v[6]) and np.isneginf(v[7]) and v[8] == 12.5
    np.testing.assert_array_equal(v[9:], [0.5, 5.0, 1.0])


def test_obj_errors(dump, tmp_path):
    p = tmp_path / "bad.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nf 1 2 7\n")
    assert dump(p) == f"error: bad OBJ vertex index: {p}"
    assert dump(tmp_path / "missing.obj") == f"error: Loading model failed: {tmp_path / 'missing.obj'}"


def test_generated_mesh_round_trips(dump, tmp_path):
    rng = np.random.default_rng(5)
    verts = (rng.standard_normal((500, 3)) * 3).astype(np.float32)
    faces = rng.integers(0, 500, size=(900, 3))
    uvs = rng.random((500, 2)).astype(np.float32)
    spec = SceneSpec({"type": "pin_hole", "pos": [0, 0, 5], "look_at": [0, 0, 0], "up": [0, 1, 0]},
                     {"width": 4, "height": 4, "spp": 1},
                     [{"name": "m", "type": "lambert_diffuse", "basecolor": [0.5, 0.5, 0.5]}],
                     [Mesh(verts, faces, "m", uvs=uvs)])
    spec.write(tmp_path)
    objs = sorted(tmp_path.rglob("*.obj"))
    assert len(objs) == 1
    v, vt, _, f = dump(objs[0])
    np.testing.assert_array_equal(v, verts.reshape(-1))
    np.testing.assert_array_equal(vt, uvs.reshape(-1))
    np.testing.assert_array_equal(f[:, :, 0], faces)
