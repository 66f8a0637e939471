"""The C-ABI library builds, loads and exports every entry point include/*.h declares
(CPU only: no compute calls)."""
import ctypes as C
import re
from pathlib import Path

import fumeng_b200

ROOT = Path(__file__).resolve().parents[1]


def declared_entry_points():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        src = h.read_text()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(fm_[a-z_0-9]+)\s*\(", src))
    return sorted(names)


def test_library_exports_declared_symbols(fm_lib):
    names = declared_entry_points()
    assert "fm_render" in names and "fm_trace_closest" in names
    lib = C.CDLL(str(fumeng_b200.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_covers_declared_symbols():
    assert set(declared_entry_points()) <= set(fumeng_b200.EXPORTED_SYMBOLS)


def test_errors_without_device(fm_lib):
    import torch
    if torch.cuda.is_available():
        return
    h = C.c_void_p()
    st = fm_lib.fm_ctx_create(0, C.byref(h))
    assert st == fumeng_b200.FM_ERR_NO_DEVICE
    assert not h.value
    assert fm_lib.fm_last_error(None) == b"null context"


def test_struct_layouts_match_the_header(tmp_path):
    # the ctypes mirrors of the header's structs have the C compiler's sizes and offsets
    import subprocess
    structs = {"fm_texture_desc": fumeng_b200.TextureDesc, "fm_tex_ref": fumeng_b200.TexRef,
               "fm_material_desc": fumeng_b200.MaterialDesc, "fm_light_desc": fumeng_b200.LightDesc,
               "fm_scene_desc": fumeng_b200.SceneDesc, "fm_camera": fumeng_b200.Camera,
               "fm_render_params": fumeng_b200.RenderParams, "fm_render_stats": fumeng_b200.RenderStats,
               "fm_tuning": fumeng_b200.Tuning, "fm_grad_desc": fumeng_b200.GradDesc,
               "fm_post_step": fumeng_b200.PostStep}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "fumeng_b200.h"', 'int main(void) {']
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"
