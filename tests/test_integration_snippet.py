"""The reference-side binding shown in INTEGRATION.md compiles against the reference's
own headers and links against the reference's compiled engine (the oracle's float build)
and libfumeng_b200.so; the linked program constructs the renderer and calls it.  On a
machine without a GPU the call must come back through the C-ABI as the reference's own
error form (a std::runtime_error from fm_ctx_create's status), not crash.  CPU only."""
import re
import subprocess
from pathlib import Path

import pytest

import fumeng_b200

ROOT = Path(__file__).resolve().parents[1]
FLAGS = ROOT / "oracle" / "_ref" / "ref_flags.txt"
REF_LIB = ROOT / "oracle" / "_ref" / "libfmref_f.so"

MAIN = r"""
#include <cstdio>
#include <stdexcept>
int main(int argc, char** argv)
{
    fumeng::engine::PathTracerConfig cfg;
    fumeng::engine::GpuPathTracer r(cfg, argc > 1 ? argv[1] : "scene.json");
    try {
        r.DrawFrameFile();
        std::printf("rendered\n");
    } catch (const std::runtime_error& e) {
        std::printf("runtime_error: %s\n", e.what());
    }
    return 0;
}
"""


def snippet() -> str:
    text = (ROOT / "INTEGRATION.md").read_text()
    blocks = re.findall(r"```cpp\n(.*?)```", text, flags=re.S)
    assert blocks, "INTEGRATION.md has no C++ binding snippet"
    return blocks[0]


@pytest.mark.skipif(not (FLAGS.exists() and REF_LIB.exists()), reason="the oracle's reference build is absent here")
def test_integration_binding_compiles_links_and_runs(fm_lib, tmp_path):
    src = tmp_path / "gpu_path_tracing.cpp"
    src.write_text("#include <string>\n#include <utility>\n" + snippet() + MAIN)
    exe = tmp_path / "binding"
    flags = FLAGS.read_text().split()
    incs = [f[2:] for f in flags if f.startswith("-I")]
    if not any((Path(i) / "engine" / "core" / "renderer.h").exists() for i in incs):
        pytest.skip("the reference's headers are not on this machine")
    cmd = ["g++", *flags, "-I", str(ROOT / "include"), str(src), "-o", str(exe),
           "-L", str(REF_LIB.parent), "-lfmref_f", "-L", str(fumeng_b200.LIB_PATH.parent), "-lfumeng_b200",
           f"-Wl,-rpath,{REF_LIB.parent}", f"-Wl,-rpath,{fumeng_b200.LIB_PATH.parent}", "-pthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    run = subprocess.run([str(exe), str(tmp_path / "missing.json")], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stderr[-2000:]
    import torch
    if not torch.cuda.is_available():
        assert run.stdout.strip() == "runtime_error: no CUDA device", run.stdout
    else:
        # a missing scene file is the loader's error, reported through fm_last_error
        assert run.stdout.startswith("runtime_error:") and "missing.json" in run.stdout, run.stdout
