"""Build the fumeng_b200 shared library in-tree with nvcc for sm_100a.

Usage: python -m fumeng_b200.build [--verbose] [--ptxas-v]

Compiles every fumeng_b200/csrc/*.cu and fumeng_b200/host/*.cpp into
fumeng_b200/libfumeng_b200.so (the C-ABI declared in include/fumeng_b200.h) and the
command-line renderer fumeng_b200/fumeng_b200_cli.  Objects are rebuilt only when a
source or header is newer than the object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
OBJ = PKG / "_build"
LIB = PKG / "libfumeng_b200.so"
CLI = PKG / "fumeng_b200_cli"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                  "-I", str(ROOT / "include")]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-I", str(ROOT / "include"), "-I", str(HOST)]


def _headers() -> list[Path]:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((ROOT / "include").glob("*.h"))
    if HOST.exists():
        hs += list(HOST.glob("*.h")) + list(HOST.glob("*.hpp"))
    return hs


def _stale(obj: Path, src: Path, headers: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {' '.join(cmd[:4])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(verbose: bool = False, ptxas_v: bool = False, force: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    headers = _headers()
    jobs = []
    objs = []
    for src in sorted(CSRC.glob("*.cu")):
        obj = OBJ / (src.stem + ".cu.o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            extra = ["-Xptxas", "-v"] if ptxas_v else []
            jobs.append([NVCC, *NVFLAGS, *extra, "-c", str(src), "-o", str(obj)])
    host_objs = []
    if HOST.exists():
        for src in sorted(HOST.glob("*.cpp")):
            obj = OBJ / (src.stem + ".cpp.o")
            if src.stem == "main":
                continue
            host_objs.append(obj)
            if force or _stale(obj, src, headers):
                jobs.append(["g++", *CXXFLAGS, "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        list(ex.map(lambda c: _run(c, verbose or ptxas_v), jobs))
    all_objs = objs + host_objs
    if force or jobs or not LIB.exists():
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, all_objs), "-lz"], verbose)
    main = HOST / "main.cpp"
    if main.exists() and (force or jobs or not CLI.exists() or main.stat().st_mtime > CLI.stat().st_mtime):
        _run(["g++", *CXXFLAGS, str(main), "-o", str(CLI), "-L", str(PKG), "-lfumeng_b200",
              f"-Wl,-rpath,{PKG}", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, ptxas_v=a.ptxas_v, force=a.force))
