"""Builds libmeshless_vis.so in-tree with nvcc for sm_100a.

    python -m libmeshlessvis_b200.build        (or python libmeshlessvis_b200/build.py)

Every .cu/.cpp under csrc/ is compiled with
-gencode arch=compute_100a,code=sm_100a and linked with cuFFT into
libmeshlessvis_b200/libmeshless_vis.so.  Objects go to csrc/_build/.
Rebuilds only what changed (by mtime, headers included).
"""
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = CSRC / "_build"
INCLUDE = ROOT / "include"
LIB = PKG / "libmeshless_vis.so"
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
HOST_CXX = shutil.which("g++", path="/usr/bin") or "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
          "-I", str(INCLUDE), "-I", str(CSRC), "-ccbin", HOST_CXX, "--expt-relaxed-constexpr"]


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers():
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[-1]}")
    return r.stdout + r.stderr


def build(verbose=False, force=False, ptxas_info=False):
    nvcc = str(CUDA_HOME / "bin" / "nvcc")
    OBJ.mkdir(exist_ok=True)
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0)
    objs = []
    for src in _sources():
        obj = OBJ / (src.name + ".o")
        objs.append(obj)
        stale = force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)
        if not stale:
            continue
        cmd = [nvcc, *ARCH, *COMMON, "-c", str(src), "-o", str(obj)]
        if ptxas_info and src.suffix == ".cu":
            cmd.insert(1, "-Xptxas=-v")
        out = _run(cmd)
        if verbose or ptxas_info:
            print(f"[build] {src.name}\n{out}", end="")
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-ccbin", HOST_CXX, "-o", str(LIB), *map(str, objs),
               "-L", str(CUDA_HOME / "lib64"), "-lcufft",
               "-Xlinker", f"-rpath={CUDA_HOME / 'lib64'}", "-Xlinker", "-Bsymbolic",
               "-Xlinker", "--exclude-libs=ALL"]
        _run(cmd)
        if verbose:
            print(f"[build] linked {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
