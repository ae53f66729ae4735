"""Build recipe for the engine library (vine_b200/libvine.so).

Compiles every CUDA / C++ source under vine_b200/csrc for sm_100a only and
links one shared library in-tree, so the built file travels with the source
tree.  Usage: ``python vine_b200/build.py [--force]`` (run as a file: importing
the package itself needs the built library).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libvine.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-Xptxas", "-v"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC"]


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers():
    inc = HERE.parent / "include"
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(inc.rglob("*.h"))


def _newest(paths):
    return max((p.stat().st_mtime for p in paths), default=0.0)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile and link libvine.so if any source is newer than the library."""
    srcs = _sources()
    hdr_time = _newest(_headers())
    BUILD.mkdir(exist_ok=True)
    objs = []
    for src in srcs:
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_time):
            continue
        if src.suffix == ".cu":
            cmd = [NVCC, *CUDA_FLAGS, "-c", str(src), "-o", str(obj)]
        else:
            cmd = [NVCC, "-x", "c++", *ARCH, "-Xcompiler", " ".join(CXX_FLAGS), "-std=c++17",
                   "-O3", "-c", str(src), "-o", str(obj)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        log = BUILD / (src.name + ".log")
        log.write_text(res.stdout + res.stderr)
        if verbose:
            sys.stderr.write(res.stderr)
        if res.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{res.stderr[-6000:]}")
    if force or not LIB.exists() or LIB.stat().st_mtime < _newest(objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs), "-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{res.stderr[-6000:]}")
    return LIB


if __name__ == "__main__":
    out = build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(out)
