"""Builds the in-tree shared library myrt_b200/libmyrt_b200.so with nvcc.

Device code is compiled for sm_100a only (B200). The library exports the C ABI
declared in include/myrt_cuda.h and links the CUDA runtime statically, so it
loads in any process (torch's own runtime is not involved).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libmyrt_b200.so"
BUILD = ROOT / "_build" / "myrt_b200"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_FLAGS = ["-O3", "-lineinfo", "-std=c++20", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-Xptxas",
              "-warn-spills"]
CXX_FLAGS = ["-O3", "-std=c++20", "-fPIC", "-pthread"]
# Translation units whose arithmetic must round every + and * separately (the
# shading restates GLSL expressions operation by operation).
NO_FMA = {"wavefront.cu", "physical.cu", "postprocess.cu", "raster.cu"}


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def needs_rebuild() -> bool:
    if not LIB.exists():
        return True
    mtime = LIB.stat().st_mtime
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp")) + [ROOT / "include" / "myrt_cuda.h"]
    return any(p.stat().st_mtime > mtime for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_rebuild():
        return LIB
    BUILD.mkdir(parents=True, exist_ok=True)
    objs = []
    for src in sources():
        obj = BUILD / (src.name + ".o")
        if src.suffix == ".cu":
            extra = ["-fmad=false"] if src.name in NO_FMA else []
            cmd = [NVCC, *ARCH, *CUDA_FLAGS, *extra, "-I", str(ROOT / "include"), "-c", str(src), "-o", str(obj)]
        else:
            cmd = ["g++", *CXX_FLAGS, "-I", str(ROOT / "include"), "-I", "/usr/local/cuda/include", "-c", str(src),
                   "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *objs, "-lpthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
