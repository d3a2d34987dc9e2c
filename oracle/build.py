"""Builds the CPU oracle (oracle/liboracle.so) and, when the reference tree is
present, oracle/_ref/libmyrt_ref.so (see build_ref.py).

TEST INFRASTRUCTURE ONLY: the product never loads either library.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SRCS = [HERE / "oracle.cpp", HERE / "oracle_render.cpp", HERE / "oracle_post.cpp"]
FLAGS = ["-std=c++20", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fwrapv", "-fno-fast-math", "-pthread"]


def build_oracle(force: bool = False) -> Path:
    deps = SRCS + sorted(HERE.glob("*.hpp"))
    if not force and LIB.exists() and all(p.stat().st_mtime <= LIB.stat().st_mtime for p in deps):
        return LIB
    subprocess.run(["g++", *FLAGS, *map(str, SRCS), "-o", str(LIB)], check=True)
    return LIB


def build_all(force: bool = False) -> None:
    build_oracle(force)
    from build_ref import main as build_ref_main  # noqa: E402  (sibling module)
    build_ref_main()


if __name__ == "__main__":
    sys.path.insert(0, str(HERE))
    build_all(force="--force" in sys.argv)
    print(LIB)
