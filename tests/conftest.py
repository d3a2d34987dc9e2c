"""Test configuration: the `gpu` marker, import paths and the native builds.

CPU tests (`-m "not gpu"`) need the C++ oracle (oracle/liboracle.so) and the
product library (myrt_b200/libmyrt_b200.so, cross-compiled for sm_100a); both
are built here if missing. GPU tests call the product through its C ABI and
compare with the oracle.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))
GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    for script in (ROOT / "oracle" / "build.py", ROOT / "myrt_b200" / "build.py"):
        lib = ROOT / ("oracle/liboracle.so" if "oracle" in str(script) else "myrt_b200/libmyrt_b200.so")
        if not lib.exists():
            subprocess.run([sys.executable, str(script)], check=True)


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        return np.load(GOLDEN / name, allow_pickle=False)

    return load


@pytest.fixture(scope="session")
def ctx():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import myrt_b200

    c = myrt_b200.Context(0)
    yield c
    c.close()
