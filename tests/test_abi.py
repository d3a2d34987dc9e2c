"""The C-ABI library loads and exports every symbol the public header declares.
No compute call is made here (no GPU needed)."""
import ctypes
import re
from pathlib import Path

import myrt_b200
from myrt_b200 import _abi

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"^\s*int\s+(myrt_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_abi.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_the_header():
    assert declared_functions() <= set(_abi.SIGNATURES)


def test_struct_sizes_match_header():
    assert ctypes.sizeof(_abi.myrt_drawable) == 160  # scene::drawable_geometry_t
    assert ctypes.sizeof(_abi.myrt_material_ref) == 8
    assert myrt_b200.HIT_DTYPE.itemsize == 16


def test_invalid_arguments_are_reported_without_a_device():
    L = _abi.lib()
    assert L.myrt_bvh8_build(None, 5, ctypes.byref(ctypes.c_void_p())) == _abi.MYRT_ERR_INVALID_ARGUMENT
    assert L.myrt_ctx_destroy(None) == _abi.MYRT_OK
    assert L.myrt_trace_closest(None, None, 0, None, 0) == _abi.MYRT_ERR_INVALID_ARGUMENT
    assert L.myrt_sync(None) == _abi.MYRT_ERR_INVALID_ARGUMENT
