"""The C-ABI library loads without a GPU and exports every symbol the header declares;
argument errors are reported before any CUDA call."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "us3d_b200.h").read_text()
    return sorted(set(re.findall(r"US3D_API\s+[\w\s\*]+?\b(us3d_\w+)\s*\(", text)))


def test_header_symbols_exported():
    from us3d_b200 import _lib

    lib = _lib.load()
    names = declared_symbols()
    assert "us3d_ug_bin" in names and "us3d_ug_backward" in names
    for n in names:
        assert hasattr(lib, n), n
    # the Python binding covers exactly what the header declares
    assert sorted(_lib.exported_symbols()) == names


def _declared_parameter_lists():
    text = (ROOT / "include" / "us3d_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    out = {}
    for m in re.finditer(r"US3D_API\s+([\w\s\*]+?)\b(us3d_\w+)\s*\(([^)]*)\)\s*;", text):
        params = " ".join(m.group(3).split())
        out[m.group(2)] = (m.group(1).strip(), [] if params in ("", "void") else params.split(","))
    return out


_CTYPE_OF = {"int32_t": "c_int", "int": "c_int", "int64_t": "c_long", "size_t": "c_ulong", "float": "c_float",
             "double": "c_double"}


def test_binding_signatures_match_header():
    """Every ctypes signature has the header's arity and, for scalar parameters, its type
    (pointers of any kind bind as c_void_p or POINTER(...))."""
    from us3d_b200 import _lib

    decl = _declared_parameter_lists()
    for name, (res, args) in _lib._SIGNATURES.items():
        ret, params = decl[name]
        assert len(args) == len(params), (name, len(args), len(params))
        for a, p in zip(args, params):
            p = p.strip()
            if "*" in p:
                assert a is ctypes.c_void_p or a is ctypes.c_char_p or hasattr(a, "_type_") and a.__name__.startswith(
                    "LP_"), (name, p, a)
            else:
                ctype = p.replace("const ", "").split()[0]
                assert a.__name__ == _CTYPE_OF[ctype], (name, p, a.__name__)


def test_slice_frame_layout():
    from us3d_b200 import _lib

    assert ctypes.sizeof(_lib.SliceFrame) == 96
    assert _lib.SliceFrame.height.offset == 64 and _lib.SliceFrame.tile_offset.offset == 84


def test_workspace_sizes():
    from us3d_b200 import _lib

    L = _lib.load()
    a = L.us3d_ug_workspace_bytes(1000, 1, 64, 16384, 0)
    b = L.us3d_ug_workspace_bytes(1000, 1, 64, 16384, 1000)
    assert b - a >= 20 * 1000 and a > 0
    assert L.us3d_ug_workspace_bytes(-1, 1, 64, 16384, 0) == 0
    assert L.us3d_ug_backward_scratch_bytes(10) == 480


def test_argument_errors_without_gpu():
    from us3d_b200 import _lib

    L = _lib.load()
    st = L.us3d_ug_bin(None, 0, None, 0, 0, 0, 0, None, None, None, None, 7.8, 1e-4, 1, 0, None)
    assert st == _lib.US3D_INVALID_ARG
    assert "workspace" in L.us3d_last_error().decode()
    st = L.us3d_ug_forward(None, None, 1, 1, 1, 1, 0, None, 7.8, 1e-4, 0.0, 0.0, None, None, None, None, None)
    assert st == _lib.US3D_INVALID_ARG
    with pytest.raises(ValueError, match="invalid argument"):
        _lib.check(st, "us3d_ug_forward")
    assert L.us3d_version() >= 100
