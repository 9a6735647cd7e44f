"""The C-ABI library: it builds for sm_100a, loads, and exports every entry
point include/mts.h declares.  No compute call is made here."""
import ctypes
import os
import re

import mts_b200 as M
from conftest import ROOT


def header_functions():
    with open(os.path.join(ROOT, "include", "mts.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:mts_status|int32_t|const char\*)\s+(mts_\w+)\s*\(", text, re.M)))


def test_header_lists_match_binding():
    assert header_functions() == sorted(M.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = M.load()
    for name in header_functions():
        assert hasattr(lib, name), name
    assert lib.mts_version() == 100


def test_library_is_built_for_sm100a():
    import importlib.util

    spec = importlib.util.spec_from_file_location("b", os.path.join(ROOT, "matched-time-splitting-3d_b200", "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    assert mod.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert mod.up_to_date()


def test_struct_layouts():
    from mts_b200 import _lib

    assert ctypes.sizeof(_lib.mts_grid) == 64
    assert ctypes.sizeof(_lib.mts_surface) == 64
    assert ctypes.sizeof(_lib.mts_params) == 48
    assert M.CROSSING_DTYPE.itemsize == 296
