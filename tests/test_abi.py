"""The C-ABI library loads and exports every entry point include/prt.h
declares (no compute calls: these run without a GPU)."""
import ctypes
import os
import re

from conftest import ROOT


def declared():
    src = open(os.path.join(ROOT, "include", "prt.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(prt_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    for must in ("prt_build_bottomup", "prt_build_topdown", "prt_join", "prt_overlay_run", "prt_area_bwd"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from parlllelrtree_b200 import _lib

    path = _lib.LIB_PATH
    if not os.path.exists(path):
        _lib.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(declared()) <= set(_lib.exported_symbols())


def test_no_device_is_reported_not_faked():
    from parlllelrtree_b200 import _lib

    L = _lib.lib()
    n = L.prt_device_count()
    assert n >= 0
    assert L.prt_version() == 1
