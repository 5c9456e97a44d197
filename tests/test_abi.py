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


def test_bad_arguments_are_rejected_before_any_device_work():
    from parlllelrtree_b200 import _lib

    L = _lib.lib()
    tree = ctypes.c_void_p()
    # fanout out of range, null boxes, unknown key mode, REF64 on float boxes
    assert L.prt_build_bottomup(ctypes.c_void_p(16), 1, None, 100, 1, 1, None, ctypes.byref(tree)) == _lib.PRT_ERR_INVALID
    assert L.prt_build_bottomup(None, 1, None, 100, 16, 1, None, ctypes.byref(tree)) == _lib.PRT_ERR_INVALID
    assert L.prt_build_bottomup(ctypes.c_void_p(16), 1, None, 100, 16, 7, None, ctypes.byref(tree)) == _lib.PRT_ERR_INVALID
    assert L.prt_build_bottomup(ctypes.c_void_p(16), 1, None, 100, 16, 0, None, ctypes.byref(tree)) == _lib.PRT_ERR_INVALID
    assert b"REF64" in L.prt_last_error()
    assert L.prt_tree_info(None, None) == _lib.PRT_ERR_INVALID


def test_without_a_device_compute_fails_loudly():
    """No CPU fallback: with no CUDA device a build returns PRT_ERR_CUDA/NOMEM."""
    from parlllelrtree_b200 import _lib

    L = _lib.lib()
    if L.prt_device_count() > 0:
        return  # on a GPU box this case cannot be produced
    tree = ctypes.c_void_p()
    rc = L.prt_build_bottomup(ctypes.c_void_p(256), 1, None, 100, 16, 1, None, ctypes.byref(tree))
    assert rc in (_lib.PRT_ERR_CUDA, _lib.PRT_ERR_NOMEM)
    assert L.prt_last_error()
