"""Loads libprt.so (the C ABI declared in include/prt.h) with ctypes.

There is no CPU fallback: if the library is missing or no CUDA device is
visible, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libprt.so")
CSRC = os.path.join(HERE, "csrc")

PRT_OK, PRT_ERR_INVALID, PRT_ERR_CAPACITY, PRT_ERR_TIMEOUT, PRT_ERR_CUDA, PRT_ERR_NOMEM = range(6)
COORD = {"i64": 0, "f32": 1, "f64": 2, "i32": 3}
KEY = {"ref64": 0, "morton32": 1}
OP = {"diff": 0, "int": 1, "xor": 2, "union": 3}
SCHED = {"plain": 0, "batched": 1}
MAX_LEVELS = 40

_lib = None

# name -> (restype, argtypes)
_P = C.c_void_p
_I = C.c_int
_I64 = C.c_int64
_SIGS = {
    "prt_last_error": (C.c_char_p, []),
    "prt_version": (_I, []),
    "prt_device_count": (_I, []),
    "prt_build_bottomup": (_I, [_P, _I, _P, _I64, _I, _I, _P, _P]),
    "prt_build_topdown": (_I, [_P, _I, _P, _I64, _I, _P, _P]),
    "prt_tree_free": (_I, [_P]),
    "prt_tree_info": (_I, [_P, _P]),
    "prt_tree_level_mbr": (_I, [_P, _I, _P]),
    "prt_tree_leaf_order": (_I, [_P, _P, _P]),
    "prt_tree_export_bu_size": (_I, [_P, _P]),
    "prt_tree_export_bu": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "prt_tree_export_td_size": (_I, [_P, _P, _P]),
    "prt_tree_export_td": (_I, [_P, _P, _P, _P]),
    "prt_join": (_I, [_P, _P, _I, _I64, _P, _I64, _P, _P]),
    "prt_join_sorted": (_I, [_P, _P, _I, _I64, _P, _I64, _P, _P]),
    "prt_join_noalloc": (_I, [_P, _P, _I, _I64, _P, _I64, _P, _P]),
    "prt_query_counts": (_I, [_P, _P, _I, _I64, _I, _P, _P]),
    "prt_tree_sibling_overlaps": (_I, [_P, _P, _P]),
    "prt_overlay_run": (_I, [_P, _I64, C.c_int32, _P, _P, _P, _I, _I, _P, _P]),
    "prt_overlay_run_ref": (_I, [_P, _I64, C.c_int32, _P, _P, _P, _P, _P, _I64, _P, _P, _P, _P, _I64, _I, _I,
                                 _P, _P]),
    "prt_results_sizes": (_I, [_P, _P]),
    "prt_results_device": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "prt_results_copy": (_I, [_P, _P, _P, _P, _P]),
    "prt_results_area": (_I, [_P, _P, _P]),
    "prt_results_copy_pairs": (_I, [_P, _P, _I64, _P, _P, _P, _P, _I64, _I64, _P]),
    "prt_results_free": (_I, [_P]),
    "prt_clip_pair_host": (_I, [_I, _I, _P, _P, _I, _P, _P, _P, C.c_int32, _P, _P, _P, _I64, _P]),
    "prt_schedule_set": (_I, [_P]),
    "prt_schedule_get": (_I, [_P]),
    "prt_layer_mbr": (_I, [_P, _P, _P]),
    "prt_layer_mbr_i32": (_I, [_P, C.c_double, _P, _P]),
    "prt_autotune": (_I, [_P, _P, _I, _I64, C.c_double, _P, _P]),
    "prt_pipeline_create": (_I, [_P, _P, _P, _P]),
    "prt_pipeline_run": (_I, [_P, _P]),
    "prt_pipeline_sizes": (_I, [_P, _P]),
    "prt_pipeline_pairs": (_I, [_P, _P, _I64, _P]),
    "prt_pipeline_results": (_I, [_P, _P, _P, _P, _P]),
    "prt_pipeline_free": (_I, [_P]),
    "prt_area_fwd": (_I, [_P, _P, _I64, _P, _P, _P, _P]),
    "prt_area_bwd": (_I, [_P, _P, _I64, _P, _P, _P, _P, _P, _P]),
    "prt_area_fwd_fallbacks": (_I, [_P]),
    "prt_debug_wait_limit": (_I, [_I, _I]),
    "prt_overlay_stream": (_I, [_P, _I64, C.c_int32, _P, _P, _P, _I, _I, _I64, _P, _P, _P]),
    "prt_rect_file_count": (_I, [C.c_char_p, _P]),
    "prt_read_rect_file": (_I, [C.c_char_p, _P, _P, _I64, _P]),
    "prt_write_rect_file": (_I, [C.c_char_p, _P, _P, _I64]),
    "prt_polygon_file_size": (_I, [C.c_char_p, _P, _P]),
    "prt_read_polygon_file": (_I, [C.c_char_p, _P, _P, _P, _P, _P, _P, _I64, _I64]),
    "prt_write_polygon_file": (_I, [C.c_char_p, _P, _P, _P, _I64]),
    "prt_profile_enable": (_I, [_I]),
    "prt_profile_focus": (_I, [C.c_char_p]),
    "prt_profile_reset": (_I, []),
    "prt_profile_read": (_I, [_P, _I, _P, _P, _I]),
}


def profile_enable(mode) -> None:
    """0/False off, 1/True time every launch, 2 count all and time only the
    focus kernel (profile_focus)."""
    lib().prt_profile_enable(int(mode))


def profile_focus(name: str) -> None:
    lib().prt_profile_focus(name.encode())


def profile_reset() -> None:
    lib().prt_profile_reset()


def profile_read() -> dict:
    """{kernel name: (summed device ms, launches)} since the last reset."""
    import numpy as np

    cap = 256
    names = C.create_string_buffer(1 << 16)
    ms = np.zeros(cap, dtype=np.float64)
    cnt = np.zeros(cap, dtype=np.int64)
    k = lib().prt_profile_read(names, 1 << 16, ms.ctypes.data_as(C.c_void_p), cnt.ctypes.data_as(C.c_void_p), cap)
    keys = names.value.decode().split("\n")[:k]
    return {keys[i]: (float(ms[i]), int(cnt[i])) for i in range(k)}


class PrtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"prt error {code}: {msg}")
        self.code = code


def build(force: bool = False) -> str:
    """Compiles libprt.so for sm_100a in-tree (nvcc; no GPU needed)."""
    cmd = ["make", "-s", "-C", CSRC, "-j8"]
    if force:
        cmd.insert(2, "-B")
    subprocess.run(cmd, check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with parlllelrtree_b200._lib.build() "
                               "(the library has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(rc: int) -> None:
    if rc != PRT_OK:
        msg = lib().prt_last_error()
        raise PrtError(rc, msg.decode() if msg else "")
