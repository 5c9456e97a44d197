"""Readers and writers of the reference's text input formats (libprt.so,
host code; no device needed).

* ``read_rect_file`` / ``write_rect_file``: data/Rect1024.txt of the R-tree
  programs (BotomUp-rtree.cu:669-698, TopDown-rtree.cu:487-497).
* ``read_polygon_file`` / ``write_polygon_file``: the base and overlay files
  of readData (vector_map_overlay_gpc_kernel.cu:752-888), including its
  quantised boxes (int)(v * 100000).
* ``layer_from_ref`` turns readData's single-contour CSR into a ``Layer``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import PRT_ERR_CAPACITY, check, lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def read_rect_file(path: str):
    """(boxes int64 [n, 4] as (x1, y1, x2, y2), keys int32 [n])."""
    n = C.c_int64(0)
    check(lib().prt_rect_file_count(path.encode(), C.byref(n)))
    boxes = np.zeros((n.value, 4), np.int64)
    keys = np.zeros(n.value, np.int32)
    got = C.c_int64(0)
    check(lib().prt_read_rect_file(path.encode(), _p(boxes), _p(keys), n.value, C.byref(got)))
    return boxes, keys


def write_rect_file(path: str, boxes, keys=None) -> None:
    b = np.ascontiguousarray(np.asarray(boxes, dtype=np.int64).reshape(-1, 4))
    k = None if keys is None else np.ascontiguousarray(np.asarray(keys, dtype=np.int32))
    check(lib().prt_write_rect_file(path.encode(), _p(b), _p(k), len(b)))


def read_polygon_file(path: str) -> dict:
    """readData's arrays for one file: num [P] int32, prefix [P] int64, hole
    [P] int32, mbr [P, 4] float64 (as written), rect [P, 4] int32 (readData's
    quantisation), vertex [V, 2] float64."""
    np_, nv = C.c_int64(0), C.c_int64(0)
    check(lib().prt_polygon_file_size(path.encode(), C.byref(np_), C.byref(nv)))
    P, V = np_.value, nv.value
    out = {"num": np.zeros(P, np.int32), "prefix": np.zeros(P, np.int64), "hole": np.zeros(P, np.int32),
           "mbr": np.zeros((P, 4), np.float64), "rect": np.zeros((P, 4), np.int32),
           "vertex": np.zeros((V, 2), np.float64)}
    rc = lib().prt_read_polygon_file(path.encode(), _p(out["num"]), _p(out["prefix"]), _p(out["hole"]),
                                     _p(out["mbr"]), _p(out["rect"]), _p(out["vertex"]), P, V)
    if rc == PRT_ERR_CAPACITY:
        raise RuntimeError(f"{path} changed while it was read")
    check(rc)
    return out


def write_polygon_file(path: str, num, hole, vertex) -> None:
    n = np.ascontiguousarray(np.asarray(num, dtype=np.int32))
    h = np.ascontiguousarray(np.asarray(hole, dtype=np.int32))
    v = np.ascontiguousarray(np.asarray(vertex, dtype=np.float64).reshape(-1, 2))
    assert int(n.sum()) == len(v), "vertex count differs from sum(num)"
    check(lib().prt_write_polygon_file(path.encode(), _p(n), _p(h), _p(v), len(n)))


def layer_from_ref(d: dict):
    """A Layer (one ring per polygon) from readData's num / prefix / hole /
    vertex arrays, as prt_overlay_run_ref interprets them."""
    from . import Layer

    P = len(d["num"])
    ring_vert = np.zeros(P + 1, np.int64)
    ring_vert[:P] = d["prefix"]
    ring_vert[P] = (d["prefix"][-1] + d["num"][-1]) if P else 0
    return Layer(np.arange(P + 1, dtype=np.int64), ring_vert, d["hole"], d["vertex"])


def layer_to_ref(layer_dict: dict) -> dict:
    """readData's arrays (num, prefix, hole, vertex) of a layer dict whose
    polygons each have one ring."""
    pr, rv = np.asarray(layer_dict["poly_ring"]), np.asarray(layer_dict["ring_vert"])
    assert np.array_equal(pr, np.arange(len(pr))), "one ring per polygon"
    num = np.diff(rv).astype(np.int32)
    return {"num": num, "prefix": rv[:-1].astype(np.int64), "hole": np.asarray(layer_dict["ring_hole"], np.int32),
            "vertex": np.asarray(layer_dict["xy"], np.float64)}
