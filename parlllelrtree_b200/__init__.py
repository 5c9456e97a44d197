"""B200-native filter-and-refine spatial join and polygon overlay.

Python host mirror of the C ABI in ``include/prt.h`` (libprt.so, hand-written
sm_100a kernels).  PyTorch supplies device memory and streams only; every
computation runs in the library's CUDA kernels and there is no CPU fallback.

Reference path mirrored (ParlllelRtree):
  * ``build_bottomup``  BotomUp-rtree.cu:73-266, 373-426, 756-874 (Z-order
    keys, radix sort, level packing; leaves first, root last)
  * ``build_topdown``   TopDown-rtree.cu:162-353, 465-481, 504-687
  * ``Tree.join``       init/query1 BFS (BotomUp-rtree.cu:592-630), emitting
    the rtree_search {nodeid, queryid} pairs of
    vector_map_overlay_gpc_kernel.cu:89-90
  * ``Tree.query_counts`` RtreeSearch counters (BotomUp-rtree.cu:439-483)
  * ``overlay``         run()/Execute/gpc_polygon_clip
    (vector_map_overlay_gpc_kernel.cu:61-750)
  * ``intersection_area`` area of the GPC intersection with a hand-written
    adjoint (no reference counterpart).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import COORD, KEY, OP, SCHED, PrtError, check, lib

__all__ = [
    "Tree", "Layer", "Results", "build_bottomup", "build_topdown", "overlay", "overlay_ref", "clip_pair",
    "intersection_area", "IntersectionArea", "PrtError", "device_count", "Pipeline", "get_schedule",
    "set_schedule", "schedule", "autotune", "overlay_stream",
]

_DT2COORD = {torch.int64: COORD["i64"], torch.float32: COORD["f32"], torch.float64: COORD["f64"],
             torch.int32: COORD["i32"]}


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev_tensor(x, dtype=None):
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(np.ascontiguousarray(x))
    if dtype is not None:
        x = x.to(dtype)
    if not x.is_cuda:
        x = x.cuda()
    return x.contiguous()


def device_count() -> int:
    return int(lib().prt_device_count())


class Tree:
    """A device-resident R-tree (see include/prt.h for the layout)."""

    def __init__(self, handle: C.c_void_p, boxes: torch.Tensor):
        self._h = handle
        self._boxes = boxes  # keep the records alive (leaf MBRs are copies; ids are not)
        info = np.zeros(8 + _lib.MAX_LEVELS, dtype=np.int64)
        check(lib().prt_tree_info(self._h, info.ctypes.data_as(C.c_void_p)))
        self.n = int(info[0])
        self.fanout = int(info[1])
        self.levels = int(info[2])
        self.kind = "bottomup" if info[3] == 0 else "topdown"
        self.coord = int(info[4])
        self.level_counts = [int(c) for c in info[8:8 + self.levels]]

    def __del__(self):
        try:
            if self._h:
                lib().prt_tree_free(self._h)
                self._h = None
        except Exception:
            pass

    def level_mbr(self, level: int) -> np.ndarray:
        out = np.empty((self.level_counts[level], 4), dtype=np.float64)
        check(lib().prt_tree_level_mbr(self._h, level, out.ctypes.data_as(C.c_void_p)))
        return out

    def levels_mbr(self):
        return [self.level_mbr(l) for l in range(self.levels)]

    def leaf_order(self) -> torch.Tensor:
        """Record id of every leaf entry (the zOrder[].index remap), int32 [n]."""
        out = torch.empty(self.n, dtype=torch.int32, device="cuda")
        check(lib().prt_tree_leaf_order(self._h, _ptr(out), _stream()))
        return out

    def export_bu(self) -> dict:
        nn = C.c_int64(0)
        check(lib().prt_tree_export_bu_size(self._h, C.byref(nn)))
        n, F = nn.value, self.fanout
        flag = np.zeros(n, np.int32)
        num = np.zeros(n, np.int32)
        mbr = np.zeros((n, F, 4), np.float64)
        ch = np.zeros((n, F), np.int32)
        data = np.zeros((n, F), np.int32)
        root = C.c_int32(0)
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        check(lib().prt_tree_export_bu(self._h, p(flag), p(num), p(mbr), p(ch), p(data), C.byref(root)))
        return {"flag": flag, "num": num, "mbr": mbr, "children": ch, "data": data, "root": root.value}

    def export_td(self) -> dict:
        ns, no = C.c_int64(0), C.c_int32(0)
        check(lib().prt_tree_export_td_size(self._h, C.byref(ns), C.byref(no)))
        idx = np.zeros(ns.value, np.int32)
        mbr = np.zeros((ns.value, 4), np.float64)
        offs = np.zeros(no.value, np.int32)
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        check(lib().prt_tree_export_td(self._h, p(idx), p(mbr), p(offs)))
        return {"nodes_index": idx, "nodes_mbr": mbr, "offsets": offs}

    def _queries(self, q):
        q = _dev_tensor(q)
        if _DT2COORD.get(q.dtype) != self.coord:
            raise PrtError(_lib.PRT_ERR_INVALID, f"query dtype {q.dtype} differs from the tree's coordinates")
        return q

    def join(self, queries, cap: int | None = None, sorted: bool = False) -> torch.Tensor:
        """All intersecting (leaf entry, query) pairs, int32 [P, 2] on the device."""
        q = self._queries(queries)
        fn = lib().prt_join_sorted if sorted else lib().prt_join
        count = C.c_int64(0)
        if cap is None:
            check(lib().prt_join(self._h, _ptr(q), self.coord, len(q), None, 0, C.byref(count), _stream()))
            cap = max(int(count.value), 1)
        out = torch.empty((cap, 2), dtype=torch.int32, device="cuda")
        rc = fn(self._h, _ptr(q), self.coord, len(q), _ptr(out), cap, C.byref(count), _stream())
        if rc == _lib.PRT_ERR_CAPACITY:
            return self.join(queries, cap=int(count.value), sorted=sorted)
        check(rc)
        return out[: count.value]

    def query_counts(self, queries, td_slots: bool = False) -> torch.Tensor:
        """Per query (entries examined, sum of max(0, hits - 1) per node, leaf hits)."""
        q = self._queries(queries)
        out = torch.zeros((len(q), 3), dtype=torch.int64, device="cuda")
        check(lib().prt_query_counts(self._h, _ptr(q), self.coord, len(q), 1 if td_slots else 0, _ptr(out),
                                     _stream()))
        return out

    def sibling_overlaps(self) -> int:
        """Overlapping sibling-entry pairs over all nodes: the reference's
        RtreeSearch1 digest (BotomUp-rtree.cu:574-590)."""
        n = C.c_int64(0)
        check(lib().prt_tree_sibling_overlaps(self._h, C.byref(n), _stream()))
        return int(n.value)

    def digests(self, queries, td_slots: bool = False):
        """The reference programs' printed digests sum, sum1, sum2, sum3 for a
        self-join (BotomUp-rtree.cu:1023-1027, TopDown-rtree.cu:794-798)."""
        c = self.query_counts(queries, td_slots).cpu().numpy()
        return int(c[:, 0].sum()), int(c[:, 1].sum()), int(c[:, 2].sum()) // 2, self.sibling_overlaps()


def _build(fn, boxes, *args):
    b = _dev_tensor(boxes)
    if b.dim() != 2 or b.shape[1] != 4:
        raise PrtError(_lib.PRT_ERR_INVALID, "boxes must be [n, 4] (x1, y1, x2, y2)")
    coord = _DT2COORD.get(b.dtype)
    if coord is None:
        raise PrtError(_lib.PRT_ERR_INVALID, f"unsupported box dtype {b.dtype}")
    h = C.c_void_p()
    return b, coord, h


def build_bottomup(boxes, fanout: int = 16, key_mode: str = "morton32", ids=None) -> Tree:
    b, coord, h = _build(None, boxes)
    idt = _dev_tensor(ids, torch.int32) if ids is not None else None
    check(lib().prt_build_bottomup(_ptr(b), coord, _ptr(idt), len(b), fanout, KEY[key_mode], _stream(),
                                   C.byref(h)))
    t = Tree(h, b)
    t._ids = idt
    return t


def build_topdown(boxes, fanout: int = 16, ids=None) -> Tree:
    b, coord, h = _build(None, boxes)
    idt = _dev_tensor(ids, torch.int32) if ids is not None else None
    check(lib().prt_build_topdown(_ptr(b), coord, _ptr(idt), len(b), fanout, _stream(), C.byref(h)))
    t = Tree(h, b)
    t._ids = idt
    return t


class _LayerStruct(C.Structure):
    _fields_ = [("poly_ring", C.c_void_p), ("ring_vert", C.c_void_p), ("ring_hole", C.c_void_p),
                ("xy", C.c_void_p), ("n_poly", C.c_int64)]


class Layer:
    """A polygon layer on the device (ring CSR; see datagen.py)."""

    def __init__(self, poly_ring, ring_vert, ring_hole, xy):
        self.poly_ring = _dev_tensor(poly_ring, torch.int64)
        self.ring_vert = _dev_tensor(ring_vert, torch.int64)
        self.ring_hole = _dev_tensor(ring_hole, torch.int32)
        self.xy = _dev_tensor(xy, torch.float64)
        self.n_poly = len(self.poly_ring) - 1

    @classmethod
    def from_dict(cls, d: dict) -> "Layer":
        return cls(d["poly_ring"], d["ring_vert"], d["ring_hole"], d["xy"])

    def struct(self, xy: torch.Tensor | None = None) -> _LayerStruct:
        x = self.xy if xy is None else xy
        return _LayerStruct(self.poly_ring.data_ptr(), self.ring_vert.data_ptr(), self.ring_hole.data_ptr(),
                            x.data_ptr(), self.n_poly)

    def mbr(self, xy: torch.Tensor | None = None) -> torch.Tensor:
        """float64 [P, 4] polygon bounding boxes (x1, y1, x2, y2) over all
        rings (prt_layer_mbr), optionally for replacement coordinates xy."""
        out = torch.empty((self.n_poly, 4), dtype=torch.float64, device=self.xy.device)
        s = self.struct(xy)
        check(lib().prt_layer_mbr(C.byref(s), _ptr(out), _stream()))
        return out

    def mbr_quantised(self, scale: float = 1e5, xy: torch.Tensor | None = None) -> torch.Tensor:
        """int32 [P, 4] polygon bounding boxes quantised as the reference's
        readData does, (int)(v * scale) truncated toward zero
        (vector_map_overlay_gpc_kernel.cu:805-808, 845-848); a tree built on
        them (PRT_COORD_I32) gives the reference's candidate set."""
        out = torch.empty((self.n_poly, 4), dtype=torch.int32, device=self.xy.device)
        s = self.struct(xy)
        check(lib().prt_layer_mbr_i32(C.byref(s), C.c_double(scale), _ptr(out), _stream()))
        return out


class Results:
    """Per-pair GPC results, device resident (the reference's gpc_polygon array)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        s = np.zeros(8, dtype=np.int64)
        check(lib().prt_results_sizes(self._h, s.ctypes.data_as(C.c_void_p)))
        self.n_pairs, self.n_contours, self.n_vertices, self.nonempty, self.retried = (int(x) for x in s[:5])

    def __del__(self):
        try:
            if self._h:
                lib().prt_results_free(self._h)
                self._h = None
        except Exception:
            pass

    def to_host(self):
        """(pair_cont_off [P+1], cont_nverts [C], cont_hole [C], xy [V, 2]) in pair order."""
        off = np.zeros(self.n_pairs + 1, np.int64)
        nv = np.zeros(max(self.n_contours, 1), np.int32)
        hole = np.zeros(max(self.n_contours, 1), np.int32)
        xy = np.zeros((max(self.n_vertices, 1), 2), np.float64)
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        check(lib().prt_results_copy(self._h, p(off), p(nv), p(hole), p(xy)))
        return off, nv[: self.n_contours], hole[: self.n_contours], xy

    def contours(self):
        """List per pair of (hole, [k, 2] vertices) contours, GPC order."""
        off, nv, hole, xy = self.to_host()
        vo = np.zeros(len(nv) + 1, np.int64)
        np.cumsum(nv, out=vo[1:])
        out = []
        for i in range(self.n_pairs):
            out.append([(int(hole[c]), xy[vo[c]:vo[c + 1]]) for c in range(off[i], off[i + 1])])
        return out

    def contours_of(self, pairs) -> list:
        """Contours of the listed pairs only (prt_results_copy_pairs), as
        contours() gives them: per pair a list of (hole, [k, 2] vertices)."""
        idx = np.ascontiguousarray(np.asarray(pairs, dtype=np.int64))
        k = len(idx)
        off = np.zeros(k + 1, np.int64)
        need = np.zeros(2, np.int64)
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        cc, vc = 64, 4096
        while True:
            nv = np.zeros(cc, np.int32)
            hole = np.zeros(cc, np.int32)
            xy = np.zeros((vc, 2), np.float64)
            rc = lib().prt_results_copy_pairs(self._h, p(idx), k, p(off), p(nv), p(hole), p(xy), cc, vc, p(need))
            if rc == _lib.PRT_ERR_CAPACITY:
                cc, vc = max(cc, int(need[0])), max(vc, int(need[1]))
                continue
            check(rc)
            break
        vo = np.zeros(int(need[0]) + 1, np.int64)
        np.cumsum(nv[: int(need[0])], out=vo[1:])
        return [[(int(hole[c]), xy[vo[c]:vo[c + 1]].copy()) for c in range(off[j], off[j + 1])] for j in range(k)]

    def area(self) -> torch.Tensor:
        out = torch.empty(self.n_pairs, dtype=torch.float64, device="cuda")
        check(lib().prt_results_area(self._h, _ptr(out), _stream()))
        return out


def overlay(pairs, base: Layer, over: Layer, leaf_to_poly=None, offset: int = 0, op: str = "int",
            sched: str = "batched") -> Results:
    """Clips every (nodeid, queryid) pair: subject = base polygon
    leaf_to_poly[nodeid - offset], clip = overlay polygon queryid."""
    p = _dev_tensor(pairs, torch.int32)
    l2p = _dev_tensor(leaf_to_poly, torch.int32) if leaf_to_poly is not None else None
    h = C.c_void_p()
    sb, so = base.struct(), over.struct()
    check(lib().prt_overlay_run(_ptr(p), len(p), offset, _ptr(l2p), C.byref(sb), C.byref(so), OP[op], SCHED[sched],
                                _stream(), C.byref(h)))
    return Results(h)


_CHUNK_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                       C.POINTER(C.c_int32), C.POINTER(C.c_double))


def overlay_stream(pairs, base: Layer, over: Layer, fn, leaf_to_poly=None, offset: int = 0, op: str = "int",
                   sched: str = "batched", chunk_pairs: int = 1 << 18) -> None:
    """Clips the pairs in chunks of at most ``chunk_pairs`` (prt_overlay_stream):
    device memory holds at most two chunks' results.  For every chunk, in pair
    order, ``fn(first_pair, pair_cont_off, cont_nverts, cont_hole, xy)`` gets
    read-only numpy views of its results in host memory (pair_cont_off
    relative to the chunk, xy [V, 2]), valid only during the call: copy what
    must outlive it (a chunk is gigabytes at full size, and the library's
    buffers are reused for the next chunk).  A truthy return value stops the
    stream with an error."""
    p = _dev_tensor(pairs, torch.int32)
    l2p = _dev_tensor(leaf_to_poly, torch.int32) if leaf_to_poly is not None else None
    sb, so = base.struct(), over.struct()
    err = []

    def cb(user, first, n, off, nv, hole, xy):
        try:
            o = np.ctypeslib.as_array(off, shape=(n + 1,))
            nc = int(o[-1])
            nvv = np.ctypeslib.as_array(nv, shape=(max(nc, 1),))[:nc] if nc else np.zeros(0, np.int32)
            hh = np.ctypeslib.as_array(hole, shape=(max(nc, 1),))[:nc] if nc else np.zeros(0, np.int32)
            tv = int(nvv.sum(dtype=np.int64))
            xx = np.ctypeslib.as_array(xy, shape=(max(tv, 1), 2))[:tv] if tv else np.zeros((0, 2), np.float64)
            for a in (o, nvv, hh, xx):
                a.flags.writeable = False
            return 1 if fn(int(first), o, nvv, hh, xx) else 0
        except BaseException as e:  # surfaced after the C call returns
            err.append(e)
            return 1

    cfn = _CHUNK_FN(cb)
    rc = lib().prt_overlay_stream(_ptr(p), len(p), offset, _ptr(l2p), C.byref(sb), C.byref(so), OP[op], SCHED[sched],
                                  int(chunk_pairs), C.cast(cfn, C.c_void_p), None, _stream())
    if err:
        raise err[0]
    check(rc)


MAX_BINS = 8


class _Schedule(C.Structure):
    _fields_ = [("nbins", C.c_int32), ("aet_slots", C.c_int32), ("bin_thresholds", C.c_int64 * MAX_BINS),
                ("bin_warp_mode", C.c_int32 * MAX_BINS), ("warps_per_sm", C.c_int32), ("reserved", C.c_int32)]

    @classmethod
    def from_dict(cls, d: dict) -> "_Schedule":
        s = cls()
        thr = list(d["thresholds"])
        s.nbins = len(thr)
        s.aet_slots = int(d.get("aet_slots", 64))
        wm = list(d.get("warp_mode", [1] * len(thr)))
        s.warps_per_sm = int(d.get("warps_per_sm", 12))
        for b in range(len(thr)):
            s.bin_thresholds[b] = int(thr[b])
            s.bin_warp_mode[b] = int(wm[b])
        return s

    def to_dict(self) -> dict:
        n = self.nbins
        return {"thresholds": [int(self.bin_thresholds[b]) for b in range(n)],
                "warp_mode": [int(self.bin_warp_mode[b]) for b in range(n)],
                "warps_per_sm": int(self.warps_per_sm), "aet_slots": int(self.aet_slots)}


def get_schedule() -> dict:
    """The batched schedule in use (prt_schedule_get): size-bin thresholds
    (descending vertex-count upper bounds), per-bin warp mode (1 = one pair
    per warp), persistent warps per SM, and the warp clipper's shared-memory
    slots."""
    s = _Schedule()
    check(lib().prt_schedule_get(C.byref(s)))
    return s.to_dict()


def set_schedule(sched: dict | None) -> None:
    """Sets the batched schedule for later calls (None = built-in default)."""
    if sched is None:
        check(lib().prt_schedule_set(None))
    else:
        check(lib().prt_schedule_set(C.byref(_Schedule.from_dict(sched))))


class schedule:
    """Context manager: ``with prt.schedule(d): ...`` runs with schedule ``d``."""

    def __init__(self, sched: dict | None):
        self.sched = sched

    def __enter__(self):
        self.prev = get_schedule()
        set_schedule(self.sched)
        return self

    def __exit__(self, *exc):
        set_schedule(self.prev)
        return False


class _Tuning(C.Structure):
    _fields_ = [("fanout", C.c_int32), ("candidates", C.c_int32), ("sample_pairs", C.c_int64),
                ("build_join_ms", C.c_double), ("clip_ms", C.c_double), ("seconds", C.c_double),
                ("sched", _Schedule)]


def _tuning_cache_path(cache):
    import os

    if cache:
        return cache
    return os.environ.get("PRT_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "parlllelrtree_b200", "tuning.json"))


def autotune(base: Layer, over: Layer, op: str = "int", max_sample_pairs: int = 200_000,
             time_budget_s: float = 30.0, cache: str | None = None, use_cache: bool = True) -> dict:
    """Chooses the tree fanout and the batched schedule for these layers
    (prt_autotune: build + join timed per fanout, the batched clip timed per
    candidate schedule on a strided sample of the candidate pairs) and
    installs the schedule.  Results are cached in a JSON file keyed by the GPU
    name and the layers' sizes; a cached entry is installed without timing."""
    import json
    import os

    key = "|".join([torch.cuda.get_device_name(), op, str(base.n_poly), str(over.n_poly),
                    str(int(base.ring_vert[-1])), str(int(over.ring_vert[-1]))])
    path = _tuning_cache_path(cache)
    db = {}
    if use_cache and os.path.exists(path):
        with open(path) as f:
            db = json.load(f)
        if key in db:
            set_schedule(db[key]["schedule"])
            return dict(db[key], cached=True)
    t = _Tuning()
    sb, so = base.struct(), over.struct()
    check(lib().prt_autotune(C.byref(sb), C.byref(so), OP[op], int(max_sample_pairs), float(time_budget_s),
                             _stream(), C.byref(t)))
    res = {"fanout": int(t.fanout), "candidates": int(t.candidates), "sample_pairs": int(t.sample_pairs),
           "build_join_ms": float(t.build_join_ms), "clip_ms": float(t.clip_ms), "seconds": float(t.seconds),
           "schedule": t.sched.to_dict()}
    if use_cache:
        db[key] = res
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        with open(path, "w") as f:
            json.dump(db, f, indent=1)
    return dict(res, cached=False)


class _PipelineConfig(C.Structure):
    _fields_ = [("fanout", C.c_int32), ("op", C.c_int32), ("max_pairs", C.c_int64), ("max_frontier", C.c_int64),
                ("max_out_contours", C.c_int64), ("max_out_vertices", C.c_int64),
                ("arena_budget_bytes", C.c_int64), ("sched", C.c_void_p)]


class Pipeline:
    """The build -> join -> clip overlay captured as one CUDA graph
    (prt_pipeline_*): tree over ``base``'s polygon MBRs, join of ``over``'s,
    batched clip of every candidate pair.  ``run()`` replays the graph on the
    current stream (which must not be the legacy default stream)."""

    def __init__(self, base: Layer, over: Layer, fanout: int = 16, op: str = "int", max_pairs: int = 0,
                 max_frontier: int = 0, max_out_contours: int = 0, max_out_vertices: int = 0,
                 arena_budget_bytes: int = 0, sched: dict | None = None):
        self.base, self.over = base, over  # the graph reads their buffers
        cfg = _PipelineConfig()
        cfg.fanout, cfg.op = fanout, OP[op]
        cfg.max_pairs, cfg.max_frontier = max_pairs, max_frontier
        cfg.max_out_contours, cfg.max_out_vertices = max_out_contours, max_out_vertices
        cfg.arena_budget_bytes = arena_budget_bytes
        self._sched = _Schedule.from_dict(sched) if sched is not None else None
        cfg.sched = C.addressof(self._sched) if self._sched is not None else None
        self._sb, self._so = base.struct(), over.struct()
        self._h = C.c_void_p()
        check(lib().prt_pipeline_create(C.byref(self._sb), C.byref(self._so), C.byref(cfg), C.byref(self._h)))
        self._max_pairs = max_pairs if max_pairs > 0 else 8 * max(base.n_poly, over.n_poly)

    def __del__(self):
        try:
            if self._h:
                lib().prt_pipeline_free(self._h)
                self._h = None
        except Exception:
            pass

    def run(self) -> None:
        check(lib().prt_pipeline_run(self._h, _stream()))

    def sizes(self) -> dict:
        s = np.zeros(8, dtype=np.int64)
        check(lib().prt_pipeline_sizes(self._h, s.ctypes.data_as(C.c_void_p)))
        keys = ("pairs", "contours", "vertices", "nonempty", "failed", "max_frontier", "overflow", "timeout")
        return dict(zip(keys, (int(x) for x in s)))

    def pairs(self):
        """(pairs int32 [n, 2] {nodeid, queryid}, leaf_to_poly int32 [P]) of the last run, on the device."""
        n = min(self.sizes()["pairs"], self._max_pairs)
        pairs = torch.empty((max(n, 1), 2), dtype=torch.int32, device="cuda")
        l2p = torch.empty(self.base.n_poly, dtype=torch.int32, device="cuda")
        check(lib().prt_pipeline_pairs(self._h, _ptr(pairs), n, _ptr(l2p)))
        return pairs[:n], l2p

    def to_host(self):
        """(pair_cont_off, cont_nverts, cont_hole, xy) in pair order, as Results.to_host."""
        s = self.sizes()
        n = s["pairs"]
        off = np.zeros(n + 1, np.int64)
        nv = np.zeros(max(s["contours"], 1), np.int32)
        hole = np.zeros(max(s["contours"], 1), np.int32)
        xy = np.zeros((max(s["vertices"], 1), 2), np.float64)
        p = lambda a: a.ctypes.data_as(C.c_void_p)
        check(lib().prt_pipeline_results(self._h, p(off), p(nv), p(hole), p(xy)))
        return off, nv[: s["contours"]], hole[: s["contours"]], xy


def overlay_ref(pairs, num_base, prefix_base, vertex_base, hole_base, num_over, prefix_over, vertex_over, hole_over,
                leaf_to_poly=None, offset: int = 0, op: str = "int", sched: str = "plain") -> Results:
    """run() with the reference's single-contour CSR arguments
    (vector_map_overlay_gpc_kernel.cu:61)."""
    t = lambda x, d: _dev_tensor(x, d)
    p = t(pairs, torch.int32)
    nb, pb, vb, hb = t(num_base, torch.int32), t(prefix_base, torch.int64), t(vertex_base, torch.float64), t(hole_base, torch.int32)
    no, po, vo, ho = t(num_over, torch.int32), t(prefix_over, torch.int64), t(vertex_over, torch.float64), t(hole_over, torch.int32)
    l2p = t(leaf_to_poly, torch.int32) if leaf_to_poly is not None else None
    h = C.c_void_p()
    check(lib().prt_overlay_run_ref(_ptr(p), len(p), offset, _ptr(l2p), _ptr(nb), _ptr(pb), _ptr(vb), _ptr(hb), len(nb),
                                    _ptr(no), _ptr(po), _ptr(vo), _ptr(ho), len(no), OP[op], SCHED[sched], _stream(),
                                    C.byref(h)))
    return Results(h)


def clip_pair(subj, clip, op: str = "int"):
    """Clips one pair of host polygons (lists of [k, 2] rings) on the device.
    Returns a list of (hole, [k, 2] vertices) contours in GPC's order."""
    def rings(poly):
        nv = np.array([len(r) for r in poly], dtype=np.int32)
        xy = np.ascontiguousarray(np.concatenate([np.asarray(r, np.float64) for r in poly])) if len(poly) else np.zeros((0, 2))
        return len(poly), nv, xy
    sn, snv, sxy = rings(subj)
    cn, cnv, cxy = rings(clip)
    cap_c, cap_v = 64, 4096
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    while True:
        oc, ov = C.c_int32(0), C.c_int64(0)
        onv = np.zeros(cap_c, np.int32)
        oh = np.zeros(cap_c, np.int32)
        oxy = np.zeros((cap_v, 2), np.float64)
        rc = lib().prt_clip_pair_host(OP[op], sn, p(snv), p(sxy), cn, p(cnv), p(cxy), C.byref(oc), cap_c, p(onv),
                                      p(oh), C.byref(ov), cap_v, p(oxy))
        if rc == _lib.PRT_ERR_CAPACITY and (oc.value > cap_c or ov.value > cap_v):
            cap_c, cap_v = max(cap_c, oc.value), max(cap_v, ov.value)
            continue
        check(rc)
        out, o = [], 0
        for c in range(oc.value):
            out.append((int(oh[c]), oxy[o:o + onv[c]].copy()))
            o += onv[c]
        return out


class IntersectionArea(torch.autograd.Function):
    """area_i = area(base[pa_i] ∩ overlay[pb_i]); backward by the adjoint
    kernel, recomputing the clip boundary (nothing stored but the inputs)."""

    @staticmethod
    def forward(ctx, base_xy, over_xy, pa, pb, base: Layer, over: Layer):
        pa = pa.to(torch.int32).contiguous()
        pb = pb.to(torch.int32).contiguous()
        area = torch.empty(len(pa), dtype=torch.float64, device=base_xy.device)
        sb, so = base.struct(base_xy.detach().contiguous()), over.struct(over_xy.detach().contiguous())
        check(lib().prt_area_fwd(_ptr(pa), _ptr(pb), len(pa), C.byref(sb), C.byref(so), _ptr(area), _stream()))
        ctx.save_for_backward(base_xy, over_xy, pa, pb)
        ctx.layers = (base, over)
        return area

    @staticmethod
    def backward(ctx, g):
        base_xy, over_xy, pa, pb = ctx.saved_tensors
        base, over = ctx.layers
        g = g.contiguous().to(torch.float64)
        gb = torch.zeros_like(base_xy, dtype=torch.float64)
        go = torch.zeros_like(over_xy, dtype=torch.float64)
        sb, so = base.struct(base_xy.detach().contiguous()), over.struct(over_xy.detach().contiguous())
        check(lib().prt_area_bwd(_ptr(pa), _ptr(pb), len(pa), C.byref(sb), C.byref(so), _ptr(g), _ptr(gb), _ptr(go),
                                 _stream()))
        return gb, go, None, None, None, None


def intersection_area(base: Layer, over: Layer, pa, pb, base_xy=None, over_xy=None) -> torch.Tensor:
    bx = base.xy if base_xy is None else base_xy
    ox = over.xy if over_xy is None else over_xy
    return IntersectionArea.apply(bx, ox, _dev_tensor(pa, torch.int32), _dev_tensor(pb, torch.int32), base, over)
