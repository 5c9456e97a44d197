"""ORACLE — test infrastructure only.

ctypes bindings for the CPU restatement (``liboracle.so``) and for the
reference's own CPU code built into ``oracle/_ref`` (``ref/build_ref.sh``).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline
import this package, and only as the checker; the library in
``parlllelrtree_b200`` never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_LIB = None
_REF = {}

COORD = {"i64": 0, "f32": 1, "f64": 2, "i32": 3}
_DT = {0: np.int64, 1: np.float32, 2: np.float64, 3: np.int32}


def build(force: bool = False) -> None:
    """Builds liboracle.so (and oracle/_ref when the reference is present)."""
    subprocess.run(["make", "-s", "-C", HERE] + (["-B"] if force else []), check=True)


def build_ref() -> bool:
    """Builds oracle/_ref from the reference sources; False if they are absent."""
    if not os.path.isdir(os.environ.get("PRT_REFERENCE_DIR", "/root/reference")):
        return False
    subprocess.run(["bash", os.path.join(HERE, "ref", "build_ref.sh")], check=True,
                   stdout=subprocess.DEVNULL)
    return True


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        _LIB = C.CDLL(path)
        _LIB.orc_keys_ref64.restype = C.c_int64
        _LIB.orc_interleave4.restype = C.c_uint64
        _LIB.orc_interleave4.argtypes = [C.c_uint64] * 4
        _LIB.orc_pack.restype = C.c_int64
        _LIB.orc_join_pairs.restype = C.c_int64
        _LIB.orc_sibling_overlaps.restype = C.c_int64
        _LIB.orc_level_count.restype = C.c_int64
        _LIB.orc_level_count.argtypes = [C.c_int64, C.c_int, C.c_int]
        _LIB.orc_num_levels.argtypes = [C.c_int64, C.c_int]
        _LIB.orc_result_area.restype = C.c_double
        _LIB.orc_area_grad.restype = C.c_double
    return _LIB


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_gpc.so"))


def ref_lib(name: str) -> C.CDLL:
    if name not in _REF:
        _REF[name] = C.CDLL(os.path.join(REF_DIR, name))
    return _REF[name]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _coord(boxes: np.ndarray):
    for k, dt in _DT.items():
        if boxes.dtype == dt:
            return k
    raise TypeError(f"unsupported coordinate dtype {boxes.dtype}")


# ---------------------------------------------------------------- keys / sort

def keys_ref64(rects: np.ndarray):
    rects = np.ascontiguousarray(rects, dtype=np.int64)
    n = len(rects)
    keys = np.empty(n, dtype=np.uint64)
    shift = np.zeros(2, dtype=np.int64)
    scale = lib().orc_keys_ref64(_p(rects), C.c_int64(n), _p(keys), _p(shift))
    return keys, int(scale), shift


def keys_morton32(boxes: np.ndarray):
    boxes = np.ascontiguousarray(boxes)
    n = len(boxes)
    keys = np.empty(n, dtype=np.uint32)
    ext = np.zeros(3, dtype=np.float64)
    lib().orc_keys_morton32(_p(boxes), C.c_int(_coord(boxes)), C.c_int64(n), _p(keys), _p(ext))
    return keys, ext


def interleave4(a, b, c, d) -> int:
    return int(lib().orc_interleave4(a, b, c, d))


def stable_argsort(keys: np.ndarray) -> np.ndarray:
    k = np.ascontiguousarray(keys, dtype=np.uint64)
    perm = np.empty(len(k), dtype=np.int64)
    lib().orc_stable_argsort_u64(_p(k), C.c_int64(len(k)), _p(perm))
    return perm


def td_order(boxes: np.ndarray, fanout: int) -> np.ndarray:
    boxes = np.ascontiguousarray(boxes)
    perm = np.empty(len(boxes), dtype=np.int64)
    lib().orc_td_order(_p(boxes), C.c_int(_coord(boxes)), C.c_int64(len(boxes)), C.c_int(fanout), _p(perm))
    return perm


def level_counts(n: int, fanout: int):
    L = lib().orc_num_levels(C.c_int64(n), C.c_int(fanout))
    return [int(lib().orc_level_count(C.c_int64(n), C.c_int(fanout), C.c_int(l))) for l in range(L)]


def pack(boxes: np.ndarray, fanout: int, perm: np.ndarray):
    """Returns the list of level MBR arrays (float64 [n_l, 4]), level 0 first."""
    boxes = np.ascontiguousarray(boxes)
    perm = np.ascontiguousarray(perm, dtype=np.int64)
    counts = level_counts(len(boxes), fanout)
    flat = np.empty((sum(counts), 4), dtype=np.float64)
    lib().orc_pack(_p(boxes), C.c_int(_coord(boxes)), C.c_int64(len(boxes)), C.c_int(fanout), _p(perm), _p(flat))
    out, o = [], 0
    for c in counts:
        out.append(flat[o:o + c])
        o += c
    return out


def build_bottomup(boxes: np.ndarray, fanout: int, key_mode: str = "morton32"):
    if key_mode == "ref64":
        keys, _, _ = keys_ref64(boxes)
    else:
        keys, _ = keys_morton32(boxes)
    perm = stable_argsort(keys.astype(np.uint64))
    return perm, pack(boxes, fanout, perm)


def build_topdown(boxes: np.ndarray, fanout: int):
    perm = td_order(boxes, fanout)
    return perm, pack(boxes, fanout, perm)


def query_counts(levels, fanout: int, queries: np.ndarray, td_slots: bool = False) -> np.ndarray:
    flat = np.ascontiguousarray(np.concatenate(levels, axis=0))
    q = np.ascontiguousarray(queries)
    out = np.empty((len(q), 3), dtype=np.int64)
    lib().orc_query_counts(_p(flat), C.c_int64(len(levels[0])), C.c_int(fanout), _p(q), C.c_int(_coord(q)),
                           C.c_int64(len(q)), C.c_int(1 if td_slots else 0), _p(out))
    return out


def join_pairs(levels, fanout: int, queries: np.ndarray, cap: int | None = None) -> np.ndarray:
    """(leaf position, query id) pairs, int64 [P, 2]."""
    flat = np.ascontiguousarray(np.concatenate(levels, axis=0))
    q = np.ascontiguousarray(queries)
    L = lib()
    if cap is None:
        cap = 1 << 16
    while True:
        pairs = np.empty((cap, 2), dtype=np.int64)
        n = L.orc_join_pairs(_p(flat), C.c_int64(len(levels[0])), C.c_int(fanout), _p(q), C.c_int(_coord(q)),
                             C.c_int64(len(q)), _p(pairs), C.c_int64(cap))
        if n <= cap:
            return pairs[:n]
        cap = int(n)


def sibling_overlaps(levels, fanout: int) -> int:
    flat = np.ascontiguousarray(np.concatenate(levels, axis=0))
    return int(lib().orc_sibling_overlaps(_p(flat), C.c_int64(len(levels[0])), C.c_int(fanout)))


def digests(levels, fanout: int, queries: np.ndarray, td_slots: bool = False):
    """The reference's printed digests: sum (entries examined), sum1, sum2
    (leaf hits / 2), sum3 (sibling overlaps)."""
    c = query_counts(levels, fanout, queries, td_slots)
    return (int(c[:, 0].sum()), int(c[:, 1].sum()), int(c[:, 2].sum()) // 2, sibling_overlaps(levels, fanout))


# ---------------------------------------------------------------- GPC clip

def _rings(poly):
    """poly: list of [k, 2] rings -> (ncont, nverts int32, xy float64)."""
    nverts = np.array([len(r) for r in poly], dtype=np.int32)
    xy = np.ascontiguousarray(np.concatenate([np.asarray(r, dtype=np.float64) for r in poly])
                              if len(poly) else np.zeros((0, 2)))
    return len(poly), nverts, xy


def _unpack_result(ncont, nverts, hole, xy):
    out, o = [], 0
    for c in range(ncont):
        k = int(nverts[c])
        out.append((int(hole[c]), xy[o:o + k].copy()))
        o += k
    return out


def gpc_clip(subj, clip, op: int = 1, stats: bool = False):
    """Oracle clip of two polygons given as lists of rings.  Returns a list of
    (hole, [k, 2] vertices) contours in GPC's output order."""
    sn, snv, sxy = _rings(subj)
    cn, cnv, cxy = _rings(clip)
    L = lib()
    cap_c, cap_v = 64, 4096
    st = np.zeros(8, dtype=np.int32)
    while True:
        oc = C.c_int(0)
        ov = C.c_int64(0)
        onv = np.zeros(cap_c, dtype=np.int32)
        oh = np.zeros(cap_c, dtype=np.int32)
        oxy = np.zeros((cap_v, 2), dtype=np.float64)
        rc = L.orc_gpc_clip(C.c_int(op), C.c_int(sn), _p(snv), _p(sxy), C.c_int(cn), _p(cnv), _p(cxy),
                            C.byref(oc), C.c_int(cap_c), _p(onv), _p(oh), C.byref(ov), C.c_int64(cap_v), _p(oxy),
                            _p(st))
        if rc == 0:
            res = _unpack_result(oc.value, onv, oh, oxy)
            return (res, st[:6].copy()) if stats else res
        cap_c = max(cap_c, oc.value)
        cap_v = max(cap_v, int(ov.value))


def ref_gpc_clip(subj, clip, op: int = 1):
    """The reference's own clip core (oracle/_ref/libref_gpc.so)."""
    sn, snv, sxy = _rings(subj)
    cn, cnv, cxy = _rings(clip)
    L = ref_lib("libref_gpc.so")
    cap_c, cap_v = 64, 4096
    sh = np.zeros(max(sn, 1), dtype=np.int32)
    ch = np.zeros(max(cn, 1), dtype=np.int32)
    while True:
        oc = C.c_int(0)
        ov = C.c_int64(0)
        onv = np.zeros(cap_c, dtype=np.int32)
        oh = np.zeros(cap_c, dtype=np.int32)
        oxy = np.zeros((cap_v, 2), dtype=np.float64)
        rc = L.ref_gpc_clip(C.c_int(op), C.c_int(sn), _p(snv), _p(sh), _p(sxy), C.c_int(cn), _p(cnv), _p(ch),
                            _p(cxy), C.byref(oc), C.c_int(cap_c), _p(onv), _p(oh), C.byref(ov), C.c_int64(cap_v),
                            _p(oxy))
        if rc == 0:
            return _unpack_result(oc.value, onv, oh, oxy)
        cap_c = max(cap_c, oc.value)
        cap_v = max(cap_v, int(ov.value))


def result_area(contours) -> float:
    """Sum of |shoelace| over contours (holes negative), by the C oracle
    (coordinates relative to each contour's first vertex)."""
    if not contours:
        return 0.0
    nv = np.array([len(v) for _, v in contours], dtype=np.int32)
    hole = np.array([h for h, _ in contours], dtype=np.int32)
    xy = np.ascontiguousarray(np.concatenate([v for _, v in contours]), dtype=np.float64)
    return float(lib().orc_result_area(C.c_int(len(contours)), _p(nv), _p(hole), _p(xy)))


def area_grad(subj, clip, subj_hole=None, clip_hole=None):
    """(area, grad_subj [V_s, 2], grad_clip [V_c, 2]) of area(subj ∩ clip)."""
    sn, snv, sxy = _rings(subj)
    cn, cnv, cxy = _rings(clip)
    sh = np.ascontiguousarray(subj_hole if subj_hole is not None else np.zeros(sn), dtype=np.int32)
    ch = np.ascontiguousarray(clip_hole if clip_hole is not None else np.zeros(cn), dtype=np.int32)
    gs = np.zeros_like(sxy)
    gc = np.zeros_like(cxy)
    a = lib().orc_area_grad(C.c_int(sn), _p(snv), _p(sh), _p(sxy), C.c_int(cn), _p(cnv), _p(ch), _p(cxy),
                            _p(gs), _p(gc))
    return float(a), gs, gc


# ---------------------------------------------------------------- reference CPU paths

def ref_bu_run(rects: np.ndarray, fanout: int, ids=None, query: bool = True):
    """The reference's bottom-up CPU path at fanout m (10, 16 or 32)."""
    L = ref_lib(f"libref_bu_m{fanout}.so")
    L.ref_bu_run.restype = C.c_longlong
    rects = np.ascontiguousarray(rects, dtype=np.int64)
    n = len(rects)
    ids = np.ascontiguousarray(np.arange(n, dtype=np.int32) if ids is None else ids, dtype=np.int32)
    cap = n + 64
    keys = np.empty(n, dtype=np.uint64)
    scale = C.c_longlong(0)
    flag = np.zeros(cap, dtype=np.int32)
    num = np.zeros(cap, dtype=np.int32)
    mbr = np.zeros((cap, fanout, 4), dtype=np.int64)
    children = np.zeros((cap, fanout), dtype=np.int32)
    data = np.zeros((cap, fanout), dtype=np.int32)
    root = C.c_int(0)
    sorted_ids = np.zeros(n, dtype=np.int32)
    dig = np.zeros(4, dtype=np.int64)
    ms = np.zeros(2, dtype=np.float64)
    nn = L.ref_bu_run(_p(rects), _p(ids), C.c_int(n), _p(keys), C.byref(scale), C.c_int(cap), _p(flag), _p(num),
                      _p(mbr), _p(children), _p(data), C.byref(root), _p(sorted_ids), _p(dig), _p(ms),
                      C.c_int(1 if query else 0))
    if nn < 0:
        raise RuntimeError("ref_bu_run: node capacity")
    return {
        "keys": keys, "scale": int(scale.value), "n_nodes": int(nn), "root": int(root.value),
        "flag": flag[:nn], "num": num[:nn], "mbr": mbr[:nn], "children": children[:nn], "data": data[:nn],
        "sorted_ids": sorted_ids, "digests": tuple(int(x) for x in dig), "ms": ms.copy(),
    }


def ref_td_run(rects: np.ndarray, fanout: int, query: bool = True):
    """The reference's top-down CPU path at fanout M (10, 16 or 32)."""
    L = ref_lib(f"libref_td_m{fanout}.so")
    L.ref_td_run.restype = C.c_longlong
    rects = np.ascontiguousarray(rects, dtype=np.int64)
    n = len(rects)
    cap = 2 * n + 64 * fanout
    idx = np.zeros(cap, dtype=np.int32)
    mbr = np.zeros((cap, 4), dtype=np.int64)
    offs = np.zeros(64, dtype=np.int32)
    noffs = C.c_int(0)
    srt = np.zeros((n, 4), dtype=np.int64)
    dig = np.zeros(4, dtype=np.int64)
    ms = np.zeros(2, dtype=np.float64)
    ns = L.ref_td_run(_p(rects), C.c_int(n), C.c_longlong(cap), _p(idx), _p(mbr), _p(offs), C.byref(noffs),
                      _p(srt), _p(dig), _p(ms), C.c_int(1 if query else 0))
    if ns < 0:
        raise RuntimeError("ref_td_run: slot capacity")
    return {
        "nodes_index": idx[:ns], "nodes_mbr": mbr[:ns], "offsets": offs[:noffs.value].copy(),
        "sorted_rects": srt, "digests": tuple(int(x) for x in dig), "ms": ms.copy(),
    }


def ref_interleave(a, b, c, d) -> int:
    L = ref_lib("libref_bu_m10.so")
    L.ref_bu_interleave.restype = C.c_ulonglong
    L.ref_bu_interleave.argtypes = [C.c_ulonglong] * 4
    return int(L.ref_bu_interleave(a, b, c, d))


def ref_overlap(a, b, which: str = "bu") -> int:
    a = np.ascontiguousarray(a, dtype=np.int64)
    b = np.ascontiguousarray(b, dtype=np.int64)
    if which == "bu":
        return int(ref_lib("libref_bu_m10.so").ref_bu_overlap(_p(a), _p(b)))
    return int(ref_lib("libref_td_m10.so").ref_td_overlap(_p(a), _p(b)))


def ref_read_data(base: str, overlay: str, min_xy=(2**31 - 1, 2**31 - 1)) -> dict:
    """The reference's own readData (vector_map_overlay_gpc_kernel.cu:752-888,
    host build in oracle/_ref/libref_readdata.so) on two polygon files:
    {"base": {...}, "overlay": {...}, "min_xy": (minX, minY)} with num, prefix,
    hole, rect (P x 4, its quantised boxes) and vertex (V x 2) per layer."""
    L = ref_lib("libref_readdata.so")
    counts = np.zeros(4, np.int64)
    mxy = np.array(min_xy, np.int32)
    cap_p = cap_v = 0
    while True:
        bufs = [{"num": np.zeros(max(cap_p, 1), np.int32), "prefix": np.zeros(max(cap_p, 1), np.int64),
                 "hole": np.zeros(max(cap_p, 1), np.int32), "rect": np.zeros((max(cap_p, 1), 4), np.int32),
                 "vertex": np.zeros((max(cap_v, 1), 2), np.float64)} for _ in range(2)]
        m = mxy.copy()
        args = [base.encode(), overlay.encode(), _p(counts)]
        for b in bufs:
            args += [_p(b["num"]), _p(b["prefix"]), _p(b["hole"]), _p(b["rect"]), _p(b["vertex"])]
        args += [C.c_int64(cap_p), C.c_int64(cap_v), _p(m)]
        rc = L.ref_read_data(*args)
        if rc == 0:
            break
        cap_p, cap_v = int(max(counts[0], counts[1])), int(max(counts[2], counts[3]))
    out = {}
    for k, (name, b) in enumerate(zip(("base", "overlay"), bufs)):
        P, V = int(counts[k]), int(counts[2 + k])
        out[name] = {"num": b["num"][:P], "prefix": b["prefix"][:P], "hole": b["hole"][:P], "rect": b["rect"][:P],
                     "vertex": b["vertex"][:V]}
    out["min_xy"] = (int(m[0]), int(m[1]))
    return out


def write_rect_file(path: str, rects: np.ndarray, keys=None) -> None:
    """Writes boxes in the format TopDown-rtree.cu / BotomUp-rtree.cu read
    (N, then per box "x1 x2", "y1 y2", "key"; BU:671-698, TD:487-497)."""
    rects = np.asarray(rects, dtype=np.int64)
    n = len(rects)
    keys = np.arange(n) if keys is None else keys
    with open(path, "w") as f:
        f.write(f"{n}\n")
        for i in range(n):
            x1, y1, x2, y2 = (int(v) for v in rects[i])
            f.write(f"{x1} {x2}\n{y1} {y2}\n{int(keys[i])}\n")


def run_td_program(rects: np.ndarray, workdir: str, timeout: float = 600.0) -> dict:
    """Runs the unchanged TopDown-rtree.cu program (oracle/_ref/td_ref) on
    ``rects`` with no GPU visible, so only its CPU build and CPU query run, and
    parses its printed digests and timings."""
    os.makedirs(os.path.join(workdir, "data"), exist_ok=True)
    write_rect_file(os.path.join(workdir, "data", "Rect1024.txt"), rects)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([os.path.join(REF_DIR, "td_ref")], cwd=workdir, env=env, capture_output=True,
                         text=True, timeout=timeout).stdout
    res = {"stdout": out}
    for line in out.splitlines():
        line = line.strip()
        if line.startswith("CPU Construction:"):
            res["cpu_build_ms"] = float(line.split(":")[1].replace("ms", ""))
        elif line.startswith("qeury run:"):
            res["cpu_query_ms"] = float(line.split(":")[1].replace("ms", ""))
        elif line.startswith("sum ="):
            res["sum"] = int(line.split("=")[1].split()[0])
        elif line.startswith("sum1 ="):
            res["sum1"] = int(line.split("=")[1].split()[0])
        elif line.startswith("sum2 ="):
            res["sum2"] = int(line.split("=")[1].split()[0])
        elif line.startswith("sum3 ="):
            res["sum3"] = int(line.split("=")[1].split()[0])
    return res
