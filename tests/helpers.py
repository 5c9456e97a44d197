"""Test helpers: conversions from the level representation (level 0 = records
in leaf order, entry j of level l+1 = union of node j of level l) to the
reference's two tree layouts, and small utilities."""
from __future__ import annotations

import numpy as np


def levels_to_bu(levels, fanout: int, leaf_ids):
    """Reference bottom-up node array (BotomUp-rtree.cu:47-54, 788-830):
    node levels bottom-up, children of node j of level l+1 = nodes jF.. of l."""
    F = fanout
    counts = [len(l) for l in levels]
    nodes = [(c + F - 1) // F for c in counts]
    first = np.concatenate([[0], np.cumsum(nodes)])
    n = int(first[-1])
    flag = np.zeros(n, np.int32)
    num = np.zeros(n, np.int32)
    mbr = np.zeros((n, F, 4), np.float64)
    ch = np.full((n, F), -1, np.int32)
    data = np.full((n, F), -1, np.int32)
    for l, lv in enumerate(levels):
        for j in range(nodes[l]):
            k = first[l] + j
            a, e = j * F, min(j * F + F, counts[l])
            flag[k] = 0 if l == 0 else 1
            num[k] = e - a
            mbr[k, : e - a] = lv[a:e]
            if l == 0:
                data[k, : e - a] = leaf_ids[a:e]
            else:
                ch[k, : e - a] = first[l - 1] + np.arange(a, e)
    return {"flag": flag, "num": num, "mbr": mbr, "children": ch, "data": data, "root": n - 1}


def levels_to_td(levels, fanout: int):
    """Reference top-down slot arrays (TopDown-rtree.cu:504-624): levels
    top-down, nodes_index > 0 child's first slot, < 0 -(leaf position)-1."""
    F = fanout
    L = len(levels)
    padded = [((len(lv) + F - 1) // F) * F for lv in levels]
    off = [0]
    for p in range(L):
        off.append(off[-1] + padded[L - 1 - p])
    idx = np.zeros(off[-1], np.int32)
    mbr = np.zeros((off[-1], 4), np.float64)
    for p in range(L):
        l = L - 1 - p
        c = len(levels[l])
        s = off[p]
        mbr[s:s + c] = levels[l]
        if l == 0:
            idx[s:s + c] = -np.arange(c) - 1
        else:
            idx[s:s + c] = off[p + 1] + np.arange(c) * F
    return {"nodes_index": idx, "nodes_mbr": mbr, "offsets": np.array(off, np.int32)}


def compare_bu(a: dict, b: dict) -> None:
    """Exact comparison of two BU layouts (only live entries)."""
    assert np.array_equal(a["flag"], b["flag"])
    assert np.array_equal(a["num"], b["num"])
    assert a["root"] == b["root"]
    for k in range(len(a["num"])):
        m = a["num"][k]
        assert np.array_equal(a["mbr"][k, :m], b["mbr"][k, :m]), f"node {k} mbr"
        if a["flag"][k] == 0:
            assert np.array_equal(a["data"][k, :m], b["data"][k, :m]), f"node {k} data"
        else:
            assert np.array_equal(a["children"][k, :m], b["children"][k, :m]), f"node {k} children"


def compare_td(a: dict, b: dict) -> None:
    assert np.array_equal(a["offsets"], b["offsets"])
    assert np.array_equal(a["nodes_index"], b["nodes_index"])
    live = a["nodes_index"] != 0
    assert np.array_equal(a["nodes_mbr"][live], b["nodes_mbr"][live])


def rings_of(layer, p):
    pr, rv, xy = layer["poly_ring"], layer["ring_vert"], layer["xy"]
    return [xy[rv[r]:rv[r + 1]] for r in range(pr[p], pr[p + 1])]


def same_contours(a, b) -> bool:
    return len(a) == len(b) and all(h1 == h2 and np.array_equal(v1, v2) for (h1, v1), (h2, v2) in zip(a, b))


def brute_pairs(boxes: np.ndarray, queries: np.ndarray) -> set:
    """All (record, query) index pairs with intersecting closed boxes."""
    b = np.asarray(boxes, dtype=np.float64)
    q = np.asarray(queries, dtype=np.float64)
    out = set()
    for j in range(len(q)):
        m = (b[:, 0] <= q[j, 2]) & (q[j, 0] <= b[:, 2]) & (b[:, 1] <= q[j, 3]) & (q[j, 1] <= b[:, 3])
        out.update((int(i), j) for i in np.nonzero(m)[0])
    return out
