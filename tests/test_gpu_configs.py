"""Parity at the stated configurations' own sizes (not scaled-down shapes).

* Small overlay: 2 x 10,000 star polygons (8-32 vertices, radius log-uniform
  1e-3..1e-2, centres uniform, seed 0 / 1), fanout-16 bottom-up Morton tree
  over layer A's MBRs, join of layer B's MBRs, GPC intersection of every
  candidate pair with the plain and the batched schedule: candidate set equal
  to the brute-force box intersection set, every contour bit-exact against
  the oracle, areas within 1e-9 relative.
* Build and query: 10M float32 mixture boxes, bottom-up (Morton) and top-down
  builds at fanout 16 and 32: leaf order and every level bit-exact against the
  oracle; 1M window queries against the fanout-16 tree: every query's counters
  and the total pair count equal to the oracle's DFS, and the pairs of a
  strided sample of 2,000 windows equal to the oracle's.
"""
import numpy as np
import pytest
import torch

import oracle
from helpers import rings_of, same_contours
from parlllelrtree_b200 import datagen as dg

pytestmark = pytest.mark.gpu


def _brute_candidates(ba, bb):
    out = set()
    for j in range(len(bb)):
        m = (ba[:, 0] <= bb[j, 2]) & (bb[j, 0] <= ba[:, 2]) & (ba[:, 1] <= bb[j, 3]) & (bb[j, 1] <= ba[:, 3])
        out.update((int(i), j) for i in np.nonzero(m)[0])
    return out


@pytest.fixture(scope="module")
def small_overlay(cuda):
    import parlllelrtree_b200 as prt

    A = dg.star_layer(10000, seed=0)
    B = dg.star_layer(10000, seed=1)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    t = prt.build_bottomup(LA.mbr(), fanout=16, key_mode="morton32")
    pairs = t.join(LB.mbr(), sorted=True)
    l2p = t.leaf_order()
    return A, B, LA, LB, pairs, l2p


def test_small_overlay_candidates(small_overlay):
    A, B, LA, LB, pairs, l2p = small_overlay
    p, perm = pairs.cpu().numpy(), l2p.cpu().numpy()
    assert len(p) > 15000  # ~20.9k candidate pairs at this configuration
    got = {(int(perm[a]), int(b)) for a, b in p}
    assert len(got) == len(p)
    assert got == _brute_candidates(dg.layer_bboxes(A), dg.layer_bboxes(B))
    # the device MBRs are the layers' exact bounding boxes
    assert np.array_equal(LA.mbr().cpu().numpy(), dg.layer_bboxes(A))


@pytest.mark.parametrize("sched", ["plain", "batched"])
def test_small_overlay_clip_exact(small_overlay, sched):
    import parlllelrtree_b200 as prt

    A, B, LA, LB, pairs, l2p = small_overlay
    res = prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched=sched)
    got = res.contours()
    p, perm = pairs.cpu().numpy(), l2p.cpu().numpy()
    nonempty = 0
    for k, (leaf, q) in enumerate(p):
        ref = oracle.gpc_clip(rings_of(A, perm[leaf]), rings_of(B, q), 1)
        assert same_contours(got[k], ref), k
        nonempty += len(ref) > 0
    assert res.nonempty == nonempty


def test_small_overlay_areas(small_overlay):
    import parlllelrtree_b200 as prt

    A, B, LA, LB, pairs, l2p = small_overlay
    p, perm = pairs.cpu().numpy(), l2p.cpu().numpy()
    pa = torch.from_numpy(perm[p[:, 0]].astype(np.int32)).cuda()
    pb = pairs[:, 1].contiguous()
    area = prt.intersection_area(LA, LB, pa, pb).cpu().numpy()
    for k, (leaf, q) in enumerate(p):
        ref = oracle.result_area(oracle.gpc_clip(rings_of(A, perm[leaf]), rings_of(B, q), 1))
        assert abs(area[k] - ref) <= 1e-9 * abs(ref) + 1e-22, k


@pytest.fixture(scope="module")
def boxes_10m(cuda):
    b = dg.mixture_boxes(10_000_000, seed=0)
    return b, torch.from_numpy(b).cuda()


@pytest.mark.parametrize("F", [16, 32])
def test_build_10m_bottomup(boxes_10m, F):
    import parlllelrtree_b200 as prt

    b, bd = boxes_10m
    keys, _ = oracle.keys_morton32(b)
    perm = oracle.stable_argsort(keys)
    t = prt.build_bottomup(bd, fanout=F, key_mode="morton32")
    assert np.array_equal(t.leaf_order().cpu().numpy(), perm)
    lv = oracle.pack(b, F, perm)
    assert t.levels == len(lv)
    for l in range(t.levels):
        assert np.array_equal(t.level_mbr(l), lv[l]), l
    assert t.sibling_overlaps() == oracle.sibling_overlaps(lv, F)


@pytest.mark.parametrize("F", [16, 32])
def test_build_10m_topdown(boxes_10m, F):
    import parlllelrtree_b200 as prt

    b, bd = boxes_10m
    perm = oracle.td_order(b, F)
    t = prt.build_topdown(bd, fanout=F)
    assert np.array_equal(t.leaf_order().cpu().numpy(), perm)
    lv = oracle.pack(b, F, perm)
    for l in range(t.levels):
        assert np.array_equal(t.level_mbr(l), lv[l]), l


def test_join_10m_1m_windows(boxes_10m):
    import parlllelrtree_b200 as prt

    b, bd = boxes_10m
    t = prt.build_bottomup(bd, fanout=16)
    w = dg.window_queries(1_000_000, seed=1)
    wd = torch.from_numpy(w).cuda()
    lv = t.levels_mbr()
    ref = oracle.query_counts(lv, 16, w)
    got = t.query_counts(wd).cpu().numpy()
    assert np.array_equal(got, ref)
    pairs = t.join(wd)
    assert len(pairs) == int(ref[:, 2].sum())
    # a strided sample of windows: their pairs exactly
    sample = np.arange(0, len(w), 500)
    got_s = pairs[pairs[:, 1] % 500 == 0].cpu().numpy().astype(np.int64)
    got_s = got_s[np.lexsort((got_s[:, 0], got_s[:, 1]))]
    exp = oracle.join_pairs(lv, 16, w[sample])
    exp[:, 1] = sample[exp[:, 1]]
    exp = exp[np.lexsort((exp[:, 0], exp[:, 1]))]
    assert np.array_equal(got_s, exp)
