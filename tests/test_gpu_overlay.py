"""GPC clipping on the GPU: contours, hole flags and vertex order bit-exact
against the oracle and the reference's golden fixtures."""
import os

import numpy as np
import pytest
import torch

import oracle
from conftest import GOLDEN
from helpers import rings_of, same_contours
from parlllelrtree_b200 import datagen as dg

pytestmark = pytest.mark.gpu

OPS = ["diff", "int", "xor", "union"]


def golden():
    g = np.load(os.path.join(GOLDEN, "gpc.npz"))
    A = {k[2:]: g[k] for k in g.files if k.startswith("a_")}
    B = {k[2:]: g[k] for k in g.files if k.startswith("b_")}
    return g, A, B


@pytest.mark.parametrize("sched", ["plain", "batched"])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_golden_pairs(cuda, sched, op):
    import parlllelrtree_b200 as prt

    g, A, B = golden()
    pairs = g["pairs"].astype(np.int32)
    res = prt.overlay(torch.from_numpy(pairs).cuda(), prt.Layer.from_dict(A), prt.Layer.from_dict(B),
                      op=OPS[op], sched=sched)
    got = res.contours()
    nc, nv, hole, xy = g[f"op{op}_ncont"], g[f"op{op}_nverts"], g[f"op{op}_hole"], g[f"op{op}_xy"]
    c = v = 0
    for k in range(len(pairs)):
        ref = []
        for _ in range(nc[k]):
            ref.append((int(hole[c]), xy[v:v + nv[c]]))
            v += nv[c]
            c += 1
        assert same_contours(got[k], ref), f"pair {k}"


def small_config(n=2500, seed=0):
    """The small plain config's shape: stars of 8-32 vertices, radius
    log-uniform 1e-3..1e-2; denser (fewer polygons per unit area) to keep the
    oracle fast."""
    A = dg.star_layer(n, seed=seed, r_lo=5e-3, r_hi=3e-2)
    B = dg.star_layer(n, seed=seed + 1, r_lo=5e-3, r_hi=3e-2)
    return A, B


@pytest.mark.parametrize("sched", ["plain", "batched"])
def test_join_then_clip_pipeline(cuda, sched):
    """Tree over layer A's MBRs -> join layer B -> clip every candidate pair,
    remapped through the leaf order like Execute (GPC:89-90)."""
    import parlllelrtree_b200 as prt

    A, B = small_config()
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    t = prt.build_bottomup(LA.mbr(), fanout=16)
    pairs = t.join(LB.mbr(), sorted=True)
    l2p = t.leaf_order()
    res = prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched=sched)
    got = res.contours()
    p = pairs.cpu().numpy()
    perm = l2p.cpu().numpy()
    # candidate set == brute-force MBR intersections
    ba, bb = dg.layer_bboxes(A), dg.layer_bboxes(B)
    exp = set()
    for j in range(len(bb)):
        m = (ba[:, 0] <= bb[j, 2]) & (bb[j, 0] <= ba[:, 2]) & (ba[:, 1] <= bb[j, 3]) & (bb[j, 1] <= ba[:, 3])
        exp.update((int(i), j) for i in np.nonzero(m)[0])
    assert {(int(perm[a]), int(b)) for a, b in p} == exp
    for k, (leaf, q) in enumerate(p):
        ref = oracle.gpc_clip(rings_of(A, perm[leaf]), rings_of(B, q), 1)
        assert same_contours(got[k], ref), k
    assert res.nonempty > 0


def test_plain_equals_batched_with_holes(cuda):
    import parlllelrtree_b200 as prt

    A = dg.star_layer(300, seed=5, nv_lo=4, nv_hi=200, r_lo=0.02, r_hi=0.1, hole_frac=0.3, zipf=1.2)
    B = dg.star_layer(300, seed=6, nv_lo=4, nv_hi=200, r_lo=0.02, r_hi=0.1, hole_frac=0.3, zipf=1.2)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    t = prt.build_bottomup(LA.mbr(), fanout=16)
    pairs = t.join(LB.mbr(), sorted=True)
    l2p = t.leaf_order()
    r1 = prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched="plain").contours()
    r2 = prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched="batched").contours()
    p = pairs.cpu().numpy()
    perm = l2p.cpu().numpy()
    for k, (leaf, q) in enumerate(p):
        ref = oracle.gpc_clip(rings_of(A, perm[leaf]), rings_of(B, q), 1)
        assert same_contours(r1[k], ref), k
        assert same_contours(r2[k], ref), k


def comb(k, x0, y0, w, h, vertical=False):
    """A comb polygon with k teeth (4k vertices)."""
    pts = []
    for i in range(k):
        pts += [(x0 + (2 * i) * w, y0), (x0 + (2 * i + 1) * w, y0), (x0 + (2 * i + 1) * w, y0 + h),
                (x0 + (2 * i + 2) * w, y0 + h)]
    pts += [(x0 + 2 * k * w, y0 - h), (x0, y0 - h)]
    a = np.array(pts, float)
    if vertical:
        a = a[:, ::-1].copy()[::-1].copy()
    return a


def test_many_intersections_retry_path(cuda):
    """Two crossing combs give O(k^2) output vertices: more than the first
    arena slice holds, so the pair is retried with a larger slice."""
    import parlllelrtree_b200 as prt

    s = [comb(40, 0.0, 0.0, 0.01, 0.9)]
    c = [comb(40, -0.05, -0.05, 0.0101, 0.95, vertical=True)]
    for op in OPS:
        got = prt.clip_pair(s, c, op)
        ref = oracle.gpc_clip(s, c, OPS.index(op))
        assert same_contours(got, ref), op


def test_clip_pair_degenerate(cuda):
    import parlllelrtree_b200 as prt

    sq = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float)
    cases = [([sq], [sq]), ([sq], [sq + [1, 0]]), ([sq], [sq + [1, 1]]), ([sq], [sq * 0.5 + 0.25]),
             ([sq], [sq + [5, 5]]), ([sq], []), ([], [sq]), ([sq, sq * 0.5 + 0.25], [sq + [0.5, 0.5]]),
             ([np.array([[0, 0], [2, 0], [2, 0], [1, 1]], float)], [sq]),
             ([np.array([[0, 0], [1, 0], [2, 0], [1, 1]], float)], [sq])]
    for s, c in cases:
        for op in OPS:
            assert same_contours(prt.clip_pair(s, c, op), oracle.gpc_clip(s, c, OPS.index(op))), (op,)


def test_reference_csr_entry_point(cuda):
    """run() with the reference's num/prefix/vertex/hole arrays."""
    import parlllelrtree_b200 as prt

    A, B = small_config(800, seed=9)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    t = prt.build_bottomup(LA.mbr(), fanout=10)
    pairs = t.join(LB.mbr(), sorted=True)
    l2p = t.leaf_order()
    numA = np.diff(A["ring_vert"]).astype(np.int32)
    numB = np.diff(B["ring_vert"]).astype(np.int32)
    r1 = prt.overlay_ref(pairs, numA, A["ring_vert"][:-1], A["xy"], A["ring_hole"], numB, B["ring_vert"][:-1],
                         B["xy"], B["ring_hole"], leaf_to_poly=l2p).contours()
    r2 = prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched="plain").contours()
    assert all(same_contours(x, y) for x, y in zip(r1, r2))


def test_results_area_matches_oracle(cuda):
    import parlllelrtree_b200 as prt

    g, A, B = golden()
    pairs = g["pairs"].astype(np.int32)
    res = prt.overlay(torch.from_numpy(pairs).cuda(), prt.Layer.from_dict(A), prt.Layer.from_dict(B))
    area = res.area().cpu().numpy()
    for k, (i, j) in enumerate(pairs):
        # same contours, same centred shoelace in the same order as the oracle
        ref = oracle.result_area(oracle.gpc_clip(rings_of(A, i), rings_of(B, j), 1))
        assert abs(area[k] - ref) <= 1e-12 * abs(ref) + 1e-24
