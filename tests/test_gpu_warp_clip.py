"""The warp-cooperative clipper (one pair per warp, active edge table in
registers up to 32 edges, in shared memory beyond) against the oracle, the
thread clipper and the reference's golden fixtures: the
batched schedule forced to warp mode for every pair, with 256 slots and with
32 slots (pairs whose active edge table outgrows 32 slots move it to their
arena), and a mixed warp / thread schedule."""
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
WARP = {"thresholds": [1 << 40], "warp_mode": [1], "warps_per_sm": 8, "aet_slots": 256}
WARP32 = {"thresholds": [1 << 40], "warp_mode": [1], "warps_per_sm": 8, "aet_slots": 32}
MIXED = {"thresholds": [1 << 40, 512, 64], "warp_mode": [1, 0, 1], "warps_per_sm": 4, "aet_slots": 64}
SCHEDS = {"warp": WARP, "warp32": WARP32, "mixed": MIXED}


def _overlay(prt, sched, pairs, LA, LB, l2p=None, op="int"):
    with prt.schedule(SCHEDS[sched]):
        return prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, op=op, sched="batched")


def _layer(polys):
    """Layer dict from a list of polygons, each a list of rings."""
    rings, holes, per = [], [], []
    for p in polys:
        per.append(len(p))
        for k, r in enumerate(p):
            rings.append(np.asarray(r, float))
            holes.append(1 if k else 0)
    return dg.layer_from_rings(rings, holes, per)


@pytest.mark.parametrize("sched", ["warp", "warp32"])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_golden_pairs_warp(cuda, sched, op):
    import parlllelrtree_b200 as prt

    g = np.load(os.path.join(GOLDEN, "gpc.npz"))
    A = {k[2:]: g[k] for k in g.files if k.startswith("a_")}
    B = {k[2:]: g[k] for k in g.files if k.startswith("b_")}
    pairs = torch.from_numpy(g["pairs"].astype(np.int32)).cuda()
    res = _overlay(prt, sched, pairs, prt.Layer.from_dict(A), prt.Layer.from_dict(B), op=OPS[op])
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


@pytest.mark.parametrize("sched", ["warp", "warp32", "mixed"])
def test_holes_and_uneven_sizes(cuda, sched):
    import parlllelrtree_b200 as prt

    A = dg.star_layer(300, seed=5, nv_lo=4, nv_hi=600, r_lo=0.02, r_hi=0.1, hole_frac=0.3, zipf=1.2)
    B = dg.star_layer(300, seed=6, nv_lo=4, nv_hi=600, r_lo=0.02, r_hi=0.1, hole_frac=0.3, zipf=1.2)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    t = prt.build_bottomup(LA.mbr(), fanout=16)
    pairs = t.join(LB.mbr(), sorted=True)
    l2p = t.leaf_order()
    p = pairs.cpu().numpy()
    perm = l2p.cpu().numpy()
    for op in OPS:
        got = _overlay(prt, sched, pairs, LA, LB, l2p, op).contours()
        for k, (leaf, q) in enumerate(p):
            ref = oracle.gpc_clip(rings_of(A, perm[leaf]), rings_of(B, q), OPS.index(op))
            assert same_contours(got[k], ref), (op, k)


def test_large_lobed_stars(cuda):
    """Pairs of up to 4096 + 4096 vertices, the batched config's shapes."""
    import parlllelrtree_b200 as prt

    rng = np.random.default_rng(11)
    K = 24
    nv = rng.choice([300, 1024, 2500, 4096], size=K)
    cen = rng.random((K, 2))
    ra = np.full(K, 6e-4)
    rb = rng.uniform(2e-4, 6e-4, size=K)
    rva, xya = dg._star_rings(rng, cen, ra, nv)
    rvb, xyb = dg._star_rings(rng, cen + rng.uniform(-3e-4, 3e-4, size=(K, 2)), rb, nv[::-1].copy())
    A = {"poly_ring": np.arange(K + 1), "ring_vert": rva, "ring_hole": np.zeros(K, np.int32), "xy": xya}
    B = {"poly_ring": np.arange(K + 1), "ring_vert": rvb, "ring_hole": np.zeros(K, np.int32), "xy": xyb}
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    pairs = torch.from_numpy(np.stack([np.arange(K), np.arange(K)], 1).astype(np.int32)).cuda()
    plain = prt.overlay(pairs, LA, LB, sched="plain").contours()
    for sched in ("warp", "warp32"):
        got = _overlay(prt, sched, pairs, LA, LB).contours()
        for k in range(K):
            assert same_contours(got[k], plain[k]), (sched, k)
    for k in range(0, K, 4):
        ref = oracle.gpc_clip(rings_of(A, k), rings_of(B, k), 1)
        assert same_contours(plain[k], ref), k


def comb(k, x0, y0, w, h, vertical=False):
    pts = []
    for i in range(k):
        pts += [(x0 + (2 * i) * w, y0), (x0 + (2 * i + 1) * w, y0), (x0 + (2 * i + 1) * w, y0 + h),
                (x0 + (2 * i + 2) * w, y0 + h)]
    pts += [(x0 + 2 * k * w, y0 - h), (x0, y0 - h)]
    a = np.array(pts, float)
    if vertical:
        a = a[:, ::-1].copy()[::-1].copy()
    return a


SQ = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float)
DEGENERATE = [([SQ], [SQ]), ([SQ], [SQ + [1, 0]]), ([SQ], [SQ + [1, 1]]), ([SQ], [SQ * 0.5 + 0.25]),
              ([SQ], [SQ + [5, 5]]), ([SQ, SQ * 0.5 + 0.25], [SQ + [0.5, 0.5]]),
              ([np.array([[0, 0], [2, 0], [2, 0], [1, 1]], float)], [SQ]),
              ([np.array([[0, 0], [1, 0], [2, 0], [1, 1]], float)], [SQ]),
              ([comb(12, 0.0, 0.0, 0.01, 0.9)], [comb(12, -0.05, -0.05, 0.0101, 0.95, vertical=True)]),
              ([comb(6, 0.0, 0.0, 0.01, 0.5)], [comb(6, 0.0, 0.0, 0.01, 0.5)]),
              ([comb(6, 0.0, 0.0, 0.01, 0.5)], [comb(6, 0.01, 0.0, 0.01, 0.5)])]


@pytest.mark.parametrize("sched", ["warp", "warp32"])
def test_degenerate_and_bundled(cuda, sched):
    """Coincident polygons and shared edges (bundles), horizontal edges,
    repeated and collinear vertices, holes, crossing combs."""
    import parlllelrtree_b200 as prt

    A = _layer([s for s, _ in DEGENERATE])
    B = _layer([c if len(c) else [SQ + [9, 9]] for _, c in DEGENERATE])
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    n = len(DEGENERATE)
    pairs = torch.from_numpy(np.stack([np.arange(n), np.arange(n)], 1).astype(np.int32)).cuda()
    for op in OPS:
        got = _overlay(prt, sched, pairs, LA, LB, op=op).contours()
        for k in range(n):
            ref = oracle.gpc_clip(rings_of(A, k), rings_of(B, k), OPS.index(op))
            assert same_contours(got[k], ref), (op, k)


def test_shared_edge_tessellations(cuda):
    """Two grids of squares / hexagons sharing edges exactly: every pair has
    bundled edges above and below scanbeams."""
    import parlllelrtree_b200 as prt

    cells = []
    for i in range(6):
        for j in range(6):
            cells.append([SQ * 0.1 + [0.1 * i, 0.1 * j]])
    hexes = []
    for i in range(6):
        for j in range(6):
            c = np.array([0.1 * i + 0.05 * (j % 2), 0.087 * j])
            a = np.arange(6) * np.pi / 3
            hexes.append([c + 0.058 * np.stack([np.cos(a), np.sin(a)], 1)])
    A, B = _layer(cells), _layer(cells[7:] + cells[:7])
    C = _layer(hexes)
    LA, LB, LC = prt.Layer.from_dict(A), prt.Layer.from_dict(B), prt.Layer.from_dict(C)
    for (X, Y, LX, LY) in ((A, B, LA, LB), (A, C, LA, LC), (C, C, LC, LC)):
        t = prt.build_bottomup(LX.mbr(), fanout=8)
        pairs = t.join(LY.mbr(), sorted=True)
        l2p = t.leaf_order()
        p = pairs.cpu().numpy()
        perm = l2p.cpu().numpy()
        for op in OPS:
            got = _overlay(prt, "warp", pairs, LX, LY, l2p, op).contours()
            for k, (leaf, q) in enumerate(p):
                ref = oracle.gpc_clip(rings_of(X, perm[leaf]), rings_of(Y, q), OPS.index(op))
                assert same_contours(got[k], ref), (op, k)


def test_area_mode_warp(cuda):
    """The area forward (clip + shoelace, area-only results) on the warp path."""
    import parlllelrtree_b200 as prt

    A = dg.star_layer(200, seed=21, nv_lo=16, nv_hi=900, r_lo=0.02, r_hi=0.06, zipf=1.1)
    B = dg.star_layer(200, seed=22, nv_lo=16, nv_hi=900, r_lo=0.02, r_hi=0.06, zipf=1.1)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    t = prt.build_bottomup(LA.mbr(), fanout=16)
    pairs = t.join(LB.mbr(), sorted=True)
    l2p = t.leaf_order().long()
    pa = l2p[pairs[:, 0].long()].int()
    pb = pairs[:, 1].int()
    a0 = prt.intersection_area(LA, LB, pa, pb)
    with prt.schedule(WARP):
        a1 = prt.intersection_area(LA, LB, pa, pb)
    assert torch.equal(a0, a1)


def _spiky(n_spikes, r_in, r_out, rot=0.0, centre=(0.0, 0.0), scale=1.0):
    a = rot + np.arange(2 * n_spikes) * np.pi / n_spikes
    r = np.where(np.arange(2 * n_spikes) % 2 == 0, r_out, r_in) * scale
    return np.stack([centre[0] + r * np.cos(a), centre[1] + r * np.sin(a)], 1)


@pytest.mark.parametrize("sched", ["warp", "warp32"])
def test_many_crossings_per_beam(cuda, sched):
    """Spiky stars against rotated, scaled and shifted copies of themselves:
    active edge tables of at most 32 edges with several crossings in one
    scanbeam (the register loop's crossing table, its sort by y and the
    bundle swaps), for all four ops; the warp clipper must give the thread
    clipper's contours."""
    import parlllelrtree_b200 as prt

    polys_a, polys_b = [], []
    rng = np.random.default_rng(5)
    for k in range(48):
        n = int(rng.integers(3, 9))
        base = _spiky(n, 0.3, 1.0, rot=rng.uniform(0, np.pi))
        polys_a.append([base])
        kind = k % 4
        if kind == 0:
            other = _spiky(n, 0.3, 1.0, rot=rng.uniform(0.02, 0.3))
        elif kind == 1:
            other = _spiky(n, 0.35, 1.1, rot=rng.uniform(0, np.pi), scale=rng.uniform(0.8, 1.2))
        elif kind == 2:
            other = _spiky(n + 1, 0.25, 0.9, rot=rng.uniform(0, np.pi), centre=rng.uniform(-0.2, 0.2, 2))
        else:
            other = base[::-1].copy() * 0.97 + rng.uniform(-0.05, 0.05, 2)
            other = other[::-1].copy()
        polys_b.append([other])
    A, B = _layer(polys_a), _layer(polys_b)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    n = len(polys_a)
    pairs = torch.from_numpy(np.stack([np.arange(n), np.arange(n)], 1).astype(np.int32)).cuda()
    for op in OPS:
        plain = prt.overlay(pairs, LA, LB, op=op, sched="plain").contours()
        got = _overlay(prt, sched, pairs, LA, LB, op=op).contours()
        for k in range(n):
            assert same_contours(got[k], plain[k]), (op, k)
        for k in range(0, n, 6):
            ref = oracle.gpc_clip(rings_of(A, k), rings_of(B, k), OPS.index(op))
            assert same_contours(plain[k], ref), (op, k)
