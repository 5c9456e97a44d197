"""Pins the oracle (CPU restatement) to the reference's own outputs: the
committed golden fixtures (made by tests/golden/gen_golden.py from the
reference's code) and, when oracle/_ref is built here, live runs of the
reference's CPU code on fresh seeded inputs."""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN
from helpers import compare_bu, compare_td, levels_to_bu, levels_to_td, rings_of, same_contours
from parlllelrtree_b200 import datagen as dg

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (reference absent)")


def shifted(rects):
    """The BU program shifts the stored boxes by (min x1, min y1) (BU:704-709)."""
    r = rects.copy()
    r[:, [0, 2]] -= r[:, 0].min()
    r[:, [1, 3]] -= r[:, 1].min()
    return r


@pytest.mark.parametrize("F", [10, 16, 32])
def test_bu_golden(F):
    g = np.load(os.path.join(GOLDEN, f"bu_m{F}.npz"))
    rects = g["rects"]
    keys, scale, _ = oracle.keys_ref64(rects)
    assert scale == int(g["scale"])
    assert np.array_equal(keys, g["keys"])
    perm = oracle.stable_argsort(keys)
    assert np.array_equal(perm, g["sorted_ids"])
    lv = oracle.pack(shifted(rects), F, perm)
    compare_bu(levels_to_bu(lv, F, perm), {k: g[k] for k in ("flag", "num", "mbr", "children", "data")}
               | {"root": int(g["root"])})
    assert oracle.digests(lv, F, shifted(rects)) == tuple(int(x) for x in g["digests"])


@pytest.mark.parametrize("F", [10, 16, 32])
def test_td_golden(F):
    g = np.load(os.path.join(GOLDEN, f"td_m{F}.npz"))
    rects = g["rects"]
    perm = oracle.td_order(rects, F)
    assert np.array_equal(rects[perm], g["sorted_rects"])
    lv = oracle.pack(rects, F, perm)
    compare_td(levels_to_td(lv, F), {k: g[k] for k in ("nodes_index", "nodes_mbr", "offsets")})
    assert oracle.digests(lv, F, rects, td_slots=True) == tuple(int(x) for x in g["digests"])


def test_td_program_golden():
    with open(os.path.join(GOLDEN, "td_program.json")) as f:
        g = json.load(f)
    rects = np.load(os.path.join(GOLDEN, "td_m10.npz"))["rects"]
    assert len(rects) == g["n"]
    perm = oracle.td_order(rects, 10)
    lv = oracle.pack(rects, 10, perm)
    assert oracle.digests(lv, 10, rects, td_slots=True) == (g["sum"], g["sum1"], g["sum2"], g["sum3"])


def _golden_gpc():
    g = np.load(os.path.join(GOLDEN, "gpc.npz"))
    A = {k[2:]: g[k] for k in g.files if k.startswith("a_")}
    B = {k[2:]: g[k] for k in g.files if k.startswith("b_")}
    return g, A, B


@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_gpc_golden(op):
    g, A, B = _golden_gpc()
    nc, nv, hole, xy = g[f"op{op}_ncont"], g[f"op{op}_nverts"], g[f"op{op}_hole"], g[f"op{op}_xy"]
    c = v = 0
    for k, (i, j) in enumerate(g["pairs"]):
        ref = []
        for _ in range(nc[k]):
            ref.append((int(hole[c]), xy[v:v + nv[c]]))
            v += nv[c]
            c += 1
        got = oracle.gpc_clip(rings_of(A, i), rings_of(B, j), op)
        assert same_contours(got, ref), f"pair {k} op {op}"


def test_interleave_spreads_low_16_bits():
    assert oracle.interleave4(0xFFFF, 0, 0, 0) == 0xC0C0C0C0C0C0C0C0
    assert oracle.interleave4(0, 0, 0, 0xFFFF) == 0x0303030303030303
    assert oracle.interleave4(0x10000, 0, 0, 0) == 0


@needs_ref
def test_interleave_matches_reference():
    rng = np.random.default_rng(5)
    for _ in range(2000):
        a = [int(x) for x in rng.integers(0, 1 << 16, size=4)]
        assert oracle.interleave4(*a) == oracle.ref_interleave(*a)


@needs_ref
def test_overlap_predicate_matches_reference():
    rng = np.random.default_rng(6)
    for _ in range(3000):
        a = np.sort(rng.integers(0, 50, size=(2, 2)), axis=0).T.reshape(-1)[[0, 2, 1, 3]]
        b = np.sort(rng.integers(0, 50, size=(2, 2)), axis=0).T.reshape(-1)[[0, 2, 1, 3]]
        mine = a[0] <= b[2] and b[0] <= a[2] and a[1] <= b[3] and b[1] <= a[3]
        assert oracle.ref_overlap(a, b, "bu") == int(mine)
        assert oracle.ref_overlap(a, b, "td") == int(mine)


@needs_ref
@pytest.mark.parametrize("n", [1, 2, 9, 10, 11, 16, 17, 100, 257, 5000])
@pytest.mark.parametrize("F", [10, 16, 32])
def test_bu_live_reference(n, F):
    rects = dg.quantise(dg.mixture_boxes(n, seed=n + F, mean_side=5e-3))
    ref = oracle.ref_bu_run(rects, F)
    keys, _, _ = oracle.keys_ref64(rects)
    assert np.array_equal(keys, ref["keys"])
    perm = oracle.stable_argsort(keys)
    assert np.array_equal(perm, ref["sorted_ids"])
    lv = oracle.pack(shifted(rects), F, perm)
    compare_bu(levels_to_bu(lv, F, perm), ref)
    assert oracle.digests(lv, F, shifted(rects)) == ref["digests"]


@needs_ref
@pytest.mark.parametrize("n", [2, 9, 10, 11, 100, 101, 1000, 4097])
@pytest.mark.parametrize("F", [10, 16, 32])
def test_td_live_reference(n, F):
    rects = dg.quantise(dg.mixture_boxes(n, seed=3 * n + F, mean_side=5e-3))
    rects -= rects[:, [0, 1, 0, 1]].min()
    ref = oracle.ref_td_run(rects, F)
    perm = oracle.td_order(rects, F)
    assert np.array_equal(rects[perm], ref["sorted_rects"])
    lv = oracle.pack(rects, F, perm)
    compare_td(levels_to_td(lv, F), ref)
    assert oracle.digests(lv, F, rects, td_slots=True) == ref["digests"]


@needs_ref
def test_gpc_live_reference_with_holes():
    A = dg.star_layer(60, seed=31, nv_lo=4, nv_hi=40, r_lo=0.05, r_hi=0.2, hole_frac=0.5)
    B = dg.star_layer(60, seed=32, nv_lo=4, nv_hi=40, r_lo=0.05, r_hi=0.2, hole_frac=0.5)
    n = 0
    for i in range(60):
        for j in range(60):
            for op in (0, 1, 2, 3):
                got = oracle.gpc_clip(rings_of(A, i), rings_of(B, j), op)
                ref = oracle.ref_gpc_clip(rings_of(A, i), rings_of(B, j), op)
                assert same_contours(got, ref), (i, j, op)
                n += len(got) > 0
    assert n > 100


@needs_ref
def test_gpc_degenerate_cases():
    sq = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float)
    cases = [
        ([sq], [sq]),                                  # identical
        ([sq], [sq + [1, 0]]),                          # shared edge
        ([sq], [sq + [1, 1]]),                          # shared corner
        ([sq], [sq * 0.5 + 0.25]),                      # containment
        ([sq], [sq + [5, 5]]),                          # disjoint
        ([sq], []),                                     # empty clip
        ([], [sq]),                                     # empty subject
        ([sq, sq * 0.5 + 0.25], [sq + [0.5, 0.5]]),     # ring inside ring
        ([np.array([[0, 0], [2, 0], [2, 0], [1, 1]], float)], [sq]),  # repeated vertex
        ([np.array([[0, 0], [1, 0], [2, 0], [1, 1]], float)], [sq]),  # collinear horizontal run
    ]
    for s, c in cases:
        for op in (0, 1, 2, 3):
            assert same_contours(oracle.gpc_clip(s, c, op), oracle.ref_gpc_clip(s, c, op)), (s, c, op)


def test_area_gradient_matches_finite_differences():
    A = dg.star_layer(5, seed=41, nv_lo=16, nv_hi=24, r_lo=0.1, r_hi=0.1, centre_xy=np.full((5, 2), 0.5))
    B = dg.star_layer(5, seed=42, nv_lo=16, nv_hi=24, r_lo=0.1, r_hi=0.1, centre_xy=np.full((5, 2), 0.52))
    h = 1e-6
    for p in range(3):
        s, c = rings_of(A, p), rings_of(B, p)
        area, gs, gc = oracle.area_grad(s, c)
        assert abs(area - oracle.result_area(oracle.gpc_clip(s, c, 1))) < 1e-12 * max(area, 1e-30) + 1e-18
        fd = np.zeros_like(gs)
        for v in range(len(s[0])):
            for d in range(2):
                sp, sm = s[0].copy(), s[0].copy()
                sp[v, d] += h
                sm[v, d] -= h
                fd[v, d] = (oracle.result_area(oracle.gpc_clip([sp], c, 1)) -
                            oracle.result_area(oracle.gpc_clip([sm], c, 1))) / (2 * h)
        # tolerance: central differences with h = 1e-6 (truncation ~h^2 f''',
        # rounding ~eps * area / h)
        assert np.abs(fd - gs).max() <= 1e-6 * np.abs(gs).max() + 1e-9
