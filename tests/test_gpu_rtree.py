"""R-tree build / join / query counters on the GPU, checked bit-exactly
against the oracle (and through it against the reference's fixtures)."""
import os

import numpy as np
import pytest
import torch

import oracle
from conftest import GOLDEN
from helpers import brute_pairs, compare_bu, compare_td, levels_to_bu, levels_to_td
from parlllelrtree_b200 import datagen as dg

pytestmark = pytest.mark.gpu

DT = {"i64": torch.int64, "f32": torch.float32, "f64": torch.float64, "i32": torch.int32}


def boxes_of(kind, n, seed, side=2e-3):
    b = dg.mixture_boxes(n, seed=seed, mean_side=side)
    if kind == "f32":
        return b
    if kind == "f64":
        return b.astype(np.float64) + np.float64(1e-9) * np.arange(4)
    if kind == "i64":
        return dg.quantise(b)
    return dg.quantise(b).astype(np.int32)


def check_levels(tree, ref_levels):
    assert tree.levels == len(ref_levels)
    for l in range(tree.levels):
        got = tree.level_mbr(l)
        assert np.array_equal(got, ref_levels[l]), f"level {l}"


@pytest.mark.parametrize("kind", ["f32", "f64", "i64", "i32"])
@pytest.mark.parametrize("F", [10, 16, 32])
@pytest.mark.parametrize("n", [1, 7, 16, 17, 1000, 70001])
def test_bottomup_morton32(cuda, kind, F, n):
    import parlllelrtree_b200 as prt

    b = boxes_of(kind, n, seed=n + F)
    keys, _ = oracle.keys_morton32(b)
    perm = oracle.stable_argsort(keys)
    lv = oracle.pack(b, F, perm)
    t = prt.build_bottomup(torch.from_numpy(b).cuda(), fanout=F, key_mode="morton32")
    check_levels(t, lv)
    assert np.array_equal(t.leaf_order().cpu().numpy(), perm)


@pytest.mark.parametrize("F", [10, 16, 32])
def test_bottomup_ref64_golden(cuda, F):
    """The reference's own BU node array (golden fixture) from the device build."""
    import parlllelrtree_b200 as prt

    g = np.load(os.path.join(GOLDEN, f"bu_m{F}.npz"))
    rects = g["rects"]
    t = prt.build_bottomup(torch.from_numpy(rects).cuda(), fanout=F, key_mode="ref64")
    assert np.array_equal(t.leaf_order().cpu().numpy(), g["sorted_ids"])
    ex = t.export_bu()
    sx, sy = rects[:, 0].min(), rects[:, 1].min()
    ex["mbr"] = ex["mbr"] - np.array([sx, sy, sx, sy], np.float64)  # the reference stores shifted boxes
    compare_bu(ex, {k: g[k] for k in ("flag", "num", "mbr", "children", "data")} | {"root": int(g["root"])})
    sh = rects - np.array([sx, sy, sx, sy])
    d = t.digests(torch.from_numpy(rects).cuda())
    assert d == tuple(int(x) for x in g["digests"][:4])


@pytest.mark.parametrize("F", [10, 16, 32])
def test_topdown_golden(cuda, F):
    import parlllelrtree_b200 as prt

    g = np.load(os.path.join(GOLDEN, f"td_m{F}.npz"))
    rects = g["rects"]
    t = prt.build_topdown(torch.from_numpy(rects).cuda(), fanout=F)
    compare_td(t.export_td(), {k: g[k] for k in ("nodes_index", "nodes_mbr", "offsets")})
    d = t.digests(torch.from_numpy(rects).cuda(), td_slots=True)
    assert d == tuple(int(x) for x in g["digests"][:4])


@pytest.mark.parametrize("kind", ["f32", "f64", "i64", "i32"])
@pytest.mark.parametrize("F", [10, 16, 32])
@pytest.mark.parametrize("n", [1, 10, 11, 5000, 40000])
def test_topdown(cuda, kind, F, n):
    import parlllelrtree_b200 as prt

    b = boxes_of(kind, n, seed=7 * n + F)
    perm = oracle.td_order(b, F)
    lv = oracle.pack(b, F, perm)
    t = prt.build_topdown(torch.from_numpy(b).cuda(), fanout=F)
    check_levels(t, lv)
    assert np.array_equal(t.leaf_order().cpu().numpy(), perm)
    compare_td(t.export_td(), levels_to_td(lv, F))
    compare_bu(t.export_bu(), levels_to_bu(lv, F, perm))


@pytest.mark.parametrize("kind", ["f32", "i64"])
@pytest.mark.parametrize("F", [2, 4, 8])
@pytest.mark.parametrize("n", [1, 5000, 40000])
def test_small_fanouts(cuda, kind, F, n):
    """Fanouts below 10: many short-run levels (at F=2 more than one
    shared-memory launch holds), the last level's runs of F records sorted by
    counting ranks; bottom-up and top-down both bit-exact against the oracle."""
    import parlllelrtree_b200 as prt

    b = boxes_of(kind, n, seed=11 * n + F)
    perm = oracle.td_order(b, F)
    lv = oracle.pack(b, F, perm)
    t = prt.build_topdown(torch.from_numpy(b).cuda(), fanout=F)
    check_levels(t, lv)
    assert np.array_equal(t.leaf_order().cpu().numpy(), perm)
    compare_td(t.export_td(), levels_to_td(lv, F))
    modes = [("morton32", oracle.keys_morton32(b)[0])]
    if kind == "i64":
        modes.append(("ref64", oracle.keys_ref64(b)[0]))
    for mode, keys in modes:
        perm_bu = oracle.stable_argsort(keys)
        tb = prt.build_bottomup(torch.from_numpy(b).cuda(), fanout=F, key_mode=mode)
        assert np.array_equal(tb.leaf_order().cpu().numpy(), perm_bu)
        check_levels(tb, oracle.pack(b, F, perm_bu))


def test_sort_stability_many_ties(cuda):
    """Heavy key ties: the leaf order must keep input order inside each tie."""
    import parlllelrtree_b200 as prt

    rng = np.random.default_rng(3)
    c = rng.integers(0, 8, size=(300000, 2)).astype(np.float32)
    b = np.concatenate([c, c + 1], axis=1).astype(np.float32)
    keys, _ = oracle.keys_morton32(b)
    perm = oracle.stable_argsort(keys)
    t = prt.build_bottomup(torch.from_numpy(b).cuda(), fanout=16)
    assert np.array_equal(t.leaf_order().cpu().numpy(), perm)


@pytest.mark.parametrize("kind", ["f32", "i64"])
@pytest.mark.parametrize("F", [10, 16, 32])
@pytest.mark.parametrize("build", ["bottomup", "topdown"])
def test_join_pairs_exact(cuda, kind, F, build):
    import parlllelrtree_b200 as prt

    b = boxes_of(kind, 20000, seed=F, side=4e-3)
    q = boxes_of(kind, 3000, seed=F + 100, side=8e-3)
    fn = prt.build_bottomup if build == "bottomup" else prt.build_topdown
    t = fn(torch.from_numpy(b).cuda(), fanout=F)
    pairs = t.join(torch.from_numpy(q).cuda(), sorted=True).cpu().numpy()
    lv = t.levels_mbr()
    ref = oracle.join_pairs(lv, F, q)
    # sorted by (query, leaf); the oracle's DFS order per query is increasing leaf
    ref = ref[np.lexsort((ref[:, 0], ref[:, 1]))]
    assert np.array_equal(pairs.astype(np.int64), ref)
    # and the candidate set equals the brute-force box intersection set
    perm = t.leaf_order().cpu().numpy()
    got = {(int(perm[a]), int(qq)) for a, qq in pairs}
    assert got == brute_pairs(b, q)


def test_join_empty_and_edge(cuda):
    import parlllelrtree_b200 as prt

    b = np.array([[0, 0, 1, 1], [2, 2, 3, 3]], np.float32)
    t = prt.build_bottomup(torch.from_numpy(b).cuda(), fanout=16)
    q = np.array([[1, 1, 2, 2], [5, 5, 6, 6], [-1, -1, -0.5, -0.5]], np.float32)  # touching both, none, none
    p = t.join(torch.from_numpy(q).cuda(), sorted=True).cpu().numpy()
    assert p.tolist() == [[0, 0], [1, 0]] or p.tolist() == [[1, 0], [0, 0]]
    assert len(t.join(torch.zeros((0, 4), dtype=torch.float32).cuda())) == 0


@pytest.mark.parametrize("F", [10, 16, 32])
def test_query_counts_match_oracle(cuda, F):
    import parlllelrtree_b200 as prt

    b = boxes_of("i64", 30000, seed=F + 5, side=3e-3)
    for build, td in (("bottomup", False), ("topdown", True)):
        fn = prt.build_bottomup if build == "bottomup" else prt.build_topdown
        t = fn(torch.from_numpy(b).cuda(), fanout=F)
        got = t.query_counts(torch.from_numpy(b).cuda(), td_slots=td).cpu().numpy()
        ref = oracle.query_counts(t.levels_mbr(), F, b, td_slots=td)
        assert np.array_equal(got, ref)


def test_large_build_parity(cuda):
    """2M float32 boxes: levels and leaf order bit-exact, bottom-up and top-down."""
    import parlllelrtree_b200 as prt

    b = dg.mixture_boxes(2_000_000, seed=0)
    keys, _ = oracle.keys_morton32(b)
    perm = oracle.stable_argsort(keys)
    t = prt.build_bottomup(torch.from_numpy(b).cuda(), fanout=16)
    assert np.array_equal(t.leaf_order().cpu().numpy(), perm)
    check_levels(t, oracle.pack(b, 16, perm))
    perm = oracle.td_order(b, 32)
    t = prt.build_topdown(torch.from_numpy(b).cuda(), fanout=32)
    assert np.array_equal(t.leaf_order().cpu().numpy(), perm)
