"""Streaming overlay (results copied out chunk by chunk) and the overlay of
layers read from the reference's polygon files through its quantised boxes."""
import os

import numpy as np
import pytest
import torch

import oracle
from helpers import rings_of, same_contours
from parlllelrtree_b200 import datagen as dg

pytestmark = pytest.mark.gpu


def _overlay_inputs(n=3000, seed=40):
    import parlllelrtree_b200 as prt

    A = dg.star_layer(n, seed=seed, nv_lo=4, nv_hi=300, r_lo=0.005, r_hi=0.03, hole_frac=0.1, zipf=1.3)
    B = dg.star_layer(n, seed=seed + 1, nv_lo=4, nv_hi=300, r_lo=0.005, r_hi=0.03, hole_frac=0.1, zipf=1.3)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    t = prt.build_bottomup(LA.mbr(), fanout=16)
    pairs = t.join(LB.mbr(), sorted=True)
    return A, B, LA, LB, pairs, t.leaf_order()


@pytest.mark.parametrize("sched,chunk", [("batched", 777), ("plain", 2048), ("batched", 1 << 20)])
def test_stream_equals_one_shot(cuda, sched, chunk):
    import parlllelrtree_b200 as prt

    A, B, LA, LB, pairs, l2p = _overlay_inputs()
    whole = prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched=sched)
    off, nv, hole, xy = whole.to_host()
    seen = []

    def take(first, o, n_, h_, x_):
        # the arrays are views valid only during the call
        seen.append((first, o.copy(), n_.copy(), h_.copy(), x_.copy()))
        return 0

    prt.overlay_stream(pairs, LA, LB, take, leaf_to_poly=l2p, sched=sched, chunk_pairs=chunk)
    assert [s[0] for s in seen] == list(range(0, len(pairs), chunk))
    # concatenated chunks == the one-shot result set, bit for bit
    c0 = v0 = 0
    for first, o, n_, h_, x_ in seen:
        k = len(o) - 1
        assert k <= chunk
        assert np.array_equal(o + c0, off[first:first + k + 1])
        assert np.array_equal(n_, nv[c0:c0 + len(n_)]) and np.array_equal(h_, hole[c0:c0 + len(h_)])
        assert np.array_equal(x_, xy[v0:v0 + len(x_)])
        c0 += len(n_)
        v0 += len(x_)
    assert c0 == whole.n_contours and v0 == whole.n_vertices


def test_stream_callback_stop_and_errors(cuda):
    import parlllelrtree_b200 as prt

    A, B, LA, LB, pairs, l2p = _overlay_inputs(800, seed=50)
    calls = []
    with pytest.raises(prt.PrtError, match="callback returned"):
        prt.overlay_stream(pairs, LA, LB, lambda *a: calls.append(a[0]) or True, leaf_to_poly=l2p, chunk_pairs=100)
    assert calls == [0]

    def boom(*a):
        raise ValueError("from the callback")

    with pytest.raises(ValueError, match="from the callback"):
        prt.overlay_stream(pairs, LA, LB, boom, leaf_to_poly=l2p, chunk_pairs=100)
    # the context is fine afterwards
    r = prt.overlay(pairs[:50], LA, LB, leaf_to_poly=l2p)
    assert r.n_pairs == 50


def test_results_copy_pairs(cuda):
    import parlllelrtree_b200 as prt

    A, B, LA, LB, pairs, l2p = _overlay_inputs(1500, seed=60)
    r = prt.overlay(pairs, LA, LB, leaf_to_poly=l2p)
    allc = r.contours()
    pick = [len(pairs) - 1, 0, 17, 17, len(pairs) // 2]
    sub = r.contours_of(pick)
    for j, i in enumerate(pick):
        assert same_contours(sub[j], allc[i])


@pytest.mark.skipif(not os.path.exists(os.path.join(oracle.REF_DIR, "libref_readdata.so")),
                    reason="oracle/_ref (the reference's CPU code) is not built")
def test_overlay_from_reference_files_with_quantised_boxes(cuda, tmp_path):
    """Polygon files -> the reference's readData and ours agree -> device
    quantised boxes equal readData's (int)(v * 1e5) boxes -> an int32 tree
    over them joins to the brute-force candidate set of those integer boxes ->
    the pairs clipped through the reference CSR entry point equal the
    oracle's clips."""
    import parlllelrtree_b200 as prt
    from parlllelrtree_b200 import io

    base = io.layer_to_ref(dg.star_layer(1200, seed=70, nv_lo=3, nv_hi=40, r_lo=2e-3, r_hi=2e-2))
    over = io.layer_to_ref(dg.star_layer(900, seed=71, nv_lo=3, nv_hi=40, r_lo=2e-3, r_hi=2e-2))
    pb, po = str(tmp_path / "base.txt"), str(tmp_path / "overlay.txt")
    io.write_polygon_file(pb, base["num"], base["hole"], base["vertex"])
    io.write_polygon_file(po, over["num"], over["hole"], over["vertex"])
    ref = oracle.ref_read_data(pb, po)
    rb, ro = io.read_polygon_file(pb), io.read_polygon_file(po)
    LA, LB = io.layer_from_ref(rb), io.layer_from_ref(ro)
    qa, qb = LA.mbr_quantised(), LB.mbr_quantised()
    assert np.array_equal(qa.cpu().numpy(), ref["base"]["rect"])
    assert np.array_equal(qb.cpu().numpy(), ref["overlay"]["rect"])
    t = prt.build_bottomup(qa, fanout=16)
    assert t.coord == 3  # PRT_COORD_I32
    pairs = t.join(qb, sorted=True)
    l2p = t.leaf_order()
    p, perm = pairs.cpu().numpy(), l2p.cpu().numpy()
    ra, ro_ = ref["base"]["rect"].astype(np.int64), ref["overlay"]["rect"].astype(np.int64)
    exp = set()
    for j in range(len(ro_)):
        m = (ra[:, 0] <= ro_[j, 2]) & (ro_[j, 0] <= ra[:, 2]) & (ra[:, 1] <= ro_[j, 3]) & (ro_[j, 1] <= ra[:, 3])
        exp.update((int(i), j) for i in np.nonzero(m)[0])
    assert {(int(perm[a]), int(b)) for a, b in p} == exp
    res = prt.overlay_ref(pairs, rb["num"], rb["prefix"], rb["vertex"], rb["hole"], ro["num"], ro["prefix"],
                          ro["vertex"], ro["hole"], leaf_to_poly=l2p, sched="batched").contours()
    Ad = {"poly_ring": np.arange(len(rb["num"]) + 1), "ring_vert": np.r_[rb["prefix"], len(rb["vertex"])],
          "xy": rb["vertex"]}
    Bd = {"poly_ring": np.arange(len(ro["num"]) + 1), "ring_vert": np.r_[ro["prefix"], len(ro["vertex"])],
          "xy": ro["vertex"]}
    for k, (leaf, q) in enumerate(p):
        exp_c = oracle.gpc_clip(rings_of(Ad, perm[leaf]), rings_of(Bd, q), 1)
        assert same_contours(res[k], exp_c), k
