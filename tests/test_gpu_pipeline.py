"""The graph-captured pipeline (prt_pipeline_*): MBRs -> bottom-up tree ->
join -> batched clip as one CUDA graph.  Its candidate pairs must equal a
separate build + join bit for bit, and its per-pair contours must equal the
non-graph overlay of the same pairs, on the first run, on replays, and after
the layer coordinates change between replays."""
import numpy as np
import pytest
import torch

from helpers import same_contours
from parlllelrtree_b200 import datagen as dg

pytestmark = pytest.mark.gpu


def _layers(n=2000, seed=0, holes=0.0, zipf=None, nv_hi=32):
    A = dg.star_layer(n, seed=seed, r_lo=5e-3, r_hi=3e-2, zipf=zipf, nv_lo=4 if zipf else 8, nv_hi=nv_hi,
                      hole_frac=holes)
    B = dg.star_layer(n, seed=seed + 1, r_lo=5e-3, r_hi=3e-2, zipf=zipf, nv_lo=4 if zipf else 8, nv_hi=nv_hi,
                      hole_frac=holes)
    return A, B


def _split(off, nv, hole, xy):
    vo = np.zeros(len(nv) + 1, np.int64)
    np.cumsum(nv, out=vo[1:])
    return [[(int(hole[c]), xy[vo[c]:vo[c + 1]]) for c in range(off[i], off[i + 1])] for i in range(len(off) - 1)]


def _check_against_overlay(prt, pipe, LA, LB):
    s = pipe.sizes()
    assert s["overflow"] == 0 and s["timeout"] == 0 and s["failed"] == 0, s
    pairs, l2p = pipe.pairs()
    # the same candidate set as a separate build + join
    t = prt.build_bottomup(LA.mbr(), fanout=16)
    ref_pairs = t.join(LB.mbr()).cpu().numpy()
    got = pairs.cpu().numpy()
    got = got[np.lexsort((got[:, 1], got[:, 0]))]
    ref_pairs = ref_pairs[np.lexsort((ref_pairs[:, 1], ref_pairs[:, 0]))]
    assert np.array_equal(got, ref_pairs)
    assert torch.equal(l2p, t.leaf_order())
    # the same contours as the non-graph overlay of the same pairs
    res = prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched="plain")
    want = res.contours()
    have = _split(*pipe.to_host())
    assert len(have) == len(want) == s["pairs"]
    for k in range(len(want)):
        assert same_contours(have[k], want[k]), f"pair {k}"
    assert s["nonempty"] == res.nonempty and s["contours"] == res.n_contours and s["vertices"] == res.n_vertices


@pytest.mark.parametrize("holes,zipf,nv_hi", [(0.0, None, 32), (0.05, 1.2, 512)])
def test_pipeline_matches_overlay(cuda, holes, zipf, nv_hi):
    import parlllelrtree_b200 as prt

    A, B = _layers(holes=holes, zipf=zipf, nv_hi=nv_hi)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        pipe = prt.Pipeline(LA, LB)
        pipe.run()
        _check_against_overlay(prt, pipe, LA, LB)
        pipe.run()  # graph replay
        pipe.run()
        _check_against_overlay(prt, pipe, LA, LB)


def test_pipeline_replay_after_coordinates_change(cuda):
    """The graph reads the layers in place: moving layer B changes the
    candidate set and the clips, and a replay follows."""
    import parlllelrtree_b200 as prt

    A, B = _layers(seed=7)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        pipe = prt.Pipeline(LA, LB)
        pipe.run()
        n0 = pipe.sizes()["pairs"]
        LB.xy[:, 0] += 0.013
        LB.xy[:, 1] -= 0.007
        LB.xy.mul_(1.01)
        pipe.run()
        _check_against_overlay(prt, pipe, LA, LB)
        assert pipe.sizes()["pairs"] != n0


def test_pipeline_reports_pair_overflow(cuda):
    import parlllelrtree_b200 as prt

    A, B = _layers(n=500, seed=3)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        pipe = prt.Pipeline(LA, LB, max_pairs=16)
        pipe.run()
        s = pipe.sizes()
        assert s["overflow"] == 1 and s["pairs"] > 16


def test_pipeline_rejects_default_stream(cuda):
    import parlllelrtree_b200 as prt

    A, B = _layers(n=200, seed=4)
    pipe = prt.Pipeline(prt.Layer.from_dict(A), prt.Layer.from_dict(B))
    with torch.cuda.stream(torch.cuda.default_stream()):
        with pytest.raises(prt.PrtError):
            pipe.run()


def test_autotune_installs_a_valid_schedule(cuda, tmp_path):
    """prt_autotune times fanouts and schedules on a sample, installs the
    best schedule (which then gives the same contours), and its JSON cache
    returns the same choice without timing."""
    import parlllelrtree_b200 as prt

    A, B = _layers(n=600, seed=11, zipf=1.2, nv_hi=400)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    saved = prt.get_schedule()
    try:
        cache = str(tmp_path / "tune.json")
        r = prt.autotune(LA, LB, max_sample_pairs=2000, time_budget_s=20.0, cache=cache)
        assert not r["cached"] and r["fanout"] in (8, 12, 16, 24, 32) and r["candidates"] >= 6
        assert prt.get_schedule() == r["schedule"]
        r2 = prt.autotune(LA, LB, cache=cache)
        assert r2["cached"] and r2["schedule"] == r["schedule"]
        t = prt.build_bottomup(LA.mbr(), fanout=r["fanout"])
        pairs = t.join(LB.mbr(), sorted=True)
        l2p = t.leaf_order()
        tuned = prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched="batched").contours()
        plain = prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched="plain").contours()
        assert all(same_contours(x, y) for x, y in zip(tuned, plain))
    finally:
        prt.set_schedule(saved)
