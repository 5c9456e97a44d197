"""The reference's text input formats: Rect1024.txt of the R-tree programs
and readData's polygon files, read and written by libprt.so's host code.
Checked against the reference's own readData (built from its sources into
oracle/_ref) and against the file writer the reference TD program's golden
digests were produced with.  No device needed."""
import os

import numpy as np
import pytest

import oracle
from parlllelrtree_b200 import datagen as dg

needs_ref = pytest.mark.skipif(not os.path.exists(os.path.join(oracle.REF_DIR, "libref_readdata.so")),
                               reason="oracle/_ref (the reference's CPU code) is not built")


def test_rect_file_round_trip_and_format(tmp_path):
    from parlllelrtree_b200 import io

    rects = dg.quantise(dg.mixture_boxes(5000, seed=3))
    keys = np.arange(5000, dtype=np.int32)[::-1].copy()
    p1, p2 = str(tmp_path / "ours.txt"), str(tmp_path / "oracle.txt")
    io.write_rect_file(p1, rects, keys)
    oracle.write_rect_file(p2, rects, keys)
    # byte for byte the format the reference programs read (the TD program's
    # golden digests were produced from oracle.write_rect_file's files)
    assert open(p1).read() == open(p2).read()
    b, k = io.read_rect_file(p2)
    assert np.array_equal(b, rects) and np.array_equal(k, keys)


def test_rect_file_whitespace_and_errors(tmp_path):
    from parlllelrtree_b200 import PrtError, io

    p = tmp_path / "r.txt"
    p.write_text("2\n  1 5 2 6 7\n\n\t-3   -1\n-4 0\n9\n")
    b, k = io.read_rect_file(str(p))
    assert b.tolist() == [[1, 2, 5, 6], [-3, -4, -1, 0]] and k.tolist() == [7, 9]
    p.write_text("2\n1 5 2 6 7\n1 x 2 3 4\n")
    with pytest.raises(PrtError, match="record 1 is malformed"):
        io.read_rect_file(str(p))
    with pytest.raises(PrtError, match="cannot open"):
        io.read_rect_file(str(tmp_path / "missing.txt"))


def _single_ring_layer(n, seed, **kw):
    from parlllelrtree_b200 import io

    L = dg.star_layer(n, seed=seed, **kw)
    d = io.layer_to_ref(L)
    d["hole"] = (np.arange(n) % 7 == 3).astype(np.int32)  # readData carries the flag through
    return d


@needs_ref
def test_polygon_files_match_reference_readdata(tmp_path):
    from parlllelrtree_b200 import io

    base = _single_ring_layer(700, seed=4, nv_lo=3, nv_hi=40)
    over = _single_ring_layer(500, seed=5, nv_lo=3, nv_hi=40, r_lo=1e-2, r_hi=5e-2)
    pb, po = str(tmp_path / "base.txt"), str(tmp_path / "overlay.txt")
    io.write_polygon_file(pb, base["num"], base["hole"], base["vertex"])
    io.write_polygon_file(po, over["num"], over["hole"], over["vertex"])
    ref = oracle.ref_read_data(pb, po)
    for path, src, name in ((pb, base, "base"), (po, over, "overlay")):
        got = io.read_polygon_file(path)
        r = ref[name]
        for k in ("num", "prefix", "hole", "rect", "vertex"):
            assert np.array_equal(got[k], r[k]), (name, k)
        # the doubles round-trip exactly and the box is the exact vertex bound
        assert np.array_equal(got["vertex"], src["vertex"])
        assert np.array_equal(got["num"], src["num"]) and np.array_equal(got["hole"], src["hole"])
        bb = dg.layer_bboxes({"poly_ring": np.arange(len(src["num"]) + 1), "ring_vert": np.r_[src["prefix"], len(src["vertex"])],
                              "xy": src["vertex"]})
        assert np.array_equal(got["mbr"], bb)
    assert ref["min_xy"] == (int(ref["base"]["rect"][:, 0].min()), int(ref["base"]["rect"][:, 1].min()))


@needs_ref
def test_polygon_file_negative_and_edge_values(tmp_path):
    """Negative coordinates (truncation toward zero) and values whose product
    with 1e5 lands next to an integer."""
    from parlllelrtree_b200 import io

    vert = np.array([[-0.000015, 0.3], [0.7, -1e-5], [0.12345678901234, 0.00001], [-2.5, 1.0]], np.float64)
    num = np.array([3, 1], np.int32)
    hole = np.array([0, 1], np.int32)
    pb, po = str(tmp_path / "b.txt"), str(tmp_path / "o.txt")
    io.write_polygon_file(pb, num, hole, vert)
    io.write_polygon_file(po, num[::-1].copy(), hole, np.r_[vert[3:], vert[:3]])
    ref = oracle.ref_read_data(pb, po)
    got = io.read_polygon_file(pb)
    assert np.array_equal(got["rect"], ref["base"]["rect"])
    assert np.array_equal(got["vertex"], ref["base"]["vertex"])
    got = io.read_polygon_file(po)
    assert np.array_equal(got["rect"], ref["overlay"]["rect"])
