"""Generates the golden fixtures in this directory by running the REFERENCE's
own code (oracle/_ref, built from the reference sources by
oracle/ref/build_ref.sh) on seeded synthetic inputs.

    python tests/golden/gen_golden.py

Fixtures (all small, committed):
  bu_m{F}.npz      BotomUp-rtree.cu CPU path at fanout F: keys, qsort order,
                   rtree_node array, digests sum/sum1/sum2/sum3
  td_m{F}.npz      TopDown-rtree.cu CPU path: slot arrays, level offsets,
                   final record order, digests
  td_program.json  digests printed by the unchanged TopDown-rtree.cu program
  gpc.npz          the reference clip core on star-polygon pairs, all four ops
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from parlllelrtree_b200 import datagen as dg  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def rect_input(n: int, seed: int) -> np.ndarray:
    """int64 boxes on the 1e6 grid, shifted to be non-negative (the top-down
    program keys raw coordinates as unsigned integers, TopDown-rtree.cu:579)."""
    r = dg.quantise(dg.mixture_boxes(n, seed=seed, mean_side=2e-3))
    return r - r[:, [0, 1, 0, 1]].min()


def star_pairs(n_layer: int, seed: int, max_pairs: int):
    A = dg.star_layer(n_layer, seed=seed, nv_lo=3, nv_hi=24, r_lo=0.02, r_hi=0.08)
    B = dg.star_layer(n_layer, seed=seed + 1, nv_lo=3, nv_hi=24, r_lo=0.02, r_hi=0.08)
    ba, bb = dg.layer_bboxes(A), dg.layer_bboxes(B)
    pairs = []
    for i in range(len(ba)):
        m = (ba[i, 0] <= bb[:, 2]) & (bb[:, 0] <= ba[i, 2]) & (ba[i, 1] <= bb[:, 3]) & (bb[:, 1] <= ba[i, 3])
        pairs.extend((i, int(j)) for j in np.nonzero(m)[0])
    rng = np.random.default_rng(seed)
    pairs = np.array(pairs, dtype=np.int64)
    pairs = pairs[rng.permutation(len(pairs))[:max_pairs]]
    return A, B, pairs


def rings_of(layer, p):
    pr, rv, xy = layer["poly_ring"], layer["ring_vert"], layer["xy"]
    return [xy[rv[r]:rv[r + 1]] for r in range(pr[p], pr[p + 1])]


def main() -> None:
    if not oracle.build_ref():
        raise SystemExit("the reference sources are needed to generate the fixtures")
    rects = rect_input(3000, seed=11)
    for F in (10, 16, 32):
        r = oracle.ref_bu_run(rects, F)
        np.savez_compressed(os.path.join(OUT, f"bu_m{F}.npz"), rects=rects, keys=r["keys"], scale=r["scale"],
                            sorted_ids=r["sorted_ids"], flag=r["flag"], num=r["num"], mbr=r["mbr"],
                            children=r["children"], data=r["data"], root=r["root"],
                            digests=np.array(r["digests"], dtype=np.int64))
        t = oracle.ref_td_run(rects, F)
        np.savez_compressed(os.path.join(OUT, f"td_m{F}.npz"), rects=rects, nodes_index=t["nodes_index"],
                            nodes_mbr=t["nodes_mbr"], offsets=t["offsets"], sorted_rects=t["sorted_rects"],
                            digests=np.array(t["digests"], dtype=np.int64))
    with tempfile.TemporaryDirectory() as d:
        res = oracle.run_td_program(rects, d)
    res.pop("stdout", None)
    with open(os.path.join(OUT, "td_program.json"), "w") as f:
        json.dump({"n": int(len(rects)), "seed": 11, **res}, f, indent=1)

    A, B, pairs = star_pairs(400, seed=21, max_pairs=600)
    recs = {"pairs": pairs}
    for key, layer in (("a", A), ("b", B)):
        for k, v in layer.items():
            recs[f"{key}_{k}"] = v
    for op in (0, 1, 2, 3):
        ncont, nverts, holes, xys = [], [], [], []
        for (i, j) in pairs:
            res = oracle.ref_gpc_clip(rings_of(A, i), rings_of(B, j), op)
            ncont.append(len(res))
            for h, v in res:
                nverts.append(len(v))
                holes.append(h)
                xys.append(v)
        recs[f"op{op}_ncont"] = np.array(ncont, dtype=np.int32)
        recs[f"op{op}_nverts"] = np.array(nverts, dtype=np.int32)
        recs[f"op{op}_hole"] = np.array(holes, dtype=np.int32)
        recs[f"op{op}_xy"] = np.concatenate(xys) if xys else np.zeros((0, 2))
    np.savez_compressed(os.path.join(OUT, "gpc.npz"), **recs)
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
