"""The map-alignment loop: gradient ascent on total overlap (R-tree rebuild,
join, GPC clip, area adjoint every step) recovers the affine transform that
was applied to a parcel map, to well below the vertex noise."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_fit_recovers_affine(cuda):
    from parlllelrtree_b200 import alignment as al

    A, B, T = al.parcel_layers(20_000, seed=3)
    assert al.recovery_error(np.zeros(6), T) > 5e-3  # the transform moves parcels by several widths
    theta, rec, stage_s = al.fit_affine(A, B, steps=200)
    assert len(rec) == 200 and len(stage_s) == 4
    assert al.recovery_error(theta, T) < 1e-4  # vertex noise is 1e-4 per coordinate
    assert rec[-1]["overlap"] > 0.9 and rec[-1]["parcels"] == 20_000


def test_parcel_layers_are_disjoint_and_ccw(cuda):
    import torch

    import parlllelrtree_b200 as prt
    from parlllelrtree_b200 import alignment as al

    A, _, _ = al.parcel_layers(5000, seed=1)
    L = prt.Layer.from_dict(A)
    t = prt.build_bottomup(L.mbr(), fanout=16)
    pairs = t.join(L.mbr())
    l2p = t.leaf_order()
    pa = l2p[pairs[:, 0].long()]
    pb = pairs[:, 1]
    # neighbouring parcels' boxes are apart: the self-join finds only (i, i)
    assert len(pairs) == 5000 and bool(torch.all(pa == pb))
    # and an empty pair list is a valid call with an empty result
    empty = torch.empty(0, dtype=torch.int32, device="cuda")
    assert prt.intersection_area(L, L, empty, empty).numel() == 0
    xy, rv = A["xy"], A["ring_vert"]
    for i in range(0, 5000, 97):
        r = xy[rv[i]:rv[i + 1]]
        assert 0.5 * np.sum(r[:, 0] * np.roll(r[:, 1], -1) - np.roll(r[:, 0], -1) * r[:, 1]) > 0
