"""Intersection area forward and the hand-written adjoint: against the
oracle's area and reference gradient, and against central finite
differences (h = 1e-6)."""
import numpy as np
import pytest
import torch

import oracle
from helpers import rings_of
from parlllelrtree_b200 import datagen as dg

pytestmark = pytest.mark.gpu


def overlapping_pairs(n, seed, nv_lo=16, nv_hi=64, hole_frac=0.0):
    """Star pairs with overlap guaranteed by a centre offset <= 0.5 r."""
    rng = np.random.default_rng(seed)
    r = np.exp(rng.uniform(np.log(1e-3), np.log(1e-2), size=n))
    c = rng.random((n, 2))
    ang = rng.uniform(0, 2 * np.pi, size=n)
    off = 0.5 * r * rng.random(n)
    c2 = c + np.stack([off * np.cos(ang), off * np.sin(ang)], axis=1)
    A = dg.star_layer(n, seed=seed + 1, nv_lo=nv_lo, nv_hi=nv_hi, centre_xy=c, radii=r, hole_frac=hole_frac)
    B = dg.star_layer(n, seed=seed + 2, nv_lo=nv_lo, nv_hi=nv_hi, centre_xy=c2, radii=r, hole_frac=hole_frac)
    return A, B


@pytest.mark.parametrize("hole_frac", [0.0, 0.5])
def test_forward_and_adjoint_match_oracle(cuda, hole_frac):
    import parlllelrtree_b200 as prt

    n = 2000
    A, B = overlapping_pairs(n, seed=int(hole_frac * 10) + 1, hole_frac=hole_frac)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    idx = torch.arange(n, dtype=torch.int32, device="cuda")
    xa = LA.xy.clone().requires_grad_(True)
    xb = LB.xy.clone().requires_grad_(True)
    w = torch.from_numpy(np.random.default_rng(0).uniform(0.5, 2.0, n)).cuda()
    area = prt.intersection_area(LA, LB, idx, idx, xa, xb)
    (area * w).sum().backward()
    area = area.detach().cpu().numpy()
    ga = xa.grad.cpu().numpy()
    gb = xb.grad.cpu().numpy()
    wn = w.cpu().numpy()
    for i in range(n):
        s, c = rings_of(A, i), rings_of(B, i)
        ref = oracle.result_area(oracle.gpc_clip(s, c, 1))
        assert abs(area[i] - ref) <= 1e-9 * abs(ref) + 1e-22, i
        hs = A["ring_hole"][A["poly_ring"][i]:A["poly_ring"][i + 1]]
        hc = B["ring_hole"][B["poly_ring"][i]:B["poly_ring"][i + 1]]
        _, rs, rc = oracle.area_grad(s, c, hs, hc)
        va = slice(A["ring_vert"][A["poly_ring"][i]], A["ring_vert"][A["poly_ring"][i + 1]])
        vb = slice(B["ring_vert"][B["poly_ring"][i]], B["ring_vert"][B["poly_ring"][i + 1]])
        scale = max(np.abs(rs).max(), np.abs(rc).max(), 1e-30)
        # tolerance 1e-9 relative: the device sums atomically in another order
        assert np.abs(ga[va] - wn[i] * rs).max() <= 1e-9 * wn[i] * scale, i
        assert np.abs(gb[vb] - wn[i] * rc).max() <= 1e-9 * wn[i] * scale, i


def test_adjoint_matches_finite_differences(cuda):
    import parlllelrtree_b200 as prt

    n = 6
    A, B = overlapping_pairs(n, seed=17)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    idx = torch.arange(n, dtype=torch.int32, device="cuda")
    xa = LA.xy.clone().requires_grad_(True)
    prt.intersection_area(LA, LB, idx, idx, xa, LB.xy).sum().backward()
    g = xa.grad.cpu().numpy()
    h = 1e-6
    x0 = LA.xy.clone()
    fd = np.zeros_like(g)
    for v in range(len(g)):
        for d in range(2):
            xp = x0.clone()
            xp[v, d] += h
            xm = x0.clone()
            xm[v, d] -= h
            ap = prt.intersection_area(LA, LB, idx, idx, xp, LB.xy).sum().item()
            am = prt.intersection_area(LA, LB, idx, idx, xm, LB.xy).sum().item()
            fd[v, d] = (ap - am) / (2 * h)
    # central differences, h = 1e-6: error ~ h^2 |f'''| + eps |area| / h
    assert np.abs(fd - g).max() <= 1e-6 * np.abs(g).max() + 1e-9


def test_shared_polygons_accumulate(cuda):
    """A polygon in several pairs receives the sum of their gradients."""
    import parlllelrtree_b200 as prt

    A, B = overlapping_pairs(50, seed=23)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    pa = torch.tensor([0, 0, 0, 1], dtype=torch.int32, device="cuda")
    pb = torch.tensor([0, 0, 1, 1], dtype=torch.int32, device="cuda")
    xa = LA.xy.clone().requires_grad_(True)
    prt.intersection_area(LA, LB, pa, pb, xa, LB.xy).sum().backward()
    g = xa.grad.cpu().numpy()
    s0 = rings_of(A, 0)
    _, g00, _ = oracle.area_grad(s0, rings_of(B, 0))
    _, g01, _ = oracle.area_grad(s0, rings_of(B, 1))
    v0 = slice(A["ring_vert"][0], A["ring_vert"][1])
    ref = 2 * g00 + g01
    assert np.abs(g[v0] - ref).max() <= 1e-9 * np.abs(ref).max() + 1e-20
