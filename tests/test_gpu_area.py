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


@pytest.mark.parametrize("hole_frac,nv", [(0.0, (16, 64)), (0.5, (16, 64)), (0.0, (40, 100)), (0.3, (100, 200))])
def test_forward_and_adjoint_match_oracle(cuda, hole_frac, nv):
    """Pairs of up to 64 vertices per polygon take the first slab-indexed
    stage, up to 128 the second, larger ones the brute-force adjoint; all
    must give the oracle's area and gradient."""
    import parlllelrtree_b200 as prt

    n = 2000 if nv[1] <= 64 else 300
    A, B = overlapping_pairs(n, seed=int(hole_frac * 10) + nv[0], nv_lo=nv[0], nv_hi=nv[1], hole_frac=hole_frac)
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


def _fd_check(prt, A, B, n, h=1e-6):
    """Central differences (h = 1e-6) of the device forward area against the
    adjoint, coordinate by coordinate.  The area is piecewise smooth: it has
    a kink wherever a vertex crosses the other polygon's boundary, and on
    polygons of radius ~1e-3 a stencil of +-1e-6 straddles one for a few
    percent of the vertices.  A coordinate whose one-sided slopes disagree by
    more than 1e-3 of the gradient scale is such a case: there the adjoint
    must lie between the two one-sided slopes.  Everywhere else the central
    difference must match it to 1e-5 of the gradient scale (truncation
    h^2 f'''/6 ~ 1e-12 / r reaches ~1e-6 relative at r = 1e-3) plus half the
    one-sided disagreement (a milder kink inside the stencil)."""
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    idx = torch.arange(n, dtype=torch.int32, device="cuda")
    xa = LA.xy.clone().requires_grad_(True)
    prt.intersection_area(LA, LB, idx, idx, xa, LB.xy).sum().backward()
    g = xa.grad.cpu().numpy()
    scale = np.abs(g).max()
    x0 = LA.xy.clone()
    f0 = prt.intersection_area(LA, LB, idx, idx, x0, LB.xy).sum().item()
    smooth = kinked = 0
    for v in range(len(g)):
        for d in range(2):
            xp = x0.clone()
            xp[v, d] += h
            xm = x0.clone()
            xm[v, d] -= h
            fp = prt.intersection_area(LA, LB, idx, idx, xp, LB.xy).sum().item()
            fm = prt.intersection_area(LA, LB, idx, idx, xm, LB.xy).sum().item()
            dp, dm = (fp - f0) / h, (f0 - fm) / h
            if abs(dp - dm) <= 1e-3 * scale:
                smooth += 1
                assert abs((fp - fm) / (2 * h) - g[v, d]) <= 1e-5 * scale + 0.5 * abs(dp - dm), (v, d)
            else:
                kinked += 1
                lo, hi = min(dp, dm), max(dp, dm)
                assert lo - 1e-6 * scale <= g[v, d] <= hi + 1e-6 * scale, (v, d)
    return smooth, kinked


def test_adjoint_matches_finite_differences(cuda):
    import parlllelrtree_b200 as prt

    A, B = overlapping_pairs(6, seed=17)  # radius log-uniform 1e-3..1e-2
    smooth, kinked = _fd_check(prt, A, B, 6)
    assert smooth >= 0.9 * (smooth + kinked)


def test_adjoint_matches_finite_differences_large(cuda):
    """Radius 0.05: kinks inside a 1e-6 stencil become rare."""
    import parlllelrtree_b200 as prt

    n = 4
    rng = np.random.default_rng(29)
    c = rng.random((n, 2)) * 0.5 + 0.25
    r = np.full(n, 0.05)
    A = dg.star_layer(n, seed=30, nv_lo=16, nv_hi=40, centre_xy=c, radii=r)
    B = dg.star_layer(n, seed=31, nv_lo=16, nv_hi=40, centre_xy=c + 0.02, radii=r)
    smooth, kinked = _fd_check(prt, A, B, n)
    assert smooth >= 0.98 * (smooth + kinked)


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


def _degenerate_pairs():
    """Pairs where the boundary integral's crossings are not clean or the
    area is a sliver: identical polygons, a shared edge, a vertex on an edge,
    one polygon inside the other, disjoint polygons with overlapping boxes,
    a thin sliver, and a square against a square with a square hole."""
    sq = lambda x0, y0, s: np.array([[x0, y0], [x0 + s, y0], [x0 + s, y0 + s], [x0, y0 + s]], np.float64)
    tri = np.array([[0.5, 0.5], [0.52, 0.5], [0.51, 0.52]])
    ring_a, ring_b, hole_a, hole_b, rpa, rpb = [], [], [], [], [], []

    def add(a_rings, b_rings, a_holes=None, b_holes=None):
        ring_a.extend(a_rings)
        ring_b.extend(b_rings)
        hole_a.extend(a_holes or [0] * len(a_rings))
        hole_b.extend(b_holes or [0] * len(b_rings))
        rpa.append(len(a_rings))
        rpb.append(len(b_rings))

    s0 = sq(0.3, 0.3, 0.01)
    add([s0], [s0.copy()])                                          # identical
    add([s0], [sq(0.31, 0.3, 0.01)])                                # shared edge
    add([s0], [np.array([[0.305, 0.31], [0.32, 0.315], [0.31, 0.33]])])  # vertex on an edge
    add([s0], [sq(0.302, 0.302, 0.004)])                            # nested, no crossing
    add([tri], [np.array([[0.52, 0.505], [0.53, 0.505], [0.53, 0.52]])])  # boxes overlap, disjoint
    add([sq(0.4, 0.4, 0.01)], [sq(0.4 + 0.01 - 1e-13, 0.403, 0.01)])      # sliver 1e-13 wide
    add([sq(0.6, 0.6, 0.02)], [sq(0.605, 0.605, 0.02), sq(0.61, 0.61, 0.005)[::-1]], None, [0, 1])  # hole
    add([sq(0.7, 0.7, 0.01)], [sq(0.705, 0.695, 0.01)])             # two clean crossings
    A = dg.layer_from_rings(ring_a, hole_a, rpa)
    B = dg.layer_from_rings(ring_b, hole_b, rpb)
    return A, B


def test_forward_falls_back_to_gpc_on_degenerate_pairs(cuda):
    import parlllelrtree_b200 as prt
    from parlllelrtree_b200 import _lib

    A, B = _degenerate_pairs()
    n = len(A["poly_ring"]) - 1
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    idx = torch.arange(n, dtype=torch.int32, device="cuda")
    area = prt.intersection_area(LA, LB, idx, idx).cpu().numpy()
    for i in range(n):
        ref = oracle.result_area(oracle.gpc_clip(rings_of(A, i), rings_of(B, i), 1))
        assert abs(area[i] - ref) <= 1e-9 * abs(ref) + 1e-22, (i, area[i], ref)
    fb = __import__("ctypes").c_int64(-1)
    _lib.check(_lib.lib().prt_area_fwd_fallbacks(__import__("ctypes").byref(fb)))
    # identical, shared edge, vertex on edge, sliver at least go to GPC
    assert fb.value >= 4


def test_forward_differentiable_configuration(cuda):
    """The differentiable-area configuration's pairs (16-64 vertices, overlap
    guaranteed): the device forward against the oracle's GPC area on 20,000
    pairs, and most pairs on the boundary-integral path."""
    import ctypes

    import parlllelrtree_b200 as prt
    from parlllelrtree_b200 import _lib

    n = 20000
    Ad, Bd = dg.overlapping_pairs_device(n, seed=5)
    LA, LB = prt.Layer.from_dict(Ad), prt.Layer.from_dict(Bd)
    idx = torch.arange(n, dtype=torch.int32, device="cuda")
    area = prt.intersection_area(LA, LB, idx, idx).cpu().numpy()
    fb = ctypes.c_int64(-1)
    _lib.check(_lib.lib().prt_area_fwd_fallbacks(ctypes.byref(fb)))
    assert fb.value < 0.1 * n  # most pairs on the boundary-integral path
    A = {k: v.cpu().numpy() for k, v in Ad.items()}
    B = {k: v.cpu().numpy() for k, v in Bd.items()}
    for i in range(n):
        ref = oracle.result_area(oracle.gpc_clip(rings_of(A, i), rings_of(B, i), 1))
        assert abs(area[i] - ref) <= 1e-9 * abs(ref) + 1e-22, (i, area[i], ref)
