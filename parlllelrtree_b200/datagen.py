"""Seeded synthetic inputs in the shapes of the benchmark configurations.

The reference ships no data (its programs read ``data/Rect1024.txt`` and two
polygon files that are not part of it), so every workload here is generated:

* ``star_layer``      star-shaped polygons, ring CSR (small overlay, batched
                      overlay, differentiable-area workloads);
* ``mixture_boxes``   axis-aligned float32 boxes around a 64-Gaussian mixture
                      (R-tree build and query workload);
* ``window_queries``  square query windows;
* ``quantise``        the integer form the reference consumes
                      (``round(v * 1e6)`` as int64).

A polygon layer is a dict of numpy arrays:
  ``poly_ring``  int64 [P+1]  ring offsets per polygon
  ``ring_vert``  int64 [R+1]  vertex offsets per ring
  ``ring_hole``  int32 [R]    1 for a hole ring
  ``xy``         float64 [V, 2]
Single-ring polygons map one-to-one onto the reference's per-polygon CSR
(``num[]``, ``prefix[]``, ``vertex[]``, ``hole[]``; vector_map_overlay_gpc_kernel.cu:792-863).
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "star_layer",
    "mixture_centres",
    "mixture_boxes",
    "window_queries",
    "quantise",
    "layer_bboxes",
    "layer_from_rings",
    "star_layer_device",
    "mixture_means",
]


def mixture_means(k: int = 64, seed: int = 0) -> np.ndarray:
    """The mixture's ``k`` means, uniform in the unit square; one fixed set
    (seed 0) shared by every layer and box set so that layers overlap."""
    return np.random.default_rng(10_000 + seed).random((k, 2))


def mixture_centres(rng: np.random.Generator, n: int, k: int = 64, sigma: float = 0.02) -> np.ndarray:
    """``n`` points from a mixture of ``k`` isotropic Gaussians (the fixed
    means of ``mixture_means``), clipped to the unit square."""
    means = mixture_means(k)
    comp = rng.integers(0, k, size=n)
    pts = means[comp] + rng.normal(0.0, sigma, size=(n, 2))
    np.clip(pts, 0.0, 1.0, out=pts)
    return pts


def mixture_boxes(n: int, seed: int = 0, k: int = 64, sigma: float = 0.02,
                  mean_side: float = 1e-4) -> np.ndarray:
    """float32 boxes [n, 4] as (x1, y1, x2, y2): centres from the mixture,
    widths and heights exponential with mean ``mean_side``."""
    rng = np.random.default_rng(seed)
    c = mixture_centres(rng, n, k, sigma)
    wh = rng.exponential(mean_side, size=(n, 2))
    out = np.empty((n, 4), dtype=np.float32)
    out[:, 0] = c[:, 0] - 0.5 * wh[:, 0]
    out[:, 1] = c[:, 1] - 0.5 * wh[:, 1]
    out[:, 2] = c[:, 0] + 0.5 * wh[:, 0]
    out[:, 3] = c[:, 1] + 0.5 * wh[:, 1]
    # float32 rounding can invert a tiny box; keep x1 <= x2, y1 <= y2
    np.minimum(out[:, 0], out[:, 2], out=out[:, 0])
    np.minimum(out[:, 1], out[:, 3], out=out[:, 1])
    return out


def window_queries(n: int, seed: int = 1, side_lo: float = 1e-4, side_hi: float = 1e-2) -> np.ndarray:
    """float32 square windows [n, 4]: centres uniform, side uniform."""
    rng = np.random.default_rng(seed)
    c = rng.random((n, 2))
    s = rng.uniform(side_lo, side_hi, size=n)
    out = np.empty((n, 4), dtype=np.float32)
    out[:, 0] = c[:, 0] - 0.5 * s
    out[:, 1] = c[:, 1] - 0.5 * s
    out[:, 2] = c[:, 0] + 0.5 * s
    out[:, 3] = c[:, 1] + 0.5 * s
    return out


def quantise(boxes: np.ndarray, scale: float = 1e6) -> np.ndarray:
    """int64 boxes ``round(v * scale)``, the integer grid the reference's
    R-tree programs read (BotomUp-rtree.cu:679-681)."""
    return np.rint(np.asarray(boxes, dtype=np.float64) * scale).astype(np.int64)


def _lobe_weight(nv):
    """Weight of the smooth radial profile: 0 up to 32 vertices (radii
    r * U(0.5, 1) per vertex, the small star configuration), growing towards 1
    for large rings, whose radius then follows a few smooth lobes plus a small
    per-vertex jitter.  Independent per-vertex jitter on thousands of vertices
    would give spiky rings that every scanline crosses hundreds of times."""
    nv = np.asarray(nv, dtype=np.float64)
    return np.clip((nv - 32.0) / np.maximum(nv, 1.0), 0.0, 1.0)


def _star_rings(rng, centres, radii, nverts):
    """CCW star rings: jittered sorted angles; radius r * ((1 - w) U(0.5, 1)
    + w (0.75 + 0.25 L(theta))) with L a sum of 5 random sine lobes scaled to
    [-1, 1] and w = _lobe_weight(n), so every vertex lies between 0.5 r and r."""
    nv = np.asarray(nverts, dtype=np.int64)
    total = int(nv.sum())
    ring_vert = np.zeros(len(nv) + 1, dtype=np.int64)
    np.cumsum(nv, out=ring_vert[1:])
    owner = np.repeat(np.arange(len(nv)), nv)
    k = np.arange(total, dtype=np.int64) - ring_vert[owner]
    step = 2.0 * np.pi / nv[owner]
    # jitter inside each vertex's own angular slot keeps the angles sorted
    theta = (k + 0.1 + 0.8 * rng.random(total)) * step
    jit = rng.uniform(0.5, 1.0, size=total)
    amp = rng.random((len(nv), 5))
    amp /= amp.sum(axis=1, keepdims=True)
    phase = rng.uniform(0.0, 2.0 * np.pi, size=(len(nv), 5))
    lobe = np.zeros(total)
    for m in range(5):
        lobe += amp[owner, m] * np.sin((m + 1) * theta + phase[owner, m])
    w = _lobe_weight(nv)[owner]
    rad = radii[owner] * ((1.0 - w) * jit + w * (0.75 + 0.25 * lobe))
    xy = np.empty((total, 2), dtype=np.float64)
    xy[:, 0] = centres[owner, 0] + rad * np.cos(theta)
    xy[:, 1] = centres[owner, 1] + rad * np.sin(theta)
    return ring_vert, xy


def star_layer(n: int, seed: int, nv_lo: int = 8, nv_hi: int = 32,
               r_lo: float = 1e-3, r_hi: float = 1e-2, centres: str = "uniform",
               zipf: float | None = None, hole_frac: float = 0.0,
               centre_xy: np.ndarray | None = None, radii: np.ndarray | None = None) -> dict:
    """A layer of ``n`` star polygons (float64, outer rings CCW).

    ``nverts`` is uniform in [nv_lo, nv_hi], or ``clip(zipf(s), nv_lo, nv_hi)``
    when ``zipf`` is given.  A fraction ``hole_frac`` of the polygons gets 1-3
    clockwise hole rings (small triangles/quads) inside the disk of radius
    0.5 r, which the star always contains.
    """
    rng = np.random.default_rng(seed)
    if zipf is not None:
        nverts = np.clip(rng.zipf(zipf, size=n), nv_lo, nv_hi).astype(np.int64)
    else:
        nverts = rng.integers(nv_lo, nv_hi + 1, size=n).astype(np.int64)
    if radii is None:
        radii = np.exp(rng.uniform(np.log(r_lo), np.log(r_hi), size=n))
    if centre_xy is None:
        if centres == "mixture":
            centre_xy = mixture_centres(rng, n)
        else:
            centre_xy = rng.random((n, 2))
    outer_vert, outer_xy = _star_rings(rng, centre_xy, radii, nverts)
    if hole_frac <= 0.0:
        return {
            "poly_ring": np.arange(n + 1, dtype=np.int64),
            "ring_vert": outer_vert,
            "ring_hole": np.zeros(n, dtype=np.int32),
            "xy": outer_xy,
        }
    has_holes = rng.random(n) < hole_frac
    nholes = np.where(has_holes, rng.integers(1, 4, size=n), 0).astype(np.int64)
    return _with_holes(rng, outer_vert, outer_xy, nverts, nholes, centre_xy, radii)


def _with_holes(rng, outer_vert, outer_xy, nverts, nholes, centre_xy, radii) -> dict:
    """Interleaves 1-3 clockwise hole rings (3-4 vertices each) after each
    polygon's outer ring.  Hole j of h sits in its own angular sector, at radii
    below the star's guaranteed inner radius: consecutive outer vertices are
    at radius >= 0.5 r and at most 1.8 * 2 pi / n apart in angle, so the outer
    boundary stays beyond 0.5 r cos(1.8 pi / n)."""
    n = len(nverts)
    rings_per_poly = 1 + nholes
    poly_ring = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(rings_per_poly, out=poly_ring[1:])
    n_rings = int(poly_ring[-1])
    ring_poly = np.repeat(np.arange(n), rings_per_poly)
    ring_j = np.arange(n_rings) - poly_ring[ring_poly]          # 0 = outer, k >= 1 = hole k-1
    is_hole = ring_j > 0
    hole_m = rng.integers(3, 5, size=n_rings)                   # vertices of each hole ring
    ring_nv = np.where(is_hole, hole_m, nverts[ring_poly])
    ring_vert = np.zeros(n_rings + 1, dtype=np.int64)
    np.cumsum(ring_nv, out=ring_vert[1:])
    xy = np.empty((int(ring_vert[-1]), 2), dtype=np.float64)
    # outer rings: move each polygon's block of vertices to its ring's slot
    outer_ring = poly_ring[:-1]
    owner = np.repeat(np.arange(n), nverts)
    k = np.arange(len(outer_xy)) - outer_vert[owner]
    xy[ring_vert[outer_ring][owner] + k] = outer_xy
    # hole rings
    hr = np.nonzero(is_hole)[0]
    if len(hr):
        hp = ring_poly[hr]
        h = nholes[hp]
        j = ring_j[hr] - 1
        m = ring_nv[hr]
        hv_owner = np.repeat(np.arange(len(hr)), m)
        hk = np.arange(int(m.sum())) - np.repeat(np.cumsum(m) - m, m)
        # each hole spans at most 0.9 pi of its sector, so no two consecutive
        # hole vertices are more than pi apart in angle (a simple CW ring)
        sector = 2.0 * np.pi / h[hv_owner]
        span = np.minimum(sector, 0.9 * np.pi)
        a0 = sector * j[hv_owner] + 0.5 * (sector - span)
        # angles inside the sector, descending within each ring (clockwise):
        # sort by (ring, -value); rings occupy contiguous slots, so the sorted
        # values land on their own ring's vertices
        raw = rng.random(len(hk))
        frac = raw[np.lexsort((-raw, hv_owner))]
        ang = a0 + span * (0.15 + 0.7 * frac)
        nv_out = nverts[hp][hv_owner]
        rin = 0.5 * np.cos(np.minimum(1.8 * np.pi / np.maximum(nv_out, 4), 1.45))
        # one radius per hole: its vertices lie on a circle arc in descending
        # angle, a convex clockwise ring
        rr = (radii[hp] * rng.uniform(0.3, 0.9, size=len(hr)))[hv_owner] * rin
        xy[ring_vert[hr][hv_owner] + hk, 0] = centre_xy[hp][hv_owner, 0] + rr * np.cos(ang)
        xy[ring_vert[hr][hv_owner] + hk, 1] = centre_xy[hp][hv_owner, 1] + rr * np.sin(ang)
    return {
        "poly_ring": poly_ring,
        "ring_vert": ring_vert,
        "ring_hole": is_hole.astype(np.int32),
        "xy": xy,
    }


def layer_from_rings(rings, holes, rings_per_poly) -> dict:
    """Builds a layer dict from a list of [k, 2] rings."""
    poly_ring = np.zeros(len(rings_per_poly) + 1, dtype=np.int64)
    np.cumsum(np.asarray(rings_per_poly, dtype=np.int64), out=poly_ring[1:])
    nv = np.array([len(r) for r in rings], dtype=np.int64)
    ring_vert = np.zeros(len(rings) + 1, dtype=np.int64)
    np.cumsum(nv, out=ring_vert[1:])
    xy = np.concatenate([np.asarray(r, dtype=np.float64) for r in rings], axis=0) if rings else np.zeros((0, 2))
    return {
        "poly_ring": poly_ring,
        "ring_vert": ring_vert,
        "ring_hole": np.asarray(holes, dtype=np.int32),
        "xy": np.ascontiguousarray(xy),
    }


def layer_bboxes(layer: dict) -> np.ndarray:
    """float64 [P, 4] (xmin, ymin, xmax, ymax) of each polygon."""
    pr, rv, xy = layer["poly_ring"], layer["ring_vert"], layer["xy"]
    npoly = len(pr) - 1
    vstart = rv[pr[:-1]]
    vend = rv[pr[1:]]
    out = np.empty((npoly, 4), dtype=np.float64)
    out[:, 0] = np.minimum.reduceat(xy[:, 0], vstart)
    out[:, 1] = np.minimum.reduceat(xy[:, 1], vstart)
    out[:, 2] = np.maximum.reduceat(xy[:, 0], vstart)
    out[:, 3] = np.maximum.reduceat(xy[:, 1], vstart)
    assert np.all(vend > vstart)
    return out


def star_layer_device(n: int, seed: int, nv_lo: int = 4, nv_hi: int = 4096, r_lo: float = 1e-3,
                      r_hi: float = 1e-2, zipf: float | None = 1.2, hole_frac: float = 0.05,
                      centres: str = "mixture", device: str = "cuda", chunk: int = 1 << 16,
                      centre_xy: np.ndarray | None = None, radii: np.ndarray | None = None) -> dict:
    """``star_layer`` for large layers: the per-polygon draws (vertex counts,
    radii, centres, holes, lobes) come from numpy, the per-vertex draws and
    trigonometry run in torch on ``device``, ``chunk`` polygons at a time so
    the temporaries stay a few GB for any layer size.  Returns the same dict
    with torch tensors on the device.  Same distribution as ``star_layer``,
    not the same numbers."""
    import torch

    rng = np.random.default_rng(seed)
    if zipf is not None:
        nverts = np.clip(rng.zipf(zipf, size=n), nv_lo, nv_hi).astype(np.int64)
    else:
        nverts = rng.integers(nv_lo, nv_hi + 1, size=n).astype(np.int64)
    r_draw = np.exp(rng.uniform(np.log(r_lo), np.log(r_hi), size=n))
    radii = r_draw if radii is None else np.asarray(radii, dtype=np.float64)
    c_draw = mixture_centres(rng, n) if centres == "mixture" else rng.random((n, 2))
    centre_xy = c_draw if centre_xy is None else np.asarray(centre_xy, dtype=np.float64)
    has_holes = rng.random(n) < hole_frac
    nholes = np.where(has_holes, rng.integers(1, 4, size=n), 0).astype(np.int64)
    amp = rng.random((n, 5))
    amp /= amp.sum(axis=1, keepdims=True)
    phase = rng.uniform(0.0, 2.0 * np.pi, size=(n, 5))
    hole_r = rng.uniform(0.3, 0.9, size=n)
    # ring CSR on the host (one outer ring + holes per polygon)
    rings_per_poly = 1 + nholes
    poly_ring = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(rings_per_poly, out=poly_ring[1:])
    n_rings = int(poly_ring[-1])
    ring_poly = np.repeat(np.arange(n), rings_per_poly)
    ring_j = np.arange(n_rings) - poly_ring[ring_poly]
    hole_m = np.random.default_rng(seed + 7919).integers(3, 5, size=n_rings)
    ring_nv = np.where(ring_j > 0, hole_m, nverts[ring_poly])
    ring_vert = np.zeros(n_rings + 1, dtype=np.int64)
    np.cumsum(ring_nv, out=ring_vert[1:])
    total = int(ring_vert[-1])
    dev = torch.device(device)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    xy = torch.empty((total, 2), dtype=torch.float64, device=dev)
    lobe_w = _lobe_weight(nverts)
    for c0 in range(0, n, chunk):
        c1 = min(n, c0 + chunk)
        r0, r1 = int(poly_ring[c0]), int(poly_ring[c1])
        v0, v1 = int(ring_vert[r0]), int(ring_vert[r1])
        t = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        rnv = t(ring_nv[r0:r1])
        rpoly = t(ring_poly[r0:r1] - c0)
        rj = t(ring_j[r0:r1])
        rv = t(ring_vert[r0:r1] - v0)
        m_v = v1 - v0
        owner = torch.repeat_interleave(torch.arange(r1 - r0, device=dev), rnv)
        k = torch.arange(m_v, device=dev) - rv[owner]
        p = rpoly[owner]
        hole_v = rj[owner] > 0
        nv_p = t(nverts[c0:c1])[p].to(torch.float64)
        u = torch.rand(m_v, generator=g, device=dev, dtype=torch.float64)
        jit = 0.5 + 0.5 * torch.rand(m_v, generator=g, device=dev, dtype=torch.float64)
        # outer rings: jittered angle slots, CCW, radius r * ((1-w) jitter + w lobes)
        theta = (k.to(torch.float64) + 0.1 + 0.8 * u) * (2.0 * np.pi / nv_p)
        A = t(amp[c0:c1])[p]
        P = t(phase[c0:c1])[p]
        lobe = torch.zeros(m_v, dtype=torch.float64, device=dev)
        for mm in range(5):
            lobe += A[:, mm] * torch.sin((mm + 1) * theta + P[:, mm])
        del A, P
        w = t(lobe_w[c0:c1])[p]
        rad_p = t(radii[c0:c1])[p]
        rr = rad_p * ((1.0 - w) * jit + w * (0.75 + 0.25 * lobe))
        del lobe, w, jit, u
        # holes: on a circle arc of their sector, descending angle (CW)
        h = t(nholes[c0:c1])[p].clamp(min=1).to(torch.float64)
        sector = 2.0 * np.pi / h
        span = torch.clamp(sector, max=0.9 * np.pi)
        a0 = sector * (rj[owner] - 1).clamp(min=0).to(torch.float64) + 0.5 * (sector - span)
        m = rnv[owner].to(torch.float64)
        frac = (m - 1 - k.to(torch.float64) + 0.5) / m
        hang = a0 + span * (0.15 + 0.7 * frac)
        rin = 0.5 * torch.cos(torch.clamp(1.8 * np.pi / nv_p.clamp(min=4), max=1.45))
        hr = rad_p * t(hole_r[c0:c1])[p] * rin
        ang = torch.where(hole_v, hang, theta)
        r_all = torch.where(hole_v, hr, rr)
        cen = t(centre_xy[c0:c1])[p]
        xy[v0:v1, 0] = cen[:, 0] + r_all * torch.cos(ang)
        xy[v0:v1, 1] = cen[:, 1] + r_all * torch.sin(ang)
        del owner, k, p, hole_v, nv_p, theta, rr, h, sector, span, a0, m, frac, hang, rin, hr, ang, r_all, cen
    return {"poly_ring": torch.from_numpy(poly_ring).to(dev), "ring_vert": torch.from_numpy(ring_vert).to(dev),
            "ring_hole": torch.from_numpy((ring_j > 0).astype(np.int32)).to(dev), "xy": xy}


def overlapping_pairs_device(n: int, seed: int = 0, nv_lo: int = 16, nv_hi: int = 64, r_lo: float = 1e-3,
                             r_hi: float = 1e-2, device: str = "cuda"):
    """The differentiable-area configuration: n pairs (A_i, B_i) of star
    polygons with nv_lo..nv_hi vertices (uniform), float64, radius log-uniform
    r_lo..r_hi, centres uniform in the unit square, no holes; B_i's centre is
    A_i's moved by at most 0.5 r_A, inside the disk of radius 0.5 r_A that
    every star contains, so each pair overlaps.  B_i's radius is r_A times
    U(0.5, 1.5).  Returns the two layer dicts (torch, on ``device``); pair i
    is (i, i)."""
    rng = np.random.default_rng(seed + 424242)
    cen = rng.random((n, 2))
    ra = np.exp(rng.uniform(np.log(r_lo), np.log(r_hi), size=n))
    ang = rng.uniform(0.0, 2.0 * np.pi, size=n)
    dist = 0.5 * ra * np.sqrt(rng.random(n))
    cb = cen + np.stack([dist * np.cos(ang), dist * np.sin(ang)], 1)
    rb = ra * rng.uniform(0.5, 1.5, size=n)
    A = star_layer_device(n, seed, nv_lo=nv_lo, nv_hi=nv_hi, zipf=None, hole_frac=0.0, device=device,
                          centre_xy=cen, radii=ra)
    B = star_layer_device(n, seed + 1, nv_lo=nv_lo, nv_hi=nv_hi, zipf=None, hole_frac=0.0, device=device,
                          centre_xy=cb, radii=rb)
    return A, B
