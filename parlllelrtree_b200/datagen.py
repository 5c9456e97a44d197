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
]


def mixture_centres(rng: np.random.Generator, n: int, k: int = 64, sigma: float = 0.02) -> np.ndarray:
    """``n`` points from a mixture of ``k`` isotropic Gaussians with means
    uniform in the unit square, clipped to the square."""
    means = rng.random((k, 2))
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


def _star_rings(rng, centres, radii, nverts):
    """CCW star rings: jittered sorted angles, radii r * U(0.5, 1)."""
    nv = np.asarray(nverts, dtype=np.int64)
    total = int(nv.sum())
    ring_vert = np.zeros(len(nv) + 1, dtype=np.int64)
    np.cumsum(nv, out=ring_vert[1:])
    owner = np.repeat(np.arange(len(nv)), nv)
    k = np.arange(total, dtype=np.int64) - ring_vert[owner]
    step = 2.0 * np.pi / nv[owner]
    # jitter inside each vertex's own angular slot keeps the angles sorted
    theta = (k + 0.1 + 0.8 * rng.random(total)) * step
    rad = radii[owner] * rng.uniform(0.5, 1.0, size=total)
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
    nholes = np.where(has_holes, rng.integers(1, 4, size=n), 0)
    rings, holes = [], []
    for p in range(n):
        rings.append(outer_xy[outer_vert[p]:outer_vert[p + 1]])
        holes.append(0)
        h = int(nholes[p])
        for j in range(h):
            # hole j sits in its own angular sector of the inner disk
            a0 = 2.0 * np.pi * j / h
            span = 2.0 * np.pi / h
            m = int(rng.integers(3, 5))
            ang = a0 + span * (0.15 + 0.7 * np.sort(rng.random(m)))[::-1]  # CW
            rr = radii[p] * rng.uniform(0.15, 0.45, size=m)
            ring = np.stack([centre_xy[p, 0] + rr * np.cos(ang),
                             centre_xy[p, 1] + rr * np.sin(ang)], axis=1)
            rings.append(ring)
            holes.append(1)
    counts = [1 + int(nholes[p]) for p in range(n)]
    return layer_from_rings(rings, holes, counts)


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
