"""Map alignment by maximising polygon overlap (no reference counterpart).

Layer A is a map of parcels; layer B is the same parcels after an unknown
affine transform plus vertex noise.  ``fit_affine`` recovers the 6-parameter
affine that maps B back onto A by gradient ascent on the total intersection
area of the two layers.  Every step runs the whole differentiable path on
the device: the transformed B's MBRs, a bottom-up R-tree over A's MBRs, the
join, the GPC clip of every candidate pair (area forward) and the adjoint
kernel (area backward, prt_area_bwd), with torch autograd carrying the vertex
gradients to the 6 parameters.

The overlap objective is sharp: it peaks at the true transform with a width
of about one parcel, while a 2 degree rotation moves parcels at the edge of
the unit square by ~15 parcel widths.  The fit therefore runs a
coarse-to-fine pyramid: early stages keep every q-th parcel (q = stride**2 on
the parcel grid) and dilate each kept parcel by `stride` about its vertex
centroid, which scales the parcels and the basin of attraction together.
Dilation about a polygon's own centroid commutes with affine maps
(T(c + s (x - c)) = T(c) + s (T(x) - T(c))), so every stage has the same
optimum; the last stage uses all parcels at their own size.
"""
from __future__ import annotations

import math

import numpy as np
import torch

CENTRE = (0.5, 0.5)


def parcel_layers(n: int = 200_000, seed: int = 0, rot_deg: float = 2.0, scale: float = 0.01, shift: float = 0.005,
                  noise: float = 1e-4):
    """Layer A: n parcels on a jittered square grid over the unit square, each
    a hexagon or a quadrilateral (random, with per-vertex radial jitter),
    float64, CCW, disjoint.  Layer B: A under an affine transform (rotation
    uniform in +-rot_deg, isotropic scale 1 +- scale, translation uniform in
    +-shift, about the centre (0.5, 0.5)) plus Gaussian vertex noise (sigma
    `noise`).  Returns (A, B, T) with layer dicts (numpy) and T the 2x3 matrix
    of the applied transform (x_B = T[:, :2] (x_A - c) + c + T[:, 2])."""
    rng = np.random.default_rng(seed)
    g = int(math.ceil(math.sqrt(n)))
    h = 1.0 / g
    ij = np.stack(np.meshgrid(np.arange(g), np.arange(g), indexing="ij"), -1).reshape(-1, 2)[:n]
    cen = (ij + 0.5) * h + rng.uniform(-0.15, 0.15, size=(n, 2)) * h
    nv = np.where(rng.random(n) < 0.5, 6, 4).astype(np.int64)
    ring_vert = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(nv, out=ring_vert[1:])
    owner = np.repeat(np.arange(n), nv)
    k = np.arange(int(ring_vert[-1])) - ring_vert[owner]
    rot = rng.uniform(0.0, 2.0 * np.pi, size=n)
    ang = rot[owner] + 2.0 * np.pi * k / nv[owner]
    rad = 0.33 * h * rng.uniform(0.85, 1.0, size=len(k))
    xa = np.stack([cen[owner, 0] + rad * np.cos(ang), cen[owner, 1] + rad * np.sin(ang)], 1)
    phi = math.radians(rng.uniform(-rot_deg, rot_deg))
    s = 1.0 + rng.uniform(-scale, scale)
    t = rng.uniform(-shift, shift, size=2)
    L = s * np.array([[math.cos(phi), -math.sin(phi)], [math.sin(phi), math.cos(phi)]])
    c = np.array(CENTRE)
    xb = (xa - c) @ L.T + c + t + rng.normal(0.0, noise, size=xa.shape)
    base = {"poly_ring": np.arange(n + 1, dtype=np.int64), "ring_vert": ring_vert,
            "ring_hole": np.zeros(n, dtype=np.int32)}
    A = dict(base, xy=np.ascontiguousarray(xa))
    B = dict(base, xy=np.ascontiguousarray(xb))
    return A, B, np.concatenate([L, t[:, None]], 1)


def _apply(theta: torch.Tensor, xy: torch.Tensor) -> torch.Tensor:
    """x' = (I + [[a, b], [c, d]]) (x - centre) + centre + (tx, ty)."""
    c = torch.tensor(CENTRE, dtype=xy.dtype, device=xy.device)
    M = torch.eye(2, dtype=xy.dtype, device=xy.device) + theta[:4].reshape(2, 2)
    return (xy - c) @ M.T + c + theta[4:]


def _subset(layer: dict, keep: np.ndarray):
    """Ring CSR of the kept polygons (single-ring layers) and the vertex index."""
    rv = np.asarray(layer["ring_vert"])
    nv = rv[keep + 1] - rv[keep]
    ring_vert = np.zeros(len(keep) + 1, dtype=np.int64)
    np.cumsum(nv, out=ring_vert[1:])
    vidx = np.concatenate([np.arange(rv[i], rv[i + 1]) for i in keep]) if len(keep) < 4096 else \
        np.repeat(rv[keep], nv) + (np.arange(int(ring_vert[-1])) - np.repeat(ring_vert[:-1], nv))
    return ring_vert, vidx


def _dilate(xy: torch.Tensor, ring_vert: torch.Tensor, owner: torch.Tensor, s: float) -> torch.Tensor:
    if s == 1.0:
        return xy
    n = len(ring_vert) - 1
    cnt = (ring_vert[1:] - ring_vert[:-1]).to(xy.dtype)
    cen = torch.zeros((n, 2), dtype=xy.dtype, device=xy.device).index_add_(0, owner, xy) / cnt[:, None]
    return cen[owner] + s * (xy - cen[owner])


def fit_affine(A: dict, B: dict, steps: int = 200, stages=((30, 50), (10, 50), (3, 50), (1, 50)), lr: float = 0.1,
               fanout: int = 16, device: str = "cuda", log=None):
    """Recovers theta (6 parameters, see _apply) maximising the total overlap
    of A and theta(B) with `steps` Adam steps split over the pyramid `stages`
    ((stride, steps) pairs; stride 1 = all parcels at their own size).  The
    Adam learning rate is lr * stride * (grid spacing): a step moves the
    parcels by a fixed fraction of their (dilated) size; it decays over each
    stage (cosine).  Returns (theta as numpy, per-step records, device seconds
    per stage)."""
    import parlllelrtree_b200 as prt

    n = len(A["ring_vert"]) - 1
    g = int(math.ceil(math.sqrt(n)))
    ij = np.stack(np.meshgrid(np.arange(g), np.arange(g), indexing="ij"), -1).reshape(-1, 2)[:n]
    theta = torch.zeros(6, dtype=torch.float64, device=device, requires_grad=True)
    xa_all = torch.from_numpy(np.asarray(A["xy"])).to(device)
    xb_all = torch.from_numpy(np.asarray(B["xy"])).to(device)
    records, stage_s = [], []
    budget = steps
    for stride, k_steps in stages:
        k_steps = min(k_steps, budget)
        if k_steps <= 0:
            break
        budget -= k_steps
        keep = np.nonzero((ij[:, 0] % stride == 0) & (ij[:, 1] % stride == 0))[0] if stride > 1 else np.arange(n)
        ring_vert, vidx = _subset(A, keep)
        m = len(keep)
        rv = torch.from_numpy(ring_vert).to(device)
        owner = torch.repeat_interleave(torch.arange(m, device=device), rv[1:] - rv[:-1])
        vi = torch.from_numpy(vidx).to(device)
        xa = _dilate(xa_all[vi], rv, owner, float(stride))
        struct = {"poly_ring": np.arange(m + 1, dtype=np.int64), "ring_vert": ring_vert,
                  "ring_hole": np.zeros(m, dtype=np.int32)}
        LA = prt.Layer.from_dict(dict(struct, xy=xa))
        LB = prt.Layer.from_dict(dict(struct, xy=xb_all[vi]))
        qa = LA.mbr()  # A does not move: its MBRs are the join's queries
        ids = torch.arange(m, device=device, dtype=torch.int32)
        own_area = float(prt.intersection_area(LA, LA, ids, ids).sum())
        opt = torch.optim.Adam([theta], lr=lr * stride / g)
        sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=k_steps)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        stage_rec, stage_ov = [], []
        cap = None  # pair capacity: the previous step's count plus a margin
        for it in range(k_steps):
            opt.zero_grad()
            xb = _dilate(_apply(theta, xb_all[vi]), rv, owner, float(stride))
            LB.xy = xb.detach().contiguous()
            # every step: R-tree over the moved layer's MBRs, join, clip, adjoint
            tree = prt.build_bottomup(LB.mbr(), fanout=fanout)
            # one traversal when the capacity suffices (the join reports the
            # count and is re-run only when it does not)
            pairs = tree.join(qa, cap=cap)
            cap = len(pairs) + len(pairs) // 4 + 1024
            pb = tree.leaf_order()[pairs[:, 0].long()]
            pa = pairs[:, 1].contiguous()
            area = prt.intersection_area(LA, LB, pa, pb, base_xy=LA.xy, over_xy=xb)
            loss = -area.sum() / own_area
            loss.backward()
            opt.step()
            sched.step()
            # the overlap stays on the device (no host round trip per step)
            # unless a logger wants it now
            stage_rec.append({"stride": stride, "parcels": m, "pairs": int(len(pairs))})
            stage_ov.append(-loss.detach())
            if log:
                stage_rec[-1]["overlap"] = float(stage_ov[-1])
                log(stage_rec[-1])
        ev1.record()
        ev1.synchronize()
        stage_s.append(ev0.elapsed_time(ev1) * 1e-3)
        for r, v in zip(stage_rec, torch.stack(stage_ov).cpu().tolist()):
            r["overlap"] = v
        records.extend(stage_rec)
    return theta.detach().cpu().numpy(), records, stage_s


def recovery_error(theta: np.ndarray, T: np.ndarray) -> float:
    """Largest displacement over the unit square of theta(T(x)) - x: how far
    the fitted transform is from inverting the applied one."""
    c = np.array(CENTRE)
    M = np.eye(2) + theta[:4].reshape(2, 2)
    corners = np.array([[0, 0], [1, 0], [0, 1], [1, 1]], dtype=np.float64)
    xb = (corners - c) @ T[:, :2].T + c + T[:, 2]
    back = (xb - c) @ M.T + c + theta[4:]
    return float(np.abs(back - corners).max())
