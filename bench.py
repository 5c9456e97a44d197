#!/usr/bin/env python
"""Benchmark of the R-tree build / join / overlay path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the R-tree build-and-query configuration): 10M axis-aligned float32
boxes around a 64-Gaussian mixture (sigma 0.02), widths/heights exponential
with mean 1e-4, seed = rank.  A step = one bottom-up bulk load at fanout 16
(MORTON32 keys of box centres -> onesweep radix sort -> level packing) of the
whole 10M-box array; `value` = boxes of all ranks / max-over-ranks device time
per step, in Mboxes/s.  Inputs (160 MB) are larger than the 126 MB L2 and L2
is also flushed (256 MB write) between timed steps.

Reported beside it (same JSON line, `secondary`): the other builds of that
configuration (bottom-up/top-down at fanout 16 and 32); 1M window queries
(side uniform 1e-4..1e-2) joined against the fanout-16 tree, with the join's
HBM roofline; the batched uneven overlay at its full size (2 x 1M stars, ~4M
candidate pairs: batched schedule, graph pipeline, plain schedule on a
labelled strided subset, 400 pairs checked bit for bit against the oracle);
the differentiable-area configuration (1M pairs, forward and adjoint, the
adjoint's HBM roofline); the map-alignment loop (200k parcels x 200 steps);
and the small overlay configuration (2 x 10,000 stars, 8-32 vertices, radius
log-uniform 1e-3..1e-2) clipped with the plain and the batched schedule.

--impl reference times the reference's own CPU build (BotomUp-rtree.cu:776-833,
qsort + packing, built from its sources into oracle/_ref) on the same boxes
quantised to int64 (round(v * 1e6)), a bounded sample per step.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BOXES = 10_000_000
N_WINDOWS = 1_000_000
FANOUT = 16
METRIC = "overlay pairs/s & R-tree build Mboxes/s on 1 B200; batched+grad vs plain"
WORKLOAD = "rtree_build_10M_f32_mixture64_bottomup_f16_morton32"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-extras", action="store_true", help="skip the secondary measurements")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t_end = time.perf_counter() + 5.0
            while not self.lines and time.perf_counter() < t_end:  # sampler running before timing starts
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t0 = time.perf_counter()
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append((time.perf_counter(), ln.strip()))

    def __exit__(self, *a):
        self.t1 = time.perf_counter()
        if self.proc:
            time.sleep(0.06)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # samples taken while the timed steps ran (plus one sampling period)
        for ts, ln in self.lines:
            if not (self.t0 <= ts <= self.t1 + 0.06):
                continue
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The largest x over all ranks (device "cpu" under the gloo backend)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def time_steps(fn, steps, warmup, flush, world, before=None, after=None):
    """Runs warmup + steps; returns per-step device ms (CUDA events on the
    current stream, L2 flushed between steps) and the bracketed wall time."""
    import torch

    for _ in range(warmup):
        r = fn()
        if after:
            after(r)
    torch.cuda.synchronize()
    ms = []
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        flush()
        if before:
            before()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        r = fn()
        b.record()
        b.synchronize()
        ms.append(a.elapsed_time(b))
        if after:
            after(r)
        del r  # the step's outputs are released outside the timed window
    barrier(world)
    torch.cuda.synchronize()
    return ms, time.perf_counter() - t0


def reference_cpu_build(rects: np.ndarray) -> float:
    """The reference's CPU bottom-up build (qsort + packing) on rects; returns ms."""
    import oracle

    res = oracle.ref_bu_run(rects, FANOUT, query=False)
    return float(res["ms"][0])


def _ref_worker(job):
    """One host process of the reference arm: the reference's CPU build on
    its own sample (same distribution, seed per worker), warm-up + timed
    steps; returns the step times in ms."""
    w, sample, steps, warmup = job
    from parlllelrtree_b200 import datagen as dg

    rects = dg.quantise(dg.mixture_boxes(sample, seed=1000 + w))
    for _ in range(warmup):
        reference_cpu_build(rects)
    return [reference_cpu_build(rects) for _ in range(steps)]


def run_reference(args):
    """The reference's own CPU bottom-up build (BotomUp-rtree.cu:776-833,
    built from its sources into oracle/_ref), one process per host core (the
    code is single-threaded), each on its own 1M-box sample of the
    configuration per step; value = boxes of all processes / mean step time."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp

    import oracle

    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference's CPU code) is not built"}))
        return
    sample = 1_000_000
    cores = os.cpu_count() or 1
    steps = max(1, min(args.steps, 20))
    with mp.get_context("spawn").Pool(cores) as pool:
        times = pool.map(_ref_worker, [(w, sample, steps, max(1, min(args.warmup, 3))) for w in range(cores)])
    mean = float(np.mean([np.mean(t) for t in times]))
    v = sum(sample / (np.mean(t) * 1e-3) for t in times) / 1e6
    print(json.dumps({
        "metric": METRIC, "impl": "reference", "value": v, "unit": "Mboxes/s", "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": mean, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_boxes": N_BOXES, "fanout": FANOUT,
                   "sample_boxes_per_step_per_process": sample, "processes": cores,
                   "coords": "int64 round(v*1e6)"},
        "cpu_baseline": {"value": v, "unit": "Mboxes/s", "cores": cores, "kind": "reference",
                         "sample": f"{cores} processes x {sample} boxes per step (1M-box samples of the "
                                   "configuration), qsort + packing (BotomUp-rtree.cu:776-833) as written"},
        "e2e": {"value": v, "unit": "Mboxes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import parlllelrtree_b200 as prt
    from parlllelrtree_b200 import _lib
    from parlllelrtree_b200 import datagen as dg

    boxes_h = dg.mixture_boxes(N_BOXES, seed=rank)
    boxes = torch.from_numpy(boxes_h).cuda()
    boxes_pin = torch.from_numpy(boxes_h).pin_memory()
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def flush():
        flush_buf.zero_()

    def step():
        return prt.build_bottomup(boxes, fanout=FANOUT, key_mode="morton32")

    def drop(t):
        del t

    # warm-up, then one untimed step with every launch timed (kernel shares
    # and the dominant kernel), then the timed steps with launches counted and
    # only the dominant kernel bracketed by events (on its launching stream)
    _lib.profile_enable(0)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    _lib.profile_reset()
    _lib.profile_enable(1)
    flush()
    step()
    torch.cuda.synchronize()
    _lib.profile_enable(0)
    shares = _lib.profile_read()
    _lib.profile_reset()
    dom_name = max(shares.items(), key=lambda kv: kv[1][0])[0]
    _lib.profile_focus(dom_name)
    _lib.profile_enable(2)
    with ClockSampler(local) as clk:
        ms, wall = time_steps(step, args.steps, 0, flush, world)
    _lib.profile_enable(0)
    prof = _lib.profile_read()
    _lib.profile_reset()
    mean_ms = float(np.mean(ms))
    t_max = max_over_ranks(mean_ms, world)
    value = N_BOXES * world / (t_max * 1e-3) / 1e6

    # end to end through the public API: pinned host boxes -> device -> build
    # -> top level read back
    def step_e2e():
        d = boxes_pin.to("cuda", non_blocking=True)
        t = prt.build_bottomup(d, fanout=FANOUT, key_mode="morton32")
        top = t.level_mbr(t.levels - 1)
        return t, top

    ms_e2e, _ = time_steps(step_e2e, args.steps, 1, flush, world)
    t_e2e = max_over_ranks(float(np.mean(ms_e2e)), world)
    e2e = N_BOXES * world / (t_e2e * 1e-3) / 1e6
    top_levels = prt.build_bottomup(boxes, fanout=FANOUT).level_counts[-1]

    # roofline of the dominant kernel, timed live in the timed steps
    total = sum(v[0] for v in shares.values()) or 1.0
    peak, peak_kind = hbm_peak()
    dom_ms, dom_n = prof.get(dom_name, (0.0, 0))
    per_launch_ms = dom_ms / max(dom_n, 1)
    algo_bytes = {
        # one radix pass moves every (key, value): read 4 + 4 B, write 4 + 4 B
        "onesweep_pass": 16 * N_BOXES,
        # gather of a 16 B box by index + 4 B index read + 16 B entry + 4 B id
        # writes
        "pack_leaf": 40 * N_BOXES,
        "morton32": 24 * N_BOXES,
        "hist": 4 * N_BOXES,
    }.get(dom_name)
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic_per_launch.json")
    if os.path.exists(tf):
        try:
            with open(tf) as f:
                traffic = json.load(f).get(f"{WORKLOAD}:{dom_name}")
        except Exception:
            traffic = None
    roofline = None
    if algo_bytes:
        achieved = algo_bytes / (per_launch_ms * 1e-3) / 1e9
        roofline = {"kernel": dom_name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                    "algorithmic_bytes_per_launch": algo_bytes, "launch_ms": per_launch_ms}

    out = {
        "metric": METRIC, "value": value, "unit": "Mboxes/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_boxes_per_gpu": N_BOXES, "fanout": FANOUT, "key_mode": "morton32",
                   "l2": "inputs (160 MB) larger than L2; 256 MB L2 flush between timed steps",
                   "parallelism": f"replicas x{world} (independent box sets, no collective)"},
        "e2e": {"value": e2e, "unit": "Mboxes/s", "h2d_bytes_per_step": int(boxes_h.nbytes),
                "d2h_bytes_per_step": int(top_levels * 32)},
        "gpu_launches": int(sum(v[1] for v in prof.values())),
        "kernel_share": {k: round(v[0] / total, 4) for k, v in sorted(shares.items(), key=lambda kv: -kv[1][0])},
        "roofline": roofline,
        "clocks": clk.summary(),
        "wall_s_timed": wall,
    }

    if rank == 0 and world == 1 and not args.no_extras:
        out["secondary"] = secondary(prt, boxes, flush, world)
        # CPU baseline: the reference's own CPU build on a bounded sample
        sample = N_BOXES
        rects = dg.quantise(boxes_h[:sample])
        try:
            cms = reference_cpu_build(rects)
            out["cpu_baseline"] = {"value": sample / (cms * 1e-3) / 1e6, "unit": "Mboxes/s", "cores": 1,
                                   "kind": "reference",
                                   "sample": f"all {sample} boxes quantised to int64, one qsort + packing pass "
                                             "(BotomUp-rtree.cu:776-833) as written"}
        except Exception as e:  # oracle/_ref missing
            out["cpu_baseline"] = {"value": None, "unit": "Mboxes/s", "cores": 1, "kind": "reference",
                                   "sample": f"unavailable: {e}"}
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def secondary(prt, boxes, flush, world):
    """Other builds of the configuration, the 1M-window join and the small
    overlay configuration, each timed with CUDA events (median of 5)."""
    import torch
    from parlllelrtree_b200 import datagen as dg

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            flush()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            r = fn()
            b.record()
            b.synchronize()
            ms.append(a.elapsed_time(b))
            del r
        return float(np.median(ms))

    res = {}
    n = len(boxes)
    for name, fn in (("bottomup_f16", lambda: prt.build_bottomup(boxes, 16)),
                     ("bottomup_f32", lambda: prt.build_bottomup(boxes, 32)),
                     ("topdown_f16", lambda: prt.build_topdown(boxes, 16)),
                     ("topdown_f32", lambda: prt.build_topdown(boxes, 32))):
        ms = timed(fn)
        res[f"build_{name}_mboxes_s"] = n / (ms * 1e-3) / 1e6
    tree = prt.build_bottomup(boxes, 16)
    win = torch.from_numpy(dg.window_queries(N_WINDOWS, seed=1)).cuda()
    npairs = len(tree.join(win))
    cap = npairs + 1024
    out = torch.empty((cap, 2), dtype=torch.int32, device="cuda")
    import ctypes as C

    from parlllelrtree_b200 import _lib

    cnt = C.c_int64(0)

    def join():
        _lib.check(_lib.lib().prt_join(tree._h, C.c_void_p(win.data_ptr()), tree.coord, len(win),
                                       C.c_void_p(out.data_ptr()), cap, C.byref(cnt),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return cnt.value

    ms = timed(join)
    res["join_1M_windows_queries_s"] = N_WINDOWS / (ms * 1e-3)
    res["join_1M_windows_pairs_s"] = npairs / (ms * 1e-3)
    res["join_1M_windows_pairs"] = npairs
    # join roofline: 20 B per entry examined (the reference's `num` counter),
    # 16 B per query box, 8 B per emitted pair
    examined = int(tree.query_counts(win)[:, 0].sum())
    algo = 20 * examined + 16 * N_WINDOWS + 8 * npairs
    peak, kind = hbm_peak()
    res["join_roofline"] = {"bound": "hbm", "achieved": algo / (ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                            "frac": algo / (ms * 1e-3) / 1e9 / peak, "peak_source": kind,
                            "algorithmic_bytes": algo, "entries_examined": examined, "ms": ms}

    # the batched uneven overlay at its full size (1M x 1M polygons)
    res["uneven_overlay_1.0"] = batched_overlay(prt, 1.0)
    # the differentiable-area configuration at full size
    res["differentiable_area_1M"] = differentiable_area(prt, 1_000_000)
    # the map-alignment loop, 200k parcels x 200 steps
    res["alignment_200k"] = alignment(200_000)

    # small overlay configuration: 2 x 10,000 stars
    A = dg.star_layer(10000, seed=0)
    B = dg.star_layer(10000, seed=1)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    t = prt.build_bottomup(LA.mbr(), fanout=16)
    pairs = t.join(LB.mbr())
    l2p = t.leaf_order()
    res["overlay_small_pairs"] = len(pairs)
    for sched in ("plain", "batched"):
        ms = timed(lambda: prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched=sched))
        res[f"overlay_small_{sched}_pairs_s"] = len(pairs) / (ms * 1e-3)
    ms = timed(lambda: prt.intersection_area(LA, LB, torch.arange(10000, device="cuda"),
                                             torch.arange(10000, device="cuda")))
    res["area_fwd_10k_pairs_s"] = 10000 / (ms * 1e-3)
    return res


def differentiable_area(prt, n: int = 1_000_000, reps: int = 5):
    """The differentiable intersection-area configuration: n overlapping pairs
    of star polygons (16-64 vertices, float64; datagen.overlapping_pairs_device),
    loss = sum of intersection areas.  Times (CUDA events, median of `reps`
    after a warm-up) the forward (GPC clip + shoelace, area only) and the
    backward adjoint kernel through the C ABI, and reports the backward
    against the HBM roofline: algorithmic bytes = 32 B per vertex of both
    polygons of every pair (16 B read, 16 B gradient written) + 16 B per pair
    (ids and upstream gradient)."""
    import ctypes as C

    import torch
    from parlllelrtree_b200 import _lib
    from parlllelrtree_b200 import datagen as dg

    A, B = dg.overlapping_pairs_device(n, seed=0)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    pa = torch.arange(n, dtype=torch.int32, device="cuda")
    pb = pa.clone()
    area = torch.empty(n, dtype=torch.float64, device="cuda")
    up = torch.ones(n, dtype=torch.float64, device="cuda")
    gb = torch.zeros_like(LA.xy)
    go = torch.zeros_like(LB.xy)
    sb, so = LA.struct(), LB.struct()
    L = _lib.lib()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: C.c_void_p(t.data_ptr())

    def fwd():
        _lib.check(L.prt_area_fwd(p(pa), p(pb), n, C.byref(sb), C.byref(so), p(area), st))

    def bwd():
        _lib.check(L.prt_area_bwd(p(pa), p(pb), n, C.byref(sb), C.byref(so), p(up), p(gb), p(go), st))

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return float(np.median(ms))

    f_ms = timed(fwd)
    fb = C.c_int64(0)
    _lib.check(L.prt_area_fwd_fallbacks(C.byref(fb)))
    b_ms = timed(bwd)
    nv = int(len(LA.xy) + len(LB.xy))
    algo = 32 * nv + 16 * n
    peak, kind = hbm_peak()
    achieved = algo / (b_ms * 1e-3) / 1e9
    return {"pairs": n, "vertices": nv, "loss": float(area.sum()),
            "fwd_ms": f_ms, "fwd_pairs_s": n / (f_ms * 1e-3), "fwd_gpc_fallback_pairs": int(fb.value),
            "bwd_ms": b_ms, "bwd_pairs_s": n / (b_ms * 1e-3),
            "bwd_roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_source": kind, "algorithmic_bytes": algo}}


def alignment(n: int = 200_000):
    """The map-alignment configuration: 200k parcels (jittered-grid hexagons
    and quadrilaterals), the second layer under a random affine (rotation
    +-2 deg, scale +-1%, translation +-0.005) plus vertex noise sigma 1e-4;
    200 Adam steps, each rebuilding the R-tree, joining, clipping and running
    the area adjoint (parlllelrtree_b200.alignment).  `loop_s` is the time
    between CUDA events at the start and end of each pyramid stage, summed:
    it includes the host's work between launches (Python, torch's small ops,
    the library's count read-backs), which bounds this loop.  A second run
    with the library's launch profiler on gives `kernel_s`, the device time of
    the library's own kernels alone.  Also the recovery error."""
    from parlllelrtree_b200 import _lib
    from parlllelrtree_b200 import alignment as al

    A, B, T = al.parcel_layers(n, seed=3)
    theta, rec, stage_s = al.fit_affine(A, B, steps=200)
    total = sum(stage_s)
    _lib.profile_reset()
    _lib.profile_enable(1)
    al.fit_affine(A, B, steps=200)
    _lib.profile_enable(0)
    prof = _lib.profile_read()
    _lib.profile_reset()
    kernel_ms = sum(v[0] for v in prof.values())
    top = sorted(prof.items(), key=lambda kv: -kv[1][0])[:6]
    return {"parcels": n, "steps": len(rec), "loop_s": total, "steps_s": len(rec) / total,
            "stage_s": stage_s, "full_res_ms_per_step": stage_s[-1] / 50 * 1e3,
            "kernel_s": kernel_ms * 1e-3, "kernel_ms_top": {k: round(v[0], 2) for k, v in top},
            "recovery_error": al.recovery_error(theta, T), "initial_error": al.recovery_error(np.zeros(6), T),
            "final_overlap": rec[-1]["overlap"]}


def _oracle_rings(L, i):
    pr = L.poly_ring[i:i + 2].cpu().numpy()
    rv = L.ring_vert[pr[0]:pr[1] + 1].cpu().numpy()
    xy = L.xy[rv[0]:rv[-1]].cpu().numpy()
    return [xy[rv[k] - rv[0]:rv[k + 1] - rv[0]] for k in range(len(rv) - 1)]


def _overlay_sample(LA, LB, pairs, l2p, sample: int = 400):
    """An evenly strided sample of the candidate pairs: their positions and
    both polygons' rings (host copies) for the CPU clip."""
    n = len(pairs)
    step = max(1, n // sample)
    idx = np.arange(0, n, step)[:sample]
    p = pairs[torch_index(idx)].cpu().numpy()
    perm = l2p.cpu().numpy()
    polys = [(_oracle_rings(LA, int(perm[a])), _oracle_rings(LB, int(b))) for a, b in p]
    return idx, step, polys


def torch_index(idx):
    import torch

    return torch.from_numpy(np.asarray(idx, dtype=np.int64)).cuda()


def _cpu_overlay_sample(polys, n, step, budget_s: float = 20.0):
    """CPU baseline of the clip: the GPC restatement in oracle/ (C, one
    thread) on the strided sample, within a time budget.  The reference's own
    CPU clip core (oracle/_ref) overflows its fixed stack[400] on pairs with
    thousands of vertices, so the port stands in for it here.  Returns the
    baseline record and the clipped contours (for the parity check)."""
    import oracle

    t0 = time.perf_counter()
    out = []
    for s_, c_ in polys:
        out.append(oracle.gpc_clip(s_, c_, 1))
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": len(out) / dt, "unit": "pairs/s", "cores": 1, "kind": "port",
            "sample": f"{len(out)} of {n} candidate pairs (every {step}th), GPC restatement in oracle/ (C), "
                      "one thread"}, out


def _same(a, b):
    return len(a) == len(b) and all(h1 == h2 and np.array_equal(v1, v2) for (h1, v1), (h2, v2) in zip(a, b))


def batched_overlay(prt, scale: float = 1.0, plain_stride: int = 8):
    """The batched uneven overlay configuration: two layers of `scale` x 1M
    star polygons (vertex count clip(Zipf(1.2), 4, 4096), 5% with 1-3 clockwise
    holes, centres from the 64-Gaussian mixture, radius log-uniform
    6.5e-5..6.5e-4, calibrated for ~4M candidate pairs at 1M x 1M), generated
    on the device; tree over layer A's MBRs (fanout 16), join layer B, clip
    every candidate pair with the batched schedule (CUDA events; inputs in
    HBM; after an untimed warm-up on a 1% strided subset that sizes the
    allocator pools), and the whole build-join-clip graph (prt.Pipeline) on a
    side stream.  The plain schedule (one thread per pair in join order) is
    timed on an evenly strided subset (every plain_stride-th pair, labelled;
    on the full list it takes ~8 minutes), and the batched schedule on the
    same subset: batched_over_plain compares the two on equal work.  Parity: 400 evenly strided pairs of
    the batched results against the oracle's GPC clip, contour for contour and
    bit for bit; the same pairs give the CPU baseline."""
    import torch
    from parlllelrtree_b200 import datagen as dg

    n = int(1_000_000 * scale)
    A = dg.star_layer_device(n, seed=101, r_lo=6.5e-5, r_hi=6.5e-4)
    B = dg.star_layer_device(n, seed=102, r_lo=6.5e-5, r_hi=6.5e-4)
    LA, LB = prt.Layer.from_dict(A), prt.Layer.from_dict(B)
    del A, B
    t = prt.build_bottomup(LA.mbr(), fanout=16)
    pairs = t.join(LB.mbr())
    l2p = t.leaf_order()
    np_ = int(len(pairs))
    out = {"polygons_per_layer": n, "vertices_per_layer": [int(len(LA.xy)), int(len(LB.xy))],
           "pairs": np_, "schedule": prt.get_schedule()}
    del t

    def timed(fn):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        r = fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b), r

    warm = prt.overlay(pairs[::100].contiguous(), LA, LB, leaf_to_poly=l2p, sched="batched")
    del warm
    ms, r = timed(lambda: prt.overlay(pairs, LA, LB, leaf_to_poly=l2p, sched="batched"))
    out["batched_ms"] = ms
    out["batched_pairs_s"] = np_ / (ms * 1e-3)
    out["batched_nonempty"], out["batched_retried"] = r.nonempty, r.retried
    out["batched_contours"], out["batched_vertices"] = r.n_contours, r.n_vertices
    # parity on the strided sample (its CPU clip is the baseline too)
    idx, step, polys = _overlay_sample(LA, LB, pairs, l2p)
    got = r.contours_of(idx)
    del r
    base, ref = _cpu_overlay_sample(polys, np_, step)
    mism = sum(0 if _same(g, e) else 1 for g, e in zip(got, ref))
    out["parity_checked"], out["parity_mismatches"] = len(ref), mism
    out["cpu_baseline"] = base
    # plain schedule on a strided subset of the same pairs
    sub = pairs[::plain_stride].contiguous()
    warm = prt.overlay(sub[::10].contiguous(), LA, LB, leaf_to_poly=l2p, sched="plain")
    del warm
    ms_p, r = timed(lambda: prt.overlay(sub, LA, LB, leaf_to_poly=l2p, sched="plain"))
    out["plain_sample"] = f"every {plain_stride}th candidate pair ({len(sub)} pairs), join order"
    out["plain_ms"] = ms_p
    out["plain_pairs_s"] = len(sub) / (ms_p * 1e-3)
    out["plain_nonempty"] = r.nonempty
    del r
    # the batched schedule on the same subset: the ratio compares equal work
    ms_b, r = timed(lambda: prt.overlay(sub, LA, LB, leaf_to_poly=l2p, sched="batched"))
    out["subset_batched_ms"] = ms_b
    out["subset_batched_pairs_s"] = len(sub) / (ms_b * 1e-3)
    out["subset_matches_plain"] = bool(r.nonempty == out["plain_nonempty"])
    del r
    out["batched_over_plain"] = out["subset_batched_pairs_s"] / out["plain_pairs_s"]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        pipe = prt.Pipeline(LA, LB, max_pairs=int(np_ * 1.25) + 1024)
        pipe.run()  # first run: uncaptured pass + capture
        stream.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        pipe.run()
        b.record(stream)
        b.synchronize()
        sz = pipe.sizes()
    out["pipeline_ms"] = a.elapsed_time(b)
    out["pipeline_pairs_s"] = sz["pairs"] / (out["pipeline_ms"] * 1e-3)
    out["pipeline_sizes"] = sz
    out["pipeline_matches_batched"] = bool(sz["pairs"] == np_ and sz["contours"] == out["batched_contours"]
                                           and sz["vertices"] == out["batched_vertices"])
    del pipe
    out["e2e"] = overlay_e2e(prt, LA, LB)
    return out


def overlay_e2e(prt, LA, LB, chunk_pairs: int = 1 << 20):
    """The overlay end to end through the public API, from host memory to
    host memory: both layers' arrays copied from pinned host memory to the
    device, polygon MBRs, bottom-up tree over layer A, join of layer B, and
    the batched clip streamed in chunks of `chunk_pairs` pairs
    (prt.overlay_stream) whose results land in host memory, chunk by chunk,
    and are handed to a callback (here it counts them).  Wall time around it
    all, the device synchronised at both ends."""
    import psutil
    import torch

    hosts = [[t.cpu().pin_memory() for t in (L.poly_ring, L.ring_vert, L.ring_hole, L.xy)] for L in (LA, LB)]
    h2d = int(sum(t.numel() * t.element_size() for hs in hosts for t in hs))
    if psutil.virtual_memory().available < 2 * h2d:
        return {"unavailable": f"host memory: {psutil.virtual_memory().available >> 30} GiB free for {h2d >> 30} GiB of layers"}
    got = {"d2h": 0, "pairs": 0, "vertices": 0}

    def take(first, off, nv, hole, xy):
        got["d2h"] += off.nbytes + nv.nbytes + hole.nbytes + xy.nbytes
        got["pairs"] += len(off) - 1
        got["vertices"] += len(xy)
        return 0

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dev = [[t.to("cuda", non_blocking=True) for t in hs] for hs in hosts]
    A, B = prt.Layer(*dev[0]), prt.Layer(*dev[1])
    tree = prt.build_bottomup(A.mbr(), fanout=16)
    pairs = tree.join(B.mbr())
    prt.overlay_stream(pairs, A, B, take, leaf_to_poly=tree.leaf_order(), chunk_pairs=chunk_pairs)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    return {"value": got["pairs"] / dt, "unit": "pairs/s", "seconds": dt, "h2d_bytes": h2d, "d2h_bytes": got["d2h"],
            "chunk_pairs": chunk_pairs, "vertices_out": got["vertices"],
            "path": "pinned host layers -> device -> MBRs -> tree -> join -> streamed batched clip -> host arrays"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
