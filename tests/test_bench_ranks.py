"""The multi-process paths of bench.py on CPU: two gloo ranks take the
max-over-ranks time and meet at the barrier as the NCCL ranks do on GPUs,
and the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    m = bench.max_over_ranks(float(rank + 1) * 1.5, world, device="cpu")
    bench.barrier(world)
    out[rank] = m
    dist.destroy_process_group()


def test_max_over_ranks_gloo_world_2():
    port = _free_port()
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
    assert dict(out) == {0: 3.0, 1: 3.0}


def test_reference_arm_runs_on_rank_0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120, cwd=ROOT)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line():
    """Rank 0 of the reference arm prints one JSON line with the driver's keys."""
    import oracle

    if not oracle.ref_available():
        oracle.build_ref()
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference"
    if "unavailable" not in d:
        assert d["value"] > 0 and d["cpu_baseline"]["cores"] >= 1 and d["e2e"]["h2d_bytes_per_step"] == 0
