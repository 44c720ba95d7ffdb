"""The N > 1 path of bench.py on the host: one process per rank, the
slowest rank's time as the job's, and the reference arm's single line from
rank 0.  world_size 2 with the gloo backend; no GPU."""
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


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_env()[:2] == (rank, world)
        bench.barrier(world)
        out[rank] = bench.max_over_ranks(1.5 + rank, world)
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    assert dict(out) == {0: 2.5, 1: 2.5}


def test_reference_arm_under_torchrun_prints_once():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--workload", "static_drop_64", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"


def test_dominant_kernel_is_a_single_kernel_scope():
    """The roofline's dominant kernel is the largest scope of one kernel
    launch: a multi-kernel scope (the five passes of solver2d) that takes
    longer is passed over; with no single-kernel scope the largest stands."""
    sys.path.insert(0, ROOT)
    import bench
    table = {"solver2d": {"ms": 10.0, "launches": 100, "timed": 20},
             "ab2": {"ms": 9.8, "launches": 20, "timed": 20},
             "adv_stage": {"ms": 6.0, "launches": 60, "timed": 60},
             "unused": {"ms": 0.0, "launches": 0, "timed": 0}}
    assert bench.dominant_scope(table)[0] == "ab2"
    assert bench.dominant_scope({"solver2d": table["solver2d"]})[0] == "solver2d"
