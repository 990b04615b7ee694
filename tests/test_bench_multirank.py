"""Multi-rank plumbing of bench.py on CPU with the gloo backend (world size 2).

The reaction step shards without any exchange (replicas only): every rank
integrates its own batch, the job time is the slowest rank's, and the
reference arm runs on rank 0 alone while the other ranks exit cleanly.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 100.0 * (rank + 1)          # rank 1 is the slow one
        slow = bench.max_over_ranks(ms, world, torch.device("cpu"))
        rate = bench.whole_job_rate(1000, 3, slow, world)
        q.put((rank, slow, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, slow, rate in res:
        assert slow == 200.0                       # both ranks see the slowest rank's time
        assert rate == pytest.approx(2 * 1000 * 3 / 0.2)   # all cells of all ranks / job time


def test_reference_arm_two_ranks_gloo():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "1", "--cells", "2048", "--cpu-sample", "64"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1                          # rank 0 alone prints
    out = lines[0]
    assert out["impl"] == "reference" and out["n_gpus"] == 2
    assert out["value"] > 0 and out["cpu_baseline"]["kind"] == "port"
    assert out["e2e"]["h2d_bytes_per_step"] == 0
