"""The N>1 path of bench.py on the CPU: two gloo ranks (no GPU).

N ranks run independent replicas of the workload; the job's time is the
slowest rank's and its value the sum of all ranks' updates.  The reference
arm prints only on rank 0.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    local_ms = 100.0 * (rank + 1)          # rank 1 is the slow one
    ms, value = bench.aggregate(dist, torch, local_ms, updates_per_step=1_000_000, steps=4, world=world,
                                device="cpu")
    q.put((rank, ms, value))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks_aggregate():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, value in got:
        assert ms == 200.0                         # max over ranks
        assert value == pytest.approx(2 * 1_000_000 * 4 / 0.2)


def test_reference_arm_runs_on_rank0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
