"""bench.py's multi-rank logic on CPU: world_size 2 over gloo.

With N GPUs the bench runs one independent network per rank (replicas; the
path has no per-tick exchange in this mode). What must hold across ranks:
every rank takes the same collective steps, the timed value is the max over
ranks, and each rank simulates a distinct seeded network. Under torchrun, the
reference arm prints only on rank 0; the other ranks exit 0 without work.
"""
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


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench.rank_barrier(dist, "cpu")
        got = bench.max_over_ranks(1.0 + 3.0 * rank, dist, "cpu")
        bench.rank_barrier(dist, "cpu")
        same = bench.max_over_ranks(5.0, dist, "cpu")
        out.put((rank, got, same, bench.rank_seed(20260, rank)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_distinct_rank_networks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [4.0, 4.0]
    assert [r[2] for r in res] == [5.0, 5.0]
    assert res[0][3] != res[1][3]


def test_reference_arm_prints_only_on_rank_zero():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
