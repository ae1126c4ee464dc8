"""Ensemble members dealt to ranks and gathered (bioneuroncore_b200/shard.py).

On CPU: the deal (greedy size balance), and world_size 2 over gloo, where each rank
runs its members through a runner and one all-gather brings the results back; the
gathered results must equal one process's run of all members bit for bit.  The CPU
runner here is the oracle (test infrastructure).  On the GPU: the device runner's
per-member results equal the oracle's for each member.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TICKS = 60
DT = 0.025


def _params():
    sys.path.insert(0, ROOT)
    from bioneuroncore_b200 import ensemble_params
    ps = ensemble_params(31, 5, 64, 600)
    for p in ps:
        p.stim_pA = 3000.0
    return list(ps)


def oracle_runner(params, ticks, dt):
    """Each member alone through the CPU oracle; the fields the device runner returns."""
    from bioneuroncore_b200 import Network
    from oracle.oracle import Oracle
    out = []
    for p in params:
        o = Oracle(Network(p))
        o.run(ticks, dt)
        out.append({"V[0]": o.segment_field("V"), "spikes[0]": o.segment_field("spikes"),
                    "ion_in[1]": o.segment_field("ion_in", 1), "bouton_Ca[0]": o.synapse_field("bouton_Ca"),
                    "refractory[0]": o.synapse_field("refractory")})
    return out


def test_deal_balances_sizes_and_covers_every_member():
    from bioneuroncore_b200.shard import deal_members
    sizes = [900, 100, 500, 500, 300, 200, 2000, 50]
    for world in (1, 2, 3, 8):
        deal = deal_members(sizes, world)
        flat = sorted(m for part in deal for m in part)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[m] for m in part) for part in deal]
        assert max(loads) - min(loads) <= max(sizes)
    assert deal_members(sizes, 2) == deal_members(sizes, 2)   # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, sizes, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from bioneuroncore_b200.shard import run_sharded
    import test_shard
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        res, deal = run_sharded(test_shard._params(), TICKS, DT, test_shard.oracle_runner, dist=dist, sizes=sizes)
        out.put((rank, [{k: v.tobytes() for k, v in r.items()} for r in res], deal))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_what_one_process_computes():
    import torch.multiprocessing as mp
    from bioneuroncore_b200.shard import member_segments, run_sharded
    ps = _params()
    sizes = member_segments(ps)
    single, _ = run_sharded(ps, TICKS, DT, oracle_runner, dist=None, sizes=sizes)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted((q.get(timeout=300) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    deal = got[0][2]
    assert deal == got[1][2] and all(len(part) > 0 for part in deal)
    for rank, res, _ in got:
        for m, (a, b) in enumerate(zip(res, single)):
            for k in b:
                assert a[k] == b[k].tobytes(), "rank %d member %d %s" % (rank, m, k)


@pytest.mark.gpu
def test_device_runner_members_equal_the_oracle():
    from bioneuroncore_b200.shard import device_runner, run_sharded
    ps = _params()
    dev, _ = run_sharded(ps, TICKS, DT, device_runner(0))
    ora, _ = run_sharded(ps, TICKS, DT, oracle_runner)
    for m, (a, b) in enumerate(zip(dev, ora)):
        for k in b:
            x = np.asarray(a[k], np.float32)
            y = np.asarray(b[k], np.float32)
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), "member %d %s" % (m, k)
