"""Ensemble members dealt to ranks, one process per GPU, and their results gathered.

Ensemble members are independent networks (a parameter sweep, or the batched-ensemble
workload): nothing crosses between them during a run, so a multi-GPU run deals whole
members to ranks and needs no data-path collective.  Each rank builds one ensemble of
its members on its GPU and runs the ticks; at the end one all-gather brings every
member's results to every rank, in member order.

Members are dealt by greedy size balance: largest first, each to the rank with the
fewest segments so far (the lowest rank on a tie), which bounds the imbalance by the
largest member.
"""
import numpy as np


def deal_members(sizes, world):
    """Per-rank lists of member indices (ascending) for members of `sizes` segments."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = [0] * world
    out = [[] for _ in range(world)]
    for m in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(m)
        loads[r] += int(sizes[m])
    return [sorted(x) for x in out]


def member_segments(params):
    """Segments of each generated member (host-only planning, no device)."""
    from . import plan_generated
    return [int(plan_generated(p).n_segments) for p in params]


def device_runner(device=0, fields=(("V", 0), ("spikes", 0), ("ion_in", 1)), syn_fields=(("bouton_Ca", 0),
                                                                                          ("refractory", 0))):
    """A runner for run_sharded: the members as one ensemble on `device`, the tick loop
    as one graph launch; returns per member a dict of its segment and synapse fields."""
    def run(params, ticks, dt):
        from . import Backend, NetgenParams
        if not params:
            return []
        b = Backend(device)
        try:
            b.load_ensemble((NetgenParams * len(params))(*params))
            b.run_ticks_graph(ticks, dt)
            n_syn = b.info().n_synapses
            seg = {"%s[%d]" % f: np.asarray(b.segment_field(*f)) for f in fields}
            syn = {"%s[%d]" % f: np.asarray(b.synapse_field(f[0], f[1], n_syn)) for f in syn_fields}
            out = []
            for m in range(len(params)):
                r = b.ensemble_member(m)
                d = {k: v[r.seg_begin:r.seg_begin + r.n_segments].copy() for k, v in seg.items()}
                d.update({k: v[r.syn_begin:r.syn_begin + r.n_synapses].copy() for k, v in syn.items()})
                out.append(d)
            return out
        finally:
            b.close()
    return run


def run_sharded(params, ticks, dt, runner, dist=None, sizes=None):
    """Runs the members dealt to this rank with `runner(params, ticks, dt)` (a list of
    per-member results) and gathers all members' results on every rank (one
    all_gather_object).  dist: torch.distributed after init_process_group, or None for
    one process.  Returns (results in member order, the deal)."""
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    sizes = member_segments(params) if sizes is None else sizes
    deal = deal_members(sizes, world)
    mine = deal[rank]
    local = runner([params[m] for m in mine], ticks, dt)
    if len(local) != len(mine):
        raise RuntimeError("runner returned %d results for %d members" % (len(local), len(mine)))
    if dist is None:
        parts = [list(zip(mine, local))]
    else:
        parts = [None] * world
        dist.all_gather_object(parts, list(zip(mine, local)))
    results = [None] * len(params)
    for part in parts:
        for m, res in part:
            results[m] = res
    return results, deal
