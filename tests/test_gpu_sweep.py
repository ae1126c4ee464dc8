"""Parameter sweeps on the device: every task of a sweep runs as one member of one
ensemble (bnc_sweep_run); each member must equal the oracle's standalone batch run of
its task bit for bit, and its metrics must be the reference's (the fixture made by
tests/golden/make_sweep_golden.py from the reference's own batch runs)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from golden_cases import GOLDEN

FIXTURE = os.path.join(GOLDEN, "sweep", "small_n8_s7_batch.npz")

pytestmark = pytest.mark.gpu


def _spec(g):
    spec = {k[len("param_"):]: float(g[k]) for k in g.files if k.startswith("param_")}
    for k in ("family", "n_neurons", "seed"):
        spec[k] = int(spec[k])
    return spec


def _tasks(g):
    return [([(int(t), float(v)) for t, v in g["task%d_overrides" % q]], int(g["task%d_seed" % q])) for q in range(3)]


def test_sweep_members_equal_standalone_batch_runs():
    from bioneuroncore_b200 import (Backend, Network, NetgenParams, EnsembleMember, load_library, sweep_run,
                                    sweep_tasks)
    from oracle.oracle import Oracle
    g = np.load(FIXTURE)
    spec = _spec(g)
    ticks, dt = int(g["ticks"]), float(g["dt"])
    tasks = _tasks(g)
    base = Network(NetgenParams(**spec))
    b = Backend()
    res = sweep_run(b, base, tasks, ticks, dt)
    V = np.asarray(b.segment_field("V", 0), np.float32)
    spikes = np.asarray(b.segment_field("spikes", 0))
    for q, (ov, seed) in enumerate(tasks):
        m = b.ensemble_member(q)
        net = Network(NetgenParams(**spec))
        arr, keep = sweep_tasks([(ov, seed)])
        assert load_library().bnc_sweep_apply(C.byref(net.data), arr) == 0
        o = Oracle(net)
        o.run(ticks, dt, tick_stride=2)
        mine = V[m.seg_begin:m.seg_begin + m.n_segments]
        ref = o.segment_field("V", 0)
        same = mine.view(np.uint32) == ref.view(np.uint32)
        assert same.all(), "task %d: %d segments differ" % (q, int((~same).sum()))
        assert np.array_equal(spikes[m.seg_begin:m.seg_begin + m.n_segments], o.segment_field("spikes", 0).astype(spikes.dtype))
        # metrics against the reference's core_compute_metrics on its FP64 run
        want = json.loads(str(g["task%d_metrics" % q]))
        got = json.loads(res[q].metrics_json.decode())
        assert got["tick"] == want["tick"] == 2 * ticks
        assert got["spike_count"] == want["spike_count"]
        assert abs(got["mean_vm"] - want["mean_vm"]) <= 0.011
        assert abs(got["synchrony"] - want["synchrony"]) <= 1e-4
        assert got["type_vm"].keys() == want["type_vm"].keys()
        assert res[q].tick == 2 * ticks


def test_single_tick_flag_steps_the_counter_once():
    from bioneuroncore_b200 import Backend, Network, NetgenParams, sweep_run
    from oracle.oracle import Oracle
    g = np.load(FIXTURE)
    spec = _spec(g)
    base = Network(NetgenParams(**spec))
    b = Backend()
    res = sweep_run(b, base, [([], 0), ([(107, 50.0)], 0)], 120, 0.1, single_tick=True)
    assert [r.tick for r in res] == [120, 120]
    o = Oracle(Network(NetgenParams(**spec)))
    o.run(120, 0.1)
    m = b.ensemble_member(0)
    mine = np.asarray(b.segment_field("V", 0), np.float32)[m.seg_begin:m.seg_begin + m.n_segments]
    assert (mine.view(np.uint32) == o.segment_field("V", 0).view(np.uint32)).all()
