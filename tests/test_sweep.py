"""Parameter sweeps (bnc_sweep_*): the reference's parameter-JSON reader, the task's
overrides and seed, and the batch mode's doubled tick counter, on the CPU.

The fixture tests/golden/sweep/small_n8_s7_batch.npz holds the reference's own batch
runs of three tasks (made by tests/golden/make_sweep_golden.py).  The oracle, given
the library's task application and the doubled counter, must reproduce them within
the relative tolerance of the other golden cases, with equal spike counts.
"""
import importlib.util
import os

import numpy as np
import pytest

from golden_cases import GOLDEN, REL_TOL, _rel

FIXTURE = os.path.join(GOLDEN, "sweep", "small_n8_s7_batch.npz")


def _gen():
    spec = importlib.util.spec_from_file_location("make_sweep_golden", os.path.join(GOLDEN, "make_sweep_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _task(g, q):
    ov = [(int(t), float(v)) for t, v in g["task%d_overrides" % q]]
    return ov, int(g["task%d_seed" % q])


def test_parse_params_follows_the_reference_reader():
    from bioneuroncore_b200 import sweep_parse_params
    got = sweep_parse_params('{"141": 0.05, "123" : 0.3, "nav": 2.5, 999: 1, 107:0.01}',
                             {"Nav1.6_channel": 141, "navX": 142})
    assert [t for t, _ in got] == [141, 123, 141, 107]     # 999 is not a type; "nav" -> lowest ID
    assert got[0][1] == np.float32(0.05) and got[3][1] == np.float32(0.01)
    assert sweep_parse_params("{}") == []
    assert [t for t, _ in sweep_parse_params('{"12": 1.0, "x": }')] == [12]   # stops at a value it cannot read


def test_apply_matches_the_reference_semantics():
    import ctypes as C
    from bioneuroncore_b200 import Network, NetgenParams, load_library, sweep_tasks
    gen = _gen()
    for ov, seed in gen.TASKS:
        a = Network(NetgenParams(**gen.SPEC))
        b = Network(NetgenParams(**gen.SPEC))
        gen.apply_task(a, ov, seed)
        arr, keep = sweep_tasks([(ov, seed)])
        assert load_library().bnc_sweep_apply(C.byref(b.data), arr) == 0
        assert np.array_equal(a.segments["modifiers"]["state"], b.segments["modifiers"]["state"])
        assert np.array_equal(a.synapses["release_probability"], b.synapses["release_probability"])
        if seed:
            assert not np.array_equal(b.synapses["release_probability"],
                                      Network(NetgenParams(**gen.SPEC)).synapses["release_probability"])


def test_fixture_exists():
    assert os.path.exists(FIXTURE)


@pytest.mark.parametrize("q", [0, 1, 2])
def test_oracle_batch_run_matches_the_reference_fixture(q):
    """The task applied by the library, the oracle's tick with the counter stepped twice
    per tick (dt 0.1 ms, 300 ticks) against the reference's batch run."""
    import ctypes as C
    from bioneuroncore_b200 import Network, NetgenParams, load_library, sweep_tasks
    from oracle.oracle import Oracle
    g = np.load(FIXTURE)
    gen = _gen()
    net = Network(NetgenParams(**gen.SPEC))
    arr, keep = sweep_tasks([_task(g, q)])
    assert load_library().bnc_sweep_apply(C.byref(net.data), arr) == 0
    o = Oracle(net)
    o.run(int(g["ticks"]), float(g["dt"]), tick_stride=2)
    err = _rel(o.segment_field("V", 0), g["task%d_V" % q], 1.0)
    assert err <= REL_TOL, err
    assert np.array_equal(o.segment_field("spikes", 0).astype(np.int64), g["task%d_spikes" % q].astype(np.int64))
