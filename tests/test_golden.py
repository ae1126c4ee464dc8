"""The oracle against the reference-generated fixtures in tests/golden/.

The fixtures hold the reference's own state (FP64 V_m and ions) after a few
hundred ticks of seeded networks; the oracle keeps FP32 state, so the bar is
the relative tolerance in tests/golden_cases.py, and spike counts must be equal.
"""
import numpy as np
import pytest

import golden_cases
from oracle.oracle import Oracle, reference_available


@pytest.mark.parametrize("name", golden_cases.cases())
def test_oracle_matches_reference_fixture(name):
    from bioneuroncore_b200 import Network, NetgenParams
    g, spec = golden_cases.load(name)
    net = Network(NetgenParams(**spec))
    o = Oracle(net)
    log = None
    if "release_syn" in g.files:
        trace, log = golden_cases.run_scheduled(o, name, net, int(g["ticks"]), float(g["dt"]), g["somata"],
                                                lambda: o.segment_field("V"),
                                                read_refractory=lambda: o.synapse_field("refractory"))
        assert len(log) > 0
    elif golden_cases.stimulus_schedule(name, net):
        trace = golden_cases.run_scheduled(o, name, net, int(g["ticks"]), float(g["dt"]), g["somata"],
                                           lambda: o.segment_field("V"))
    else:
        trace = o.trace(int(g["ticks"]), float(g["dt"]), g["somata"])
    golden_cases.compare(g, trace, o.segment_field, o.synapse_field, log=log)


@pytest.mark.parametrize("name", golden_cases.release_cases())
def test_fp64_restatement_reproduces_release_fixture(name):
    """The oracle's FP64-state build (-DBO_FP64 -DBO_LIBM: the reference's state types
    and C library functions) against a fixture of the reference's own run with
    releases: the same release decisions (synapse, tick) and every held state word
    equal bit for bit.  Needs only the fixture, not the reference's sources."""
    from bioneuroncore_b200 import Network, NetgenParams
    g, spec = golden_cases.load(name)
    net = Network(NetgenParams(**spec))
    o = Oracle(net, fp64=True)
    _, log = golden_cases.run_scheduled(o, name, net, int(g["ticks"]), float(g["dt"]), g["somata"],
                                        lambda: o.segment_field("V"),
                                        read_refractory=lambda: o.synapse_field("refractory"))
    assert len(log) > 0 and log == golden_cases.release_log(g)
    bad = []
    for f, q in golden_cases.SEG_FULL:
        if not np.array_equal(o.segment_field(f, q), g["full_seg_%s_%d" % (f, q)]):
            bad.append("%s[%d]" % (f, q))
    for f, q in golden_cases.SYN_FULL:
        if not np.array_equal(o.synapse_field(f, q), g["full_syn_%s_%d" % (f, q)]):
            bad.append("syn %s[%d]" % (f, q))
    assert not bad, "FP64 restatement differs from the reference's run: %r" % bad
    assert np.array_equal(o.segment_field("spikes").astype(np.int64), g["spikes"].astype(np.int64))


def test_fixtures_exist():
    assert set(golden_cases.cases()) >= {"small_n8_s7", "large_n4_s3", "stimuli_n8_s7", "releases_extras_n8_s6"}
    assert set(golden_cases.release_cases()) >= {"releases_extras_n8_s6", "releases_large_n12_s3"}


@pytest.mark.skipif(not reference_available(), reason="reference CPU library not built here")
def test_fixtures_are_reproducible_from_the_reference():
    """Re-runs the reference for the smallest fixture and checks it reproduces bit for bit."""
    import importlib.util
    import os
    spec_ = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(golden_cases.GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec_)
    spec_.loader.exec_module(mg)
    g, spec = golden_cases.load("large_n4_s3")
    fresh = mg.run_reference(spec, int(g["ticks"]))
    for k in ("V", "ion_in", "ion_out", "soma_trace", "spikes", "syn_weight"):
        assert np.array_equal(fresh[k], g[k]), k
