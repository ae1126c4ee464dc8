"""Mechano stimuli through bnc_upload_mechano, against the CPU oracle.

The reference applies a mechano stimulus -- a value written into one state word of
the first modifier of a type on a segment, found by the segment's id -- once, before
the modifier currents of the tick it is passed to (simulation_host.cpp:211-230).  The
oracle's restatement of that is pinned to the reference's own tick by
tests/test_oracle_vs_reference.py::test_mechano_stimuli_bit_identical, with the same
schedule as here: gates, parameter words (which switch the item to reading its
parameters), the effective-area word, a myelin-blocked slot, and stimuli that match
nothing.  The device state must equal the oracle's bit for bit, and so must the
records a drop-in caller reads.
"""
import ctypes

import numpy as np
import pytest

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

DT = 0.025


def _same(a, b, what):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    ok = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
    if not ok.all():
        i = int(np.argmax(~ok))
        raise AssertionError("%s differs at %d: gpu %r oracle %r (%d mismatches)"
                             % (what, i, a[i], b[i], int((~ok).sum())))


def test_mechano_stimuli_equal_the_oracle():
    import test_oracle_vs_reference as pin
    from bioneuroncore_b200 import Backend, Network, NetgenParams, NET_SMALL
    p = NetgenParams(family=NET_SMALL, n_neurons=8, seed=7, stim_pA=3000.0)
    net_g, net_o = Network(p), Network(p)
    sched = pin.mechano_schedule(net_g)
    gpu = Backend()
    gpu.load_network(net_g)
    ora = Oracle(net_o)
    nmod = int(net_g.segments["modifier_count"].max())
    for t in range(200):
        if t in sched:
            gpu.upload_mechano(sched[t])
            ora.upload_mechano(sched[t])
        gpu.run_ticks(1, DT)
        ora.run(1, DT)
        if t in sched or t + 1 == 200:
            label = "tick %d" % (t + 1)
            _same(gpu.segment_field("V"), ora.segment_field("V"), label + " V")
            for q in range(7):
                _same(gpu.segment_field("ion_in", q), ora.segment_field("ion_in", q), "%s ion_in[%d]" % (label, q))
            for slot in range(nmod):
                for k in range(7):
                    _same(gpu.segment_field("mod_state", slot * 8 + k), ora.segment_field("mod_state", slot * 8 + k),
                          "%s slot %d state %d" % (label, slot, k))


def test_mechano_stimuli_reach_the_dropin_records(tmp_path):
    """Through the reference-facing calls: the records after each tick hold the
    stimulated words, the blocked slot's word included."""
    import test_oracle_vs_reference as pin
    from bioneuroncore_b200 import Backend, Network, NetgenParams, NET_SMALL, load_library
    from bioneuroncore_b200.abi import SEGMENT_DTYPE, view
    p = NetgenParams(family=NET_SMALL, n_neurons=8, seed=7, stim_pA=3000.0)
    net = Network(p)
    path = tmp_path / "net.bion"
    assert load_library().bnc_bion_save(str(path).encode(), ctypes.byref(net.data)) == 0
    sched = pin.mechano_schedule(net)
    b = Backend()
    b.load_bion(str(path))
    n = net.data.num_segments
    for t in range(70):
        if t in sched:
            b.upload_mechano(sched[t])
        b.run_tick(DT)
        if t in sched:
            seg = view(b.bion_data().segments, SEGMENT_DTYPE, n)
            for sid, mt, idx, val in sched[t]:
                hit = np.flatnonzero(seg["id"] == sid)
                if not len(hit) or not (0 <= idx < 7):
                    continue
                i = int(hit[0])
                slots = np.flatnonzero(seg["modifiers"][i]["type"][:seg["modifier_count"][i]] == mt)
                if not len(slots):
                    continue
                st = seg["modifiers"][i, slots[0]]["state"][idx]
                # a gate moves on in the tick after the write; parameter words (Nav 5,
                # K2P 0 and 1) and a myelin-blocked slot keep the value written
                blocked = mt in (107, 123) and 4 in seg["modifiers"][i]["type"][:seg["modifier_count"][i]]
                if (mt, idx) in ((141, 5), (142, 5), (107, 0), (107, 1)) or blocked:
                    later = [v for s2, m2, i2, v in sched[t] if (s2, m2, i2) == (sid, mt, idx)][-1]
                    assert st == np.float64(np.float32(later)), (t, sid, mt, idx, st)


def test_mechano_needs_records():
    from bioneuroncore_b200 import Backend, NetgenParams, NET_SMALL, BackendError
    b = Backend()
    b.load_generated(NetgenParams(family=NET_SMALL, n_neurons=2, seed=1))
    with pytest.raises(BackendError):
        b.upload_mechano([(0, 123, 0, 1.0)])
