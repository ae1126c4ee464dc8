"""bnc_run_ticks_static_scratch against bnc_run_ticks, through the C ABI.

Some callers cannot call cudaMalloc while they drive the simulation: a host
whose pool allocator owns the device memory and refuses any other allocation,
or a control loop that cannot take the device-wide synchronisation of a
cudaFree.  For them the library has a tick entry point that allocates nothing:
the per-segment presynaptic records that the tile kernel hands to the synapse
kernel every tick live in a fixed array inside the library instead of buffers
of the network.  This file checks that it computes exactly what the regular
entry point computes -- bit for bit, the bar of every GPU test here -- on two
calls in a row (the second call finds the first call's records in the shared
array), and that a network larger than the array is refused.

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 0.025
BNC_ERR_ARG = -20
MAX_SEGMENTS = 131072  # BNC_STATIC_SCRATCH_MAX_SEGMENTS in include/bnc_b200.h

SEG_FIELDS = [("V", 0), ("ion_in", 2), ("ion_out", 2), ("ATP", 0), ("spikes", 0), ("neurotransmitter", 0)] + [
    ("mod_state", slot * 8 + k) for slot in range(4) for k in range(2)]
SYN_FIELDS = [("bouton_Ca", 0), ("spine_Ca", 0), ("weight", 0), ("refractory", 0), ("facilitation", 0),
              ("cleft", 0), ("cleft", 1), ("receptor_state", 0), ("receptor_state", 1)]


def _static_ticks(backend, n):
    rc = backend.lib.bnc_run_ticks_static_scratch(backend.h, n, C.c_float(DT))
    if rc != 0:
        raise AssertionError("bnc_run_ticks_static_scratch returned %d: %s" % (rc, backend.lib.bnc_last_error().decode()))


def _assert_same(a, b, what):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    same = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
    if not same.all():
        i = int(np.argmax(~same))
        raise AssertionError("%s differs at %d of %d: static scratch %r, regular %r (%d mismatches)"
                             % (what, i, a.size, a[i], b[i], int((~same).sum())))


def _compare(static, regular, n_syn, label):
    for f, i in SEG_FIELDS:
        _assert_same(static.segment_field(f, i), regular.segment_field(f, i), "%s %s[%d]" % (label, f, i))
    if n_syn:
        for f, i in SYN_FIELDS:
            _assert_same(static.synapse_field(f, i, n_syn), regular.synapse_field(f, i, n_syn),
                         "%s synapse %s[%d]" % (label, f, i))


@pytest.mark.parametrize("family,n_neurons,n_synapses,seed", [("large", 12, 300, 5), ("small", 16, 0, 11)])
def test_static_scratch_matches_regular_ticks(family, n_neurons, n_synapses, seed):
    from bioneuroncore_b200 import Backend, Network, NetgenParams, NET_LARGE, NET_SMALL
    p = NetgenParams(family=NET_LARGE if family == "large" else NET_SMALL, n_neurons=n_neurons,
                     n_synapses=n_synapses, seed=seed)
    net_s, net_r = Network(p), Network(p)
    static, regular = Backend(), Backend()
    static.load_network(net_s)
    regular.load_network(net_r)
    n_syn = net_r.data.num_synapses
    assert n_syn > 0
    assert static.info().n_segments <= MAX_SEGMENTS
    for call, n in enumerate((7, 23)):
        _static_ticks(static, n)
        regular.run_ticks(n, DT)
        assert static.info().ticks == regular.info().ticks
        _compare(static, regular, n_syn, "%s network, call %d (+%d ticks)" % (family, call + 1, n))


def test_static_scratch_with_presynaptic_ions_and_injections():
    """Synapses with readily releasable pools and bouton autoreceptor channels make the
    tile kernel also write the presynaptic ion records, which this entry point keeps in
    the fixed array as well; ion and ligand injections uploaded before the first call
    are applied by its first tick.  3 nA somatic steps make the network release within
    the run.  Both calls must equal the regular ticks bit for bit."""
    from bioneuroncore_b200 import Backend, Network, NetgenParams, NET_SMALL, NETGEN_SYNAPSE_EXTRAS
    from bioneuroncore_b200.abi import stimulus_data
    p = NetgenParams(family=NET_SMALL, n_neurons=16, seed=6, flags=NETGEN_SYNAPSE_EXTRAS, stim_pA=3000.0)
    net_s, net_r = Network(p), Network(p)
    syn = net_r.synapses
    assert (syn["RRP_max"] > 0).any() and (syn["pre_autoreceptor_count"] > 0).any()
    static, regular = Backend(), Backend()
    static.load_network(net_s)
    regular.load_network(net_r)
    cur = [tuple(int(r[f]) if f in ("segment_id", "start_tick") else float(r[f])
                 for f in ("segment_id", "amplitude_pA", "duration_ms", "start_tick")) for r in net_r.stimuli]
    inj = stimulus_data(current=cur, ion_inj=[(32, 0, 2.0, 0), (64, 1, 0.5, 1)], lig_inj=[(96, 0, 0.4, 1)])
    static.upload_stimuli(inj)
    regular.upload_stimuli(inj)
    n_syn = net_r.data.num_synapses
    rrp0 = np.asarray(regular.synapse_field("RRP", 0, n_syn)).copy()
    for call, n in enumerate((150, 350)):
        _static_ticks(static, n)
        regular.run_ticks(n, DT)
        assert static.info().ticks == regular.info().ticks
        _compare(static, regular, n_syn, "extras network, call %d (+%d ticks)" % (call + 1, n))
        _assert_same(static.synapse_field("RRP", 0, n_syn), regular.synapse_field("RRP", 0, n_syn), "RRP")
        for f, i in (("intra_nt", 0), ("ion_in", 0), ("ion_out", 1)):
            _assert_same(static.segment_field(f, i), regular.segment_field(f, i), "%s[%d]" % (f, i))
    assert (np.asarray(regular.synapse_field("RRP", 0, n_syn)) != rrp0).any(), "the run must release"


def test_static_scratch_rejects_networks_above_its_limit():
    from bioneuroncore_b200 import Backend, NetgenParams, NET_LARGE, plan_generated
    p = NetgenParams(family=NET_LARGE, n_neurons=MAX_SEGMENTS // 64 + 1, n_synapses=1000, seed=3)
    assert plan_generated(p).n_segments > MAX_SEGMENTS
    b = Backend()
    b.load_generated(p)
    rc = b.lib.bnc_run_ticks_static_scratch(b.h, 1, C.c_float(DT))
    assert rc == BNC_ERR_ARG
    assert "at most %d" % MAX_SEGMENTS in b.lib.bnc_last_error().decode()
    assert b.info().ticks == 0
    b.run_ticks(1, DT)  # the refusal leaves the handle usable
    assert b.info().ticks == 1
