"""GPU tick vs the CPU oracle on runs long enough to release transmitter.

The oracle (oracle/bnc_oracle.c) is pinned bit for bit to the reference's own tick by
tests/test_oracle_vs_reference.py, on these same generator families.  Here each case
runs until synapses release and the GPU must equal the oracle bit for bit: the release
decisions tick by tick (from the refractory counters: a synapse releases only while
its counter is 0 and a release leaves it above 0; simulation_host.cpp:421-459, 591),
the clefts, pools, bouton Ca2+ and the receptor states, and all segment state.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

DT = 0.025


def _pair(params):
    from bioneuroncore_b200 import Backend, Network
    net_o = Network(params)
    net_g = Network(params)
    gpu = Backend()
    gpu.load_network(net_g)
    return Oracle(net_o), gpu, net_g


def _same(a, b, what):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    ok = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
    if not ok.all():
        i = int(np.argmax(~ok))
        raise AssertionError("%s differs at %d of %d: gpu %r oracle %r (%d mismatches)"
                             % (what, i, a.size, a[i], b[i], int((~ok).sum())))


def _compare_everything(ora, gpu, net, label):
    seg = net.segments
    n_syn = net.data.num_synapses
    for f, i in [("V", 0), ("ATP", 0), ("temperature", 0), ("transcription", 0), ("spikes", 0)]:
        _same(gpu.segment_field(f, i), ora.segment_field(f, i), "%s %s" % (label, f))
    for q in range(7):
        _same(gpu.segment_field("ion_in", q), ora.segment_field("ion_in", q), "%s ion_in[%d]" % (label, q))
        _same(gpu.segment_field("ion_out", q), ora.segment_field("ion_out", q), "%s ion_out[%d]" % (label, q))
    for q in range(15):
        _same(gpu.segment_field("neurotransmitter", q), ora.segment_field("neurotransmitter", q),
              "%s neurotransmitter[%d]" % (label, q))
        _same(gpu.segment_field("intra_nt", q), ora.segment_field("intra_nt", q), "%s intra_nt[%d]" % (label, q))
    for slot in range(int(seg["modifier_count"].max())):
        for k in range(7):
            _same(gpu.segment_field("mod_state", slot * 8 + k), ora.segment_field("mod_state", slot * 8 + k),
                  "%s modifier slot %d state %d" % (label, slot, k))
    if not n_syn:
        return
    for f in ("bouton_Ca", "spine_Ca", "weight", "refractory", "facilitation", "spine_camkii",
              "spine_calcineurin", "RRP"):
        _same(gpu.synapse_field(f, 0, n_syn), ora.synapse_field(f, 0), "%s synapse %s" % (label, f))
    for q in range(15):
        _same(gpu.synapse_field("cleft", q, n_syn), ora.synapse_field("cleft", q), "%s cleft[%d]" % (label, q))
    for j in range(int(net.synapses["post_receptor_count"].max())):
        for k in range(3):   # the receptor models keep three state words
            _same(gpu.synapse_field("receptor_state", j * 8 + k, n_syn), ora.synapse_field("receptor_state", j * 8 + k),
                  "%s receptor %d state %d" % (label, j, k))


def _run(params, ticks, full_every):
    """Ticks GPU and oracle side by side; returns the common release decision log."""
    ora, gpu, net = _pair(params)
    n_syn = net.data.num_synapses
    log_g, log_o = [], []
    rg = gpu.synapse_field("refractory", 0, n_syn)
    ro = ora.synapse_field("refractory", 0)
    for t in range(ticks):
        ora.run(1, DT)
        gpu.run_ticks(1, DT)
        ng = gpu.synapse_field("refractory", 0, n_syn)
        no = ora.synapse_field("refractory", 0)
        log_g += [(int(i), t) for i in np.flatnonzero((rg == 0) & (ng > 0))]
        log_o += [(int(i), t) for i in np.flatnonzero((ro == 0) & (no > 0))]
        rg, ro = ng, no
        if log_g != log_o:
            raise AssertionError("release decisions differ at tick %d" % t)
        if (t + 1) % full_every == 0 or t + 1 == ticks:
            _compare_everything(ora, gpu, net, "tick %d" % (t + 1))
    return log_o, net


def test_large_set_releases_bitexact():
    """All 24 large-set models, 8 receptors per synapse (AMPA/NMDA, GABA-A/glycine),
    1,000 ticks: the network releases from about tick 100 on."""
    from bioneuroncore_b200 import NetgenParams, NET_LARGE
    log, _ = _run(NetgenParams(family=NET_LARGE, n_neurons=12, seed=3), 1000, 100)
    assert len(log) > 0


def test_large_set_draw_order_releases_bitexact():
    """The same with the modifiers kept in draw order (not listed by type ID)."""
    from bioneuroncore_b200 import NetgenParams, NET_LARGE, NETGEN_DRAW_ORDER
    log, _ = _run(NetgenParams(family=NET_LARGE, n_neurons=16, seed=4, flags=NETGEN_DRAW_ORDER), 400, 100)
    assert len(log) > 0


def test_synapse_extras_releases_bitexact():
    """Readily releasable pools, bouton autoreceptor channels (the extended presynaptic
    record) and delays (the delay slots), 1,000 ticks of the small family with 3 nA
    somatic steps; pooled, autoreceptor-carrying and delayed synapses all release."""
    from bioneuroncore_b200 import NetgenParams, NET_SMALL, NETGEN_SYNAPSE_EXTRAS
    p = NetgenParams(family=NET_SMALL, n_neurons=16, seed=6, flags=NETGEN_SYNAPSE_EXTRAS, stim_pA=3000.0)
    log, net = _run(p, 1000, 100)
    syn = net.synapses
    released = {s for s, _ in log}
    assert any(syn["delay"][s] > 0 for s in released)
    assert any(syn["RRP_max"][s] > 0 for s in released)
    assert any(syn["pre_autoreceptor_count"][s] > 0 for s in released)


def test_full_small_workload_bitexact():
    """The small workload at its full size and length: 64 neurons x 32 segments, 400
    synapses, 4,000 ticks at dt 0.025 ms, 0.2 nA steps on 10% of somata."""
    from bioneuroncore_b200 import NetgenParams, NET_SMALL
    _run(NetgenParams(family=NET_SMALL, n_neurons=64, seed=7), 4000, 1000)


def test_release_modulators_bitexact():
    """Presynaptic release modulators (Gi/o, Gs and ionotropic autoreceptors) beside
    bouton channels, pools and delays, 1,000 ticks: the modulators' state words, the
    release decisions and all other state equal the oracle's bit for bit."""
    from bioneuroncore_b200 import NetgenParams, NET_SMALL, NETGEN_SYNAPSE_EXTRAS, NETGEN_RELEASE_MODULATORS
    p = NetgenParams(family=NET_SMALL, n_neurons=16, seed=6,
                     flags=NETGEN_SYNAPSE_EXTRAS | NETGEN_RELEASE_MODULATORS, stim_pA=3000.0)
    log, net = _run(p, 1000, 100)
    assert len(log) > 0
    ora, gpu, net = _pair(p)
    ora.run(400, DT)
    gpu.run_ticks(400, DT)
    n_syn = net.data.num_synapses
    nmod = 0
    for j in range(int(net.synapses["pre_autoreceptor_count"].max())):
        g = gpu.synapse_field("autoreceptor_state", j * 8, n_syn)
        o = ora.synapse_field("autoreceptor_state", j * 8)
        types = np.where(net.synapses["pre_autoreceptor_count"] > j, net.synapses["pre_autoreceptors"][:, j]["type"], 0)
        is_mod = np.isin(types, [13, 18, 19, 22, 27, 29, 30, 35, 36, 38, 44, 46])
        nmod += int(is_mod.sum())
        _same(g[is_mod], o[is_mod], "modulator state, autoreceptor %d" % j)
    assert nmod > 0


def test_endocannabinoid_signalling_bitexact():
    """eCB synthesis on the post segments, its retrograde release into the clefts (the
    modifier losing a tenth per synapse, in synapse order) and CB1 autoreceptors reading
    it, 1,000 ticks: eCB clefts, neurotransmitter 9, modifier states and release
    decisions equal the oracle's bit for bit."""
    from bioneuroncore_b200 import NetgenParams, NET_SMALL, NETGEN_SYNAPSE_EXTRAS, NETGEN_ECB
    p = NetgenParams(family=NET_SMALL, n_neurons=16, seed=6, flags=NETGEN_SYNAPSE_EXTRAS | NETGEN_ECB,
                     stim_pA=3000.0)
    log, net = _run(p, 1000, 100)
    assert len(log) > 0


def test_glial_capture_bitexact():
    """Glial segments with a GLAST transporter: each cleft hands a share of its
    transmitter to the glial segment nearest in z (summed there in synapse order),
    the transporter takes it up in step 1, and no cleft clears it by its own time
    constant; 1,000 ticks equal the oracle's bit for bit."""
    from bioneuroncore_b200 import NetgenParams, NET_SMALL, NETGEN_SYNAPSE_EXTRAS, NETGEN_GLIA
    p = NetgenParams(family=NET_SMALL, n_neurons=16, seed=6, flags=NETGEN_SYNAPSE_EXTRAS | NETGEN_GLIA,
                     stim_pA=3000.0)
    log, net = _run(p, 1000, 100)
    assert len(log) > 0


def test_gap_junctions_bitexact():
    """Electrical synapses and dendritic bridges between somata, spread among the
    chemical synapses: connexin items, the slow gate, Cx43's Vj gate, the filtered
    current of delayed junctions, both segments' I_buffer in synapse order; 1,000 ticks
    equal the oracle's bit for bit, the junctions' gate and filter included."""
    from bioneuroncore_b200 import NetgenParams, NET_SMALL, NETGEN_GAP_JUNCTIONS
    p = NetgenParams(family=NET_SMALL, n_neurons=16, seed=6, flags=NETGEN_GAP_JUNCTIONS, stim_pA=3000.0)
    ora, gpu, net = _pair(p)
    n_syn = net.data.num_synapses
    gap = net.synapses["type"] > 0
    assert gap.sum() == 15
    for t in range(10):
        ora.run(100, DT)
        gpu.run_ticks(100, DT)
        _compare_everything(ora, gpu, net, "tick %d" % (100 * (t + 1)))
        _same(gpu.synapse_field("depression", 0, n_syn)[gap], ora.synapse_field("depression", 0)[gap],
              "tick %d gap slow gate" % (100 * (t + 1)))
    assert (ora.synapse_field("depression", 0)[gap] > 0).all()
