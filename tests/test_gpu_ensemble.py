"""Batched ensembles and the captured tick loop, on the GPU, through the C ABI.

An ensemble is one device structure holding many independent networks; every
member must evolve exactly as it does when simulated alone (same kernels, same
per-member synapse ids and hence the same release stream), so the bar is bit
equality per member.  The captured loop (bnc_run_ticks_graph) must equal plain
launches bit for bit, including across calls (the tick counter lives on the
device there).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 0.025
SEG = [("V", 0), ("ion_in", 0), ("ion_in", 1), ("ion_in", 2), ("ion_out", 1), ("ATP", 0), ("spikes", 0),
       ("neurotransmitter", 0), ("mod_state", 0), ("mod_state", 1), ("mod_state", 9)]
SYN = [("bouton_Ca", 0), ("spine_Ca", 0), ("weight", 0), ("refractory", 0), ("cleft", 0),
       ("receptor_state", 0)]


def _same(a, b, what):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    eq = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
    assert eq.all(), "%s: %d of %d differ (first at %d: %r vs %r)" % (
        what, int((~eq).sum()), a.size, int(np.argmax(~eq)), a[np.argmax(~eq)], b[np.argmax(~eq)])


def test_ensemble_members_match_separate_runs():
    from bioneuroncore_b200 import Backend, ensemble_params
    ps = ensemble_params(11, 5, 64, 1200)
    ens = Backend()
    ens.load_ensemble(ps)
    singles = []
    for p in ps:
        b = Backend()
        b.load_generated(p)
        singles.append(b)
    for step in (1, 24):
        ens.run_ticks(step, DT)
        for b in singles:
            b.run_ticks(step, DT)
        for f, i in SEG:
            whole = ens.segment_field(f, i)
            for m, b in enumerate(singles):
                r = ens.ensemble_member(m)
                _same(whole[r.seg_begin:r.seg_begin + r.n_segments], b.segment_field(f, i),
                      "member %d %s[%d] after +%d" % (m, f, i, step))
        n_total = ens.info().n_synapses
        for f, i in SYN:
            whole = ens.synapse_field(f, i, n_total)
            for m, b in enumerate(singles):
                r = ens.ensemble_member(m)
                _same(whole[r.syn_begin:r.syn_begin + r.n_synapses], b.synapse_field(f, i),
                      "member %d synapse %s[%d] after +%d" % (m, f, i, step))


def test_ensemble_of_host_networks_matches_generated_ensemble():
    from bioneuroncore_b200 import Backend, Network, ensemble_params
    ps = ensemble_params(5, 3, 64, 400)
    a, b = Backend(), Backend()
    a.load_ensemble(ps)
    nets = [Network(p) for p in ps]
    b.load_ensemble_networks(nets)
    a.run_ticks(10, DT)
    b.run_ticks(10, DT)
    for f, i in SEG:
        _same(a.segment_field(f, i), b.segment_field(f, i), "%s[%d]" % (f, i))


@pytest.mark.parametrize("family", ["small", "large"])
def test_graph_ticks_match_plain_ticks(family):
    from bioneuroncore_b200 import Backend, NetgenParams, NET_SMALL, NET_LARGE
    p = NetgenParams(family=NET_SMALL if family == "small" else NET_LARGE, n_neurons=10, n_synapses=200, seed=4)
    g, r = Backend(), Backend()
    g.load_generated(p)
    r.load_generated(p)
    for n in (70, 40, 3):        # two replays + 6 plain; one replay + 8 plain; plain only
        g.run_ticks_graph(n, DT)
        r.run_ticks(n, DT)
        assert g.info().ticks == r.info().ticks
        for f, i in SEG:
            _same(g.segment_field(f, i), r.segment_field(f, i), "%s %s[%d] after %d" % (family, f, i, n))
        for f, i in SYN:
            _same(g.synapse_field(f, i), r.synapse_field(f, i), "%s synapse %s[%d]" % (family, f, i))


def test_autotuned_grouping_gives_identical_results():
    from bioneuroncore_b200 import Backend, ensemble_params
    ps = ensemble_params(21, 6, 64, 3000)
    tuned, plain = Backend(), Backend()
    t = tuned.load_ensemble_tuned(ps, 32, DT)
    plain.load_ensemble(ps)
    assert t.candidates_tried >= 3 and t.ms_per_tick > 0
    assert (tuned.info().warp_cap, tuned.info().tile_segs) == (t.warp_cap, t.tile_segs)
    for step in (1, 40):
        tuned.run_ticks_graph(step, DT)
        plain.run_ticks(step, DT)
        for f, i in SEG:
            _same(tuned.segment_field(f, i), plain.segment_field(f, i), "%s[%d] after +%d" % (f, i, step))
        n = plain.info().n_synapses
        for f, i in SYN:
            _same(tuned.synapse_field(f, i, n), plain.synapse_field(f, i, n), "synapse %s[%d]" % (f, i))


def test_ensemble_members_equal_the_oracle_with_releases():
    """Each member of a seeded uneven ensemble (own conductance scales and seed), with
    3 nA somatic steps so that members release, run through the captured tick loop,
    equals the CPU oracle's run of that member alone, bit for bit, after 600 ticks."""
    from bioneuroncore_b200 import Backend, Network, ensemble_params
    from oracle.oracle import Oracle
    ps = ensemble_params(23, 6, 64, 900)
    for p in ps:
        p.stim_pA = 3000.0
    ens = Backend()
    ens.load_ensemble(ps)
    ticks = 600
    ens.run_ticks_graph(ticks, DT)
    n_total = ens.info().n_synapses
    released = 0
    for m, p in enumerate(ps):
        ora = Oracle(Network(p))
        log = ora.run_logged(ticks, DT)
        released += len(log[0])
        r = ens.ensemble_member(m)
        for f, i in SEG + [("ion_out", 0), ("ion_in", 3)]:
            whole = ens.segment_field(f, i)
            _same(whole[r.seg_begin:r.seg_begin + r.n_segments], ora.segment_field(f, i), "member %d %s[%d]" % (m, f, i))
        for f, i in SYN + [("RRP", 0), ("receptor_state", 1)]:
            whole = ens.synapse_field(f, i, n_total)
            _same(whole[r.syn_begin:r.syn_begin + r.n_synapses], ora.synapse_field(f, i),
                  "member %d synapse %s[%d]" % (m, f, i))
    assert released > 0, "the members must release transmitter"
