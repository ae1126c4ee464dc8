"""The state conversion on the device: the loader's records gathered into the device
layout by the conversion kernels (csrc/convert.cu), read back before any tick.

Every value the records hold -- segment state, modifier state words and densities'
flags, synapse state -- must come back as the record held it, whatever the value: the
records are filled with seeded random values here rather than the generator's
defaults, so a word taken from the wrong record or slot shows.  A receptor override
out of range on a modifier item must still fail the load with the builder's message.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _net(seed=11):
    from bioneuroncore_b200 import Network, NetgenParams, NET_LARGE
    return Network(NetgenParams(family=NET_LARGE, n_neurons=6, seed=seed))


def _same(got, want, what):
    got = np.asarray(got, np.float32)
    want = np.asarray(want, np.float32)
    bad = got.view(np.uint32) != want.view(np.uint32)
    assert not bad.any(), "%s: %d mismatches, first at %d (%r vs %r)" % (
        what, int(bad.sum()), int(np.argmax(bad)), got[np.argmax(bad)], want[np.argmax(bad)])


def test_segment_and_item_state_round_trip():
    from bioneuroncore_b200 import Backend
    net = _net()
    seg = net.segments
    rng = np.random.default_rng(5)
    n = len(seg)
    seg["V_m"] = rng.uniform(-80.0, -50.0, n)
    seg["intra_ions"] = seg["intra_ions"] * rng.uniform(0.9, 1.1, seg["intra_ions"].shape)
    seg["extra_ions"] = seg["extra_ions"] * rng.uniform(0.9, 1.1, seg["extra_ions"].shape)
    seg["ATP_level"] = rng.uniform(1.0, 3.0, n)
    mods = seg["modifiers"]
    cnt = seg["modifier_count"]
    for i in range(n):
        for j in range(int(cnt[i])):
            # gates in (0, 1): every model accepts them as a starting state
            mods[i, j]["state"][:3] = rng.uniform(0.05, 0.95, 3)
    b = Backend()
    b.load_network(net)
    _same(b.segment_field("V"), seg["V_m"], "V")
    for q in range(7):
        _same(b.segment_field("ion_in", q), seg["intra_ions"][:, q], "ion_in[%d]" % q)
        _same(b.segment_field("ion_out", q), seg["extra_ions"][:, q], "ion_out[%d]" % q)
    _same(b.segment_field("ATP"), seg["ATP_level"], "ATP")
    for slot in range(int(cnt.max())):
        has = cnt > slot
        for k in range(3):
            got = b.segment_field("mod_state", slot * 8 + k)[has]
            _same(got, mods[has, slot]["state"][:, k], "slot %d state %d" % (slot, k))


def test_synapse_state_round_trip():
    from bioneuroncore_b200 import Backend
    net = _net(seed=12)
    syn = net.synapses
    rng = np.random.default_rng(6)
    k = len(syn)
    for f in ("bouton_Ca", "spine_Ca", "spine_camkii", "spine_calcineurin", "facilitation", "weight"):
        syn[f] = rng.uniform(0.1, 2.0, k)
    b = Backend()
    b.load_network(net)
    for f in ("bouton_Ca", "spine_Ca", "spine_camkii", "spine_calcineurin", "facilitation", "weight"):
        _same(b.synapse_field(f, 0, k), syn[f], f)


def test_item_receptor_override_out_of_range_fails_the_load():
    from bioneuroncore_b200 import Backend, BackendError, last_error
    net = _net(seed=13)
    seg = net.segments
    mods = seg["modifiers"]
    hit = None
    for i in range(len(seg)):
        for j in range(int(seg["modifier_count"][i])):
            if mods[i, j]["type"] == 8:
                hit = (i, j)
                break
        if hit:
            break
    assert hit, "the large family carries AMPA items"
    mods[hit[0], hit[1]]["active_vars"] = 9
    b = Backend()
    with pytest.raises(BackendError):
        b.load_network(net)
    assert "active_vars 9 out of range" in last_error()
