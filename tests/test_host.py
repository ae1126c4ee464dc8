"""Host-side logic without a GPU: the seeded generator, the builder's planning
(tiles, phase schedule, validation and the supported-type checks), and .bion
I/O, the latter also against the reference's own loader when it is built here
(bion_load_host / bion_save, src/bion_loader_host.cpp:26-504).
"""
import ctypes as C

import numpy as np
import pytest

from oracle.oracle import reference_available, REF_LIB

BNC_ERR_UNSUPPORTED = -21
BNC_ERR_FORMAT = -9
BNC_BION_ERR_BAD_CONN = -6
BNC_BION_ERR_BAD_MAGIC = -2
BNC_BION_ERR_FILE_OPEN = -1


def _net(**kw):
    from bioneuroncore_b200 import Network, NetgenParams
    return Network(NetgenParams(**kw))


def _plan_aos(net):
    from bioneuroncore_b200 import load_library, NetInfo
    info = NetInfo()
    rc = load_library().bnc_plan_aos(C.byref(net.data), net.stim_ptr, net.n_stim, C.byref(info))
    return rc, info


def _bytes(net):
    return (net.segments.tobytes(), net.synapses.tobytes(), net.connections.tobytes(), net.stimuli.tobytes())


def test_generator_is_deterministic_per_seed():
    a = _net(family=1, n_neurons=6, seed=42)
    b = _net(family=1, n_neurons=6, seed=42)
    c = _net(family=1, n_neurons=6, seed=43)
    assert _bytes(a) == _bytes(b)
    assert _bytes(a)[0] != _bytes(c)[0]


def test_small_family_shape():
    """64 x 32-segment neurons: soma + 15-segment dendrite chain + 16-segment axon,
    6 modifier kinds, 80% AMPA / 20% GABA-A synapses, stimuli on 10% of somata."""
    net = _net(family=1, n_neurons=20, seed=1)
    seg = net.segments
    assert net.data.num_segments == 20 * 32
    assert (seg["segment_type"][::32] == 1).all()
    assert np.allclose(seg["V_m"], -65.0)
    assert np.allclose(seg["intra_ions"][:, 0], 12.0) and np.allclose(seg["extra_ions"][:, 1], 4.0)
    assert net.data.num_connections == 20 * 31
    rtype = net.synapses["post_receptors"]["type"][:, 0]
    assert set(np.unique(rtype)) <= {8, 11}
    assert net.n_stim == 2
    assert (net.stimuli["amplitude_pA"] == 200.0).all()


def test_plan_of_generated_networks():
    from bioneuroncore_b200 import plan_generated, NetgenParams, NET_SMALL, NET_LARGE, NET_TREES
    inf = plan_generated(NetgenParams(family=NET_SMALL, n_neurons=64, seed=1))
    assert inf.n_segments == 2048 and inf.n_connections == 64 * 31
    assert inf.max_tile_segs <= 1024 and inf.n_tiles >= 2
    assert inf.n_synapses == 400 and inf.flags & 1 and inf.flags & 2
    big = plan_generated(NetgenParams(family=NET_LARGE, n_neurons=200, seed=1))
    assert big.n_segments == 200 * 64 and big.n_receptors == big.n_synapses * 8
    # 16 modifiers per segment from the large set, plus Cav2.1 on axon segments
    assert big.n_items >= 16 * big.n_segments
    assert big.algo_bytes_per_tick == pytest.approx(big.tile_bytes_per_tick + big.synapse_kernel_bytes_per_tick)
    trees = plan_generated(NetgenParams(family=NET_TREES, n_neurons=2, tree_depth=9, seed=1))
    assert trees.n_segments == 2 * 1023 and trees.max_tile_segs <= 1024
    # depth 10: 2,047-segment trees split over tile pairs (2-CTA clusters)
    big = plan_generated(NetgenParams(family=NET_TREES, n_neurons=3, tree_depth=10, seed=1))
    assert big.n_segments == 3 * 2047 and big.n_tiles == 6 and big.max_tile_segs == 1024
    assert big.smem_bytes <= 227 * 1024


def test_modifier_phase_groups():
    """Phase groups form on slot-order schedules only: the large set (16 modifiers per
    segment, slot order) runs 17 phases in ceil(17 / F) launches; the small set keeps
    its greedy type-uniform phases, one launch each; F is capped at 32."""
    from bioneuroncore_b200 import plan_generated, BuildOptions, NetgenParams, NET_SMALL, NET_LARGE
    p = NetgenParams(family=NET_LARGE, n_neurons=50, seed=2)
    for f, want in ((1, 1), (2, 2), (4, 4), (17, 17), (40, 32)):
        inf = plan_generated(p, BuildOptions(fuse_phases=f))
        assert inf.fuse_phases == want
        assert inf.modifier_launches == 1 + -(-inf.n_phases // want)
    assert plan_generated(p).fuse_phases == 4            # the default
    # from 65,536 segments on, the depth drops while warps would run more than 1.3
    # models per item on average: slots listed by type ID keep 4, slots in draw order
    # (no common order between segments) get 2 at 128k segments
    from bioneuroncore_b200 import NETGEN_DRAW_ORDER
    assert plan_generated(NetgenParams(family=NET_LARGE, n_neurons=2000, seed=2)).fuse_phases == 4
    assert plan_generated(NetgenParams(family=NET_LARGE, n_neurons=2000, seed=2, flags=NETGEN_DRAW_ORDER)).fuse_phases == 2
    assert plan_generated(NetgenParams(family=NET_LARGE, n_neurons=2000, seed=2, flags=NETGEN_DRAW_ORDER),
                          BuildOptions(fuse_phases=4)).fuse_phases == 4   # an explicit depth is kept
    small = plan_generated(NetgenParams(family=NET_SMALL, n_neurons=16, seed=2), BuildOptions(fuse_phases=3))
    assert small.fuse_phases == 1 and small.modifier_launches == 1 + small.n_phases
    # chunked modifier passes keep one launch per phase and chunk
    ch = plan_generated(p, BuildOptions(fuse_phases=3, chunk_segs=1000))
    assert ch.fuse_phases == 1


def test_synapse_step_launches():
    """Steps 3 and 4 run as k_release (the synapses' presynaptic half, one thread per
    synapse) and k_synapse for networks without release modulators, eCB, glia or gap
    junctions, and as one fused k_synapse (plus k_glia, k_gj_commit) otherwise."""
    from bioneuroncore_b200 import (plan_generated, NetgenParams, NET_SMALL, NET_LARGE, NETGEN_NO_SYNAPSES,
                                    NETGEN_GAP_JUNCTIONS, NETGEN_GLIA, NETGEN_RELEASE_MODULATORS)
    assert plan_generated(NetgenParams(family=NET_LARGE, n_neurons=20, seed=1)).synapse_launches == 2
    assert plan_generated(NetgenParams(family=NET_SMALL, n_neurons=8, seed=1)).synapse_launches == 2
    assert plan_generated(NetgenParams(family=NET_SMALL, n_neurons=8, seed=1,
                                       flags=NETGEN_NO_SYNAPSES)).synapse_launches == 1
    assert plan_generated(NetgenParams(family=NET_SMALL, n_neurons=8, seed=1,
                                       flags=NETGEN_RELEASE_MODULATORS)).synapse_launches == 1
    assert plan_generated(NetgenParams(family=NET_SMALL, n_neurons=8, seed=1,
                                       flags=NETGEN_GLIA | NETGEN_GAP_JUNCTIONS)).synapse_launches == 3


def test_diffusion_barrier_groups():
    """Tiles whose connections stay inside aligned groups of 32 or 64 threads get
    barriers of that group (32-segment neurons: a warp each; 64-segment neurons: a
    named 64-thread barrier), with a CTA of whole 64-thread groups; trees split over
    2-CTA clusters keep cluster barriers; the option turns the groups off."""
    from bioneuroncore_b200 import BuildOptions, plan_generated, NetgenParams, NET_SMALL, NET_LARGE, NET_TREES
    small = plan_generated(NetgenParams(family=NET_SMALL, n_neurons=64, seed=1))
    assert small.group_tiles_32 == small.n_tiles and small.group_tiles_64 == 0
    large = plan_generated(NetgenParams(family=NET_LARGE, n_neurons=100, seed=1))
    assert large.group_tiles_64 == large.n_tiles and large.group_tiles_32 == 0
    assert large.diffusion_threads % 64 == 0 and large.diffusion_threads <= 960
    off = plan_generated(NetgenParams(family=NET_LARGE, n_neurons=100, seed=1), BuildOptions(cta_barriers=1))
    assert off.group_tiles_32 == off.group_tiles_64 == 0
    trees = plan_generated(NetgenParams(family=NET_TREES, n_neurons=2, tree_depth=10, seed=1))
    assert trees.group_tiles_32 == trees.group_tiles_64 == 0


def test_plan_aos_accepts_generated_network():
    net = _net(family=1, n_neurons=4, seed=5)
    rc, info = _plan_aos(net)
    assert rc == 0
    assert info.n_segments == 128


def test_unsupported_modifier_type_is_rejected_not_skipped():
    from bioneuroncore_b200 import last_error
    net = _net(family=1, n_neurons=2, seed=5)
    net.segments["modifiers"][3, 0]["type"] = 50   # no device model for this built-in ID
    rc, _ = _plan_aos(net)
    assert rc == BNC_ERR_UNSUPPORTED
    assert "50" in last_error()


def test_user_plugin_type_is_rejected():
    from bioneuroncore_b200 import last_error
    net = _net(family=1, n_neurons=2, seed=5)
    net.segments["modifiers"][0, 1]["type"] = 7 + 0   # NaK pump is supported
    assert _plan_aos(net)[0] == 0
    net.segments["modifiers"][0, 1]["type"] = 60      # user ID range 0-127 without a device entry
    assert _lib().bnc_device_modifier_registered(60) == 0
    assert _plan_aos(net)[0] == BNC_ERR_UNSUPPORTED
    assert last_error()


def test_gap_junction_rules():
    """Electrical synapses and dendritic bridges are accepted; a junction whose segment
    an earlier synapse with an NMDA receptor targets (its Ca2+ would move before the
    junction reads it), a segment with two connexin-36, and synapse types above 2 are
    refused."""
    from bioneuroncore_b200 import NETGEN_GAP_JUNCTIONS, last_error
    net = _net(family=1, n_neurons=4, seed=5, flags=NETGEN_GAP_JUNCTIONS)
    syn = net.synapses
    assert (syn["type"] > 0).sum() == 3 and _plan_aos(net)[0] == 0
    g = int(np.flatnonzero(syn["type"] > 0)[-1])
    k = int(np.flatnonzero(syn["type"][:g] == 0)[0])
    syn["post_segment"][k] = syn["post_segment"][g]
    syn["post_receptors"][k, 0]["type"] = 9                      # NMDA onto the junction's segment, earlier
    assert _plan_aos(net)[0] == BNC_ERR_UNSUPPORTED and "NMDA" in last_error()
    net2 = _net(family=1, n_neurons=4, seed=5, flags=NETGEN_GAP_JUNCTIONS)
    seg = net2.segments
    c = int(seg["modifier_count"][0])
    seg["modifiers"][0, c] = seg["modifiers"][0, int(np.flatnonzero(seg["modifiers"][0]["type"] == 114)[0])]
    seg["modifier_count"][0] = c + 1
    assert _plan_aos(net2)[0] == BNC_ERR_UNSUPPORTED and "connexin" in last_error()
    net3 = _net(family=1, n_neurons=4, seed=5)
    net3.synapses["type"][0] = 3
    assert _plan_aos(net3)[0] == BNC_ERR_UNSUPPORTED


def test_modifier_count_out_of_range_is_a_format_error():
    net = _net(family=1, n_neurons=2, seed=5)
    net.segments["modifier_count"][1] = 33
    assert _plan_aos(net)[0] == BNC_ERR_FORMAT


def _lib():
    from bioneuroncore_b200 import load_library
    return load_library()


def test_bion_roundtrip(tmp_path):
    from bioneuroncore_b200.abi import BionData
    net = _net(family=2, n_neurons=3, n_synapses=40, seed=9)
    path = str(tmp_path / "net.bion").encode()
    assert _lib().bnc_bion_save(path, C.byref(net.data)) == 0
    back = BionData()
    assert _lib().bnc_bion_load(path, C.byref(back)) == 0
    try:
        from bioneuroncore_b200.abi import view, SEGMENT_DTYPE, SYNAPSE_DTYPE
        s = view(back.segments, SEGMENT_DTYPE, back.num_segments)
        y = view(back.synapses, SYNAPSE_DTYPE, back.num_synapses)
        assert back.num_segments == net.data.num_segments and back.num_synapses == 40
        # intra_connection_ids are rebuilt on load, as the reference loader does
        fields = [f for f in SEGMENT_DTYPE.names if f not in ("intra_connection_ids", "intra_connection_count")]
        for f in fields:
            assert s[f].tobytes() == net.segments[f].tobytes(), f
        assert y.tobytes() == net.synapses.tobytes()
    finally:
        _lib().bnc_bion_unload(C.byref(back))


def test_bion_errors(tmp_path):
    from bioneuroncore_b200.abi import BionData
    d = BionData()
    assert _lib().bnc_bion_load(str(tmp_path / "missing.bion").encode(), C.byref(d)) == BNC_BION_ERR_FILE_OPEN
    bad = tmp_path / "bad.bion"
    bad.write_bytes(b"\0" * 200)
    assert _lib().bnc_bion_load(str(bad).encode(), C.byref(d)) == BNC_BION_ERR_BAD_MAGIC
    net = _net(family=1, n_neurons=2, seed=5)
    net.connections["segment_b"][0] = 10 ** 6
    p = str(tmp_path / "conn.bion").encode()
    assert _lib().bnc_bion_save(p, C.byref(net.data)) == 0
    assert _lib().bnc_bion_load(p, C.byref(d)) == BNC_BION_ERR_BAD_CONN


@pytest.mark.skipif(not reference_available(), reason="reference CPU library not built here")
def test_bion_files_interchange_with_the_reference_loader(tmp_path):
    from bioneuroncore_b200.abi import BionData, view, SEGMENT_DTYPE
    ref = C.CDLL(REF_LIB)
    load = getattr(ref, "_Z14bion_load_hostPKcP8BionData")
    save = getattr(ref, "_Z9bion_savePKcPK8BionData")
    unload = getattr(ref, "_Z16bion_unload_hostP8BionData")
    for f in (load, save):
        f.argtypes = [C.c_char_p, C.c_void_p]
        f.restype = C.c_int
    unload.argtypes = [C.c_void_p]
    net = _net(family=1, n_neurons=3, seed=2)
    ours = str(tmp_path / "ours.bion").encode()
    theirs = str(tmp_path / "theirs.bion").encode()
    assert _lib().bnc_bion_save(ours, C.byref(net.data)) == 0
    r = BionData()
    assert load(ours, C.byref(r)) == 0            # the reference reads our file
    assert save(theirs, C.byref(r)) == 0          # and writes it back
    unload(C.byref(r))
    b = BionData()
    assert _lib().bnc_bion_load(theirs, C.byref(b)) == 0   # we read the reference's file
    try:
        s = view(b.segments, SEGMENT_DTYPE, b.num_segments)
        assert s["V_m"].tobytes() == net.segments["V_m"].tobytes()
        assert s["modifiers"].tobytes() == net.segments["modifiers"].tobytes()
        assert b.num_synapses == net.data.num_synapses
    finally:
        _lib().bnc_bion_unload(C.byref(b))


def test_ensemble_params_are_seeded_and_in_range():
    from bioneuroncore_b200 import ensemble_params
    a = ensemble_params(7, 64, 200, 20000)
    b = ensemble_params(7, 64, 200, 20000)
    c = ensemble_params(8, 64, 200, 20000)
    assert bytes(a) == bytes(b) and bytes(a) != bytes(c)
    segs = np.array([m.n_neurons * 32 for m in a])
    assert segs.min() >= 200 - 16 and segs.max() <= 20000 + 16
    assert len(set(m.seed for m in a)) == 64
    scales = np.array([list(m.conductance_scale) for m in a])
    assert scales.min() >= 0.5 and scales.max() <= 2.0
    assert all(m.family == 4 for m in a)


def test_ensemble_plan_is_the_union_of_its_members():
    from bioneuroncore_b200 import ensemble_params, plan_ensemble, plan_generated
    ps = ensemble_params(3, 5, 64, 2000)
    inf = plan_ensemble(ps)
    singles = [plan_generated(p) for p in ps]
    assert inf.n_segments == sum(x.n_segments for x in singles)
    assert inf.n_synapses == sum(x.n_synapses for x in singles)
    assert inf.n_items == sum(x.n_items for x in singles)
    assert inf.n_tiles <= sum(x.n_tiles for x in singles)


def test_ensemble_members_must_agree_on_the_network_switches():
    from bioneuroncore_b200 import ensemble_params, plan_ensemble, BackendError, last_error
    ps = ensemble_params(3, 3, 64, 600)
    ps[1].flags = 1   # BNC_NETGEN_NO_SYNAPSES
    with pytest.raises(BackendError):
        plan_ensemble(ps)
    assert "member 1" in last_error()
