"""The oracle's restatement pinned against the reference's own compiled tick.

oracle/liboracle64.so is oracle/bnc_oracle.c (and bo_*.h) built with -DBO_FP64
-DBO_LIBM: V_m, ions and modifier densities/states are stored as double, as the
reference's Segment and Modifier hold them (types.h:451-500), and exp/log/pow are the
C library's, as the reference's build calls them.  Nothing else differs from the
FP32 oracle that the GPU path is compared with bit for bit.  So if this build equals
the reference's core_run_tick (oracle/_ref, compiled from the reference's sources by
oracle/Makefile) bit for bit, tick after tick, the FP32 oracle computes the
reference's operations in the reference's order, and its remaining distance from the
reference is FP32 storage and the own elementary functions alone.

Every case runs until releases happen; the release decisions (synapse, tick) are
read from the refractory counters, which the reference sets on a release
(simulation_host.cpp:458) and counts down every tick (:591), and must be identical.
The release draw itself is checked on random inputs through the reference's own
xorshift32_rnd and seed expression (oracle/ref_harness.cpp).
"""
import ctypes as C

import numpy as np
import pytest

from oracle.oracle import Oracle, Reference, oracle64_lib, reference_available, REF_LIB

pytestmark = pytest.mark.skipif(not reference_available(), reason="reference CPU library not built here")

DT = 0.025


def _net(family, n, seed, flags=0, stim_pA=0.0, tree_depth=0):
    from bioneuroncore_b200 import Network, NetgenParams
    return Network(NetgenParams(family=family, n_neurons=n, seed=seed, flags=flags, stim_pA=stim_pA,
                                tree_depth=tree_depth))


def _fresh_reference(net):
    """A Reference whose static delay buffer starts empty: core_run_tick keeps it in a
    function-local static that it only clears when the synapse count changes
    (simulation_host.cpp:322-326, 679-682), so a call with no synapses comes first."""
    ref = Reference(net)
    zero = C.c_uint32(0)
    tick = C.c_uint64(0)
    ref.lib.core_run_tick(None, 0, None, 0, None, 0, 0, C.byref(tick), C.c_float(DT), None, C.byref(zero),
                          *([None] * 10))
    return ref


def _seg_fields(net):
    seg = net.segments
    out = {"V": seg["V_m"], "ATP": seg["ATP_level"], "temperature": seg["temperature"],
           "transcription": seg["transcription_signal"]}
    for q in range(7):
        out["ion_in[%d]" % q] = seg["intra_ions"][:, q]
        out["ion_out[%d]" % q] = seg["extra_ions"][:, q]
    for q in range(15):
        out["intra_nt[%d]" % q] = seg["intra_nt"][:, q]
        out["neurotransmitter[%d]" % q] = seg["neurotransmitter"][:, q]
    nmod = int(seg["modifier_count"].max())
    for j in range(nmod):
        for k in range(7):
            st = np.where(seg["modifier_count"] > j, seg["modifiers"][:, j]["state"][:, k], 0.0)
            out["mod_state[%d]" % (j * 8 + k)] = st
    return out


def _syn_fields(net):
    syn = net.synapses
    out = {}
    for f in ("bouton_Ca", "spine_Ca", "weight", "refractory", "facilitation", "depression", "spine_camkii",
              "spine_calcineurin", "RRP"):
        out[f] = syn[f]
    for q in range(15):
        out["cleft[%d]" % q] = syn["cleft_neurotransmitter"][:, q]
    nrec = int(syn["post_receptor_count"].max()) if len(syn) else 0
    for j in range(nrec):
        for k in range(7):
            out["receptor_state[%d]" % (j * 8 + k)] = np.where(
                syn["post_receptor_count"] > j, syn["post_receptors"][:, j]["state"][:, k], 0.0)
    return out


def _oracle_value(ora, name):
    base, _, idx = name.partition("[")
    idx = int(idx[:-1]) if idx else 0
    if base in ("bouton_Ca", "spine_Ca", "weight", "refractory", "facilitation", "depression", "spine_camkii",
                "spine_calcineurin", "RRP", "cleft", "receptor_state"):
        return ora.synapse_field(base, idx)
    return ora.segment_field(base, idx)


def _assert_same(net_r, ora, names=None):
    ref_vals = dict(_seg_fields(net_r))
    if net_r.data.num_synapses:
        ref_vals.update(_syn_fields(net_r))
    bad = []
    for name, want in ref_vals.items():
        if names is not None and name not in names:
            continue
        got = _oracle_value(ora, name)
        want = np.asarray(want, np.float64)
        if not np.array_equal(got, want):
            bad.append((name, float(np.abs(got - want).max())))
    assert not bad, "FP64 oracle differs from the reference's tick: %r" % bad[:8]


def _decisions(before, after, tick):
    """(synapse, tick) of every release decided this tick: a synapse can release only
    while its refractory counter is 0, and a release leaves it above 0."""
    return [(int(i), tick) for i in np.flatnonzero((before == 0) & (after > 0))]


def _run_pinned(net_r, net_o, ticks, schedule=(), full_every=50):
    """Runs both a tick at a time and compares; returns the release decision log."""
    ref = _fresh_reference(net_r)
    ora = Oracle(net_o, fp64=True)
    sched = dict(schedule)
    log_r, log_o = [], []
    every_tick = {"V", "refractory", "bouton_Ca", "RRP"} | {"cleft[%d]" % q for q in range(15)}
    for t in range(ticks):
        if t in sched:
            ref.upload_stimuli(sched[t])
            ora.upload_stimuli(sched[t])
        if net_r.data.num_synapses:
            rb = net_r.synapses["refractory"].copy()
            ob = ora.synapse_field("refractory")
        ref.run(1, DT)
        ora.run(1, DT)
        if net_r.data.num_synapses:
            log_r += _decisions(rb, net_r.synapses["refractory"], t)
            log_o += _decisions(ob, ora.synapse_field("refractory"), t)
        _assert_same(net_r, ora, None if (t + 1) % full_every == 0 or t + 1 == ticks else every_tick)
    assert log_r == log_o, "release decisions differ"
    ora.close()
    return log_r


def test_small_network_with_stimuli_bit_identical():
    from bioneuroncore_b200 import NET_SMALL
    _run_pinned(_net(NET_SMALL, 8, 7), _net(NET_SMALL, 8, 7), 200)


def test_full_small_workload_bit_identical():
    """The small workload at its full size: 64 neurons x 32 segments, 400 synapses,
    4,000 ticks (compared every tick on V and synapse state, everything every 500)."""
    from bioneuroncore_b200 import NET_SMALL
    _run_pinned(_net(NET_SMALL, 64, 7), _net(NET_SMALL, 64, 7), 4000, full_every=500)


def test_trees_with_perturbed_ions_bit_identical():
    """Binary dendritic trees (the electrodiffusion workload's morphology) with ions
    perturbed per segment, so every Nernst-Planck flux and the bath relaxation act."""
    from bioneuroncore_b200 import NET_TREES, NETGEN_PERTURB_IONS
    spec = dict(family=NET_TREES, n=3, seed=11, flags=NETGEN_PERTURB_IONS, tree_depth=6)
    _run_pinned(_net(**spec), _net(**spec), 100)


def test_large_set_with_releases_bit_identical():
    """All 24 large-set models and 8 receptors per synapse; releases from ~100 ticks on."""
    from bioneuroncore_b200 import NET_LARGE
    log = _run_pinned(_net(NET_LARGE, 12, 3), _net(NET_LARGE, 12, 3), 400)
    assert len(log) > 0, "the case must release"


def test_synapse_extras_with_releases_bit_identical():
    """Readily releasable pools, bouton autoreceptor channels and delayed releases
    (the delay buffer), 1,000 ticks of the small family driven by 3 nA somatic steps."""
    from bioneuroncore_b200 import NET_SMALL, NETGEN_SYNAPSE_EXTRAS
    spec = dict(family=NET_SMALL, n=16, seed=6, flags=NETGEN_SYNAPSE_EXTRAS, stim_pA=3000.0)
    net_r = _net(**spec)
    syn = net_r.synapses
    assert (syn["RRP_max"] > 0).any() and (syn["pre_autoreceptor_count"] > 0).any() and (syn["delay"] > 0).any()
    log = _run_pinned(net_r, _net(**spec), 1000, full_every=100)
    assert len(log) > 0, "the case must release"
    released = {s for s, _ in log}
    assert any(syn["delay"][s] > 0 for s in released), "a delayed synapse must release"
    assert any(syn["RRP_max"][s] > 0 for s in released), "a synapse with a pool must release"
    assert any(syn["pre_autoreceptor_count"][s] > 0 for s in released), "a synapse with autoreceptors must release"


def test_release_modulators_bit_identical():
    """Presynaptic release-modulator autoreceptors (Gi/o, Gs and ionotropic types,
    receptors_biological.cpp:428-509) beside bouton channels, pools and delays: the
    modulators' state[0] and every release decision, 1,000 ticks."""
    from bioneuroncore_b200 import NET_SMALL, NETGEN_SYNAPSE_EXTRAS, NETGEN_RELEASE_MODULATORS
    spec = dict(family=NET_SMALL, n=16, seed=6, flags=NETGEN_SYNAPSE_EXTRAS | NETGEN_RELEASE_MODULATORS,
                stim_pA=3000.0)
    net_r = _net(**spec)
    syn = net_r.synapses
    types = {int(syn["pre_autoreceptors"][k, j]["type"]) for k in range(len(syn))
             for j in range(int(syn["pre_autoreceptor_count"][k]))}
    assert {29, 30} & types and types & {18, 19, 22, 27, 35, 36, 38} and types & {44, 46}
    log = _run_pinned(net_r, _net(**spec), 1000, full_every=100)
    assert len(log) > 0, "the case must release"
    ora_net = _net(**spec)
    ora = Oracle(ora_net, fp64=True)
    ref = _fresh_reference(net_r2 := _net(**spec))
    ora.run(300, DT)
    ref.run(300, DT)
    for j in range(3):
        want = np.where(net_r2.synapses["pre_autoreceptor_count"] > j,
                        net_r2.synapses["pre_autoreceptors"][:, j]["state"][:, 0], 0.0)
        assert np.array_equal(ora.synapse_field("autoreceptor_state", j * 8), want), j
    ora.close()


def test_endocannabinoid_signalling_bit_identical():
    """eCB synthesis on the post segments (hh_biological.cpp:1746-1767), its retrograde
    release into each cleft with the modifier's decay per synapse
    (simulation_host.cpp:578-589), and CB1 autoreceptors reading it: 1,000 ticks with
    releases, every state word and release decision equal."""
    from bioneuroncore_b200 import NET_SMALL, NETGEN_SYNAPSE_EXTRAS, NETGEN_ECB
    spec = dict(family=NET_SMALL, n=16, seed=6, flags=NETGEN_SYNAPSE_EXTRAS | NETGEN_ECB, stim_pA=3000.0)
    net_r = _net(**spec)
    assert (net_r.segments["modifiers"]["type"] == 86).any()
    log = _run_pinned(net_r, _net(**spec), 1000, full_every=100)
    assert len(log) > 0
    assert (net_r.synapses["cleft_neurotransmitter"][:, 9] > 0).any(), "eCB must reach the clefts"


def test_glial_capture_bit_identical():
    """Glial segments (a GLAST transporter, hh_biological.cpp:725-733): each cleft
    hands a share of its glutamate, glycine or GABA to the glial segment nearest in z
    instead of clearing it (simulation_host.cpp:467-487, 505-510), and the transporter
    takes it up in step 1; 1,000 ticks with releases, everything equal."""
    from bioneuroncore_b200 import NET_SMALL, NETGEN_SYNAPSE_EXTRAS, NETGEN_GLIA
    spec = dict(family=NET_SMALL, n=16, seed=6, flags=NETGEN_SYNAPSE_EXTRAS | NETGEN_GLIA, stim_pA=3000.0)
    net_r = _net(**spec)
    glial = np.flatnonzero((net_r.segments["modifiers"]["type"] == 147).any(axis=1))
    assert len(glial) > 1
    log = _run_pinned(net_r, _net(**spec), 1000, full_every=100)
    assert len(log) > 0
    nt = net_r.segments["neurotransmitter"]
    assert (nt[glial][:, [0, 1, 7]] > 0).any(), "the glia must have taken up transmitter"


def test_gap_junctions_bit_identical():
    """Electrical synapses and dendritic bridges between somata (simulation_host.cpp:
    373-402; run_tick_common.h:79-122): connexin-36/43 models in step 1, the slow
    Ca2+/CaM gate, Cx43's Vj gate, the filtered current of delayed junctions, both
    segments' I_buffer in synapse order among the chemical synapses; 1,000 ticks."""
    from bioneuroncore_b200 import NET_SMALL, NETGEN_GAP_JUNCTIONS
    spec = dict(family=NET_SMALL, n=16, seed=6, flags=NETGEN_GAP_JUNCTIONS, stim_pA=3000.0)
    net_r = _net(**spec)
    syn = net_r.synapses
    assert (syn["type"] == 1).any() and (syn["type"] == 2).any()
    log = _run_pinned(net_r, _net(**spec), 1000, full_every=100)
    assert len(log) > 0
    gj = syn["type"] > 0
    assert (syn["depression"][gj] > 0).all() and (syn["cleft_neurotransmitter"][gj & (syn["delay"] > 0), 0] != 0).any()


def mechano_schedule(net):
    """Mechano stimuli at three ticks of the small family (tick -> (segment_id, mod_type,
    state_idx, value) list): a gate (dynamic word), parameter words of Nav1.x and K2P,
    the effective-area word 7, the Kv delayed rectifier of a myelinated axon segment
    (myelin blocks it: kernel_dispatch.h:301-309, so its modifier never runs), and
    stimuli that match nothing (absent type, index out of range, absent segment id);
    two on one slot in one call, the later winning."""
    seg = net.segments
    types = seg["modifiers"]["type"]
    cnt = seg["modifier_count"]

    def first(t, pred=lambda i: True):
        for i in range(len(seg)):
            if pred(i) and t in types[i, :cnt[i]]:
                return int(seg["id"][i])
        raise AssertionError("no segment with type %d" % t)
    myel = lambda i: 4 in types[i, :cnt[i]]                        # noqa: E731
    nav = 141 if (types == 141).any() else 142
    s_kv, s_k2p, s_nav = first(123), first(107), first(nav, lambda i: not myel(i))
    s_blocked = first(123, myel)
    return {
        20: [(s_kv, 123, 0, 0.9), (s_nav, nav, 5, 4.0), (s_k2p, 107, 0, 3.5), (s_k2p, 107, 7, 123.0),
             (s_blocked, 123, 0, 0.7), (s_kv, 200, 0, 1.0), (s_kv, 123, 9, 1.0), (10 ** 7, 123, 0, 1.0)],
        60: [(s_kv, 123, 0, 0.2), (s_kv, 123, 0, 0.95), (s_nav, nav, 1, 0.1)],
        61: [(s_k2p, 107, 1, 2.0)],
    }


def test_mechano_stimuli_bit_identical():
    """Mechano stimuli, core_run_tick's own argument (simulation_host.cpp:211-230): one
    shot, before the tick's modifier currents; every state word after each call and
    200 ticks equal."""
    from bioneuroncore_b200 import NET_SMALL
    net_r, net_o = _net(NET_SMALL, 8, 7, stim_pA=3000.0), _net(NET_SMALL, 8, 7, stim_pA=3000.0)
    sched = mechano_schedule(net_r)
    ref = _fresh_reference(net_r)
    ora = Oracle(net_o, fp64=True)
    for t in range(200):
        if t in sched:
            ref.upload_mechano(sched[t])
            ora.upload_mechano(sched[t])
        ref.run(1, DT)
        ora.run(1, DT)
        if t in sched or t + 1 == 200:
            _assert_same(net_r, ora)
    ora.close()


def test_stimulus_uploads_bit_identical():
    """Every stimulus kind of GpuStimulusData, uploaded twice (the stimuli fixture's schedule)."""
    import golden_cases
    from bioneuroncore_b200 import NET_SMALL
    net_r, net_o = _net(NET_SMALL, 8, 7), _net(NET_SMALL, 8, 7)
    sched = golden_cases.stimulus_schedule("stimuli_n8_s7", net_r)
    assert sched
    _run_pinned(net_r, net_o, 200, schedule=sched)


def _harness():
    lib = C.CDLL(REF_LIB.replace("libbiocore_ref.so", "libref_harness.so"))
    lib.ref_xorshift32_rnd.argtypes = [C.c_uint32]; lib.ref_xorshift32_rnd.restype = C.c_float
    lib.ref_release_seed.argtypes = [C.c_uint32, C.c_uint64, C.c_double]; lib.ref_release_seed.restype = C.c_uint32
    lib.ref_release_decision.argtypes = [C.c_uint32, C.c_uint64, C.c_double, C.c_float]
    lib.ref_release_decision.restype = C.c_int
    return lib


def test_release_draw_matches_the_reference():
    """The seed id ^ tick ^ (uint32)(V_m*1000) and the xorshift32 draw of the oracle
    (both builds) against the reference's own code on random (id, tick, V_m, p),
    negative V_m included, and on the FP32-representable V_m the FP32 state holds."""
    h = _harness()
    o64 = oracle64_lib()
    from oracle.oracle import oracle_lib
    o32 = oracle_lib()
    rng = np.random.default_rng(20261204)
    n = 200000
    ids = rng.integers(0, 2**32, n, dtype=np.uint64)
    ticks = rng.integers(0, 2**40, n, dtype=np.uint64)
    V = rng.uniform(-130.0, 160.0, n)
    V[:1000] = np.round(V[:1000], 1)          # values near the x1000 rounding boundaries
    V32 = V.astype(np.float32).astype(np.float64)
    p = rng.uniform(0.0, 1.0, n).astype(np.float32)
    for i in range(n):
        sid, tk = int(ids[i]), int(ticks[i])
        for v, ora in ((float(V[i]), o64), (float(V32[i]), o32)):
            seed_ref = h.ref_release_seed(sid, tk, v)
            seed_ora = (sid ^ (tk & 0xFFFFFFFF)) ^ ora.bo_seed_bits(v)
            assert seed_ref == seed_ora, (sid, tk, v)
        assert h.ref_xorshift32_rnd(seed_ref) == o32.bo_xorshift_f(seed_ref)
        assert h.ref_release_decision(sid, tk, float(V32[i]), float(p[i])) == \
            int(o32.bo_xorshift_f(seed_ref) < float(p[i]))


def test_protein_mapping_matches_the_reference():
    """The nucleus protein -> release parameter mapping of the oracle against the
    reference's own rrp_apply_protein_mapping (kernel_dispatch.h:651-663), through
    oracle/ref_harness.cpp, on random protein levels that reach both clamps."""
    h = C.CDLL(REF_LIB.replace("libbiocore_ref.so", "libref_harness.so"))
    h.ref_protein_mapping.argtypes = [C.c_void_p, C.c_void_p]
    from oracle.oracle import oracle_lib
    o = oracle_lib()
    o.bo_protein_mapping.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(7)
    for _ in range(2000):
        pl = rng.uniform(-3.0, 3.0, 57).astype(np.float32)
        want = np.zeros(3, np.float32)
        h.ref_protein_mapping(pl.ctypes.data, want.ctypes.data)
        got = np.zeros(3, np.float32)
        o.bo_protein_mapping(pl.ctypes.data, got[0:].ctypes.data, got[1:].ctypes.data, got[2:].ctypes.data)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def _nuclei(n, seed):
    """n 500-byte nucleus records (types.h:508-524) with random protein levels."""
    rng = np.random.default_rng(seed)
    buf = np.zeros(n * 500, np.uint8)
    for i in range(n):
        buf[i * 500:i * 500 + 4] = np.frombuffer(np.uint32(i).tobytes(), np.uint8)
        buf[i * 500 + 244:i * 500 + 244 + 57 * 4] = np.frombuffer(rng.uniform(0.0, 1.5, 57).astype(np.float32).tobytes(),
                                                                 np.uint8)
    return buf


def test_nuclei_are_read_as_the_reference_reads_them(tmp_path):
    """A .bion with nuclei written by the reference's bion_save (500-byte records), and
    the same file rewritten with the 46-gene 412-byte records of older files: this
    library's reader returns the reference loader's nucleus records byte for byte."""
    from bioneuroncore_b200 import Network, NetgenParams, NET_SMALL, load_library
    from bioneuroncore_b200.abi import BionData
    ref = C.CDLL(REF_LIB)
    load = getattr(ref, "_Z14bion_load_hostPKcP8BionData")
    save = getattr(ref, "_Z9bion_savePKcPK8BionData")
    unload = getattr(ref, "_Z16bion_unload_hostP8BionData")
    for f in (load, save):
        f.argtypes = [C.c_char_p, C.c_void_p]
        f.restype = C.c_int
    unload.argtypes = [C.c_void_p]
    net = Network(NetgenParams(family=NET_SMALL, n_neurons=4, seed=2))
    nu = _nuclei(4, 3)
    net.data.nuclei = nu.ctypes.data
    net.data.num_nuclei = 4
    p500 = tmp_path / "n500.bion"
    try:
        assert save(str(p500).encode(), C.byref(net.data)) == 0
    finally:
        net.data.nuclei = None
        net.data.num_nuclei = 0
    raw = bytearray(p500.read_bytes())
    hdr = 100
    n_nuc_off = len(raw) - 4 * 500
    old = bytearray()
    for i in range(4):
        r = raw[n_nuc_off + i * 500:n_nuc_off + (i + 1) * 500]
        rec = bytearray(412)
        rec[0:16] = r[0:16]
        rec[16:16 + 184] = r[16:16 + 184]          # genes 0..45 of gene_activity
        rec[200:200 + 184] = r[244:244 + 184]      # genes 0..45 of protein_level
        rec[384:408] = r[472:496]                  # the six levels after them
        old += rec
    raw412 = raw[:n_nuc_off] + old
    struct_off = 84   # NetworkHeader.file_sz_nucleus (types.h:577-599)
    raw412[struct_off:struct_off + 4] = np.uint32(412).tobytes()
    p412 = tmp_path / "n412.bion"
    p412.write_bytes(bytes(raw412))
    lib = load_library()
    for path in (p500, p412):
        r, o = BionData(), BionData()
        assert load(str(path).encode(), C.byref(r)) == 0
        assert lib.bnc_bion_load(str(path).encode(), C.byref(o)) == 0
        try:
            assert r.num_nuclei == o.num_nuclei == 4
            assert C.string_at(r.nuclei, 4 * 500) == C.string_at(o.nuclei, 4 * 500), path.name
        finally:
            unload(C.byref(r))
            lib.bnc_bion_unload(C.byref(o))
