"""GPU tick vs the CPU oracle, through the C ABI.

The kernels restate the reference's arithmetic operation by operation with FP32
state (the oracle's precision rule), the same elementary functions and no fused
multiply-adds, and every accumulation follows the reference's loop order.  So the
bar here is bit-exact equality of every state variable, tick by tick: V_m, ions,
modifier gates, synapse state, spike counts and release decisions.  Networks are
small seeded instances of the workload families.
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
    ora = Oracle(net_o)
    gpu = Backend()
    gpu.load_network(net_g)
    return ora, gpu, net_g


def _assert_same(a, b, what):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    same = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
    if not same.all():
        i = int(np.argmax(~same))
        raise AssertionError("%s differs at %d of %d: gpu %r oracle %r (%d mismatches)"
                             % (what, i, a.size, a[i], b[i], int((~same).sum())))


SEG_CHECKS = [("V", 0)] + [("ion_in", q) for q in range(7)] + [("ion_out", q) for q in range(7)] + [
    ("ATP", 0), ("temperature", 0), ("transcription", 0), ("spikes", 0)] + [("neurotransmitter", q) for q in (0, 1, 7)]
SYN_CHECKS = [("bouton_Ca", 0), ("spine_Ca", 0), ("weight", 0), ("refractory", 0), ("facilitation", 0),
              ("spine_camkii", 0), ("spine_calcineurin", 0), ("cleft", 0), ("cleft", 1),
              ("receptor_state", 0), ("receptor_state", 1), ("RRP", 0)]


def _compare_all(ora, gpu, n_syn, label):
    for f, i in SEG_CHECKS:
        _assert_same(gpu.segment_field(f, i), ora.segment_field(f, i), "%s %s[%d]" % (label, f, i))
    for slot in range(6):
        for k in range(3):
            _assert_same(gpu.segment_field("mod_state", slot * 8 + k), ora.segment_field("mod_state", slot * 8 + k),
                         "%s modifier slot %d state %d" % (label, slot, k))
    if n_syn:
        for f, i in SYN_CHECKS:
            _assert_same(gpu.synapse_field(f, i, n_syn), ora.synapse_field(f, i), "%s synapse %s[%d]" % (label, f, i))


@pytest.mark.parametrize("flags", [0, 1 | 2, 1, 2, 32])
def test_small_network_bitexact(flags):
    from bioneuroncore_b200 import NetgenParams, NET_SMALL
    p = NetgenParams(family=NET_SMALL, n_neurons=16, seed=11, flags=flags)
    ora, gpu, net = _pair(p)
    for step in (1, 9, 40):
        ora.run(step, DT)
        gpu.run_ticks(step, DT)
        _compare_all(ora, gpu, net.data.num_synapses, "small flags=%d after +%d" % (flags, step))


@pytest.mark.parametrize("flags", [0, 32])
def test_large_set_bitexact(flags):
    from bioneuroncore_b200 import NetgenParams, NET_LARGE
    p = NetgenParams(family=NET_LARGE, n_neurons=12, n_synapses=300, seed=5, flags=flags)
    ora, gpu, net = _pair(p)
    for step in (1, 20, 30):
        ora.run(step, DT)
        gpu.run_ticks(step, DT)
        _compare_all(ora, gpu, net.data.num_synapses, "large after +%d" % step)


@pytest.mark.parametrize("name", __import__("golden_cases").cases())
def test_gpu_matches_reference_fixture(name):
    """The GPU path against the reference's own FP64 CPU tick (fixtures made by
    tests/golden/make_golden.py), within the relative tolerance of golden_cases."""
    import golden_cases
    from bioneuroncore_b200 import Backend, Network, NetgenParams
    g, spec = golden_cases.load(name)
    net = Network(NetgenParams(**spec))
    gpu = Backend()
    gpu.load_network(net)
    n_syn = net.data.num_synapses
    log = None
    if "release_syn" in g.files:
        trace, log = golden_cases.run_scheduled(gpu, name, net, int(g["ticks"]), float(g["dt"]), g["somata"],
                                                lambda: gpu.segment_field("V"),
                                                read_refractory=lambda: gpu.synapse_field("refractory", 0, n_syn))
        assert len(log) > 0
    else:
        trace = golden_cases.run_scheduled(gpu, name, net, int(g["ticks"]), float(g["dt"]), g["somata"],
                                           lambda: gpu.segment_field("V"))
    golden_cases.compare(g, trace, gpu.segment_field, lambda f: gpu.synapse_field(f, 0, n_syn), log=log)


@pytest.mark.parametrize("chunk", [64, 300])
def test_chunked_modifier_pass_bitexact(chunk):
    """The modifier pass run chunk by chunk (all phases of a chunk of segments before
    the next) computes what the oracle computes: chunking only reorders independent
    segments."""
    from bioneuroncore_b200 import Backend, BuildOptions, Network, NetgenParams, NET_LARGE
    p = NetgenParams(family=NET_LARGE, n_neurons=12, n_synapses=300, seed=5)
    ora = Oracle(Network(p))
    gpu = Backend()
    gpu.load_generated(p, BuildOptions(chunk_segs=chunk))
    n_syn = ora.n_syn
    for step in (1, 20):
        ora.run(step, DT)
        gpu.run_ticks(step, DT)
        _compare_all(ora, gpu, n_syn, "chunk %d after +%d" % (chunk, step))


@pytest.mark.parametrize("family,cta_barriers", [("small", 0), ("small", 1), ("large", 0), ("large", 1)])
def test_diffusion_barrier_groups_bitexact(family, cta_barriers):
    """The diffusion kernel with barriers over a warp (32-segment neurons) or a pair of
    warps (64-segment neurons), and with CTA-wide barriers: both are the oracle's tick,
    bit for bit, through releases."""
    from bioneuroncore_b200 import Backend, BuildOptions, Network, NetgenParams, NET_LARGE, NET_SMALL
    if family == "small":
        p = NetgenParams(family=NET_SMALL, n_neurons=40, seed=6, flags=32, stim_pA=3000.0)
    else:
        p = NetgenParams(family=NET_LARGE, n_neurons=20, seed=3)
    ora = Oracle(Network(p))
    gpu = Backend()
    gpu.load_generated(p, BuildOptions(cta_barriers=cta_barriers))
    info = gpu.info()
    grouped = info.group_tiles_32 + info.group_tiles_64
    assert (grouped == 0) if cta_barriers else (grouped == info.n_tiles)
    n_syn = ora.n_syn
    for step in (1, 99, 200):
        ora.run(step, DT)
        gpu.run_ticks(step, DT)
        label = "%s cta_barriers=%d after +%d" % (family, cta_barriers, step)
        for f, i in SEG_CHECKS:
            _assert_same(gpu.segment_field(f, i), ora.segment_field(f, i), "%s %s[%d]" % (label, f, i))
        # gate words of the channel slots (a generated network loaded without host
        # records reads back only the state words its models update)
        for slot in range(5):
            for k in range(2):
                _assert_same(gpu.segment_field("mod_state", slot * 8 + k), ora.segment_field("mod_state", slot * 8 + k),
                             "%s modifier slot %d state %d" % (label, slot, k))
        for f, i in SYN_CHECKS:
            _assert_same(gpu.synapse_field(f, i, n_syn), ora.synapse_field(f, i), "%s synapse %s[%d]" % (label, f, i))


@pytest.mark.parametrize("fuse", [1, 3, 4, 17])
def test_fused_modifier_phases_bitexact(fuse):
    """Several modifier phases per launch (each segment's items of those phases run on
    its record in registers) compute what the oracle computes, bit for bit; so do one
    launch per phase and one launch for all 17 phases.  The large set has 16 modifiers
    per segment (17 on axon segments with Cav2.1), so groups of 3 and 4 leave a
    shorter last group."""
    from bioneuroncore_b200 import Backend, BuildOptions, Network, NetgenParams, NET_LARGE
    p = NetgenParams(family=NET_LARGE, n_neurons=12, n_synapses=300, seed=6)
    ora = Oracle(Network(p))
    gpu = Backend()
    gpu.load_generated(p, BuildOptions(fuse_phases=fuse))
    info = gpu.info()
    assert info.fuse_phases == fuse
    assert info.modifier_launches == 1 + -(-info.n_phases // fuse)
    n_syn = ora.n_syn
    for step in (1, 20):
        ora.run(step, DT)
        gpu.run_ticks(step, DT)
        _compare_all(ora, gpu, n_syn, "fuse %d after +%d" % (fuse, step))


def test_trees_bitexact():
    """Depth-10 dendritic trees (2,047 segments each) exceed one CTA's tile: each tree
    runs on a 2-CTA cluster, its halves exchanging ghost segments through distributed
    shared memory.  The result must still be the oracle's, bit for bit."""
    from bioneuroncore_b200 import NetgenParams, NET_TREES
    p = NetgenParams(family=NET_TREES, n_neurons=3, tree_depth=10, seed=8, flags=8)   # perturbed ions
    ora, gpu, net = _pair(p)
    assert gpu.info().n_tiles % 2 == 0
    for step in (1, 9, 20):
        ora.run(step, DT)
        gpu.run_ticks(step, DT)
        _compare_all(ora, gpu, 0, "trees after +%d" % step)


def test_components_split_across_a_cluster_bitexact():
    """The large set with 48-segment tiles: every 64-segment neuron spans a tile pair,
    with synapses, stimuli and all 24 channel types."""
    from bioneuroncore_b200 import Backend, BuildOptions, Network, NetgenParams, NET_LARGE
    p = NetgenParams(family=NET_LARGE, n_neurons=6, n_synapses=200, seed=9)
    ora = Oracle(Network(p))
    gpu = Backend()
    gpu.load_generated(p, BuildOptions(tile_segs=48))
    assert gpu.info().n_tiles == 12
    for step in (1, 20):
        ora.run(step, DT)
        gpu.run_ticks(step, DT)
        _compare_all(ora, gpu, ora.n_syn, "split components after +%d" % step)


def _mode_net(case):
    from bioneuroncore_b200 import NetgenParams, NET_TREES, NET_LARGE, NET_SMALL, NETGEN_PERTURB_IONS
    if case == "trees":   # 2,047-segment trees on 2-CTA clusters
        return NetgenParams(family=NET_TREES, n_neurons=3, tree_depth=10, seed=8, flags=NETGEN_PERTURB_IONS)
    if case == "large":   # one tile holding twelve neurons (twelve convergence groups)
        return NetgenParams(family=NET_LARGE, n_neurons=12, n_synapses=300, seed=5)
    if case == "split":   # 48-segment tiles: each 64-segment neuron on its own tile pair
        return NetgenParams(family=NET_LARGE, n_neurons=6, n_synapses=200, seed=9)
    return NetgenParams(family=NET_SMALL, n_neurons=16, seed=11)


@pytest.mark.parametrize("case", ["trees", "large", "split", "small"])
@pytest.mark.parametrize("cap", [100000, 5])
def test_residual_diffusion_mode_bitexact(case, cap):
    """The residual-controlled FP64 Jacobi mode and the ion ledger (bnc_set_diffusion_mode)
    against the oracle's restatement of the same mode: the state bit for bit, the same
    sweep counts and capped group solves (each convergence group -- a connected
    component -- stops on its own, as the oracle's loop over groups does), and the FP64
    ledger within summation-order rounding (1e-9 relative)."""
    from bioneuroncore_b200 import Backend, BuildOptions, Network, DIFFUSION_RESIDUAL, DIFFUSION_LEDGER
    p = _mode_net(case)
    ora = Oracle(Network(p))
    gpu = Backend()
    if case == "split":
        gpu.load_generated(p, BuildOptions(tile_segs=48))
    else:
        gpu.load_network(Network(p))
    flags = DIFFUSION_RESIDUAL | DIFFUSION_LEDGER
    ora.set_diffusion_mode(flags, 1e-6, cap)
    gpu.set_diffusion_mode(flags, 1e-6, cap)
    n_syn = ora.n_syn
    for step in (1, 3):
        ora.run(step, DT)
        gpu.run_ticks(step, DT)
        _compare_all(ora, gpu, n_syn, "%s residual cap %d after +%d" % (case, cap, step))
    st_o, led_o = ora.diffusion_stats()
    st = gpu.diffusion_stats()
    assert (st.max_sweeps_v, st.max_sweeps_phi, st.capped_v, st.capped_phi) == tuple(int(x) for x in st_o)
    if cap == 5:
        assert st.capped_v > 0
    else:
        assert st.capped_v == 0 and st.capped_phi == 0
    led = np.array(list(st.rounding) + list(st.bath))
    assert np.all(np.abs(led - led_o) <= 1e-9 * np.abs(led_o).max() + 1e-300), (led, led_o)


def test_ledger_closes_the_mass_balance_on_the_gpu():
    """On a network where only step 2.5 moves ions, each ion's total amount in the
    device state (FP32, summed in FP64) changes by the device ledger's rounding plus
    bath terms, up to FP64 rounding of the sums."""
    import test_diffusion_modes as tdm
    from bioneuroncore_b200 import Backend, DIFFUSION_LEDGER
    net = tdm.diffusion_only(depth=10)
    ora = Oracle(tdm.diffusion_only(depth=10))   # the volumes the updates divide by
    vol = ora.segment_field(10).astype(np.float64)
    vx = (ora.segment_field(10) * tdm.EXTRA_VOLUME_RATIO).astype(np.float64)
    gpu = Backend()
    gpu.load_network(net)
    gpu.set_diffusion_mode(DIFFUSION_LEDGER)

    def amounts():
        return np.array([(np.asarray(gpu.segment_field("ion_in", q), np.float64) * vol).sum() +
                         (np.asarray(gpu.segment_field("ion_out", q), np.float64) * vx).sum() for q in range(7)])

    before = amounts()
    gpu.run_ticks(5, DT)
    after = amounts()
    st = gpu.diffusion_stats()
    booked = np.array(st.rounding) + np.array(st.bath)
    assert np.all(np.abs((after - before) - booked) <= 1e-11 * (np.abs(before) + 1.0)), (after - before, booked)


def _compare_nt(ora, gpu, label):
    for f in ("intra_nt", "neurotransmitter"):
        for q in range(15):
            _assert_same(gpu.segment_field(f, q), ora.segment_field(f, q), "%s %s[%d]" % (label, f, q))


@pytest.mark.parametrize("graph", [False, True])
def test_stimulus_uploads_bitexact(graph):
    """gpu_backend_upload_stimuli with every stimulus kind, twice: current steps, ramps
    (rising, falling, empty, flat), voltage clamps (overlapping on one segment), ion
    injections (repeated into one ion, extracellular, invalid index and segment) and
    ligand injections (intracellular, which turns on intra_nt diffusion, and
    extracellular, which the synapse pass wipes).  Injections apply once, at the next
    tick; each upload replaces every list.  Through plain launches and through the
    captured tick loop, which an upload must invalidate."""
    import golden_cases
    from bioneuroncore_b200 import NetgenParams, NET_SMALL
    p = NetgenParams(family=NET_SMALL, n_neurons=8, seed=7)
    ora, gpu, net = _pair(p)
    (t0, first), (t1, second) = golden_cases.stimulus_schedule("stimuli", net)
    assert (t0, t1) == (0, 100)
    run = gpu.run_ticks_graph if graph else gpu.run_ticks
    n_syn = net.data.num_synapses
    ora.upload_stimuli(first)
    gpu.upload_stimuli(first)
    for step in (1, 40, 59):
        ora.run(step, DT)
        run(step, DT)
        _compare_all(ora, gpu, n_syn, "first upload, graph=%s, +%d" % (graph, step))
        _compare_nt(ora, gpu, "first upload +%d" % step)
    ora.upload_stimuli(second)
    gpu.upload_stimuli(second)
    for step in (1, 64, 35):
        ora.run(step, DT)
        run(step, DT)
        _compare_all(ora, gpu, n_syn, "second upload, graph=%s, +%d" % (graph, step))
        _compare_nt(ora, gpu, "second upload +%d" % step)


def test_injections_without_synapses_bitexact():
    """On dendritic trees (no synapses) an extracellular ligand injection stays in the
    neurotransmitter field and diffuses through step 2.5, as intracellular ones and
    ions do; ramps and clamps act as on any network."""
    from bioneuroncore_b200 import NetgenParams, NET_TREES
    from bioneuroncore_b200.abi import stimulus_data
    p = NetgenParams(family=NET_TREES, n_neurons=2, tree_depth=6, seed=4)
    ora, gpu, net = _pair(p)
    n = int(net.data.num_segments)
    data = stimulus_data(ramps=[(0, 100.0, -40.0, 2, 60)], vclamps=[(n - 1, -50.0, 5, 40)],
                         ion_inj=[(3, 1, 2.0, 1), (3, 1, -0.25, 1), (70, 0, 1.0, 0)],
                         lig_inj=[(5, 1, 0.4, 0), (9, 0, 0.3, 1), (5, 14, 0.1, 0), (66, 7, 0.2, 0)])
    ora.upload_stimuli(data)
    gpu.upload_stimuli(data)
    for step in (1, 10, 49):
        ora.run(step, DT)
        gpu.run_ticks(step, DT)
        _compare_all(ora, gpu, 0, "trees with injections +%d" % step)
        _compare_nt(ora, gpu, "trees with injections +%d" % step)
    assert gpu.segment_field("neurotransmitter", 1).astype(np.float64).sum() > 0.3
