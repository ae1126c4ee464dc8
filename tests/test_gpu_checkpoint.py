"""Checkpoints (bnc_save_checkpoint / bnc_load_checkpoint): a run saved half way and
loaded into a fresh backend continues bit for bit as the uninterrupted run.  The
network has transmission delays, readily releasable pools and presynaptic
autoreceptors (BNC_NETGEN_SYNAPSE_EXTRAS), so pending delayed releases and the tick
counter that seeds the release draws must both survive the checkpoint."""
import numpy as np
import pytest

from bioneuroncore_b200 import Backend, Network, NetgenParams, NET_SMALL, BackendError

pytestmark = pytest.mark.gpu

DT = 0.025
SEG_FIELDS = [("V", 0), ("ATP", 0)] + [("ion_in", q) for q in range(7)] + [("ion_out", q) for q in range(7)] + \
             [("neurotransmitter", q) for q in (0, 1)] + [("mod_state", q) for q in (0, 1, 8, 9)]
SYN_FIELDS = ["weight", "bouton_Ca", "spine_Ca", "RRP", "cleft", "refractory", "receptor_state"]


def _state(b):
    out = {"%s[%d]" % f: np.asarray(b.segment_field(*f), np.float32) for f in SEG_FIELDS}
    out.update({f: np.asarray(b.synapse_field(f), np.float32) for f in SYN_FIELDS})
    return out


def _same(x, y):
    for k in x:
        eq = x[k].view(np.uint32) == y[k].view(np.uint32)
        assert eq.all(), "%s: %d values differ" % (k, int((~eq).sum()))


def test_checkpoint_resumes_bit_for_bit(tmp_path):
    p = NetgenParams(family=NET_SMALL, n_neurons=8, seed=7, flags=32)
    whole = Backend()
    whole.load_network(Network(p))
    whole.run_ticks(800, DT)
    half = Backend()
    half.load_network(Network(p))
    half.run_ticks(400, DT)
    path = tmp_path / "run.bion"
    half.save_checkpoint(path)
    assert path.exists() and (tmp_path / "run.bion.state").exists()
    resumed = Backend()
    resumed.load_checkpoint(path)
    resumed.run_ticks(400, DT)
    _same(_state(whole), _state(resumed))
    # the .bion alone restarts the tick counter and drops the pending releases
    plain = Backend()
    plain.load_bion(str(path))
    plain.run_ticks(400, DT)
    a, c = _state(whole), _state(plain)
    assert any((a[k].view(np.uint32) != c[k].view(np.uint32)).any() for k in a)


def test_checkpoint_keeps_ramps_and_pending_injections(tmp_path):
    """A ramp that spans the save point and ion and ligand injections uploaded just
    before the save (applied by the first tick after it) survive the checkpoint: the
    resumed run equals the uninterrupted one bit for bit."""
    from bioneuroncore_b200.abi import stimulus_data
    p = NetgenParams(family=NET_SMALL, n_neurons=8, seed=7, flags=32)
    soma = [32 * k for k in range(8)]   # segment 0 of each 32-segment neuron

    def uploads(sim, net, t):
        cur = [tuple(int(r[f]) if f in ("segment_id", "start_tick") else float(r[f])
                     for f in ("segment_id", "amplitude_pA", "duration_ms", "start_tick")) for r in net.stimuli]
        if t == 100:
            sim.upload_stimuli(stimulus_data(current=cur, ramps=[(soma[1], 0.0, 400.0, 150, 350),
                                                                 (soma[2], 300.0, -100.0, 180, 260)]))
        if t == 200:
            sim.upload_stimuli(stimulus_data(current=cur, ramps=[(soma[1], 0.0, 400.0, 150, 350)],
                                             ion_inj=[(soma[3], 0, 1.5, 0), (soma[4], 1, 0.5, 1)],
                                             lig_inj=[(soma[5], 0, 0.3, 1), (soma[6], 2, 0.1, 0)]))

    net_w = Network(p)
    whole = Backend()
    whole.load_network(net_w)
    for t in range(400):
        uploads(whole, net_w, t)
        whole.run_ticks(1, DT)
    net_h = Network(p)
    half = Backend()
    half.load_network(net_h)
    for t in range(200):
        uploads(half, net_h, t)
        half.run_ticks(1, DT)
    uploads(half, net_h, 200)          # uploaded, not yet applied: pending at the save
    path = tmp_path / "run.bion"
    half.save_checkpoint(path)
    resumed = Backend()
    resumed.load_checkpoint(path)
    resumed.run_ticks(200, DT)
    _same(_state(whole), _state(resumed))


def test_checkpoint_refuses_version_1_state_files(tmp_path):
    import struct
    p = NetgenParams(family=NET_SMALL, n_neurons=4, seed=3)
    b = Backend()
    b.load_network(Network(p))
    b.run_ticks(5, DT)
    path = tmp_path / "run.bion"
    b.save_checkpoint(path)
    raw = bytearray((tmp_path / "run.bion.state").read_bytes())
    struct.pack_into("<I", raw, 8, 1)
    (tmp_path / "run.bion.state").write_bytes(bytes(raw))
    with pytest.raises(BackendError, match="version 1"):
        Backend().load_checkpoint(path)


def test_checkpoint_errors(tmp_path):
    b = Backend()
    with pytest.raises(BackendError):
        b.load_checkpoint(tmp_path / "missing.bion")
    (tmp_path / "bad.bion.state").write_bytes(b"not a state file")
    with pytest.raises(BackendError):
        b.load_checkpoint(tmp_path / "bad.bion")


def test_state_frame_is_the_daemon_layout():
    """bnc_state_frame: tick, counts and the Segment/Synapse records of the current state,
    byte for byte the records of the synced host arrays (the daemon's frame,
    daemon_state.cpp:66-79)."""
    import ctypes as C
    import struct
    from bioneuroncore_b200 import BionData
    p = NetgenParams(family=NET_SMALL, n_neurons=4, seed=3)
    b = Backend()
    b.load_network(Network(p))
    b.run_ticks(37, DT)
    frame = b.state_frame()
    tick, n_seg, n_syn = struct.unpack_from("<QII", frame, 0)
    assert tick == 37
    b.sync_to_host()
    d = C.cast(b.lib.gpu_backend_bion_data(b.h), C.POINTER(BionData)).contents
    seg_bytes = C.string_at(d.segments, n_seg * 3216)
    syn_bytes = C.string_at(d.synapses, n_syn * 1568)
    assert n_seg == d.num_segments and n_syn == d.num_synapses
    assert frame[16:16 + len(seg_bytes)] == seg_bytes
    assert frame[16 + len(seg_bytes):] == syn_bytes
