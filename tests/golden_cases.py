"""Shared comparison of a simulator's state with the reference-generated fixtures
in tests/golden/ (made by tests/golden/make_golden.py from the reference's own
CPU tick).  Used by the oracle test (CPU) and the GPU test alike."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REL_TOL = 1e-4   # relative, V_m floored at 1 mV and concentrations at 1e-6 mM


# State words a release fixture holds in full (the reference's FP64 values), by the
# field names of Oracle.segment_field / synapse_field.
SEG_FULL = [("V", 0), ("ATP", 0), ("temperature", 0), ("transcription", 0)] + \
    [("ion_in", q) for q in range(7)] + [("ion_out", q) for q in range(7)] + \
    [("intra_nt", q) for q in range(15)] + [("neurotransmitter", q) for q in range(15)]
SYN_FULL = [(f, 0) for f in ("bouton_Ca", "spine_Ca", "weight", "refractory", "facilitation", "depression",
                             "spine_camkii", "spine_calcineurin", "RRP")] + [("cleft", q) for q in range(15)]


def _all():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def cases():
    """Fixtures an FP32-state path must match within REL_TOL.  A fixture whose release
    draws an FP32 V_m can flip (the seed truncates V_m * 1000 to an integer) is a pin
    for the FP64 restatement only (release_cases), and is left out here."""
    out = []
    for name in _all():
        with np.load(os.path.join(GOLDEN, name + ".npz")) as g:
            if "fp32_tolerance" not in g.files or int(g["fp32_tolerance"]):
                out.append(name)
    return out


def release_cases():
    """Fixtures that hold the reference's release decisions and its full FP64 state."""
    out = []
    for name in _all():
        with np.load(os.path.join(GOLDEN, name + ".npz")) as g:
            if "release_syn" in g.files:
                out.append(name)
    return out


def release_log(g):
    return list(zip((int(x) for x in g["release_syn"]), (int(x) for x in g["release_tick"])))


def decisions(before, after, tick):
    """(synapse, tick) of every release decided in a tick: a synapse releases only while
    its refractory counter is 0 (simulation_host.cpp:458), and a release leaves it
    above 0 (it counts down every tick, :591)."""
    before = np.asarray(before)
    after = np.asarray(after)
    return [(int(i), tick) for i in np.flatnonzero((before == 0) & (after > 0))]


def load(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    spec = {k[len("param_"):]: int(g[k]) for k in g.files if k.startswith("param_")}
    return g, spec


def _rel(a, b, floor):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max()) if b.size else 0.0


def compare(g, trace, seg_field, syn_field, log=None):
    """Returns a dict of max relative errors; raises AssertionError past REL_TOL, on
    any spike-count difference, or (given the run's release decisions `log` and a
    fixture that holds the reference's) on any release decision that differs."""
    if log is not None and "release_syn" in g.files:
        want = release_log(g)
        assert log == want, "release decisions differ from the reference: %d vs %d, first difference %r" % (
            len(log), len(want), next(((a, b) for a, b in zip(log, want) if a != b), None))
    errs = {"soma_trace": _rel(trace, g["soma_trace"], 1.0), "V": _rel(seg_field("V", 0), g["V"], 1.0),
            "ATP": _rel(seg_field("ATP", 0), g["ATP"], 1e-6)}
    for q in range(7):
        errs["ion_in[%d]" % q] = _rel(seg_field("ion_in", q), g["ion_in"][:, q], 1e-6)
        errs["ion_out[%d]" % q] = _rel(seg_field("ion_out", q), g["ion_out"][:, q], 1e-6)
    errs["syn_weight"] = _rel(syn_field("weight"), g["syn_weight"], 1e-9)
    errs["syn_spine_Ca"] = _rel(syn_field("spine_Ca"), g["syn_spine_Ca"], 1e-9)
    errs["syn_bouton_Ca"] = _rel(syn_field("bouton_Ca"), g["syn_bouton_Ca"], 1e-9)
    if "syn_RRP" in g.files:
        errs["syn_RRP"] = _rel(syn_field("RRP"), g["syn_RRP"], 1e-6)
    if "intra_nt" in g.files:
        for q in range(15):
            errs["intra_nt[%d]" % q] = _rel(seg_field("intra_nt", q), g["intra_nt"][:, q], 1e-6)
    bad = {k: v for k, v in errs.items() if not v <= REL_TOL}
    assert not bad, "relative error above %g: %r" % (REL_TOL, bad)
    spikes = np.asarray(seg_field("spikes", 0)).astype(np.int64)
    assert np.array_equal(spikes, g["spikes"].astype(np.int64)), "spike counts differ from the reference"
    return errs


def stimulus_schedule(name, net):
    """The uploads (gpu_backend_upload_stimuli / core_run_tick's stimulus arguments) a
    fixture case makes: a list of (tick, GpuStimulusData), each uploaded before that
    tick runs.  Empty for cases without one.  The "stimuli" case keeps the generator's
    current steps and adds ramps (rising, falling, empty), voltage clamps, ion
    injections (repeated into one ion, extracellular, out-of-range index and segment)
    and ligand injections (intracellular, which then diffuses, and extracellular)."""
    if not name.startswith("stimuli"):
        return []
    from bioneuroncore_b200.abi import stimulus_data
    cur = [tuple(int(r[f]) if f in ("segment_id", "start_tick") else float(r[f])
                 for f in ("segment_id", "amplitude_pA", "duration_ms", "start_tick")) for r in net.stimuli]
    soma = [int(i) for i in np.flatnonzero(net.segments["segment_type"] == 1)]
    n = int(net.data.num_segments)
    first = stimulus_data(
        current=cur,
        ramps=[(soma[0], 0.0, 300.0, 10, 150), (soma[1], 200.0, -100.0, 50, 120), (soma[2], 50.0, 80.0, 30, 30),
               (soma[0], 25.0, 25.0, 100, 180)],
        vclamps=[(soma[3], -30.0, 60, 90), (soma[3] + 1, -80.0, 20, 200), (soma[3], -20.0, 80, 85)],
        ion_inj=[(soma[4], 0, 2.0, 0), (soma[4], 0, 0.5, 0), (soma[5] + 2, 1, 1.5, 1), (soma[5], 9, 1.0, 0),
                 (n + 5, 0, 1.0, 0), (soma[6], 2, 1e-4, 0)],
        lig_inj=[(soma[1] + 3, 0, 0.5, 1), (soma[2], 1, 0.2, 0), (soma[2] + 1, 7, 0.3, 1)])
    second = stimulus_data(
        current=cur,
        ramps=[(soma[1], -50.0, 150.0, 100, 190)],
        ion_inj=[(soma[0], 3, 4.0, 0), (soma[7], 1, -0.5, 1)],
        lig_inj=[(soma[0], 0, 0.25, 1)])
    return [(0, first), (100, second)]


def run_scheduled(sim, name, net, ticks, dt, somata, read_v, read_refractory=None):
    """Runs `ticks` single ticks on `sim` (anything with run(n, dt) or run_ticks(n, dt)
    and upload_stimuli), uploading the case's schedule; returns the soma V_m trace, and
    with read_refractory (the synapses' refractory counters) also the release decisions
    (synapse, tick) in tick order."""
    sched = dict(stimulus_schedule(name, net))
    step = getattr(sim, "run_ticks", None) or sim.run
    trace = np.empty((ticks, len(somata)), np.float64)
    log = []
    for t in range(ticks):
        if t in sched:
            sim.upload_stimuli(sched[t])
        before = np.array(read_refractory(), copy=True) if read_refractory else None
        step(1, dt)
        if read_refractory:
            log += decisions(before, read_refractory(), t)
        trace[t] = read_v()[somata]
    return (trace, log) if read_refractory else trace

