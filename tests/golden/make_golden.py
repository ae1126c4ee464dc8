"""Generates the golden fixtures in this folder from the reference's own CPU tick.

The reference's core_run_tick (src/simulation_host.cpp:660-669) is compiled from
its sources into oracle/_ref/libbiocore_ref.so by oracle/Makefile and run here on
seeded networks from the project's generator; the resulting state is stored as
.npz so that tests can pin the oracle (and the GPU path) to the reference on
machines where the reference sources are absent.

    python tests/golden/make_golden.py [case ...]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

DT = 0.025

# name -> (generator parameters, ticks)
CASES = {
    "small_n8_s7": (dict(family=1, n_neurons=8, seed=7), 200),
    "large_n4_s3": (dict(family=2, n_neurons=4, n_synapses=80, seed=3), 100),
    # RRP, presynaptic autoreceptors and transmission delays (BNC_NETGEN_SYNAPSE_EXTRAS)
    "extras_n8_s7": (dict(family=1, n_neurons=8, seed=7, flags=32), 200),
    # every stimulus kind of gpu_backend_upload_stimuli, two uploads (golden_cases.stimulus_schedule)
    "stimuli_n8_s7": (dict(family=1, n_neurons=8, seed=7), 200),
    # releases: RRP, autoreceptors and delays driven by 3 nA somatic steps (7 releases,
    # an FP32-state path decides them all alike)
    "releases_extras_n8_s6": (dict(family=1, n_neurons=8, seed=6, flags=32, stim_pA=3000), 300),
    # releases on the large set (42 releases); FP32 V_m flips some draws, so this one
    # pins the FP64 restatement only
    "releases_large_n12_s3": (dict(family=2, n_neurons=12, seed=3), 200),
}
# Cases that hold the release decisions and the full FP64 state, and whether an
# FP32-state path is held to the fixture's tolerance.
RELEASES = {"releases_extras_n8_s6": True, "releases_large_n12_s3": False}


def params(spec):
    from bioneuroncore_b200 import NetgenParams
    return NetgenParams(**spec)


def run_reference(spec, ticks, name=""):
    import ctypes as C
    sys.path.insert(0, os.path.dirname(HERE))
    import golden_cases
    from bioneuroncore_b200 import Network
    from oracle.oracle import Reference, reference_lib
    net = Network(params(spec))
    ref = Reference(net)
    lib = reference_lib()
    # core_run_tick keeps its delay buffer in a function-local static that it clears
    # only when the synapse count changes (simulation_host.cpp:322-326): a call with
    # no synapses first, so every case starts with an empty buffer
    zero, tick0 = C.c_uint32(0), C.c_uint64(0)
    lib.core_run_tick(None, 0, None, 0, None, 0, 0, C.byref(tick0), C.c_float(DT), None, C.byref(zero),
                      *([None] * 10))
    spikes = np.zeros(net.data.num_segments, np.uint32)
    lib.core_enable_spike_count(spikes.ctypes.data, net.data.num_segments)
    somata = np.flatnonzero(net.segments["segment_type"] == 1).astype(np.uint32)
    log = None
    if name in RELEASES:
        trace, log = golden_cases.run_scheduled(ref, name, net, ticks, DT, somata, lambda: net.segments["V_m"],
                                                read_refractory=lambda: net.synapses["refractory"])
    else:
        trace = golden_cases.run_scheduled(ref, name, net, ticks, DT, somata, lambda: net.segments["V_m"])
    lib.core_disable_spike_tracking()
    seg = net.segments
    syn = net.synapses
    out = dict(
        ticks=np.int64(ticks), dt=np.float32(DT), somata=somata, soma_trace=trace,
        V=seg["V_m"].copy(), ion_in=seg["intra_ions"][:, :7].copy(), ion_out=seg["extra_ions"][:, :7].copy(),
        ATP=seg["ATP_level"].astype(np.float64), spikes=spikes.copy(),
        syn_weight=syn["weight"].astype(np.float64), syn_spine_Ca=syn["spine_Ca"].astype(np.float64),
        syn_bouton_Ca=syn["bouton_Ca"].astype(np.float64), syn_RRP=syn["RRP"].astype(np.float64),
    )
    if golden_cases.stimulus_schedule(name, net):
        out["intra_nt"] = seg["intra_nt"].astype(np.float64)
    if log is not None:
        out["release_syn"] = np.array([x for x, _ in log], np.int64)
        out["release_tick"] = np.array([t for _, t in log], np.int64)
        out["fp32_tolerance"] = np.int8(RELEASES[name])
        for f, q in golden_cases.SEG_FULL:
            out["full_seg_%s_%d" % (f, q)] = _seg_value(net, f, q)
        for f, q in golden_cases.SYN_FULL:
            out["full_syn_%s_%d" % (f, q)] = _syn_value(net, f, q)
    out.update({"param_" + k: np.int64(v) for k, v in spec.items()})
    return out


def _seg_value(net, f, q):
    seg = net.segments
    col = {"V": "V_m", "ATP": "ATP_level", "temperature": "temperature",
           "transcription": "transcription_signal"}
    if f in col:
        return seg[col[f]].astype(np.float64)
    arr = {"ion_in": "intra_ions", "ion_out": "extra_ions", "intra_nt": "intra_nt",
           "neurotransmitter": "neurotransmitter"}[f]
    return seg[arr][:, q].astype(np.float64)


def _syn_value(net, f, q):
    syn = net.synapses
    if f == "cleft":
        return syn["cleft_neurotransmitter"][:, q].astype(np.float64)
    return syn[f].astype(np.float64)


def main():
    from oracle.oracle import reference_available
    if not reference_available():
        raise SystemExit("oracle/_ref/libbiocore_ref.so is not built (make -C oracle)")
    only = set(sys.argv[1:])   # case names; all cases when none is given
    for name, (spec, ticks) in CASES.items():
        if only and name not in only:
            continue
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **run_reference(spec, ticks, name))
        print("wrote", name)


if __name__ == "__main__":
    main()
