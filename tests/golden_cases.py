"""Shared comparison of a simulator's state with the reference-generated fixtures
in tests/golden/ (made by tests/golden/make_golden.py from the reference's own
CPU tick).  Used by the oracle test (CPU) and the GPU test alike."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REL_TOL = 1e-4   # relative, V_m floored at 1 mV and concentrations at 1e-6 mM


def cases():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    spec = {k[len("param_"):]: int(g[k]) for k in g.files if k.startswith("param_")}
    return g, spec


def _rel(a, b, floor):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float((np.abs(a - b) / np.maximum(np.abs(b), floor)).max()) if b.size else 0.0


def compare(g, trace, seg_field, syn_field):
    """Returns a dict of max relative errors; raises AssertionError past REL_TOL or on
    any spike-count difference."""
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
    bad = {k: v for k, v in errs.items() if not v <= REL_TOL}
    assert not bad, "relative error above %g: %r" % (REL_TOL, bad)
    spikes = np.asarray(seg_field("spikes", 0)).astype(np.int64)
    assert np.array_equal(spikes, g["spikes"].astype(np.int64)), "spike counts differ from the reference"
    return errs
