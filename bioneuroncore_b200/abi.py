"""ctypes / numpy views of the reference data model (include/bnc_abi.h).

The layouts are the reference's `.bion` v14 structs (reference include/types.h:446-603,
include/bion_loader.h:16-28); sizes and offsets are asserted at import.
"""
import ctypes as C

import numpy as np

MOD_DTYPE = np.dtype({
    "names": ["type", "density", "state", "active_vars", "flags"],
    "formats": ["u1", "<f8", ("<f8", 8), "u1", "u1"],
    "offsets": [0, 8, 16, 80, 81],
    "itemsize": 88,
})

SEGMENT_DTYPE = np.dtype({
    "names": ["id", "neuron_id", "position", "direction", "length", "radius", "V_m", "intra_ions",
              "extra_ions", "intra_nt", "neurotransmitter", "modifiers", "modifier_count",
              "segment_type", "ATP_level", "temperature", "I_buffer", "transcription_signal",
              "intra_connection_ids", "intra_connection_count", "ER_Ca2"],
    "formats": ["<u4", "<u4", ("<f4", 3), ("<f4", 3), "<f4", "<f4", "<f8", ("<f8", 8), ("<f8", 8),
                ("<f4", 15), ("<f4", 15), (MOD_DTYPE, 32), "u1", "u1", "<f4", "<f4", "<f8", "<f4",
                ("<u4", 16), "u1", "<f4"],
    "offsets": [0, 4, 8, 20, 32, 36, 40, 48, 112, 176, 236, 296, 3112, 3113, 3120, 3124, 3128, 3136,
                3140, 3204, 3212],
    "itemsize": 3216,
})

SYNAPSE_DTYPE = np.dtype({
    "names": ["id", "pre_segment", "post_segment", "type", "weight", "delay", "pre_area", "post_area",
              "pre_autoreceptors", "pre_autoreceptor_count", "post_receptors", "post_receptor_count",
              "release_probability", "release_amount", "cleft_neurotransmitter", "facilitation",
              "depression", "tau_clearance", "refractory", "RRP", "RRP_max", "RRP_recovery",
              "bouton_Ca", "spine_Ca", "spine_camkii", "spine_calcineurin"],
    "formats": ["<u4", "<u4", "<u4", "u1", "<f4", "<f4", "<f4", "<f4", (MOD_DTYPE, 8), "u1",
                (MOD_DTYPE, 8), "u1", "<f4", "<f4", ("<f4", 15), "<f4", "<f4", "<f4", "u1", "<f4",
                "<f4", "<f4", "<f4", "<f4", "<f4", "<f4"],
    "offsets": [0, 4, 8, 12, 16, 20, 24, 28, 32, 736, 744, 1448, 1452, 1456, 1460, 1520, 1524, 1528,
                1532, 1540, 1544, 1548, 1552, 1556, 1560, 1564],
    "itemsize": 1568,
})

CONN_DTYPE = np.dtype({
    "names": ["segment_a", "segment_b", "is_intracellular"],
    "formats": ["<u4", "<u4", "u1"],
    "offsets": [0, 4, 8],
    "itemsize": 16,
})

STIM_DTYPE = np.dtype({
    "names": ["segment_id", "amplitude_pA", "duration_ms", "start_tick"],
    "formats": ["<u4", "<f4", "<f4", "<u8"],
    "offsets": [0, 4, 8, 12],
    "itemsize": 20,
})


MAX_STIMULI = 256   # BNC_GPU_MAX_STIMULI


class CurrentStimulus(C.Structure):
    _pack_ = 1
    _fields_ = [("segment_id", C.c_uint32), ("amplitude_pA", C.c_float), ("duration_ms", C.c_float),
                ("start_tick", C.c_uint64)]


class VoltageClamp(C.Structure):
    _pack_ = 1
    _fields_ = [("segment_id", C.c_uint32), ("target_mV", C.c_float), ("start_tick", C.c_uint64),
                ("end_tick", C.c_uint64)]


class RampStimulus(C.Structure):
    _pack_ = 1
    _fields_ = [("segment_id", C.c_uint32), ("start_pA", C.c_float), ("end_pA", C.c_float),
                ("start_tick", C.c_uint64), ("end_tick", C.c_uint64)]


class IonInjection(C.Structure):
    _pack_ = 1
    _fields_ = [("segment_id", C.c_uint32), ("ion_idx", C.c_int32), ("amount_mM", C.c_float),
                ("extracellular", C.c_uint8), ("_pad", C.c_uint8 * 3)]


class LigandInjection(C.Structure):
    _pack_ = 1
    _fields_ = [("segment_id", C.c_uint32), ("nt_idx", C.c_int32), ("amount", C.c_float),
                ("intracellular", C.c_uint8), ("_pad2", C.c_uint8 * 3)]


class MechanoStimulus(C.Structure):
    """types.h:645-655 (packed, 13 bytes)."""
    _pack_ = 1
    _fields_ = [("segment_id", C.c_uint32), ("mod_type", C.c_uint8), ("state_idx", C.c_int32), ("value", C.c_float)]


def mechano_data(items):
    """A ctypes array of MechanoStimulus from (segment_id, mod_type, state_idx, value)."""
    arr = (MechanoStimulus * max(len(items), 1))()
    for i, (sid, t, idx, v) in enumerate(items):
        arr[i].segment_id, arr[i].mod_type, arr[i].state_idx, arr[i].value = sid, t, idx, v
    return arr, len(items)


class GpuStimulusData(C.Structure):
    """BncGpuStimulusData, the argument of gpu_backend_upload_stimuli (reference
    include/types.h:662-674): up to 256 entries of each stimulus kind."""
    _pack_ = 1
    _fields_ = [("current_stim_count", C.c_uint32), ("vclamp_count", C.c_uint32), ("ramp_count", C.c_uint32),
                ("ion_inj_count", C.c_uint32), ("lig_inj_count", C.c_uint32), ("current_tick", C.c_uint64),
                ("current_stim", CurrentStimulus * MAX_STIMULI), ("vclamps", VoltageClamp * MAX_STIMULI),
                ("ramps", RampStimulus * MAX_STIMULI), ("ion_inj", IonInjection * MAX_STIMULI),
                ("lig_inj", LigandInjection * MAX_STIMULI)]


def stimulus_data(current=(), vclamps=(), ramps=(), ion_inj=(), lig_inj=()):
    """A GpuStimulusData from tuples in field order: current (segment_id, amplitude_pA,
    duration_ms, start_tick), vclamps (segment_id, target_mV, start_tick, end_tick), ramps
    (segment_id, start_pA, end_pA, start_tick, end_tick), ion_inj (segment_id, ion_idx,
    amount_mM, extracellular), lig_inj (segment_id, nt_idx, amount, intracellular)."""
    d = GpuStimulusData()
    for name, cnt, rows, cls in (("current_stim", "current_stim_count", current, CurrentStimulus),
                                 ("vclamps", "vclamp_count", vclamps, VoltageClamp),
                                 ("ramps", "ramp_count", ramps, RampStimulus),
                                 ("ion_inj", "ion_inj_count", ion_inj, IonInjection),
                                 ("lig_inj", "lig_inj_count", lig_inj, LigandInjection)):
        rows = list(rows)
        if len(rows) > MAX_STIMULI:
            raise ValueError("at most %d entries of each stimulus kind" % MAX_STIMULI)
        arr = getattr(d, name)
        for k, r in enumerate(rows):
            arr[k] = cls(*r)
        setattr(d, cnt, len(rows))
    return d


assert C.sizeof(CurrentStimulus) == 20 and C.sizeof(VoltageClamp) == 24 and C.sizeof(RampStimulus) == 28
assert C.sizeof(IonInjection) == 16 and C.sizeof(LigandInjection) == 16
assert C.sizeof(GpuStimulusData) == 28 + MAX_STIMULI * (20 + 24 + 28 + 16 + 16)


class BionData(C.Structure):
    """Reference BionData (include/bion_loader.h:16-28); not packed."""
    _fields_ = [
        ("header", C.c_uint8 * 100),
        ("neurons", C.c_void_p),
        ("segments", C.c_void_p),
        ("connections", C.c_void_p),
        ("synapses", C.c_void_p),
        ("nuclei", C.c_void_p),
        ("num_neurons", C.c_uint32),
        ("num_segments", C.c_uint32),
        ("num_connections", C.c_uint32),
        ("num_synapses", C.c_uint32),
        ("num_nuclei", C.c_uint32),
    ]


class NetgenParams(C.Structure):
    """BncNetgenParams (include/bnc_b200.h)."""
    _fields_ = [
        ("family", C.c_uint32),
        ("n_neurons", C.c_uint32),
        ("n_synapses", C.c_uint64),
        ("seed", C.c_uint64),
        ("segs_per_neuron", C.c_uint32),
        ("tree_depth", C.c_uint32),
        ("conductance_scale", C.c_float * 4),
        ("flags", C.c_uint32),
        ("stim_pA", C.c_float),
        ("stim_duration_ms", C.c_float),
    ]


NET_SMALL, NET_LARGE, NET_TREES, NET_ENSEMBLE_MEMBER, NET_ADJOINT = 1, 2, 3, 4, 5
NETGEN_NO_SYNAPSES, NETGEN_NO_CONNECTIONS, NETGEN_NO_STIMULI, NETGEN_PERTURB_IONS = 1, 2, 4, 8
NETGEN_DRAW_ORDER = 16
NETGEN_SYNAPSE_EXTRAS = 32
NETGEN_FULL_SMALL_SET = 64
NETGEN_GLYCINE = 128
NETGEN_RELEASE_MODULATORS = 256
NETGEN_ECB = 512
NETGEN_GLIA = 1024
NETGEN_GAP_JUNCTIONS = 2048
NETGEN_NMDA = 4096

assert SEGMENT_DTYPE.itemsize == 3216 and SYNAPSE_DTYPE.itemsize == 1568 and MOD_DTYPE.itemsize == 88
assert BionData.segments.offset == 112 and BionData.num_segments.offset == 148


def view(ptr, dtype, count):
    """numpy view (no copy) of `count` records of `dtype` at address `ptr`."""
    if count == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    buf = (C.c_uint8 * (dtype.itemsize * count)).from_address(ptr)
    return np.frombuffer(buf, dtype=dtype, count=count)
