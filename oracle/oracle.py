"""CPU oracle bindings -- TEST INFRASTRUCTURE ONLY.

`Oracle` drives oracle/liboracle.so, the C restatement of the reference tick with
FP32 state (oracle/bnc_oracle.c).  `Reference` drives oracle/_ref/libbiocore_ref.so,
the reference's own CPU library compiled from its sources by oracle/Makefile, when
that build is present.  Only tests/, the smoke check and bench.py's CPU-baseline
leg use this module; the product path never does.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libbiocore_ref.so")

_ora = None
_ref = None


def oracle_lib():
    global _ora
    if _ora is None:
        if not os.path.exists(ORACLE_LIB):
            from bioneuroncore_b200 import build
            build.build_oracle()   # gcc only; the oracle is plain C
        lib = C.CDLL(ORACLE_LIB)
        vp = C.c_void_p
        lib.bo_create.argtypes = [vp, vp, C.c_uint32, C.c_char_p, C.c_int]
        lib.bo_create.restype = vp
        lib.bo_destroy.argtypes = [vp]
        lib.bo_run.argtypes = [vp, C.c_uint32, C.c_float]
        lib.bo_run_trace.argtypes = [vp, C.c_uint32, C.c_float, vp, C.c_uint32, vp]
        lib.bo_get_seg_field.argtypes = [vp, C.c_int, C.c_int, vp]
        lib.bo_get_syn_field.argtypes = [vp, C.c_int, C.c_int, vp]
        lib.bo_set_syn_scale.argtypes = [vp, vp]
        lib.bo_tick_count.argtypes = [vp]
        lib.bo_tick_count.restype = C.c_uint64
        lib.bo_exp_d.argtypes = [C.c_double]; lib.bo_exp_d.restype = C.c_double
        lib.bo_expf_f.argtypes = [C.c_float]; lib.bo_expf_f.restype = C.c_float
        lib.bo_log_d.argtypes = [C.c_double]; lib.bo_log_d.restype = C.c_double
        lib.bo_pow_d.argtypes = [C.c_double, C.c_double]; lib.bo_pow_d.restype = C.c_double
        lib.bo_xorshift_f.argtypes = [C.c_uint32]; lib.bo_xorshift_f.restype = C.c_float
        lib.bo_seed_bits.argtypes = [C.c_float]; lib.bo_seed_bits.restype = C.c_uint32
        for name in ("bo_ghk_mono_d", "bo_ghk_div_d", "bo_ghk_anion_d"):
            getattr(lib, name).argtypes = [C.c_double] * 3
            getattr(lib, name).restype = C.c_double
        lib.bo_nernst_f.argtypes = [C.c_float] * 3; lib.bo_nernst_f.restype = C.c_float
        lib.bo_const.argtypes = [C.c_int]; lib.bo_const.restype = C.c_double
        lib.bo_register_modifier.argtypes = [C.c_uint8, C.c_void_p]; lib.bo_register_modifier.restype = C.c_int
        _ora = lib
    return _ora


def reference_available():
    return os.path.exists(REF_LIB)


def reference_lib():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_LIB)
        vp = C.c_void_p
        lib.core_run_tick.argtypes = [vp, C.c_uint32, vp, C.c_uint32, vp, C.c_uint32, C.c_uint8,
                                      C.POINTER(C.c_uint64), C.c_float, vp, C.POINTER(C.c_uint32)] + [vp] * 10
        lib.core_run_tick.restype = None
        lib.core_enable_spike_count.argtypes = [vp, C.c_uint32]
        lib.core_disable_spike_tracking.argtypes = []
        _ref = lib
    return _ref


SEG = {"V": 0, "ion_in": 1, "ion_out": 2, "ATP": 3, "temperature": 4, "transcription": 5, "intra_nt": 6,
       "neurotransmitter": 7, "mod_state": 8, "spikes": 9}
SYN = {"bouton_Ca": 0, "spine_Ca": 1, "weight": 2, "refractory": 3, "cleft": 4, "receptor_state": 5,
       "facilitation": 6, "spine_camkii": 7, "spine_calcineurin": 8, "RRP": 9}


class Oracle:
    """FP32-state CPU restatement of the reference tick over a generated Network."""

    def __init__(self, net):
        lib = oracle_lib()
        err = C.create_string_buffer(256)
        self.h = lib.bo_create(C.byref(net.data), net.stim_ptr, net.n_stim, err, 256)
        if err.value:
            lib.bo_destroy(self.h)
            self.h = None
            raise ValueError(err.value.decode())
        self.n_seg = net.data.num_segments
        self.n_syn = net.data.num_synapses

    def run(self, ticks, dt):
        oracle_lib().bo_run(self.h, ticks, C.c_float(dt))

    def trace(self, ticks, dt, rec):
        rec = np.ascontiguousarray(rec, np.uint32)
        out = np.empty((ticks, rec.size), np.float32)
        oracle_lib().bo_run_trace(self.h, ticks, C.c_float(dt), rec.ctypes.data, rec.size, out.ctypes.data)
        return out

    def segment_field(self, field, index=0):
        out = np.empty(self.n_seg, np.float32)
        oracle_lib().bo_get_seg_field(self.h, SEG.get(field, field), index, out.ctypes.data)
        return out

    def synapse_field(self, field, index=0):
        out = np.empty(max(self.n_syn, 1), np.float32)
        oracle_lib().bo_get_syn_field(self.h, SYN.get(field, field), index, out.ctypes.data)
        return out[:self.n_syn]

    def set_synapse_scale(self, scale):
        s = np.ascontiguousarray(scale, np.float32)
        oracle_lib().bo_set_syn_scale(self.h, s.ctypes.data)

    def close(self):
        if self.h:
            oracle_lib().bo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Reference:
    """The reference's own core_run_tick (FP64 state) applied in place to a Network's AoS."""

    def __init__(self, net):
        self.net = net
        self.lib = reference_lib()
        self.tick = C.c_uint64(0)
        self.n_stim = C.c_uint32(net.n_stim)

    def run(self, ticks, dt):
        d = self.net.data
        for _ in range(ticks):
            self.lib.core_run_tick(d.segments, d.num_segments, d.connections, d.num_connections, d.synapses,
                                   d.num_synapses, 0, C.byref(self.tick), C.c_float(dt), self.net.stim_ptr,
                                   C.byref(self.n_stim), *([None] * 10))

    def trace(self, ticks, dt, rec):
        out = np.empty((ticks, len(rec)), np.float64)
        for t in range(ticks):
            self.run(1, dt)
            out[t] = self.net.segments["V_m"][rec]
        return out
