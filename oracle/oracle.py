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
        lib.bo_upload_stimuli.argtypes = [vp, vp]
        lib.bo_upload_mechano.argtypes = [vp, vp, C.c_uint32]
        lib.bo_run.argtypes = [vp, C.c_uint32, C.c_float]
        lib.bo_set_diffusion_mode.argtypes = [vp, C.c_uint32, C.c_double, C.c_uint32]
        lib.bo_diffusion_stats.argtypes = [vp, vp, vp, C.c_int]
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
        lib.bo_seed_bits.argtypes = [C.c_double]; lib.bo_seed_bits.restype = C.c_uint32
        for name in ("bo_ghk_mono_d", "bo_ghk_div_d", "bo_ghk_anion_d"):
            getattr(lib, name).argtypes = [C.c_double] * 3
            getattr(lib, name).restype = C.c_double
        lib.bo_nernst_f.argtypes = [C.c_float] * 3; lib.bo_nernst_f.restype = C.c_float
        lib.bo_const.argtypes = [C.c_int]; lib.bo_const.restype = C.c_double
        lib.bo_register_modifier.argtypes = [C.c_uint8, C.c_void_p]; lib.bo_register_modifier.restype = C.c_int
        lib.bo_set_release_log.argtypes = [vp, vp, vp, vp, vp, C.c_uint32]
        lib.bo_run_stride.argtypes = [vp, C.c_uint32, C.c_float, C.c_uint32]
        lib.bo_release_log_count.argtypes = [vp]; lib.bo_release_log_count.restype = C.c_uint32
        _ora = lib
    return _ora


_ora64 = None


def oracle64_lib():
    """oracle/liboracle64.so: the same restatement built with FP64 state and the C
    library's elementary functions (-DBO_FP64 -DBO_LIBM), the build that is compared
    with the reference's own tick."""
    global _ora64
    if _ora64 is None:
        from bioneuroncore_b200 import build
        if not os.path.exists(build.ORACLE64_LIB):
            build.build_oracle()
        lib = C.CDLL(build.ORACLE64_LIB)
        vp = C.c_void_p
        lib.bo_create.argtypes = [vp, vp, C.c_uint32, C.c_char_p, C.c_int]
        lib.bo_create.restype = vp
        lib.bo_destroy.argtypes = [vp]
        lib.bo_upload_stimuli.argtypes = [vp, vp]
        lib.bo_upload_mechano.argtypes = [vp, vp, C.c_uint32]
        lib.bo_run.argtypes = [vp, C.c_uint32, C.c_float]
        lib.bo_run_stride.argtypes = [vp, C.c_uint32, C.c_float, C.c_uint32]
        lib.bo_get_seg_field64.argtypes = [vp, C.c_int, C.c_int, vp]
        lib.bo_get_syn_field64.argtypes = [vp, C.c_int, C.c_int, vp]
        lib.bo_set_release_log.argtypes = [vp, vp, vp, vp, vp, C.c_uint32]
        lib.bo_release_log_count.argtypes = [vp]; lib.bo_release_log_count.restype = C.c_uint32
        lib.bo_tick_count.argtypes = [vp]
        lib.bo_tick_count.restype = C.c_uint64
        lib.bo_seed_bits.argtypes = [C.c_double]; lib.bo_seed_bits.restype = C.c_uint32
        lib.bo_xorshift_f.argtypes = [C.c_uint32]; lib.bo_xorshift_f.restype = C.c_float
        _ora64 = lib
    return _ora64


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
       "facilitation": 6, "spine_camkii": 7, "spine_calcineurin": 8, "RRP": 9, "depression": 10,
       "autoreceptor_state": 11}


class Oracle:
    """FP32-state CPU restatement of the reference tick over a generated Network.
    With fp64=True, the same restatement with FP64 state and the C library's
    elementary functions (oracle64_lib); its fields then come back as float64."""

    def __init__(self, net, fp64=False):
        self.fp64 = fp64
        lib = self._lib()
        err = C.create_string_buffer(256)
        self.h = lib.bo_create(C.byref(net.data), net.stim_ptr, net.n_stim, err, 256)
        if err.value:
            lib.bo_destroy(self.h)
            self.h = None
            raise ValueError(err.value.decode())
        self.n_seg = net.data.num_segments
        self.n_syn = net.data.num_synapses

    def _lib(self):
        return oracle64_lib() if self.fp64 else oracle_lib()

    def set_diffusion_mode(self, flags, tol=1e-6, max_sweeps=100000):
        """bo_set_diffusion_mode: residual-controlled FP64 Jacobi solves (flag 1) and
        the per-ion ledger (flag 2), as the backend's bnc_set_diffusion_mode."""
        self._lib().bo_set_diffusion_mode(self.h, flags, C.c_double(tol), max_sweeps)

    def diffusion_stats(self, reset=False):
        """(stats[4], ledger[14]): max V and phi sweeps, capped V and phi group solves;
        per ion the FP32 rounding of the Nernst-Planck updates, then the bath exchange."""
        st = np.zeros(4, np.uint32)
        led = np.zeros(14, np.float64)
        self._lib().bo_diffusion_stats(self.h, st.ctypes.data, led.ctypes.data, 1 if reset else 0)
        return st, led

    def upload_stimuli(self, data):
        """bo_upload_stimuli with a GpuStimulusData: every list replaced, injections once."""
        self._lib().bo_upload_stimuli(self.h, C.byref(data))

    def upload_mechano(self, items):
        """bo_upload_mechano: (segment_id, mod_type, state_idx, value) for the next tick."""
        from bioneuroncore_b200.abi import mechano_data
        arr, n = mechano_data(items)
        self._lib().bo_upload_mechano(self.h, arr, C.c_uint32(n))

    def run(self, ticks, dt, tick_stride=1):
        if tick_stride == 1:
            self._lib().bo_run(self.h, ticks, C.c_float(dt))
        else:
            self._lib().bo_run_stride(self.h, ticks, C.c_float(dt), tick_stride)

    def trace(self, ticks, dt, rec):
        rec = np.ascontiguousarray(rec, np.uint32)
        out = np.empty((ticks, rec.size), np.float32)
        self._lib().bo_run_trace(self.h, ticks, C.c_float(dt), rec.ctypes.data, rec.size, out.ctypes.data)
        return out

    def segment_field(self, field, index=0):
        if self.fp64:
            out = np.empty(self.n_seg, np.float64)
            self._lib().bo_get_seg_field64(self.h, SEG.get(field, field), index, out.ctypes.data)
            return out
        out = np.empty(self.n_seg, np.float32)
        self._lib().bo_get_seg_field(self.h, SEG.get(field, field), index, out.ctypes.data)
        return out

    def synapse_field(self, field, index=0):
        if self.fp64:
            out = np.empty(max(self.n_syn, 1), np.float64)
            self._lib().bo_get_syn_field64(self.h, SYN.get(field, field), index, out.ctypes.data)
            return out[:self.n_syn]
        out = np.empty(max(self.n_syn, 1), np.float32)
        self._lib().bo_get_syn_field(self.h, SYN.get(field, field), index, out.ctypes.data)
        return out[:self.n_syn]

    def set_synapse_scale(self, scale):
        s = np.ascontiguousarray(scale, np.float32)
        self._lib().bo_set_syn_scale(self.h, s.ctypes.data)

    def run_logged(self, ticks, dt, cap=None):
        """Runs `ticks` ticks and returns the release log they produce, sorted by
        (synapse, tick, slot): every transmitter amount that entered a cleft."""
        cap = cap or max(64, self.n_syn * (ticks // 16 + 4))
        syn = np.zeros(cap, np.uint32)
        tick = np.zeros(cap, np.uint64)
        amt = np.zeros(cap, np.float32)
        slot = np.zeros(cap, np.uint8)
        lib = self._lib()
        lib.bo_set_release_log(self.h, syn.ctypes.data, tick.ctypes.data, amt.ctypes.data, slot.ctypes.data, cap)
        lib.bo_run(self.h, ticks, C.c_float(dt))
        n = lib.bo_release_log_count(self.h)
        lib.bo_set_release_log(self.h, None, None, None, None, 0)
        if n > cap:
            raise RuntimeError("release log overflow")
        order = np.lexsort((slot[:n], tick[:n], syn[:n]))
        return syn[:n][order], tick[:n][order], amt[:n][order]

    def close(self):
        if self.h:
            self._lib().bo_destroy(self.h)
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
        self.stim_ptr = net.stim_ptr
        self.rest = [None] * 10   # vclamps, ramps, ion and ligand injections, mechano: array, count

    def upload_stimuli(self, data):
        """Hands the lists of a GpuStimulusData to core_run_tick's own stimulus arguments
        (simulation_host.cpp:660-669), which it expires and clears in place."""
        self._data = data
        self.stim_ptr = C.addressof(data.current_stim)
        self.n_stim = C.c_uint32(data.current_stim_count)
        self._counts = [C.c_uint32(data.vclamp_count), C.c_uint32(data.ramp_count),
                        C.c_uint32(data.ion_inj_count), C.c_uint32(data.lig_inj_count)]
        arrs = [data.vclamps, data.ramps, data.ion_inj, data.lig_inj]
        self.rest = []
        for a, c in zip(arrs, self._counts):
            self.rest += [C.addressof(a), C.cast(C.pointer(c), C.c_void_p)]
        self.rest += [None, None]

    def upload_mechano(self, items):
        """The mechano argument of the next core_run_tick call (simulation_host.cpp:211-230),
        which applies the stimuli and sets the count to 0."""
        from bioneuroncore_b200.abi import mechano_data
        self._mech, n = mechano_data(items)
        self._mech_n = C.c_uint32(n)
        self.rest = list(self.rest[:8]) + [C.addressof(self._mech), C.cast(C.pointer(self._mech_n), C.c_void_p)]

    def run(self, ticks, dt, tick_stride=1):
        d = self.net.data
        for _ in range(ticks):
            self.lib.core_run_tick(d.segments, d.num_segments, d.connections, d.num_connections, d.synapses,
                                   d.num_synapses, 0, C.byref(self.tick), C.c_float(dt), self.stim_ptr,
                                   C.byref(self.n_stim), *self.rest)
            self.tick.value += tick_stride - 1   # the batch mode's second increment

    def trace(self, ticks, dt, rec):
        out = np.empty((ticks, len(rec)), np.float64)
        for t in range(ticks):
            self.run(1, dt)
            out[t] = self.net.segments["V_m"][rec]
        return out


_tan = None


def tangent_lib():
    """oracle/libbo_tangent.so: the FP64 forward-mode replay (bo_tangent.cpp)."""
    global _tan
    if _tan is None:
        from bioneuroncore_b200 import build
        path = build.TANGENT_LIB
        if not os.path.exists(path):
            build.build_oracle()
        lib = C.CDLL(path)
        vp = C.c_void_p
        lib.bo_tangent_run.argtypes = [vp, vp, C.c_uint32, vp, vp, vp, C.c_uint32, C.c_uint64, C.c_uint32, C.c_float,
                                       C.c_uint32] + [vp] * 8 + [vp, C.c_uint32, vp, vp, vp]
        lib.bo_tangent_run.restype = C.c_int
        _tan = lib
    return _tan


def tangent_loss(net, log, ticks, dt, params, direction, soma, target, stride=1):
    """Loss and its derivative along `direction` (FP64 forward mode) for the replayed
    tick.  params / direction: (gNa, gK, gleak per segment, w per synapse)."""
    syn, tick, amt = [np.ascontiguousarray(a) for a in log]
    syn = syn.astype(np.uint32); tick = tick.astype(np.uint64); amt = amt.astype(np.float32)
    p = [np.ascontiguousarray(a, np.float64) for a in params]
    d = [np.ascontiguousarray(a, np.float64) for a in direction]
    soma = np.ascontiguousarray(soma, np.uint32)
    target = np.ascontiguousarray(target, np.float32)
    loss, dloss = C.c_double(), C.c_double()
    rc = tangent_lib().bo_tangent_run(C.byref(net.data), net.stim_ptr, net.n_stim, syn.ctypes.data, tick.ctypes.data,
                                      amt.ctypes.data, syn.size, 0, ticks, C.c_float(dt), stride,
                                      *[a.ctypes.data for a in p], *[a.ctypes.data for a in d],
                                      soma.ctypes.data, soma.size, target.ctypes.data, C.byref(loss), C.byref(dloss))
    if rc != 0:
        raise ValueError("network not modelled by the tangent replay")
    return loss.value, dloss.value
