"""bioneuroncore_b200 -- B200 backend for BioNeuronCore's per-tick simulation loop.

Python view of the C ABI in include/bnc_b200.h.  The compute path is the CUDA
library libbnc_b200.so built in-tree (``python -m bioneuroncore_b200.build``);
there is no CPU fallback: `Backend` raises when the library or a device is missing.

    from bioneuroncore_b200 import Backend, NetgenParams
    b = Backend()                                  # gpu_backend_create
    b.load_generated(NetgenParams(family=2))       # 6.4M-segment network on device
    b.run_ticks(100, 0.025)
    v = b.segment_field("V")                       # V_m in original segment order
"""
import ctypes as C
import os

import numpy as np

from .abi import (BionData, NetgenParams, SEGMENT_DTYPE, SYNAPSE_DTYPE, CONN_DTYPE, STIM_DTYPE, view,
                  NET_SMALL, NET_LARGE, NET_TREES, NET_ENSEMBLE_MEMBER, NET_ADJOINT, NETGEN_NO_SYNAPSES,
                  NETGEN_NO_CONNECTIONS, NETGEN_NO_STIMULI, NETGEN_PERTURB_IONS, NETGEN_SYNAPSE_EXTRAS,
                  NETGEN_FULL_SMALL_SET, NETGEN_GLYCINE, NETGEN_DRAW_ORDER, NETGEN_RELEASE_MODULATORS, NETGEN_ECB, NETGEN_GLIA, NETGEN_GAP_JUNCTIONS,
                  NETGEN_NMDA)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbnc_b200.so")

SEG_FIELDS = {"V": 0, "ion_in": 1, "ion_out": 2, "ATP": 3, "temperature": 4, "transcription": 5,
              "intra_nt": 6, "neurotransmitter": 7, "mod_state": 8, "spikes": 9}
SYN_FIELDS = {"bouton_Ca": 0, "spine_Ca": 1, "weight": 2, "refractory": 3, "cleft": 4, "receptor_state": 5,
              "facilitation": 6, "spine_camkii": 7, "spine_calcineurin": 8, "RRP": 9, "depression": 10,
              "autoreceptor_state": 11}

# Symbols the reference's loader requires (reference tests/smoke_cuda.sh:24-29) plus the
# ABI probes and this backend's own entry points; include/*.h declares every one.
DROPIN_SYMBOLS = ["gpu_backend_create", "gpu_backend_create_on_device", "gpu_backend_destroy",
                  "gpu_backend_load_bion", "gpu_backend_run_tick", "gpu_backend_bion_data",
                  "gpu_backend_upload_stimuli", "gpu_backend_device_count", "gpu_backend_get_device_info",
                  "gpu_backend_ibuf_offset", "gpu_backend_vm_offset", "gpu_backend_seg_size"]
NEW_SYMBOLS = ["bnc_netgen_aos", "bnc_netgen_free", "bnc_last_error", "bnc_load_aos", "bnc_load_generated",
               "bnc_run_ticks", "bnc_time_ticks", "bnc_sync_to_host", "bnc_records_managed", "bnc_set_records_residency",
               "bnc_upload_mechano",
               "register_modifier_current", "register_modulator_release", "bnc_plugin_load",
               "bnc_plugin_load_directory", "bnc_plugin_registered", "bnc_plugin_count", "bnc_plugin_unregister_all",
               "bnc_read_segment_field",
               "bnc_read_synapse_field", "bnc_set_synapse_scale", "bnc_network_info", "bnc_save_bion",
               "bnc_plan_generated", "bnc_step_io", "bnc_profile_ticks", "bnc_run_ticks_static_scratch",
               "bnc_plan_aos", "bnc_bion_load", "bnc_bion_unload", "bnc_bion_save", "bnc_load_ensemble_generated",
               "bnc_load_ensemble_aos", "bnc_ensemble_member", "bnc_plan_ensemble_generated", "bnc_ensemble_params",
               "bnc_run_ticks_graph", "bnc_load_ensemble_tuned", "bnc_time_ticks_graph", "bnc_load_generated_opts",
               "bnc_plan_generated_opts", "biocore_gpu_register_device_modifier", "bnc_register_device_modifier",
               "bnc_device_modifier_registered", "bnc_adjoint_create", "bnc_adjoint_destroy", "bnc_adjoint_info",
               "bnc_adjoint_soma", "bnc_adjoint_record", "bnc_adjoint_release_count", "bnc_adjoint_set_params",
               "bnc_adjoint_get_params", "bnc_adjoint_set_target", "bnc_adjoint_forward", "bnc_adjoint_backward",
               "bnc_adjoint_timings", "bnc_sweep_parse_params", "bnc_sweep_apply", "bnc_sweep_run",
               "bnc_save_checkpoint", "bnc_load_checkpoint", "bnc_state_frame", "bnc_set_diffusion_mode",
               "bnc_diffusion_stats"]

DIFFUSION_RESIDUAL = 1
DIFFUSION_LEDGER = 2


class DiffusionStats(C.Structure):
    """bnc_diffusion_stats: sweep counts of the residual-controlled solves and the
    per-ion FP64 ledger of step 2.5 (rounding of the FP32 updates, bath exchange)."""
    _fields_ = [("max_sweeps_v", C.c_uint32), ("max_sweeps_phi", C.c_uint32), ("capped_v", C.c_uint32),
                ("capped_phi", C.c_uint32), ("rounding", C.c_double * 7), ("bath", C.c_double * 7)]


class NetInfo(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("n_segments", "n_connections", "n_synapses", "n_tiles", "n_items",
                                          "n_phases", "n_receptors", "max_tile_segs", "max_tile_edges",
                                          "smem_bytes", "flags")] + [
        ("ticks", C.c_uint64), ("algo_bytes_per_tick", C.c_double), ("seg_bytes_per_tick", C.c_double),
        ("syn_bytes_per_tick", C.c_double), ("tile_bytes_per_tick", C.c_double),
        ("synapse_kernel_bytes_per_tick", C.c_double), ("warp_cap", C.c_uint32), ("tile_segs", C.c_uint32),
        ("modifier_kernel_bytes", C.c_double), ("diffusion_kernel_bytes", C.c_double),
        ("modifier_launches", C.c_uint32), ("fuse_phases", C.c_uint32), ("group_tiles_32", C.c_uint32),
        ("group_tiles_64", C.c_uint32), ("diffusion_threads", C.c_uint32), ("synapse_launches", C.c_uint32)]


class BuildOptions(C.Structure):
    """Device-layout options (include/bnc_b200.h BncBuildOptions); 0 = default."""
    _fields_ = [("warp_cap", C.c_uint32), ("tile_segs", C.c_uint32), ("phase_cap", C.c_uint32),
                ("chunk_segs", C.c_uint32), ("fuse_phases", C.c_uint32), ("cta_barriers", C.c_uint32)]


class Tuning(C.Structure):
    _fields_ = [("warp_cap", C.c_uint32), ("tile_segs", C.c_uint32), ("ms_per_tick", C.c_float),
                ("candidates_tried", C.c_uint32), ("sample_members", C.c_uint32)]


def plan_generated(params, options=None):
    """Host-only planning of a generated network (no device needed); returns NetInfo."""
    inf = NetInfo()
    if options is None:
        _check(load_library().bnc_plan_generated(C.byref(params), C.byref(inf)), "bnc_plan_generated")
    else:
        _check(load_library().bnc_plan_generated_opts(C.byref(params), C.byref(options), C.byref(inf)),
               "bnc_plan_generated_opts")
    return inf


class EnsembleMember(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("seg_begin", "n_segments", "syn_begin", "n_synapses", "stim_begin",
                                          "n_stimuli")]


def ensemble_params(seed, n_members, min_segments=200, max_segments=20000):
    """Seeded uneven ensemble (sizes log-uniform, gNa/gK/gleak/gCa x U[0.5, 2]); returns a
    ctypes array of NetgenParams."""
    arr = (NetgenParams * n_members)()
    _check(load_library().bnc_ensemble_params(seed, n_members, min_segments, max_segments, arr),
           "bnc_ensemble_params")
    return arr


def plan_ensemble(params):
    """Host-only planning of a generated ensemble; returns NetInfo."""
    arr = params if isinstance(params, C.Array) else (NetgenParams * len(params))(*params)
    inf = NetInfo()
    _check(load_library().bnc_plan_ensemble_generated(arr, len(arr), C.byref(inf)), "bnc_plan_ensemble_generated")
    return inf


def register_device_modifier(type_id, source, entry):
    """Compiles CUDA C++ `source` (see include/bnc_device_modifier.h) with NVRTC and
    registers its extern "C" kernel `entry` for modifier type `type_id` (0-127)."""
    _check(load_library().bnc_register_device_modifier(type_id, source.encode(), entry.encode()),
           "bnc_register_device_modifier")


class BackendError(RuntimeError):
    pass


_lib = None


def load_library(path=LIB_PATH):
    """Loads libbnc_b200.so; raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise BackendError("libbnc_b200.so is not built; run `python -m bioneuroncore_b200.build`")
    lib = C.CDLL(path)
    vp, i32, u32, f32 = C.c_void_p, C.c_int, C.c_uint32, C.c_float
    sig = {
        "gpu_backend_create": ([], vp), "gpu_backend_create_on_device": ([i32], vp),
        "gpu_backend_destroy": ([vp], None), "gpu_backend_load_bion": ([vp, C.c_char_p], i32),
        "gpu_backend_run_tick": ([vp, f32], None), "gpu_backend_bion_data": ([vp], vp),
        "gpu_backend_upload_stimuli": ([vp, vp], None), "gpu_backend_device_count": ([], i32),
        "gpu_backend_get_device_info": ([i32, vp], i32), "gpu_backend_ibuf_offset": ([], i32),
        "gpu_backend_vm_offset": ([], i32), "gpu_backend_seg_size": ([], i32),
        "bnc_netgen_aos": ([vp, vp, vp, vp], i32), "bnc_netgen_free": ([vp, vp], None),
        "bnc_last_error": ([], C.c_char_p), "bnc_load_aos": ([vp, vp, vp, u32], i32),
        "bnc_load_generated": ([vp, vp], i32), "bnc_run_ticks": ([vp, u32, f32], i32),
        "bnc_time_ticks": ([vp, u32, f32, vp], i32), "bnc_sync_to_host": ([vp], i32), "bnc_records_managed": ([vp], i32),
        "bnc_set_records_residency": ([vp, i32], i32), "bnc_upload_mechano": ([vp, vp, u32], i32),
        "bnc_read_segment_field": ([vp, i32, i32, vp, u32], i32),
        "bnc_read_synapse_field": ([vp, i32, i32, vp, u32], i32),
        "bnc_set_synapse_scale": ([vp, vp, u32], i32), "bnc_network_info": ([vp, vp], i32),
        "bnc_save_bion": ([vp, C.c_char_p], i32), "bnc_plan_generated": ([vp, vp], i32),
        "bnc_step_io": ([vp, f32, vp, u32, vp, u32], i32), "bnc_profile_ticks": ([vp, u32, f32, vp, vp, vp], i32),
        "bnc_run_ticks_static_scratch": ([vp, u32, f32], i32),
        "bnc_plan_aos": ([vp, vp, u32, vp], i32), "bnc_bion_load": ([C.c_char_p, vp], i32),
        "bnc_bion_unload": ([vp], None), "bnc_bion_save": ([C.c_char_p, vp], i32),
        "bnc_load_ensemble_generated": ([vp, vp, u32], i32), "bnc_load_ensemble_aos": ([vp, vp, vp, vp, u32], i32),
        "bnc_ensemble_member": ([vp, u32, vp], i32), "bnc_plan_ensemble_generated": ([vp, u32, vp], i32),
        "bnc_ensemble_params": ([C.c_uint64, u32, u32, u32, vp], i32), "bnc_run_ticks_graph": ([vp, u32, f32], i32),
        "bnc_load_ensemble_tuned": ([vp, vp, u32, u32, f32, vp], i32), "bnc_time_ticks_graph": ([vp, u32, f32, vp], i32),
        "bnc_load_generated_opts": ([vp, vp, vp], i32), "bnc_plan_generated_opts": ([vp, vp, vp], i32),
        "biocore_gpu_register_device_modifier": ([C.c_uint8, C.c_char_p, C.c_char_p], i32),
        "bnc_register_device_modifier": ([C.c_uint8, C.c_char_p, C.c_char_p], i32),
        "bnc_device_modifier_registered": ([C.c_uint8], i32),
        "bnc_adjoint_create": ([vp, vp], vp), "bnc_adjoint_destroy": ([vp], None),
        "bnc_adjoint_info": ([vp, vp], i32), "bnc_adjoint_soma": ([vp, vp, u32], i32),
        "bnc_adjoint_record": ([vp, vp], i32), "bnc_adjoint_release_count": ([vp, vp], i32),
        "bnc_adjoint_set_params": ([vp, u32, vp, vp, vp, vp], i32),
        "bnc_adjoint_get_params": ([vp, u32, vp, vp, vp, vp], i32),
        "bnc_adjoint_set_target": ([vp, vp], i32), "bnc_adjoint_forward": ([vp, vp, vp], i32),
        "bnc_adjoint_backward": ([vp, vp, vp, vp, vp], i32), "bnc_adjoint_timings": ([vp, vp, vp], i32),
        "bnc_sweep_parse_params": ([C.c_char_p, vp, vp, u32, vp, vp, u32, vp], i32),
        "bnc_sweep_apply": ([vp, vp], i32),
        "bnc_sweep_run": ([vp, vp, vp, u32, vp, u32, u32, f32, u32, vp], i32),
        "bnc_save_checkpoint": ([vp, C.c_char_p], i32), "bnc_load_checkpoint": ([vp, C.c_char_p], i32),
        "bnc_state_frame": ([vp, vp, C.c_uint64, vp], i32),
        "bnc_set_diffusion_mode": ([vp, u32, C.c_double, u32], i32),
        "bnc_diffusion_stats": ([vp, vp, i32], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def last_error():
    return load_library().bnc_last_error().decode()


def _check(rc, what):
    if rc != 0:
        raise BackendError("%s failed (%d): %s" % (what, rc, last_error()))


class Network:
    """A generated network in host AoS arrays (reference layout), owned by the library."""

    def __init__(self, params):
        lib = load_library()
        self.params = params
        self.data = BionData()
        self._stim = C.c_void_p()
        ns = C.c_uint32()
        _check(lib.bnc_netgen_aos(C.byref(params), C.byref(self.data), C.byref(self._stim), C.byref(ns)),
               "bnc_netgen_aos")
        self.n_stim = ns.value

    @property
    def segments(self):
        return view(self.data.segments, SEGMENT_DTYPE, self.data.num_segments)

    @property
    def synapses(self):
        return view(self.data.synapses, SYNAPSE_DTYPE, self.data.num_synapses)

    @property
    def connections(self):
        return view(self.data.connections, CONN_DTYPE, self.data.num_connections)

    @property
    def stimuli(self):
        return view(self._stim.value, STIM_DTYPE, self.n_stim)

    @property
    def stim_ptr(self):
        return self._stim.value

    def close(self):
        if self.data.segments:
            load_library().bnc_netgen_free(C.byref(self.data), self._stim)
            self._stim = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Backend:
    """One simulation on one GPU (the reference's `Simulation` behind gpu_backend_*)."""

    def __init__(self, device=0):
        self.lib = load_library()
        if self.lib.gpu_backend_device_count() <= 0:
            raise BackendError("no CUDA device visible")
        self.h = self.lib.gpu_backend_create_on_device(device)
        if not self.h:
            raise BackendError("gpu_backend_create_on_device failed: " + last_error())

    def close(self):
        if self.h:
            self.lib.gpu_backend_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # drop-in calls
    def load_bion(self, path):
        _check(self.lib.gpu_backend_load_bion(self.h, path.encode()), "gpu_backend_load_bion")

    def run_tick(self, dt):
        self.lib.gpu_backend_run_tick(self.h, C.c_float(dt))

    def bion_data(self):
        p = self.lib.gpu_backend_bion_data(self.h)
        return BionData.from_address(p) if p else None

    # new calls
    def load_network(self, net):
        _check(self.lib.bnc_load_aos(self.h, C.byref(net.data), net.stim_ptr, net.n_stim), "bnc_load_aos")

    def load_generated(self, params, options=None):
        if options is None:
            _check(self.lib.bnc_load_generated(self.h, C.byref(params)), "bnc_load_generated")
        else:
            _check(self.lib.bnc_load_generated_opts(self.h, C.byref(params), C.byref(options)),
                   "bnc_load_generated_opts")

    def upload_mechano(self, items):
        """bnc_upload_mechano with (segment_id, mod_type, state_idx, value) tuples."""
        from .abi import mechano_data
        arr, n = mechano_data(items)
        _check(self.lib.bnc_upload_mechano(self.h, arr, n), "bnc_upload_mechano")

    def upload_stimuli(self, data):
        """gpu_backend_upload_stimuli with a GpuStimulusData (abi.stimulus_data): replaces
        every stimulus list; ion and ligand injections apply once, at the next tick.  The
        reference call returns nothing, so a rejected upload shows as bnc_last_error()."""
        self.lib.gpu_backend_upload_stimuli(self.h, C.byref(data))
        err = last_error()
        if err:
            raise BackendError("gpu_backend_upload_stimuli: " + err)

    def run_ticks(self, n, dt):
        _check(self.lib.bnc_run_ticks(self.h, n, C.c_float(dt)), "bnc_run_ticks")

    def run_ticks_graph(self, n, dt):
        _check(self.lib.bnc_run_ticks_graph(self.h, n, C.c_float(dt)), "bnc_run_ticks_graph")

    def load_ensemble(self, params):
        arr = params if isinstance(params, C.Array) else (NetgenParams * len(params))(*params)
        _check(self.lib.bnc_load_ensemble_generated(self.h, arr, len(arr)), "bnc_load_ensemble_generated")

    def load_ensemble_networks(self, nets):
        """Ensemble of host-AoS Networks (copied; the Networks stay valid)."""
        from .abi import BionData
        data = (BionData * len(nets))(*[n.data for n in nets])
        stims = (C.c_void_p * len(nets))(*[n.stim_ptr for n in nets])
        counts = (C.c_uint32 * len(nets))(*[n.n_stim for n in nets])
        _check(self.lib.bnc_load_ensemble_aos(self.h, data, stims, counts, len(nets)), "bnc_load_ensemble_aos")

    def load_ensemble_tuned(self, params, trial_ticks, dt):
        arr = params if isinstance(params, C.Array) else (NetgenParams * len(params))(*params)
        t = Tuning()
        _check(self.lib.bnc_load_ensemble_tuned(self.h, arr, len(arr), trial_ticks, C.c_float(dt), C.byref(t)),
               "bnc_load_ensemble_tuned")
        return t

    def time_ticks_graph(self, n, dt):
        ms = C.c_float()
        _check(self.lib.bnc_time_ticks_graph(self.h, n, C.c_float(dt), C.byref(ms)), "bnc_time_ticks_graph")
        return ms.value

    def ensemble_member(self, m):
        out = EnsembleMember()
        _check(self.lib.bnc_ensemble_member(self.h, m, C.byref(out)), "bnc_ensemble_member")
        return out

    def time_ticks(self, n, dt):
        ms = C.c_float()
        _check(self.lib.bnc_time_ticks(self.h, n, C.c_float(dt), C.byref(ms)), "bnc_time_ticks")
        return ms.value

    def step_io(self, dt, stim_amp_ptr=0, n_amp=0, v_out_ptr=0, n_v=0):
        """One tick with host<->device copies (pointers to host buffers, pinned for async)."""
        _check(self.lib.bnc_step_io(self.h, C.c_float(dt), stim_amp_ptr or None, n_amp, v_out_ptr or None, n_v),
               "bnc_step_io")

    def profile_ticks(self, n, dt):
        """Runs n ticks; returns summed ms in (k_modifiers, k_diffusion, k_synapse)."""
        a, b, c = C.c_float(), C.c_float(), C.c_float()
        _check(self.lib.bnc_profile_ticks(self.h, n, C.c_float(dt), C.byref(a), C.byref(b), C.byref(c)),
               "bnc_profile_ticks")
        return a.value, b.value, c.value

    def sync_to_host(self):
        _check(self.lib.bnc_sync_to_host(self.h), "bnc_sync_to_host")

    def info(self):
        inf = NetInfo()
        _check(self.lib.bnc_network_info(self.h, C.byref(inf)), "bnc_network_info")
        return inf

    def segment_field(self, field, index=0):
        n = self.info().n_segments
        out = np.empty(n, np.float32)
        _check(self.lib.bnc_read_segment_field(self.h, SEG_FIELDS.get(field, field), index,
                                               out.ctypes.data, n), "bnc_read_segment_field")
        return out

    def synapse_field(self, field, index=0, n_total=None):
        n = n_total if n_total is not None else self.info().n_synapses
        out = np.empty(max(n, 1), np.float32)
        _check(self.lib.bnc_read_synapse_field(self.h, SYN_FIELDS.get(field, field), index,
                                               out.ctypes.data, n), "bnc_read_synapse_field")
        return out[:n]

    def set_synapse_scale(self, scale):
        s = np.ascontiguousarray(scale, np.float32)
        _check(self.lib.bnc_set_synapse_scale(self.h, s.ctypes.data, s.size), "bnc_set_synapse_scale")

    def state_frame(self):
        """The daemon's state-frame payload (bytes) from the device state."""
        n = C.c_uint64()
        self.lib.bnc_state_frame(self.h, None, 0, C.byref(n))
        buf = (C.c_uint8 * n.value)()
        _check(self.lib.bnc_state_frame(self.h, buf, n.value, C.byref(n)), "bnc_state_frame")
        return bytes(buf)

    def set_diffusion_mode(self, flags, tol=1e-6, max_sweeps=100000):
        """Step 2.5 options: DIFFUSION_RESIDUAL (FP64 Jacobi solves to `tol`, at most
        `max_sweeps` sweeps) and DIFFUSION_LEDGER (the per-ion FP64 ledger); 0 restores
        the reference's fixed 50 sweeps."""
        _check(self.lib.bnc_set_diffusion_mode(self.h, flags, C.c_double(tol), max_sweeps), "bnc_set_diffusion_mode")

    def diffusion_stats(self, reset=False):
        out = DiffusionStats()
        _check(self.lib.bnc_diffusion_stats(self.h, C.byref(out), 1 if reset else 0), "bnc_diffusion_stats")
        return out

    def save_checkpoint(self, path):
        _check(self.lib.bnc_save_checkpoint(self.h, str(path).encode()), "bnc_save_checkpoint")

    def load_checkpoint(self, path):
        _check(self.lib.bnc_load_checkpoint(self.h, str(path).encode()), "bnc_load_checkpoint")

    def save_bion(self, path):
        _check(self.lib.bnc_save_bion(self.h, path.encode()), "bnc_save_bion")


__all__ = ["Backend", "Network", "Adjoint", "AdjointConfig", "AdjointInfo", "SweepTask", "SweepResult",
           "sweep_parse_params", "sweep_tasks", "sweep_run", "SWEEP_SINGLE_TICK", "NetgenParams", "BionData", "BackendError", "load_library", "last_error",
           "NET_SMALL", "NET_LARGE", "NET_TREES", "NET_ENSEMBLE_MEMBER", "NET_ADJOINT", "NETGEN_NO_SYNAPSES",
           "NETGEN_NO_CONNECTIONS", "NETGEN_NO_STIMULI", "NETGEN_PERTURB_IONS", "NETGEN_SYNAPSE_EXTRAS", "NETGEN_FULL_SMALL_SET", "NETGEN_GLYCINE", "NETGEN_DRAW_ORDER", "NETGEN_RELEASE_MODULATORS", "NETGEN_ECB", "NETGEN_GLIA", "NETGEN_GAP_JUNCTIONS", "NETGEN_NMDA", "SEG_FIELDS", "SYN_FIELDS",
           "DROPIN_SYMBOLS", "NEW_SYMBOLS", "EnsembleMember", "Tuning", "BuildOptions", "register_device_modifier", "ensemble_params", "plan_ensemble", "plan_generated",
           "DIFFUSION_RESIDUAL", "DIFFUSION_LEDGER", "DiffusionStats"]


class AdjointConfig(C.Structure):
    _fields_ = [("n_sets", C.c_uint32), ("ticks", C.c_uint32), ("checkpoint_every", C.c_uint32),
                ("sample_every", C.c_uint32), ("dt", C.c_float)]


class AdjointInfo(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("n_neurons", "n_segments", "n_synapses", "n_samples", "n_sets", "ticks",
                                          "checkpoint_every", "threads", "smem_forward", "smem_backward")] + \
               [(n, C.c_uint64) for n in ("checkpoint_bytes", "window_bytes", "scratch_bytes")]


def _fptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Adjoint:
    """Gradients of a somatic voltage-trace loss w.r.t. per-segment gNa/gK/gleak and
    per-synapse weights, for `n_sets` parameter sets at once (bnc_adjoint_*).

    Built from the network loaded in `backend` at its current tick; `record()` then runs
    the plain tick for `ticks` ticks on that backend and keeps the release log that the
    forward and backward passes replay (releases are pathwise fixed)."""

    def __init__(self, backend, n_sets, ticks, dt, checkpoint_every=256, sample_every=1):
        lib = load_library()
        self.cfg = AdjointConfig(n_sets, ticks, checkpoint_every, sample_every, dt)
        h = lib.bnc_adjoint_create(backend.h, C.byref(self.cfg))
        if not h:
            raise BackendError("bnc_adjoint_create failed: %s" % last_error())
        self.h = h
        self.backend = backend
        inf = AdjointInfo()
        _check(lib.bnc_adjoint_info(h, C.byref(inf)), "bnc_adjoint_info")
        self.info = inf
        import numpy as np
        self.soma = np.zeros(inf.n_neurons, np.uint32)
        _check(lib.bnc_adjoint_soma(h, _fptr(self.soma), inf.n_neurons), "bnc_adjoint_soma")

    def close(self):
        if getattr(self, "h", None):
            load_library().bnc_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def record(self):
        _check(load_library().bnc_adjoint_record(self.h, self.backend.h), "bnc_adjoint_record")

    def release_count(self):
        n = C.c_uint64()
        _check(load_library().bnc_adjoint_release_count(self.h, C.byref(n)), "bnc_adjoint_release_count")
        return n.value

    def set_params(self, p, gNa=None, gK=None, gleak=None, w=None):
        import numpy as np
        arr = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (gNa, gK, gleak, w)]
        _check(load_library().bnc_adjoint_set_params(self.h, p, *[_fptr(a) for a in arr]), "bnc_adjoint_set_params")

    def get_params(self, p):
        import numpy as np
        i = self.info
        out = [np.zeros(i.n_segments, np.float32) for _ in range(3)] + [np.zeros(max(i.n_synapses, 1), np.float32)]
        _check(load_library().bnc_adjoint_get_params(self.h, p, *[_fptr(a) for a in out]), "bnc_adjoint_get_params")
        out[3] = out[3][:i.n_synapses]
        return out

    def set_target(self, target):
        import numpy as np
        t = np.ascontiguousarray(target, np.float32).reshape(self.info.n_samples, self.info.n_neurons)
        _check(load_library().bnc_adjoint_set_target(self.h, _fptr(t)), "bnc_adjoint_set_target")

    def forward(self, trace=False):
        """Returns (loss[n_sets], trace[n_sets][n_samples][n_neurons] or None)."""
        import numpy as np
        i = self.info
        loss = np.zeros(i.n_sets, np.float64)
        tr = np.zeros((i.n_sets, i.n_samples, i.n_neurons), np.float32) if trace else None
        _check(load_library().bnc_adjoint_forward(self.h, _fptr(loss), _fptr(tr)), "bnc_adjoint_forward")
        return loss, tr

    def backward(self):
        """Returns (g_gNa, g_gK, g_gleak) as [n_sets][n_segments] and g_w as [n_sets][n_synapses]."""
        import numpy as np
        i = self.info
        g = [np.zeros((i.n_sets, i.n_segments), np.float32) for _ in range(3)]
        gw = np.zeros((i.n_sets, max(i.n_synapses, 1)), np.float32)
        _check(load_library().bnc_adjoint_backward(self.h, *[_fptr(a) for a in g], _fptr(gw)), "bnc_adjoint_backward")
        return g[0], g[1], g[2], gw[:, :i.n_synapses]

    def timings(self):
        f, b = C.c_float(), C.c_float()
        _check(load_library().bnc_adjoint_timings(self.h, C.byref(f), C.byref(b)), "bnc_adjoint_timings")
        return f.value, b.value


SWEEP_SINGLE_TICK = 1


class SweepTask(C.Structure):
    _fields_ = [("type_ids", C.c_void_p), ("values", C.c_void_p), ("n_overrides", C.c_uint32), ("seed", C.c_uint32)]


class SweepResult(C.Structure):
    _fields_ = [("mean_vm", C.c_float), ("spike_count", C.c_uint32), ("synchrony", C.c_float), ("tick", C.c_uint64),
                ("metrics_json", C.c_char * 2048)]


def sweep_parse_params(text, names=None):
    """The reference's parameter JSON as [(type_id, value), ...] (bnc_sweep_parse_params);
    `names` maps modifier names to type IDs for non-numeric keys."""
    import numpy as np
    names = names or {}
    nm = (C.c_char_p * max(len(names), 1))(*[k.encode() for k in names])
    ids = np.array(list(names.values()) or [0], np.uint8)
    cap = 256
    tid = np.zeros(cap, np.uint8)
    val = np.zeros(cap, np.float32)
    n = C.c_uint32()
    _check(load_library().bnc_sweep_parse_params(text.encode(), nm, ids.ctypes.data_as(C.c_void_p), len(names),
                                                 tid.ctypes.data_as(C.c_void_p), val.ctypes.data_as(C.c_void_p),
                                                 cap, C.byref(n)), "bnc_sweep_parse_params")
    return [(int(tid[q]), float(val[q])) for q in range(n.value)]


def sweep_tasks(tasks):
    """[(overrides [(type_id, value)], seed), ...] -> (ctypes array of SweepTask, keep-alive arrays)."""
    import numpy as np
    keep = []
    arr = (SweepTask * len(tasks))()
    for q, (ov, seed) in enumerate(tasks):
        ids = np.array([t for t, _ in ov] or [0], np.uint8)
        vals = np.array([v for _, v in ov] or [0.0], np.float32)
        keep += [ids, vals]
        arr[q] = SweepTask(ids.ctypes.data_as(C.c_void_p), vals.ctypes.data_as(C.c_void_p), len(ov), seed)
    return arr, keep


def sweep_run(backend, net, tasks, ticks, dt=0.1, single_tick=False):
    """Runs the tasks as one ensemble in `backend` (bnc_sweep_run); returns the
    per-task SweepResult list."""
    arr, keep = sweep_tasks(tasks)
    res = (SweepResult * len(tasks))()
    _check(load_library().bnc_sweep_run(backend.h, C.byref(net.data), net.stim_ptr, net.n_stim, arr, len(tasks), ticks,
                                        C.c_float(dt), SWEEP_SINGLE_TICK if single_tick else 0, res), "bnc_sweep_run")
    return list(res)
