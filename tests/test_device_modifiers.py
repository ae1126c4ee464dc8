"""User modifiers on the device (modifier IDs 0-127), registered as CUDA source.

CPU part: registration compiles with NVRTC without a GPU; compile errors and
out-of-range IDs are reported; the planner rejects a network that uses an ID
with neither a built-in model nor a registration, and accepts it afterwards.

GPU part (marked gpu): the same model as a device modifier and as a C plugin of
the oracle (the reference's CPU plugin path, kernel_dispatch.h:336-343) give
bit-identical ticks, with the modifier placed between built-in ones in the
segment's slot order.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

USER_TYPE = 20   # in the reference's plugin range 0-127, no built-in model

DEVICE_SRC = r'''
#include "bnc_device_modifier.h"
// linear leak towards -70 mV that also counts time in state word 0 and moves K+
extern "C" __global__ void lin_leak(BncDeviceModifierArgs a) {
    unsigned int q = a.begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.end) return;
    BncSegmentState* s = a.seg + a.item_seg[q];
    float I = a.density[q] * (-70.0f - s->V);
    a.state[q] = a.state[q] + a.dt;
    s->in[1] = s->in[1] + 1e-7f * I;
    s->itot += (double)I;
}
'''

ORACLE_SRC = r'''
typedef struct {
    float* V; float* in; float* out; float* atp;
    float area; double vol; float density; float* state; unsigned char type;
} BoPluginView;
double lin_leak(BoPluginView* v, float dt) {
    float I = v->density * (-70.0f - *v->V);
    v->state[0] = v->state[0] + dt;
    v->in[1] = v->in[1] + 1e-7f * I;
    return (double)I;
}
'''


def _register_device():
    from bioneuroncore_b200 import register_device_modifier
    register_device_modifier(USER_TYPE, DEVICE_SRC, "lin_leak")


def _with_user_modifiers(net, every=3, density=0.5):
    """Inserts a USER_TYPE modifier at slot 1 of every `every`-th segment."""
    seg = net.segments
    for i in range(0, net.data.num_segments, every):
        c = int(seg["modifier_count"][i])
        mods = seg["modifiers"][i]
        mods[2:c + 1] = mods[1:c].copy()
        mods[1] = np.zeros((), dtype=mods.dtype)
        mods[1]["type"] = USER_TYPE
        mods[1]["density"] = np.float32(density)
        seg["modifier_count"][i] = c + 1
    return net


def _plan(net):
    from bioneuroncore_b200 import load_library, NetInfo
    info = NetInfo()
    return load_library().bnc_plan_aos(C.byref(net.data), net.stim_ptr, net.n_stim, C.byref(info))


def test_registration_errors():
    from bioneuroncore_b200 import register_device_modifier, BackendError, last_error, load_library
    with pytest.raises(BackendError):
        register_device_modifier(128, DEVICE_SRC, "lin_leak")
    with pytest.raises(BackendError):
        register_device_modifier(21, "this is not CUDA", "k")
    assert "does not compile" in last_error()
    assert load_library().bnc_device_modifier_registered(21) == 0


def test_registration_from_file(tmp_path):
    from bioneuroncore_b200 import load_library
    f = tmp_path / "leak.cu"
    f.write_text(DEVICE_SRC)
    lib = load_library()
    assert lib.biocore_gpu_register_device_modifier(22, str(f).encode(), b"lin_leak") == 0
    assert lib.bnc_device_modifier_registered(22) == 1
    assert lib.biocore_gpu_register_device_modifier(23, str(tmp_path / "missing.cu").encode(), b"x") == -1


def test_planner_needs_a_registration_for_user_ids():
    from bioneuroncore_b200 import Network, NetgenParams, NET_SMALL, load_library
    net = _with_user_modifiers(Network(NetgenParams(family=NET_SMALL, n_neurons=2, seed=3)))
    if not load_library().bnc_device_modifier_registered(USER_TYPE):
        assert _plan(net) == -21
    _register_device()
    assert _plan(net) == 0


def _oracle_plugin(tmp_path):
    src = tmp_path / "plugin.c"
    src.write_text(ORACLE_SRC)
    so = tmp_path / "plugin.so"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(so), str(src)], check=True)
    lib = C.CDLL(str(so))
    return lib, C.cast(lib.lin_leak, C.c_void_p).value


@pytest.mark.gpu
def test_device_modifier_matches_oracle_plugin(tmp_path):
    from bioneuroncore_b200 import Backend, Network, NetgenParams, NET_SMALL
    from oracle.oracle import Oracle, oracle_lib
    _register_device()
    plugin_lib, fn = _oracle_plugin(tmp_path)
    assert oracle_lib().bo_register_modifier(USER_TYPE, fn) == 0
    try:
        p = NetgenParams(family=NET_SMALL, n_neurons=6, seed=13)
        net_o = _with_user_modifiers(Network(p))
        net_g = _with_user_modifiers(Network(p))
        ora = Oracle(net_o)
        gpu = Backend()
        gpu.load_network(net_g)
        for step in (1, 15, 30):
            ora.run(step, 0.025)
            gpu.run_ticks(step, 0.025)
            for f, i in [("V", 0), ("ion_in", 0), ("ion_in", 1), ("ion_out", 1), ("ATP", 0), ("spikes", 0)] + [
                    ("mod_state", slot * 8 + k) for slot in range(4) for k in range(2)]:
                a = np.asarray(gpu.segment_field(f, i), np.float32)
                b = np.asarray(ora.segment_field(f, i), np.float32)
                same = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
                assert same.all(), "%s[%d] after +%d: %d differ" % (f, i, step, int((~same).sum()))
        # the user modifier ran: its time counter advanced by dt every tick
        t = np.asarray(gpu.segment_field("mod_state", 1 * 8 + 0), np.float32)[::3]
        assert (t > 0).all()
    finally:
        oracle_lib().bo_register_modifier(USER_TYPE, None)
