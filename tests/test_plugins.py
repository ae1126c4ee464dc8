"""Reference modifier plugins binding to this backend (plugin_host.cpp).

A reference plugin exports biocore_plugin_init and biocore_plugin_desc and registers
CPU functions through register_modifier_current / register_modulator_release (C
linkage) or register_user_modifier / register_user_modulator (C++ linkage), as
plugins/builtin/*.cpp do against modifier_interface.h:38-39 and
plugin_manager.h:98-99.  Here tiny plugins of both kinds are compiled with the
reference's declarations restated and loaded through bnc_plugin_load: they must bind
to this library's exports, their registrations must be recorded, and a network that
uses a registered ID must be refused (no CPU fallback) until device code is registered
for it.  The loader's error codes follow plugin_load (plugin_manager.cpp:208-258).
"""
import ctypes as C
import shutil
import subprocess

import numpy as np
import pytest

BNC_ERR_UNSUPPORTED = -21

C_PLUGIN = r'''
#include <stdint.h>
struct Modifier; struct Segment;
typedef double (*ModifierFunc)(struct Modifier*, struct Segment*, float);
typedef float (*ReleaseModulatorFunc)(struct Modifier*, float*, float);
extern void register_modifier_current(uint8_t type, ModifierFunc func);
extern void register_modulator_release(uint8_t type, ReleaseModulatorFunc func);
static double cur(struct Modifier* m, struct Segment* s, float dt) { (void)m; (void)s; (void)dt; return 0.0; }
static float rel(struct Modifier* m, float* nt, float dt) { (void)m; (void)nt; (void)dt; return 1.0f; }
int biocore_plugin_init(void) {
    register_modifier_current(44, cur);     /* a user ID */
    register_modifier_current(7, cur);      /* overrides the built-in Na/K pump */
    register_modulator_release(45, rel);
    register_modifier_current(200, cur);    /* >= 128: ignored, as by the reference */
    return 4;
}
const char* biocore_plugin_desc(void) {
    return "{\"name\":\"test_c\",\"version\":\"1.0\",\"author\":\"t\",\"modifiers\":["
           "{\"id\":44,\"name\":\"a\",\"release\":false},{\"id\":7,\"name\":\"b\",\"release\":false},"
           "{\"id\":45,\"name\":\"c\",\"release\":true}]}";
}
'''

CPP_PLUGIN = r'''
#include <cstdint>
struct Modifier; struct Segment;
typedef double (*ModifierFunc)(Modifier* mod, Segment* seg, float dt);
void register_user_modifier(uint8_t type, ModifierFunc func);   // C++ linkage, as plugin_manager.h:98
static double cur(Modifier*, Segment*, float) { return 0.0; }
extern "C" int biocore_plugin_init() { register_user_modifier(46, cur); return 1; }
'''

NO_INIT = "int something_else(void) { return 1; }\n"
ZERO_INIT = "int biocore_plugin_init(void) { return 0; }\n"


@pytest.fixture()
def lib():
    from bioneuroncore_b200 import load_library
    L = load_library()
    L.bnc_plugin_load.argtypes = [C.c_char_p]
    L.bnc_plugin_load_directory.argtypes = [C.c_char_p]
    L.bnc_plugin_registered.argtypes = [C.c_uint8]
    L.bnc_plugin_unregister_all()
    yield L
    L.bnc_plugin_unregister_all()


def _build(tmp_path, name, src, cpp=False):
    cc = shutil.which("g++" if cpp else "gcc")
    if cc is None:
        pytest.skip("no compiler")
    f = tmp_path / (name + (".cpp" if cpp else ".c"))
    f.write_text(src)
    so = tmp_path / (name + ".so")
    # undefined register_* stay unresolved until load time, as in a reference plugin
    subprocess.run([cc, "-O2", "-fPIC", "-shared", "-o", str(so), str(f)], check=True)
    return so


def _net_with_type(t, family="small"):
    from bioneuroncore_b200 import Network, NetgenParams, NET_SMALL
    net = Network(NetgenParams(family=NET_SMALL, n_neurons=2, seed=3))
    if t is not None:
        seg = net.segments
        c = int(seg["modifier_count"][0])
        mods = seg["modifiers"][0]
        mods[c] = np.zeros((), dtype=mods.dtype)
        mods[c]["type"] = t
        mods[c]["density"] = np.float32(0.5)
        seg["modifier_count"][0] = c + 1
    return net


def _plan(net):
    from bioneuroncore_b200 import load_library, NetInfo
    info = NetInfo()
    return load_library().bnc_plan_aos(C.byref(net.data), net.stim_ptr, net.n_stim, C.byref(info))


def test_c_and_cpp_plugins_bind_and_register(tmp_path, lib):
    so_c = _build(tmp_path, "plug_c", C_PLUGIN)
    so_cpp = _build(tmp_path, "plug_cpp", CPP_PLUGIN, cpp=True)
    n0 = lib.bnc_plugin_count()
    assert lib.bnc_plugin_load(str(so_c).encode()) == 4
    assert lib.bnc_plugin_load(str(so_cpp).encode()) == 1
    assert lib.bnc_plugin_count() == n0 + 2
    assert lib.bnc_plugin_registered(44) == 1
    assert lib.bnc_plugin_registered(7) == 1
    assert lib.bnc_plugin_registered(45) == 2
    assert lib.bnc_plugin_registered(46) == 1      # through the C++-linkage entry
    assert lib.bnc_plugin_registered(200) == 0     # IDs >= 128 are ignored
    assert lib.bnc_plugin_registered(43) == 0


def test_networks_using_host_registered_ids_are_refused(tmp_path, lib):
    from bioneuroncore_b200 import last_error
    assert _plan(_net_with_type(None)) == 0
    so_c = _build(tmp_path, "plug_c", C_PLUGIN)
    assert lib.bnc_plugin_load(str(so_c).encode()) == 4
    # the small family carries the Na/K pump (7) on every segment: the plugin overrides
    # it on the reference's CPU path, which this backend cannot run
    assert _plan(_net_with_type(None)) == BNC_ERR_UNSUPPORTED
    assert "host plugin" in last_error()
    lib.bnc_plugin_unregister_all()
    assert _plan(_net_with_type(None)) == 0
    lib.register_modifier_current.argtypes = [C.c_uint8, C.c_void_p]
    lib.register_modifier_current(44, C.cast(lib.bnc_plugin_count, C.c_void_p))   # any non-null function
    assert _plan(_net_with_type(44)) == BNC_ERR_UNSUPPORTED
    assert "host plugin" in last_error()


def test_device_code_registered_for_the_id_is_accepted(tmp_path, lib):
    from bioneuroncore_b200 import register_device_modifier
    src = r'''
#include "bnc_device_modifier.h"
extern "C" __global__ void leak47(BncDeviceModifierArgs a) {
    unsigned int q = a.begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.end) return;
    BncSegmentState* s = a.seg + a.item_seg[q];
    s->itot += (double)(a.density[q] * (-70.0f - s->V));
}
'''
    lib.register_modifier_current.argtypes = [C.c_uint8, C.c_void_p]
    lib.register_modifier_current(47, C.cast(lib.bnc_plugin_count, C.c_void_p))
    assert _plan(_net_with_type(47)) == BNC_ERR_UNSUPPORTED
    register_device_modifier(47, src, "leak47")
    assert _plan(_net_with_type(47)) == 0


def test_loader_error_codes(tmp_path, lib):
    assert lib.bnc_plugin_load(str(tmp_path / "missing.so").encode()) == -1
    assert lib.bnc_plugin_load(str(_build(tmp_path, "noinit", NO_INIT)).encode()) == -2
    assert lib.bnc_plugin_load(str(_build(tmp_path, "zeroinit", ZERO_INIT)).encode()) == -3


def test_directory_load(tmp_path, lib):
    d = tmp_path / "plugins"
    d.mkdir()
    _build(d, "a", C_PLUGIN)
    _build(d, "b", CPP_PLUGIN, cpp=True)
    (d / "notes.txt").write_text("not a plugin")
    for p in d.glob("*.c*"):
        p.unlink()
    assert lib.bnc_plugin_load_directory(str(d).encode()) == 5
