"""ABI checks that need no GPU.

- The structures of include/bnc_abi.h have the reference's sizes and field
  offsets (the values asserted by the reference's
  tests/test_abi_segment_layout.cpp:14-57), both as compiled C and as the numpy
  dtypes the Python side uses.
- libbnc_b200.so loads and exports every function include/bnc_b200.h declares,
  including the 12 drop-in gpu_backend_* symbols the reference's loader needs
  (tests/smoke_cuda.sh:24-29).
- The host-only entry points work without a device.
"""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")

# tests/test_abi_segment_layout.cpp:14-57 of the reference
REFERENCE_LAYOUT = {
    "sizeof(BncSegment)": 3216, "offsetof(BncSegment, V_m)": 40, "offsetof(BncSegment, I_buffer)": 3128,
    "offsetof(BncSegment, intra_ions)": 48, "offsetof(BncSegment, extra_ions)": 112,
    "offsetof(BncSegment, segment_type)": 3113, "offsetof(BncSegment, modifier_count)": 3112,
    "offsetof(BncBionData, header)": 0, "offsetof(BncBionData, segments)": 112,
    "offsetof(BncBionData, num_segments)": 148, "sizeof(BncModifier)": 88, "sizeof(BncSynapse)": 1568,
    "sizeof(BncIntraConnection)": 16, "sizeof(BncNeuron)": 24, "sizeof(BncNetworkHeader)": 100,
    "BNC_ION_COUNT": 7, "BNC_ION_MAX": 8, "BNC_NT_COUNT": 15, "BNC_MAX_MODIFIERS": 32,
}

DROPIN = ["gpu_backend_create", "gpu_backend_create_on_device", "gpu_backend_destroy", "gpu_backend_load_bion",
          "gpu_backend_run_tick", "gpu_backend_bion_data", "gpu_backend_upload_stimuli", "gpu_backend_device_count",
          "gpu_backend_get_device_info", "gpu_backend_ibuf_offset", "gpu_backend_vm_offset", "gpu_backend_seg_size"]


def declared_functions():
    text = open(os.path.join(INCLUDE, "bnc_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*\b((?:gpu_backend|bnc|biocore_gpu|register)_[a-z0-9_]+)\s*\(",
                       text, flags=re.M)
    return sorted(set(names))


def test_struct_layout_compiled(tmp_path):
    src = tmp_path / "layout.c"
    body = "\n".join('    printf("%%s %%zu\\n", "%s", (size_t)(%s));' % (k, k) for k in REFERENCE_LAYOUT)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "bnc_abi.h"\nint main(void) {\n%s\n'
                   '    return 0;\n}\n' % body)
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", INCLUDE, "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        k, v = line.rsplit(" ", 1)
        got[k] = int(v)
    assert got == REFERENCE_LAYOUT


def test_numpy_dtypes_match_reference_layout():
    from bioneuroncore_b200.abi import SEGMENT_DTYPE, SYNAPSE_DTYPE, MOD_DTYPE, CONN_DTYPE
    assert SEGMENT_DTYPE.itemsize == 3216
    assert SYNAPSE_DTYPE.itemsize == 1568
    assert MOD_DTYPE.itemsize == 88
    assert CONN_DTYPE.itemsize == 16
    f = SEGMENT_DTYPE.fields
    assert f["V_m"][1] == 40 and f["intra_ions"][1] == 48 and f["extra_ions"][1] == 112
    assert f["modifier_count"][1] == 3112 and f["segment_type"][1] == 3113 and f["I_buffer"][1] == 3128


def test_header_declares_the_dropin_set():
    names = declared_functions()
    for n in DROPIN:
        assert n in names, n


def test_library_exports_every_declared_function():
    from bioneuroncore_b200 import load_library, DROPIN_SYMBOLS, NEW_SYMBOLS
    lib = load_library()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert sorted(DROPIN_SYMBOLS) == sorted(DROPIN)
    assert sorted(DROPIN_SYMBOLS + NEW_SYMBOLS) == names


def test_abi_probe_functions_need_no_device():
    from bioneuroncore_b200 import load_library
    lib = load_library()
    assert lib.gpu_backend_vm_offset() == 40
    assert lib.gpu_backend_ibuf_offset() == 3128
    assert lib.gpu_backend_seg_size() == 3216


def test_null_handles_are_rejected():
    from bioneuroncore_b200 import load_library
    lib = load_library()
    assert lib.bnc_run_ticks(None, 1, C.c_float(0.025)) == -20
    assert lib.bnc_run_ticks_static_scratch(None, 1, C.c_float(0.025)) == -20
    assert lib.gpu_backend_load_bion(None, b"x.bion") == -1
    assert lib.bnc_plan_generated(None, None) == -20
    assert "null" in lib.bnc_last_error().decode()
