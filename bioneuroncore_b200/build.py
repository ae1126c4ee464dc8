"""Builds the backend's shared library (and, for tests, the CPU oracle).

    python -m bioneuroncore_b200.build            # product library only
    python -m bioneuroncore_b200.build --oracle   # also oracle/liboracle.so (+ reference if present)

The CUDA translation units are compiled for sm_100a only, with --fmad=false so no
multiply-add is contracted behind the source's back (the kernels restate the
reference's arithmetic operation by operation).  Outputs stay in the source tree.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libbnc_b200.so")
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle.so")
ORACLE64_LIB = os.path.join(ORACLE_DIR, "liboracle64.so")

CU_SOURCES = ["modifiers.cu", "diffuse.cu", "synapse.cu", "backend.cu", "plugins.cu", "adjoint.cu", "convert.cu"]
CPP_SOURCES = ["netgen.cpp", "capi_host.cpp", "builder.cpp", "sweep.cpp", "plugin_host.cpp", "bion_file.cpp"]
HEADERS = sorted(f for f in os.listdir(CSRC) if f.endswith((".h", ".cuh")))

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-I" + os.path.join(ROOT, "include"), "-I" + BUILD]


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def _embed_header():
    """Writes include/bnc_device_modifier.h as a C++ raw string literal into the build
    folder; plugins.cu hands it to NVRTC so user sources can include it."""
    src = os.path.join(ROOT, "include", "bnc_device_modifier.h")
    out = os.path.join(BUILD, "bnc_device_modifier_h.inc")
    if _stale(out, [src]):
        text = open(src).read()
        assert ")BNCH\"" not in text
        with open(out, "w") as f:
            f.write('R"BNCH(' + text + ')BNCH"\n')


def build_library(verbose=False, ptxas_info=False):
    """Compiles libbnc_b200.so (sm_100a) if any source changed; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", f)
                                                        for f in ("bnc_abi.h", "bnc_b200.h",
                                                                  "bnc_device_modifier.h")]
    _embed_header()
    jobs = []
    objs = []
    for src in CU_SOURCES + CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers + [__file__]):
            cmd = [nvcc] + GENCODE + NVCC_FLAGS + ["-c", s, "-o", o]
            if src.endswith(".cpp"):
                cmd = [nvcc] + GENCODE + NVCC_FLAGS + ["-x", "c++", "-c", s, "-o", o]
            if ptxas_info and src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)
    logs = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            logs = list(ex.map(_run, jobs))
    if jobs or _stale(LIB, objs):
        _run([nvcc] + GENCODE + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    if verbose:
        for l in logs:
            if l.strip():
                print(l)
    return LIB


TANGENT_LIB = os.path.join(ORACLE_DIR, "libbo_tangent.so")


def build_oracle():
    """Compiles the CPU oracle (test infrastructure) with contraction disabled: the FP32
    tick restatement, the same source with FP64 state and the C library's elementary
    functions (liboracle64.so, checked against the reference's own tick), and the FP64
    forward-mode replay that checks the adjoint."""
    srcs = [os.path.join(ORACLE_DIR, f) for f in ("bnc_oracle.c", "bo_math.h", "bo_physics.h", "bo_modifiers.h")]
    abi = os.path.join(ROOT, "include", "bnc_abi.h")
    if _stale(ORACLE_LIB, srcs + [abi]):
        _run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", ORACLE_LIB,
              os.path.join(ORACLE_DIR, "bnc_oracle.c"), "-lm"])
    if _stale(ORACLE64_LIB, srcs + [abi]):
        _run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-DBO_FP64", "-DBO_LIBM", "-fPIC", "-shared",
              "-o", ORACLE64_LIB, os.path.join(ORACLE_DIR, "bnc_oracle.c"), "-lm"])
    tsrc = os.path.join(ORACLE_DIR, "bo_tangent.cpp")
    if _stale(TANGENT_LIB, [tsrc, abi]):
        _run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", TANGENT_LIB, tsrc, "-lm"])
    return ORACLE_LIB


def build_reference(ref_dir=None):
    """Builds the reference CPU library into oracle/_ref/ from the reference checkout
    at `ref_dir` (else $BNC_REFERENCE_DIR); returns None when neither names one."""
    ref_dir = ref_dir or os.environ.get("BNC_REFERENCE_DIR")
    if not ref_dir or not os.path.isdir(os.path.join(ref_dir, "src")):
        return None
    _run(["make", "-s", "-C", ORACLE_DIR, "-j8", "REF=" + os.path.abspath(ref_dir)])
    return os.path.join(ORACLE_DIR, "_ref", "libbiocore_ref.so")


def ensure_built():
    """Builds the product library and the oracle only when their files are missing."""
    if not os.path.exists(LIB):
        build_library()
    if not all(os.path.exists(p) for p in (ORACLE_LIB, ORACLE64_LIB, TANGENT_LIB)):
        build_oracle()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--oracle", action="store_true")
    ap.add_argument("--ptxas", action="store_true")
    ap.add_argument("--reference", default=None, help="reference checkout to build oracle/_ref/ from")
    a = ap.parse_args(argv)
    print(build_library(verbose=True, ptxas_info=a.ptxas))
    if a.oracle:
        print(build_oracle())
        print(build_reference(a.reference))


if __name__ == "__main__":
    sys.exit(main())
