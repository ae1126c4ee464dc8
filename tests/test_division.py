"""The diffusion kernel's divisions by a precomputed reciprocal (diffuse.cu).

div_by_float: a / b from y = RN(1 / b) with one fma correction; the claim is that the
result is the IEEE binary64 quotient for every double a and every b that holds a
float value.  div_rn_f and div_rn_d: the same correction (Markstein's) for binary32
and binary64 operands, inside a guarded range (else the hardware division); the claim
is the IEEE quotient of the operands' own precision.  This test restates the same
operations in C (IEEE arithmetic with a fused multiply-add, as on the GPU) and
compares them bit for bit with a / b on random operands, on operands whose quotient
lies next to a rounding midpoint (the hard cases of rounding), on divisors whose
significand is all ones or a power of two, and on zeros, infinities, NaNs and tiny
values.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

SRC = r"""
#include <math.h>
#include <stdint.h>
#include <string.h>

static double div_by_float(double a, double b, double y) {
    const double q0 = a * y;
    const double r = fma(-q0, b, a);
    const double aq = fabs(q0);
    if (aq >= 0x1p-900 && aq <= 0x1.fffffffffffffp+1023) return fma(r, y, q0);
    if (aq == 0.0) return q0;
    return a / b;
}

static float div_rn_f(float a, float b, float y) {
    const float aa = fabsf(a), ab = fabsf(b);
    if (aa >= 0x1p-64f && aa <= 0x1p64f && ab >= 0x1p-32f && ab <= 0x1p32f) {
        const float q0 = a * y;
        const float r = fmaf(-q0, b, a);
        return fmaf(r, y, q0);
    }
    return a / b;
}

static double div_rn_d(double a, double b, double y) {
    const double q0 = a * y;
    const double aq = fabs(q0), ab = fabs(b);
    if (aq >= 0x1p-500 && aq <= 0x1p500 && ab >= 0x1p-500 && ab <= 0x1p500) {
        const double r = fma(-q0, b, a);
        return fma(r, y, q0);
    }
    return a / b;
}

long check_f(const float* a, const float* b, long n, long* first) {
    long bad = 0;
    *first = -1;
    for (long k = 0; k < n; k++) {
        const float q = div_rn_f(a[k], b[k], 1.0f / b[k]), ref = a[k] / b[k];
        uint32_t x, z;
        memcpy(&x, &q, 4);
        memcpy(&z, &ref, 4);
        if (x != z && !(isnan(q) && isnan(ref))) { if (*first < 0) *first = k; bad++; }
    }
    return bad;
}

long check_d(const double* a, const double* b, long n, long* first) {
    long bad = 0;
    *first = -1;
    for (long k = 0; k < n; k++) {
        const double q = div_rn_d(a[k], b[k], 1.0 / b[k]), ref = a[k] / b[k];
        uint64_t x, z;
        memcpy(&x, &q, 8);
        memcpy(&z, &ref, 8);
        if (x != z && !(isnan(q) && isnan(ref))) { if (*first < 0) *first = k; bad++; }
    }
    return bad;
}

/* counts mismatches between div_by_float(a[k], b[k], 1 / b[k]) and a[k] / b[k] */
long check(const double* a, const float* b, long n, long* first) {
    long bad = 0;
    *first = -1;
    for (long k = 0; k < n; k++) {
        const double bd = (double)b[k];
        const double y = 1.0 / bd;
        const double q = div_by_float(a[k], bd, y);
        const double ref = a[k] / bd;
        uint64_t x, z;
        memcpy(&x, &q, 8);
        memcpy(&z, &ref, 8);
        if (x != z && !(isnan(q) && isnan(ref))) { if (*first < 0) *first = k; bad++; }
    }
    return bad;
}
"""


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    gcc = shutil.which("gcc") or shutil.which("cc")
    if gcc is None:
        pytest.skip("no C compiler")
    d = tmp_path_factory.mktemp("div")
    src = d / "div.c"
    src.write_text(SRC)
    so = d / "libdiv.so"
    subprocess.run([gcc, "-O2", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC", str(src), "-o", str(so),
                    "-lm"], check=True)
    L = C.CDLL(str(so))
    for f in (L.check, L.check_f, L.check_d):
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_long, C.POINTER(C.c_long)]
        f.restype = C.c_long
    return L


def _run(lib, a, b):
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float32)
    first = C.c_long()
    bad = lib.check(a.ctypes.data, b.ctypes.data, a.size, C.byref(first))
    assert bad == 0, "%d mismatches, first a=%r b=%r" % (bad, a[first.value], b[first.value])


def test_random_operands(lib):
    rng = np.random.default_rng(1)
    n = 4_000_000
    # full 53-bit dividends over a wide range, float divisors like segment volumes
    a = rng.standard_normal(n) * np.exp2(rng.integers(-60, 60, n))
    b = (np.exp2(rng.uniform(-20, 40, n))).astype(np.float32)
    _run(lib, a, b)
    # float-valued dividends (the intracellular fluxes)
    _run(lib, rng.standard_normal(n).astype(np.float32).astype(np.float64) * 1e-3, b)


def test_quotients_next_to_rounding_midpoints(lib):
    """a = b * m rounded, m a midpoint of the binary64 grid: the quotient a / b lies
    within an ulp's fraction of m, where a wrong rounding would show."""
    rng = np.random.default_rng(2)
    n = 4_000_000
    b = rng.uniform(1.0, 2.0, n).astype(np.float32).astype(np.float64) * np.exp2(rng.integers(-10, 20, n))
    base = rng.uniform(1.0, 2.0, n)
    ulp = np.spacing(base)
    m = base + ulp / 2                      # a midpoint (not representable itself)
    for shift in (0.0, 1.0, -1.0):
        a = (base + ulp * (0.5 + shift * 2.0 ** -20)) * b
        _run(lib, a, b)
        a = np.nextafter(m * b, np.inf)
        _run(lib, a, b)
        a = np.nextafter(m * b, -np.inf)
        _run(lib, a, b)


def test_special_values(lib):
    tiny = np.array([0.0, -0.0, 5e-324, -5e-324, 1e-300, 2.0 ** -900, 2.0 ** -899, 1e-310, np.inf, -np.inf,
                     np.nan, 1.7976931348623157e308, -1e308, 1.0, -3.0])
    b = np.array([1.0, 1e-6, 3.0, 7.0, 1e6, np.float32(0.1), np.float32(3.4e38), np.float32(1e-38)], np.float32)
    A, B = np.meshgrid(tiny, b)
    _run(lib, A.ravel(), B.ravel())


def _run_prec(lib, a, b, dtype):
    a = np.ascontiguousarray(a, dtype)
    b = np.ascontiguousarray(b, dtype)
    first = C.c_long()
    fn = lib.check_f if dtype == np.float32 else lib.check_d
    bad = fn(a.ctypes.data, b.ctypes.data, a.size, C.byref(first))
    assert bad == 0, "%d mismatches, first a=%r b=%r" % (bad, a[first.value], b[first.value])


@pytest.mark.parametrize("dtype,bits,emax", [(np.float32, 24, 40), (np.float64, 53, 520)])
def test_markstein_division(lib, dtype, bits, emax):
    """div_rn_f / div_rn_d: random operands (inside and outside the guarded range),
    divisors with all-ones and power-of-two significands, and dividends that put the
    quotient next to a rounding midpoint of the operands' precision."""
    rng = np.random.default_rng(3 if dtype == np.float32 else 4)
    n = 3_000_000
    a = rng.standard_normal(n) * np.exp2(rng.integers(-emax, emax, n).astype(np.float64))
    b = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-emax, emax, n).astype(np.float64))
    b[::7] = np.exp2(rng.integers(-30, 30, b[::7].size).astype(np.float64))                       # powers of two
    b[3::7] = (2.0 - 2.0 ** (1 - bits)) * np.exp2(rng.integers(-30, 30, b[3::7].size).astype(np.float64))   # all ones
    _run_prec(lib, a.astype(dtype), b.astype(dtype), dtype)
    # midpoints: m = q + ulp(q) / 2, a = RN(m * b) and its neighbours
    q = rng.uniform(1.0, 2.0, n).astype(dtype)
    bb = (rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-20, 20, n).astype(np.float64))).astype(dtype)
    bb[::5] = (2.0 - 2.0 ** (1 - bits))
    m = q.astype(np.longdouble) + np.spacing(q).astype(np.longdouble) / 2
    a0 = (m * bb.astype(np.longdouble)).astype(dtype)
    for k in (0, 1, -1, 2, -2):
        ak = a0
        for _ in range(abs(k)):
            ak = np.nextafter(ak, np.array(np.inf if k > 0 else -np.inf, dtype))
        _run_prec(lib, ak, bb, dtype)
    tiny = np.array([0.0, -0.0, 1e-30, -1e-30, np.inf, -np.inf, np.nan, 1.0, -3.0, 2.0 ** -33, 2.0 ** 33], dtype)
    div = np.array([1.0, 1e-6, 3.0, 7.0, 1e6, 0.1, 2.0 ** -33, 2.0 ** 33], dtype)
    A, B = np.meshgrid(tiny, div)
    _run_prec(lib, A.ravel(), B.ravel(), dtype)
