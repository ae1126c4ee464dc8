"""The elementary functions shared by the oracle and the kernels, the release RNG,
and the reference's ionic known-answer tests, all on the CPU.

The kernels compile the same exp/log/pow (bioneuroncore_b200/csrc/device_math.cuh
restates oracle/bo_math.h operation by operation), so these bounds hold on the
device too; the GPU parity tests check the two agree bit for bit.
"""
import math

import numpy as np
import pytest

from oracle.oracle import oracle_lib


def _ulps(got, want, dtype):
    got = np.asarray(got, dtype).astype(np.float64)
    want = np.asarray(want, dtype)
    return np.abs(got - want.astype(np.float64)) / np.spacing(np.abs(want)).astype(np.float64)


def test_exp_double_within_one_ulp():
    lib = oracle_lib()
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-700, 700, 4000), rng.uniform(-5, 5, 4000), [0.0, 1.0, -1.0, 1e-300]])
    assert _ulps([lib.bo_exp_d(v) for v in x], np.exp(x), np.float64).max() <= 1.0
    assert lib.bo_exp_d(800.0) == math.inf and lib.bo_exp_d(-800.0) == 0.0
    assert math.isnan(lib.bo_exp_d(math.nan))


def test_expf_within_one_ulp():
    lib = oracle_lib()
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.uniform(-87, 88, 4000), rng.uniform(-5, 5, 4000)]).astype(np.float32)
    want = np.exp(x.astype(np.float64)).astype(np.float32)
    assert _ulps([lib.bo_expf_f(float(v)) for v in x], want, np.float32).max() <= 1.0


def test_log_within_two_ulp():
    lib = oracle_lib()
    rng = np.random.default_rng(3)
    y = np.exp(rng.uniform(-700, 700, 4000))
    assert _ulps([lib.bo_log_d(v) for v in y], np.log(y), np.float64).max() <= 2.0
    assert lib.bo_log_d(0.0) == -math.inf and math.isnan(lib.bo_log_d(-1.0))
    assert lib.bo_log_d(1.0) == 0.0


def test_pow_integer_exponents_exact_products_and_general_bound():
    lib = oracle_lib()
    # integer exponents by binary powering: exact for small integers
    assert lib.bo_pow_d(3.0, 4.0) == 81.0
    assert lib.bo_pow_d(2.0, -3.0) == 0.125
    assert lib.bo_pow_d(7.5, 0.0) == 1.0
    rng = np.random.default_rng(4)
    xs = rng.uniform(0.01, 100, 2000)
    ys = rng.uniform(-4, 4, 2000)
    # exp(y*log x): the rounding of y*log(x) is amplified by |y log x|; 32 ulp bounds it here
    assert _ulps([lib.bo_pow_d(a, b) for a, b in zip(xs, ys)], xs ** ys, np.float64).max() <= 32.0


def _xorshift32_unit(seed):
    # simulation_host.cpp:150-156 of the reference
    x = seed & 0xFFFFFFFF
    x ^= (x << 13) & 0xFFFFFFFF
    x ^= x >> 17
    x ^= (x << 5) & 0xFFFFFFFF
    return np.float32(np.float32(x & 0x7FFFFFFF) / np.float32(0x7FFFFFFF))


def test_release_rng_matches_the_reference_xorshift32():
    lib = oracle_lib()
    rng = np.random.default_rng(5)
    for s in list(rng.integers(0, 2 ** 32, 2000, dtype=np.uint64)) + [0, 1, 0xFFFFFFFF, 0x80000000]:
        assert np.float32(lib.bo_xorshift_f(int(s))) == _xorshift32_unit(int(s))


def test_seed_bits_follow_the_x86_double_to_uint32_conversion():
    """(uint32_t)(V_m * 1000.0f) with V_m double: truncation toward zero to int64,
    then the low 32 bits (how g++ on x86-64 compiles simulation_host.cpp:438-439)."""
    lib = oracle_lib()
    for v in (-65.0, -64.99, -40.0, 0.0, 0.0004, 12.3456, -119.9999, 149.5):
        want = int(math.trunc(float(np.float32(v)) * 1000.0)) & 0xFFFFFFFF
        assert lib.bo_seed_bits(float(np.float32(v))) == want
    assert lib.bo_seed_bits(-65.0) == 4294902296


# ---- reference known-answer tests, restated ----

def _textbook_flux(V_mV, c_in, c_out, z, F, R, T):
    # tests/test_ghk_reference.cpp:14-27 of the reference
    V = V_mV * 0.001
    Vn = z * F * V / (R * T)
    e = math.exp(-Vn)
    k = z * z * F * F / (R * T)
    if abs(Vn) < 1e-6:
        return z * F * (c_in - c_out)
    if Vn > 20.0:
        return k * V * c_in
    if Vn < -20.0:
        return k * V * c_out
    return k * V * (c_in - c_out * e) / (1.0 - e)


@pytest.mark.parametrize("V", [-100.0, -70.0, -40.0, 0.0, 40.0])
def test_ghk_flux_terms_match_textbook(V):
    """tests/test_ghk_reference.cpp:29-75: K+, Na+ (monovalent), Ca2+ (divalent),
    Cl- (anion, c_in and c_out swapped) to relative 1e-4."""
    lib = oracle_lib()
    F, R, T = lib.bo_const(0), lib.bo_const(1), lib.bo_const(2)
    cases = [(lib.bo_ghk_mono_d, 140e-3, 5e-3, 1.0, False), (lib.bo_ghk_mono_d, 12e-3, 140e-3, 1.0, False),
             (lib.bo_ghk_div_d, 0.0001e-3, 1.2e-3, 2.0, False), (lib.bo_ghk_anion_d, 5e-3, 130e-3, 1.0, True)]
    for fn, ci, co, z, anion in cases:
        got = fn(V, ci, co)
        want = _textbook_flux(V, co, ci, z, F, R, T) if anion else _textbook_flux(V, ci, co, z, F, R, T)
        assert got == pytest.approx(want, rel=1e-4, abs=1e-12)


def test_ghk_flux_signs():
    """tests/test_ghk_reference.cpp:77-83: at -70 mV K+ flows out, Na+ in."""
    lib = oracle_lib()
    assert lib.bo_ghk_mono_d(-70.0, 140e-3, 5e-3) > 0.0
    assert lib.bo_ghk_mono_d(-70.0, 12e-3, 140e-3) < 0.0


def test_nernst_known_answers():
    """tests/test_reference_ionics.cpp:22-31."""
    lib = oracle_lib()
    F, R, T = lib.bo_const(0), np.float32(lib.bo_const(1)), np.float32(lib.bo_const(2))
    ref = float(R * T) / (1.0 * F) * math.log(0.005 / 0.140) * 1000.0
    assert lib.bo_nernst_f(0.140, 0.005, 1.0) == pytest.approx(ref, rel=1e-4)
    assert lib.bo_nernst_f(0.140, 0.005, 1.0) == pytest.approx(-89.0, abs=0.5)
    assert lib.bo_nernst_f(0.012, 0.140, 1.0) == pytest.approx(65.7, abs=0.5)
    assert lib.bo_nernst_f(0.0001, 0.0012, 2.0) == pytest.approx(33.2, abs=0.5)
    assert lib.bo_nernst_f(0.005, 0.130, -1.0) == pytest.approx(-87.1, abs=0.5)
