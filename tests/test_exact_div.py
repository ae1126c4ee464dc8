"""bioneuroncore_b200/csrc/exact_div.h returns the IEEE quotient.

The diffusion kernel divides by the same denominators many times per tick
(segment volumes, the phi_e diagonal) and uses div_by with a reciprocal
computed once.  It must return exactly what a / b returns, since the parity
bar is bit equality with the oracle's plain divisions.  The header compiles as
host C++ too; this test builds it with g++ (no contraction, as the oracle is
built) and compares both on random operands of mixed magnitudes and on edge
cases.
"""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r'''
#include "exact_div.h"
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>
static long bad = 0, n = 0;
static void check(double a, double b) {
    double q = bnc::div_by(a, b, bnc::recip_for_div(b)), r = a / b;
    n++;
    bool same = std::memcmp(&q, &r, 8) == 0 || (q != q && r != r);
    if (!same) { if (bad < 5) std::printf("%.17g / %.17g: %.17g vs %.17g\n", a, b, q, r); bad++; }
}
int main() {
    std::mt19937_64 g(7);
    std::uniform_real_distribution<double> u(-1, 1);
    for (int i = 0; i < 3000000; i++) {
        double a = std::ldexp(u(g), (int)(g() % 120) - 60);
        double b = std::ldexp(u(g), (int)(g() % 120) - 60);
        if (i % 3 == 0) b = (double)(float)b;
        if (i % 4 == 0) a = (double)(float)a;
        if (b != 0.0) check(a, b);
    }
    const double inf = std::numeric_limits<double>::infinity(), nan = std::numeric_limits<double>::quiet_NaN();
    const double edge[] = {0.0, -0.0, 1.0, -1.0, 3.0, 0.1, 1e-300, 1e300, 4.9e-324, 2.2250738585072014e-308,
                           inf, -inf, nan, 1.0000000000000002, 0.9999999999999999, 1e-250, 1e250};
    for (double a : edge) for (double b : edge) check(a, b);
    std::printf("%ld %ld\n", n, bad);
    return bad != 0;
}
'''


def test_div_by_equals_ieee_division(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "t"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "bioneuroncore_b200", "csrc"),
                    "-o", str(exe), str(src)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    n, bad = map(int, r.stdout.split()[-2:])
    assert n > 2_900_000 and bad == 0
