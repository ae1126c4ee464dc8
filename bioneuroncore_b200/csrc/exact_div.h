// exact_div.h -- a / b, correctly rounded, for a denominator b reused many times.
//
// With y = RN(1/b) computed once, q0 = RN(a*y) is within a couple of ulps of a/b;
// one correction q1 = RN(q0 + RN(a - q0*b) * y), the remainder taken exactly by a
// fused multiply-add, gives the correctly rounded quotient in all but rare cases
// (P. Markstein, "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990; J.-M. Muller et al., Handbook of
// Floating-Point Arithmetic, 2nd ed., 2018, sec. 4.7).  The result is then checked
// exactly: the remainder r = a - q1*b (exact by fma for a quotient this close)
// must satisfy |r| < ulp(q1)/2 * |b| -- the exact quotient of two binary64 numbers
// is never halfway between two binary64 numbers, so the bound is strict and
// certifies RN(a/b).  Whenever the check cannot certify the result (zero,
// subnormal or non-finite operands and results, a power-of-two quotient whose
// rounding interval is asymmetric, or a failed bound), the IEEE division a / b
// is returned instead.  Either way the value is the IEEE quotient.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define BNC_HD __host__ __device__ __forceinline__
#else
#define BNC_HD inline
#endif

namespace bnc {

BNC_HD uint64_t ed_bits(double x) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return u;
#endif
}

BNC_HD double ed_from_bits(uint64_t u) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double x;
    std::memcpy(&x, &u, 8);
    return x;
#endif
}

BNC_HD double ed_fma(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return fma(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

// Reciprocal to pass as `y` below (one IEEE division per denominator).
BNC_HD double recip_for_div(double b) { return 1.0 / b; }

// a / b, given y = recip_for_div(b).
BNC_HD double div_by(double a, double b, double y) {
    const double aa = a < 0.0 ? -a : a, ab = b < 0.0 ? -b : b;
    // operands well inside the normal range: no step below can underflow or overflow
    if (aa >= 1.0e-250 && aa <= 1.0e250 && ab >= 1.0e-250 && ab <= 1.0e250) {
        const double q0 = a * y;
        const double q1 = ed_fma(ed_fma(-q0, b, a), y, q0);
        const uint64_t qb = ed_bits(q1);
        const uint32_t e = (uint32_t)((qb >> 52) & 0x7FFu);
        // a normal quotient that is not a power of two (symmetric rounding interval)
        if (e > 54u && e < 0x7FFu && (qb & 0x000FFFFFFFFFFFFFull) != 0) {
            const double r = ed_fma(-q1, b, a);                                  // exact remainder
            const double half_ulp = ed_from_bits((uint64_t)(e - 53u) << 52);   // ulp(q1) / 2
            const double bound = half_ulp * ab;                                 // exact: power-of-two scaling
            const double ar = r < 0.0 ? -r : r;
            if (ar < bound) return q1;
        }
    }
    return a / b;
}

}  // namespace bnc
