/*
 * bo_math.h -- elementary functions for the CPU oracle (test infrastructure).
 *
 * The reference calls the C library's exp/expf/log/pow.  The oracle and the CUDA
 * kernels must evaluate these identically on both sides, so both use this same
 * published method instead of their platform's library:
 *
 *   exp: Cody & Waite argument reduction x = k*ln2 + r (ln2 split into a high
 *        part with trailing zero bits and a low part), Taylor polynomial of
 *        exp(r) by Horner's rule (degree 13 in double, 7 in float), scaling by
 *        2^k built from the exponent bits.
 *   log: x = m*2^e with m in [sqrt(1/2), sqrt(2)); log(m) = 2*atanh(s),
 *        s = (m-1)/(m+1), odd series in s by Horner's rule.
 *   pow: exact-integer exponents |y| <= 64 by binary powering in double; other
 *        exponents as exp(y*log(x)).
 *
 * Compiled without floating-point contraction (-ffp-contract=off) so every
 * operation rounds exactly as written.  Accuracy against the C library is
 * checked in tests/test_oracle_math.py.
 */
#ifndef BO_MATH_H
#define BO_MATH_H
#include <stdint.h>
#include <string.h>
#include <math.h>

static inline double bo_u2d(uint64_t u) { double d; memcpy(&d, &u, 8); return d; }
static inline uint64_t bo_d2u(double d) { uint64_t u; memcpy(&u, &d, 8); return u; }
static inline float bo_u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t bo_f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* 2^k as a double for k in [-1074, 1023] (two factors below the normal range). */
static inline double bo_scale2(double p, int k) {
    if (k > 1023) return p * bo_u2d((uint64_t)(1023 + 1023) << 52) * bo_u2d((uint64_t)(k - 1023 + 1023) << 52);
    if (k >= -1022) return p * bo_u2d((uint64_t)(k + 1023) << 52);
    return (p * bo_u2d((uint64_t)(k + 54 + 1023) << 52)) * bo_u2d((uint64_t)(-54 + 1023) << 52);
}

static inline double bo_exp(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return bo_u2d(0x7FF0000000000000ull);
    if (x < -745.1332191019412) return 0.0;
    const double LOG2E = 1.4426950408889634;
    const double LN2_HI = 6.93147180369123816490e-01;
    const double LN2_LO = 1.90821492927058770002e-10;
    double kd = floor(x * LOG2E + 0.5);
    double r = x - kd * LN2_HI;
    r = r - kd * LN2_LO;
    double p = 1.0 / 6227020800.0;         /* 1/13! */
    p = p * r + 1.0 / 479001600.0;         /* 1/12! */
    p = p * r + 1.0 / 39916800.0;
    p = p * r + 1.0 / 3628800.0;
    p = p * r + 1.0 / 362880.0;
    p = p * r + 1.0 / 40320.0;
    p = p * r + 1.0 / 5040.0;
    p = p * r + 1.0 / 720.0;
    p = p * r + 1.0 / 120.0;
    p = p * r + 1.0 / 24.0;
    p = p * r + 1.0 / 6.0;
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    return bo_scale2(p, (int)kd);
}

static inline float bo_scale2f(float p, int k) {
    if (k > 127) return p * bo_u2f((uint32_t)(127 + 127) << 23) * bo_u2f((uint32_t)(k - 127 + 127) << 23);
    if (k >= -126) return p * bo_u2f((uint32_t)(k + 127) << 23);
    return (p * bo_u2f((uint32_t)(k + 25 + 127) << 23)) * bo_u2f((uint32_t)(-25 + 127) << 23);
}

static inline float bo_expf(float x) {
    if (x != x) return x;
    if (x > 88.7228394f) return bo_u2f(0x7F800000u);
    if (x < -103.972084f) return 0.0f;
    const float LOG2E = 1.44269504f;
    const float LN2_HI = 0.693145751953125f;     /* 0x3F317200 */
    const float LN2_LO = 1.42860676e-06f;
    float kf = floorf(x * LOG2E + 0.5f);
    float r = x - kf * LN2_HI;
    r = r - kf * LN2_LO;
    float p = 1.0f / 5040.0f;
    p = p * r + 1.0f / 720.0f;
    p = p * r + 1.0f / 120.0f;
    p = p * r + 1.0f / 24.0f;
    p = p * r + 1.0f / 6.0f;
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    return bo_scale2f(p, (int)kf);
}

static inline double bo_log(double x) {
    if (x != x) return x;
    if (x < 0.0) return bo_u2d(0x7FF8000000000000ull);
    if (x == 0.0) return -bo_u2d(0x7FF0000000000000ull);
    if (x == bo_u2d(0x7FF0000000000000ull)) return x;
    int e = 0;
    if (x < 2.2250738585072014e-308) { x = x * 18014398509481984.0; e = -54; }  /* 2^54 */
    uint64_t b = bo_d2u(x);
    e += (int)((b >> 52) & 0x7FF) - 1023;
    double m = bo_u2d((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
    if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double s2 = s * s;
    double t = 1.0 / 23.0;
    t = t * s2 + 1.0 / 21.0;
    t = t * s2 + 1.0 / 19.0;
    t = t * s2 + 1.0 / 17.0;
    t = t * s2 + 1.0 / 15.0;
    t = t * s2 + 1.0 / 13.0;
    t = t * s2 + 1.0 / 11.0;
    t = t * s2 + 1.0 / 9.0;
    t = t * s2 + 1.0 / 7.0;
    t = t * s2 + 1.0 / 5.0;
    t = t * s2 + 1.0 / 3.0;
    t = t * s2 + 1.0;
    double lm = 2.0 * s * t;
    double ed = (double)e;
    const double LN2_HI = 6.93147180369123816490e-01;
    const double LN2_LO = 1.90821492927058770002e-10;
    return ed * LN2_HI + (ed * LN2_LO + lm);
}

static inline float bo_logf(float x) { return (float)bo_log((double)x); }

static inline double bo_pow(double x, double y) {
    if (y == 0.0) return 1.0;
    if (x != x || y != y) return x + y;
    double yi = floor(y);
    if (yi == y && y >= -64.0 && y <= 64.0) {
        int n = (int)y;
        int neg = n < 0;
        unsigned int u = (unsigned int)(neg ? -n : n);
        double base = x, acc = 1.0;
        while (u) {
            if (u & 1u) acc = acc * base;
            u >>= 1;
            if (u) base = base * base;
        }
        return neg ? 1.0 / acc : acc;
    }
    if (x == 0.0) return y > 0.0 ? 0.0 : bo_u2d(0x7FF0000000000000ull);
    if (x < 0.0) return bo_u2d(0x7FF8000000000000ull);
    return bo_exp(y * bo_log(x));
}

static inline float bo_powf(float x, float y) { return (float)bo_pow((double)x, (double)y); }

#ifdef BO_LIBM
/* The FP64-state build (-DBO_FP64 -DBO_LIBM) calls the C library's functions,
 * exactly as the reference's compiled tick does, so that it can be compared with
 * the reference bit for bit. */
#define bo_exp(x) exp(x)
#define bo_expf(x) expf(x)
#define bo_log(x) log(x)
#define bo_logf(x) logf(x)
#define bo_pow(x, y) pow(x, y)
#define bo_powf(x, y) powf(x, y)
#endif

#endif
