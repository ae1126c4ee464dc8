// device_math.cuh -- elementary functions for the device physics.
//
// The reference calls the C library's exp/expf/log/pow.  For results that agree
// bit-for-bit with a CPU evaluation of the same algorithm, the kernels use one
// published method instead of CUDA's math library:
//   exp: Cody & Waite reduction x = k*ln2 + r with ln2 split into a high part with
//        trailing zero bits and a low part, Taylor polynomial of exp(r) by Horner's
//        rule (degree 13 in double, 7 in float), scaling by 2^k from exponent bits;
//   log: x = m*2^e, m in [sqrt(1/2), sqrt(2)), log(m) = 2*atanh((m-1)/(m+1)) by an
//        odd series in Horner form;
//   pow: exact-integer exponents |y| <= 64 by binary powering in double, others as
//        exp(y*log(x)).
// The translation unit is compiled with --fmad=false so each operation rounds as
// written.
#pragma once
#include <cstdint>

// Translation units whose kernels run many different channel models in one launch
// define BNC_MATH_OUTLINE before including this header: the elementary functions are
// then called, not inlined at every call site, which keeps the kernel's instruction
// footprint within the instruction cache.  Results are the same either way.
#ifdef BNC_MATH_OUTLINE
#define BNC_MATH_FN static __device__ __noinline__
#else
#define BNC_MATH_FN static __device__ __forceinline__
#endif

namespace bnc {

static __device__ __forceinline__ double dm_scale2(double p, int k) {
    if (k > 1023)
        return p * __longlong_as_double((long long)(1023 + 1023) << 52) *
               __longlong_as_double((long long)(k - 1023 + 1023) << 52);
    if (k >= -1022) return p * __longlong_as_double((long long)(k + 1023) << 52);
    return (p * __longlong_as_double((long long)(k + 54 + 1023) << 52)) *
           __longlong_as_double((long long)(-54 + 1023) << 52);
}

BNC_MATH_FN double dm_exp(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return __longlong_as_double(0x7FF0000000000000ll);
    if (x < -745.1332191019412) return 0.0;
    const double LOG2E = 1.4426950408889634;
    const double LN2_HI = 6.93147180369123816490e-01;
    const double LN2_LO = 1.90821492927058770002e-10;
    double kd = floor(x * LOG2E + 0.5);
    double r = x - kd * LN2_HI;
    r = r - kd * LN2_LO;
    double p = 1.0 / 6227020800.0;
    p = p * r + 1.0 / 479001600.0;
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
    return dm_scale2(p, (int)kd);
}

static __device__ __forceinline__ float dm_scale2f(float p, int k) {
    if (k > 127)
        return p * __uint_as_float((uint32_t)(127 + 127) << 23) * __uint_as_float((uint32_t)(k - 127 + 127) << 23);
    if (k >= -126) return p * __uint_as_float((uint32_t)(k + 127) << 23);
    return (p * __uint_as_float((uint32_t)(k + 25 + 127) << 23)) * __uint_as_float((uint32_t)(-25 + 127) << 23);
}

BNC_MATH_FN float dm_expf(float x) {
    if (x != x) return x;
    if (x > 88.7228394f) return __uint_as_float(0x7F800000u);
    if (x < -103.972084f) return 0.0f;
    const float LOG2E = 1.44269504f;
    const float LN2_HI = 0.693145751953125f;
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
    return dm_scale2f(p, (int)kf);
}

BNC_MATH_FN double dm_log(double x) {
    if (x != x) return x;
    if (x < 0.0) return __longlong_as_double(0x7FF8000000000000ll);
    if (x == 0.0) return -__longlong_as_double(0x7FF0000000000000ll);
    if (x == __longlong_as_double(0x7FF0000000000000ll)) return x;
    int e = 0;
    if (x < 2.2250738585072014e-308) { x = x * 18014398509481984.0; e = -54; }
    unsigned long long b = (unsigned long long)__double_as_longlong(x);
    e += (int)((b >> 52) & 0x7FF) - 1023;
    double m = __longlong_as_double((long long)((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull));
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

static __device__ __forceinline__ float dm_logf(float x) { return (float)dm_log((double)x); }

BNC_MATH_FN double dm_pow(double x, double y) {
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
    if (x == 0.0) return y > 0.0 ? 0.0 : __longlong_as_double(0x7FF0000000000000ll);
    if (x < 0.0) return __longlong_as_double(0x7FF8000000000000ll);
    return dm_exp(y * dm_log(x));
}

static __device__ __forceinline__ float dm_powf(float x, float y) { return (float)dm_pow((double)x, (double)y); }

}  // namespace bnc
