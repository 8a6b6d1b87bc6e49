/* Common definitions shared by the CUDA kernels and the CPU oracle.
 *
 * Elementary functions.  The solver needs exp, log, log10 and pow in two
 * places: the PRIMORDIAL rate laws (src/odevec_commons.F90:101-384) and the
 * step-size factors of the order selection (src/odevec.F90:561-572).  The
 * CPU library and the CUDA library implement these differently, so the same
 * program gives results that differ in the last bit on the two processors,
 * and one such bit can change an accept/reject decision of the integrator.
 * The functions below are written once, with plain IEEE-754 double
 * operations only, and compiled for both, so the GPU path and the CPU
 * oracle evaluate bit-identical values.  Methods:
 *
 *   ov_exp  - Cody & Waite argument reduction x = k ln2 + r, |r| <= ln2/2,
 *             with ln2 split into a 32-bit head and a tail (W. J. Cody and
 *             W. Waite, "Software Manual for the Elementary Functions",
 *             1980), then the Taylor series of e^r to degree 13 (truncation
 *             error below 5e-18) in Horner form, then scaling by 2^k.
 *   ov_log  - x = 2^e (1+f) with 1+f in [sqrt(1/2), sqrt(2)); with
 *             u = f/(2+f), log(1+f) = 2 atanh(u) = f - u (f - R),
 *             R = sum_{j>=1} 2 u^(2j) / (2j+1), summed to j = 11
 *             (|u| <= 0.1716, truncation below 1e-18).
 *   ov_pow  - exp(y log x) for x > 0, with the usual special cases.
 *
 * Measured against the C library: |error| <= 2 ulp for exp and log over
 * their ranges (tests/test_math.py).  Division and square root are IEEE
 * correctly rounded on both processors and are used directly.
 *
 * Floating-point contraction must be off for both compilers (gcc
 * -ffp-contract=off, nvcc --fmad=false) wherever bit parity is expected. */
#ifndef OV_COMMON_H
#define OV_COMMON_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define OV_HD __host__ __device__
#define OV_INLINE __forceinline__
#else
#define OV_HD
#define OV_INLINE inline
#endif
#define OV_RESTRICT __restrict__

/* A scheduling fence for long straight-line network code: the compiler
   moves no memory access across it, so values loaded before it are not
   kept live (and spilled) for uses long after.  No effect on results. */
#if defined(__CUDA_ARCH__)
#define OV_SCHED() asm volatile("" ::: "memory")
#else
#define OV_SCHED() ((void)0)
#endif

OV_HD static OV_INLINE double ov_bits2d(uint64_t b)
{
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
#endif
}

OV_HD static OV_INLINE uint64_t ov_d2bits(double d)
{
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t b;
    memcpy(&b, &d, sizeof b);
    return b;
#endif
}

/* 2^m for -1022 <= m <= 1023 */
OV_HD static OV_INLINE double ov_pow2i(int m)
{
    return ov_bits2d((uint64_t)(m + 1023) << 52);
}

/* p * 2^k for p in [0.5, 2] and -1080 < k < 1030, one rounding at most */
OV_HD static OV_INLINE double ov_scale2(double p, int k)
{
    if (k > 1000)
        return p * ov_pow2i(1000) * ov_pow2i(k - 1000);
    if (k < -1000)
        return p * ov_pow2i(k + 1000) * ov_pow2i(-1000);
    return p * ov_pow2i(k);
}

#define OV_LN2_HI 0x1.62e42fee00000p-1  /* ln 2 truncated to 32 bits */
#define OV_LN2_LO 0x1.a39ef35793c76p-33 /* ln 2 - OV_LN2_HI, rounded */
#define OV_INV_LN2 0x1.71547652b82fep+0
#define OV_INV_LN10 0x1.bcb7b1526e50ep-2
#define OV_SQRT2 0x1.6a09e667f3bcdp+0

OV_HD static OV_INLINE double ov_exp(double x)
{
    if (x != x)
        return x;
    if (x > 709.782712893384)
        return INFINITY;
    if (x < -745.1332191019412)
        return 0.0;
    /* nearest integer of x/ln2 (|x/ln2| < 2^11, so the shift trick is exact) */
    const double shift = 6755399441055744.0; /* 1.5 * 2^52 */
    double kd = (x * OV_INV_LN2 + shift) - shift;
    int k = (int)kd;
    double r = (x - kd * OV_LN2_HI) - kd * OV_LN2_LO;
    double p = 1.0 / 6227020800.0;            /* 1/13! */
    p = 1.0 / 479001600.0 + r * p;            /* 1/12! */
    p = 1.0 / 39916800.0 + r * p;             /* 1/11! */
    p = 1.0 / 3628800.0 + r * p;
    p = 1.0 / 362880.0 + r * p;
    p = 1.0 / 40320.0 + r * p;
    p = 1.0 / 5040.0 + r * p;
    p = 1.0 / 720.0 + r * p;
    p = 1.0 / 120.0 + r * p;
    p = 1.0 / 24.0 + r * p;
    p = 1.0 / 6.0 + r * p;
    p = 0.5 + r * p;
    p = 1.0 + r * p;
    p = 1.0 + r * p;
    return ov_scale2(p, k);
}

OV_HD static OV_INLINE double ov_log(double x)
{
    if (x != x)
        return x;
    if (x < 0.0)
        return NAN;
    if (x == 0.0)
        return -INFINITY;
    if (x == INFINITY)
        return x;
    int e = 0;
    uint64_t b = ov_d2bits(x);
    if ((b >> 52) == 0) { /* subnormal */
        x *= 18014398509481984.0; /* 2^54 */
        e = -54;
        b = ov_d2bits(x);
    }
    e += (int)(b >> 52) - 1023;
    double m = ov_bits2d((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1,2) */
    if (m > OV_SQRT2) {
        m *= 0.5;
        e += 1;
    }
    double f = m - 1.0; /* exact */
    double u = f / (2.0 + f);
    double z = u * u;
    double R = 2.0 / 23.0;
    R = 2.0 / 21.0 + z * R;
    R = 2.0 / 19.0 + z * R;
    R = 2.0 / 17.0 + z * R;
    R = 2.0 / 15.0 + z * R;
    R = 2.0 / 13.0 + z * R;
    R = 2.0 / 11.0 + z * R;
    R = 2.0 / 9.0 + z * R;
    R = 2.0 / 7.0 + z * R;
    R = 2.0 / 5.0 + z * R;
    R = 2.0 / 3.0 + z * R;
    R = z * R;
    double ed = (double)e;
    double lm = f - u * (f - R);
    return ed * OV_LN2_HI + (lm + ed * OV_LN2_LO);
}

OV_HD static OV_INLINE double ov_log10(double x)
{
    return ov_log(x) * OV_INV_LN10;
}

OV_HD static OV_INLINE double ov_pow(double x, double y)
{
    if (y == 0.0 || x == 1.0)
        return 1.0;
    if (x != x || y != y)
        return x + y;
    if (x == 0.0)
        return y > 0.0 ? 0.0 : INFINITY;
    if (x < 0.0) {
        double yi = floor(y);
        if (yi != y)
            return NAN;
        double a = ov_exp(y * ov_log(-x));
        double h = 0.5 * y;
        return (floor(h) == h) ? a : -a;
    }
    return ov_exp(y * ov_log(x));
}

/* Branch-free restatements of ov_exp, ov_log and ov_pow.  Every input runs
   the main path (special inputs on a harmless stand-in) and the special
   cases are selected afterwards, in the order the branches above test them,
   so each result is bit-identical to the branching function's; factors of
   1.0 stand in for the skipped scalings and are exact.  Without branches the
   compiler can interleave independent calls (the step-size selection needs
   three powers at once, the PRIMORDIAL rate laws about forty). */
OV_HD static OV_INLINE double ov_scale2_sel(double p, int k)
{
    const int a = k > 1000 ? 1000 : (k < -1000 ? k + 1000 : k);
    const int b = k > 1000 ? k - 1000 : (k < -1000 ? -1000 : 0);
    return p * ov_pow2i(a) * ov_pow2i(b);
}

OV_HD static OV_INLINE double ov_exp_sel(double x)
{
    const int ok = x >= -745.1332191019412 && x <= 709.782712893384;
    const double xs = ok ? x : 0.0;
    const double shift = 6755399441055744.0; /* 1.5 * 2^52 */
    double kd = (xs * OV_INV_LN2 + shift) - shift;
    int k = (int)kd;
    double r = (xs - kd * OV_LN2_HI) - kd * OV_LN2_LO;
    double p = 1.0 / 6227020800.0;
    p = 1.0 / 479001600.0 + r * p;
    p = 1.0 / 39916800.0 + r * p;
    p = 1.0 / 3628800.0 + r * p;
    p = 1.0 / 362880.0 + r * p;
    p = 1.0 / 40320.0 + r * p;
    p = 1.0 / 5040.0 + r * p;
    p = 1.0 / 720.0 + r * p;
    p = 1.0 / 120.0 + r * p;
    p = 1.0 / 24.0 + r * p;
    p = 1.0 / 6.0 + r * p;
    p = 0.5 + r * p;
    p = 1.0 + r * p;
    p = 1.0 + r * p;
    double v = ov_scale2_sel(p, k);
    v = x < -745.1332191019412 ? 0.0 : v;
    v = x > 709.782712893384 ? INFINITY : v;
    v = x != x ? x : v;
    return v;
}

OV_HD static OV_INLINE double ov_log_sel(double x)
{
    const int ok = x > 0.0 && x < INFINITY;
    double xs = ok ? x : 1.0;
    uint64_t b = ov_d2bits(xs);
    const int sub = (b >> 52) == 0;
    xs = xs * (sub ? 18014398509481984.0 : 1.0); /* 2^54 */
    int e = sub ? -54 : 0;
    b = ov_d2bits(xs);
    e += (int)(b >> 52) - 1023;
    double m = ov_bits2d((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1,2) */
    const int hi = m > OV_SQRT2;
    m = m * (hi ? 0.5 : 1.0);
    e += hi;
    double f = m - 1.0;
    double u = f / (2.0 + f);
    double z = u * u;
    double R = 2.0 / 23.0;
    R = 2.0 / 21.0 + z * R;
    R = 2.0 / 19.0 + z * R;
    R = 2.0 / 17.0 + z * R;
    R = 2.0 / 15.0 + z * R;
    R = 2.0 / 13.0 + z * R;
    R = 2.0 / 11.0 + z * R;
    R = 2.0 / 9.0 + z * R;
    R = 2.0 / 7.0 + z * R;
    R = 2.0 / 5.0 + z * R;
    R = 2.0 / 3.0 + z * R;
    R = z * R;
    double ed = (double)e;
    double lm = f - u * (f - R);
    double v = ed * OV_LN2_HI + (lm + ed * OV_LN2_LO);
    v = x == INFINITY ? x : v;
    v = x == 0.0 ? -INFINITY : v;
    v = x < 0.0 ? NAN : v;
    v = x != x ? x : v;
    return v;
}

OV_HD static OV_INLINE double ov_log10_sel(double x)
{
    return ov_log_sel(x) * OV_INV_LN10;
}

OV_HD static OV_INLINE double ov_pow_sel(double x, double y)
{
    const double a = ov_exp_sel(y * ov_log_sel(x < 0.0 ? -x : x));
    const double h = 0.5 * y;
    double v = x < 0.0 ? (floor(y) != y ? NAN : (floor(h) == h ? a : -a)) : a;
    v = x == 0.0 ? (y > 0.0 ? 0.0 : INFINITY) : v;
    v = (x != x || y != y) ? x + y : v;
    v = (y == 0.0 || x == 1.0) ? 1.0 : v;
    return v;
}

/* Pivots of the numeric LU.  In FP64 the factorisation and the solves divide
   by each pivot as the reference does (src/odevec.F90:906-969, :864-889).
   An FP32 LU stores each pivot's reciprocal in place once the pivot is final
   (ov_pivot) and multiplies by it (ov_divp): one correctly rounded division
   per pivot instead of one per use, at most one more rounding per product,
   which the modified Newton iteration's FP64 residual absorbs. */
#ifdef __cplusplus
template <class T>
OV_HD static OV_INLINE T ov_pivot(T p) { return p; }
template <>
OV_HD OV_INLINE float ov_pivot<float>(float p) { return 1.0f / p; }
template <class T>
OV_HD static OV_INLINE T ov_divp(T x, T p) { return x / p; }
template <>
OV_HD OV_INLINE float ov_divp<float>(float x, float p) { return x * p; }
#endif

/* Host builds of the CPU oracle with OV_LIBM defined call the C library's
   exp, log, log10 and pow instead, as the reference's Fortran does, so that
   the oracle can be compared bit for bit with runs of the reference's own
   solver module.  Device code never sees this. */
#if defined(OV_LIBM) && !defined(__CUDACC__)
#define ov_exp(x) exp(x)
#define ov_log(x) log(x)
#define ov_log10(x) log10(x)
#define ov_pow(x, y) pow((x), (y))
#define ov_exp_sel(x) exp(x)
#define ov_log_sel(x) log(x)
#define ov_log10_sel(x) log10(x)
#define ov_pow_sel(x, y) pow((x), (y))
#endif

#endif /* OV_COMMON_H */
