/*
 * portable_math.h — exp, log and cbrt that give the same bits on the GPU and on the host.
 *
 * The SP step calls exp and log in the friction factors, the singular head loss and the
 * critical depth of 'q' boundaries.  CUDA's and the host libm's versions differ in the last
 * ulp on some arguments, and wetting/drying flows amplify such differences (a one-ulp change
 * of exp in the CPU oracle moves some 200-step runs by 1e-5..1e-2).  These two functions use
 * only IEEE binary64 +, -, *, / (each rounded once: the CUDA build uses -fmad=false, the host
 * builds -ffp-contract=off without FMA) and exact bit manipulation, so they return identical
 * results on both sides.
 *
 * Methods (textbook, not taken from any library):
 *  - exp: Cody & Waite argument reduction x = k ln2 + r, |r| <= ln2/2, with ln2 split in a
 *    head whose low 21 mantissa bits are zero (k*ln2_hi exact for |k| < 2^21) and a tail;
 *    exp(r) by its Taylor series to degree 13 in Horner form (truncation < 2^-56 relative);
 *    2^k applied through the exponent field, in two factors near the subnormal range.
 *  - log: x = m 2^e with m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(s), s = (m-1)/(m+1),
 *    |s| <= 0.1716, by the odd series 2(s + s^3/3 + ... + s^23/23) (truncation < 2^-56);
 *    log x = e ln2_hi + (e ln2_lo + log m).
 * Accuracy: exp and log within 2 ulp of the true value over the argument ranges the step uses,
 * cbrt within 1 ulp (checked against the host libm by tests/test_portable_math.py and against
 * CUDA's exp/log/cbrt on the GPU).
 *
 * Constants: 1/n! and 1/(2n+1) are the binary64 values nearest the exact rationals; ln2,
 * 1/ln2 and sqrt(2) are the nearest binary64 values of the real numbers.
 */
#ifndef SW2D_PORTABLE_MATH_H
#define SW2D_PORTABLE_MATH_H

#include <stdint.h>

#if defined(__CUDACC__)
#define SW2D_PM_FN __host__ __device__ __forceinline__
#else
#include <string.h>
#define SW2D_PM_FN static inline
#endif

SW2D_PM_FN uint64_t sw2d_pm_bits(double x)
{
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t b;
    memcpy(&b, &x, sizeof b);
    return b;
#endif
}

SW2D_PM_FN double sw2d_pm_from_bits(uint64_t b)
{
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
#endif
}

/* 2^n for n in [-1022, 1023] */
SW2D_PM_FN double sw2d_pm_pow2(int n) { return sw2d_pm_from_bits((uint64_t)(n + 1023) << 52); }

SW2D_PM_FN double sw2d_exp(double x)
{
    const double kInvLn2 = 1.4426950408889634;          /* 1/ln2 */
    const double kLn2Hi = 0.6931471803691238;           /* ln2, low 21 mantissa bits cleared */
    const double kLn2Lo = 1.9082149292705877e-10;       /* ln2 - kLn2Hi */
    const double kShift = 6755399441055744.0;           /* 1.5 * 2^52: rounds to an integer, ties to even */
    if (x != x) return x;                               /* NaN */
    if (x > 709.782712893384) return sw2d_pm_from_bits(0x7ff0000000000000ULL); /* overflow: +inf */
    if (x < -745.1332191019412) return 0.0;             /* below half the smallest subnormal */
    double kd = x * kInvLn2 + kShift;
    kd = kd - kShift;
    int k = (int)kd;
    double r = (x - kd * kLn2Hi) - kd * kLn2Lo;
    double p = 1.6059043836821613e-10;                  /* 1/13! */
    p = p * r + 2.08767569878681e-09;                   /* 1/12! */
    p = p * r + 2.505210838544172e-08;                  /* 1/11! */
    p = p * r + 2.755731922398589e-07;                  /* 1/10! */
    p = p * r + 2.7557319223985893e-06;                 /* 1/9!  */
    p = p * r + 2.48015873015873e-05;                   /* 1/8!  */
    p = p * r + 0.0001984126984126984;                  /* 1/7!  */
    p = p * r + 0.001388888888888889;                   /* 1/6!  */
    p = p * r + 0.008333333333333333;                   /* 1/5!  */
    p = p * r + 0.041666666666666664;                   /* 1/4!  */
    p = p * r + 0.16666666666666666;                    /* 1/3!  */
    p = p * r + 0.5;                                    /* 1/2!  */
    p = p * r + 1.0;                                    /* 1/1!  */
    p = p * r + 1.0;                                    /* 1/0!  */
    if (k > 1023) return (p * 2.0) * sw2d_pm_pow2(k - 1);
    if (k < -1022) return (p * sw2d_pm_pow2(k + 1000)) * sw2d_pm_pow2(-1000);
    return p * sw2d_pm_pow2(k);
}

SW2D_PM_FN double sw2d_log(double x)
{
    const double kLn2Hi = 0.6931471803691238;
    const double kLn2Lo = 1.9082149292705877e-10;
    const double kSqrt2 = 1.4142135623730951;
    if (x != x) return x;                                             /* NaN */
    if (x < 0.0) return sw2d_pm_from_bits(0x7ff8000000000000ULL);     /* NaN */
    if (x == 0.0) return sw2d_pm_from_bits(0xfff0000000000000ULL);    /* -inf */
    uint64_t b = sw2d_pm_bits(x);
    if ((b >> 52) == 0x7ff) return x;                                 /* +inf */
    int e = 0;
    if ((b >> 52) == 0) {                                             /* subnormal: scale by 2^54 */
        x = x * 18014398509481984.0;
        b = sw2d_pm_bits(x);
        e = -54;
    }
    e += (int)((b >> 52) & 0x7ff) - 1023;
    double m = sw2d_pm_from_bits((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1, 2) */
    if (m > kSqrt2) {
        m = m * 0.5;
        e += 1;
    }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double z = s * s;
    double t = 0.043478260869565216;                    /* 1/23 */
    t = t * z + 0.047619047619047616;                   /* 1/21 */
    t = t * z + 0.05263157894736842;                    /* 1/19 */
    t = t * z + 0.058823529411764705;                   /* 1/17 */
    t = t * z + 0.06666666666666667;                    /* 1/15 */
    t = t * z + 0.07692307692307693;                    /* 1/13 */
    t = t * z + 0.09090909090909091;                    /* 1/11 */
    t = t * z + 0.1111111111111111;                     /* 1/9  */
    t = t * z + 0.14285714285714285;                    /* 1/7  */
    t = t * z + 0.2;                                    /* 1/5  */
    t = t * z + 0.3333333333333333;                     /* 1/3  */
    t = t * z;
    double s2 = s + s;
    double lm = s2 + s2 * t;
    double ed = (double)e;
    return ed * kLn2Hi + (ed * kLn2Lo + lm);
}

/*
 * cbrt (the Strickler friction of the differentiated step takes h^(4/3) = h cbrt(h)):
 * |x| = m 2^e with m in [1, 2); e = 3k + j, j in {0, 1, 2}; t = m 2^j in [1, 8) (exact);
 * cbrt|x| = 2^k cbrt(t).  A first guess (3/4 + m/4) c_j, within 2 % of cbrt(t), is refined by
 * five steps of Newton's iteration for y^3 = t, y <- y - (y^3 - t) / (3 y^2) (quadratic
 * convergence: 2e-2, 4e-4, 2e-7, 3e-14, then rounding level); the sign of x is restored.
 * The c_j are rough guesses of 2^(j/3); their error only changes the starting point.
 */
SW2D_PM_FN double sw2d_cbrt(double x)
{
    if (x != x || x == 0.0) return x;                                 /* NaN, +-0 */
    uint64_t b = sw2d_pm_bits(x);
    const uint64_t sign = b & 0x8000000000000000ULL;
    b &= 0x7fffffffffffffffULL;
    if ((b >> 52) == 0x7ff) return x;                                 /* +-inf */
    int e = 0;
    if ((b >> 52) == 0) {                                             /* subnormal: scale by 2^54 */
        b = sw2d_pm_bits(sw2d_pm_from_bits(b) * 18014398509481984.0);
        e = -54;
    }
    e += (int)(b >> 52) - 1023;
    const double m = sw2d_pm_from_bits((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    int k = e / 3, j = e - 3 * k;
    if (j < 0) {
        j += 3;
        k -= 1;
    }
    const double t = (j == 0) ? m : ((j == 1) ? m * 2.0 : m * 4.0);
    double y = (0.75 + 0.25 * m) * ((j == 0) ? 1.0 : ((j == 1) ? 1.26 : 1.5874));
    for (int it = 0; it < 5; it++) y = y - (y * y * y - t) / (3.0 * (y * y));
    const double r = y * sw2d_pm_pow2(k);
    return sw2d_pm_from_bits(sw2d_pm_bits(r) | sign);
}

#endif
