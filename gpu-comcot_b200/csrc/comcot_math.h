/*
 * Deterministic elementary functions shared by the CUDA kernels and the CPU
 * restatement, so that a float exp() or pow() rounds identically on both.
 *
 * The reference evaluates EXP(-REF) in WAVE_BREAKING (moment.f90:1318) and
 * DF**(2.3333333) in the Manning friction terms (moment.f90:460,633,234,260)
 * with the compiler's libm.  Two different libm implementations can differ by
 * one ulp, which in a wet/dry stencil can flip a mask.  Both sides therefore
 * call these functions instead.
 *
 * Method (no table, no vendor code):
 *   exp(x): Cody & Waite argument reduction x = k*ln2 + r with ln2 split in a
 *           high part exact in 32 bits and a low correction (W. J. Cody and
 *           W. Waite, "Software Manual for the Elementary Functions", 1980),
 *           then the Taylor series of e^r to degree 14 (|r| <= 0.35, truncation
 *           < 1e-18), evaluated by Horner in double, scaled by 2^k built from
 *           the exponent bits, rounded once to float.
 *   log(x): x = m * 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s),
 *           s = (m-1)/(m+1), |s| < 0.172, odd series to s^25 (error < 1e-19).
 *   pow(x,y) = exp(y * log(x)) for x > 0, all in double, rounded once.
 * Every operation is a separately rounded IEEE double add/mul/div; on the
 * device the _rn intrinsics forbid contraction into FMA, on the host the
 * library is compiled with -ffp-contract=off.  The double result carries
 * ~50 correct bits, so the float rounding agrees with a correctly rounded
 * libm except within 2^-26 of a rounding midpoint.
 */
#ifndef COMCOT_MATH_H
#define COMCOT_MATH_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define CCM_FN static __host__ __device__ __forceinline__
#else
#define CCM_FN static inline
#endif

#if defined(__CUDA_ARCH__)
#define CCM_DADD(a, b) __dadd_rn((a), (b))
#define CCM_DSUB(a, b) __dsub_rn((a), (b))
#define CCM_DMUL(a, b) __dmul_rn((a), (b))
#define CCM_DDIV(a, b) __ddiv_rn((a), (b))
#else
#define CCM_DADD(a, b) ((a) + (b))
#define CCM_DSUB(a, b) ((a) - (b))
#define CCM_DMUL(a, b) ((a) * (b))
#define CCM_DDIV(a, b) ((a) / (b))
#endif

CCM_FN float ccm_inff(void) {
#if defined(__CUDA_ARCH__)
    return __int_as_float(0x7f800000);
#else
    uint32_t u = 0x7f800000u;
    float f;
    memcpy(&f, &u, sizeof f);
    return f;
#endif
}

CCM_FN double ccm_bits_to_double(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double d;
    memcpy(&d, &u, sizeof d);
    return d;
#endif
}

CCM_FN uint64_t ccm_double_to_bits(double d) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t u;
    memcpy(&u, &d, sizeof u);
    return u;
#endif
}

/* e^x in double for |x| < 708, reduced by Cody-Waite. */
CCM_FN double ccm_exp_d(double x) {
    const double INV_LN2 = 1.4426950408889634;
    const double LN2_HI = 0.693145751953125;          /* 22 significant bits */
    const double LN2_LO = 1.4286068203094172321e-6;   /* ln2 - LN2_HI        */
    double t = CCM_DADD(CCM_DMUL(x, INV_LN2), 0.5);
    double kf = t >= 0.0 ? (double)(int64_t)t : -(double)(int64_t)(-t);
    if (kf > t) kf = CCM_DSUB(kf, 1.0);               /* floor */
    int k = (int)kf;
    double r = CCM_DSUB(CCM_DSUB(x, CCM_DMUL(kf, LN2_HI)), CCM_DMUL(kf, LN2_LO));
    /* Horner evaluation of sum_{n=0}^{14} r^n / n! */
    double p = 1.0 / 87178291200.0;                   /* 1/14! */
    p = CCM_DADD(CCM_DMUL(p, r), 1.0 / 6227020800.0);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0 / 479001600.0);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0 / 39916800.0);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0 / 3628800.0);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0 / 362880.0);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0 / 40320.0);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0 / 5040.0);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0 / 720.0);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0 / 120.0);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0 / 24.0);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0 / 6.0);
    p = CCM_DADD(CCM_DMUL(p, r), 0.5);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0);
    p = CCM_DADD(CCM_DMUL(p, r), 1.0);
    /* 2^k for k in [-1022, 1023]; callers keep k inside that range */
    double twok = ccm_bits_to_double((uint64_t)(int64_t)(k + 1023) << 52);
    return CCM_DMUL(p, twok);
}

/* natural log in double for finite x > 0 (normal or subnormal). */
CCM_FN double ccm_log_d(double x) {
    const double LN2 = 0.69314718055994530942;
    const double SQRT2 = 1.4142135623730951;
    int e = 0;
    uint64_t u = ccm_double_to_bits(x);
    int ex = (int)((u >> 52) & 0x7ff);
    if (ex == 0) {                                      /* subnormal: rescale */
        x = CCM_DMUL(x, 18014398509481984.0);          /* 2^54 */
        u = ccm_double_to_bits(x);
        ex = (int)((u >> 52) & 0x7ff);
        e = -54;
    }
    e += ex - 1023;
    double m = ccm_bits_to_double((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (m > SQRT2) { m = CCM_DMUL(m, 0.5); e += 1; }
    double s = CCM_DDIV(CCM_DSUB(m, 1.0), CCM_DADD(m, 1.0));
    double s2 = CCM_DMUL(s, s);
    double q = 1.0 / 25.0;
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0 / 23.0);
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0 / 21.0);
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0 / 19.0);
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0 / 17.0);
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0 / 15.0);
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0 / 13.0);
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0 / 11.0);
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0 / 9.0);
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0 / 7.0);
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0 / 5.0);
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0 / 3.0);
    q = CCM_DADD(CCM_DMUL(q, s2), 1.0);
    double logm = CCM_DMUL(CCM_DMUL(2.0, s), q);
    return CCM_DADD(CCM_DMUL((double)e, LN2), logm);
}

/* float e^x, rounded once from the double evaluation. */
CCM_FN float cc_expf(float xf) {
    double x = (double)xf;
    if (x != x) return xf;                     /* NaN propagates            */
    if (x > 88.8) return ccm_inff();          /* overflows to +inf in float */
    if (x < -104.0) return 0.0f;                /* below half the least subnormal */
    return (float)ccm_exp_d(x);
}

/* float x**y for x >= 0 and finite y, as used by the friction terms. */
CCM_FN float cc_powf(float xf, float yf) {
    double x = (double)xf, y = (double)yf;
    if (x != x || y != y) return xf + yf;
    if (yf == 0.0f) return 1.0f;
    if (xf == 0.0f) return yf > 0.0f ? 0.0f : ccm_inff();
    if (xf < 0.0f) return (xf - xf) / (xf - xf);    /* NaN, as Fortran REAL**REAL */
    if (x > 3.4e38) return yf > 0.0f ? ccm_inff() : 0.0f;
    double l = CCM_DMUL(y, ccm_log_d(x));
    if (l > 88.8) return ccm_inff();
    if (l < -104.0) return 0.0f;
    return (float)ccm_exp_d(l);
}

#endif
