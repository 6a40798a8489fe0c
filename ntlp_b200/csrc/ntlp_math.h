/*
 * ntlp_math.h -- elementary functions shared by the host and the device.
 *
 * The droplet step calls exp (saturation vapour pressure and the Koehler
 * humidity term), log/acos/cos/pow (the cubic equilibrium-radius guess) and
 * pow (Reynolds-number corrections, the Exner factor).  The reference takes
 * these from Intel's libm (particles.f90:4305,4347-4365; les.F:10771,10781,
 * 10793).  CUDA's device libm and glibc differ from each other in the last
 * bit on some arguments, and the droplet Newton solve uses a one-sided finite
 * difference with step 1e-12 (particles.f90:4232), which turns one-ulp
 * differences into ~1e-4 relative Jacobian noise and ~1e-12 differences in
 * the converged radius.  To make the FP64 device path reproduce the CPU
 * restatement bit for bit, both sides call these functions, written once:
 *
 *   - every operation is an IEEE double add, multiply, divide, square root
 *     or an explicit fused multiply-add, each correctly rounded on both the
 *     x86-64 host (SSE2, compiled without contraction) and the GPU (compiled
 *     with --fmad=false for the FP64 kernels);
 *   - the algorithms are the classical ones: Cody & Waite argument
 *     reduction (Software Manual for the Elementary Functions, 1980) with
 *     Taylor polynomials whose coefficients are the exact series terms
 *     (1/n!, 2/(2n+1), (2n)!/(4^n (n!)^2 (2n+1))) rounded to double, and the
 *     log(1+f) = 2 atanh(f/(2+f)) identity for the logarithm.
 *
 * Accuracy against glibc is checked by the CPU test suite (exp and log within
 * 1 ulp, pow/acos/cos within a few ulp on the argument ranges used here).
 * This file is plain C99 so that the C oracle can include it as well.
 */
#ifndef NTLP_MATH_H
#define NTLP_MATH_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#ifdef __CUDACC__
#define NTLP_HD static __host__ __device__ __forceinline__
#else
#define NTLP_HD static inline
#endif

/* ---- bit access ------------------------------------------------------- */
NTLP_HD uint64_t ntlp_bits(double x) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    memcpy(&u, &x, sizeof u);
    return u;
#endif
}

NTLP_HD double ntlp_from_bits(uint64_t u) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double x;
    memcpy(&x, &u, sizeof x);
    return x;
#endif
}

NTLP_HD double ntlp_inf(void) { return ntlp_from_bits(0x7ff0000000000000ULL); }
NTLP_HD double ntlp_nan(void) { return ntlp_from_bits(0x7ff8000000000000ULL); }
NTLP_HD int ntlp_isnan(double x) { return !(x == x); }

/* ---- constants (computed to 60 digits and rounded) -------------------- */
#define NTLP_LN2_HI      0x1.62e42fefa39efp-1   /* ln 2 rounded              */
#define NTLP_LN2_LO      0x1.abc9e3b39803fp-56  /* ln 2 - NTLP_LN2_HI        */
#define NTLP_LN2_HI32    0x1.62e42fee00000p-1   /* ln 2 with 21 zero bits    */
#define NTLP_LN2_LO32    0x1.a39ef35793c76p-33  /* ln 2 - NTLP_LN2_HI32      */
#define NTLP_INV_LN2     0x1.71547652b82fep+0
#define NTLP_SQRT2       0x1.6a09e667f3bcdp+0
#define NTLP_PI_HI       0x1.921fb54442d18p+1
#define NTLP_PI_LO       0x1.1a62633145c07p-53
#define NTLP_PIO2_HI     0x1.921fb54442d18p+0
#define NTLP_PIO2_LO     0x1.1a62633145c07p-54
#define NTLP_PIO2_1      0x1.921fb54400000p+0   /* pi/2 in three 33-bit parts */
#define NTLP_PIO2_2      0x1.0b4611a600000p-34
#define NTLP_PIO2_3      0x1.3198a2e000000p-69
#define NTLP_TWO_OVER_PI 0x1.45f306dc9c883p-1
#define NTLP_RND_SHIFT   0x1.8p52               /* round-to-integer shifter  */

/* error-free sum of two doubles: s + t == a + b exactly */
NTLP_HD void ntlp_two_sum(double a, double b, double *s, double *t) {
    double sum = a + b;
    double bb = sum - a;
    *t = (a - (sum - bb)) + (b - bb);
    *s = sum;
}

/* ---- exp -------------------------------------------------------------- */
/* exp(hi + lo) for |lo| much smaller than ulp-scale of hi's reduction.   */
NTLP_HD double ntlp_exp_dd(double hi, double lo) {
    if (ntlp_isnan(hi)) return hi;
    if (hi > 709.782712893384) return ntlp_inf();
    if (hi < -745.2) return 0.0;
    /* k = nearest integer to hi / ln2 */
    double kd = fma(hi, NTLP_INV_LN2, NTLP_RND_SHIFT) - NTLP_RND_SHIFT;
    double r = fma(-kd, NTLP_LN2_HI, hi);
    r = fma(-kd, NTLP_LN2_LO, r);
    r = r + lo;
    /* e^r - 1 = r + r^2 * (1/2! + r/3! + ... + r^11/13!),  |r| <= 0.3466 */
    double q = 0x1.6124613a86d09p-33;            /* 1/13! */
    q = fma(q, r, 0x1.1eed8eff8d898p-29);        /* 1/12! */
    q = fma(q, r, 0x1.ae64567f544e4p-26);        /* 1/11! */
    q = fma(q, r, 0x1.27e4fb7789f5cp-22);        /* 1/10! */
    q = fma(q, r, 0x1.71de3a556c734p-19);        /* 1/9!  */
    q = fma(q, r, 0x1.a01a01a01a01ap-16);        /* 1/8!  */
    q = fma(q, r, 0x1.a01a01a01a01ap-13);        /* 1/7!  */
    q = fma(q, r, 0x1.6c16c16c16c17p-10);        /* 1/6!  */
    q = fma(q, r, 0x1.1111111111111p-7);         /* 1/5!  */
    q = fma(q, r, 0x1.5555555555555p-5);         /* 1/4!  */
    q = fma(q, r, 0x1.5555555555555p-3);         /* 1/3!  */
    q = fma(q, r, 0x1.0000000000000p-1);         /* 1/2!  */
    double em1 = fma(q, r * r, r);
    double m = 1.0 + em1;
    int k = (int)kd;
    if (k >= -1020 && k <= 1022)
        return m * ntlp_from_bits((uint64_t)(int64_t)(k + 1023) << 52);
    if (k > 1022)
        return (m * 2.0) * ntlp_from_bits((uint64_t)(int64_t)(k - 1 + 1023) << 52);
    /* deep underflow: scale into the normal range first, round once at the end */
    return (m * ntlp_from_bits((uint64_t)(int64_t)(k + 200 + 1023) << 52)) * 0x1p-200;
}

NTLP_HD double ntlp_exp(double x) { return ntlp_exp_dd(x, 0.0); }

/* ---- log -------------------------------------------------------------- */
/* Natural log of x > 0 as an unevaluated sum hi + *lo.                    */
NTLP_HD double ntlp_log_dd(double x, double *lo) {
    *lo = 0.0;
    if (ntlp_isnan(x)) return x;
    if (x < 0.0) return ntlp_nan();
    if (x == 0.0) return -ntlp_inf();
    if (x == ntlp_inf()) return x;
    uint64_t u = ntlp_bits(x);
    int e = 0;
    if (u < 0x0010000000000000ULL) {            /* subnormal */
        x *= 0x1p54;
        u = ntlp_bits(x);
        e = -54;
    }
    e += (int)(u >> 52) - 1023;
    double m = ntlp_from_bits((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (m > NTLP_SQRT2) {
        m *= 0.5;
        e += 1;
    }
    double f = m - 1.0;                          /* exact */
    double s = f / (2.0 + f);
    double z = s * s;
    /* R = 2z/3 + 2z^2/5 + ... + 2z^11/23 */
    double R = 0x1.642c8590b2164p-4;             /* 2/23 */
    R = fma(R, z, 0x1.8618618618618p-4);         /* 2/21 */
    R = fma(R, z, 0x1.af286bca1af28p-4);         /* 2/19 */
    R = fma(R, z, 0x1.e1e1e1e1e1e1ep-4);         /* 2/17 */
    R = fma(R, z, 0x1.1111111111111p-3);         /* 2/15 */
    R = fma(R, z, 0x1.3b13b13b13b14p-3);         /* 2/13 */
    R = fma(R, z, 0x1.745d1745d1746p-3);         /* 2/11 */
    R = fma(R, z, 0x1.c71c71c71c71cp-3);         /* 2/9  */
    R = fma(R, z, 0x1.2492492492492p-2);         /* 2/7  */
    R = fma(R, z, 0x1.999999999999ap-2);         /* 2/5  */
    R = fma(R, z, 0x1.5555555555555p-1);         /* 2/3  */
    R = R * z;
    double hfsq = 0.5 * f * f;
    double corr = hfsq - s * (hfsq + R);         /* f - log(1+f) */
    double dk = (double)e;
    double s1, t1;
    ntlp_two_sum(dk * NTLP_LN2_HI32, f, &s1, &t1);   /* both addends exact */
    double low = t1 + (dk * NTLP_LN2_LO32 - corr);
    double hi = s1 + low;
    *lo = low - (hi - s1);
    return hi;
}

NTLP_HD double ntlp_log(double x) {
    double lo;
    double hi = ntlp_log_dd(x, &lo);
    return hi;
}

/* log10(x) = log(x) / ln(10): the double-double log times 1/ln(10) split
 * into two doubles (computed to 60 digits from the definition).           */
#define NTLP_INV_LN10_HI 0x1.bcb7b1526e50ep-2
#define NTLP_INV_LN10_LO 0x1.95355baaafad3p-57
NTLP_HD double ntlp_log10(double x) {
    double lo;
    double hi = ntlp_log_dd(x, &lo);
    if (!(hi == hi) || hi == ntlp_inf() || hi == -ntlp_inf()) return hi;
    double p = hi * NTLP_INV_LN10_HI;
    double e = fma(hi, NTLP_INV_LN10_HI, -p);
    e = fma(hi, NTLP_INV_LN10_LO, e);
    e = fma(lo, NTLP_INV_LN10_HI, e);
    return p + e;
}

/* ---- pow -------------------------------------------------------------- */
NTLP_HD int ntlp_is_int(double y) { return floor(y) == y && fabs(y) < 0x1p53; }

NTLP_HD double ntlp_pow(double x, double y) {
    if (y == 0.0 || x == 1.0) return 1.0;
    if (ntlp_isnan(x) || ntlp_isnan(y)) return x + y;
    double sign = 1.0;
    if (x < 0.0) {
        if (!ntlp_is_int(y)) return ntlp_nan();
        if (fmod(y, 2.0) != 0.0) sign = -1.0;
        x = -x;
    }
    if (x == 0.0) return y > 0.0 ? 0.0 * sign : sign * ntlp_inf();
    if (x == ntlp_inf()) return y > 0.0 ? sign * ntlp_inf() : 0.0 * sign;
    double llo;
    double lhi = ntlp_log_dd(x, &llo);
    double phi = y * lhi;
    double plo = fma(y, lhi, -phi) + y * llo;
    return sign * ntlp_exp_dd(phi, plo);
}

/* ---- acos ------------------------------------------------------------- */
/* asin(x) for |x| <= 0.5 by its Maclaurin series, 26 terms. */
NTLP_HD double ntlp_asin_small(double x) {
    double z = x * x;
    double p = 0x1.1052bc5fa960ap-9;
    p = fma(p, z, 0x1.208d3570ae5a6p-9);
    p = fma(p, z, 0x1.3275586c5f2f0p-9);
    p = fma(p, z, 0x1.464c0950f7d47p-9);
    p = fma(p, z, 0x1.5c5f56efaaaabp-9);
    p = fma(p, z, 0x1.750de64d7d05fp-9);
    p = fma(p, z, 0x1.90cb77f60c7cep-9);
    p = fma(p, z, 0x1.b026f57b13b14p-9);
    p = fma(p, z, 0x1.d3d2a8e0dd67dp-9);
    p = fma(p, z, 0x1.fcaf8fb6db6dbp-9);
    p = fma(p, z, 0x1.15ee9d45d1746p-8);
    p = fma(p, z, 0x1.31683bdef7bdfp-8);
    p = fma(p, z, 0x1.51ba308d3dcb1p-8);
    p = fma(p, z, 0x1.782dda12f684cp-8);
    p = fma(p, z, 0x1.a6863d70a3d71p-8);
    p = fma(p, z, 0x1.df3bd37a6f4dfp-8);
    p = fma(p, z, 0x1.12ef3cf3cf3cfp-7);
    p = fma(p, z, 0x1.3fde50d79435ep-7);
    p = fma(p, z, 0x1.7a87878787878p-7);
    p = fma(p, z, 0x1.c99999999999ap-7);
    p = fma(p, z, 0x1.1c4ec4ec4ec4fp-6);
    p = fma(p, z, 0x1.6e8ba2e8ba2e9p-6);
    p = fma(p, z, 0x1.f1c71c71c71c7p-6);
    p = fma(p, z, 0x1.6db6db6db6db7p-5);
    p = fma(p, z, 0x1.3333333333333p-4);
    p = fma(p, z, 0x1.5555555555555p-3);
    return fma(x * z, p, x);
}

NTLP_HD double ntlp_acos(double x) {
    if (ntlp_isnan(x) || x > 1.0 || x < -1.0) return ntlp_nan();
    if (fabs(x) <= 0.5)
        return NTLP_PIO2_HI - (ntlp_asin_small(x) - NTLP_PIO2_LO);
    if (x > 0.0) {
        double s = sqrt((1.0 - x) * 0.5);
        return 2.0 * ntlp_asin_small(s);
    }
    double s = sqrt((1.0 + x) * 0.5);
    return NTLP_PI_HI - (2.0 * ntlp_asin_small(s) - NTLP_PI_LO);
}

/* ---- cos -------------------------------------------------------------- */
/* cos(r), sin(r) for |r| <= pi/4 by their Maclaurin series. */
NTLP_HD double ntlp_cos_small(double r) {
    double z = r * r;
    double c = 0x1.e542ba4020225p-62;            /*  1/20! */
    c = fma(c, z, -0x1.6827863b97d97p-53);       /* -1/18! */
    c = fma(c, z, 0x1.ae7f3e733b81fp-45);        /*  1/16! */
    c = fma(c, z, -0x1.93974a8c07c9dp-37);       /* -1/14! */
    c = fma(c, z, 0x1.1eed8eff8d898p-29);        /*  1/12! */
    c = fma(c, z, -0x1.27e4fb7789f5cp-22);       /* -1/10! */
    c = fma(c, z, 0x1.a01a01a01a01ap-16);        /*  1/8!  */
    c = fma(c, z, -0x1.6c16c16c16c17p-10);       /* -1/6!  */
    c = fma(c, z, 0x1.5555555555555p-5);         /*  1/4!  */
    double hz = 0.5 * z;
    double w = 1.0 - hz;
    return w + (((1.0 - w) - hz) + (z * z) * c);
}

NTLP_HD double ntlp_sin_small(double r) {
    double z = r * r;
    double s = 0x1.71b8ef6dcf572p-66;            /*  1/21! */
    s = fma(s, z, -0x1.2f49b46814157p-57);       /* -1/19! */
    s = fma(s, z, 0x1.952c77030ad4ap-49);        /*  1/17! */
    s = fma(s, z, -0x1.ae7f3e733b81fp-41);       /* -1/15! */
    s = fma(s, z, 0x1.6124613a86d09p-33);        /*  1/13! */
    s = fma(s, z, -0x1.ae64567f544e4p-26);       /* -1/11! */
    s = fma(s, z, 0x1.71de3a556c734p-19);        /*  1/9!  */
    s = fma(s, z, -0x1.a01a01a01a01ap-13);       /* -1/7!  */
    s = fma(s, z, 0x1.1111111111111p-7);         /*  1/5!  */
    s = fma(s, z, -0x1.5555555555555p-3);        /* -1/3!  */
    return fma(r * z, s, r);
}

/* cos(x); the three-part reduction is accurate for |x| below ~1e5. */
NTLP_HD double ntlp_cos(double x) {
    if (ntlp_isnan(x) || fabs(x) == ntlp_inf()) return ntlp_nan();
    double a = fabs(x);
    if (a < 0x1p-27) return 1.0;
    double nd = fma(a, NTLP_TWO_OVER_PI, NTLP_RND_SHIFT) - NTLP_RND_SHIFT;
    double r = fma(-nd, NTLP_PIO2_1, a);
    r = fma(-nd, NTLP_PIO2_2, r);
    r = fma(-nd, NTLP_PIO2_3, r);
    int n = ((int)nd) & 3;
    if (n == 0) return ntlp_cos_small(r);
    if (n == 1) return -ntlp_sin_small(r);
    if (n == 2) return -ntlp_cos_small(r);
    return ntlp_sin_small(r);
}

#endif /* NTLP_MATH_H */
