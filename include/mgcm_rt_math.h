/*
 * mgcm_rt_math.h -- the FP64 exponential used by the radiation path.
 *
 * The reference two-stream IR solver is ill-conditioned in optically thin
 * layers: EP = EXP(LAMDA*DTAU) enters the tridiagonal rows through EP-EM
 * (code/gfluxi.f90:113-123, code/dsolver.f90:74-80), so a one-ulp change of
 * EXP moves IR fluxes by up to ~1e-6 relative (visible: ~1e-13).  Results of
 * the reference therefore depend on the libm it links.  To make the FP64 path
 * reproducible to 1e-12 across host and device, both the CPU oracle and the
 * FP64 kernels evaluate every per-column exponential with this one routine:
 * the same IEEE operations in the same order, no fused multiply-add, so host
 * and device results are bit-identical.
 *
 * Method: P. T. P. Tang, "Table-driven implementation of the exponential
 * function in IEEE floating-point arithmetic", ACM TOMS 15(2), 1989:
 *   x = (32 m + j) ln2/32 + r,  |r| <= ln2/64,
 *   exp(x) = 2^m (S_j + S_j p(r)),  S_j = 2^(j/32) held as lead + trail,
 *   p(r) = r + r^2/2! + ... + r^6/6!  (Taylor; truncation < 2^-60 on |r|).
 * The table entries are 2^(j/32) rounded to double (lead) and the rounded
 * remainder (trail), generated with 60-digit decimal arithmetic.  Accuracy is
 * below one ulp; it is not a copy of any libm's algorithm or constants.
 */
#ifndef MGCM_RT_MATH_H
#define MGCM_RT_MATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define MGCM_RT_HD __host__ __device__ __forceinline__
#else
#define MGCM_RT_HD static inline
#endif

#define MGCM_RT_EXP_TABLE                                                                     \
    {0x1.0000000000000p+0, 0x1.059b0d3158574p+0, 0x1.0b5586cf9890fp+0, 0x1.11301d0125b51p+0, \
     0x1.172b83c7d517bp+0, 0x1.1d4873168b9aap+0, 0x1.2387a6e756238p+0, 0x1.29e9df51fdee1p+0, \
     0x1.306fe0a31b715p+0, 0x1.371a7373aa9cbp+0, 0x1.3dea64c123422p+0, 0x1.44e086061892dp+0, \
     0x1.4bfdad5362a27p+0, 0x1.5342b569d4f82p+0, 0x1.5ab07dd485429p+0, 0x1.6247eb03a5585p+0, \
     0x1.6a09e667f3bcdp+0, 0x1.71f75e8ec5f74p+0, 0x1.7a11473eb0187p+0, 0x1.82589994cce13p+0, \
     0x1.8ace5422aa0dbp+0, 0x1.93737b0cdc5e5p+0, 0x1.9c49182a3f090p+0, 0x1.a5503b23e255dp+0, \
     0x1.ae89f995ad3adp+0, 0x1.b7f76f2fb5e47p+0, 0x1.c199bdd85529cp+0, 0x1.cb720dcef9069p+0, \
     0x1.d5818dcfba487p+0, 0x1.dfc97337b9b5fp+0, 0x1.ea4afa2a490dap+0, 0x1.f50765b6e4540p+0, \
     0x0.0p+0,              0x1.d73e2a475b465p-55,  0x1.8a62e4adc610bp-54,  -0x1.6c51039449b3ap-54, \
     -0x1.19041b9d78a76p-55, 0x1.e016e00a2643cp-54,  0x1.9b07eb6c70573p-54,  0x1.612e8afad1255p-55, \
     0x1.6f46ad23182e4p-55,  -0x1.63aeabf42eae2p-54, 0x1.ada0911f09ebcp-55,  0x1.89b7a04ef80d0p-59, \
     0x1.d4397afec42e2p-56,  -0x1.07abe1db13cadp-55, 0x1.6324c054647adp-54,  -0x1.383c17e40b497p-54, \
     -0x1.bdd3413b26456p-54, -0x1.16e4786887a99p-55, -0x1.41577ee04992fp-55, -0x1.d4c1dd41532d8p-54, \
     0x1.6e9f156864b27p-54,  -0x1.75fc781b57ebcp-57, 0x1.c7c46b071f2bep-56,  -0x1.d2f6edb8d41e1p-54, \
     0x1.7a1cd345dcc81p-54,  -0x1.5584f7e54ac3bp-56, 0x1.11065895048ddp-55,  0x1.503cbd1e949dbp-56, \
     0x1.2ed02d75b3707p-55,  -0x1.1a5cd4f184b5cp-54, -0x1.e9c23179c2893p-54, 0x1.9d3e12dd8a18bp-54}

#if defined(__CUDACC__)
static __device__ const double mgcm_rt_exp_tab_dev[64] = MGCM_RT_EXP_TABLE;
#endif
static const double mgcm_rt_exp_tab_host[64] = MGCM_RT_EXP_TABLE;

#if defined(__CUDA_ARCH__)
#define MGCM_RT_MUL(a, b) __dmul_rn((a), (b))
#define MGCM_RT_ADD(a, b) __dadd_rn((a), (b))
#define MGCM_RT_RINT(x) rint(x)
#define MGCM_RT_TAB(i) __ldg(&mgcm_rt_exp_tab_dev[i])
#define MGCM_RT_UNROLL _Pragma("unroll")
#else
#define MGCM_RT_MUL(a, b) ((a) * (b))
#define MGCM_RT_ADD(a, b) ((a) + (b))
#define MGCM_RT_RINT(x) nearbyint(x)
#define MGCM_RT_TAB(i) (mgcm_rt_exp_tab_host[i])
#define MGCM_RT_UNROLL
#endif

MGCM_RT_HD double mgcm_rt_pow2i(int m) {
    const uint64_t bits = (uint64_t)(m + 1023) << 52;
    double r;
    memcpy(&r, &bits, sizeof r);
    return r;
}

/* exp(x), bit-identical on host (compiled without FMA contraction) and device. */
MGCM_RT_HD double mgcm_rt_exp(double x) {
    const double INV_L = 0x1.71547652b82fep+5;   /* 32/ln2 */
    const double L1 = 0x1.62e42fee00000p-6;      /* ln2/32, 32 significant bits */
    const double L2 = 0x1.a39ef35793c76p-38;     /* ln2/32 - L1 */
    const double A1 = 0x1.0000000000000p-1, A2 = 0x1.5555555555555p-3;
    const double A3 = 0x1.5555555555555p-5, A4 = 0x1.1111111111111p-7;
    const double A5 = 0x1.6c16c16c16c17p-10;
    if (!(x == x)) return x;                      /* NaN */
    if (x > 709.782712893383) return HUGE_VAL;
    if (x < -745.2) return 0.0;
    const double nf = MGCM_RT_RINT(MGCM_RT_MUL(x, INV_L));
    const int n = (int)nf;
    const int j = n & 31;
    const int m = (n - j) / 32;
    const double r1 = MGCM_RT_ADD(x, -MGCM_RT_MUL(nf, L1));
    const double r2 = -MGCM_RT_MUL(nf, L2);
    const double r = MGCM_RT_ADD(r1, r2);
    double q = MGCM_RT_ADD(A4, MGCM_RT_MUL(r, A5));
    q = MGCM_RT_ADD(A3, MGCM_RT_MUL(r, q));
    q = MGCM_RT_ADD(A2, MGCM_RT_MUL(r, q));
    q = MGCM_RT_ADD(A1, MGCM_RT_MUL(r, q));
    q = MGCM_RT_MUL(MGCM_RT_MUL(r, r), q);
    const double p = MGCM_RT_ADD(r1, MGCM_RT_ADD(r2, q));
    const double sl = MGCM_RT_TAB(j), st = MGCM_RT_TAB(32 + j);
    const double s = MGCM_RT_ADD(sl, st);
    const double v = MGCM_RT_ADD(sl, MGCM_RT_ADD(st, MGCM_RT_MUL(s, p)));
    if (m > 1023) return MGCM_RT_MUL(MGCM_RT_MUL(v, mgcm_rt_pow2i(m - 1)), 2.0);
    if (m >= -1022) return MGCM_RT_MUL(v, mgcm_rt_pow2i(m));
    return MGCM_RT_MUL(MGCM_RT_MUL(v, mgcm_rt_pow2i(m + 200)), mgcm_rt_pow2i(-200));
}

/* log10(x) for the interpolation weight of tpindex (code/tpindex.f90:93,106),
 * which the reference IR solver is as sensitive to as to EXP.  Method:
 * x = 2^e m, m in [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s), s = (m-1)/(m+1),
 * by its Taylor series in s^2 to s^23 (|s| <= 0.1716: truncation < 2^-57),
 * log10 x = e log10(2) + ln(m) log10(e) with log10(2) split so that
 * e*hi is exact.  About one ulp; identical on host and device. */
MGCM_RT_HD double mgcm_rt_log10(double x) {
    const double L2HI = 0x1.3441350800000p-2, L2LO = 0x1.f79fef311f12bp-34;
    const double LOG10E = 0x1.bcb7b1526e50ep-2, SQRT2 = 0x1.6a09e667f3bcdp+0;
    const double C[11] = {0x1.5555555555555p-2, 0x1.999999999999ap-3, 0x1.2492492492492p-3,
                          0x1.c71c71c71c71cp-4, 0x1.745d1745d1746p-4, 0x1.3b13b13b13b14p-4,
                          0x1.1111111111111p-4, 0x1.e1e1e1e1e1e1ep-5, 0x1.af286bca1af28p-5,
                          0x1.8618618618618p-5, 0x1.642c8590b2164p-5};
    if (!(x > 0.0)) return x == 0.0 ? -HUGE_VAL : (x - x) / (x - x);
    if (x == HUGE_VAL) return x;
    int e = 0;
    if (x < 0x1.0p-1022) {
        x = MGCM_RT_MUL(x, 0x1.0p+54);
        e = -54;
    }
    uint64_t bits;
    memcpy(&bits, &x, sizeof bits);
    e += (int)((bits >> 52) & 0x7ff) - 1023;
    bits = (bits & 0x000fffffffffffffull) | 0x3ff0000000000000ull;
    double m;
    memcpy(&m, &bits, sizeof m);
    if (m > SQRT2) {
        m = MGCM_RT_MUL(m, 0.5);
        e += 1;
    }
    const double f = MGCM_RT_ADD(m, -1.0);
    const double s = f / MGCM_RT_ADD(2.0, f);
    const double z = MGCM_RT_MUL(s, s);
    double r = C[10];
    for (int k = 9; k >= 0; --k) r = MGCM_RT_ADD(C[k], MGCM_RT_MUL(z, r));
    r = MGCM_RT_MUL(z, r);
    const double s2 = MGCM_RT_ADD(s, s);
    const double lnm = MGCM_RT_ADD(s2, MGCM_RT_MUL(s2, r));
    const double ed = (double)e;
    return MGCM_RT_ADD(MGCM_RT_MUL(ed, L2HI),
                       MGCM_RT_ADD(MGCM_RT_MUL(ed, L2LO), MGCM_RT_MUL(lnm, LOG10E)));
}

/* Natural logarithm, the same reduction and series as mgcm_rt_log10:
 * ln x = e ln2 + 2 atanh(s), ln2 split so that e*hi is exact.  About one ulp;
 * identical on host and device. */
MGCM_RT_HD double mgcm_rt_ln(double x) {
    const double LN2HI = 0x1.62e42fee00000p-1, LN2LO = 0x1.a39ef35793c76p-33;
    const double SQRT2 = 0x1.6a09e667f3bcdp+0;
    const double C[11] = {0x1.5555555555555p-2, 0x1.999999999999ap-3, 0x1.2492492492492p-3,
                          0x1.c71c71c71c71cp-4, 0x1.745d1745d1746p-4, 0x1.3b13b13b13b14p-4,
                          0x1.1111111111111p-4, 0x1.e1e1e1e1e1e1ep-5, 0x1.af286bca1af28p-5,
                          0x1.8618618618618p-5, 0x1.642c8590b2164p-5};
    if (!(x > 0.0)) return x == 0.0 ? -HUGE_VAL : (x - x) / (x - x);
    if (x == HUGE_VAL) return x;
    int e = 0;
    if (x < 0x1.0p-1022) {
        x = MGCM_RT_MUL(x, 0x1.0p+54);
        e = -54;
    }
    uint64_t bits;
    memcpy(&bits, &x, sizeof bits);
    e += (int)((bits >> 52) & 0x7ff) - 1023;
    bits = (bits & 0x000fffffffffffffull) | 0x3ff0000000000000ull;
    double m;
    memcpy(&m, &bits, sizeof m);
    if (m > SQRT2) {
        m = MGCM_RT_MUL(m, 0.5);
        e += 1;
    }
    const double f = MGCM_RT_ADD(m, -1.0);
    const double s = f / MGCM_RT_ADD(2.0, f);
    const double z = MGCM_RT_MUL(s, s);
    double r = C[10];
    for (int k = 9; k >= 0; --k) r = MGCM_RT_ADD(C[k], MGCM_RT_MUL(z, r));
    r = MGCM_RT_MUL(z, r);
    const double s2 = MGCM_RT_ADD(s, s);
    const double lnm = MGCM_RT_ADD(s2, MGCM_RT_MUL(s2, r));
    const double ed = (double)e;
    return MGCM_RT_ADD(MGCM_RT_MUL(ed, LN2HI), MGCM_RT_ADD(MGCM_RT_MUL(ed, LN2LO), lnm));
}

/* x**y for x > 0 as exp(y ln x) (the aerosol optics' real powers,
 * code/opt_dst.f:98,108, code/opt_cld.f:99,127,137).  Relative error about
 * (1 + |y ln x|) ulp. */
MGCM_RT_HD double mgcm_rt_pow(double x, double y) {
    return mgcm_rt_exp(MGCM_RT_MUL(y, mgcm_rt_ln(x)));
}

/* Error function (the DERF of the aerosol size-bin weights,
 * code/opt_dst.f:116-117).  |x| < 1.5: Maclaurin series
 *   erf x = 2/sqrt(pi) sum_n (-1)^n x^(2n+1) / (n! (2n+1)),
 * each term the previous one times -x^2 times the reciprocals 1/n and
 * 1/(2n+1) (correctly rounded: constants once the device unrolls the loop,
 * a division on the host), summed until the terms fall below 2^-60 of the
 * sum (at most 60 terms, 26 below 1.5);
 * 1.5 <= |x| < 6: erf x = 1 - erfc x with the continued fraction
 *   erfc x = exp(-x^2)/sqrt(pi) / (x + (1/2)/(x + 1/(x + (3/2)/(x + ...)))),
 * its 80th convergent A/B from the forward three-term recurrences (A, B stay
 * below 1e100 on this range; 80 terms converge to 1e-16 from x = 1.5 on);
 * |x| >= 6: +-1.  Absolute error below 1e-15 (8.9e-16 at most over a
 * 140,001-point scan of [-7, 7] against libm); identical on host and
 * device. */
MGCM_RT_HD double mgcm_rt_erf(double x) {
    const double TWO_RSQPI = 0x1.20dd750429b6dp+0, RSQPI = 0x1.20dd750429b6dp-1;
    const double ax = x < 0.0 ? -x : x;
    double r;
    if (ax < 1.5) {
        const double mx2 = -MGCM_RT_MUL(x, x);
        double t = x, sum = x;
        MGCM_RT_UNROLL
        for (int n = 1; n <= 60; ++n) {
            t = MGCM_RT_MUL(MGCM_RT_MUL(t, mx2), 1.0 / (double)n);
            const double term = MGCM_RT_MUL(t, 1.0 / (double)(2 * n + 1));
            sum = MGCM_RT_ADD(sum, term);
            const double at = term < 0.0 ? -term : term, as = sum < 0.0 ? -sum : sum;
            if (at < MGCM_RT_MUL(as, 0x1.0p-60)) break;
        }
        return MGCM_RT_MUL(TWO_RSQPI, sum);
    }
    if (ax >= 6.0) {
        r = 1.0;
    } else {
        double a1 = 1.0, a0 = ax, b1 = 0.0, b0 = 1.0;
        MGCM_RT_UNROLL
        for (int n = 1; n <= 80; ++n) {
            const double an = MGCM_RT_MUL(0.5, (double)n);
            const double a = MGCM_RT_ADD(MGCM_RT_MUL(ax, a0), MGCM_RT_MUL(an, a1));
            const double b = MGCM_RT_ADD(MGCM_RT_MUL(ax, b0), MGCM_RT_MUL(an, b1));
            a1 = a0;
            a0 = a;
            b1 = b0;
            b0 = b;
        }
        const double erfc = MGCM_RT_MUL(MGCM_RT_MUL(mgcm_rt_exp(-MGCM_RT_MUL(ax, ax)), RSQPI), b0 / a0);
        r = MGCM_RT_ADD(1.0, -erfc);
    }
    return x < 0.0 ? -r : r;
}

#endif /* MGCM_RT_MATH_H */
