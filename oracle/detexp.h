/*
 * detexp.h -- ORACLE (test infrastructure only).
 *
 * Deterministic single-precision exponential used by the oracle's
 * mixed-precision mode in place of the Fortran intrinsic EXP(REAL) that
 * get_kg.f:355-360 applies to the interpolated ln k.
 *
 * Method: Cody & Waite argument reduction (W. J. Cody, W. Waite, "Software
 * Manual for the Elementary Functions", Prentice-Hall 1980) with the two-part
 * ln 2 split published in fdlibm's e_exp.c (ln2_hi has 21 trailing zero bits,
 * so n*ln2_hi is exact for |n| < 2^21), followed by the degree-12 Taylor
 * polynomial of e^r on |r| <= ln2/2 (truncation error < 2e-16) evaluated by
 * Horner's rule in IEEE double with no fused multiply-add, scaled by 2^n and
 * rounded once to float.  Every step is a correctly rounded IEEE operation,
 * so the CUDA kernels (which use the same steps with __dmul_rn/__dadd_rn)
 * produce bit-identical results.  The result differs from the correctly
 * rounded e^x only when e^x lies within ~3e-16 (relative) of a float
 * rounding midpoint.
 *
 * Compile with -ffp-contract=off.
 */
#ifndef ORACLE_DETEXP_H
#define ORACLE_DETEXP_H

#include <math.h>
#include <stdint.h>
#include <string.h>

static inline double orc_pow2i(int n) {
    uint64_t bits = (uint64_t)(int64_t)(n + 1023) << 52;
    double d;
    memcpy(&d, &bits, sizeof d);
    return d;
}

static inline float orc_det_expf(float xf) {
    const double x = (double)xf;
    if (x != x) return xf;                       /* NaN propagates */
    if (x > 89.0) return INFINITY;               /* above ln(FLT_MAX) */
    if (x < -104.0) return 0.0f;                 /* below the float subnormal range */
    const double inv_ln2 = 1.44269504088896338700e+00;
    const double ln2_hi = 6.93147180369123816490e-01;
    const double ln2_lo = 1.90821492927058770002e-10;
    const double n = nearbyint(x * inv_ln2);     /* round half to even */
    const double r = (x - n * ln2_hi) - n * ln2_lo;
    /* 1/k!, k = 12..0 */
    static const double c[13] = {
        2.08767569878680989792e-09, 2.50521083854417187751e-08,
        2.75573192239858906526e-07, 2.75573192239858906526e-06,
        2.48015873015873015873e-05, 1.98412698412698412698e-04,
        1.38888888888888888889e-03, 8.33333333333333333333e-03,
        4.16666666666666666667e-02, 1.66666666666666666667e-01,
        5.00000000000000000000e-01, 1.00000000000000000000e+00,
        1.00000000000000000000e+00};
    double p = c[0];
    for (int k = 1; k < 13; ++k) p = p * r + c[k];
    return (float)(p * orc_pow2i((int)n));
}

#endif
