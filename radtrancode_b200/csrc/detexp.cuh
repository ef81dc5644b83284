// detexp.cuh -- deterministic single-precision exponential for the k-table
// interpolation (the EXP(REAL) of radtran/cirsradg/get_kg.f:355-360).
//
// Cody & Waite argument reduction (Cody, Waite, "Software Manual for the
// Elementary Functions", 1980) with fdlibm's published two-part ln 2
// (ln2_hi carries 21 trailing zero bits, so n*ln2_hi is exact for the
// |n| <= 150 reached here), then the degree-12 Taylor polynomial of e^r on
// |r| <= ln2/2 by Horner's rule in IEEE double.  Every operation is an
// explicitly rounded intrinsic (no fused multiply-add), so the result is the
// same bit pattern on any IEEE-754 machine that performs the same steps; the
// host-side restatement used to check this kernel performs them in the same
// order.  The sort keys of the random-overlap rebinning are built from these
// values, which is what makes the integer g-bin assignment reproducible.
#pragma once

namespace rtb {

__device__ __forceinline__ float det_expf(float xf) {
    const double x = (double)xf;
    if (x != x) return xf;
    if (x > 89.0) return __int_as_float(0x7f800000);
    if (x < -104.0) return 0.0f;
    const double inv_ln2 = 1.44269504088896338700e+00;
    const double ln2_hi = 6.93147180369123816490e-01;
    const double ln2_lo = 1.90821492927058770002e-10;
    const double n = rint(__dmul_rn(x, inv_ln2));
    const double r = __dsub_rn(__dsub_rn(x, __dmul_rn(n, ln2_hi)), __dmul_rn(n, ln2_lo));
    double p = 2.08767569878680989792e-09;
    p = __dadd_rn(__dmul_rn(p, r), 2.50521083854417187751e-08);
    p = __dadd_rn(__dmul_rn(p, r), 2.75573192239858906526e-07);
    p = __dadd_rn(__dmul_rn(p, r), 2.75573192239858906526e-06);
    p = __dadd_rn(__dmul_rn(p, r), 2.48015873015873015873e-05);
    p = __dadd_rn(__dmul_rn(p, r), 1.98412698412698412698e-04);
    p = __dadd_rn(__dmul_rn(p, r), 1.38888888888888888889e-03);
    p = __dadd_rn(__dmul_rn(p, r), 8.33333333333333333333e-03);
    p = __dadd_rn(__dmul_rn(p, r), 4.16666666666666666667e-02);
    p = __dadd_rn(__dmul_rn(p, r), 1.66666666666666666667e-01);
    p = __dadd_rn(__dmul_rn(p, r), 5.00000000000000000000e-01);
    p = __dadd_rn(__dmul_rn(p, r), 1.00000000000000000000e+00);
    p = __dadd_rn(__dmul_rn(p, r), 1.00000000000000000000e+00);
    const long long bits = (long long)((int)n + 1023) << 52;
    return __double2float_rn(__dmul_rn(p, __longlong_as_double(bits)));
}

}  // namespace rtb
