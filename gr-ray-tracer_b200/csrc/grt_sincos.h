// Deterministic sin/cos for the isotropic scattering and emission directions.
//
// Method: Cody & Waite argument reduction by pi/2 (pi/2 split into a 50-bit
// head, so k * head is exact for |k| <= 4, and a tail), then the Taylor
// series of sin and cos (coefficients 1/n!) on |r| <= pi/4 by Horner's rule
// in r^2, truncated where the next term is below 1e-21.  The same IEEE
// operations in the same order on the host and the device (no contraction:
// the kernels are built with -fmad=false, the oracle with -ffp-contract=off)
// give bit-identical results on both, which keeps the GPU and the oracle on
// the same trajectory after a scattering event.  Accuracy: a few ulp of the
// true values for |x| <= 2 pi (checked against mpmath).
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define GRT_SC_HD __host__ __device__ __forceinline__
#else
#define GRT_SC_HD inline
#endif

namespace grt {

GRT_SC_HD void det_sincos(double x, double* s, double* c) {
    const double k = rint(x * 0.6366197723675814);  // nearest integer to x / (pi/2)
    const double r = (x - k * 1.5707963267948966) - k * 6.123233995736766e-17;
    const double r2 = r * r;
    // sin r = r (1 - r^2/3! + r^4/5! - ... - r^20/21!)
    double ps = 1.9572941063391263e-20;
    ps = -8.22063524662433e-18 + r2 * ps;
    ps = 2.8114572543455206e-15 + r2 * ps;
    ps = -7.647163731819816e-13 + r2 * ps;
    ps = 1.6059043836821613e-10 + r2 * ps;
    ps = -2.505210838544172e-08 + r2 * ps;
    ps = 2.7557319223985893e-06 + r2 * ps;
    ps = -0.0001984126984126984 + r2 * ps;
    ps = 0.008333333333333333 + r2 * ps;
    ps = 0.16666666666666666 - r2 * ps;
    const double sr = r - (r * r2) * ps;
    // cos r = 1 - r^2/2! + r^4/4! - ... + r^20/20!
    double pc = 4.110317623312165e-19;
    pc = -1.5619206968586225e-16 + r2 * pc;
    pc = 4.779477332387385e-14 + r2 * pc;
    pc = -1.1470745597729725e-11 + r2 * pc;
    pc = 2.08767569878681e-09 + r2 * pc;
    pc = -2.755731922398589e-07 + r2 * pc;
    pc = 2.48015873015873e-05 + r2 * pc;
    pc = -0.001388888888888889 + r2 * pc;
    pc = 0.041666666666666664 + r2 * pc;
    pc = 0.5 - r2 * pc;
    const double cr = 1.0 - r2 * pc;
    const long long q = static_cast<long long>(k) & 3;
    if (q == 0) {
        *s = sr;
        *c = cr;
    } else if (q == 1) {
        *s = cr;
        *c = -sr;
    } else if (q == 2) {
        *s = -sr;
        *c = -cr;
    } else {
        *s = -cr;
        *c = sr;
    }
}

}  // namespace grt
