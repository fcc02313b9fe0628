// Correctly rounded FP64 quotients from a shared reciprocal.
//
// The right-hand side of Hamilton's equations divides 21 times by only six
// distinct values.  Each quotient a/b is formed from y = RN(1/b) (CUDA's
// correctly rounded reciprocal __drcp_rn, once per denominator) with the
// residual corrections of Markstein's division theorem (P. W. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990; Muller et al., Handbook of
// Floating-Point Arithmetic, ch. 4):
//   q0 = RN(a y)                  within 1.5 ulp of a/b (|y - 1/b| <= 2^-53 / |b|)
//   q1 = RN(q0 + RN(a - b q0) y)  within 1/2 ulp plus a negligible term: faithful
//   r1 = a - b q1                 exact (the remainder of a faithful quotient)
//   q2 = RN(q1 + r1 y)            = RN(a/b) by the theorem (y = RN(1/b), q1 faithful)
// Each residual and correction is one fused multiply-add (one rounding).  A
// zero numerator gives q0 = a y, the signed zero the division gives.  The
// theorem needs every value away from underflow and overflow; the caller
// guarantees it (ks_rhs_rcp checks its inputs against a box in which every
// numerator, denominator and quotient of the right-hand side stays inside
// [2^-900, 2^900]) and uses IEEE divisions outside.  A single-warp ncu probe
// on B200 counts 17 instructions for an IEEE FP64 division, 12 for
// __drcp_rn and 5 for div_by.
#pragma once

#include <cuda_runtime.h>

namespace grt {
namespace dev {

__device__ __forceinline__ double div_recip(double b) { return __drcp_rn(b); }

__device__ __forceinline__ double div_by(double a, double b, double y) {
    const double q0 = a * y;
    const double r0 = fma(-b, q0, a);
    const double q1 = fma(r0, y, q0);
    const double r1 = fma(-b, q1, a);
    const double q2 = fma(r1, y, q1);
    return a == 0.0 ? q0 : q2;
}

// Biased exponent of v (0 for zeros and subnormals, 2047 for inf/NaN).
__device__ __forceinline__ unsigned div_exponent(double v) {
    return (static_cast<unsigned>(__double2hiint(v)) >> 20) & 0x7FFu;
}

// v is an exact zero or 2^lo <= |v| < 2^(hi+1) (lo, hi unbiased).
template <int LO, int HI>
__device__ __forceinline__ bool div_zero_or_within(double v) {
    const unsigned e = div_exponent(v);
    return e == 0u ? (v == 0.0) : (e - static_cast<unsigned>(1023 + LO)) <= static_cast<unsigned>(HI - LO);
}

// 2^lo <= |v| < 2^(hi+1), v finite and normal.
template <int LO, int HI>
__device__ __forceinline__ bool div_within(double v) {
    return (div_exponent(v) - static_cast<unsigned>(1023 + LO)) <= static_cast<unsigned>(HI - LO);
}

}  // namespace dev
}  // namespace grt
