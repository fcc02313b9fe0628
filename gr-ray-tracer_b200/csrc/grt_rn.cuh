// Branch-free, correctly rounded FP64 reciprocal and square root for the
// arguments of ks_rhs_rcp (grt_metric.cuh).
//
// CUDA's __drcp_rn and sqrt handle every input, zeros, subnormals and
// infinities included, and so carry a branch to a slow path.  Each such
// branch ends a basic block, and the compiler does not move independent work
// across it: the seven reciprocals and square roots of one right-hand side
// then run one after another, and a lone warp waits out each of them.  These
// forms have no branch.  They are exact (equal to __drcp_rn and to the IEEE
// square root bit for bit) on the ranges stated below, which contain every
// argument that reaches them.
//
// Both start from the PTX approximation instructions (rcp.approx.ftz.f64 and
// rsqrt.approx.ftz.f64; on 1.9e7 random arguments on B200 the largest
// |b y - 1| was 2^-19.9 and the largest |v y^2 - 1| 2^-19.0) and refine with
// two Newton-Raphson steps, each of which squares the relative error: about
// 2^-78 before rounding, so the refined value is faithful.
// The last step of each is Markstein's correction (P. W. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990; M. Cornea, J. Harrison,
// P. T. P. Tang, "Scientific Computing on Itanium-based Systems", 2002,
// ch. 8), each residual formed exactly by one fused multiply-add:
//   reciprocal:  y faithful to 1/b, e = 1 - b y (exact), RN(y + y e) = RN(1/b),
//                except when b's significand is all ones.  There
//                1/b = 2^(-E-1) (1 + 2^-53 + 2^-106 + ...), just above the
//                midpoint, so RN(1/b) = 2^(-E-1) (1 + 2^-52), set directly;
//   square root: y close to 1/sqrt(v), s = RN(v y), r = v - s^2 (exact),
//                RN(s + r y/2) = RN(sqrt(v)).
// Ranges: rcp_rn_box is exact for |b| in [2^-1000, 2^1000]; sqrt_rn_box for v
// in [2^-900, 2^1000] (below that the residual v - s^2 can leave the normal
// range and lose bits, and the result can be an ulp off).  For any other
// argument sqrt_rn_box gives NaN (zero, a subnormal, +inf, NaN) or a value
// outside [2^-450, 2^500], so a box check on the result rejects it as it
// rejects the exact square root.  In ks_rhs_rcp every square root whose
// result passes the box has its argument in [2^-120, 2^86], and every
// reciprocal's argument lies in [2^-192, 2^164].  The device self-test
// (grt_selftest_rn_box) compares both with CUDA's functions on random,
// all-ones and midpoint-square arguments.
#pragma once

#include <cuda_runtime.h>

namespace grt {
namespace dev {

__device__ __forceinline__ double rcp_seed(double b) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    return y;
}

__device__ __forceinline__ double rsqrt_seed(double v) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(v));
    return y;
}

__device__ __forceinline__ double rcp_rn_box(double b) {
    double y = rcp_seed(b);
    double e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    e = fma(-b, y, 1.0);
    y = fma(y, e, y);
    // all-ones significand: RN(1/b) = sign(b) 2^(-E-1) (1 + 2^-52); with b's
    // biased exponent eb = E + 1023 that is biased exponent 2045 - eb
    const unsigned hi = static_cast<unsigned>(__double2hiint(b));
    const unsigned lo = static_cast<unsigned>(__double2loint(b));
    const bool ones = (hi & 0x000FFFFFu) == 0x000FFFFFu && lo == 0xFFFFFFFFu;
    const unsigned eb = (hi >> 20) & 0x7FFu;
    const unsigned hi_ones = (hi & 0x80000000u) | ((2045u - eb) << 20);
    return ones ? __hiloint2double(static_cast<int>(hi_ones), 1) : y;
}

__device__ __forceinline__ double sqrt_rn_box(double v) {
    double y = rsqrt_seed(v);
    double h = 0.5 * y;
    double e = fma(-(v * y), y, 1.0);
    y = fma(h, e, y);
    h = 0.5 * y;
    e = fma(-(v * y), y, 1.0);
    y = fma(h, e, y);
    h = 0.5 * y;
    const double s = v * y;
    const double r = fma(-s, s, v);
    return fma(r, h, s);
}

}  // namespace dev
}  // namespace grt
