// Mixed FP32/FP64 right-hand-side policy of the trace kernels.
//
// Right-hand side of Hamilton's equations (kerr_schild_core.hpp:157-192):
//   * FP32 form (ks_rhs_fp32): the exact flat-space part dx^mu/dlambda =
//     eta^{mu nu} p_nu stays FP64, the Kerr-Schild correction -2H l^mu (l.p)
//     and dp/dlambda are evaluated in FP32; being O(M/r) of the flat part,
//     their FP32 rounding enters the trajectory at ~1e-7 M/r relative;
//   * otherwise the FP64 parity form (ks_rhs), bit-identical to the plain
//     kernel (the trace kernels are built with -fmad=false).
// Which one a call uses: RK4 calls (fixed step) use FP32; an RK45 call uses
// FP32 only after emission (not ImageBackward) and outside the fluid grid.
// Before that, the adaptive step sequence decides where the backward ray
// first lands inside the grid -- the cell that emits it -- and any change of
// the step sequence, even at the last bit of FP64 (FMA contraction or a
// reciprocal in place of a division), moves that landing point for some rays
// and changes their emitted intensity.  After emission outside the grid the
// Stokes vector no longer changes, so FP32 there leaves the image intact.
//
// Kept in FP64:
//   * the state x^mu / p_mu and every Runge-Kutta stage combination and
//     update (the FP32 derivatives are accumulated in FP64, so no FP32
//     rounding of the accumulation itself enters the state);
//   * the step-size controller (error norm, pow, accept/reject);
//   * the whole right-hand side inside x^2+y^2+z^2 < fp64_radius_sq
//     (default (4M)^2 + a^2, i.e. r < 4M) and within the polar-axis cone
//     (x^2+y^2) < fp64_axis_sin2 (x^2+y^2+z^2);
//   * the null-constraint renormalisation after each accepted step: the
//     spatial p_i are rescaled (p_t, the conserved energy, is kept) so that
//     g^{mu nu} p_mu p_nu = 0 again;
//   * fluid sampling, radiative transfer, scattering and the camera test
//     (shared FP64 device code), so cell indices and Stokes updates follow
//     the FP64 form.
#pragma once

#include "grt_metric_fast.cuh"
#include "grt_trace.cuh"

namespace grt {
namespace dev {

// BF: the FP64 part is Fp64RhsT<BF>.
template <bool BF>
struct MixedRhsT {
    static GRT_DEV V7 eval(const double s[8], const KParams& kp, int fast) {
        const double x = s[1], y = s[2], z = s[3];
        const double rho2 = x * x + y * y;
        const double rsq = rho2 + z * z;
        if (!fast || rsq < kp.fp64_radius_sq || rho2 < kp.fp64_axis_sin2 * rsq)
            return Fp64RhsT<BF>::eval(s, kp, 0);
        return to_v7(ks_rhs_fp32(x, y, z, rsq, s[4], s[5], s[6], s[7], kp.a, kp.M));
    }

    // Null-constraint renormalisation in FP64 after a call that used the FP32
    // right-hand side: with l.p = -p_t + q, q = l_i p_i,
    // g^{mu nu} p_mu p_nu = alpha^2 (|p|^2 - 2H q^2) + alpha (4H p_t q) - (1+2H) p_t^2
    // for p_i -> alpha p_i; take the root near 1.
    static GRT_DEV void after_accept(double s[8], const KParams& kp, int fast) {
        if (!kp.renormalize || !fast) return;
        const double x = s[1], y = s[2], z = s[3];
        const double pt = s[4], px = s[5], py = s[6], pz = s[7];
        const double r = ks_radius(x, y, z, kp.a);
        const double B = r * r + kp.a * kp.a;
        const double l1 = (r * x + kp.a * y) / B, l2 = (r * y - kp.a * x) / B, l3 = z / r;
        const double H = kp.M * r * r * r / (r * r * r * r + kp.a * kp.a * z * z);
        const double q = l1 * px + l2 * py + l3 * pz;
        const double A = px * px + py * py + pz * pz - 2.0 * H * q * q;
        const double Bq = 4.0 * H * pt * q;
        const double C = -(1.0 + 2.0 * H) * pt * pt;
        const double disc = Bq * Bq - 4.0 * A * C;
        if (!(A > 0.0) || !(disc >= 0.0)) return;
        const double alpha = (-Bq + sqrt(disc)) / (2.0 * A);
        if (!(fabs(alpha - 1.0) < 1.0e-3)) return;
        s[5] = alpha * px;
        s[6] = alpha * py;
        s[7] = alpha * pz;
    }
};
using MixedRhs = MixedRhsT<false>;

}  // namespace dev
}  // namespace grt
