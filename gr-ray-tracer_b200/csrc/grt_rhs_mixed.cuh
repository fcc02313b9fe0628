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

// The renormalisation's root near 1 with IEEE division and sqrt (out of line:
// the fallback outside the box).
static __device__ __noinline__ double renorm_alpha_ieee(double Bq, double disc, double A) {
    return (-Bq + sqrt(disc)) / (2.0 * A);
}

// BF: the FP64 part is Fp64RhsT<BF>.  LAT: as for Fp64RhsT; the
// renormalisation also takes the branch-free forms there.
template <bool BF, bool LAT = false>
struct MixedRhsT {
    static constexpr bool kLatency = LAT;
    static GRT_DEV V7 eval(const double s[8], const KParams& kp, int fast) {
        const double x = s[1], y = s[2], z = s[3];
        const double rho2 = x * x + y * y;
        const double rsq = rho2 + z * z;
        if (!fast || rsq < kp.fp64_radius_sq || rho2 < kp.fp64_axis_sin2 * rsq)
            return Fp64RhsT<BF, LAT>::eval(s, kp, 0);
        return to_v7(ks_rhs_fp32(x, y, z, rsq, s[4], s[5], s[6], s[7], kp.a, kp.M));
    }

    // Null-constraint renormalisation in FP64 after a call that used the FP32
    // right-hand side: with l.p = -p_t + q, q = l_i p_i,
    // g^{mu nu} p_mu p_nu = alpha^2 (|p|^2 - 2H q^2) + alpha (4H p_t q) - (1+2H) p_t^2
    // for p_i -> alpha p_i; take the root near 1.  Returns the Kerr-Schild
    // radius of the position (unchanged by the rescale), which post_step
    // then takes instead of computing it again, or -1 when nothing was done.
    // With LAT its quotients and square roots are the branch-free forms
    // (grt_div.cuh, grt_rn.cuh) inside the box where they equal IEEE division
    // and sqrt (the box of ks_rhs_rcp for l and H; [2^-400, 2^400] for the
    // operands of alpha), IEEE outside: the result is the same either way.
    static GRT_DEV double after_accept(double s[8], const KParams& kp, int fast) {
        if (!kp.renormalize || !fast) return -1.0;
        const double x = s[1], y = s[2], z = s[3];
        const double pt = s[4], px = s[5], py = s[6], pz = s[7];
        const double a = kp.a;
        const double r = LAT ? ks_radius_bf(x, y, z, a) : ks_radius(x, y, z, a);
        const double B = r * r + a * a;
        const double nH = kp.M * r * r * r;
        const double Dn = r * r * r * r + a * a * z * z;
        double l1, l2, l3, H;
        if (LAT && kp.rcp_ok && div_zero_or_within<-20, 19>(x) && div_zero_or_within<-20, 19>(y) &&
            div_zero_or_within<-20, 19>(z) && div_within<-24, 19>(r)) {
            const double yB = rcp_rn_box(B), yr = rcp_rn_box(r), yD = rcp_rn_box(Dn);
            l1 = div_by(r * x + a * y, B, yB);
            l2 = div_by(r * y - a * x, B, yB);
            l3 = div_by(z, r, yr);
            H = div_by(nH, Dn, yD);
        } else {
            l1 = (r * x + a * y) / B;
            l2 = (r * y - a * x) / B;
            l3 = z / r;
            H = nH / Dn;
        }
        const double q = l1 * px + l2 * py + l3 * pz;
        const double A = px * px + py * py + pz * pz - 2.0 * H * q * q;
        const double Bq = 4.0 * H * pt * q;
        const double C = -(1.0 + 2.0 * H) * pt * pt;
        const double disc = Bq * Bq - 4.0 * A * C;
        if (!(A > 0.0) || !(disc >= 0.0)) return r;
        double alpha;
        if constexpr (LAT) {
            const double twoA = 2.0 * A;
            const double num = -Bq + sqrt_rn_box(disc);
            alpha = div_by(num, twoA, rcp_rn_box(twoA));
            if (!(div_within<-900, 999>(disc) && div_within<-400, 399>(twoA) && div_zero_or_within<-400, 399>(num)))
                alpha = renorm_alpha_ieee(Bq, disc, A);
        } else {
            alpha = (-Bq + sqrt(disc)) / (2.0 * A);
        }
        if (!(fabs(alpha - 1.0) < 1.0e-3)) return r;
        s[5] = alpha * px;
        s[6] = alpha * py;
        s[7] = alpha * pz;
        return r;
    }
};
using MixedRhs = MixedRhsT<false>;

}  // namespace dev
}  // namespace grt
