// Kerr-Schild metric core and Hamilton's equations, FP64, for sm_100a.
//
// Same mathematics as the reference's kerr_schild namespace
// (src/metrics/kerr_schild_core.hpp:27-227): g_{mu nu} = eta + 2 H l_mu l_nu,
// r(x,y,z) from x^2+y^2+z^2 = r^2 + a^2 z^2 / r^2, H = M r^3 / (r^4 + a^2 z^2).
// The right-hand side is written out per component with the derivative
// selectors (dx/dx^k in {0,1}) resolved at compile time, but every non-trivial
// product and sum keeps the reference's association, so with FMA contraction
// disabled (this file is built with -fmad=false for the FP64 parity form) it
// rounds exactly like the reference's host code.  Multiplications by the
// literal 0/1 selectors and additions of the resulting zeros are omitted: they
// can change only the sign of an exact zero.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "grt_div.cuh"
#include "grt_rn.cuh"

namespace grt {
namespace dev {

#define GRT_DEV __device__ __forceinline__

constexpr double kPi = 3.14159265358979323846;

// Right-hand side of the photon ODE in the seven non-trivial components
// (dt, dx, dy, dz, dpx, dpy, dpz); dp_t/dlambda = 0 for the stationary metric.
struct Rhs7 {
    double t, x, y, z, px, py, pz;
};

// kerr_schild_core.hpp:27-33
GRT_DEV double ks_radius(double x, double y, double z, double a) {
    const double rsq = x * x + y * y + z * z;
    const double A = rsq - a * a;
    double r = A * A + 4.0 * ((a * z) * (a * z));
    // S = sqrt(A^2 + 4 (a z)^2), then r = sqrt((A + S) / 2), through one
    // sqrt site (a rolled loop keeps the step loop's code small)
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
        const double v = sqrt(r);
        r = k == 0 ? 0.5 * (A + v) : v;
    }
    return r;
}

// ks_radius out of line: the fallback of ks_radius_bf.
static __device__ __noinline__ double ks_radius_ieee(double x, double y, double z, double a) {
    return ks_radius(x, y, z, a);
}

// ks_radius with the branch-free square root (grt_rn.cuh) when both of its
// arguments lie in that function's exact range, [2^-900, 2^1000]; otherwise
// ks_radius itself.  The same value as ks_radius for every input: the test
// comes after both square roots, so they overlap with the work around them
// instead of waiting behind sqrt's slow-path branch.
GRT_DEV double ks_radius_bf(double x, double y, double z, double a) {
    const double rsq = x * x + y * y + z * z;
    const double A = rsq - a * a;
    const double v1 = A * A + 4.0 * ((a * z) * (a * z));
    const double S = sqrt_rn_box(v1);
    const double v2 = 0.5 * (A + S);
    const double r = sqrt_rn_box(v2);
    if (div_within<-900, 999>(v1) && div_within<-900, 999>(v2)) return r;
    return ks_radius_ieee(x, y, z, a);
}

// kerr_schild_core.hpp:157-192 (with compute_r_and_deriv :36-46,
// compute_l_and_deriv :58-77, compute_H_and_deriv :85-95 inlined).
GRT_DEV Rhs7 ks_rhs(double x, double y, double z, double pt, double px, double py, double pz,
                    double a, double M) {
    // r and dr/dx^k
    const double rsq = x * x + y * y + z * z;
    const double A = rsq - a * a;
    const double S = sqrt(A * A + 4.0 * ((a * z) * (a * z)));
    const double r = sqrt(0.5 * (A + S));
    const double opas = 1.0 + A / S;
    const double two_r = 2.0 * r;
    const double dr0 = x * opas / two_r;
    const double dr1 = y * opas / two_r;
    const double dr2 = (z * opas + 2.0 * (a * a) * z / S) / two_r;
    // l_mu and dl_mu/dx^k
    const double B = r * r + a * a;
    const double l1 = (r * x + a * y) / B;
    const double l2 = (r * y - a * x) / B;
    const double l3 = z / r;
    const double dB0 = 2.0 * r * dr0;
    const double dB1 = 2.0 * r * dr1;
    const double dB2 = 2.0 * r * dr2;
    const double dl01 = ((dr0 * x + r) - l1 * dB0) / B;
    const double dl02 = ((dr0 * y - a) - l2 * dB0) / B;
    const double dl03 = (0.0 - l3 * dr0) / r;
    const double dl11 = ((dr1 * x + a) - l1 * dB1) / B;
    const double dl12 = ((dr1 * y + r) - l2 * dB1) / B;
    const double dl13 = (0.0 - l3 * dr1) / r;
    const double dl21 = (dr2 * x - l1 * dB2) / B;
    const double dl22 = (dr2 * y - l2 * dB2) / B;
    const double dl23 = (1.0 - l3 * dr2) / r;
    // H and dH/dx^k
    const double r2 = r * r;
    const double r3 = r2 * r;
    const double D = r3 * r + (a * z) * (a * z);
    const double H = M * r3 / D;
    const double four_r3 = 4.0 * r3;
    const double dD0 = four_r3 * dr0;
    const double dD1 = four_r3 * dr1;
    const double dD2 = four_r3 * dr2 + 2.0 * (a * a) * z;
    const double three_r2 = 3.0 * r2;
    const double DD = D * D;
    const double dH0 = M * (three_r2 * dr0 * D - r3 * dD0) / DD;
    const double dH1 = M * (three_r2 * dr1 * D - r3 * dD1) / DD;
    const double dH2 = M * (three_r2 * dr2 * D - r3 * dD2) / DD;
    // contraction with p_mu (l^mu = (-1, l1, l2, l3))
    const double ldp = ((-pt + l1 * px) + l2 * py) + l3 * pz;
    const double twoH = 2.0 * H;
    Rhs7 o;
    o.t = -pt - (-twoH) * ldp;
    o.x = px - twoH * l1 * ldp;
    o.y = py - twoH * l2 * ldp;
    o.z = pz - twoH * l3 * ldp;
    const double ldp2 = ldp * ldp;
    const double twoHl = twoH * ldp;
    o.px = dH0 * ldp2 + twoHl * ((dl01 * px + dl02 * py) + dl03 * pz);
    o.py = dH1 * ldp2 + twoHl * ((dl11 * px + dl12 * py) + dl13 * pz);
    o.pz = dH2 * ldp2 + twoHl * ((dl21 * px + dl22 * py) + dl23 * pz);
    return o;
}

// ks_rhs with every quotient formed from the correctly rounded reciprocal of
// its denominator (six of them: S, 2r, B, r, D, D^2; five reciprocal
// evaluations, since RN(1/(2r)) = RN(1/r) / 2) by div_by, which rounds like an
// IEEE division while no value under- or overflows.  That holds in
// the box this checks first: x, y, z each an exact zero or of magnitude in
// [2^-20, 2^20], r in [2^-24, 2^20] and S in [2^-60, 2^42], with a spin of
// magnitude 0 or in [2^-20, 2] and a mass in [2^-20, 2^20] (checked on the
// host: rcp_ok).  Inside it every numerator, quotient and denominator stays
// in [2^-900, 2^900]: products of at most eight factors of at least 2^-60,
// differences of such products (zero, or at least 2^-52 of the smaller),
// divided by at most r^8 <= 2^160.  Outside it `ok` is false and the caller
// evaluates ks_rhs.  The expression tree is ks_rhs's, so the result equals
// ks_rhs bit for bit.
// BF selects the branch-free reciprocal and square root of grt_rn.cuh (equal
// to __drcp_rn and sqrt on every argument that reaches them here: the square
// roots' results are checked against the box before use, and every
// reciprocal's argument lies in [2^-192, 2^164]); without it, CUDA's.
template <bool BF>
GRT_DEV double rhs_recip(double b) {
    if constexpr (BF) return rcp_rn_box(b);
    else return div_recip(b);
}

template <bool BF>
GRT_DEV double rhs_sqrt(double v) {
    if constexpr (BF) return sqrt_rn_box(v);
    else return sqrt(v);
}

template <bool BF = false>
GRT_DEV Rhs7 ks_rhs_rcp(double x, double y, double z, double pt, double px, double py, double pz,
                        double a, double M, bool& ok) {
    const double rsq = x * x + y * y + z * z;
    const double A = rsq - a * a;
    // Two square-root sites (unlike ks_radius): the reciprocal of S and the
    // quotients that use it then overlap the second square root, which
    // measured 3% faster on a lane-per-SM workload than one rolled site.
    const double S = rhs_sqrt<BF>(A * A + 4.0 * ((a * z) * (a * z)));
    const double r = rhs_sqrt<BF>(0.5 * (A + S));
    ok = div_zero_or_within<-20, 19>(x) && div_zero_or_within<-20, 19>(y) && div_zero_or_within<-20, 19>(z) &&
         div_within<-24, 19>(r) && div_within<-60, 41>(S);
    Rhs7 o{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (!ok) return o;
    const double yS = rhs_recip<BF>(S);
    const double opas = 1.0 + div_by(A, S, yS);
    const double two_r = 2.0 * r;
    // RN(1/(2r)) = RN(1/r) / 2 exactly: r is inside the box, so no rounding
    // step under- or overflows
    const double yr = rhs_recip<BF>(r);
    const double y2r = 0.5 * yr;
    const double dr0 = div_by(x * opas, two_r, y2r);
    const double dr1 = div_by(y * opas, two_r, y2r);
    const double dr2 = div_by(z * opas + div_by(2.0 * (a * a) * z, S, yS), two_r, y2r);
    const double B = r * r + a * a;
    const double yB = rhs_recip<BF>(B);
    const double l1 = div_by(r * x + a * y, B, yB);
    const double l2 = div_by(r * y - a * x, B, yB);
    const double l3 = div_by(z, r, yr);
    const double dB0 = 2.0 * r * dr0;
    const double dB1 = 2.0 * r * dr1;
    const double dB2 = 2.0 * r * dr2;
    const double dl01 = div_by((dr0 * x + r) - l1 * dB0, B, yB);
    const double dl02 = div_by((dr0 * y - a) - l2 * dB0, B, yB);
    const double dl03 = div_by(0.0 - l3 * dr0, r, yr);
    const double dl11 = div_by((dr1 * x + a) - l1 * dB1, B, yB);
    const double dl12 = div_by((dr1 * y + r) - l2 * dB1, B, yB);
    const double dl13 = div_by(0.0 - l3 * dr1, r, yr);
    const double dl21 = div_by(dr2 * x - l1 * dB2, B, yB);
    const double dl22 = div_by(dr2 * y - l2 * dB2, B, yB);
    const double dl23 = div_by(1.0 - l3 * dr2, r, yr);
    const double r2 = r * r;
    const double r3 = r2 * r;
    const double D = r3 * r + (a * z) * (a * z);
    const double yD = rhs_recip<BF>(D);
    const double H = div_by(M * r3, D, yD);
    const double four_r3 = 4.0 * r3;
    const double dD0 = four_r3 * dr0;
    const double dD1 = four_r3 * dr1;
    const double dD2 = four_r3 * dr2 + 2.0 * (a * a) * z;
    const double three_r2 = 3.0 * r2;
    const double DD = D * D;
    const double yDD = rhs_recip<BF>(DD);
    const double dH0 = div_by(M * (three_r2 * dr0 * D - r3 * dD0), DD, yDD);
    const double dH1 = div_by(M * (three_r2 * dr1 * D - r3 * dD1), DD, yDD);
    const double dH2 = div_by(M * (three_r2 * dr2 * D - r3 * dD2), DD, yDD);
    const double ldp = ((-pt + l1 * px) + l2 * py) + l3 * pz;
    const double twoH = 2.0 * H;
    o.t = -pt - (-twoH) * ldp;
    o.x = px - twoH * l1 * ldp;
    o.y = py - twoH * l2 * ldp;
    o.z = pz - twoH * l3 * ldp;
    const double ldp2 = ldp * ldp;
    const double twoHl = twoH * ldp;
    o.px = dH0 * ldp2 + twoHl * ((dl01 * px + dl02 * py) + dl03 * pz);
    o.py = dH1 * ldp2 + twoHl * ((dl11 * px + dl12 * py) + dl13 * pz);
    o.pz = dH2 * ldp2 + twoHl * ((dl21 * px + dl22 * py) + dl23 * pz);
    return o;
}

// Metric pieces at a point: r, l_mu (l0 = 1) and H (compute_metric,
// kerr_schild_core.hpp:98-110).  g_{mu nu} = 2 H l_mu l_nu + eta_{mu nu}.
struct MetricAt {
    double l[4];
    double twoH;
    double g[4][4];
};

GRT_DEV void ks_metric_from_r(double x, double y, double z, double r, double a, double M,
                              MetricAt& m) {
    const double B = r * r + a * a;
    m.l[0] = 1.0;
    m.l[1] = (r * x + a * y) / B;
    m.l[2] = (r * y - a * x) / B;
    m.l[3] = z / r;
    const double D = r * r * r * r + (a * z) * (a * z);
    const double H = M * (r * r * r) / D;
    m.twoH = 2.0 * H;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) {
            const double v = m.twoH * m.l[mu] * m.l[nu];
            m.g[mu][nu] = (mu == nu) ? v + (mu == 0 ? -1.0 : 1.0) : v;
        }
    }
}

GRT_DEV void ks_metric(double x, double y, double z, double a, double M, MetricAt& m) {
    ks_metric_from_r(x, y, z, ks_radius(x, y, z, a), a, M, m);
}

// fluid_frame.hpp:6-13: sum over mu, nu of g[mu][nu]*u[mu]*v[nu], mu-major.
GRT_DEV double metric_dot(const double g[4][4], const double u[4], const double v[4]) {
    double s = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu)
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) s += g[mu][nu] * u[mu] * v[nu];
    return s;
}

// metric_dot(g, u, e_axis) for the unit coordinate vector e_axis.
GRT_DEV double metric_dot_unit(const double g[4][4], const double u[4], int axis) {
    double s = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) s += g[mu][axis] * u[mu];
    return s;
}

// kerr_schild_core.hpp:200-227: future-directed null p_mu from a spatial K^i.
GRT_DEV bool ks_null_momentum(const double X[4], const double K[3], double a, double M,
                              double p[4]) {
    MetricAt m;
    ks_metric(X[1], X[2], X[3], a, M, m);
    const double qa = m.g[0][0];
    const double qb = 2.0 * (m.g[0][1] * K[0] + m.g[0][2] * K[1] + m.g[0][3] * K[2]);
    double qc = 0.0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) qc += m.g[i + 1][j + 1] * K[i] * K[j];
    const double disc = qb * qb - 4.0 * qa * qc;
    if (disc < 0.0) return false;
    const double sq = sqrt(disc);
    const double K01 = (-qb + sq) / (2.0 * qa);
    const double K02 = (-qb - sq) / (2.0 * qa);
    const double K0 = (K01 > 0.0) ? K01 : K02;
    if (!(K0 > 0.0)) return false;
    const double Kc[4] = {K0, K[0], K[1], K[2]};
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        double s = 0.0;
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) s += m.g[mu][nu] * Kc[nu];
        p[mu] = s;
    }
    return true;
}

}  // namespace dev
}  // namespace grt
