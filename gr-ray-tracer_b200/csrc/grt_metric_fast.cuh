// Fast FP64 and FP32 right-hand sides of Hamilton's equations for the mixed
// trace form (grt_kernels_mixed.cu).  Same mathematics as ks_rhs
// (grt_metric.cuh; reference kerr_schild_core.hpp:157-192), reorganised for
// throughput instead of bitwise agreement with the reference's host build:
//   * the 21 divisions become 4 reciprocals (1/S, 1/r, 1/B, 1/D) and products;
//   * each reciprocal is one FP32 reciprocal refined by two Newton-Raphson
//     iterations x <- x + x (1 - a x) in FP64 (relative error ~1e-16);
//   * FMA contraction is on (the mixed translation unit is built with it).
#pragma once

#include "grt_metric.cuh"

namespace grt {
namespace dev {

// 1/a for positive normal a within FP32 range; other inputs take the IEEE path.
GRT_DEV double fast_rcp(double a) {
    if (!(a > 1e-30 && a < 1e30)) return 1.0 / a;
    double x = static_cast<double>(__frcp_rn(static_cast<float>(a)));
    double e = fma(-a, x, 1.0);
    x = fma(x, e, x);
    e = fma(-a, x, 1.0);
    return fma(x, e, x);
}

// FP64 right-hand side with reciprocals: the seven evolving components.
GRT_DEV Rhs7 ks_rhs_fast(double x, double y, double z, double pt, double px, double py, double pz,
                         double a, double M) {
    const double a2 = a * a;
    const double A = x * x + y * y + z * z - a2;
    const double az = a * z;
    const double S = sqrt(A * A + 4.0 * az * az);
    const double r = sqrt(0.5 * (A + S));
    const double invS = fast_rcp(S);
    const double invr = fast_rcp(r);
    const double opas = 1.0 + A * invS;
    const double h = 0.5 * invr * opas;
    const double dr0 = x * h, dr1 = y * h;
    const double dr2 = (z * opas + 2.0 * a2 * z * invS) * (0.5 * invr);
    const double B = r * r + a2;
    const double invB = fast_rcp(B);
    const double l1 = (r * x + a * y) * invB;
    const double l2 = (r * y - a * x) * invB;
    const double l3 = z * invr;
    const double twor = 2.0 * r;
    const double dB0 = twor * dr0, dB1 = twor * dr1, dB2 = twor * dr2;
    const double dl01 = ((dr0 * x + r) - l1 * dB0) * invB;
    const double dl02 = ((dr0 * y - a) - l2 * dB0) * invB;
    const double dl03 = -(l3 * dr0) * invr;
    const double dl11 = ((dr1 * x + a) - l1 * dB1) * invB;
    const double dl12 = ((dr1 * y + r) - l2 * dB1) * invB;
    const double dl13 = -(l3 * dr1) * invr;
    const double dl21 = (dr2 * x - l1 * dB2) * invB;
    const double dl22 = (dr2 * y - l2 * dB2) * invB;
    const double dl23 = (1.0 - l3 * dr2) * invr;
    const double r2 = r * r, r3 = r2 * r;
    const double D = r3 * r + az * az;
    const double invD = fast_rcp(D);
    const double H = M * r3 * invD;
    const double four_r3 = 4.0 * r3;
    const double MinvD2 = M * invD * invD;
    const double three_r2D = 3.0 * r2 * D;
    const double dH0 = (three_r2D * dr0 - r3 * (four_r3 * dr0)) * MinvD2;
    const double dH1 = (three_r2D * dr1 - r3 * (four_r3 * dr1)) * MinvD2;
    const double dH2 = (three_r2D * dr2 - r3 * (four_r3 * dr2 + 2.0 * a2 * z)) * MinvD2;
    const double ldp = ((-pt + l1 * px) + l2 * py) + l3 * pz;
    const double c = 2.0 * H * ldp;
    Rhs7 o;
    o.t = -pt + c;
    o.x = px - c * l1;
    o.y = py - c * l2;
    o.z = pz - c * l3;
    const double ldp2 = ldp * ldp;
    o.px = dH0 * ldp2 + c * ((dl01 * px + dl02 * py) + dl03 * pz);
    o.py = dH1 * ldp2 + c * ((dl11 * px + dl12 * py) + dl13 * pz);
    o.pz = dH2 * ldp2 + c * ((dl21 * px + dl22 * py) + dl23 * pz);
    return o;
}

// FP32 Kerr-Schild corrections on top of the exact flat-space part.  The
// flat part dx^mu/dlambda = eta^{mu nu} p_nu stays FP64; the correction
// -2H l^mu (l.p) and the whole dp/dlambda = dH (l.p)^2 + 2H (l.p)(dl.p) are
// O(M/r) and O(M/r^2) and carry FP32 rounding only at that scale.
GRT_DEV Rhs7 ks_rhs_fp32(double x, double y, double z, double rsq, double pt, double px, double py,
                         double pz, double a, double M) {
    const float xf = static_cast<float>(x), yf = static_cast<float>(y), zf = static_cast<float>(z);
    const float ptf = static_cast<float>(pt), pxf = static_cast<float>(px);
    const float pyf = static_cast<float>(py), pzf = static_cast<float>(pz);
    const float af = static_cast<float>(a), Mf = static_cast<float>(M);
    const float a2 = af * af;
    const float A = static_cast<float>(rsq) - a2;
    const float az = af * zf;
    const float S = sqrtf(A * A + 4.0f * az * az);
    const float r = sqrtf(0.5f * (A + S));
    const float invS = __frcp_rn(S);
    const float invr = __frcp_rn(r);
    const float opas = 1.0f + A * invS;
    const float h = 0.5f * invr * opas;
    const float dr0 = xf * h, dr1 = yf * h;
    const float dr2 = (zf * opas + 2.0f * a2 * zf * invS) * (0.5f * invr);
    const float B = r * r + a2;
    const float invB = __frcp_rn(B);
    const float l1 = (r * xf + af * yf) * invB;
    const float l2 = (r * yf - af * xf) * invB;
    const float l3 = zf * invr;
    const float twor = 2.0f * r;
    const float dB0 = twor * dr0, dB1 = twor * dr1, dB2 = twor * dr2;
    const float dl01 = ((dr0 * xf + r) - l1 * dB0) * invB;
    const float dl02 = ((dr0 * yf - af) - l2 * dB0) * invB;
    const float dl03 = -(l3 * dr0) * invr;
    const float dl11 = ((dr1 * xf + af) - l1 * dB1) * invB;
    const float dl12 = ((dr1 * yf + r) - l2 * dB1) * invB;
    const float dl13 = -(l3 * dr1) * invr;
    const float dl21 = (dr2 * xf - l1 * dB2) * invB;
    const float dl22 = (dr2 * yf - l2 * dB2) * invB;
    const float dl23 = (1.0f - l3 * dr2) * invr;
    const float r2 = r * r, r3 = r2 * r;
    const float D = r3 * r + az * az;
    const float invD = __frcp_rn(D);
    const float H = Mf * r3 * invD;
    const float four_r3 = 4.0f * r3;
    const float MinvD2 = Mf * invD * invD;
    const float three_r2D = 3.0f * r2 * D;
    const float dH0 = (three_r2D * dr0 - r3 * (four_r3 * dr0)) * MinvD2;
    const float dH1 = (three_r2D * dr1 - r3 * (four_r3 * dr1)) * MinvD2;
    const float dH2 = (three_r2D * dr2 - r3 * (four_r3 * dr2 + 2.0f * a2 * zf)) * MinvD2;
    const float ldp = ((-ptf + l1 * pxf) + l2 * pyf) + l3 * pzf;
    const float c = 2.0f * H * ldp;
    Rhs7 o;
    o.t = -pt + static_cast<double>(c);
    o.x = px - static_cast<double>(c * l1);
    o.y = py - static_cast<double>(c * l2);
    o.z = pz - static_cast<double>(c * l3);
    const float ldp2 = ldp * ldp;
    o.px = static_cast<double>(dH0 * ldp2 + c * ((dl01 * pxf + dl02 * pyf) + dl03 * pzf));
    o.py = static_cast<double>(dH1 * ldp2 + c * ((dl11 * pxf + dl12 * pyf) + dl13 * pzf));
    o.pz = static_cast<double>(dH2 * ldp2 + c * ((dl21 * pxf + dl22 * pyf) + dl23 * pzf));
    return o;
}

}  // namespace dev
}  // namespace grt
