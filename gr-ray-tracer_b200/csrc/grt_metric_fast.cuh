// FP32 right-hand side of Hamilton's equations for the mixed trace form
// (MixedRhs in grt_rhs_mixed.cuh).  Same mathematics as ks_rhs (grt_metric.cuh;
// reference kerr_schild_core.hpp:157-192), reorganised for FP32 throughput:
// the 21 divisions and 2 square roots become 2 reciprocal square roots and 2
// reciprocals on the special-function unit, and the multiply-adds are
// written as explicit fmaf (the mixed
// translation unit is built without automatic contraction so that its FP64
// path stays bit-identical to the parity form).
#pragma once

#include "grt_metric.cuh"

namespace grt {
namespace dev {

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
    const float S2 = fmaf(A, A, 4.0f * az * az);
    const float invS = rsqrtf(S2);  // special-function unit, ~2 ulp
    const float S = S2 * invS;
    const float r2h = 0.5f * (A + S);
    const float invr = rsqrtf(r2h);
    const float r = r2h * invr;
    const float opas = fmaf(A, invS, 1.0f);
    const float h = 0.5f * invr * opas;
    const float dr0 = xf * h, dr1 = yf * h;
    const float dr2 = fmaf(zf, opas, 2.0f * a2 * zf * invS) * (0.5f * invr);
    const float B = fmaf(r, r, a2);
    const float invB = __fdividef(1.0f, B);
    const float l1 = fmaf(r, xf, af * yf) * invB;
    const float l2 = fmaf(r, yf, -af * xf) * invB;
    const float l3 = zf * invr;
    const float twor = 2.0f * r;
    const float dB0 = twor * dr0, dB1 = twor * dr1, dB2 = twor * dr2;
    const float dl01 = fmaf(-l1, dB0, fmaf(dr0, xf, r)) * invB;
    const float dl02 = fmaf(-l2, dB0, fmaf(dr0, yf, -af)) * invB;
    const float dl03 = -(l3 * dr0) * invr;
    const float dl11 = fmaf(-l1, dB1, fmaf(dr1, xf, af)) * invB;
    const float dl12 = fmaf(-l2, dB1, fmaf(dr1, yf, r)) * invB;
    const float dl13 = -(l3 * dr1) * invr;
    const float dl21 = fmaf(-l1, dB2, dr2 * xf) * invB;
    const float dl22 = fmaf(-l2, dB2, dr2 * yf) * invB;
    const float dl23 = fmaf(-l3, dr2, 1.0f) * invr;
    const float r2 = r * r, r3 = r2 * r;
    const float D = fmaf(r3, r, az * az);
    const float invD = __fdividef(1.0f, D);
    const float H = Mf * r3 * invD;
    const float four_r3 = 4.0f * r3;
    const float MinvD2 = Mf * invD * invD;
    const float three_r2D = 3.0f * r2 * D;
    const float dH0 = fmaf(three_r2D, dr0, -r3 * (four_r3 * dr0)) * MinvD2;
    const float dH1 = fmaf(three_r2D, dr1, -r3 * (four_r3 * dr1)) * MinvD2;
    const float dH2 = fmaf(three_r2D, dr2, -r3 * fmaf(four_r3, dr2, 2.0f * a2 * zf)) * MinvD2;
    const float ldp = fmaf(l3, pzf, fmaf(l2, pyf, fmaf(l1, pxf, -ptf)));
    const float c = 2.0f * H * ldp;
    Rhs7 o;
    o.t = -pt + static_cast<double>(c);
    o.x = px - static_cast<double>(c * l1);
    o.y = py - static_cast<double>(c * l2);
    o.z = pz - static_cast<double>(c * l3);
    const float ldp2 = ldp * ldp;
    o.px = static_cast<double>(fmaf(dH0, ldp2, c * fmaf(dl03, pzf, fmaf(dl02, pyf, dl01 * pxf))));
    o.py = static_cast<double>(fmaf(dH1, ldp2, c * fmaf(dl13, pzf, fmaf(dl12, pyf, dl11 * pxf))));
    o.pz = static_cast<double>(fmaf(dH2, ldp2, c * fmaf(dl23, pzf, fmaf(dl22, pyf, dl21 * pxf))));
    return o;
}

}  // namespace dev
}  // namespace grt
