// Correctly rounded x^(1/4) for the RK45 step-size controller.
//
// The reference evaluates scale = safety * pow(1/err, 0.25)
// (src/geodesic_integrate/integrate_cart_ks.hpp:217).  pow is not correctly
// rounded in any libm we can call on both sides (glibc's errs by up to 0.52 ulp
// and misrounds ~0.1% of the controller's inputs; CUDA's by up to 2 ulp), and a
// single ulp in the proposed step changes the whole later step sequence.  This
// function returns the correctly rounded fourth root instead, so the kernels
// and the CPU oracle agree bit for bit:
//   y = RN(sqrt(RN(sqrt(x))))  (IEEE sqrt, identical on host and device) is
//   within 1.5 ulp of x^(1/4); a floating-point rounding test with a proven
//   error bound settles almost every candidate, and y is otherwise moved while
//   x lies beyond the fourth power of the rounding midpoint next to it, tested
//   exactly in 256-bit integer arithmetic (a midpoint has 54+ significant
//   bits, so x can never equal its fourth power: there are no ties).
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define GRT_FR_HD __host__ __device__ __forceinline__
#define GRT_FR_SLOW static __host__ __device__ __noinline__
#else
#define GRT_FR_HD inline
#define GRT_FR_SLOW inline
#endif

namespace grt {
namespace fr {

GRT_FR_HD uint64_t bits_of(double x) {
#if defined(__CUDA_ARCH__)
    return static_cast<uint64_t>(__double_as_longlong(x));
#else
    uint64_t b;
    __builtin_memcpy(&b, &x, 8);
    return b;
#endif
}

GRT_FR_HD double from_bits(uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double(static_cast<long long>(b));
#else
    double x;
    __builtin_memcpy(&x, &b, 8);
    return x;
#endif
}

GRT_FR_HD void mul64(uint64_t a, uint64_t b, uint64_t& lo, uint64_t& hi) {
#if defined(__CUDA_ARCH__)
    lo = a * b;
    hi = __umul64hi(a, b);
#else
    const unsigned __int128 p = static_cast<unsigned __int128>(a) * b;
    lo = static_cast<uint64_t>(p);
    hi = static_cast<uint64_t>(p >> 64);
#endif
}

// w[0..3] += (hi:lo) << (64 * at); the sums stay below 2^256 here.
GRT_FR_HD void add128(uint64_t w[4], int at, uint64_t lo, uint64_t hi) {
    const uint64_t s0 = w[at] + lo;
    uint64_t c = s0 < lo ? 1 : 0;
    w[at] = s0;
    if (at + 1 >= 4) return;
    const uint64_t t = hi + c;
    const uint64_t c1 = t < c ? 1 : 0;
    const uint64_t s1 = w[at + 1] + t;
    const uint64_t c2 = s1 < t ? 1 : 0;
    w[at + 1] = s1;
    c = c1 + c2;
    for (int q = at + 2; q < 4 && c; ++q) {
        const uint64_t sq = w[q] + c;
        c = sq < c ? 1 : 0;
        w[q] = sq;
    }
}

// A^4 for A < 2^56 as a 256-bit integer.
GRT_FR_HD void pow4(uint64_t A, uint64_t w[4]) {
    uint64_t l, h;
    mul64(A, A, l, h);  // A^2 = h*2^64 + l, h < 2^48
    w[0] = w[1] = w[2] = w[3] = 0;
    uint64_t p0l, p0h, p1l, p1h, p2l, p2h;
    mul64(l, l, p0l, p0h);
    mul64(h, l, p1l, p1h);
    mul64(h, h, p2l, p2h);
    add128(w, 0, p0l, p0h);
    add128(w, 1, p1l, p1h);
    add128(w, 1, p1l, p1h);
    add128(w, 2, p2l, p2h);
}

// sign of (A^4 * 2^0) - (X * 2^s): +1, 0 or -1 (s >= 0).
GRT_FR_HD int cmp_pow4(uint64_t A, uint64_t X, int s) {
    uint64_t P[4];
    pow4(A, P);
    uint64_t Q[4] = {0, 0, 0, 0};
    if (s < 0) return 1;  // never happens for finite positive inputs (P ~ 2^213)
    const int q = s >> 6, r = s & 63;
    if (q >= 4) return -1;
    Q[q] = X << r;
    if (r && q + 1 < 4) Q[q + 1] = X >> (64 - r);
    else if (r && q + 1 >= 4 && (X >> (64 - r)) != 0) return -1;
    for (int k = 3; k >= 0; --k) {
        if (P[k] != Q[k]) return P[k] > Q[k] ? 1 : -1;
    }
    return 0;
}

// decompose a positive finite double into integer mantissa and exponent
GRT_FR_HD void decompose(double v, uint64_t& m, int& e) {
    const uint64_t b = bits_of(v);
    const int eb = static_cast<int>((b >> 52) & 0x7FF);
    const uint64_t frac = b & ((1ull << 52) - 1);
    if (eb == 0) {
        m = frac;
        e = -1074;
    } else {
        m = frac | (1ull << 52);
        e = eb - 1075;
    }
}

}  // namespace fr

// Correctly rounded (to nearest) x^(1/4) for x >= 0 by the exact midpoint
// test alone (the fallback of fourth_root_cr).
GRT_FR_SLOW double fourth_root_exact(double x) {
    if (!(x > 0.0) || !(x < INFINITY)) return sqrt(sqrt(x));  // 0, inf, nan
    double y = sqrt(sqrt(x));
    uint64_t X;
    int F;
    fr::decompose(x, X, F);
    for (int it = 0; it < 4; ++it) {
        uint64_t M;
        int E;
        fr::decompose(y, M, E);
        // upper midpoint (2M+1) 2^(E-1): move up while x > mid^4
        if (fr::cmp_pow4(2 * M + 1, X, F - 4 * (E - 1)) < 0) {
            y = fr::from_bits(fr::bits_of(y) + 1);
            continue;
        }
        // lower midpoint: (2M-1) 2^(E-1), or (4M-1) 2^(E-2) when y is a power of two
        const bool pow2 = M == (1ull << 52);
        const uint64_t A = pow2 ? 4 * M - 1 : 2 * M - 1;
        const int sh = pow2 ? F - 4 * (E - 2) : F - 4 * (E - 1);
        if (fr::cmp_pow4(A, X, sh) > 0) {
            y = fr::from_bits(fr::bits_of(y) - 1);
            continue;
        }
        break;
    }
    return y;
}

// Correctly rounded (to nearest) x^(1/4) for x >= 0.
//
// Fast path (Ziv-style rounding test): for a candidate y = M 2^E that is not a
// power of two, with u = 2^E its ulp, y is the correctly rounded root iff
// (y - u/2)^4 < x < (y + u/2)^4.  Both gaps exceed 2 y^3 u (1 - 2^-52), so
// |x - y^4| < 2 y^3 u (1 - 2^-42) proves y.  The residual is formed with
// exact products (y^2 = p + pe, p^2 = q + qe by fma) and x - q exact by
// Sterbenz's lemma; its error is below 2^-103 y^4 < 2^-51 (2 y^3 u), and the
// computed bound 2 (p y) u (1 - 2^-40) is below 2 y^3 u (1 - 2^-41), so an
// accepted y is always the correctly rounded one.  A residual beyond the
// bound moves y one ulp and tests again; powers of two, inputs outside
// [2^-900, 2^900] (where the products could leave the normal range) and
// candidates the test cannot settle in three tries take the exact path.
GRT_FR_HD double fourth_root_cr(double x) {
    if (x > 0x1p-900 && x < 0x1p900) {
        double y = sqrt(sqrt(x));
        for (int it = 0; it < 3; ++it) {
            const uint64_t b = fr::bits_of(y);
            if ((b & ((1ull << 52) - 1)) == 0) break;  // power of two
            const double u = fr::from_bits((b & (0x7FFull << 52)) - (52ull << 52));  // 2^E
            const double p = y * y;
            const double pe = fma(y, y, -p);
            const double q = p * p;
            const double qe = fma(p, p, -q);
            const double lo = qe + (2.0 * p) * pe;
            const double r = (x - q) - lo;
            const double T = ((2.0 * (p * y)) * u) * (1.0 - 0x1p-40);
            if (r > T) {
                y = fr::from_bits(b + 1);
            } else if (r < -T) {
                y = fr::from_bits(b - 1);
            } else {
                return y;
            }
        }
    }
    return fourth_root_exact(x);
}

}  // namespace grt
