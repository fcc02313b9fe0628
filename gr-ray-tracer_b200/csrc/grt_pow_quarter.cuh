// pow(x, 0.25) for the RK45 step-size controller, rounded as glibc rounds it.
//
// The reference computes scale = safety * pow(1/err, 0.25)
// (src/geodesic_integrate/integrate_cart_ks.hpp:217) with the host libm.  One
// ulp in the proposed step changes every later step of the ray, so for the
// kernels to reproduce the reference's RK45 trajectories bit for bit this
// function must return what glibc's pow returns, including the ~0.08% of
// controller inputs that glibc rounds the other way from the exact result.
//
// glibc (2.28 and later; the image has 2.39) evaluates pow with the algorithm
// Szabolcs Nagy published in ARM's optimized-routines (math/pow.c).  This is a
// restatement of that published method for y = 1/4, written here from its
// description:
//   1. log(x) = k ln2 + log(c) + log1p(z/c - 1), x = 2^k z with z in
//      [OFF, 2 OFF); 1/c, log(c) and its tail come from a 128-entry table
//      chosen by the top mantissa bits of z, r = z/c - 1 is exact, and
//      log1p(r) - r + r^2/2 is a degree-8 polynomial.  The result is carried
//      as hi + lo with about 68 significant bits.
//   2. y*log(x) is exact for y = 1/4 (a power of two).
//   3. exp(e) = 2^(k/128) exp(r'), k = round(128 e / ln2),
//      r' = e - k ln2/128 + (the log's tail / 4), and
//      exp(r') - 1 - r' is a degree-5 polynomial; 2^(k/128) = scale (1 + tail)
//      from a 128-entry table.  The last step is fma(scale, t, scale).
// glibc on x86-64 runs this algorithm from its FMA build (ifunc-selected on
// CPUs with FMA and AVX2, which every B200 host has), where every multiply
// whose result feeds one addition is fused.  The fused/unfused choice of each
// operation below reproduces that build; three of them decide the last bit
// (the exp polynomial's two fused sums and the final fma), the rest give the
// same bits either way on the controller's inputs.  Tables and coefficients
// are generated by gen_pow_tables.py (rules and fits described there), and
// the function equals glibc's pow(x, 0.25) on 2e10 random inputs over the
// controller's unclamped range and on every tie-sensitive input found
// (tests/test_numerics.py, tests/test_gpu_division.py repeat samples of both).
//
// Kernels are built with -fmad=false and the oracle with -ffp-contract=off, so
// only the explicit fma() calls below are fused, on both sides.
#pragma once

#include <math.h>
#include <stdint.h>

#include "grt_pow_tables.h"

#if defined(__CUDACC__)
#define GRT_PQ_HD __host__ __device__ __forceinline__
#else
#define GRT_PQ_HD inline
#endif

namespace grt {
namespace pq {

static const double kLogTabH[3 * 128] = {GRT_POW_LOG_TABLE};
static const uint64_t kExpTabH[2 * 128] = {GRT_POW_EXP_TABLE};
#if defined(__CUDACC__)
static __device__ const double kLogTabD[3 * 128] = {GRT_POW_LOG_TABLE};
static __device__ const uint64_t kExpTabD[2 * 128] = {GRT_POW_EXP_TABLE};
#endif

GRT_PQ_HD double log_tab(int j) {
#if defined(__CUDA_ARCH__)
    return __ldg(&kLogTabD[j]);
#else
    return kLogTabH[j];
#endif
}

GRT_PQ_HD uint64_t exp_tab(int j) {
#if defined(__CUDA_ARCH__)
    return static_cast<uint64_t>(__ldg(reinterpret_cast<const unsigned long long*>(&kExpTabD[j])));
#else
    return kExpTabH[j];
#endif
}

GRT_PQ_HD uint64_t bits(double x) {
#if defined(__CUDA_ARCH__)
    return static_cast<uint64_t>(__double_as_longlong(x));
#else
    uint64_t b;
    __builtin_memcpy(&b, &x, 8);
    return b;
#endif
}

GRT_PQ_HD double from_bits(uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double(static_cast<long long>(b));
#else
    double x;
    __builtin_memcpy(&x, &b, 8);
    return x;
#endif
}

}  // namespace pq

// x^(1/4) as glibc's pow(x, 0.25) returns it, for every x (+-0 -> +0,
// +-inf -> +inf, other negatives and NaN -> NaN; subnormals are normalised
// first, as glibc does).
GRT_PQ_HD double pow_quarter(double x) {
    constexpr uint64_t kOff = 0x3fe6955500000000ull;
    constexpr double kA[6] = {GRT_POW_LOG_POLY};
    constexpr double kC[4] = {GRT_POW_EXP_POLY};
    uint64_t ix = pq::bits(x);
    if (ix - 0x0010000000000000ull >= 0x7ff0000000000000ull - 0x0010000000000000ull) {
        // zero, subnormal, infinite, NaN or negative
        if (x == 0.0) return 0.0;
        if ((ix << 1) == 0xffe0000000000000ull) return x * x;  // +-inf -> +inf
        if (!(x > 0.0)) return (x - x) / (x - x);               // NaN, negative -> NaN
        ix = pq::bits(x * 0x1p52) - (52ull << 52);  // subnormal: normalise
    }
    // log(x) as hi + lo
    const uint64_t tmp = ix - kOff;
    const int i = static_cast<int>((tmp >> 45) & 127u);
    const double k = static_cast<double>(static_cast<int64_t>(tmp) >> 52);
    const double z = pq::from_bits(ix - (tmp & (0xfffull << 52)));
    const double invc = pq::log_tab(3 * i), logc = pq::log_tab(3 * i + 1), logctail = pq::log_tab(3 * i + 2);
    const double r = fma(z, invc, -1.0);  // exact: 1/c has few significant bits
    const double t1 = k * GRT_POW_LN2HI + logc;  // exact
    const double t2 = t1 + r;
    const double lo1 = fma(k, GRT_POW_LN2LO, logctail);
    const double lo2 = t1 - t2 + r;
    const double ar = -0.5 * r;
    const double ar2 = r * ar;
    const double ar3 = r * ar2;
    const double hi = t2 + ar2;
    const double lo3 = fma(ar, r, -ar2);
    const double lo4 = t2 - hi + ar2;
    // log1p(r) - r + r^2/2 = ar3 * q(r); the coefficients are c_j scaled by
    // -2, -2, 4, 4, -8, -8 to absorb the powers of ar2 = -r^2/2
    const double q = fma(ar2, fma(ar2, fma(r, -8.0 * kA[5], -8.0 * kA[4]), fma(r, 4.0 * kA[3], 4.0 * kA[2])),
                         fma(r, -2.0 * kA[1], -2.0 * kA[0]));
    const double lo = fma(ar3, q, lo1 + lo2 + lo3 + lo4);
    const double y = hi + lo;
    const double ytail = hi - y + lo;
    // exp(y/4 + ytail/4)
    const double e = 0.25 * y, etail = 0.25 * ytail;
    if (((pq::bits(e) >> 52) & 0x7ff) < 0x3c9) return 1.0 + e;  // |e| < 2^-54
    constexpr double kShift = 0x1.8p52;
    double kd = fma(GRT_POW_INVLN2N, e, kShift);
    const uint64_t ki = pq::bits(kd);
    kd -= kShift;
    double rr = fma(kd, GRT_POW_NEGLN2LON, fma(kd, GRT_POW_NEGLN2HIN, e));
    rr += etail;
    const int idx = static_cast<int>(2 * (ki % 128));
    const double tail = pq::from_bits(pq::exp_tab(idx));
    const double scale = pq::from_bits(pq::exp_tab(idx + 1) + (ki << 45));
    const double r2 = rr * rr;
    const double r4 = r2 * r2;
    const double t = fma(r4, fma(rr, kC[3], kC[2]), fma(r2, fma(rr, kC[1], kC[0]), tail + rr));
    return fma(scale, t, scale);
}

}  // namespace grt
