// Host-side staging of a separable grid's axes, shared by every entry point
// that traces against a grid (grt_upload_grid in grt_api.cu and
// grt_trace_device_noalloc in grt_noalloc.cu), so that all of them derive the
// lookup's acceptance bounds with the same glibc arithmetic and agree bit for
// bit at cell edges.  Plain arrays in, plain arrays out: nothing allocates.
#pragma once

#include <cmath>
#include <cstddef>

namespace grt {
namespace axes {

constexpr double kPi = 3.14159265358979323846;  // src/utils.hpp:16

// scattering.hpp:41-46: angular distance on the circle, glibc fmod.
inline double periodic_distance(double lhs, double rhs) {
    const double d = std::fmod(std::fabs(lhs - rhs), 2.0 * kPi);
    return std::fmin(d, 2.0 * kPi - d);
}

// scattering.hpp:100-149: the acceptance half-width 0.500001 * (largest
// neighbour span) of each value of one separable axis -- log spacing for the
// radius (kind 0), linear for theta (kind 1), periodic for phi (kind 2) --
// evaluated with glibc as the reference evaluates it on every call.
inline void half_spans(const double* a, size_t n, int kind, double* h) {
    for (size_t i = 0; i < n; ++i) {
        if (n == 1) {
            h[i] = 1.0e-10;
            continue;
        }
        double span = 0.0;
        for (int side = 0; side < 2; ++side) {
            if ((side == 0 && i == 0) || (side == 1 && i + 1 >= n)) continue;
            const double nb = a[side == 0 ? i - 1 : i + 1];
            double d;
            if (kind == 0) d = std::fabs(std::log(a[i] / nb));
            else if (kind == 1) d = std::fabs(a[i] - nb);
            else d = periodic_distance(a[i], nb);
            span = std::fmax(span, d);
        }
        h[i] = 0.500001 * span;
    }
}

// Strictly increasing with a relative gap above 1e-12 (so that the staged
// binary search and the reference's nearest-value scans pick the same cell).
inline bool well_separated_increasing(const double* a, size_t n) {
    for (size_t i = 1; i < n; ++i) {
        if (!(a[i] > a[i - 1])) return false;
        const double gap = a[i] - a[i - 1];
        const double mag = std::fmax(std::fabs(a[i]), std::fabs(a[i - 1]));
        if (!(gap > 1e-12 * mag)) return false;
    }
    return true;
}

// The per-axis conditions of a stageable separable grid (the cell-by-cell
// outer-product check is the caller's).
inline bool axes_stageable(const double* ra, size_t nr, const double* ta, size_t nth, const double* pa, size_t nph) {
    return nr && nth && nph && well_separated_increasing(ra, nr) && well_separated_increasing(ta, nth) &&
           well_separated_increasing(pa, nph) && ra[0] > 0.0 && pa[0] >= 0.0 && pa[nph - 1] < 2.0 * kPi;
}

// Radii outside [lo, hi] fail within_radial_cell (scattering.hpp:100-117) for
// every cell (margin 0.6 > 0.500001 of the outermost log spacing), so a
// lookup can stop early.  lo = 0, hi = inf when there is no such bound.
inline void radial_reject_bounds(const double* ra, size_t nr, double* lo, double* hi) {
    *lo = 0.0;
    *hi = INFINITY;
    if (nr >= 2) {
        const double span_lo = std::fabs(std::log(ra[0] / ra[1]));
        const double span_hi = std::fabs(std::log(ra[nr - 1] / ra[nr - 2]));
        *lo = ra[0] * std::exp(-0.6 * span_lo);
        *hi = ra[nr - 1] * std::exp(0.6 * span_hi);
    }
}

}  // namespace axes
}  // namespace grt
