// Device-side pieces of the per-photon hot path shared by the trace kernels:
// counter-based RNG, nonuniform-grid cell lookup, fluid sampling + tetrad,
// radiative transfer, scattering, packet generators and the camera test.
//
// Each function names the reference function it replaces (file:line within the
// reference project).  Floating-point expressions keep the reference's
// association so the FP64 parity kernel (built with -fmad=false) rounds like
// the reference; differences can come only from libdevice vs glibc in log,
// acos, atan2, exp and pow, which are called, never re-implemented.
#pragma once

#include <stdint.h>

#include "grt_kparams.h"
#include "grt_metric.cuh"
#include "grt_sincos.h"
#include "grt_user_physics.h"

namespace grt {
namespace dev {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11), key = 64-bit seed,
// counter = {id_lo, id_hi, domain, block}.  Each block gives four words = two
// doubles in [0,1) with 53 random bits.  One stream per (photon id, host step),
// which replaces the reference's Kokkos::Random_XorShift64_Pool
// (src/radiative_transfer/scattering.hpp:16-17) with a reproducible generator.
// ---------------------------------------------------------------------------
struct Philox {
    uint32_t k0, k1, c0, c1, c2, c3;
    uint32_t w[4];
    int used;

    GRT_DEV Philox(uint64_t seed, uint64_t id, uint32_t domain)
        : k0(static_cast<uint32_t>(seed)), k1(static_cast<uint32_t>(seed >> 32)),
          c0(static_cast<uint32_t>(id)), c1(static_cast<uint32_t>(id >> 32)), c2(domain), c3(0),
          used(4) {}

    static GRT_DEV void block(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3, uint32_t key0,
                              uint32_t key1, uint32_t out[4]) {
#pragma unroll
        for (int round = 0; round < 10; ++round) {
            const uint32_t hi0 = __umulhi(0xD2511F53u, x0), lo0 = 0xD2511F53u * x0;
            const uint32_t hi1 = __umulhi(0xCD9E8D57u, x2), lo1 = 0xCD9E8D57u * x2;
            x0 = hi1 ^ x1 ^ key0;
            x1 = lo1;
            x2 = hi0 ^ x3 ^ key1;
            x3 = lo0;
            key0 += 0x9E3779B9u;
            key1 += 0xBB67AE85u;
        }
        out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
    }

    GRT_DEV double drand() {
        if (used >= 4) {
            block(c0, c1, c2, c3, k0, k1, w);
            ++c3;
            used = 0;
        }
        const uint64_t hi = used == 0 ? w[0] : w[2];
        const uint64_t lo = used == 0 ? w[1] : w[3];
        used += 2;
        return static_cast<double>((hi << 21) | (lo >> 11)) * (1.0 / 9007199254740992.0);
    }
};
constexpr uint32_t kInitDomain = 0xFFFFFFFFu;    // disk-mode emission draws
constexpr uint32_t kScreenDomain = 0xFFFFFFFEu;  // image-mode random screen (u, v)

// ---------------------------------------------------------------------------
// Nonuniform (r, theta, phi) grid lookup (scattering.hpp:41-180)
// ---------------------------------------------------------------------------

// scattering.hpp:41-45
GRT_DEV double periodic_angle_distance(double lhs, double rhs) {
    const double d = fmod(fabs(lhs - rhs), 2.0 * kPi);
    return fmin(d, 2.0 * kPi - d);
}

// Separable sorted axes: the reference's linear argmin with strict '<'
// (first index wins ties, scattering.hpp:55-63,73-79,89-95) computed from the
// bracketing pair found by binary search.  Valid because the distance to a
// sorted axis is monotone on each side of the query (division and log are
// monotone); the host only enables this path when every axis is strictly
// increasing with neighbouring values separated by more than 1e-12 relative,
// which rules out equal distances at non-adjacent indices.
GRT_DEV int bracket(const double* axis, int n, double q) {
    int lo = -1, hi = n;  // axis[lo] <= q < axis[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (axis[mid] <= q) lo = mid; else hi = mid;
    }
    return lo;
}

GRT_DEV int nearest_radial_sorted(const double* r, int n, double radius) {
    const int lo = bracket(r, n, radius);
    if (lo < 0) return 0;
    if (lo + 1 >= n) return lo;
    const double dlo = fabs(log(radius / r[lo]));
    const double dhi = fabs(log(radius / r[lo + 1]));
    return dhi < dlo ? lo + 1 : lo;
}

GRT_DEV int nearest_polar_sorted(const double* th, int n, double polar) {
    const int lo = bracket(th, n, polar);
    if (lo < 0) return 0;
    if (lo + 1 >= n) return lo;
    const double dlo = fabs(polar - th[lo]);
    const double dhi = fabs(polar - th[lo + 1]);
    return dhi < dlo ? lo + 1 : lo;
}

// periodic_angle_distance for |lhs - rhs| <= 4 pi: fmod(v, 2 pi) is v, or
// exactly v - 2 pi (Sterbenz) for v in [2 pi, 4 pi).  The separable path has
// azimuth queries in [0, 2 pi] and axis values in [0, 2 pi).
GRT_DEV double periodic_angle_distance_near(double lhs, double rhs) {
    const double v = fabs(lhs - rhs);
    const double d = v >= 2.0 * kPi ? v - 2.0 * kPi : v;
    return fmin(d, 2.0 * kPi - d);
}

GRT_DEV int nearest_azimuth_sorted(const double* ph, int n, double az) {
    if (n == 1) return 0;
    const int lo = bracket(ph, n, az);
    const int c1 = lo < 0 ? n - 1 : lo;
    const int c2 = lo + 1 < n ? lo + 1 : 0;
    const double d1 = periodic_angle_distance_near(az, ph[c1]);
    const double d2 = periodic_angle_distance_near(az, ph[c2]);
    if (d1 < d2) return c1;
    if (d2 < d1) return c2;
    return c1 < c2 ? c1 : c2;
}

// scattering.hpp:99-149 on one separable axis, with the neighbour half-span
// precomputed per axis value (see KGrid::r_half).
GRT_DEV bool within_radial_sorted(const double* r, const double* half, int i, double radius) {
    return fabs(log(radius / r[i])) <= half[i];
}

// nearest_radial_sorted and within_radial_sorted in one pass: the log
// distance of the chosen cell is the one the nearest-cell test computed, so it
// is evaluated once per candidate (one or two), through one site.  Ties go to
// the lower index, as in nearest_radial_sorted.
GRT_DEV bool locate_radial_sorted(const double* r, const double* half, int n, double radius, int& i) {
    const int lo = bracket(r, n, radius);
    const int c0 = lo < 0 ? 0 : lo;
    const int ncand = (lo >= 0 && lo + 1 < n) ? 2 : 1;
    double best = 0.0;
    int bi = c0;
#pragma unroll 1
    for (int k = 0; k < ncand; ++k) {
        const double d = fabs(log(radius / r[c0 + k]));
        if (k == 0 || d < best) {
            best = d;
            bi = c0 + k;
        }
    }
    i = bi;
    return best <= half[bi];
}
GRT_DEV bool within_polar_sorted(const double* th, const double* half, int j, double polar) {
    return fabs(polar - th[j]) <= half[j];
}
GRT_DEV bool within_azimuth_sorted(const double* ph, const double* half, int k, double az) {
    return periodic_angle_distance_near(az, ph[k]) <= half[k];
}

// General (non-separable) coordinates: the reference's three coordinate-descent
// passes of linear scans over the full 3-D coordinate arrays
// (scattering.hpp:151-180), used when the grid is not separable.
struct Grid3 {
    const double* r;
    const double* th;
    const double* ph;
    int nr, nth, nph;
    GRT_DEV size_t at(int i, int j, int k) const {
        return (static_cast<size_t>(i) * nth + j) * nph + k;
    }
};

static __device__ __noinline__ bool locate_general(const Grid3& g, double radius, double polar, double az, int& i, int& j,
                            int& k) {
    j = g.nth / 2;
    k = g.nph / 2;
    i = g.nr / 2;
    for (int it = 0; it < 3; ++it) {
        {  // nearest_radial_index
            const double first = g.r[g.at(0, j, k)];
            if (!(first > 0.0)) return false;
            int best_i = 0;
            double best = fabs(log(radius / first));
            for (int q = 1; q < g.nr; ++q) {
                const double c = g.r[g.at(q, j, k)];
                if (!(c > 0.0)) continue;
                const double d = fabs(log(radius / c));
                if (d < best) { best_i = q; best = d; }
            }
            i = best_i;
        }
        {  // nearest_polar_index
            int best_j = 0;
            double best = fabs(polar - g.th[g.at(i, 0, k)]);
            for (int q = 1; q < g.nth; ++q) {
                const double d = fabs(polar - g.th[g.at(i, q, k)]);
                if (d < best) { best_j = q; best = d; }
            }
            j = best_j;
        }
        {  // nearest_azimuth_index
            int best_k = 0;
            double best = periodic_angle_distance(az, g.ph[g.at(i, j, 0)]);
            for (int q = 1; q < g.nph; ++q) {
                const double d = periodic_angle_distance(az, g.ph[g.at(i, j, q)]);
                if (d < best) { best_k = q; best = d; }
            }
            k = best_k;
        }
    }
    {  // within_radial_cell
        const double center = g.r[g.at(i, j, k)];
        if (!(center > 0.0)) return false;
        const double cd = fabs(log(radius / center));
        if (g.nr == 1) {
            if (!(cd <= 1.0e-10)) return false;
        } else {
            double span = 0.0;
            if (i > 0 && g.r[g.at(i - 1, j, k)] > 0.0)
                span = fmax(span, fabs(log(center / g.r[g.at(i - 1, j, k)])));
            if (i + 1 < g.nr && g.r[g.at(i + 1, j, k)] > 0.0)
                span = fmax(span, fabs(log(center / g.r[g.at(i + 1, j, k)])));
            if (!(cd <= 0.500001 * span)) return false;
        }
    }
    {  // within_polar_cell
        const double center = g.th[g.at(i, j, k)];
        const double cd = fabs(polar - center);
        if (g.nth == 1) {
            if (!(cd <= 1.0e-10)) return false;
        } else {
            double span = 0.0;
            if (j > 0) span = fmax(span, fabs(center - g.th[g.at(i, j - 1, k)]));
            if (j + 1 < g.nth) span = fmax(span, fabs(center - g.th[g.at(i, j + 1, k)]));
            if (!(cd <= 0.500001 * span)) return false;
        }
    }
    {  // within_azimuth_cell
        const double center = g.ph[g.at(i, j, k)];
        const double cd = periodic_angle_distance(az, center);
        if (g.nph == 1) {
            if (!(cd <= 1.0e-10)) return false;
        } else {
            double span = 0.0;
            if (k > 0) span = fmax(span, periodic_angle_distance(center, g.ph[g.at(i, j, k - 1)]));
            if (k + 1 < g.nph) span = fmax(span, periodic_angle_distance(center, g.ph[g.at(i, j, k + 1)]));
            if (!(cd <= 0.500001 * span)) return false;
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// Fluid sample + tetrad (scattering.hpp:185-251, fluid_frame.hpp:51-80)
// ---------------------------------------------------------------------------
struct FluidSample {
    FluidCellCGS fluid;
    double e[4][4];  // tetrad, e[0] = fluid four-velocity
    int cell;
};

// fluid_frame.hpp:51-80 with the metric already evaluated at the photon.
GRT_DEV bool build_tetrad(const double g[4][4], const double u[4], double e[4][4]) {
    const double vn = metric_dot(g, u, u);
    if (!(vn < 0.0) || !isfinite(vn)) return false;
    const double inv = 1.0 / sqrt(-vn);
    const double ts = u[0] >= 0.0 ? 1.0 : -1.0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) e[0][mu] = ts * u[mu] * inv;
    // Rolled over the spatial axes (one square-root and one division site):
    // the tetrad is built on every fluid sample, so its code stays small.
#pragma unroll 1
    for (int axis = 0; axis < 3; ++axis) {
        double cand[4];
        const double tp = metric_dot_unit(g, e[0], axis + 1);
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) cand[mu] = (mu == axis + 1 ? 1.0 : 0.0) + tp * e[0][mu];
#pragma unroll 1
        for (int prev = 0; prev < axis; ++prev) {
            const double proj = metric_dot(g, e[prev + 1], cand);
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) cand[mu] -= proj * e[prev + 1][mu];
        }
        const double n = metric_dot(g, cand, cand);
        if (!(n > 1.0e-20) || !isfinite(n)) return false;
        const double is = 1.0 / sqrt(n);
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) e[axis + 1][mu] = cand[mu] * is;
    }
    return true;
}

// sample_scattering_fluid (scattering.hpp:185-251).  `radius` is
// compute_r(x, y, z, spin) of the state, which the caller has already.
// Cartesian velocity / magnetic four-vectors per cell are precomputed on the
// host with the reference's transform (fluid_frame.hpp:28-48) and unit scale,
// so the per-step arithmetic is exactly the reference's.
// fluid_frame.hpp:28-48 on the device, times the [units] scale (raw layout only).
GRT_DEV void spherical_to_cartesian_scaled(double r, double th, double ph, double spin, const double* sv,
                                          double scale, double c[4]) {
    double st, ct, sp, cp;
    sincos(th, &st, &ct);
    sincos(ph, &sp, &cp);
    const double radial_x = cp * st, radial_y = sp * st, radial_z = ct;
    const double theta_x = (r * cp - spin * sp) * ct;
    const double theta_y = (r * sp + spin * cp) * ct;
    const double theta_z = -r * st;
    const double phi_x = (-r * sp - spin * cp) * st;
    const double phi_y = (r * cp - spin * sp) * st;
    c[0] = sv[0] * scale;
    c[1] = (radial_x * sv[1] + theta_x * sv[2] + phi_x * sv[3]) * scale;
    c[2] = (radial_y * sv[1] + theta_y * sv[2] + phi_y * sv[3]) * scale;
    c[3] = (radial_z * sv[1] + theta_z * sv[2]) * scale;
}

// RAW selects the grid layout: false -- packed (rho, T) pairs and Cartesian
// four-vectors precomputed on the host; true -- the reference's raw arrays,
// with the spherical-to-Cartesian conversion done per sample.
// Separable axes and their half-spans staged in shared memory.
struct Axes {
    const double* r;
    const double* th;
    const double* ph;
    const double* rh;
    const double* thh;
    const double* phh;
};

template <bool RAW>
static __device__ __noinline__ bool sample_fluid_at(const KParams& kp, const Axes ax, double t, double x,
                                                    double y, double z, double radius, FluidSample* outp) {
    FluidSample& out = *outp;
    const double s[4] = {t, x, y, z};
    const KGrid& G = kp.grid;
    int i, j, k;
    if (G.separable) {
        if (!locate_radial_sorted(ax.r, ax.rh, G.nr, radius, i)) return false;
    }
    const double ct = fmax(-1.0, fmin(1.0, s[3] / radius));
    const double polar = acos(ct);
    double az = atan2(radius * s[2] - kp.a * s[1], radius * s[1] + kp.a * s[2]);
    if (az < 0.0) az += 2.0 * kPi;
    if (G.separable) {
        j = nearest_polar_sorted(ax.th, G.nth, polar);
        k = nearest_azimuth_sorted(ax.ph, G.nph, az);
        if (!within_polar_sorted(ax.th, ax.thh, j, polar) || !within_azimuth_sorted(ax.ph, ax.phh, k, az))
            return false;
    } else {
        const Grid3 g3{G.r3, G.th3, G.ph3, G.nr, G.nth, G.nph};
        if (!locate_general(g3, radius, polar, az, i, j, k)) return false;
    }
    const int cell = (i * G.nth + j) * G.nph + k;
    out.cell = cell;
    FluidCellCGS& f = out.fluid;
    f.position_cm[0] = s[1] * kp.length_scale;
    f.position_cm[1] = s[2] * kp.length_scale;
    f.position_cm[2] = s[3] * kp.length_scale;
    f.coordinate_time_s = s[0] * kp.time_scale;
    double cm[4];
    if (RAW) {
        f.density_g_cm3 = G.rho_raw[cell] * kp.density_scale;
        f.temperature_k = G.T_raw[cell] * kp.temperature_scale;
        if (!(f.density_g_cm3 > 0.0) || !isfinite(f.density_g_cm3) || !isfinite(f.temperature_k))
            return false;
        spherical_to_cartesian_scaled(G.r3[cell], G.th3[cell], G.ph3[cell], kp.a, G.vel_raw + 4 * cell,
                                      G.vel_scale, f.coordinate_four_velocity_cm_s);
        spherical_to_cartesian_scaled(G.r3[cell], G.th3[cell], G.ph3[cell], kp.a, G.mag_raw + 4 * cell,
                                      G.mag_scale, cm);
    } else {
        const double2 rt = G.rho_t[cell];
        f.density_g_cm3 = rt.x * kp.density_scale;
        f.temperature_k = rt.y * kp.temperature_scale;
        if (!(f.density_g_cm3 > 0.0) || !isfinite(f.density_g_cm3) || !isfinite(f.temperature_k))
            return false;
        const double2 u01 = G.vel[2 * cell], u23 = G.vel[2 * cell + 1];
        f.coordinate_four_velocity_cm_s[0] = u01.x;
        f.coordinate_four_velocity_cm_s[1] = u01.y;
        f.coordinate_four_velocity_cm_s[2] = u23.x;
        f.coordinate_four_velocity_cm_s[3] = u23.y;
        const double2 b01 = G.mag[2 * cell], b23 = G.mag[2 * cell + 1];
        cm[0] = b01.x; cm[1] = b01.y; cm[2] = b23.x; cm[3] = b23.y;
    }
    MetricAt m;
    ks_metric_from_r(s[1], s[2], s[3], radius, kp.a, kp.M, m);
    if (!build_tetrad(m.g, f.coordinate_four_velocity_cm_s, out.e)) return false;
    f.magnetic_gauss[0] = -metric_dot(m.g, out.e[0], cm);
#pragma unroll
    for (int axis = 1; axis < 4; ++axis) f.magnetic_gauss[axis] = metric_dot(m.g, out.e[axis], cm);
    return true;
}

// sample_scattering_fluid (scattering.hpp:185-251): the cheap early-outs
// inline, the lookup + gather + tetrad out of line.
template <bool RAW = false>
GRT_DEV bool sample_fluid(const KParams& kp, const Axes& ax, const double s[8], double radius, FluidSample& out) {
    const KGrid& G = kp.grid;
    if (!G.available) return false;
    if (!(radius > 0.0) || !isfinite(radius)) return false;
    if (radius < G.r_reject_lo || radius > G.r_reject_hi) return false;
    return sample_fluid_at<RAW>(kp, ax, s[0], s[1], s[2], s[3], radius, &out);
}

// ---------------------------------------------------------------------------
// Scattering and packet generation
// ---------------------------------------------------------------------------
constexpr double kProtonMassCgs = 1.67262192369e-24;   // scattering.hpp:256
constexpr double kSigmaThomsonCgs = 6.6524587158e-25;  // scattering.hpp:257

// State a scattering event may change, passed by copy to the out-of-line
// scatter_packet so the caller's state never has its address taken (which
// would keep it in local memory for the whole trace loop).
struct ScatterState {
    double s[8];
    double I[4];
};

// maybe_scatter_photon (scattering.hpp:259-313) in two parts.  scatter_drawn is the
// part every sampled step takes, inline: the Thomson optical depth over the
// proposed step and the first draw; it says whether the packet scatters.
GRT_DEV bool scatter_drawn(double dl, double length_scale, const FluidSample& fs, Philox& rng) {
    const double path_cm = dl * length_scale;
    const double ne = fs.fluid.density_g_cm3 / kProtonMassCgs;
    const double tau = kSigmaThomsonCgs * ne * path_cm;
    const double prob = 1.0 - exp(-tau);
    return !(rng.drand() >= prob);  // the reference's rejection test, NaN included
}

// The rest, out of line and only for a packet that scatters: the isotropic
// fluid-frame direction (two more draws), the new covariant momentum and the
// albedo weights; false leaves the state as it was.
static __device__ __noinline__ bool scatter_packet(ScatterState* st, double albedo, const FluidSample& fs, double a,
                                                   double M, Philox* rngp) {
    Philox& rng = *rngp;
    double* s = st->s;
    double* I = st->I;
    double E = 0.0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) E -= s[4 + mu] * fs.e[0][mu];
    if (!(E > 0.0) || !isfinite(E)) return false;
    const double mu_c = 2.0 * rng.drand() - 1.0;
    const double dphi = 2.0 * kPi * rng.drand();
    const double tr = sqrt(fmax(0.0, 1.0 - mu_c * mu_c));
    double sn, cs;
    det_sincos(dphi, &sn, &cs);  // the oracle's sin/cos bit for bit (grt_sincos.h)
    const double dx = tr * cs, dy = tr * sn, dz = mu_c;
    double w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) w[q] = fs.e[0][q] + dx * fs.e[1][q] + dy * fs.e[2][q] + dz * fs.e[3][q];
    MetricAt m;
    ks_metric(s[1], s[2], s[3], a, M, m);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double pq = 0.0;
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) pq += m.g[q][nu] * w[nu];
        s[4 + q] = E * pq;
    }
    I[0] *= albedo;
    I[1] *= 0.5 * albedo;
    I[2] *= 0.5 * albedo;
    I[3] *= 0.25 * albedo;
    return true;
}

// GenerateBlackbody (photon_generation.hpp:99-124): Planck spectrum as a
// mixture of Gamma(4, n) with weights 1/n^4; the four product draws are taken
// in order.
static __device__ __noinline__ bool generate_blackbody(const FluidCellCGS& cell, Philox& rng, int packets, double energy,
                                double& nu, double& E) {
    if (!(cell.temperature_k > 0.0)) return false;
    const double inverse_zeta4 = 0.9239384029215902;
    const double choose = rng.drand();
    double cumulative = 0.0;
    int m = 1;
    for (; m < 64; ++m) {
        const double n = static_cast<double>(m);
        cumulative += inverse_zeta4 / (n * n * n * n);
        if (choose <= cumulative) break;
    }
    const double d1 = rng.drand(), d2 = rng.drand(), d3 = rng.drand(), d4 = rng.drand();
    const double product = fmax(1.0e-300, d1 * d2 * d3 * d4);
    const double x = -log(product) / static_cast<double>(m);
    nu = x * 2.0836619123327576e10 * cell.temperature_k;
    E = energy / static_cast<double>(packets);
    return isfinite(nu) && nu > 0.0;
}

// GeneratePowerLaw (photon_generation.hpp:126-143)
static __device__ __noinline__ bool generate_power_law(Philox& rng, int packets, double slope, double nu_min, double nu_max,
                                double energy, double& nu, double& E) {
    const double draw = rng.drand();
    if (fabs(slope - 1.0) < 1.0e-12) {
        nu = nu_min * pow(nu_max / nu_min, draw);
    } else {
        const double ex = 1.0 - slope;
        const double lo = pow(nu_min, ex);
        const double hi = pow(nu_max, ex);
        nu = pow(lo + draw * (hi - lo), 1.0 / ex);
    }
    E = energy / static_cast<double>(packets);
    return isfinite(nu) && nu > 0.0;
}

// ---------------------------------------------------------------------------
// Camera (integrate_cart_ks.hpp:96-130); the plane basis is precomputed on the host.
// ---------------------------------------------------------------------------
GRT_DEV int camera_crossing(const KImage& im, const double s[8], double& u, double& v) {
    const double pc = s[1] * im.cam_n[0] + s[2] * im.cam_n[1] + s[3] * im.cam_n[2];
    if (pc < im.cam_D) return 0;
    const double rel0 = s[1] - im.cam_D * im.cam_n[0];
    const double rel1 = s[2] - im.cam_D * im.cam_n[1];
    const double rel2 = s[3] - im.cam_D * im.cam_n[2];
    u = rel0 * im.cam_th[0] + rel1 * im.cam_th[1] + rel2 * im.cam_th[2];
    v = rel0 * im.cam_ph[0] + rel1 * im.cam_ph[1] + rel2 * im.cam_ph[2];
    const bool inside = fabs(u) <= 0.5 * im.cam_W && fabs(v) <= 0.5 * im.cam_H;
    return inside ? 1 : -1;
}

static __device__ __noinline__ double camera_observer_energy_at(double a, double M, double x, double y, double z,
                                                                double pt) {
    MetricAt m;
    ks_metric(x, y, z, a, M, m);
    if (!(m.g[0][0] < 0.0)) return 0.0;
    const double u0 = 1.0 / sqrt(-m.g[0][0]);
    return -pt * u0;
}

GRT_DEV double camera_observer_energy(const KParams& kp, const double s[8]) {
    return camera_observer_energy_at(kp.a, kp.M, s[1], s[2], s[3], s[4]);
}

}  // namespace dev
}  // namespace grt
