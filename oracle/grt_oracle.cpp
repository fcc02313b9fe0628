// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the GR-ray-tracer per-photon hot path, used by the tests,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker for
// the sm_100a kernels.  The product never links or calls this file.
//
// Every function restates one reference function, cited by file:line within
// the reference project, and keeps the reference's order of floating-point
// operations (built with -ffp-contract=off) so that its results can be compared
// with the CUDA kernels at round-off level.  Randomness uses the same
// counter-based Philox4x32-10 streams as the kernels (written independently
// here from the published algorithm of Salmon et al., SC'11), so RNG-dependent
// paths are compared draw for draw; the reference's own Kokkos XorShift64
// streams cannot be reproduced and are compared in distribution instead.
//
// The user-editable extension points are taken from the product header
// grt_user_physics.h, exactly as a user's edit would reach both sides.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "grt.h"
#include "grt_pow_quarter.cuh"  // the kernels' controller root, checked below against std::pow
#include "grt_sincos.h"        // deterministic sin/cos shared with the kernels (scattering directions)
#include "grt_user_physics.h"

namespace oracle {

using real = double;

// How the RK45 controller evaluates pow(1/err, 0.25)
// (src/geodesic_integrate/integrate_cart_ks.hpp:217):
//   0 = std::pow, i.e. glibc, exactly like the reference's host build (default);
//   1 = grt::pow_quarter, the kernels' restatement of glibc's pow compiled for
//       the host (grt_pow_quarter.cuh), to show whole runs agree either way.
int g_pow_mode = 0;

real controller_root(real x) { return g_pow_mode == 1 ? grt::pow_quarter(x) : std::pow(x, real(0.25)); }
using grt::FluidCellCGS;

constexpr real PI = 3.14159265358979323846;  // src/utils.hpp:16
constexpr int IT = 0, IX = 1, IY = 2, IZ = 3, IKT = 4, IKX = 5, IKY = 6, IKZ = 7;

inline real SQR(real x) { return x * x; }            // src/utils.hpp:31-36
inline real CUBE(real x) { return x * x * x; }
inline real QUAD(real x) { return x * x * x * x; }

// ---------------------------------------------------------------------------
// Kerr-Schild metric core (src/metrics/kerr_schild_core.hpp)
// ---------------------------------------------------------------------------

// kerr_schild_core.hpp:27-33
real compute_r(real x, real y, real z, real a) {
    const real rsq = SQR(x) + SQR(y) + SQR(z);
    const real A = rsq - SQR(a);
    const real S = std::sqrt(SQR(A) + 4.0 * SQR(a * z));
    return std::sqrt(0.5 * (A + S));
}

// kerr_schild_core.hpp:36-46
void compute_r_and_deriv(real x, real y, real z, real a, real& r, real dr[3]) {
    const real rsq = SQR(x) + SQR(y) + SQR(z);
    const real A = rsq - SQR(a);
    const real S = std::sqrt(SQR(A) + 4.0 * SQR(a * z));
    r = std::sqrt(0.5 * (A + S));
    const real one_plus_A_over_S = 1.0 + A / S;
    dr[0] = x * one_plus_A_over_S / (2.0 * r);
    dr[1] = y * one_plus_A_over_S / (2.0 * r);
    dr[2] = (z * one_plus_A_over_S + 2.0 * SQR(a) * z / S) / (2.0 * r);
}

// kerr_schild_core.hpp:49-56
void compute_l(real x, real y, real z, real r, real a, real l[4]) {
    const real B = SQR(r) + SQR(a);
    l[0] = 1.0;
    l[1] = (r * x + a * y) / B;
    l[2] = (r * y - a * x) / B;
    l[3] = z / r;
}

// kerr_schild_core.hpp:58-77
void compute_l_and_deriv(real x, real y, real z, real r, const real dr[3], real a,
                         real l[4], real dl[3][4]) {
    const real B = SQR(r) + SQR(a);
    l[0] = 1.0;
    l[1] = (r * x + a * y) / B;
    l[2] = (r * y - a * x) / B;
    l[3] = z / r;
    for (int k = 0; k < 3; ++k) {
        const real dx_dk = (k == 0) ? 1.0 : 0.0;
        const real dy_dk = (k == 1) ? 1.0 : 0.0;
        const real dz_dk = (k == 2) ? 1.0 : 0.0;
        const real dB_dk = 2.0 * r * dr[k];
        dl[k][0] = 0.0;
        dl[k][1] = ((dr[k] * x + r * dx_dk) + a * dy_dk - l[1] * dB_dk) / B;
        dl[k][2] = ((dr[k] * y + r * dy_dk) - a * dx_dk - l[2] * dB_dk) / B;
        dl[k][3] = (dz_dk - l[3] * dr[k]) / r;
    }
}

// kerr_schild_core.hpp:79-83
real compute_H(real r, real z, real a, real M) {
    const real D = QUAD(r) + SQR(a * z);
    return M * CUBE(r) / D;
}

// kerr_schild_core.hpp:85-95
real compute_H_and_deriv(real r, real z, const real dr[3], real a, real M, real dH[3]) {
    const real D = QUAD(r) + SQR(a * z);
    const real H = M * CUBE(r) / D;
    for (int k = 0; k < 3; ++k) {
        const real dz_dk = (k == 2) ? 1.0 : 0.0;
        const real dD_dk = 4.0 * CUBE(r) * dr[k] + 2.0 * SQR(a) * z * dz_dk;
        dH[k] = M * (3.0 * SQR(r) * dr[k] * D - CUBE(r) * dD_dk) / SQR(D);
    }
    return H;
}

// kerr_schild_core.hpp:98-110
void compute_metric(const real X[4], real a, real M, real g[4][4]) {
    const real r = compute_r(X[1], X[2], X[3], a);
    real l[4];
    compute_l(X[1], X[2], X[3], r, a, l);
    const real H = compute_H(r, X[3], a, M);
    const real eta[4] = {-1.0, 1.0, 1.0, 1.0};
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu)
            g[mu][nu] = 2.0 * H * l[mu] * l[nu] + ((mu == nu) ? eta[mu] : 0.0);
}

// kerr_schild_core.hpp:113-126
void compute_inverse_metric(const real X[4], real a, real M, real ginv[4][4]) {
    const real r = compute_r(X[1], X[2], X[3], a);
    real l[4];
    compute_l(X[1], X[2], X[3], r, a, l);
    const real lup[4] = {-l[0], l[1], l[2], l[3]};
    const real H = compute_H(r, X[3], a, M);
    const real eta[4] = {-1.0, 1.0, 1.0, 1.0};
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu)
            ginv[mu][nu] = -2.0 * H * lup[mu] * lup[nu] + ((mu == nu) ? eta[mu] : 0.0);
}

// kerr_schild_core.hpp:130-155
void compute_inverse_metric_deriv(const real X[4], real a, real M, real dginv[4][4][4]) {
    real r, dr[3];
    compute_r_and_deriv(X[1], X[2], X[3], a, r, dr);
    real l[4], dl[3][4];
    compute_l_and_deriv(X[1], X[2], X[3], r, dr, a, l, dl);
    real dH[3];
    const real H = compute_H_and_deriv(r, X[3], dr, a, M, dH);
    const real lup[4] = {-l[0], l[1], l[2], l[3]};
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu) dginv[0][mu][nu] = 0.0;
    for (int k = 0; k < 3; ++k) {
        const real dlup[4] = {-dl[k][0], dl[k][1], dl[k][2], dl[k][3]};
        for (int mu = 0; mu < 4; ++mu)
            for (int nu = 0; nu < 4; ++nu)
                dginv[k + 1][mu][nu] =
                    -2.0 * (dH[k] * lup[mu] * lup[nu] + H * (dlup[mu] * lup[nu] + lup[mu] * dlup[nu]));
    }
}

// kerr_schild_core.hpp:157-192: Hamilton's equations for covariant p_mu.
void hamiltonian_rhs(const real X[4], const real p[4], real a, real M, real rhs[8]) {
    real r, dr[3];
    compute_r_and_deriv(X[1], X[2], X[3], a, r, dr);
    real l[4], dl[3][4];
    compute_l_and_deriv(X[1], X[2], X[3], r, dr, a, l, dl);
    real dH[3];
    const real H = compute_H_and_deriv(r, X[3], dr, a, M, dH);
    const real lup[4] = {-l[0], l[1], l[2], l[3]};
    real l_dot_p = 0.0;
    for (int mu = 0; mu < 4; ++mu) l_dot_p += lup[mu] * p[mu];
    rhs[0] = -p[0] - 2.0 * H * lup[0] * l_dot_p;
    for (int mu = 1; mu < 4; ++mu) rhs[mu] = p[mu] - 2.0 * H * lup[mu] * l_dot_p;
    rhs[IKT] = 0.0;
    for (int k = 0; k < 3; ++k) {
        const real dlup[4] = {-dl[k][0], dl[k][1], dl[k][2], dl[k][3]};
        real dl_dot_p = 0.0;
        for (int mu = 0; mu < 4; ++mu) dl_dot_p += dlup[mu] * p[mu];
        rhs[IKX + k] = dH[k] * SQR(l_dot_p) + 2.0 * H * l_dot_p * dl_dot_p;
    }
}

// kerr_schild_core.hpp:200-227
bool null_covariant_momentum(const real X[4], const real K[3], real a, real M, real p[4]) {
    real g[4][4];
    compute_metric(X, a, M, g);
    const real qa = g[0][0];
    const real qb = 2.0 * (g[0][1] * K[0] + g[0][2] * K[1] + g[0][3] * K[2]);
    real qc = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) qc += g[i + 1][j + 1] * K[i] * K[j];
    const real disc = SQR(qb) - 4.0 * qa * qc;
    if (disc < 0.0) return false;
    const real sq = std::sqrt(disc);
    const real K0_1 = (-qb + sq) / (2.0 * qa);
    const real K0_2 = (-qb - sq) / (2.0 * qa);
    const real K0 = (K0_1 > 0.0) ? K0_1 : K0_2;
    if (!(K0 > 0.0)) return false;
    const real Kc[4] = {K0, K[0], K[1], K[2]};
    for (int mu = 0; mu < 4; ++mu) {
        real sum = 0.0;
        for (int nu = 0; nu < 4; ++nu) sum += g[mu][nu] * Kc[nu];
        p[mu] = sum;
    }
    return true;
}

// src/metrics/cartesian_kerr_schild.hpp:10-21
real kerr_schild_norm(const real X[4], const real V[4], real a, real M) {
    real g[4][4];
    compute_inverse_metric(X, a, M, g);
    real n = 0.0;
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu) n += g[mu][nu] * V[mu] * V[nu];
    return n;
}

// ---------------------------------------------------------------------------
// Counter-based RNG: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
// Stream (key = seed, counter = {id_lo, id_hi, domain, block}); each block
// gives four 32-bit words = two doubles in [0,1) with 53 random bits.
// ---------------------------------------------------------------------------
struct Philox {
    uint32_t key[2];
    uint32_t ctr[4];
    uint32_t out[4];
    int used = 4;

    static void block(const uint32_t in[4], const uint32_t k_in[2], uint32_t res[4]) {
        uint32_t c0 = in[0], c1 = in[1], c2 = in[2], c3 = in[3];
        uint32_t k0 = k_in[0], k1 = k_in[1];
        for (int round = 0; round < 10; ++round) {
            const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
            const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
            const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
            const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
            c0 = hi1 ^ c1 ^ k0;
            c1 = lo1;
            c2 = hi0 ^ c3 ^ k1;
            c3 = lo0;
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        res[0] = c0; res[1] = c1; res[2] = c2; res[3] = c3;
    }

    Philox(uint64_t seed, uint64_t id, uint32_t domain) {
        key[0] = static_cast<uint32_t>(seed);
        key[1] = static_cast<uint32_t>(seed >> 32);
        ctr[0] = static_cast<uint32_t>(id);
        ctr[1] = static_cast<uint32_t>(id >> 32);
        ctr[2] = domain;
        ctr[3] = 0;
    }
    double drand() {
        if (used >= 4) {
            block(ctr, key, out);
            ++ctr[3];
            used = 0;
        }
        const uint64_t hi = out[used], lo = out[used + 1];
        used += 2;
        const uint64_t bits = (hi << 21) | (lo >> 11);
        return static_cast<double>(bits) * (1.0 / 9007199254740992.0);
    }
};
constexpr uint32_t kInitDomain = 0xFFFFFFFFu;

// ---------------------------------------------------------------------------
// Fluid grid sampling (src/radiative_transfer/scattering.hpp,
// src/radiative_transfer/fluid_frame.hpp)
// ---------------------------------------------------------------------------
struct Grid {
    size_t nr = 0, nth = 0, nph = 0;
    const real* r = nullptr;
    const real* th = nullptr;
    const real* ph = nullptr;
    const real* rho = nullptr;
    const real* T = nullptr;
    const real* vel = nullptr;
    const real* mag = nullptr;
    real length_scale = 1, time_scale = 1, density_scale = 1, temperature_scale = 1,
         velocity_scale = 1, magnetic_scale = 1;
    real spin = 0, mass = 1;
    bool available = false;
    size_t at(size_t i, size_t j, size_t k) const { return (i * nth + j) * nph + k; }
};

// scattering.hpp:41-45
real periodic_angle_distance(real lhs, real rhs) {
    real d = std::fmod(std::fabs(lhs - rhs), 2.0 * PI);
    return std::fmin(d, 2.0 * PI - d);
}

// scattering.hpp:47-65
int nearest_radial_index(const Grid& g, real radius, int j, int k) {
    if (g.nr == 0 || !(radius > 0.0)) return -1;
    int nearest = 0;
    const real first = g.r[g.at(0, j, k)];
    if (!(first > 0.0)) return -1;
    real best = std::fabs(std::log(radius / first));
    for (size_t i = 1; i < g.nr; ++i) {
        const real c = g.r[g.at(i, j, k)];
        if (!(c > 0.0)) continue;
        const real d = std::fabs(std::log(radius / c));
        if (d < best) { nearest = static_cast<int>(i); best = d; }
    }
    return nearest;
}

// scattering.hpp:67-81
int nearest_polar_index(const Grid& g, real polar, int i, int k) {
    if (g.nth == 0) return -1;
    int nearest = 0;
    real best = std::fabs(polar - g.th[g.at(i, 0, k)]);
    for (size_t j = 1; j < g.nth; ++j) {
        const real d = std::fabs(polar - g.th[g.at(i, j, k)]);
        if (d < best) { nearest = static_cast<int>(j); best = d; }
    }
    return nearest;
}

// scattering.hpp:83-97
int nearest_azimuth_index(const Grid& g, real azimuth, int i, int j) {
    if (g.nph == 0) return -1;
    int nearest = 0;
    real best = periodic_angle_distance(azimuth, g.ph[g.at(i, j, 0)]);
    for (size_t k = 1; k < g.nph; ++k) {
        const real d = periodic_angle_distance(azimuth, g.ph[g.at(i, j, k)]);
        if (d < best) { nearest = static_cast<int>(k); best = d; }
    }
    return nearest;
}

// scattering.hpp:99-117
bool within_radial_cell(const Grid& g, real radius, int i, int j, int k) {
    const real center = g.r[g.at(i, j, k)];
    if (!(center > 0.0) || !(radius > 0.0)) return false;
    const real cd = std::fabs(std::log(radius / center));
    if (g.nr == 1) return cd <= 1.0e-10;
    real span = 0.0;
    if (i > 0 && g.r[g.at(i - 1, j, k)] > 0.0)
        span = std::fmax(span, std::fabs(std::log(center / g.r[g.at(i - 1, j, k)])));
    if (static_cast<size_t>(i + 1) < g.nr && g.r[g.at(i + 1, j, k)] > 0.0)
        span = std::fmax(span, std::fabs(std::log(center / g.r[g.at(i + 1, j, k)])));
    return cd <= 0.500001 * span;
}

// scattering.hpp:119-133
bool within_polar_cell(const Grid& g, real polar, int i, int j, int k) {
    const real center = g.th[g.at(i, j, k)];
    const real cd = std::fabs(polar - center);
    if (g.nth == 1) return cd <= 1.0e-10;
    real span = 0.0;
    if (j > 0) span = std::fmax(span, std::fabs(center - g.th[g.at(i, j - 1, k)]));
    if (static_cast<size_t>(j + 1) < g.nth)
        span = std::fmax(span, std::fabs(center - g.th[g.at(i, j + 1, k)]));
    return cd <= 0.500001 * span;
}

// scattering.hpp:135-149
bool within_azimuth_cell(const Grid& g, real azimuth, int i, int j, int k) {
    const real center = g.ph[g.at(i, j, k)];
    const real cd = periodic_angle_distance(azimuth, center);
    if (g.nph == 1) return cd <= 1.0e-10;
    real span = 0.0;
    if (k > 0) span = std::fmax(span, periodic_angle_distance(center, g.ph[g.at(i, j, k - 1)]));
    if (static_cast<size_t>(k + 1) < g.nph)
        span = std::fmax(span, periodic_angle_distance(center, g.ph[g.at(i, j, k + 1)]));
    return cd <= 0.500001 * span;
}

// scattering.hpp:151-180: three coordinate-descent passes, then half-cell acceptance.
bool locate_cell(const Grid& g, real radius, real polar, real azimuth, int& i, int& j, int& k) {
    if (g.nr == 0 || g.nth == 0 || g.nph == 0) return false;
    i = static_cast<int>(g.nr / 2);
    j = static_cast<int>(g.nth / 2);
    k = static_cast<int>(g.nph / 2);
    for (int it = 0; it < 3; ++it) {
        i = nearest_radial_index(g, radius, j, k);
        if (i < 0) return false;
        j = nearest_polar_index(g, polar, i, k);
        if (j < 0) return false;
        k = nearest_azimuth_index(g, azimuth, i, j);
        if (k < 0) return false;
    }
    return within_radial_cell(g, radius, i, j, k) && within_polar_cell(g, polar, i, j, k) &&
           within_azimuth_cell(g, azimuth, i, j, k);
}

// fluid_frame.hpp:6-13
real metric_inner_product(const real g[4][4], const real a[4], const real b[4]) {
    real result = 0.0;
    for (int mu = 0; mu < 4; ++mu)
        for (int nu = 0; nu < 4; ++nu) result += g[mu][nu] * a[mu] * b[nu];
    return result;
}

// fluid_frame.hpp:15-26
void spherical_to_cartesian(real r, real theta, real phi, real spin, real pos[4]) {
    const real st = std::sin(theta), ct = std::cos(theta);
    const real sp = std::sin(phi), cp = std::cos(phi);
    pos[0] = 0.0;
    pos[1] = (r * cp - spin * sp) * st;
    pos[2] = (r * sp + spin * cp) * st;
    pos[3] = r * ct;
}

// fluid_frame.hpp:28-48
void spherical_vector_to_cartesian(real r, real theta, real phi, real spin,
                                   const real s[4], real c[4]) {
    const real st = std::sin(theta), ct = std::cos(theta);
    const real sp = std::sin(phi), cp = std::cos(phi);
    const real radial_x = cp * st, radial_y = sp * st, radial_z = ct;
    const real theta_x = (r * cp - spin * sp) * ct;
    const real theta_y = (r * sp + spin * cp) * ct;
    const real theta_z = -r * st;
    const real phi_x = (-r * sp - spin * cp) * st;
    const real phi_y = (r * cp - spin * sp) * st;
    c[0] = s[0];
    c[1] = radial_x * s[1] + theta_x * s[2] + phi_x * s[3];
    c[2] = radial_y * s[1] + theta_y * s[2] + phi_y * s[3];
    c[3] = radial_z * s[1] + theta_z * s[2];
}

// fluid_frame.hpp:51-80: Gram-Schmidt tetrad with e0 = u/|u|.
bool build_fluid_tetrad(const real pos[4], const real u[4], real spin, real mass, real e[4][4]) {
    real g[4][4];
    compute_metric(pos, spin, mass, g);
    const real vn = metric_inner_product(g, u, u);
    if (!(vn < 0.0) || !std::isfinite(vn)) return false;
    const real inv = 1.0 / std::sqrt(-vn);
    const real ts = u[0] >= 0.0 ? 1.0 : -1.0;
    for (int mu = 0; mu < 4; ++mu) e[0][mu] = ts * u[mu] * inv;
    for (int axis = 0; axis < 3; ++axis) {
        real cand[4] = {0.0, 0.0, 0.0, 0.0};
        cand[axis + 1] = 1.0;
        const real tp = metric_inner_product(g, e[0], cand);
        for (int mu = 0; mu < 4; ++mu) cand[mu] += tp * e[0][mu];
        for (int prev = 0; prev < axis; ++prev) {
            const real proj = metric_inner_product(g, e[prev + 1], cand);
            for (int mu = 0; mu < 4; ++mu) cand[mu] -= proj * e[prev + 1][mu];
        }
        const real n = metric_inner_product(g, cand, cand);
        if (!(n > 1.0e-20) || !std::isfinite(n)) return false;
        const real is = 1.0 / std::sqrt(n);
        for (int mu = 0; mu < 4; ++mu) e[axis + 1][mu] = cand[mu] * is;
    }
    return true;
}

// fluid_frame.hpp:82-104
void fluid_direction_to_momentum(const real pos[4], const real e[4][4], real dx, real dy,
                                 real dz, real spin, real mass, real p[4]) {
    real w[4];
    for (int mu = 0; mu < 4; ++mu) w[mu] = e[0][mu] + dx * e[1][mu] + dy * e[2][mu] + dz * e[3][mu];
    real g[4][4];
    compute_metric(pos, spin, mass, g);
    for (int mu = 0; mu < 4; ++mu) {
        p[mu] = 0.0;
        for (int nu = 0; nu < 4; ++nu) p[mu] += g[mu][nu] * w[nu];
    }
}

// scattering.hpp:185-251
bool sample_fluid(const real state[8], const Grid& g, FluidCellCGS& fluid, real tetrad[4][4],
                  int* cell_out) {
    if (!g.available) return false;
    const real radius = compute_r(state[IX], state[IY], state[IZ], g.spin);
    if (!(radius > 0.0) || !std::isfinite(radius)) return false;
    const real cos_theta = std::fmax(real(-1.0), std::fmin(real(1.0), state[IZ] / radius));
    const real polar = std::acos(cos_theta);
    real azimuth = std::atan2(radius * state[IY] - g.spin * state[IX],
                              radius * state[IX] + g.spin * state[IY]);
    if (azimuth < 0.0) azimuth += 2.0 * PI;
    int i = -1, j = -1, k = -1;
    if (!locate_cell(g, radius, polar, azimuth, i, j, k)) return false;
    const size_t c = g.at(i, j, k);
    if (cell_out) *cell_out = static_cast<int>(c);
    fluid.position_cm[0] = state[IX] * g.length_scale;
    fluid.position_cm[1] = state[IY] * g.length_scale;
    fluid.position_cm[2] = state[IZ] * g.length_scale;
    fluid.coordinate_time_s = state[IT] * g.time_scale;
    fluid.density_g_cm3 = g.rho[c] * g.density_scale;
    fluid.temperature_k = g.T[c] * g.temperature_scale;
    if (!(fluid.density_g_cm3 > 0.0) || !std::isfinite(fluid.density_g_cm3) ||
        !std::isfinite(fluid.temperature_k))
        return false;
    real sv[4], sm[4];
    for (int q = 0; q < 4; ++q) {
        sv[q] = g.vel[c * 4 + q];
        sm[q] = g.mag[c * 4 + q];
    }
    spherical_vector_to_cartesian(g.r[c], g.th[c], g.ph[c], g.spin, sv,
                                  fluid.coordinate_four_velocity_cm_s);
    for (int q = 0; q < 4; ++q) fluid.coordinate_four_velocity_cm_s[q] *= g.velocity_scale;
    const real pos[4] = {state[IT], state[IX], state[IY], state[IZ]};
    if (!build_fluid_tetrad(pos, fluid.coordinate_four_velocity_cm_s, g.spin, g.mass, tetrad))
        return false;
    real cm[4];
    spherical_vector_to_cartesian(g.r[c], g.th[c], g.ph[c], g.spin, sm, cm);
    for (int q = 0; q < 4; ++q) cm[q] *= g.magnetic_scale;
    real metric[4][4];
    compute_metric(pos, g.spin, g.mass, metric);
    fluid.magnetic_gauss[0] = -metric_inner_product(metric, tetrad[0], cm);
    for (int axis = 1; axis < 4; ++axis)
        fluid.magnetic_gauss[axis] = metric_inner_product(metric, tetrad[axis], cm);
    return true;
}

// ---------------------------------------------------------------------------
// Radiative transfer, scattering, generators
// ---------------------------------------------------------------------------

// src/radiative_transfer/radiative_transfer.hpp:80-96 (with optional per-cell
// multipliers on the returned increments, used by the adjoint checks).
void apply_rt(real stokes[4], const FluidCellCGS& fluid, real nu, real path, bool abs_on,
              bool emis_on, real kappa, real jcoef, real m_abs = 1.0, real m_emis = 1.0) {
    if (abs_on) {
        const real dtau = m_abs * grt::ComputeOpticalDepthIncrement(fluid, nu, path, kappa);
        const real att = std::exp(-dtau);
        for (int q = 0; q < 4; ++q) stokes[q] *= att;
    }
    if (emis_on) stokes[0] += m_emis * grt::ComputeEmissivityIncrement(fluid, nu, path, jcoef);
}

constexpr real proton_mass_cgs = 1.67262192369e-24;   // scattering.hpp:256
constexpr real sigma_thomson_cgs = 6.6524587158e-25;  // scattering.hpp:257

// scattering.hpp:259-313
bool maybe_scatter(real state[8], real stokes[4], bool enabled, real albedo, real dl,
                   real length_scale, const FluidCellCGS& fluid, const real e[4][4], real spin,
                   real mass, Philox& rng) {
    if (!enabled) return false;
    const real path_cm = dl * length_scale;
    const real ne = fluid.density_g_cm3 / proton_mass_cgs;
    const real tau = sigma_thomson_cgs * ne * path_cm;
    const real prob = 1.0 - std::exp(-tau);
    if (rng.drand() >= prob) return false;
    real E = 0.0;
    for (int mu = 0; mu < 4; ++mu) E -= state[IKT + mu] * e[0][mu];
    if (!(E > 0.0) || !std::isfinite(E)) return false;
    const real mu_c = 2.0 * rng.drand() - 1.0;
    const real dphi = 2.0 * PI * rng.drand();
    const real tr = std::sqrt(std::fmax(real(0.0), 1.0 - mu_c * mu_c));
    const real pos[4] = {state[IT], state[IX], state[IY], state[IZ]};
    real pm[4];
    real sn, cs;
    grt::det_sincos(dphi, &sn, &cs);  // the kernels' sin/cos (grt_sincos.h), libm within 1 ulp
    fluid_direction_to_momentum(pos, e, tr * cs, tr * sn, mu_c, spin, mass, pm);
    for (int q = 0; q < 4; ++q) state[IKT + q] = E * pm[q];
    stokes[0] *= albedo;
    stokes[1] *= 0.5 * albedo;
    stokes[2] *= 0.5 * albedo;
    stokes[3] *= 0.25 * albedo;
    return true;
}

// src/radiative_transfer/photon_generation.hpp:99-124 (draw order made explicit)
bool generate_blackbody(const FluidCellCGS& cell, Philox& rng, int packets, real energy,
                        real& nu, real& E) {
    if (!(cell.temperature_k > 0.0)) return false;
    constexpr real inverse_zeta4 = 0.9239384029215902;
    const real choose = rng.drand();
    real cumulative = 0.0;
    int m = 1;
    for (; m < 64; ++m) {
        const real n = static_cast<real>(m);
        cumulative += inverse_zeta4 / (n * n * n * n);
        if (choose <= cumulative) break;
    }
    const real d1 = rng.drand(), d2 = rng.drand(), d3 = rng.drand(), d4 = rng.drand();
    const real product = std::fmax(real(1.0e-300), d1 * d2 * d3 * d4);
    const real x = -std::log(product) / static_cast<real>(m);
    constexpr real boltzmann_over_planck = 2.0836619123327576e10;
    nu = x * boltzmann_over_planck * cell.temperature_k;
    E = energy / static_cast<real>(packets);
    return std::isfinite(nu) && nu > 0.0;
}

// photon_generation.hpp:126-143
bool generate_power_law(Philox& rng, int packets, real slope, real nu_min, real nu_max,
                        real energy, real& nu, real& E) {
    const real draw = rng.drand();
    if (std::fabs(slope - 1.0) < 1.0e-12) {
        nu = nu_min * std::pow(nu_max / nu_min, draw);
    } else {
        const real ex = 1.0 - slope;
        const real lo = std::pow(nu_min, ex);
        const real hi = std::pow(nu_max, ex);
        nu = std::pow(lo + draw * (hi - lo), 1.0 / ex);
    }
    E = energy / static_cast<real>(packets);
    return std::isfinite(nu) && nu > 0.0;
}

// ---------------------------------------------------------------------------
// The per-photon step functor (src/geodesic_integrate/integrate_cart_ks.hpp)
// ---------------------------------------------------------------------------
struct Photon {
    uint64_t id;
    real freq, emit_e;
    real s[8];
    real I[4];
    real dl, tdisp, pdisp;
    uint8_t term, phase;
};

struct Stepper {
    const grt_params* p;
    const Grid* g;
    bool scat_on, abs_on, emis_on;
    // Optional per-cell multipliers on dtau / dI (adjoint checks); NULL = 1.
    const real* m_abs = nullptr;
    const real* m_emis = nullptr;
    real nrm[3], th_hat[3], ph_hat[3];
    uint64_t accepted = 0, rejected = 0, calls = 0;

    void init_camera() {
        const real st = std::sin(p->camera_theta), ct = std::cos(p->camera_theta);
        const real sp = std::sin(p->camera_phi), cp = std::cos(p->camera_phi);
        nrm[0] = st * cp; nrm[1] = st * sp; nrm[2] = ct;
        th_hat[0] = ct * cp; th_hat[1] = ct * sp; th_hat[2] = -st;
        ph_hat[0] = -sp; ph_hat[1] = cp; ph_hat[2] = 0.0;
    }

    void rhs(const real s[8], real out[8]) const {
        hamiltonian_rhs(s, s + 4, p->spin, p->mass, out);
    }

    // integrate_cart_ks.hpp:142-155
    void rk4(real s[8], real dt) const {
        real k1[8], k2[8], k3[8], k4[8], t[8];
        rhs(s, k1);
        for (int i = 0; i < 8; ++i) t[i] = s[i] + 0.5 * dt * k1[i];
        rhs(t, k2);
        for (int i = 0; i < 8; ++i) t[i] = s[i] + 0.5 * dt * k2[i];
        rhs(t, k3);
        for (int i = 0; i < 8; ++i) t[i] = s[i] + dt * k3[i];
        rhs(t, k4);
        for (int i = 0; i < 8; ++i) s[i] += (dt / 6.0) * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
    }

    // integrate_cart_ks.hpp:159-227 (Fehlberg 4(5), 5th-order solution kept)
    int rk45(real s[8], real* dlambda, const real k1[8]) const {
        const real a21 = 1.0 / 4.0;
        const real a31 = 3.0 / 32.0, a32 = 9.0 / 32.0;
        const real a41 = 1932.0 / 2197.0, a42 = -7200.0 / 2197.0, a43 = 7296.0 / 2197.0;
        const real a51 = 439.0 / 216.0, a52 = -8.0, a53 = 3680.0 / 513.0, a54 = -845.0 / 4104.0;
        const real a61 = -8.0 / 27.0, a62 = 2.0, a63 = -3544.0 / 2565.0, a64 = 1859.0 / 4104.0,
                   a65 = -11.0 / 40.0;
        const real b4_1 = 25.0 / 216.0, b4_3 = 1408.0 / 2565.0, b4_4 = 2197.0 / 4104.0, b4_5 = -1.0 / 5.0;
        const real b5_1 = 16.0 / 135.0, b5_3 = 6656.0 / 12825.0, b5_4 = 28561.0 / 56430.0,
                   b5_5 = -9.0 / 50.0, b5_6 = 2.0 / 55.0;
        const real dt = *dlambda;
        real k2[8], k3[8], k4[8], k5[8], k6[8], t[8];
        for (int i = 0; i < 8; ++i) t[i] = s[i] + dt * a21 * k1[i];
        rhs(t, k2);
        for (int i = 0; i < 8; ++i) t[i] = s[i] + dt * (a31 * k1[i] + a32 * k2[i]);
        rhs(t, k3);
        for (int i = 0; i < 8; ++i) t[i] = s[i] + dt * (a41 * k1[i] + a42 * k2[i] + a43 * k3[i]);
        rhs(t, k4);
        for (int i = 0; i < 8; ++i)
            t[i] = s[i] + dt * (a51 * k1[i] + a52 * k2[i] + a53 * k3[i] + a54 * k4[i]);
        rhs(t, k5);
        for (int i = 0; i < 8; ++i)
            t[i] = s[i] + dt * (a61 * k1[i] + a62 * k2[i] + a63 * k3[i] + a64 * k4[i] + a65 * k5[i]);
        rhs(t, k6);
        real x4[8], x5[8], err = 0.0;
        bool finite = true;
        for (int i = 0; i < 8; ++i) {
            x4[i] = s[i] + dt * (b4_1 * k1[i] + b4_3 * k3[i] + b4_4 * k4[i] + b4_5 * k5[i]);
            x5[i] = s[i] + dt * (b5_1 * k1[i] + b5_3 * k3[i] + b5_4 * k4[i] + b5_5 * k5[i] + b5_6 * k6[i]);
            const real sc = p->atol + p->rtol * std::fmax(std::fabs(x5[i]), std::fabs(x4[i]));
            const real ratio = std::fabs(x5[i] - x4[i]) / sc;
            if (!std::isfinite(x5[i]) || !std::isfinite(ratio)) finite = false;
            err = std::fmax(err, ratio);
        }
        if (!finite) {
            *dlambda = dt * p->min_step_scale;
            return 0;
        }
        if (err == 0.0) {
            *dlambda = dt * p->max_step_scale;
            for (int i = 0; i < 8; ++i) s[i] = x5[i];
            return 1;
        }
        real scale = p->safety * controller_root(real(1.0) / err);
        scale = std::fmin(p->max_step_scale, std::fmax(p->min_step_scale, scale));
        if (err <= 1.0) {
            *dlambda = dt * scale;
            for (int i = 0; i < 8; ++i) s[i] = x5[i];
            return 1;
        }
        *dlambda = dt * scale;
        return 0;
    }

    // integrate_cart_ks.hpp:96-120
    int camera_plane_crossing(const real s[8], real& u, real& v) const {
        const real pc = s[IX] * nrm[0] + s[IY] * nrm[1] + s[IZ] * nrm[2];
        if (pc < p->camera_distance) return 0;
        const real rel[3] = {s[IX] - p->camera_distance * nrm[0], s[IY] - p->camera_distance * nrm[1],
                             s[IZ] - p->camera_distance * nrm[2]};
        u = rel[0] * th_hat[0] + rel[1] * th_hat[1] + rel[2] * th_hat[2];
        v = rel[0] * ph_hat[0] + rel[1] * ph_hat[1] + rel[2] * ph_hat[2];
        const bool inside = std::fabs(u) <= 0.5 * p->camera_width && std::fabs(v) <= 0.5 * p->camera_height;
        return inside ? 1 : -1;
    }

    // integrate_cart_ks.hpp:122-130
    real camera_observer_energy(const real s[8]) const {
        const real X[4] = {s[IT], s[IX], s[IY], s[IZ]};
        real g[4][4];
        compute_metric(X, p->spin, p->mass, g);
        if (!(g[0][0] < 0.0)) return 0.0;
        const real u0 = 1.0 / std::sqrt(-g[0][0]);
        return -s[IKT] * u0;
    }

    // integrate_cart_ks.hpp:230-419: one invocation on photon ph at host step `step`.
    // trace (optional) receives (cell, dtau_base, dI_base, I_before, scale) for
    // every radiative-transfer application -- scale = albedo when the photon
    // scattered in that step, else 1 -- and (-1, 0, 0, 0, 0) when the Stokes
    // vector is zeroed on arrival; the adjoint check replays it backwards.
    void call(Photon& ph, int64_t step, std::vector<real>* trace = nullptr) {
        if (ph.term) return;
        ++calls;
        real s[8];
        for (int i = 0; i < 8; ++i) s[i] = ph.s[i];
        const uint8_t phase = ph.phase;
        const real dist = compute_r(s[IX], s[IY], s[IZ], p->spin);
        if (dist <= p->r_term_min) {
            ph.I[0] = ph.I[1] = ph.I[2] = ph.I[3] = 0.0;
            ph.term = 1;
            ph.phase = GRT_PHASE_REJECTED;
            return;
        }
        if (dist > p->r_term_max) {
            ph.term = 1;
            ph.phase = GRT_PHASE_REJECTED;
            return;
        }
        real taken = 0.0;
        if (p->integrator == GRT_RK4) {
            taken = ph.dl;
            rk4(s, taken);
            ++accepted;
        } else if (p->integrator == GRT_RK45) {
            real k1[8];
            rhs(s, k1);
            real dl = ph.dl;
            int ok = 0;
            for (int attempt = 0; attempt < 12; ++attempt) {
                taken = dl;
                ok = rk45(s, &dl, k1);
                if (ok) break;
                ++rejected;
            }
            ph.dl = dl;
            if (!ok) {
                ph.term = 1;
                return;
            }
            ++accepted;
        } else {
            ph.term = 1;
            return;
        }
        real stokes[4] = {ph.I[0], ph.I[1], ph.I[2], ph.I[3]};
        FluidCellCGS fluid;
        real tetrad[4][4];
        const bool image = p->mode == GRT_MODE_IMAGE;
        const bool needs = scat_on || abs_on || emis_on || (image && phase == GRT_PHASE_IMAGE_BACKWARD);
        int cell = -1;
        const bool sampled = needs && sample_fluid(s, *g, fluid, tetrad, &cell);
        if (image && phase == GRT_PHASE_IMAGE_BACKWARD && sampled) {
            Philox rng(p->scattering_seed + static_cast<uint64_t>(p->rank), ph.id, static_cast<uint32_t>(step));
            real nu = 0.0, E = 0.0;
            bool generated = false;
            const real dcode = fluid.density_g_cm3 / g->density_scale;
            const int packets = grt::ComputeSuperphotonsPerCell(dcode, p->superphoton_count_normalization);
            if (packets > 0 && p->generator == GRT_GEN_BLACKBODY) {
                generated = generate_blackbody(fluid, rng, packets, p->energy_per_cell_erg, nu, E);
            } else if (packets > 0 && p->generator == GRT_GEN_POWER_LAW) {
                generated = generate_power_law(rng, packets, p->power_law_slope, p->nu_min_hz,
                                               p->nu_max_hz, p->energy_per_cell_erg, nu, E);
            } else if (packets > 0) {
                generated = grt::GeneratePhotonsCustom(fluid, rng, packets, p->custom_frequency_hz,
                                                       p->energy_per_cell_erg, nu, E);
            }
            if (generated) {
                ph.freq = nu;
                real ee = 0.0;
                for (int c = 0; c < 4; ++c) ee -= s[IKT + c] * tetrad[0][c];
                ph.emit_e = ee;
                stokes[0] = E;
                stokes[1] = stokes[2] = stokes[3] = 0.0;
                ph.dl = -std::fabs(ph.dl);
                ph.phase = GRT_PHASE_IMAGE_FORWARD;
            } else {
                stokes[0] = stokes[1] = stokes[2] = stokes[3] = 0.0;
                ph.term = 1;
                ph.phase = GRT_PHASE_REJECTED;
            }
        } else if (sampled && phase != GRT_PHASE_IMAGE_BACKWARD) {
            if (abs_on || emis_on) {
                const real ma = m_abs ? m_abs[cell] : 1.0;
                const real me = m_emis ? m_emis[cell] : 1.0;
                if (trace) {
                    trace->push_back(static_cast<real>(cell));
                    trace->push_back(abs_on ? grt::ComputeOpticalDepthIncrement(
                                                  fluid, ph.freq, taken, p->absorption_coefficient)
                                            : 0.0);
                    trace->push_back(emis_on ? grt::ComputeEmissivityIncrement(
                                                   fluid, ph.freq, taken, p->emission_coefficient)
                                             : 0.0);
                    trace->push_back(stokes[0]);
                }
                apply_rt(stokes, fluid, ph.freq, taken, abs_on, emis_on, p->absorption_coefficient,
                         p->emission_coefficient, ma, me);
            }
            bool scattered = false;
            if (scat_on) {
                Philox rng(p->scattering_seed + static_cast<uint64_t>(p->rank), ph.id, static_cast<uint32_t>(step));
                scattered = maybe_scatter(s, stokes, true, p->scattering_albedo, std::fabs(ph.dl), g->length_scale,
                                          fluid, tetrad, p->spin, p->mass, rng);
            }
            if (trace && (abs_on || emis_on)) trace->push_back(scattered ? p->scattering_albedo : 1.0);
        }
        if (image && phase == GRT_PHASE_IMAGE_FORWARD) {
            real u = 0.0, v = 0.0;
            const int crossing = camera_plane_crossing(s, u, v);
            if (crossing > 0) {
                const real eo = camera_observer_energy(s);
                const real ee = ph.emit_e;
                if (eo > 0.0 && ee > 0.0 && std::isfinite(eo) && std::isfinite(ee)) {
                    ph.freq *= eo / ee;
                } else {
                    stokes[0] = stokes[1] = stokes[2] = stokes[3] = 0.0;
                    if (trace) trace->insert(trace->end(), {-1.0, 0.0, 0.0, 0.0, 0.0});
                }
                ph.tdisp = u;
                ph.pdisp = v;
                ph.phase = GRT_PHASE_IMAGE_ARRIVED;
                ph.term = 1;
            } else if (crossing < 0) {
                stokes[0] = stokes[1] = stokes[2] = stokes[3] = 0.0;
                ph.phase = GRT_PHASE_REJECTED;
                ph.term = 1;
            }
        }
        for (int i = 0; i < 8; ++i) ph.s[i] = s[i];
        for (int q = 0; q < 4; ++q) ph.I[q] = stokes[q];
    }
};

Grid make_grid(const grt_params* p, size_t nr, size_t nth, size_t nph, const real* r, const real* th,
               const real* ph, const real* rho, const real* T, const real* vel, const real* mag) {
    Grid g;
    g.nr = nr; g.nth = nth; g.nph = nph;
    g.r = r; g.th = th; g.ph = ph; g.rho = rho; g.T = T; g.vel = vel; g.mag = mag;
    g.length_scale = p->length_cm_per_code;
    g.time_scale = p->time_s_per_code;
    g.density_scale = p->density_g_cm3_per_code;
    g.temperature_scale = p->temperature_k_per_code;
    g.velocity_scale = p->four_velocity_cm_s_per_code;
    g.magnetic_scale = p->magnetic_gauss_per_code;
    g.spin = p->spin;
    g.mass = p->mass;
    // integrate_cart_ks.hpp:436-445: fluid available iff every field is present.
    g.available = nr > 0 && nth > 0 && nph > 0 && r && th && ph && rho && T && vel && mag;
    return g;
}

void load(const grt_photon_soa* s, size_t i, Photon& ph) {
    ph.id = s->id[i];
    ph.freq = s->frequency[i];
    ph.emit_e = s->emission_frame_energy[i];
    ph.s[0] = s->x0[i]; ph.s[1] = s->x1[i]; ph.s[2] = s->x2[i]; ph.s[3] = s->x3[i];
    ph.s[4] = s->k0[i]; ph.s[5] = s->k1[i]; ph.s[6] = s->k2[i]; ph.s[7] = s->k3[i];
    ph.I[0] = s->I[i]; ph.I[1] = s->Q[i]; ph.I[2] = s->U[i]; ph.I[3] = s->V[i];
    ph.dl = s->dlambda[i];
    ph.tdisp = s->theta_disp[i];
    ph.pdisp = s->phi_disp[i];
    ph.term = s->terminate[i];
    ph.phase = s->phase[i];
}

void store(const Photon& ph, const grt_photon_soa* s, size_t i) {
    s->id[i] = ph.id;
    s->frequency[i] = ph.freq;
    s->emission_frame_energy[i] = ph.emit_e;
    s->x0[i] = ph.s[0]; s->x1[i] = ph.s[1]; s->x2[i] = ph.s[2]; s->x3[i] = ph.s[3];
    s->k0[i] = ph.s[4]; s->k1[i] = ph.s[5]; s->k2[i] = ph.s[6]; s->k3[i] = ph.s[7];
    s->I[i] = ph.I[0]; s->Q[i] = ph.I[1]; s->U[i] = ph.I[2]; s->V[i] = ph.I[3];
    s->dlambda[i] = ph.dl;
    s->theta_disp[i] = ph.tdisp;
    s->phi_disp[i] = ph.pdisp;
    s->terminate[i] = ph.term;
    s->phase[i] = ph.phase;
}

// src/radiative_transfer/observation.hpp:22-29
size_t observation_bin(real value, real lo, real hi, size_t bins) {
    if (bins <= 1 || !(hi > lo)) return 0;
    const real f = (value - lo) / (hi - lo);
    const real sc = std::fmax(real(0.0), std::fmin(real(1.0), f));
    return static_cast<size_t>(sc * static_cast<real>(bins - 1));
}

}  // namespace oracle


// ---------------------------------------------------------------------------
// Op counting: the RHS and the RK4 / RKF45 stage arithmetic above, written
// once more over a scalar type that counts +, -, *, / and sqrt (and pow, as
// one op), in the same source order, to pin the algorithmic FLOP counts the
// roofline uses.  A test checks that the Counted instantiation produces the
// same values as the double code above.
// ---------------------------------------------------------------------------
namespace opcount {
struct Counter { uint64_t add = 0, mul = 0, div = 0, sqrt = 0, pow = 0; };
Counter g;
struct N {
    double v;
    N(double x = 0.0) : v(x) {}
};
inline N operator+(N a, N b) { ++g.add; return N(a.v + b.v); }
inline N operator-(N a, N b) { ++g.add; return N(a.v - b.v); }
inline N operator*(N a, N b) { ++g.mul; return N(a.v * b.v); }
inline N operator/(N a, N b) { ++g.div; return N(a.v / b.v); }
inline N operator-(N a) { return N(-a.v); }
inline N& operator+=(N& a, N b) { a = a + b; return a; }
inline bool operator<(N a, N b) { return a.v < b.v; }
inline bool operator>(N a, N b) { return a.v > b.v; }
inline bool operator<=(N a, N b) { return a.v <= b.v; }
inline bool operator==(N a, N b) { return a.v == b.v; }
inline N Sqrt(N a) { ++g.sqrt; return N(std::sqrt(a.v)); }
inline N Fabs(N a) { return N(std::fabs(a.v)); }
inline N Fmax(N a, N b) { return N(std::fmax(a.v, b.v)); }
inline N Fmin(N a, N b) { return N(std::fmin(a.v, b.v)); }
inline N Pow(N a, N b) { ++g.pow; return N(std::pow(a.v, b.v)); }
inline bool Isfinite(N a) { return std::isfinite(a.v); }
template <class T> T SQ(T x) { return x * x; }
template <class T> T CU(T x) { return x * x * x; }
template <class T> T QU(T x) { return x * x * x * x; }

// kerr_schild_core.hpp:157-192 with :36-46, :58-77, :85-95
template <class T>
void rhs(const T X[4], const T p[4], T a, T M, T out[8]) {
    const T rsq = SQ(X[1]) + SQ(X[2]) + SQ(X[3]);
    const T A = rsq - SQ(a);
    const T S = Sqrt(SQ(A) + T(4.0) * SQ(a * X[3]));
    const T r = Sqrt(T(0.5) * (A + S));
    const T opas = T(1.0) + A / S;
    T dr[3];
    dr[0] = X[1] * opas / (T(2.0) * r);
    dr[1] = X[2] * opas / (T(2.0) * r);
    dr[2] = (X[3] * opas + T(2.0) * SQ(a) * X[3] / S) / (T(2.0) * r);
    const T B = SQ(r) + SQ(a);
    T l[4], dl[3][4];
    l[0] = T(1.0);
    l[1] = (r * X[1] + a * X[2]) / B;
    l[2] = (r * X[2] - a * X[1]) / B;
    l[3] = X[3] / r;
    for (int k = 0; k < 3; ++k) {
        const T dx = T(k == 0 ? 1.0 : 0.0), dy = T(k == 1 ? 1.0 : 0.0), dz = T(k == 2 ? 1.0 : 0.0);
        const T dB = T(2.0) * r * dr[k];
        dl[k][0] = T(0.0);
        dl[k][1] = ((dr[k] * X[1] + r * dx) + a * dy - l[1] * dB) / B;
        dl[k][2] = ((dr[k] * X[2] + r * dy) - a * dx - l[2] * dB) / B;
        dl[k][3] = (dz - l[3] * dr[k]) / r;
    }
    const T D = QU(r) + SQ(a * X[3]);
    const T H = M * CU(r) / D;
    T dH[3];
    for (int k = 0; k < 3; ++k) {
        const T dz = T(k == 2 ? 1.0 : 0.0);
        const T dD = T(4.0) * CU(r) * dr[k] + T(2.0) * SQ(a) * X[3] * dz;
        dH[k] = M * (T(3.0) * SQ(r) * dr[k] * D - CU(r) * dD) / SQ(D);
    }
    const T lup[4] = {-l[0], l[1], l[2], l[3]};
    T ldp = T(0.0);
    for (int mu = 0; mu < 4; ++mu) ldp += lup[mu] * p[mu];
    out[0] = -p[0] - T(2.0) * H * lup[0] * ldp;
    for (int mu = 1; mu < 4; ++mu) out[mu] = p[mu] - T(2.0) * H * lup[mu] * ldp;
    out[4] = T(0.0);
    for (int k = 0; k < 3; ++k) {
        const T dlup[4] = {-dl[k][0], dl[k][1], dl[k][2], dl[k][3]};
        T dldp = T(0.0);
        for (int mu = 0; mu < 4; ++mu) dldp += dlup[mu] * p[mu];
        out[5 + k] = dH[k] * SQ(ldp) + T(2.0) * H * ldp * dldp;
    }
}

template <class T>
void rhs_s(const T s[8], T a, T M, T out[8]) { rhs<T>(s, s + 4, a, M, out); }

// integrate_cart_ks.hpp:142-155
template <class T>
void rk4(T s[8], T dt, T a, T M) {
    T k1[8], k2[8], k3[8], k4[8], t[8];
    rhs_s(s, a, M, k1);
    for (int i = 0; i < 8; ++i) t[i] = s[i] + T(0.5) * dt * k1[i];
    rhs_s(t, a, M, k2);
    for (int i = 0; i < 8; ++i) t[i] = s[i] + T(0.5) * dt * k2[i];
    rhs_s(t, a, M, k3);
    for (int i = 0; i < 8; ++i) t[i] = s[i] + dt * k3[i];
    rhs_s(t, a, M, k4);
    for (int i = 0; i < 8; ++i) s[i] += (dt / T(6.0)) * (k1[i] + T(2.0) * k2[i] + T(2.0) * k3[i] + k4[i]);
}

// integrate_cart_ks.hpp:159-227, one attempt (k1 given); returns accepted
template <class T>
int rk45_attempt(T s[8], T& dl, const T k1[8], T a, T M, T atol, T rtol) {
    const T a21 = T(1.0 / 4.0), a31 = T(3.0 / 32.0), a32 = T(9.0 / 32.0);
    const T a41 = T(1932.0 / 2197.0), a42 = T(-7200.0 / 2197.0), a43 = T(7296.0 / 2197.0);
    const T a51 = T(439.0 / 216.0), a52 = T(-8.0), a53 = T(3680.0 / 513.0), a54 = T(-845.0 / 4104.0);
    const T a61 = T(-8.0 / 27.0), a62 = T(2.0), a63 = T(-3544.0 / 2565.0), a64 = T(1859.0 / 4104.0),
            a65 = T(-11.0 / 40.0);
    const T b41 = T(25.0 / 216.0), b43 = T(1408.0 / 2565.0), b44 = T(2197.0 / 4104.0), b45 = T(-1.0 / 5.0);
    const T b51 = T(16.0 / 135.0), b53 = T(6656.0 / 12825.0), b54 = T(28561.0 / 56430.0), b55 = T(-9.0 / 50.0),
            b56 = T(2.0 / 55.0);
    const T dt = dl;
    T k2[8], k3[8], k4[8], k5[8], k6[8], t[8];
    for (int i = 0; i < 8; ++i) t[i] = s[i] + dt * a21 * k1[i];
    rhs_s(t, a, M, k2);
    for (int i = 0; i < 8; ++i) t[i] = s[i] + dt * (a31 * k1[i] + a32 * k2[i]);
    rhs_s(t, a, M, k3);
    for (int i = 0; i < 8; ++i) t[i] = s[i] + dt * (a41 * k1[i] + a42 * k2[i] + a43 * k3[i]);
    rhs_s(t, a, M, k4);
    for (int i = 0; i < 8; ++i) t[i] = s[i] + dt * (a51 * k1[i] + a52 * k2[i] + a53 * k3[i] + a54 * k4[i]);
    rhs_s(t, a, M, k5);
    for (int i = 0; i < 8; ++i)
        t[i] = s[i] + dt * (a61 * k1[i] + a62 * k2[i] + a63 * k3[i] + a64 * k4[i] + a65 * k5[i]);
    rhs_s(t, a, M, k6);
    T x4[8], x5[8], err = T(0.0);
    for (int i = 0; i < 8; ++i) {
        x4[i] = s[i] + dt * (b41 * k1[i] + b43 * k3[i] + b44 * k4[i] + b45 * k5[i]);
        x5[i] = s[i] + dt * (b51 * k1[i] + b53 * k3[i] + b54 * k4[i] + b55 * k5[i] + b56 * k6[i]);
        const T sc = atol + rtol * Fmax(Fabs(x5[i]), Fabs(x4[i]));
        err = Fmax(err, Fabs(x5[i] - x4[i]) / sc);
    }
    T scale = T(0.9) * Pow(T(1.0) / err, T(0.25));
    scale = Fmin(T(10.0), Fmax(T(0.01), scale));
    dl = dt * scale;
    if (err <= T(1.0)) {
        for (int i = 0; i < 8; ++i) s[i] = x5[i];
        return 1;
    }
    return 0;
}
}  // namespace opcount

using namespace oracle;

extern "C" {

// One full run of the reference step loop (integrate_cart_ks.hpp:468-527) over
// n photons in place: the global step loop with the termination check on
// output steps.  per_photon_cap (may be NULL) receives nothing; stats gets
// counters.  m_abs/m_emis are optional per-cell multipliers (NULL = 1).
int oracle_run(const grt_params* p, size_t nr, size_t nth, size_t nph, const double* r,
               const double* th, const double* ph, const double* rho, const double* T,
               const double* vel, const double* mag, const double* m_abs, const double* m_emis,
               grt_photon_soa* soa, size_t n, grt_run_stats* stats) {
    Grid g = make_grid(p, nr, nth, nph, r, th, ph, rho, T, vel, mag);
    std::vector<Photon> photons(n);
    for (size_t i = 0; i < n; ++i) load(soa, i, photons[i]);
    uint64_t acc = 0, rej = 0, calls = 0;
    real fraction = 0.0;
    int64_t step = 0;
    int64_t steps_done = 0;
    const uint64_t interval = p->output_interval ? p->output_interval : 1;
    for (step = 0; step < p->max_steps; ++step) {
#pragma omp parallel reduction(+ : acc, rej, calls)
        {
            Stepper st{p, &g, p->scattering_enabled && g.available,
                       p->absorption_enabled && g.available, p->emission_enabled && g.available,
                       m_abs, m_emis};
            st.init_camera();
#pragma omp for schedule(dynamic, 64)
            for (int64_t i = 0; i < static_cast<int64_t>(n); ++i) st.call(photons[i], step);
            acc += st.accepted;
            rej += st.rejected;
            calls += st.calls;
        }
        steps_done = step + 1;
        if (static_cast<uint64_t>(step) % interval == 0 || step == p->max_steps - 1) {
            uint64_t term = 0;
            for (size_t i = 0; i < n; ++i) term += photons[i].term ? 1 : 0;
            fraction = static_cast<real>(term) / static_cast<real>(p->nphotons);
        }
        if (fraction >= p->termination_percent) break;
    }
    uint64_t term = 0;
    for (size_t i = 0; i < n; ++i) {
        store(photons[i], soa, i);
        term += photons[i].term ? 1 : 0;
    }
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->steps_done = steps_done;
        stats->n_terminated = term;
        stats->accepted_steps = acc;
        stats->rejected_attempts = rej;
        stats->photon_calls = calls;
    }
    return 0;
}

// FP64 reference gradient of a Stokes-I image loss with respect to the
// per-cell multipliers: every photon is stepped alone to termination (the
// termination_percent = 1 loop), recording its radiative-transfer updates, and
// ImageArrived photons replay them backwards from dL/dI of their pixel
// (observation.hpp:22-29 binning over image_nx x image_ny).  photons are
// advanced in place; g_abs/g_emis ([nr*nth*nph]) are overwritten.
int oracle_adjoint_image_I(const grt_params* p, size_t nr, size_t nth, size_t nph, const double* r,
                           const double* th, const double* ph, const double* rho, const double* T,
                           const double* vel, const double* mag, const double* m_abs, const double* m_emis,
                           grt_photon_soa* soa, size_t n, const double* dL_dI, double* g_abs, double* g_emis) {
    Grid g = make_grid(p, nr, nth, nph, r, th, ph, rho, T, vel, mag);
    const size_t ncell = nr * nth * nph;
    std::vector<real> ga(ncell, 0.0), ge(ncell, 0.0);
    Stepper st{p, &g, p->scattering_enabled && g.available, p->absorption_enabled && g.available,
               p->emission_enabled && g.available, m_abs, m_emis};
    st.init_camera();
    std::vector<real> tr;
    for (size_t i = 0; i < n; ++i) {
        Photon pho;
        load(soa, i, pho);
        tr.clear();
        for (int64_t step = 0; step < p->max_steps && !pho.term; ++step) st.call(pho, step, &tr);
        store(pho, soa, i);
        if (pho.phase != GRT_PHASE_IMAGE_ARRIVED) continue;
        const auto bin = [](real v, real lo, real hi, uint64_t bins) -> uint64_t {
            if (bins <= 1 || !(hi > lo)) return 0;
            const real f = std::fmax(0.0, std::fmin(1.0, (v - lo) / (hi - lo)));
            return static_cast<uint64_t>(f * static_cast<real>(bins - 1));
        };
        const uint64_t px = bin(pho.tdisp, -0.5 * p->camera_width, 0.5 * p->camera_width, p->image_nx);
        const uint64_t py = bin(pho.pdisp, -0.5 * p->camera_height, 0.5 * p->camera_height, p->image_ny);
        real lam = dL_dI[py * p->image_nx + px];
        if (!tr.empty() && tr[tr.size() - 5] < 0.0) lam = 0.0;  // zeroed on arrival
        for (size_t e = tr.size(); e >= 5 && lam != 0.0; e -= 5) {
            const real* q = &tr[e - 5];
            if (q[0] < 0.0) continue;
            const size_t cell = static_cast<size_t>(q[0]);
            const real tau0 = q[1], j0 = q[2], Ib = q[3], scale = q[4];
            const real ma = m_abs ? m_abs[cell] : 1.0;
            const real att = st.abs_on ? std::exp(-(ma * tau0)) : 1.0;
            const real lp = lam * scale;
            if (st.emis_on) ge[cell] += lp * j0;
            if (st.abs_on) ga[cell] += lp * Ib * att * (-tau0);
            lam = lp * att;
        }
    }
    for (size_t c = 0; c < ncell; ++c) {
        if (g_abs) g_abs[c] = ga[c];
        if (g_emis) g_emis[c] = ge[c];
    }
    return 0;
}

// initialize_photons_disk (src/radiative_transfer/initialize_photons.hpp:
// 173-327) after build_superphoton_cell_offsets (:32-64), with the kernels'
// random streams (Philox keyed by seed + rank, photon id, domain 0xFFFFFFFF;
// generator draws, then mu, phi) and the shared deterministic sin/cos for the
// direction.  out == NULL only counts the packets (*n_out).
int oracle_init_disk_photons(const grt_params* p, size_t nr, size_t nth, size_t nph, const double* r,
                             const double* th, const double* ph, const double* rho, const double* T,
                             const double* vel, const double* mag, uint64_t id_offset, grt_photon_soa* out,
                             uint64_t* n_out) {
    Grid g = make_grid(p, nr, nth, nph, r, th, ph, rho, T, vel, mag);
    const size_t ncell = nr * nth * nph;
    std::vector<uint64_t> off(ncell + 1);
    uint64_t total = 0;
    for (size_t c = 0; c < ncell; ++c) {
        off[c] = total;
        const int count = grt::ComputeSuperphotonsPerCell(rho[c], p->superphoton_count_normalization);
        total += static_cast<uint64_t>(count > 0 ? count : 0);
    }
    off[ncell] = total;
    if (n_out) *n_out = total;
    if (!out) return 0;
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < static_cast<int64_t>(total); ++ii) {
        const uint64_t i = static_cast<uint64_t>(ii);
        size_t lo = 0, hi = ncell;  // locate_superphoton_cell (:66-80)
        while (lo + 1 < hi) {
            const size_t mid = lo + (hi - lo) / 2;
            if (off[mid] <= i) lo = mid;
            else hi = mid;
        }
        const size_t c = lo;
        const int packets = static_cast<int>(off[c + 1] - off[c]);
        real pos[4];
        spherical_to_cartesian(r[c], th[c], ph[c], p->spin, pos);
        FluidCellCGS fluid;
        for (int q = 0; q < 3; ++q) fluid.position_cm[q] = pos[q + 1] * g.length_scale;
        fluid.coordinate_time_s = pos[0] * g.time_scale;
        fluid.density_g_cm3 = rho[c] * g.density_scale;
        fluid.temperature_k = T[c] * g.temperature_scale;
        real sv[4], sm[4], cm[4];
        for (int q = 0; q < 4; ++q) {
            sv[q] = vel[4 * c + q];
            sm[q] = mag[4 * c + q];
        }
        spherical_vector_to_cartesian(r[c], th[c], ph[c], p->spin, sv, fluid.coordinate_four_velocity_cm_s);
        for (int q = 0; q < 4; ++q) fluid.coordinate_four_velocity_cm_s[q] *= g.velocity_scale;
        spherical_vector_to_cartesian(r[c], th[c], ph[c], p->spin, sm, cm);
        for (int q = 0; q < 4; ++q) cm[q] *= g.magnetic_scale;
        real e[4][4];
        const bool valid = build_fluid_tetrad(pos, fluid.coordinate_four_velocity_cm_s, p->spin, p->mass, e);
        for (int q = 0; q < 4; ++q) fluid.magnetic_gauss[q] = 0.0;
        if (valid) {
            real metric[4][4];
            compute_metric(pos, p->spin, p->mass, metric);
            fluid.magnetic_gauss[0] = -metric_inner_product(metric, e[0], cm);
            for (int axis = 1; axis < 4; ++axis) fluid.magnetic_gauss[axis] = metric_inner_product(metric, e[axis], cm);
        }
        const uint64_t id = id_offset + i;
        Philox rng(p->scattering_seed + static_cast<uint64_t>(p->rank), id, 0xFFFFFFFFu);
        real nu = 0.0, E = 0.0;
        bool generated = false;
        if (valid && p->generator == GRT_GEN_BLACKBODY) {
            generated = generate_blackbody(fluid, rng, packets, p->energy_per_cell_erg, nu, E);
        } else if (valid && p->generator == GRT_GEN_POWER_LAW) {
            generated = generate_power_law(rng, packets, p->power_law_slope, p->nu_min_hz, p->nu_max_hz,
                                           p->energy_per_cell_erg, nu, E);
        } else if (valid) {
            generated = grt::GeneratePhotonsCustom(fluid, rng, packets, p->custom_frequency_hz, p->energy_per_cell_erg,
                                                   nu, E);
        }
        const real mu = 2.0 * rng.drand() - 1.0;
        const real dphi = 2.0 * PI * rng.drand();
        const real tr = std::sqrt(std::fmax(real(0.0), 1.0 - mu * mu));
        real sn, cs;
        grt::det_sincos(dphi, &sn, &cs);
        real pc[4] = {0.0, 0.0, 0.0, 0.0};
        if (generated) fluid_direction_to_momentum(pos, e, tr * cs, tr * sn, mu, p->spin, p->mass, pc);
        real ee = 0.0;
        if (generated)
            for (int q = 0; q < 4; ++q) ee -= pc[q] * e[0][q];
        out->id[i] = id;
        out->frequency[i] = nu;
        out->emission_frame_energy[i] = ee;
        out->x0[i] = pos[0]; out->x1[i] = pos[1]; out->x2[i] = pos[2]; out->x3[i] = pos[3];
        out->k0[i] = pc[0]; out->k1[i] = pc[1]; out->k2[i] = pc[2]; out->k3[i] = pc[3];
        out->I[i] = generated ? E : 0.0;
        out->Q[i] = out->U[i] = out->V[i] = 0.0;
        out->dlambda[i] = p->initial_step;
        out->terminate[i] = generated ? 0 : 1;
        out->phase[i] = generated ? GRT_PHASE_DISK : GRT_PHASE_REJECTED;
        out->theta_disp[i] = 0.0;
        out->phi_disp[i] = 0.0;
    }
    return 0;
}

// Deterministic pixel-grid variant of initialize_photons_image
// (src/radiative_transfer/initialize_photons.hpp:82-170).
// initialize_photons_image (src/radiative_transfer/initialize_photons.hpp:
// 82-170) with its random screen (:115-126): (u, v) = drand(-W/2, W/2),
// drand(-H/2, H/2), drand(lo, hi) = lo + (hi - lo) d, the pool seeded
// 12345 + rank -- here Philox keyed by (12345 + rank, photon id, domain
// 0xFFFFFFFE), the kernels' streams, in place of Kokkos's XorShift pool.
int oracle_init_image_photons_random(const grt_params* p, uint64_t n, uint64_t id_offset, grt_photon_soa* out) {
    const real D = p->camera_distance;
    const real cx = D * std::sin(p->camera_theta) * std::cos(p->camera_phi);
    const real cy = D * std::sin(p->camera_theta) * std::sin(p->camera_phi);
    const real cz = D * std::cos(p->camera_theta);
    const real th_hat[3] = {std::cos(p->camera_theta) * std::cos(p->camera_phi),
                            std::cos(p->camera_theta) * std::sin(p->camera_phi), -std::sin(p->camera_theta)};
    const real ph_hat[3] = {-std::sin(p->camera_phi), std::cos(p->camera_phi), 0.0};
    const real W = p->camera_width, H = p->camera_height;
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t id = id_offset + i;
        Philox rng(12345ull + static_cast<uint64_t>(static_cast<int64_t>(p->rank)), id, 0xFFFFFFFEu);
        const real u = -W / 2 + (W / 2 - (-W / 2)) * rng.drand();
        const real v = -H / 2 + (H / 2 - (-H / 2)) * rng.drand();
        out->id[i] = id;
        out->frequency[i] = 0.0;
        out->emission_frame_energy[i] = 1.0;
        const real x = cx + u * th_hat[0] + v * ph_hat[0];
        const real y = cy + u * th_hat[1] + v * ph_hat[1];
        const real z = cz + u * th_hat[2] + v * ph_hat[2];
        real kx = -cx, ky = -cy, kz = -cz;
        const real kn = std::sqrt(kx * kx + ky * ky + kz * kz);
        kx /= kn; ky /= kn; kz /= kn;
        out->x0[i] = 0.0; out->x1[i] = x; out->x2[i] = y; out->x3[i] = z;
        const real X[4] = {0.0, x, y, z};
        const real K[3] = {kx, ky, kz};
        real pc[4] = {0.0, 0.0, 0.0, 0.0};
        null_covariant_momentum(X, K, p->spin, p->mass, pc);
        out->k0[i] = pc[0]; out->k1[i] = pc[1]; out->k2[i] = pc[2]; out->k3[i] = pc[3];
        out->I[i] = out->Q[i] = out->U[i] = out->V[i] = 0.0;
        out->dlambda[i] = p->initial_step * D;
        out->terminate[i] = 0;
        out->phase[i] = GRT_PHASE_IMAGE_BACKWARD;
        out->theta_disp[i] = u;
        out->phi_disp[i] = v;
    }
    return 0;
}

int oracle_init_image_photons(const grt_params* p, uint64_t nx, uint64_t ny, uint64_t id_offset,
                              grt_photon_soa* out) {
    const real D = p->camera_distance;
    const real cx = D * std::sin(p->camera_theta) * std::cos(p->camera_phi);
    const real cy = D * std::sin(p->camera_theta) * std::sin(p->camera_phi);
    const real cz = D * std::cos(p->camera_theta);
    const real th_hat[3] = {std::cos(p->camera_theta) * std::cos(p->camera_phi),
                            std::cos(p->camera_theta) * std::sin(p->camera_phi), -std::sin(p->camera_theta)};
    const real ph_hat[3] = {-std::sin(p->camera_phi), std::cos(p->camera_phi), 0.0};
    for (uint64_t iy = 0; iy < ny; ++iy) {
        for (uint64_t ix = 0; ix < nx; ++ix) {
            const uint64_t i = iy * nx + ix;
            const real u = -0.5 * p->camera_width + (static_cast<real>(ix) + 0.5) * p->camera_width / static_cast<real>(nx);
            const real v = -0.5 * p->camera_height + (static_cast<real>(iy) + 0.5) * p->camera_height / static_cast<real>(ny);
            out->id[i] = id_offset + i;
            out->frequency[i] = 0.0;
            out->emission_frame_energy[i] = 1.0;
            const real x = cx + u * th_hat[0] + v * ph_hat[0];
            const real y = cy + u * th_hat[1] + v * ph_hat[1];
            const real z = cz + u * th_hat[2] + v * ph_hat[2];
            real kx = -cx, ky = -cy, kz = -cz;
            const real kn = std::sqrt(kx * kx + ky * ky + kz * kz);
            kx /= kn; ky /= kn; kz /= kn;
            out->x0[i] = 0.0; out->x1[i] = x; out->x2[i] = y; out->x3[i] = z;
            const real X[4] = {0.0, x, y, z};
            const real K[3] = {kx, ky, kz};
            real pc[4] = {0.0, 0.0, 0.0, 0.0};
            null_covariant_momentum(X, K, p->spin, p->mass, pc);
            out->k0[i] = pc[0]; out->k1[i] = pc[1]; out->k2[i] = pc[2]; out->k3[i] = pc[3];
            out->I[i] = out->Q[i] = out->U[i] = out->V[i] = 0.0;
            out->dlambda[i] = p->initial_step * D;
            out->terminate[i] = 0;
            out->phase[i] = GRT_PHASE_IMAGE_BACKWARD;
            out->theta_disp[i] = u;
            out->phi_disp[i] = v;
        }
    }
    return 0;
}

// Line-of-sight forward rays (no counterpart in the reference initialisers;
// the functor handles them as ImageForward photons): pixel-centre rays that
// start on the plane -back * n behind the scene, aimed along the camera normal
// n, with I = 0, frequency = custom_frequency_hz, emission_frame_energy = -p_t
// and dlambda = initial_step * back.
int oracle_init_forward_photons(const grt_params* p, uint64_t nx, uint64_t ny, double back, uint64_t id_offset,
                                grt_photon_soa* out) {
    const real D = p->camera_distance;
    const real cx = D * std::sin(p->camera_theta) * std::cos(p->camera_phi);
    const real cy = D * std::sin(p->camera_theta) * std::sin(p->camera_phi);
    const real cz = D * std::cos(p->camera_theta);
    const real bx = -back * std::sin(p->camera_theta) * std::cos(p->camera_phi);
    const real by = -back * std::sin(p->camera_theta) * std::sin(p->camera_phi);
    const real bz = -back * std::cos(p->camera_theta);
    const real th_hat[3] = {std::cos(p->camera_theta) * std::cos(p->camera_phi),
                            std::cos(p->camera_theta) * std::sin(p->camera_phi), -std::sin(p->camera_theta)};
    const real ph_hat[3] = {-std::sin(p->camera_phi), std::cos(p->camera_phi), 0.0};
    for (uint64_t iy = 0; iy < ny; ++iy) {
        for (uint64_t ix = 0; ix < nx; ++ix) {
            const uint64_t i = iy * nx + ix;
            const real u = -0.5 * p->camera_width + (static_cast<real>(ix) + 0.5) * p->camera_width / static_cast<real>(nx);
            const real v = -0.5 * p->camera_height + (static_cast<real>(iy) + 0.5) * p->camera_height / static_cast<real>(ny);
            const real x = bx + u * th_hat[0] + v * ph_hat[0];
            const real y = by + u * th_hat[1] + v * ph_hat[1];
            const real z = bz + u * th_hat[2] + v * ph_hat[2];
            real kx = cx, ky = cy, kz = cz;
            const real kn = std::sqrt(kx * kx + ky * ky + kz * kz);
            kx /= kn; ky /= kn; kz /= kn;
            const real X[4] = {0.0, x, y, z};
            const real K[3] = {kx, ky, kz};
            real pc[4] = {0.0, 0.0, 0.0, 0.0};
            null_covariant_momentum(X, K, p->spin, p->mass, pc);
            out->id[i] = id_offset + i;
            out->frequency[i] = p->custom_frequency_hz;
            out->emission_frame_energy[i] = -pc[0];
            out->x0[i] = 0.0; out->x1[i] = x; out->x2[i] = y; out->x3[i] = z;
            out->k0[i] = pc[0]; out->k1[i] = pc[1]; out->k2[i] = pc[2]; out->k3[i] = pc[3];
            out->I[i] = out->Q[i] = out->U[i] = out->V[i] = 0.0;
            out->dlambda[i] = p->initial_step * back;
            out->terminate[i] = 0;
            out->phase[i] = GRT_PHASE_IMAGE_FORWARD;
            out->theta_disp[i] = u;
            out->phi_disp[i] = v;
        }
    }
    return 0;
}

// observation.hpp:31-84
int oracle_image_products(const grt_params* p, const grt_photon_soa* s, size_t n,
                          grt_image_products* out) {
    const size_t nx = p->image_nx, ny = p->image_ny, bins = p->spectrum_bins;
    for (size_t q = 0; q < nx * ny; ++q) out->image_I[q] = out->image_Q[q] = out->image_U[q] = out->image_V[q] = 0.0;
    const real lmin = std::log10(p->spectrum_min_hz), lmax = std::log10(p->spectrum_max_hz);
    for (size_t b = 0; b < bins; ++b) {
        const real f = bins > 1 ? static_cast<real>(b) / static_cast<real>(bins - 1) : 0.0;
        out->spectrum_frequency_hz[b] = std::pow(real(10.0), lmin + f * (lmax - lmin));
        out->spectrum_I[b] = 0.0;
    }
    uint64_t arrived = 0;
    for (size_t i = 0; i < n; ++i) {
        if (s->phase[i] != GRT_PHASE_IMAGE_ARRIVED) continue;
        ++arrived;
        const size_t px = observation_bin(s->theta_disp[i], -0.5 * p->camera_width, 0.5 * p->camera_width, nx);
        const size_t py = observation_bin(s->phi_disp[i], -0.5 * p->camera_height, 0.5 * p->camera_height, ny);
        const size_t pix = py * nx + px;
        out->image_I[pix] += s->I[i];
        out->image_Q[pix] += s->Q[i];
        out->image_U[pix] += s->U[i];
        out->image_V[pix] += s->V[i];
        const real f = s->frequency[i];
        if (f >= p->spectrum_min_hz && f <= p->spectrum_max_hz) {
            const size_t b = observation_bin(std::log10(f), lmin, lmax, bins);
            out->spectrum_I[b] += s->I[i];
        }
    }
    out->arrived_count[0] = arrived;
    return 0;
}

// ---- unit-level entry points for the known-answer tests ----
void oracle_hamiltonian_rhs(const double X[4], const double p[4], double a, double M, double rhs[8]) {
    hamiltonian_rhs(X, p, a, M, rhs);
}
double oracle_compute_r(double x, double y, double z, double a) { return compute_r(x, y, z, a); }
void oracle_metric(const double X[4], double a, double M, double g[16]) {
    compute_metric(X, a, M, reinterpret_cast<double(*)[4]>(g));
}
void oracle_inverse_metric(const double X[4], double a, double M, double g[16]) {
    compute_inverse_metric(X, a, M, reinterpret_cast<double(*)[4]>(g));
}
void oracle_inverse_metric_deriv(const double X[4], double a, double M, double d[64]) {
    compute_inverse_metric_deriv(X, a, M, reinterpret_cast<double(*)[4][4]>(d));
}
int oracle_null_momentum(const double X[4], const double K[3], double a, double M, double p[4]) {
    return null_covariant_momentum(X, K, a, M, p) ? 1 : 0;
}
double oracle_norm(const double X[4], const double V[4], double a, double M) {
    return kerr_schild_norm(X, V, a, M);
}
// rk4/rk45 of the photon ODE with the functor's parameters (p supplies spin, mass, tolerances)
void oracle_rk4_step(const grt_params* p, double s[8], double dt) {
    Stepper st{p, nullptr, false, false, false};
    st.rk4(s, dt);
}
int oracle_rk45_step(const grt_params* p, double s[8], double* dl) {
    Stepper st{p, nullptr, false, false, false};
    double k1[8];
    st.rhs(s, k1);
    return st.rk45(s, dl, k1);
}
int oracle_locate_cell(size_t nr, size_t nth, size_t nph, const double* r, const double* th,
                       const double* ph, double radius, double polar, double azimuth, int ijk[3]) {
    Grid g;
    g.nr = nr; g.nth = nth; g.nph = nph; g.r = r; g.th = th; g.ph = ph;
    int i = -1, j = -1, k = -1;
    const bool ok = locate_cell(g, radius, polar, azimuth, i, j, k);
    ijk[0] = i; ijk[1] = j; ijk[2] = k;
    return ok ? 1 : 0;
}
// sample_scattering_fluid on a full grid; fluid_out[14] = position_cm[3], t_s, rho, T,
// magnetic_gauss[4], u[4]; tetrad_out[16]; returns 1 if sampled.
int oracle_sample_fluid(const grt_params* p, size_t nr, size_t nth, size_t nph, const double* r,
                        const double* th, const double* ph, const double* rho, const double* T,
                        const double* vel, const double* mag, const double state[8],
                        double fluid_out[14], double tetrad_out[16], int* cell) {
    Grid g = make_grid(p, nr, nth, nph, r, th, ph, rho, T, vel, mag);
    FluidCellCGS f;
    real e[4][4];
    const bool ok = sample_fluid(state, g, f, e, cell);
    if (!ok) return 0;
    for (int q = 0; q < 3; ++q) fluid_out[q] = f.position_cm[q];
    fluid_out[3] = f.coordinate_time_s;
    fluid_out[4] = f.density_g_cm3;
    fluid_out[5] = f.temperature_k;
    for (int q = 0; q < 4; ++q) fluid_out[6 + q] = f.magnetic_gauss[q];
    for (int q = 0; q < 4; ++q) fluid_out[10 + q] = f.coordinate_four_velocity_cm_s[q];
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b) tetrad_out[a * 4 + b] = e[a][b];
    return 1;
}
void oracle_apply_rt(double stokes[4], double density, double temperature, double nu, double path,
                     int abs_on, int emis_on, double kappa, double jcoef) {
    FluidCellCGS f;
    f.density_g_cm3 = density;
    f.temperature_k = temperature;
    apply_rt(stokes, f, nu, path, abs_on != 0, emis_on != 0, kappa, jcoef);
}
void oracle_philox_block(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    Philox::block(ctr, key, out);
}
double oracle_philox_drand(uint64_t seed, uint64_t id, uint32_t domain, int index) {
    Philox rng(seed, id, domain);
    double d = 0.0;
    for (int q = 0; q <= index; ++q) d = rng.drand();
    return d;
}
void oracle_set_pow_mode(int mode) { g_pow_mode = mode; }
void oracle_det_sincos(const double* x, uint64_t n, double* s, double* c) {
    for (uint64_t i = 0; i < n; ++i) grt::det_sincos(x[i], s + i, c + i);
}
// Element-wise: out_libm[i] = std::pow(x[i], 0.25) from this host's libm,
// out_product[i] = the kernels' grt::pow_quarter compiled for the host; the two
// must agree bit for bit.
void oracle_pow_quarter_pair(const double* x, uint64_t n, double* out_libm, double* out_product) {
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < static_cast<long long>(n); ++i) {
        out_libm[i] = std::pow(x[i], 0.25);
        out_product[i] = grt::pow_quarter(x[i]);
    }
}
// Algorithmic op counts (add+sub, mul, div, sqrt, pow) of one RHS, one RK4
// step and one RKF45 attempt (with k1 given) at the state X/P, from the
// Counted instantiation; checks[3] = max |Counted - double| over the results.
void oracle_op_counts(const grt_params* p, const double X[4], const double P[4], double dl,
                      uint64_t rhs_ops[5], uint64_t rk4_ops[5], uint64_t rk45_ops[5], double checks[3]) {
    using opcount::N;
    auto take = [](uint64_t out[5]) {
        const opcount::Counter c = opcount::g;
        out[0] = c.add; out[1] = c.mul; out[2] = c.div; out[3] = c.sqrt; out[4] = c.pow;
        opcount::g = opcount::Counter();
    };
    const N a(p->spin), M(p->mass);
    N Xn[4], Pn[4], o[8];
    for (int q = 0; q < 4; ++q) { Xn[q] = N(X[q]); Pn[q] = N(P[q]); }
    opcount::g = opcount::Counter();
    opcount::rhs<N>(Xn, Pn, a, M, o);
    take(rhs_ops);
    double od[8];
    hamiltonian_rhs(X, P, p->spin, p->mass, od);
    checks[0] = 0.0;
    for (int q = 0; q < 8; ++q) checks[0] = std::fmax(checks[0], std::fabs(od[q] - o[q].v));
    N s[8];
    double sd[8];
    for (int q = 0; q < 4; ++q) { s[q] = N(X[q]); s[4 + q] = N(P[q]); sd[q] = X[q]; sd[4 + q] = P[q]; }
    opcount::rk4<N>(s, N(dl), a, M);
    take(rk4_ops);
    Stepper st{p, nullptr, false, false, false};
    st.rk4(sd, dl);
    checks[1] = 0.0;
    for (int q = 0; q < 8; ++q) checks[1] = std::fmax(checks[1], std::fabs(sd[q] - s[q].v));
    N k1[8], s2[8];
    double sd2[8], kd[8];
    for (int q = 0; q < 4; ++q) { s2[q] = N(X[q]); s2[4 + q] = N(P[q]); sd2[q] = X[q]; sd2[4 + q] = P[q]; }
    opcount::rhs_s<N>(s2, a, M, k1);
    opcount::g = opcount::Counter();
    N dln(dl);
    opcount::rk45_attempt<N>(s2, dln, k1, a, M, N(p->atol), N(p->rtol));
    take(rk45_ops);
    st.rhs(sd2, kd);
    double dld = dl;
    st.rk45(sd2, &dld, kd);
    checks[2] = std::fabs(dld - dln.v);
    for (int q = 0; q < 8; ++q) checks[2] = std::fmax(checks[2], std::fabs(sd2[q] - s2[q].v));
}

uint64_t oracle_observation_bin(double value, double lo, double hi, uint64_t bins) {
    return observation_bin(value, lo, hi, bins);
}

}  // extern "C"
