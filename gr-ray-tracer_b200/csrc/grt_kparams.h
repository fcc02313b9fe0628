// Parameter block passed by value to the trace kernels (one __grid_constant__
// struct per launch), built on the host from grt_params by grt_api.cu.
#pragma once

#include <stdint.h>
#include <vector_types.h>

namespace grt {

// Device view of the fluid grid (replaces ScatteringFluidGrid,
// src/radiative_transfer/scattering.hpp:22-39).
struct KGrid {
    int nr, nth, nph;
    int available;   // fluid present (integrate_cart_ks.hpp:436-445)
    int separable;   // coordinates are sorted per-axis products (fast lookup path)
    int pad;
    const double* r_axis;   // [nr]   separable axes (staged into shared memory)
    const double* th_axis;  // [nth]
    const double* ph_axis;  // [nph]
    // within-cell acceptance half-widths per separable axis value, computed
    // on the host exactly as scattering.hpp:99-149 computes them per call:
    // 0.500001 * (largest neighbour span), or 1e-10 for a one-value axis
    const double* r_half;   // [nr]   (log spacing)
    const double* th_half;  // [nth]
    const double* ph_half;  // [nph]  (periodic spacing)
    const double* r3;       // [nr*nth*nph] full coordinates (general path)
    const double* th3;
    const double* ph3;
    const double2* rho_t;   // [ncells] (rho, T) in code units
    const double2* vel;     // [2*ncells] Cartesian KS u^mu * velocity scale
    const double2* mag;     // [2*ncells] Cartesian KS b^mu * magnetic scale
    double r_reject_lo;     // radii outside [lo, hi] cannot pass within_radial_cell
    double r_reject_hi;
    // Raw reference layout (allocation-free entry point): the seven arrays as
    // loaded from the NumPy inputs, four-vectors converted per sample.
    const double* rho_raw;  // [ncells]
    const double* T_raw;    // [ncells]
    const double* vel_raw;  // [ncells*4] spherical KS components
    const double* mag_raw;  // [ncells*4]
    double vel_scale, mag_scale;
};

// Device structure-of-arrays photon state (struct Photons, src/utils.hpp:40-133).
struct KPhotons {
    uint64_t* id;
    double* frequency;
    double* emission_frame_energy;
    double* x0; double* x1; double* x2; double* x3;
    double* k0; double* k1; double* k2; double* k3;
    double* I; double* Q; double* U; double* V;
    double* dlambda;
    double* theta_disp;
    double* phi_disp;
    uint8_t* terminate;
    uint8_t* phase;
};

// Counters one trace launch accumulates (all zeroed before the launch).
// Per-SM first-claim counters (KParams::sm_claims), indexed by %smid.
constexpr unsigned kSmClaimSlots = 1024;

struct KCounters {
    unsigned long long queue_head;        // next photon index to hand out
    unsigned long long terminated;        // photons that terminated in this launch
    unsigned long long accepted;          // accepted ray-steps
    unsigned long long rejected;          // rejected RK45 attempts
    unsigned long long calls;             // functor invocations on live photons
    unsigned long long max_term_step;     // largest global step index at which a photon terminated, +1
    unsigned long long timed_out;         // warps that hit their iteration limit
    unsigned long long pad;
};

// One image of a launch: the camera plane of integrate_cart_ks.hpp:96-107
// (basis computed on the host with libm, as the reference computes it) and
// the image's radiative coefficients -- custom generator frequency and the
// absorption/emission coefficients (frequency channels of a batch differ here).
struct KImage {
    double cam_D, cam_W, cam_H;
    double cam_n[3], cam_th[3], cam_ph[3];
    double nu_custom, kappa, jcoef;
    double pad;
};

struct KParams {
    // physics
    double a, M;
    double r_min, r_max;
    double atol, rtol, min_scale, max_scale, safety;
    double albedo;
    double length_scale, time_scale, density_scale, temperature_scale;
    double norm, energy, pl_slope, nu_min, nu_max;
    uint64_t seed;             // scattering.seed + rank
    int integrator;            // GRT_RK4 / GRT_RK45
    int image_mode;            // simulation.mode == image
    int abs_on, emis_on, scat_on;  // already ANDed with fluid availability
    int generator;
    // the single image of a one-image launch (nimages == 0)
    KImage img0;
    // batched launch: photon index q belongs to image b when
    // image_start[b] <= q < image_start[b + 1]; nimages == 0 uses img0
    const KImage* images;
    const unsigned long long* image_start;  // [nimages + 1]
    int nimages;
    // Channel groups (batched launch, scattering off): images with the same
    // camera and screen share one geodesic per pixel; queue index q in group g
    // is pixel q - group_qstart[g] of the images chan_img[group_chan[g] ..
    // group_chan[g + 1]) (the first is the group's lead).  0 = no sharing.
    int ngroups;
    const unsigned long long* group_qstart;  // [ngroups + 1]
    const int* group_chan;                  // [ngroups + 1]
    const int* chan_img;                    // [channels]
    KGrid grid;
    KPhotons ph;
    uint64_t n;                // photons in the queue
    int64_t step0;             // global step index of this launch's first call
    int64_t budget;            // calls each live photon may take in this launch
    unsigned long long max_iterations;  // per-warp loop limit (GRT_ETIMEOUT)
    KCounters* counters;
    // two-launch image mode (trace_body LEG 1 then 2): calls each photon took
    // in the backward-leg launch, by queue index, zeroed before it
    long long* calls_carry;
    // channel groups: (lead channel << 32) | finished-channel mask of each
    // geodesic as the last launch left it; zeroed with the photons' init
    // (nullptr: channel 0 leads and none finished)
    unsigned long long* share_state;
    // first-fill balance: when every queue claim fits in the resident warps,
    // a warp's first claim is allowed only while its SM (%smid) has taken
    // fewer than sm_quota first claims (sm_claims: kSmClaimSlots counters,
    // zeroed before each launch); 0 = off
    unsigned* sm_claims;
    unsigned sm_quota;
    // image mode: queue position -> queue index, so that each warp's 32
    // claims are an 8 x 4 tile of one image's pixels (nullptr = identity)
    const unsigned* order;
    int refill_threshold;      // idle lanes before a warp refills (1..32)
    int grab;                  // photons claimed per queue access (per warp)
    const double* m_abs;       // optional per-cell multipliers on dtau (nullptr = 1)
    const double* m_emis;      // optional per-cell multipliers on dI
    // mixed-precision form only
    double fp64_radius_sq;     // x^2+y^2+z^2 below this uses the FP64 right-hand side
    double fp64_axis_sin2;     // (x^2+y^2)/(x^2+y^2+z^2) below this (polar axis) uses FP64
    double fp32_min_radius_sq; // RK45 calls start r^2 above this (outside the fluid grid) for FP32
    int renormalize;           // restore g^{mu nu} p_mu p_nu = 0 in FP64 after each accepted step
    // spin and mass inside the range where the FP64 right-hand side may use
    // reciprocal quotients (ks_rhs_rcp): |a| = 0 or in [2^-20, 2], M in [2^-20, 2^20]
    int rcp_ok;
};

}  // namespace grt
