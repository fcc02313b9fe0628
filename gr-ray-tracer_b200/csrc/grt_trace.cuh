// Persistent trace kernel body, templated on the right-hand-side policy.
//
// Replaces the host step loop's per-step launch of the reference functor
// (src/geodesic_integrate/integrate_cart_ks.hpp:468-481, operator() :230-419):
// one launch advances every photon by up to `budget` functor invocations
// ("calls"), keeping its state in registers between calls.  Photons are
// independent, so this is exactly the reference's result whenever no
// termination check falls inside the launch (the host splits launches at the
// reference's output steps when termination_percent < 1).
//
// Work distribution: each warp claims contiguous blocks of `grab` photon
// indices from a global queue; lanes whose photon terminated (or used its
// budget) stay idle until at least `refill_threshold` lanes are idle, then the
// warp hands them the next indices with one ballot + prefix rank.  A loop
// iteration is one unit of work per lane: a complete RK4 call, or one RK45
// attempt (rejected attempts no longer hold the whole warp for 12 tries).
#pragma once

#include "grt_device.cuh"
#include "grt_pow_quarter.cuh"

namespace grt {
namespace dev {

constexpr unsigned kFull = 0xFFFFFFFFu;

// Fehlberg 4(5) tableau (integrate_cart_ks.hpp:166-180).
constexpr double a21 = 1.0 / 4.0;
constexpr double a31 = 3.0 / 32.0, a32 = 9.0 / 32.0;
constexpr double a41 = 1932.0 / 2197.0, a42 = -7200.0 / 2197.0, a43 = 7296.0 / 2197.0;
constexpr double a51 = 439.0 / 216.0, a52 = -8.0, a53 = 3680.0 / 513.0, a54 = -845.0 / 4104.0;
constexpr double a61 = -8.0 / 27.0, a62 = 2.0, a63 = -3544.0 / 2565.0, a64 = 1859.0 / 4104.0,
                 a65 = -11.0 / 40.0;
constexpr double b41 = 25.0 / 216.0, b43 = 1408.0 / 2565.0, b44 = 2197.0 / 4104.0, b45 = -1.0 / 5.0;
constexpr double b51 = 16.0 / 135.0, b53 = 6656.0 / 12825.0, b54 = 28561.0 / 56430.0,
                 b55 = -9.0 / 50.0, b56 = 2.0 / 55.0;

// The seven evolving components of the state (t,x,y,z,px,py,pz); p_t is constant.
struct V7 {
    double v[7];
};

GRT_DEV V7 to_v7(const Rhs7& r) {
    V7 o;
    o.v[0] = r.t; o.v[1] = r.x; o.v[2] = r.y; o.v[3] = r.z;
    o.v[4] = r.px; o.v[5] = r.py; o.v[6] = r.pz;
    return o;
}

// state index of V7 component c
GRT_DEV constexpr int sidx(int c) { return c < 4 ? c : c + 1; }

// ks_rhs with IEEE divisions, out of line: the right-hand side outside the
// box of ks_rhs_rcp.
static __device__ __noinline__ Rhs7 ks_rhs_ieee(double x, double y, double z, double pt, double px, double py,
                                                double pz, double a, double M) {
    return ks_rhs(x, y, z, pt, px, py, pz, a, M);
}

// Right-hand-side policy of the FP64 parity form: ks_rhs_rcp (reciprocal
// quotients that round like IEEE divisions) inside its box, ks_rhs outside;
// both give ks_rhs's result bit for bit.  BF: ks_rhs_rcp with the branch-free
// reciprocal and square root (grt_rn.cuh), which a lone warp per scheduler
// runs faster (C1's 4,096 rays: 3% on the trace) and the disk-mode kernel,
// at 170 registers, slower (2%); the image-mode kernels use it.
// LAT: the instantiation is latency-bound (one warp or so per scheduler: the
// 2-blocks/SM kernels), where the mixed form's renormalisation with the
// branch-free functions and the branch-free Kerr-Schild radius (ks_radius_bf)
// measured 4.6% faster on C1; at 4 blocks/SM and 128 registers the radius
// measured 1% slower, so the others keep ks_radius.
// `fast` is the per-call precision hint of the mixed form (ignored here).
template <bool BF, bool LAT = false>
struct Fp64RhsT {
    static constexpr bool kLatency = LAT;
    static GRT_DEV V7 eval(const double s[8], const KParams& kp, int /*fast*/) {
        if (kp.rcp_ok) {
            bool ok;
            const Rhs7 o = ks_rhs_rcp<BF>(s[1], s[2], s[3], s[4], s[5], s[6], s[7], kp.a, kp.M, ok);
            if (ok) return to_v7(o);
        }
        return to_v7(ks_rhs_ieee(s[1], s[2], s[3], s[4], s[5], s[6], s[7], kp.a, kp.M));
    }
    // nothing to do after an accepted step; no radius computed (-1)
    static GRT_DEV double after_accept(double*, const KParams&, int) { return -1.0; }
};
using Fp64Rhs = Fp64RhsT<false>;

struct Lane {
    double s[8];
    double I[4];
    double freq, emit, dl;
    double radius;        // ks_radius of s, valid when have_radius
    uint64_t id;
    long long idx;        // photon index, -1 when idle
    long long q;          // queue index of the lane's photon (geodesic index when sharing)
    long long calls;      // calls taken in this launch
    int phase;
    int have_radius;
    // RK45 call in progress
    int mid_call;
    int attempts;
    int img;              // image of a batched launch (0 otherwise)
    // channel group of a sharing launch: the lane traces the geodesic of
    // pixel `pix` for every channel image of group `grp`; channel `lead`
    // lives in registers, the others in their own photon slots
    int grp, lead, nchan;
    unsigned done;        // channels already finished (written) on their own
    int zero_all;         // a shared event zeroed every channel's Stokes vector
    long long pix;
    int fast;             // precision hint of the current call (mixed form)
    int gen_pending;      // backward-leg launch: stopped at first fluid contact, generation left to generate_body
    int need_k1;          // the call's k1 = f(state) is still to be evaluated
    double dl_try;
};

// GEO: the backward-leg launch, which neither reads nor changes a photon's
// id, frequency, emission-frame energy, Stokes vector or screen position
// (generation happens in generate_body; transfer, scattering and arrival in
// the forward-leg launch): only the geodesic part is loaded and stored, and the Stokes vector
// only zeroed, which keeps those fields out of the lane's registers.
template <bool GEO = false>
GRT_DEV void load_photon(const KPhotons& P, long long i, Lane& L) {
    if (!GEO) {
        L.id = P.id[i];
        L.freq = P.frequency[i];
        L.emit = P.emission_frame_energy[i];
        L.I[0] = P.I[i]; L.I[1] = P.Q[i]; L.I[2] = P.U[i]; L.I[3] = P.V[i];
    }
    L.s[0] = P.x0[i]; L.s[1] = P.x1[i]; L.s[2] = P.x2[i]; L.s[3] = P.x3[i];
    L.s[4] = P.k0[i]; L.s[5] = P.k1[i]; L.s[6] = P.k2[i]; L.s[7] = P.k3[i];
    L.dl = P.dlambda[i];
    L.phase = P.phase[i];
    L.calls = 0;
    L.have_radius = 0;
    L.mid_call = 0;
    L.gen_pending = 0;
    L.zero_all = 0;
}

template <bool GEO = false>
GRT_DEV void store_photon(const KPhotons& P, const Lane& L, int terminated, double tdisp, double pdisp,
                          int have_disp) {
    const long long i = L.idx;
    if (!GEO) {
        P.frequency[i] = L.freq;
        P.emission_frame_energy[i] = L.emit;
        P.I[i] = L.I[0]; P.Q[i] = L.I[1]; P.U[i] = L.I[2]; P.V[i] = L.I[3];
    } else if (L.zero_all) {
        P.I[i] = 0.0; P.Q[i] = 0.0; P.U[i] = 0.0; P.V[i] = 0.0;
    }
    P.x0[i] = L.s[0]; P.x1[i] = L.s[1]; P.x2[i] = L.s[2]; P.x3[i] = L.s[3];
    P.k0[i] = L.s[4]; P.k1[i] = L.s[5]; P.k2[i] = L.s[6]; P.k3[i] = L.s[7];
    P.dlambda[i] = L.dl;
    if (!GEO && have_disp) {
        P.theta_disp[i] = tdisp;
        P.phi_disp[i] = pdisp;
    }
    P.terminate[i] = static_cast<uint8_t>(terminated);
    P.phase[i] = static_cast<uint8_t>(L.phase);
}

// ---- channel groups (frequency channels sharing one geodesic) ----
GRT_DEV int chan_image(const KParams& kp, int grp, int c) { return kp.chan_img[kp.group_chan[grp] + c]; }
GRT_DEV long long chan_slot(const KParams& kp, int grp, int c, long long pix) {
    return static_cast<long long>(kp.image_start[chan_image(kp, grp, c)]) + pix;
}

// Geodesic part of the photon state of channel slot i (its id, frequency and
// Stokes vector are its own and already in place).
template <bool GEO = false>
GRT_DEV void store_follower(const KPhotons& P, const Lane& L, long long i, int terminated, int phase, double tdisp,
                            double pdisp, int have_disp, int zero_stokes, double dl) {
    if (!GEO) P.emission_frame_energy[i] = L.emit;
    P.x0[i] = L.s[0]; P.x1[i] = L.s[1]; P.x2[i] = L.s[2]; P.x3[i] = L.s[3];
    P.k0[i] = L.s[4]; P.k1[i] = L.s[5]; P.k2[i] = L.s[6]; P.k3[i] = L.s[7];
    if (zero_stokes) {
        P.I[i] = 0.0; P.Q[i] = 0.0; P.U[i] = 0.0; P.V[i] = 0.0;
    }
    P.dlambda[i] = dl;
    if (!GEO && have_disp) {
        P.theta_disp[i] = tdisp;
        P.phi_disp[i] = pdisp;
    }
    P.terminate[i] = static_cast<uint8_t>(terminated);
    P.phase[i] = static_cast<uint8_t>(phase);
}

// Store the lane's photon and, in a sharing launch, every channel still riding
// on its geodesic.  Returns the number of photons stored.  GEO (the
// backward-leg launch, see load_photon): the geodesic part only, and no
// followers when the ray is handed over with its generation pending (the
// forward-leg launch stores them when the ray finishes).
template <bool SHARE, bool GEO = false>
GRT_DEV int store_all(const KParams& kp, const Lane& L, int terminated, double tdisp, double pdisp, int have_disp) {
    store_photon<GEO>(kp.ph, L, terminated, tdisp, pdisp, have_disp);
    int stored = 1;
    if (SHARE && !(GEO && L.gen_pending)) {
        for (int c = 0; c < L.nchan; ++c) {
            if (c == L.lead || ((L.done >> c) & 1u)) continue;
            store_follower<GEO>(kp.ph, L, chan_slot(kp, L.grp, c, L.pix), terminated, L.phase, tdisp, pdisp,
                                have_disp, L.zero_all, L.dl);
            ++stored;
        }
    }
    return stored;
}

// integrate_cart_ks.hpp:142-155.  One right-hand-side site inside a stage
// loop (kept rolled: a fully unrolled step overflows the instruction cache);
// only the running weighted sum ((k1 + 2 k2) + 2 k3) + k4 is kept, which adds
// the stages in the reference's order.  Stage inputs s + (c dt) k with
// c in {1/2, 1/2, 1} round exactly like the reference's s + c*dt*k.
template <class RHS>
GRT_DEV void rk4_step(double s[8], double dt, const KParams& kp, int fast) {
    double t[8];
    V7 k, sum;
    t[4] = s[4];
#pragma unroll 1
    for (int st = 0; st < 4; ++st) {
        if (st == 0) {
#pragma unroll
            for (int c = 0; c < 7; ++c) t[sidx(c)] = s[sidx(c)];
        } else {
            const double cdt = (st == 3) ? dt : 0.5 * dt;
#pragma unroll
            for (int c = 0; c < 7; ++c) t[sidx(c)] = s[sidx(c)] + cdt * k.v[c];
        }
        k = RHS::eval(t, kp, fast);
        if (st == 0) {
            sum = k;
        } else if (st == 3) {
#pragma unroll
            for (int c = 0; c < 7; ++c) sum.v[c] = sum.v[c] + k.v[c];
        } else {
#pragma unroll
            for (int c = 0; c < 7; ++c) sum.v[c] = sum.v[c] + 2.0 * k.v[c];
        }
    }
    const double h6 = dt / 6.0;
#pragma unroll
    for (int c = 0; c < 7; ++c) s[sidx(c)] += h6 * sum.v[c];
}

// Stage-input rows of the Fehlberg tableau (a_{t,j}, j < t), zero padded.
static __constant__ double kFehlbergA[5][5] = {
    {a21, 0.0, 0.0, 0.0, 0.0},
    {a31, a32, 0.0, 0.0, 0.0},
    {a41, a42, a43, 0.0, 0.0},
    {a51, a52, a53, a54, 0.0},
    {a61, a62, a63, a64, a65}};

// Trace kernels run kTraceThreads-thread blocks (the launchers and
// __launch_bounds__ use the same constant).
constexpr int kTraceThreads = 128;

// Per-thread slots in shared memory: the stage derivatives k1..k5 (slots
// 0..4; k6 replaces k2 in slot 1 once the last stage input is formed) and the
// state (slot 5) for the error norm.  [6][7][kTraceThreads] doubles,
// thread-contiguous so a warp's accesses are conflict-free; base already
// points at this thread's column, so a slot is a constant offset from it.
// k1 stays there across the retries of one call.
constexpr int kStageSlots = 6;
struct KStore {
    double* base;
    GRT_DEV double& at(int j, int c) const { return base[(j * 7 + c) * kTraceThreads]; }
};

// pow(1/err, 0.25) of the reference as glibc's pow rounds it
// (grt_pow_quarter.cuh); out of line to keep the step loop small.
static __device__ __noinline__ double controller_root(double x) { return pow_quarter(x); }

// One Fehlberg attempt (integrate_cart_ks.hpp:159-227), preceded by the
// call's k1 = f(state) when need_k1 (integrate_cart_ks.hpp:274-275); returns 1
// if accepted (s advanced), 0 if rejected; *dl receives the next proposed step
// either way.  All right-hand sides go through one site in a rolled stage
// loop -- a lane that needs k1 runs it one iteration ahead of the others, so
// the warp stays converged on the same code -- and the derivatives live in
// shared memory (KStore), which keeps registers for the right-hand side.
// The stage sums and the error norm are rolled loops too, the norm with a
// single division site: every inline IEEE division brings its slow path into
// the step loop's instruction stream, and with seven of them unrolled the
// loop missed the instruction cache far more (the unrolled form was 11-22%
// slower on C2 and C3).  Each stage input is summed over j = 1..t-1 left to
// right, the reference's association; for the first stage, dt*(a21 k1)
// equals the reference's (dt*a21)*k1 because a21 = 1/4 is a power of two.
template <class RHS>
GRT_DEV int rk45_attempt(const KParams& kp, double s[8], double* dl, int need_k1, int fast, const KStore& kk) {
    const double dt = *dl;
    double t[8];
    t[4] = s[4];
#pragma unroll 1
    for (int st = need_k1 ? -1 : 0; st < 5; ++st) {
        if (st < 0) {
#pragma unroll
            for (int c = 0; c < 7; ++c) t[sidx(c)] = s[sidx(c)];
        } else {
            double acc[7];
            const double a0 = kFehlbergA[st][0];
#pragma unroll
            for (int c = 0; c < 7; ++c) acc[c] = a0 * kk.at(0, c);
#pragma unroll 1
            for (int j = 1; j <= st; ++j) {
                const double aj = kFehlbergA[st][j];
#pragma unroll
                for (int c = 0; c < 7; ++c) acc[c] = acc[c] + aj * kk.at(j, c);
            }
#pragma unroll
            for (int c = 0; c < 7; ++c) t[sidx(c)] = s[sidx(c)] + dt * acc[c];
        }
        const V7 k = RHS::eval(t, kp, fast);
        // k2..k5 to slots 1..4; k6 replaces k2 in slot 1 (no later use)
        const int slot = st < 4 ? st + 1 : 1;
#pragma unroll
        for (int c = 0; c < 7; ++c) kk.at(slot, c) = k.v[c];
    }
    // The state goes to slot 5 so that the error norm runs as a loop over the
    // components (one division site); x5 replaces it there.
#pragma unroll
    for (int c = 0; c < 7; ++c) kk.at(5, c) = s[sidx(c)];
    double err = 0.0;
    bool finite = isfinite(s[4]);
    // The norm is max_c RN(n_c / sc_c).  Rounding is monotone, so it equals
    // RN(n_m / sc_m) for the component m of largest exact ratio, found by
    // comparing exact cross products n_c sc_m against n_m sc_c (the product
    // and its fma residual).  One division then replaces seven serial ones.
    // That needs every x4, x5 finite and n_c, sc_c inside [2^-400, 2^400]
    // (or n_c = 0), so that no product under- or overflows; otherwise the
    // ratios are formed one by one as before.  n_c and sc_c go to slots 2
    // and 3 (k3, k4: not read again in this attempt).
    bool boxed = true;
#pragma unroll 1
    for (int c = 0; c < 7; ++c) {
        const double si = kk.at(5, c);
        const double k1 = kk.at(0, c), k3 = kk.at(2, c), k4 = kk.at(3, c), k5 = kk.at(4, c), k6 = kk.at(1, c);
        const double x4 = si + dt * (b41 * k1 + b43 * k3 + b44 * k4 + b45 * k5);
        const double x5 = si + dt * (b51 * k1 + b53 * k3 + b54 * k4 + b55 * k5 + b56 * k6);
        const double sc = kp.atol + kp.rtol * fmax(fabs(x5), fabs(x4));
        const double n = fabs(x5 - x4);
        boxed = boxed && isfinite(x4) && isfinite(x5) && div_within<-400, 399>(sc) &&
                div_zero_or_within<-400, 399>(n);
        kk.at(5, c) = x5;
        kk.at(2, c) = n;
        kk.at(3, c) = sc;
    }
    if (boxed) {
        double nm = kk.at(2, 0), sm = kk.at(3, 0);
#pragma unroll 1
        for (int c = 1; c < 7; ++c) {
            const double n = kk.at(2, c), sc = kk.at(3, c);
            const double p = n * sm, q = nm * sc;
            if (p > q || (p == q && fma(n, sm, -p) > fma(nm, sc, -q))) {
                nm = n;
                sm = sc;
            }
        }
        err = div_by(nm, sm, div_recip(sm));
    } else {
#pragma unroll 1
        for (int c = 0; c < 7; ++c) {
            const double ratio = kk.at(2, c) / kk.at(3, c);
            if (!isfinite(kk.at(5, c)) || !isfinite(ratio)) finite = false;
            err = fmax(err, ratio);
        }
    }
    if (!finite) {
        *dl = dt * kp.min_scale;
        return 0;
    }
    if (err == 0.0) {
        *dl = dt * kp.max_scale;
#pragma unroll
        for (int c = 0; c < 7; ++c) s[sidx(c)] = kk.at(5, c);
        return 1;
    }
    // 1/err rounded to nearest, as the division 1.0 / err rounds it (err is
    // finite and positive here), without a second division site
    double scale = kp.safety * controller_root(div_recip(err));
    scale = fmin(kp.max_scale, fmax(kp.min_scale, scale));
    *dl = dt * scale;
    if (err <= 1.0) {
#pragma unroll
        for (int c = 0; c < 7; ++c) s[sidx(c)] = kk.at(5, c);
        return 1;
    }
    return 0;
}

struct LaneCounters {
    unsigned long long terminated, accepted, rejected, calls, max_term_step;
};

// The image a photon belongs to: the launch's only image, or the batch entry
// whose index range holds photon index q (binary search, once per load).
GRT_DEV int image_of_photon(const KParams& kp, long long q) {
    if (kp.nimages <= 0) return 0;
    int lo = 0, hi = kp.nimages - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (kp.image_start[mid] <= static_cast<unsigned long long>(q)) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

GRT_DEV const KImage& image_params(const KParams& kp, int img) { return kp.nimages > 0 ? kp.images[img] : kp.img0; }

// observation.hpp:22-29: bin of value in [lo, hi] over `bins` bins,
// floor(clamp((value - lo) / (hi - lo)) * (bins - 1)).
GRT_DEV unsigned long long observation_bin(double value, double lo, double hi, unsigned long long bins) {
    if (bins <= 1 || !(hi > lo)) return 0;
    const double f = (value - lo) / (hi - lo);
    const double sc = fmax(0.0, fmin(1.0, f));
    return static_cast<unsigned long long>(sc * static_cast<double>(bins - 1));
}

// Observer of the radiative-transfer updates of post_step (the adjoint's
// recompute records them); the trace kernels pass NoRecord, which compiles away.
struct NoRecord {
    // one RT update in cell `cell`: I = (I_before * att + m_emis * j0) * scale,
    // att = exp(-m_abs * tau0)
    GRT_DEV void rt_step(int, double, double, double, double, double) {}
    // the Stokes vector was zeroed (invalid arrival energies)
    GRT_DEV void zeroed() {}
};

// Everything after the integration step of one call (integrate_cart_ks.hpp:307-417).
// phase0 is the phase loaded at the start of the call.  Returns 1 if the photon
// terminated.
// Packet generation of photon `id` at `step` (integrate_cart_ks.hpp:325-347).
GRT_DEV bool generate_packet(const KParams& kp, const FluidSample& fs, uint64_t id, int64_t step, int packets,
                             double nu_custom, double& nu, double& E) {
    Philox rng(kp.seed, id, static_cast<uint32_t>(step));
    if (packets > 0 && kp.generator == 0) return generate_blackbody(fs.fluid, rng, packets, kp.energy, nu, E);
    if (packets > 0 && kp.generator == 1)
        return generate_power_law(rng, packets, kp.pl_slope, kp.nu_min, kp.nu_max, kp.energy, nu, E);
    if (packets > 0) return GeneratePhotonsCustom(fs.fluid, rng, packets, nu_custom, kp.energy, nu, E);
    return false;
}

// The first fluid contact of an image-backward ray (integrate_cart_ks.hpp:
// 351-363): the cell's packet count and the generator give the packet's
// frequency and energy; the ray reverses (dlambda negated) into ImageForward,
// or is Rejected when no packet is generated.  SHARE: every other channel of
// the geodesic draws with its own id and frequency; a channel rejected on its
// own is written out (counted in *ch_term), and if the lead is rejected
// another channel is promoted.  `step` is the global index of the call.
// Returns 1 if the ray terminated.
template <bool SHARE>
GRT_DEV int generate_at_contact(const KParams& kp, Lane& L, const FluidSample& fs, int64_t step, int* ch_term) {
    const KImage& im = image_params(kp, L.img);
    int terminated = 0;
    double nu = 0.0, E = 0.0;
    const double dcode = fs.fluid.density_g_cm3 / kp.density_scale;
    const int packets = ComputeSuperphotonsPerCell(dcode, kp.norm);
    bool generated = generate_packet(kp, fs, L.id, step, packets, im.nu_custom, nu, E);
    if (SHARE) {
        // every other channel draws with its own id and frequency
        int promote = -1;
        for (int c = 0; c < L.nchan; ++c) {
            if (c == L.lead || ((L.done >> c) & 1u)) continue;
            const long long sc = chan_slot(kp, L.grp, c, L.pix);
            double nu_c = 0.0, E_c = 0.0;
            const double f_c = image_params(kp, chan_image(kp, L.grp, c)).nu_custom;
            if (generate_packet(kp, fs, kp.ph.id[sc], step, packets, f_c, nu_c, E_c)) {
                kp.ph.frequency[sc] = nu_c;
                kp.ph.I[sc] = E_c;
                kp.ph.Q[sc] = 0.0;
                kp.ph.U[sc] = 0.0;
                kp.ph.V[sc] = 0.0;
                if (!generated && promote < 0) promote = c;
            } else {
                // rejected on its own: the state after this step, Stokes zeroed
                store_follower(kp.ph, L, sc, 1, 4, 0.0, 0.0, 0, 1, L.dl);
                L.done |= 1u << c;
                ++*ch_term;
            }
        }
        if (!generated && promote >= 0) {
            // the lead is rejected on its own; channel `promote` carries on
            L.I[0] = L.I[1] = L.I[2] = L.I[3] = 0.0;
            const int ph_keep = L.phase;
            L.phase = 4;
            store_photon(kp.ph, L, 1, 0.0, 0.0, 0);
            L.phase = ph_keep;
            L.done |= 1u << L.lead;
            ++*ch_term;
            const long long sc = chan_slot(kp, L.grp, promote, L.pix);
            L.lead = promote;
            L.idx = sc;
            L.id = kp.ph.id[sc];
            L.img = chan_image(kp, L.grp, promote);
            nu = kp.ph.frequency[sc];
            E = kp.ph.I[sc];
            generated = true;
        }
    }
    if (generated) {
        L.freq = nu;
        double ee = 0.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) ee -= L.s[4 + c] * fs.e[0][c];
        L.emit = ee;
        L.I[0] = E;
        L.I[1] = L.I[2] = L.I[3] = 0.0;
        L.dl = -fabs(L.dl);
        L.phase = 2;  // ImageForward
    } else {
        L.I[0] = L.I[1] = L.I[2] = L.I[3] = 0.0;
        L.phase = 4;  // Rejected
        terminated = 1;
    }
    return terminated;
}

// SHARE: the lane also carries the other channels of its group (their
// frequencies and Stokes vectors in their photon slots); *ch_term counts the
// channels that terminated on their own in this call.
// LEG (see trace_body) removes the code the leg never runs: generation from
// the forward leg, transfer and the camera from the backward leg.
// radius_hint: the Kerr-Schild radius of L.s when the caller already has it
// (the mixed form's renormalisation computes it), else negative.  FASTR: the
// radius through ks_radius_bf (latency-bound instantiations).
template <bool RAW = false, class Rec = NoRecord, bool SHARE = false, int LEG = 0, bool FASTR = false>
GRT_DEV int post_step(const KParams& kp, const Axes& ax, Lane& L, int phase0, double taken, int64_t step,
                      double& tdisp, double& pdisp, int& have_disp, Rec rec = Rec(), int* ch_term = nullptr,
                      double radius_hint = -1.0) {
    const KImage& im = image_params(kp, L.img);
    if (radius_hint >= 0.0) L.radius = radius_hint;
    else L.radius = FASTR ? ks_radius_bf(L.s[1], L.s[2], L.s[3], kp.a) : ks_radius(L.s[1], L.s[2], L.s[3], kp.a);
    L.have_radius = 1;
    const bool backward = phase0 == 1;  // ImageBackward
    // LEG 3 (disk mode) compiles the image-mode branches out of the step loop
    const bool image_mode = LEG != 3 && kp.image_mode;
    const bool needs = kp.scat_on || kp.abs_on || kp.emis_on || (image_mode && backward);
    FluidSample fs;
    const bool sampled = needs && sample_fluid<RAW>(kp, ax, L.s, L.radius, fs);
    int terminated = 0;
    if (LEG != 2 && image_mode && backward && sampled) {
        if (LEG == 1) {
            // the backward-leg launch stops here: generate_body samples
            // this position again and generates (one call, split)
            L.gen_pending = 1;
        } else {
            terminated = generate_at_contact<SHARE>(kp, L, fs, step, ch_term);
        }
    } else if (LEG != 1 && sampled && !backward) {
        const double I_before = L.I[0];
        double tau0 = 0.0, j0 = 0.0, att = 1.0, scale = 1.0;
        if (kp.abs_on) {
            double dtau = ComputeOpticalDepthIncrement(fs.fluid, L.freq, taken, im.kappa);
            tau0 = dtau;
            if (kp.m_abs) dtau = kp.m_abs[fs.cell] * dtau;
            att = exp(-dtau);
#pragma unroll
            for (int q = 0; q < 4; ++q) L.I[q] *= att;
        }
        if (kp.emis_on) {
            double dI = ComputeEmissivityIncrement(fs.fluid, L.freq, taken, im.jcoef);
            j0 = dI;
            if (kp.m_emis) dI = kp.m_emis[fs.cell] * dI;
            L.I[0] += dI;
        }
        if (SHARE && (kp.abs_on || kp.emis_on)) {
            for (int c = 0; c < L.nchan; ++c) {
                if (c == L.lead || ((L.done >> c) & 1u)) continue;
                const long long sc = chan_slot(kp, L.grp, c, L.pix);
                const KImage& ic = image_params(kp, chan_image(kp, L.grp, c));
                const double f_c = kp.ph.frequency[sc];
                double Ic[4] = {kp.ph.I[sc], kp.ph.Q[sc], kp.ph.U[sc], kp.ph.V[sc]};
                if (kp.abs_on) {
                    double dtau = ComputeOpticalDepthIncrement(fs.fluid, f_c, taken, ic.kappa);
                    if (kp.m_abs) dtau = kp.m_abs[fs.cell] * dtau;
                    const double att_c = exp(-dtau);
                    for (int q = 0; q < 4; ++q) Ic[q] *= att_c;
                }
                if (kp.emis_on) {
                    double dI = ComputeEmissivityIncrement(fs.fluid, f_c, taken, ic.jcoef);
                    if (kp.m_emis) dI = kp.m_emis[fs.cell] * dI;
                    Ic[0] += dI;
                }
                kp.ph.I[sc] = Ic[0];
                kp.ph.Q[sc] = Ic[1];
                kp.ph.U[sc] = Ic[2];
                kp.ph.V[sc] = Ic[3];
            }
        }
        if (kp.scat_on) {
            Philox rng(kp.seed, L.id, static_cast<uint32_t>(step));
            if (scatter_drawn(fabs(L.dl), kp.length_scale, fs, rng)) {
                ScatterState st;
#pragma unroll
                for (int c = 0; c < 8; ++c) st.s[c] = L.s[c];
#pragma unroll
                for (int q = 0; q < 4; ++q) st.I[q] = L.I[q];
                if (scatter_packet(&st, kp.albedo, fs, kp.a, kp.M, &rng)) {
#pragma unroll
                    for (int c = 4; c < 8; ++c) L.s[c] = st.s[c];
#pragma unroll
                    for (int q = 0; q < 4; ++q) L.I[q] = st.I[q];
                    scale = kp.albedo;
                }
            }
        }
        rec.rt_step(fs.cell, tau0, j0, I_before, att, scale);
    }
    if (LEG != 1 && image_mode && phase0 == 2) {  // ImageForward
        double u = 0.0, v = 0.0;
        const int crossing = camera_crossing(im, L.s, u, v);
        if (crossing > 0) {
            const double eo = camera_observer_energy(kp, L.s);
            const double ee = L.emit;
            if (eo > 0.0 && ee > 0.0 && isfinite(eo) && isfinite(ee)) {
                L.freq *= eo / ee;
                if (SHARE) {
                    for (int c = 0; c < L.nchan; ++c) {
                        if (c == L.lead || ((L.done >> c) & 1u)) continue;
                        const long long sc = chan_slot(kp, L.grp, c, L.pix);
                        kp.ph.frequency[sc] *= eo / ee;
                    }
                }
            } else {
                L.I[0] = L.I[1] = L.I[2] = L.I[3] = 0.0;
                L.zero_all = 1;
                rec.zeroed();
            }
            tdisp = u;
            pdisp = v;
            have_disp = 1;
            L.phase = 3;  // ImageArrived
            terminated = 1;
        } else if (crossing < 0) {
            L.I[0] = L.I[1] = L.I[2] = L.I[3] = 0.0;
            L.zero_all = 1;
            L.phase = 4;
            terminated = 1;
        }
    }
    return terminated;
}

// State of a live photon that the next launch over the queue needs besides
// its photon slot: the calls taken (backward leg to forward leg) and, when
// channels share the geodesic, which channel leads and which finished.
// A photon the backward-leg launch stopped at its first fluid contact is
// carried as -(calls + 1).
template <bool SHARE, int LEG>
GRT_DEV void store_carry(const KParams& kp, const Lane& L) {
    if (LEG == 1) kp.calls_carry[L.q] = L.gen_pending ? -(L.calls + 1) : L.calls;
    if (SHARE && kp.share_state)
        kp.share_state[L.q] = (static_cast<unsigned long long>(L.lead) << 32) | L.done;
}

// SHARE: queue indices are geodesics of channel groups (KParams::ngroups > 0).
// LEG splits an image-mode launch into two trace launches over the same queue,
// with the generate_pending kernel between them:
//   0  whole rays (disk mode, or image mode in one launch);
//   1  the backward leg: photons in ImageBackward only; a lane hands its
//      photon over at its first fluid contact, before the packet generation
//      of that call -- stored like a budget end, with the calls taken so far
//      in KParams::calls_carry[q] (negated: -(calls + 1), generation pending);
//      generate_body then finishes those calls, one thread per photon;
//   2  everything after: photons in any live phase but ImageBackward,
//      resuming with the calls left in calls_carry[q];
//   3  disk mode: whole rays like 0, with the image-mode branches (packet
//      generation at first contact, camera arrival) compiled out, which keeps
//      the step loop's code small for the instruction cache.
// Each photon takes the same calls in the same order either way, so the split
// launches give the one-launch result bit for bit; each loop body holds only
// its own leg's code.
template <int INTEGRATOR, class RHS, bool RAW = false, bool SHARE = false, int LEG = 0>
GRT_DEV void trace_body(const KParams& kp, const Axes& ax, const KStore& kk) {
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    Lane L;
    L.idx = -1;
    LaneCounters cnt = {0, 0, 0, 0, 0};
    bool exhausted = false;
    bool first_claim = true;
    unsigned long long local_next = 0, local_end = 0;
    unsigned long long iters = 0;
    bool timed_out = false;
    double tdisp = 0.0, pdisp = 0.0;
    int have_disp = 0;

    while (true) {
        // ---- refill idle lanes from the warp's block / the global queue ----
        const unsigned idle = __ballot_sync(kFull, L.idx < 0);
        if (idle && !(exhausted && local_next >= local_end)) {
            const int nidle = __popc(idle);
            if (nidle >= kp.refill_threshold || idle == kFull) {
                unsigned long long base_a = local_next;
                unsigned long long take_a = local_end - local_next;
                if (take_a > static_cast<unsigned long long>(nidle)) take_a = nidle;
                local_next += take_a;
                unsigned long long base_b = 0, take_b = 0;
                if (first_claim && kp.sm_quota) {
                    // Spread the first fill evenly over the SMs: a warp whose
                    // SM has its share of first claims already takes nothing
                    // and ends; the other SMs' warps take the rest.  Without
                    // it the first warps to start take every claim, and few
                    // rays crowd onto a few SMs (C1's 128 warps: 30% slower).
                    unsigned allowed = 1;
                    if (lane == 0) {
                        unsigned sm;
                        asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
                        if (sm < kSmClaimSlots) allowed = atomicAdd(&kp.sm_claims[sm], 1u) < kp.sm_quota;
                    }
                    if (!__shfl_sync(kFull, allowed, 0)) exhausted = true;
                }
                first_claim = false;
                if (take_a < static_cast<unsigned long long>(nidle) && !exhausted) {
                    unsigned long long claim = 0;
                    if (lane == 0) claim = atomicAdd(&kp.counters->queue_head,
                                                     static_cast<unsigned long long>(kp.grab));
                    claim = __shfl_sync(kFull, claim, 0);
                    if (claim >= kp.n) {
                        exhausted = true;
                    } else {
                        local_next = claim;
                        local_end = claim + kp.grab < kp.n ? claim + kp.grab : kp.n;
                        take_b = local_end - local_next;
                        const unsigned long long want = nidle - take_a;
                        if (take_b > want) take_b = want;
                        base_b = local_next;
                        local_next += take_b;
                    }
                }
                if (L.idx < 0) {
                    const unsigned long long rank = __popc(idle & lt_mask);
                    long long q = -1;
                    if (rank < take_a) q = static_cast<long long>(base_a + rank);
                    else if (rank - take_a < take_b) q = static_cast<long long>(base_b + (rank - take_a));
                    // the queue hands out pixels in tiles (KParams::order); a
                    // photon's calls do not depend on which lane takes it
                    if (kp.order && q >= 0) q = static_cast<long long>(kp.order[q]);
                    long long slot = q;
                    if (SHARE && q >= 0) {
                        int lo = 0, hi = kp.ngroups - 1;
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (kp.group_qstart[mid] <= static_cast<unsigned long long>(q)) lo = mid;
                            else hi = mid - 1;
                        }
                        L.grp = lo;
                        L.pix = q - static_cast<long long>(kp.group_qstart[lo]);
                        L.nchan = kp.group_chan[lo + 1] - kp.group_chan[lo];
                        // which channel leads and which finished on their own,
                        // as an earlier launch left them (zero after an init)
                        const unsigned long long ss = kp.share_state ? kp.share_state[q] : 0ull;
                        L.done = static_cast<unsigned>(ss & 0xFFFFFFFFull);
                        L.lead = static_cast<int>((ss >> 32) & 0xFFull);
                        L.zero_all = 0;
                        slot = chan_slot(kp, lo, L.lead, L.pix);
                    }
                    if (q >= 0 && !kp.ph.terminate[slot] &&
                        (LEG == 0 || LEG == 3 || ((kp.ph.phase[slot] == 1) == (LEG == 1)))) {
                        load_photon<LEG == 1>(kp.ph, slot, L);
                        L.idx = slot;
                        L.q = q;
                        if (LEG == 2) L.calls = kp.calls_carry[q];
                        L.img = SHARE ? chan_image(kp, L.grp, L.lead) : image_of_photon(kp, q);
                        have_disp = 0;
                    }
                }
            }
        }
        const unsigned active = __ballot_sync(kFull, L.idx >= 0);
        if (!active) {
            if (exhausted && local_next >= local_end) break;
            continue;
        }
        if (++iters > kp.max_iterations) {
            timed_out = true;
            break;
        }
        if (L.idx < 0) continue;

        // ---- one unit of work for this lane ----
        int finished = 0, terminated = 0;
        if (!L.mid_call) {
            if (L.calls >= kp.budget) {
                finished = 1;  // budget of this launch used; photon stays live
            } else {
                ++L.calls;
                ++cnt.calls;
                const double r = L.have_radius   ? L.radius
                                 : RHS::kLatency ? ks_radius_bf(L.s[1], L.s[2], L.s[3], kp.a)
                                                 : ks_radius(L.s[1], L.s[2], L.s[3], kp.a);
                if (r <= kp.r_min) {
                    L.I[0] = L.I[1] = L.I[2] = L.I[3] = 0.0;
                    L.zero_all = 1;
                    L.phase = 4;
                    finished = terminated = 1;
                } else if (r > kp.r_max) {
                    L.phase = 4;
                    finished = terminated = 1;
                } else if (INTEGRATOR == 0) {
                    const int phase0 = L.phase;
                    const double taken = L.dl;
                    rk4_step<RHS>(L.s, taken, kp, 1);
                    const double rn = RHS::after_accept(L.s, kp, 1);
                    ++cnt.accepted;
                    int ch_term = 0;
                    terminated = post_step<RAW, NoRecord, SHARE, LEG, RHS::kLatency>(
                        kp, ax, L, phase0, taken, kp.step0 + L.calls - 1, tdisp, pdisp, have_disp, NoRecord(), &ch_term,
                        rn);
                    if (SHARE && ch_term) {
                        cnt.terminated += ch_term;
                        const unsigned long long ts = static_cast<unsigned long long>(kp.step0 + L.calls);
                        if (ts > cnt.max_term_step) cnt.max_term_step = ts;
                    }
                    finished = terminated || (LEG == 1 && (L.phase != 1 || L.gen_pending));
                } else {
                    // Mixed form: an RK45 call may use the FP32 right-hand side only
                    // when its step sequence cannot change which fluid cell the ray
                    // samples next: after emission (not ImageBackward) and outside
                    // the fluid grid.  Fixed-step RK4 calls may use it everywhere.
                    L.fast = (LEG != 1 && L.phase != 1 && r * r > kp.fp32_min_radius_sq) ? 1 : 0;
                    L.need_k1 = 1;
                    L.dl_try = L.dl;
                    L.attempts = 0;
                    L.mid_call = 1;
                }
            }
        }
        if (INTEGRATOR == 1 && L.mid_call) {
            const double taken = L.dl_try;
            // the backward leg never uses the FP32 right-hand side (a literal
            // 0 lets the compiler drop it from the backward kernel)
            const int ok = rk45_attempt<RHS>(kp, L.s, &L.dl_try, L.need_k1, LEG == 1 ? 0 : L.fast, kk);
            L.need_k1 = 0;
            ++L.attempts;
            if (ok) {
                const double rn = RHS::after_accept(L.s, kp, L.fast);
                ++cnt.accepted;
                L.dl = L.dl_try;
                L.mid_call = 0;
                const int phase0 = L.phase;
                int ch_term = 0;
                terminated = post_step<RAW, NoRecord, SHARE, LEG, RHS::kLatency>(
                    kp, ax, L, phase0, taken, kp.step0 + L.calls - 1, tdisp, pdisp, have_disp, NoRecord(), &ch_term, rn);
                if (SHARE && ch_term) {
                    cnt.terminated += ch_term;
                    const unsigned long long ts = static_cast<unsigned long long>(kp.step0 + L.calls);
                    if (ts > cnt.max_term_step) cnt.max_term_step = ts;
                }
                finished = terminated || (LEG == 1 && (L.phase != 1 || L.gen_pending));
            } else {
                ++cnt.rejected;
                if (L.attempts >= 12) {
                    L.dl = L.dl_try;
                    L.mid_call = 0;
                    finished = terminated = 1;  // phase and state unchanged (:294-297)
                }
            }
        }
        if (finished) {
            const int stored = store_all<SHARE, LEG == 1>(kp, L, terminated, tdisp, pdisp, have_disp);
            if (terminated) {
                cnt.terminated += stored;
                const unsigned long long ts = static_cast<unsigned long long>(kp.step0 + L.calls);
                if (ts > cnt.max_term_step) cnt.max_term_step = ts;
            } else {
                store_carry<SHARE, LEG>(kp, L);
            }
            L.idx = -1;
        }
    }
    if (timed_out) {
        // Leave every photon consistent: write back what this lane holds.
        if (L.idx >= 0) {
            store_all<SHARE, LEG == 1>(kp, L, 0, tdisp, pdisp, have_disp);
            store_carry<SHARE, LEG>(kp, L);
        }
        if (lane == 0) atomicAdd(&kp.counters->timed_out, 1ull);
    }
    // ---- flush counters: warp reduce, one atomic per counter per warp ----
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        cnt.terminated += __shfl_down_sync(kFull, cnt.terminated, off);
        cnt.accepted += __shfl_down_sync(kFull, cnt.accepted, off);
        cnt.rejected += __shfl_down_sync(kFull, cnt.rejected, off);
        cnt.calls += __shfl_down_sync(kFull, cnt.calls, off);
        const unsigned long long m = __shfl_down_sync(kFull, cnt.max_term_step, off);
        if (m > cnt.max_term_step) cnt.max_term_step = m;
    }
    if (lane == 0) {
        if (cnt.terminated) atomicAdd(&kp.counters->terminated, cnt.terminated);
        if (cnt.accepted) atomicAdd(&kp.counters->accepted, cnt.accepted);
        if (cnt.rejected) atomicAdd(&kp.counters->rejected, cnt.rejected);
        if (cnt.calls) atomicAdd(&kp.counters->calls, cnt.calls);
        if (cnt.max_term_step) atomicMax(&kp.counters->max_term_step, cnt.max_term_step);
    }
}

// Between the backward-leg and forward-leg launches: the packet generation
// of the rays the backward leg stopped at their first fluid contact
// (calls_carry[q] < 0), one thread per queue index.  It finishes that call
// (integrate_cart_ks.hpp:351-363): the same position samples the same cell,
// the packet is generated, and the photon goes on to the forward-leg launch
// in ImageForward with its calls in calls_carry[q] -- or terminates Rejected.
// Kept out of the forward-leg loop, whose lanes would otherwise sit in this
// once-per-ray code while their warp-mates step.
template <bool SHARE>
GRT_DEV void generate_body(const KParams& kp, const Axes& ax) {
    unsigned long long terminated = 0, max_ts = 0;
    const unsigned long long stride = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
    for (unsigned long long q = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; q < kp.n;
         q += stride) {
        const long long carry = kp.calls_carry[q];
        if (carry >= 0) continue;
        Lane L;
        long long slot = static_cast<long long>(q);
        if (SHARE) {
            int lo = 0, hi = kp.ngroups - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (kp.group_qstart[mid] <= q) lo = mid;
                else hi = mid - 1;
            }
            L.grp = lo;
            L.pix = static_cast<long long>(q - kp.group_qstart[lo]);
            L.nchan = kp.group_chan[lo + 1] - kp.group_chan[lo];
            const unsigned long long ss = kp.share_state ? kp.share_state[q] : 0ull;
            L.done = static_cast<unsigned>(ss & 0xFFFFFFFFull);
            L.lead = static_cast<int>((ss >> 32) & 0xFFull);
            slot = chan_slot(kp, lo, L.lead, L.pix);
        }
        load_photon<false>(kp.ph, slot, L);
        L.idx = slot;
        L.q = static_cast<long long>(q);
        L.calls = -carry - 1;
        L.img = SHARE ? chan_image(kp, L.grp, L.lead) : image_of_photon(kp, static_cast<long long>(q));
        L.radius = ks_radius(L.s[1], L.s[2], L.s[3], kp.a);
        L.have_radius = 1;
        FluidSample fs;
        int ch_term = 0, term = 0;
        if (sample_fluid<false>(kp, ax, L.s, L.radius, fs))
            term = generate_at_contact<SHARE>(kp, L, fs, kp.step0 + L.calls - 1, &ch_term);
        if (term || ch_term) {
            const unsigned long long ts = static_cast<unsigned long long>(kp.step0 + L.calls);
            if (ts > max_ts) max_ts = ts;
        }
        terminated += static_cast<unsigned long long>(ch_term);
        if (term) {
            terminated += store_all<SHARE>(kp, L, 1, 0.0, 0.0, 0);
        } else {
            // the lead only: the followers' geodesic state is stored by the
            // forward-leg launch when the ray finishes
            store_photon(kp.ph, L, 0, 0.0, 0.0, 0);
            kp.calls_carry[q] = L.calls;
            if (SHARE && kp.share_state)
                kp.share_state[q] = (static_cast<unsigned long long>(L.lead) << 32) | L.done;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        terminated += __shfl_down_sync(kFull, terminated, off);
        const unsigned long long m = __shfl_down_sync(kFull, max_ts, off);
        if (m > max_ts) max_ts = m;
    }
    if ((threadIdx.x & 31) == 0) {
        if (terminated) atomicAdd(&kp.counters->terminated, terminated);
        if (max_ts) atomicMax(&kp.counters->max_term_step, max_ts);
    }
}

// Shared-memory layout of a trace block: [stage slots (RK45)] [axes and
// half-spans of a separable grid].  Returns the staged pointers.
GRT_DEV void stage_grid(const KParams& kp, double* smem, int integrator, Axes& ax, KStore& kk) {
    const KGrid& G = kp.grid;
    double* p = smem;
    kk.base = p + threadIdx.x;
    if (integrator == 1) p += kStageSlots * 7 * kTraceThreads;
    if (G.available && G.separable) {
        double* r = p;
        double* th = r + G.nr;
        double* ph = th + G.nth;
        double* rh = ph + G.nph;
        double* thh = rh + G.nr;
        double* phh = thh + G.nth;
        for (int q = threadIdx.x; q < G.nr; q += blockDim.x) { r[q] = G.r_axis[q]; rh[q] = G.r_half[q]; }
        for (int q = threadIdx.x; q < G.nth; q += blockDim.x) { th[q] = G.th_axis[q]; thh[q] = G.th_half[q]; }
        for (int q = threadIdx.x; q < G.nph; q += blockDim.x) { ph[q] = G.ph_axis[q]; phh[q] = G.ph_half[q]; }
        ax = Axes{r, th, ph, rh, thh, phh};
    } else {
        ax = Axes{nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    }
    __syncthreads();
}


}  // namespace dev
}  // namespace grt
