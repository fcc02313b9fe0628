// Adjoint of the radiative-transfer sweep (no counterpart in the reference).
//
// The image-mode Stokes-I of a ray is a function of the per-cell multipliers
// on the optical-depth and emissivity increments (KParams::m_abs, m_emis):
// along its forward leg every sampled step does
//   I <- (I * exp(-m_abs[c] * tau0) + m_emis[c] * j0) * scale
// (radiative_transfer.hpp:80-96 with the multipliers applied to the values the
// user extension points return; scale = albedo on a scattering event,
// scattering.hpp:305-309).  The geodesic does not depend on the multipliers,
// so for a loss L over the Stokes-I image, with lambda = dL/dI after a step:
//   dL/dm_emis[c] += lambda_pre * j0,
//   dL/dm_abs[c]  += lambda_pre * I_before * att * (-tau0),
//   lambda_before  = lambda_pre * att,      lambda_pre = lambda * scale.
//
// adj_forward traces every ray (one thread per ray, the same per-call code as
// the trace kernels, so the trajectory is bit-identical) and stores the ray
// state where its radiative transfer starts -- right after the emission call
// of an image-backward ray, at the start for forward and disk photons -- and
// every K calls after that.
// adj_reverse walks each arrived ray's checkpoints from the last to the first:
// it recomputes the K calls of a segment from its checkpoint, recording the
// RT updates on a per-ray tape, then sweeps the tape backwards.
#include "grt_launch.h"
#include "grt_trace.cuh"

namespace grt {
namespace dev {

constexpr int kCkptDoubles = 16;  // s[8], I[4], freq, emit, dl, phase
constexpr int kTapeDoubles = 6;   // cell, tau0, j0, I_before, att, scale

GRT_DEV void save_checkpoint(double* c, const Lane& L) {
#pragma unroll
    for (int q = 0; q < 8; ++q) c[q] = L.s[q];
#pragma unroll
    for (int q = 0; q < 4; ++q) c[8 + q] = L.I[q];
    c[12] = L.freq;
    c[13] = L.emit;
    c[14] = L.dl;
    c[15] = static_cast<double>(L.phase);
}

GRT_DEV void load_checkpoint(const double* c, Lane& L) {
#pragma unroll
    for (int q = 0; q < 8; ++q) L.s[q] = c[q];
#pragma unroll
    for (int q = 0; q < 4; ++q) L.I[q] = c[8 + q];
    L.freq = c[12];
    L.emit = c[13];
    L.dl = c[14];
    L.phase = static_cast<int>(c[15]);
    L.have_radius = 0;
    L.mid_call = 0;
}

// One call of the reference functor on this ray (the trace kernels' per-call
// sequence: termination radii, RK4 step or up to 12 RKF45 attempts, post_step).
// Returns 1 if the photon terminated.  The right-hand side takes the
// branch-free reciprocal and square root (Fp64RhsT<true>): with one ray per
// thread and about one warp per scheduler, both passes measured 5% faster.
template <int INTEGRATOR, class Rec>
GRT_DEV int run_call(const KParams& kp, const Axes& ax, const KStore& kk, Lane& L, double& tdisp, double& pdisp,
                     int& have_disp, Rec rec) {
    ++L.calls;
    const double r = L.have_radius ? L.radius : ks_radius(L.s[1], L.s[2], L.s[3], kp.a);
    if (r <= kp.r_min) {
        L.I[0] = L.I[1] = L.I[2] = L.I[3] = 0.0;
        L.phase = 4;
        return 1;
    }
    if (r > kp.r_max) {
        L.phase = 4;
        return 1;
    }
    const int64_t step = kp.step0 + L.calls - 1;
    if (INTEGRATOR == 0) {
        const int phase0 = L.phase;
        const double taken = L.dl;
        rk4_step<Fp64RhsT<true>>(L.s, taken, kp, 1);
        return post_step<false, Rec>(kp, ax, L, phase0, taken, step, tdisp, pdisp, have_disp, rec);
    }
    L.dl_try = L.dl;
    for (int attempt = 0; attempt < 12; ++attempt) {
        const double taken = L.dl_try;
        if (rk45_attempt<Fp64RhsT<true>>(kp, L.s, &L.dl_try, attempt == 0, 0, kk)) {
            L.dl = L.dl_try;
            const int phase0 = L.phase;
            return post_step<false, Rec>(kp, ax, L, phase0, taken, step, tdisp, pdisp, have_disp, rec);
        }
    }
    L.dl = L.dl_try;
    return 1;  // integrate_cart_ks.hpp:294-297: give up, phase and state unchanged
}

struct TapeRecord {
    double* tape;  // this thread's K entries
    int* count;
    int* zero_flag;
    int cap;
    GRT_DEV void rt_step(int cell, double tau0, double j0, double I_before, double att, double scale) const {
        const int t = *count;
        if (t < cap) {
            double* e = tape + static_cast<long long>(t) * kTapeDoubles;
            e[0] = static_cast<double>(cell);
            e[1] = tau0;
            e[2] = j0;
            e[3] = I_before;
            e[4] = att;
            e[5] = scale;
        }
        *count = t + 1;
    }
    GRT_DEV void zeroed() const { *zero_flag = 1; }
};

}  // namespace dev

template <int INTEGRATOR>
__global__ void __launch_bounds__(128, 2) adj_forward(const __grid_constant__ KParams kp,
                                                      const __grid_constant__ AdjointArgs aa) {
    extern __shared__ double smem[];
    dev::Axes ax;
    dev::KStore kk;
    dev::stage_grid(kp, smem, INTEGRATOR, ax, kk);
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
         i < static_cast<long long>(kp.n); i += stride) {
        aa.nckpt[i] = 0;
        aa.call0[i] = -1;
        if (kp.ph.terminate[i]) continue;
        dev::Lane L;
        dev::load_photon(kp.ph, i, L);
        L.idx = i;
        L.img = dev::image_of_photon(kp, i);
        double tdisp = 0.0, pdisp = 0.0;
        int have_disp = 0, terminated = 0, nck = 0;
        // radiative transfer starts after the emission call (image backward
        // rays) or at once (forward and disk photons)
        long long c0 = L.phase == 1 ? -1 : 0;
        while (L.calls < kp.budget) {
            if (c0 >= 0 && (L.calls - c0) % aa.K == 0) {
                if (nck < aa.cap) {
                    dev::save_checkpoint(aa.ckpt + (i * aa.cap + nck) * dev::kCkptDoubles, L);
                    ++nck;
                } else {
                    atomicAdd(aa.overflow, 1);
                }
            }
            const int phase_before = L.phase;
            terminated = dev::run_call<INTEGRATOR>(kp, ax, kk, L, tdisp, pdisp, have_disp, dev::NoRecord());
            if (terminated) break;
            if (c0 < 0 && phase_before == 1 && L.phase == 2) c0 = L.calls;  // emitted in this call
        }
        dev::store_photon(kp.ph, L, terminated, tdisp, pdisp, have_disp);
        aa.nckpt[i] = nck;
        aa.call0[i] = c0;
        atomicAdd(&kp.counters->calls, static_cast<unsigned long long>(L.calls));
        if (terminated) atomicAdd(&kp.counters->terminated, 1ull);
    }
}

template <int INTEGRATOR>
__global__ void __launch_bounds__(128, 2) adj_reverse(const __grid_constant__ KParams kp,
                                                      const __grid_constant__ AdjointArgs aa) {
    extern __shared__ double smem[];
    dev::Axes ax;
    dev::KStore kk;
    dev::stage_grid(kp, smem, INTEGRATOR, ax, kk);
    const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
         i < static_cast<long long>(kp.n); i += stride) {
        if (kp.ph.phase[i] != 3) continue;  // only ImageArrived rays enter the image
        const int nck = aa.nckpt[i];
        if (nck <= 0) continue;
        const unsigned long long px = dev::observation_bin(kp.ph.theta_disp[i], -0.5 * aa.W, 0.5 * aa.W, aa.nx);
        const unsigned long long py = dev::observation_bin(kp.ph.phi_disp[i], -0.5 * aa.H, 0.5 * aa.H, aa.ny);
        double lam = aa.dL_dI[py * aa.nx + px];
        if (lam == 0.0) continue;
        double* tape = aa.tape + static_cast<long long>(blockIdx.x * blockDim.x + threadIdx.x) * aa.K *
                                     dev::kTapeDoubles;
        const long long c0 = aa.call0[i];
        dev::Lane L;
        L.id = kp.ph.id[i];
        L.idx = i;
        L.img = dev::image_of_photon(kp, i);
        for (int m = nck - 1; m >= 0 && lam != 0.0; --m) {
            dev::load_checkpoint(aa.ckpt + (i * aa.cap + m) * dev::kCkptDoubles, L);
            L.calls = c0 + static_cast<long long>(m) * aa.K;
            const long long end = (m == nck - 1) ? kp.budget : L.calls + aa.K;
            int count = 0, zeroed = 0;
            dev::TapeRecord rec{tape, &count, &zeroed, aa.K};
            double tdisp = 0.0, pdisp = 0.0;
            int have_disp = 0;
            while (L.calls < end && L.calls < kp.budget) {
                if (dev::run_call<INTEGRATOR>(kp, ax, kk, L, tdisp, pdisp, have_disp, rec)) break;
            }
            if (count > aa.K) {
                atomicAdd(aa.overflow, 1);
                count = aa.K;
            }
            if (m == nck - 1 && zeroed) break;  // Stokes zeroed at arrival: no dependence
            for (int t = count - 1; t >= 0; --t) {
                const double* e = tape + static_cast<long long>(t) * dev::kTapeDoubles;
                const int cell = static_cast<int>(e[0]);
                const double lp = lam * e[5];
                if (kp.emis_on) atomicAdd(aa.g_emis + cell, lp * e[2]);
                if (kp.abs_on) atomicAdd(aa.g_abs + cell, lp * e[3] * e[4] * (-e[1]));
                lam = lp * e[4];
            }
        }
    }
}

cudaError_t launch_adjoint_forward(const KParams& kp, const AdjointArgs& aa, int blocks, size_t smem,
                                   cudaStream_t stream) {
    if (kp.integrator == 0) {
        cudaFuncSetAttribute(adj_forward<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        adj_forward<0><<<blocks, 128, smem, stream>>>(kp, aa);
    } else {
        cudaFuncSetAttribute(adj_forward<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        adj_forward<1><<<blocks, 128, smem, stream>>>(kp, aa);
    }
    return cudaGetLastError();
}

cudaError_t launch_adjoint_reverse(const KParams& kp, const AdjointArgs& aa, int blocks, size_t smem,
                                   cudaStream_t stream) {
    if (kp.integrator == 0) {
        cudaFuncSetAttribute(adj_reverse<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        adj_reverse<0><<<blocks, 128, smem, stream>>>(kp, aa);
    } else {
        cudaFuncSetAttribute(adj_reverse<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        adj_reverse<1><<<blocks, 128, smem, stream>>>(kp, aa);
    }
    return cudaGetLastError();
}

}  // namespace grt
