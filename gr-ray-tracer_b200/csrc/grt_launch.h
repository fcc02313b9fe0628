// Host-side launch interface between the C ABI (grt_api.cu) and the kernel
// translation units.  Internal to the library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#include "grt_kparams.h"

namespace grt {

struct InitImageArgs {
    KPhotons ph;
    unsigned long long offset;     // first photon slot written
    unsigned long long nx, ny;
    unsigned long long row0, nrows;  // pixel rows [row0, row0 + nrows) of the ny-row screen
    unsigned long long id_offset;
    double W, H;
    double cx, cy, cz;
    double th_hat[3], ph_hat[3];
    double a, M;
    double dlambda0;               // initial_step * camera_distance (forward: * back distance)
    // line-of-sight forward rays: start on the plane -back * n, aimed along +n,
    // ImageForward, I = 0, frequency nu0, emission_frame_energy = -p_t
    int forward;
    double bx, by, bz;             // -back * n
    double nu0;
    // the reference's random screen instead of pixel centres: (u, v) from
    // Philox keyed by (seed, photon id), see kScreenDomain
    int random_screen;
    unsigned long long seed;
};

// initialize_photons_disk (initialize_photons.hpp:173-327): one photon per
// packet; the packet's cell comes from the prefix sum of per-cell counts.
struct DiskInitArgs {
    KPhotons ph;
    unsigned long long n;                // packets = offsets[ncell]
    const unsigned long long* offsets;   // [ncell + 1]
    unsigned long long ncell;
    const double* pos;                   // [ncell][3] Cartesian KS cell positions (host libm)
    const double2* rho_t;                // [ncell] (rho, T) code units
    const double2* vel;                  // [2 * ncell] Cartesian u^mu * velocity scale
    const double2* mag;                  // [2 * ncell] Cartesian b^mu * magnetic scale
    double density_scale, temperature_scale, length_scale, time_scale;
    double a, M;
    int generator;
    int pad;
    double energy, pl_slope, nu_min, nu_max, nu_custom;
    uint64_t seed;                       // scattering seed + rank (Philox key)
    unsigned long long id_offset;
    double dlambda0;                     // initial_step (disk mode: unscaled)
};

// One image of a products launch: its photon slots, screen and output buffers.
struct ProductsImage {
    unsigned long long offset, n;  // photon slots [offset, offset + n)
    unsigned long long nx, ny;
    double W, H;
    double* image;                 // [4][ny][nx] (I, Q, U, V), zeroed before the launch
    double* spectrum;              // [bins], zeroed
    unsigned long long* arrived;   // [1], zeroed
    unsigned block0;               // first block of this image in the launch
    unsigned pad;
};

// build_observation_products over up to kProductsMaxImages images in one
// launch; each block belongs to one image.
constexpr int kProductsMaxImages = 32;
constexpr unsigned long long kProductsSharedBins = 4096;  // spectrum privatised in shared memory up to this
struct ProductsSet {
    KPhotons ph;
    unsigned long long bins;
    double spec_min, spec_max, log_min, log_max;
    int nimages;
    unsigned blocks;
    ProductsImage img[kProductsMaxImages];
};

// Strided gather of an output step's photon fields (write_output_step):
// elements src[k][j * stride], j < count, of field k packed at dst + dst_off[k].
constexpr int kGatherMaxFields = 40;  // a selection's fields, "all" after 20 names included
struct GatherArgs {
    const void* src[kGatherMaxFields];
    unsigned long long dst_off[kGatherMaxFields];
    int item[kGatherMaxFields];  // element bytes: 8 or 1
    int nfields;
    int pad;
    unsigned long long count, stride;
    unsigned char* dst;
};

// Buffers of the adjoint pass (grt_adjoint.cu).
struct AdjointArgs {
    double* ckpt;              // [n][cap][16] ray state after emission and every K calls
    int cap;                   // checkpoints per ray
    int K;                     // calls between checkpoints
    int* nckpt;                // [n] checkpoints written
    long long* call0;          // [n] calls taken when checkpoint 0 was written (-1: never emitted)
    int* overflow;             // checkpoint/tape capacity errors
    const double* dL_dI;       // [ny][nx] dL/d(image_I)
    unsigned long long nx, ny;
    double W, H;
    double* g_abs;             // [ncell] dL/dm_abs (accumulated)
    double* g_emis;            // [ncell] dL/dm_emis
    double* tape;              // [threads][K][6]
};

// Camera plane basis of integrate_cart_ks.hpp:97-107 with host libm, plus the
// image's coefficients.
inline KImage make_kimage(double theta, double phi, double distance, double width, double height, double nu_custom,
                          double kappa, double jcoef) {
    KImage im{};
    im.cam_D = distance;
    im.cam_W = width;
    im.cam_H = height;
    im.cam_n[0] = std::sin(theta) * std::cos(phi);
    im.cam_n[1] = std::sin(theta) * std::sin(phi);
    im.cam_n[2] = std::cos(theta);
    im.cam_th[0] = std::cos(theta) * std::cos(phi);
    im.cam_th[1] = std::cos(theta) * std::sin(phi);
    im.cam_th[2] = -std::sin(theta);
    im.cam_ph[0] = -std::sin(phi);
    im.cam_ph[1] = std::cos(phi);
    im.cam_ph[2] = 0.0;
    im.nu_custom = nu_custom;
    im.kappa = kappa;
    im.jcoef = jcoef;
    return im;
}

// Whether the spin a and mass M admit the reciprocal-quotient right-hand side
// (KParams::rcp_ok): |a| = 0 or in [2^-20, 2], M in [2^-20, 2^20].
inline int rcp_params_ok(double a, double M) {
    const double fa = std::fabs(a);
    const bool a_ok = fa == 0.0 || (fa >= std::ldexp(1.0, -20) && fa <= 2.0);
    const bool m_ok = M >= std::ldexp(1.0, -20) && M <= std::ldexp(1.0, 20);
    return a_ok && m_ok ? 1 : 0;
}

// Dynamic shared memory of a trace launch: the stage slots for RK45 (6*7
// doubles per thread: k1..k5, then the state) plus the separable axes and
// their half-spans (2*(nr+nth+nph)).
inline size_t dev_trace_smem_bytes(int integrator, int threads, bool separable, int nr, int nth, int nph) {
    size_t n = integrator == 1 ? static_cast<size_t>(6 * 7) * threads : 0;
    if (separable) n += 2 * static_cast<size_t>(nr + nth + nph);
    return n * sizeof(double);
}

// Adjoint pass: checkpointed forward trace and reverse sweep, 128-thread blocks.
cudaError_t launch_adjoint_forward(const KParams& kp, const AdjointArgs& aa, int blocks, size_t smem,
                                   cudaStream_t stream);
cudaError_t launch_adjoint_reverse(const KParams& kp, const AdjointArgs& aa, int blocks, size_t smem,
                                   cudaStream_t stream);

// Persistent trace launches (grt_trace_inst.cu): `blocks` blocks of 128
// threads; blocks_per_sm in {2, 3, 4} picks the register cap (255 / 170 /
// 128); leg 0 traces whole rays, legs 1 and 2 the backward leg and the rest
// of image-mode rays, leg 3 whole disk-mode rays (trace_body).
cudaError_t launch_trace_fp64_leg0(const KParams& kp, int integrator, int blocks_per_sm, int blocks, size_t smem,
                                   cudaStream_t stream);
cudaError_t launch_trace_fp64_leg1(const KParams& kp, int integrator, int blocks_per_sm, int blocks, size_t smem,
                                   cudaStream_t stream);
cudaError_t launch_trace_fp64_leg2(const KParams& kp, int integrator, int blocks_per_sm, int blocks, size_t smem,
                                   cudaStream_t stream);
cudaError_t launch_trace_mixed_leg0(const KParams& kp, int integrator, int blocks_per_sm, int blocks, size_t smem,
                                    cudaStream_t stream);
cudaError_t launch_trace_mixed_leg1(const KParams& kp, int integrator, int blocks_per_sm, int blocks, size_t smem,
                                    cudaStream_t stream);
cudaError_t launch_trace_mixed_leg2(const KParams& kp, int integrator, int blocks_per_sm, int blocks, size_t smem,
                                    cudaStream_t stream);
cudaError_t launch_trace_fp64_leg3(const KParams& kp, int integrator, int blocks_per_sm, int blocks, size_t smem,
                                   cudaStream_t stream);
cudaError_t launch_trace_mixed_leg3(const KParams& kp, int integrator, int blocks_per_sm, int blocks, size_t smem,
                                    cudaStream_t stream);
// Packet generation between the backward-leg and forward-leg launches
// (photons with calls_carry < 0), one thread per queue index; smem holds the
// staged axes (dev_trace_smem_bytes with integrator 0).
cudaError_t launch_generate_pending(const KParams& kp, int sm_count, size_t smem, cudaStream_t stream);
// sm_count * blocks_per_sm blocks of the form's (FP64 or mixed) kernel for `leg`.
cudaError_t launch_trace(const KParams& kp, bool mixed, int leg, int integrator, int sm_count, int blocks_per_sm,
                         size_t smem, cudaStream_t stream);
cudaError_t launch_init_image(const InitImageArgs& args, cudaStream_t stream);
cudaError_t launch_init_disk(const DiskInitArgs& a, cudaStream_t stream);
// Fills block0 / blocks of `set` and launches it.
cudaError_t launch_image_products(ProductsSet& set, cudaStream_t stream);
cudaError_t launch_gather_fields(const GatherArgs& a, int sm_count, cudaStream_t stream);
cudaError_t launch_count_terminated(const uint8_t* term, unsigned long long n, unsigned long long* out,
                                    int sm_count, cudaStream_t stream);

}  // namespace grt
