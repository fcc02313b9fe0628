// FP64 parity-form kernels.  Built with -fmad=false so that every product and
// sum rounds separately, as in the reference's host build.
//
//   trace_fp64<RK4|RK45>  -- persistent per-photon step loop (integrate_cart_ks.hpp:230-419)
//   init_image_pixels     -- pixel-grid camera rays (initialize_photons.hpp:82-170)
//   image_products        -- build_observation_products (observation.hpp:31-84)
//   count_terminated      -- "Count Terminated Photons" (integrate_cart_ks.hpp:496-503)
#include "grt_launch.h"
#include "grt_trace.cuh"

namespace grt {

// 128-thread blocks; MINB resident blocks per SM caps the registers per
// thread at 65536 / (128 * MINB): 255, 170 and 128 for MINB = 2, 3, 4.
template <int INTEGRATOR, int MINB>
__global__ void __launch_bounds__(128, MINB) trace_fp64(const __grid_constant__ KParams kp) {
    extern __shared__ double smem[];
    dev::Axes ax;
    dev::KStore kk;
    dev::stage_grid(kp, smem, INTEGRATOR, ax, kk);
    dev::trace_body<INTEGRATOR, dev::Fp64Rhs>(kp, ax, kk);
}

// initialize_photons.hpp:116-169 with screen (u, v) at pixel centres; the
// camera centre and basis come from the host (glibc sin/cos, like the reference).
// With args.forward, line-of-sight forward rays instead (see InitImageArgs).
__global__ void init_image_pixels(const __grid_constant__ InitImageArgs args) {
    const unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x;
    if (i >= args.nx * args.ny) return;
    const unsigned long long iy = i / args.nx, ix = i % args.nx;
    const double u = -0.5 * args.W + (static_cast<double>(ix) + 0.5) * args.W / static_cast<double>(args.nx);
    const double v = -0.5 * args.H + (static_cast<double>(iy) + 0.5) * args.H / static_cast<double>(args.ny);
    const bool fwd = args.forward != 0;
    const double x = (fwd ? args.bx : args.cx) + u * args.th_hat[0] + v * args.ph_hat[0];
    const double y = (fwd ? args.by : args.cy) + u * args.th_hat[1] + v * args.ph_hat[1];
    const double z = (fwd ? args.bz : args.cz) + u * args.th_hat[2] + v * args.ph_hat[2];
    double kx = fwd ? args.cx : -args.cx, ky = fwd ? args.cy : -args.cy, kz = fwd ? args.cz : -args.cz;
    const double kn = sqrt(kx * kx + ky * ky + kz * kz);
    kx /= kn;
    ky /= kn;
    kz /= kn;
    const double X[4] = {0.0, x, y, z};
    const double K[3] = {kx, ky, kz};
    double p[4] = {0.0, 0.0, 0.0, 0.0};
    dev::ks_null_momentum(X, K, args.a, args.M, p);
    const KPhotons& P = args.ph;
    const unsigned long long o = args.offset + i;
    P.id[o] = args.id_offset + i;
    P.frequency[o] = fwd ? args.nu0 : 0.0;
    P.emission_frame_energy[o] = fwd ? -p[0] : 1.0;
    P.x0[o] = 0.0; P.x1[o] = x; P.x2[o] = y; P.x3[o] = z;
    P.k0[o] = p[0]; P.k1[o] = p[1]; P.k2[o] = p[2]; P.k3[o] = p[3];
    P.I[o] = 0.0; P.Q[o] = 0.0; P.U[o] = 0.0; P.V[o] = 0.0;
    P.dlambda[o] = args.dlambda0;
    P.terminate[o] = 0;
    P.phase[o] = fwd ? 2 : 1;  // ImageForward / ImageBackward
    P.theta_disp[o] = u;
    P.phi_disp[o] = v;
}


// observation.hpp:61-82: ImageArrived photons binned by arrival (u, v) and log10(nu).
__global__ void image_products(const __grid_constant__ ProductsArgs args) {
    const unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x;
    bool arrived = false;
    if (i < args.n) {
        const unsigned long long o = args.offset + i;
        if (args.ph.phase[o] == 3) {
            arrived = true;
            const unsigned long long px = dev::observation_bin(args.ph.theta_disp[o], -0.5 * args.W, 0.5 * args.W, args.nx);
            const unsigned long long py = dev::observation_bin(args.ph.phi_disp[o], -0.5 * args.H, 0.5 * args.H, args.ny);
            const unsigned long long pix = py * args.nx + px;
            const double I = args.ph.I[o];
            atomicAdd(&args.image[pix], I);
            atomicAdd(&args.image[args.nx * args.ny + pix], args.ph.Q[o]);
            atomicAdd(&args.image[2 * args.nx * args.ny + pix], args.ph.U[o]);
            atomicAdd(&args.image[3 * args.nx * args.ny + pix], args.ph.V[o]);
            const double f = args.ph.frequency[o];
            if (f >= args.spec_min && f <= args.spec_max) {
                const unsigned long long b = dev::observation_bin(log10(f), args.log_min, args.log_max, args.bins);
                atomicAdd(&args.spectrum[b], I);
            }
        }
    }
    const unsigned mask = __ballot_sync(0xFFFFFFFFu, arrived);
    if ((threadIdx.x & 31) == 0 && mask) atomicAdd(args.arrived, static_cast<unsigned long long>(__popc(mask)));
}

__global__ void count_terminated(const uint8_t* __restrict__ term, unsigned long long n,
                                 unsigned long long* out) {
    unsigned long long c = 0;
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x)
        c += term[i] ? 1 : 0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, off);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// ---- host-side launchers ----
template <int I, int B>
static cudaError_t launch_trace_fp64_v(const KParams& kp, int blocks, size_t smem, cudaStream_t stream) {
    cudaFuncSetAttribute(trace_fp64<I, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    trace_fp64<I, B><<<blocks, 128, smem, stream>>>(kp);
    return cudaGetLastError();
}

// 128-thread blocks, sm_count * blocks_per_sm of them; blocks_per_sm (2, 3
// or 4) selects the register-capped instantiation.
cudaError_t launch_trace_fp64(const KParams& kp, int integrator, int sm_count, int blocks_per_sm, size_t smem,
                           cudaStream_t stream) {
    const int blocks = sm_count * blocks_per_sm;
    if (integrator == 0) {
        switch (blocks_per_sm) {
            case 2: return launch_trace_fp64_v<0, 2>(kp, blocks, smem, stream);
            case 3: return launch_trace_fp64_v<0, 3>(kp, blocks, smem, stream);
            case 4: return launch_trace_fp64_v<0, 4>(kp, blocks, smem, stream);
            default: return cudaErrorInvalidConfiguration;
        }
    }
    switch (blocks_per_sm) {
        case 2: return launch_trace_fp64_v<1, 2>(kp, blocks, smem, stream);
        case 3: return launch_trace_fp64_v<1, 3>(kp, blocks, smem, stream);
        case 4: return launch_trace_fp64_v<1, 4>(kp, blocks, smem, stream);
        default: return cudaErrorInvalidConfiguration;
    }
}

cudaError_t launch_init_image(const InitImageArgs& args, cudaStream_t stream) {
    const unsigned long long n = args.nx * args.ny;
    if (n == 0) return cudaSuccess;
    const unsigned threads = 256;
    const unsigned blocks = static_cast<unsigned>((n + threads - 1) / threads);
    init_image_pixels<<<blocks, threads, 0, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_image_products(const ProductsArgs& args, cudaStream_t stream) {
    if (args.n == 0) return cudaSuccess;
    const unsigned threads = 256;
    const unsigned blocks = static_cast<unsigned>((args.n + threads - 1) / threads);
    image_products<<<blocks, threads, 0, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_count_terminated(const uint8_t* term, unsigned long long n, unsigned long long* out,
                                    int sm_count, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    unsigned long long want = (n + 255) / 256;
    const unsigned long long cap = static_cast<unsigned long long>(sm_count) * 8;
    const unsigned blocks = static_cast<unsigned>(want < cap ? want : cap);
    count_terminated<<<blocks, 256, 0, stream>>>(term, n, out);
    return cudaGetLastError();
}

}  // namespace grt
