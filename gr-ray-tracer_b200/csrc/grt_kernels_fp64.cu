// FP64 kernels around the trace, built with -fmad=false so that every product
// and sum rounds separately, as in the reference's host build:
//
//   init_image_pixels     -- pixel-grid camera rays (initialize_photons.hpp:82-170)
//   image_products        -- build_observation_products (observation.hpp:31-84)
//   init_disk_photons     -- initialize_photons_disk (initialize_photons.hpp:173-327)
//   count_terminated      -- "Count Terminated Photons" (integrate_cart_ks.hpp:496-503)
//   gather_fields         -- strided field gather of write_output_step (write_output.hpp:13-59)
//
// and the dispatcher over the trace kernels of grt_trace_inst.cu.
#include "grt_launch.h"
#include "grt_trace.cuh"

namespace grt {

// initialize_photons.hpp:116-169 with screen (u, v) at pixel centres, or
// with args.random_screen at the reference's uniform random screen position
// (:123-125, drand(lo, hi) = lo + (hi - lo) d) from Philox keyed by (seed,
// photon id); the camera centre and basis come from the host (glibc sin/cos,
// like the reference).  With args.forward, line-of-sight forward rays instead
// (see InitImageArgs).
__global__ void init_image_pixels(const __grid_constant__ InitImageArgs args) {
    const unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x;
    if (i >= args.nx * args.nrows) return;
    const unsigned long long iy = args.row0 + i / args.nx, ix = i % args.nx;
    const unsigned long long id = args.id_offset + args.row0 * args.nx + i;
    double u, v;
    if (args.random_screen) {
        dev::Philox rng(args.seed, id, dev::kScreenDomain);
        u = -0.5 * args.W + args.W * rng.drand();
        v = -0.5 * args.H + args.H * rng.drand();
    } else {
        u = -0.5 * args.W + (static_cast<double>(ix) + 0.5) * args.W / static_cast<double>(args.nx);
        v = -0.5 * args.H + (static_cast<double>(iy) + 0.5) * args.H / static_cast<double>(args.ny);
    }
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
    P.id[o] = id;
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


// observation.hpp:61-82: ImageArrived photons binned by arrival (u, v) and
// log10(nu).  Each block serves one image of the set.  The arrival
// frequencies of an image crowd into a few spectrum bins, so per-photon
// atomics would serialise on them: the spectrum is summed per warp (one
// shuffle reduction per distinct bin), then per block in shared memory, and
// flushed with one global atomic per non-empty bin.
__global__ void __launch_bounds__(256) image_products(const __grid_constant__ ProductsSet set) {
    extern __shared__ double hist[];
    __shared__ unsigned long long s_arrived;
    int k = 0;
    while (k + 1 < set.nimages && set.img[k + 1].block0 <= blockIdx.x) ++k;
    const ProductsImage& im = set.img[k];
    const unsigned end = k + 1 < set.nimages ? set.img[k + 1].block0 : set.blocks;
    const unsigned long long stride = static_cast<unsigned long long>(end - im.block0) * blockDim.x;
    const bool shared_spec = set.bins <= kProductsSharedBins;
    if (shared_spec)
        for (unsigned long long q = threadIdx.x; q < set.bins; q += blockDim.x) hist[q] = 0.0;
    if (threadIdx.x == 0) s_arrived = 0;
    __syncthreads();
    const unsigned long long npix = im.nx * im.ny;
    const unsigned lane = threadIdx.x & 31u;
    unsigned long long count = 0;
    // warp-uniform trip count: every lane of a warp runs each iteration, so
    // the spectrum can be summed per warp before the shared-memory atomics
    for (unsigned long long i0 = static_cast<unsigned long long>(blockIdx.x - im.block0) * blockDim.x +
                                 (threadIdx.x & ~31u);
         i0 < im.n; i0 += stride) {
        const unsigned long long i = i0 + lane;
        const unsigned long long o = im.offset + i;
        long long b = -1;
        double I = 0.0;
        if (i < im.n && set.ph.phase[o] == 3) {
            ++count;
            const unsigned long long px =
                dev::observation_bin(set.ph.theta_disp[o], -0.5 * im.W, 0.5 * im.W, im.nx);
            const unsigned long long py =
                dev::observation_bin(set.ph.phi_disp[o], -0.5 * im.H, 0.5 * im.H, im.ny);
            const unsigned long long pix = py * im.nx + px;
            I = set.ph.I[o];
            atomicAdd(&im.image[pix], I);
            atomicAdd(&im.image[npix + pix], set.ph.Q[o]);
            atomicAdd(&im.image[2 * npix + pix], set.ph.U[o]);
            atomicAdd(&im.image[3 * npix + pix], set.ph.V[o]);
            const double f = set.ph.frequency[o];
            if (set.bins > 0 && f >= set.spec_min && f <= set.spec_max)
                b = static_cast<long long>(dev::observation_bin(log10(f), set.log_min, set.log_max, set.bins));
        }
        // one sum per distinct bin of the warp (few: an image's arrival
        // frequencies crowd into a handful of bins), then one atomic
        unsigned pending = __ballot_sync(0xFFFFFFFFu, b >= 0);
        while (pending) {
            const long long b0 = __shfl_sync(0xFFFFFFFFu, b, __ffs(pending) - 1);
            const unsigned members = __ballot_sync(0xFFFFFFFFu, b == b0);
            double v = b == b0 ? I : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
            if (lane == 0) atomicAdd(shared_spec ? &hist[b0] : &im.spectrum[b0], v);
            pending &= ~members;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) count += __shfl_down_sync(0xFFFFFFFFu, count, off);
    if ((threadIdx.x & 31) == 0 && count) atomicAdd(&s_arrived, count);
    __syncthreads();
    if (shared_spec)
        for (unsigned long long q = threadIdx.x; q < set.bins; q += blockDim.x)
            if (hist[q] != 0.0) atomicAdd(&im.spectrum[q], hist[q]);
    if (threadIdx.x == 0 && s_arrived) atomicAdd(im.arrived, s_arrived);
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

// initialize_photons_disk (initialize_photons.hpp:173-327) for packet i: the
// cell is the last one whose offset is <= i (locate_superphoton_cell, :66-80);
// fluid sample, tetrad and fluid-frame magnetic field as the reference builds
// them; frequency/energy from the configured generator; an isotropic
// fluid-frame direction (mu, phi) lowered to p_mu.  Random draws: Philox
// keyed by (seed, photon id, domain 0xFFFFFFFF), generator draws first, then
// mu and phi, as in the reference.
__global__ void init_disk_photons(const __grid_constant__ DiskInitArgs args) {
    const unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x;
    if (i >= args.n) return;
    unsigned long long lo = 0, hi = args.ncell;
    while (lo + 1 < hi) {
        const unsigned long long mid = lo + (hi - lo) / 2;
        if (args.offsets[mid] <= i) lo = mid;
        else hi = mid;
    }
    const unsigned long long cell = lo;
    const int packets = static_cast<int>(args.offsets[cell + 1] - args.offsets[cell]);
    const double x = args.pos[3 * cell], y = args.pos[3 * cell + 1], z = args.pos[3 * cell + 2];
    FluidCellCGS fluid;
    fluid.position_cm[0] = x * args.length_scale;
    fluid.position_cm[1] = y * args.length_scale;
    fluid.position_cm[2] = z * args.length_scale;
    fluid.coordinate_time_s = 0.0 * args.time_scale;
    const double2 rt = args.rho_t[cell];
    fluid.density_g_cm3 = rt.x * args.density_scale;
    fluid.temperature_k = rt.y * args.temperature_scale;
    const double2 u01 = args.vel[2 * cell], u23 = args.vel[2 * cell + 1];
    fluid.coordinate_four_velocity_cm_s[0] = u01.x;
    fluid.coordinate_four_velocity_cm_s[1] = u01.y;
    fluid.coordinate_four_velocity_cm_s[2] = u23.x;
    fluid.coordinate_four_velocity_cm_s[3] = u23.y;
    const double2 b01 = args.mag[2 * cell], b23 = args.mag[2 * cell + 1];
    const double cm[4] = {b01.x, b01.y, b23.x, b23.y};
    dev::MetricAt m;
    dev::ks_metric(x, y, z, args.a, args.M, m);
    double e[4][4];
    const bool valid = dev::build_tetrad(m.g, fluid.coordinate_four_velocity_cm_s, e);
    fluid.magnetic_gauss[0] = fluid.magnetic_gauss[1] = fluid.magnetic_gauss[2] = fluid.magnetic_gauss[3] = 0.0;
    if (valid) {
        fluid.magnetic_gauss[0] = -dev::metric_dot(m.g, e[0], cm);
        for (int axis = 1; axis < 4; ++axis) fluid.magnetic_gauss[axis] = dev::metric_dot(m.g, e[axis], cm);
    }
    const uint64_t id = args.id_offset + i;
    dev::Philox rng(args.seed, id, 0xFFFFFFFFu);
    double nu = 0.0, E = 0.0;
    bool generated = false;
    if (valid && args.generator == 0) {
        generated = dev::generate_blackbody(fluid, rng, packets, args.energy, nu, E);
    } else if (valid && args.generator == 1) {
        generated = dev::generate_power_law(rng, packets, args.pl_slope, args.nu_min, args.nu_max, args.energy, nu, E);
    } else if (valid) {
        generated = GeneratePhotonsCustom(fluid, rng, packets, args.nu_custom, args.energy, nu, E);
    }
    const double mu = 2.0 * rng.drand() - 1.0;
    const double dphi = 2.0 * dev::kPi * rng.drand();
    const double tr = sqrt(fmax(0.0, 1.0 - mu * mu));
    double sn, cs;
    det_sincos(dphi, &sn, &cs);
    double p[4] = {0.0, 0.0, 0.0, 0.0};
    if (generated) {
        double w[4];
        for (int q = 0; q < 4; ++q) w[q] = e[0][q] + (tr * cs) * e[1][q] + (tr * sn) * e[2][q] + mu * e[3][q];
        for (int q = 0; q < 4; ++q) {
            double pq = 0.0;
            for (int nn = 0; nn < 4; ++nn) pq += m.g[q][nn] * w[nn];
            p[q] = pq;
        }
    }
    double ee = 0.0;
    if (generated)
        for (int c = 0; c < 4; ++c) ee -= p[c] * e[0][c];
    const KPhotons& P = args.ph;
    P.id[i] = id;
    P.frequency[i] = nu;
    P.emission_frame_energy[i] = ee;
    P.x0[i] = 0.0; P.x1[i] = x; P.x2[i] = y; P.x3[i] = z;
    P.k0[i] = p[0]; P.k1[i] = p[1]; P.k2[i] = p[2]; P.k3[i] = p[3];
    P.I[i] = generated ? E : 0.0;
    P.Q[i] = 0.0; P.U[i] = 0.0; P.V[i] = 0.0;
    P.dlambda[i] = args.dlambda0;
    P.terminate[i] = generated ? 0 : 1;
    P.phase[i] = generated ? 0 : 4;  // Disk / Rejected
    P.theta_disp[i] = 0.0;
    P.phi_disp[i] = 0.0;
}

// make_strided_host_values (write_output.hpp:13-24) for every selected field
// at once: blockIdx.y picks the field; 8-byte fields copy as 64-bit words.
__global__ void gather_fields(const __grid_constant__ GatherArgs a) {
    const int f = blockIdx.y;
    const unsigned long long step = static_cast<unsigned long long>(gridDim.x) * blockDim.x;
    for (unsigned long long j = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; j < a.count;
         j += step) {
        const unsigned long long i = j * a.stride;
        if (a.item[f] == 8)
            reinterpret_cast<unsigned long long*>(a.dst + a.dst_off[f])[j] =
                static_cast<const unsigned long long*>(a.src[f])[i];
        else
            a.dst[a.dst_off[f] + j] = static_cast<const unsigned char*>(a.src[f])[i];
    }
}

// ---- host-side launchers ----
cudaError_t launch_gather_fields(const GatherArgs& a, int sm_count, cudaStream_t stream) {
    if (a.count == 0 || a.nfields == 0) return cudaSuccess;
    if (a.nfields > kGatherMaxFields) return cudaErrorInvalidValue;
    const unsigned long long want = (a.count + 255) / 256;
    const unsigned long long cap = static_cast<unsigned long long>(sm_count) * 8;
    const dim3 grid(static_cast<unsigned>(want < cap ? want : cap), static_cast<unsigned>(a.nfields));
    gather_fields<<<grid, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_trace(const KParams& kp, bool mixed, int leg, int integrator, int sm_count, int blocks_per_sm,
                         size_t smem, cudaStream_t stream) {
    const int blocks = sm_count * blocks_per_sm;
    switch (leg + (mixed ? 4 : 0)) {
        case 0: return launch_trace_fp64_leg0(kp, integrator, blocks_per_sm, blocks, smem, stream);
        case 1: return launch_trace_fp64_leg1(kp, integrator, blocks_per_sm, blocks, smem, stream);
        case 2: return launch_trace_fp64_leg2(kp, integrator, blocks_per_sm, blocks, smem, stream);
        case 3: return launch_trace_fp64_leg3(kp, integrator, blocks_per_sm, blocks, smem, stream);
        case 4: return launch_trace_mixed_leg0(kp, integrator, blocks_per_sm, blocks, smem, stream);
        case 5: return launch_trace_mixed_leg1(kp, integrator, blocks_per_sm, blocks, smem, stream);
        case 6: return launch_trace_mixed_leg2(kp, integrator, blocks_per_sm, blocks, smem, stream);
        case 7: return launch_trace_mixed_leg3(kp, integrator, blocks_per_sm, blocks, smem, stream);
        default: return cudaErrorInvalidConfiguration;
    }
}

cudaError_t launch_init_image(const InitImageArgs& args, cudaStream_t stream) {
    const unsigned long long n = args.nx * args.nrows;
    if (n == 0) return cudaSuccess;
    const unsigned threads = 256;
    const unsigned blocks = static_cast<unsigned>((n + threads - 1) / threads);
    init_image_pixels<<<blocks, threads, 0, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_init_disk(const DiskInitArgs& a, cudaStream_t stream) {
    if (a.n == 0) return cudaSuccess;
    const unsigned threads = 128;
    const unsigned long long blocks = (a.n + threads - 1) / threads;
    if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
    init_disk_photons<<<static_cast<unsigned>(blocks), threads, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_image_products(ProductsSet& set, cudaStream_t stream) {
    const unsigned threads = 256;
    unsigned long long blocks = 0;
    for (int k = 0; k < set.nimages; ++k) {
        set.img[k].block0 = static_cast<unsigned>(blocks);
        // about four arrivals per thread: few blocks, so few spectrum flushes
        blocks += (set.img[k].n + 4 * threads - 1) / (4 * threads);
    }
    if (blocks == 0) return cudaSuccess;
    if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidConfiguration;
    set.blocks = static_cast<unsigned>(blocks);
    const size_t smem = set.bins <= kProductsSharedBins ? set.bins * sizeof(double) : 0;
    image_products<<<set.blocks, threads, smem, stream>>>(set);
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
