// Allocation-free tracing entry point (grt_trace_device_noalloc in grt.h).
//
// Some hosts cannot call cudaMalloc at the point where they trace: a framework
// that owns every byte of device memory through its own pool or a fixed
// budget, or a latency-critical loop that must not allocate after start-up
// (cudaMalloc can synchronise the device).  Such a caller keeps the grid and
// the photons in device memory it already owns; this entry point traces them
// in place and allocates nothing -- no cudaMalloc, cudaFree, event or stream.
//
// The only scratch the trace needs beyond its inputs and outputs -- the work
// queue head and launch counters, plus the separable grid axes and lookup
// bounds derived from the coordinate arrays (the bounds on the host, with the
// routine the context entry point uses, from a static host buffer) -- lives in one file-scope
// __device__ array of kNoallocScratchBytes (128 KiB) that every GPU which loads
// this library holds until the process exits.  All calls share it: each call
// clears the parts that must start at zero, and calls that overlap on the GPU
// (two streams, two host threads) race on it, so serialise calls per device.
// Its device address is looked up with cudaGetSymbolAddress on the first call
// made on each device (with that device current); make that first call before
// any stream capture.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "grt.h"
#include "grt_grid_axes.h"
#include "grt_kparams.h"
#include "grt_launch.h"
#include "grt_trace.cuh"

namespace {

constexpr size_t kNoallocScratchBytes = 128 * 1024;
constexpr size_t kCountersOffset = 0;                      // grt::KCounters
constexpr size_t kMetaOffset = 128;                        // GridMeta
constexpr size_t kAxesOffset = 256;                        // r, theta, phi axes, then their half-spans
constexpr size_t kMaxAxisValues = 8160;                    // 2 * 8160 doubles fit after kAxesOffset
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

struct GridMeta {
    int separable;
    int pad;
    double r_reject_lo;
    double r_reject_hi;
};

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Host copy of the staged axes and their half-spans while a call derives
// them (a static buffer: nothing is allocated on the host either).
std::mutex g_stage_mutex;
double g_stage_host[2 * kMaxAxisValues];

// Device address of g_noalloc_scratch on the current device (set-up once per device).
cudaError_t scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = ptr;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

// Separability test over every cell, many blocks: a cell whose coordinates
// differ from the outer product of the axes clears meta->separable (set to all
// ones before the launch).  Block 0 also copies the three axes into the
// scratch, from where the host reads them to derive the acceptance bounds.
__global__ void noalloc_check_grid(const double* r, const double* th, const double* ph, int nr, int nth, int nph,
                                   double* axes, GridMeta* meta) {
    const long long ncell = static_cast<long long>(nr) * nth * nph;
    const long long plane = static_cast<long long>(nth) * nph;
    bool ok = true;
    for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < ncell;
         q += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long i = q / plane;
        const long long j = (q / nph) % nth;
        const long long k = q % nph;
        if (!(r[q] == r[i * plane]) || !(th[q] == th[j * nph]) || !(ph[q] == ph[k])) ok = false;
    }
    if (__any_sync(0xFFFFFFFFu, !ok) && (threadIdx.x & 31) == 0) atomicAnd(&meta->separable, 0);
    if (blockIdx.x == 0) {
        for (int i = threadIdx.x; i < nr; i += blockDim.x) axes[i] = r[static_cast<long long>(i) * plane];
        for (int j = threadIdx.x; j < nth; j += blockDim.x) axes[nr + j] = th[static_cast<long long>(j) * nph];
        for (int k = threadIdx.x; k < nph; k += blockDim.x) axes[nr + nth + k] = ph[k];
    }
}

__global__ void noalloc_count_terminated(const uint8_t* term, unsigned long long n, unsigned long long* out) {
    unsigned long long c = 0;
    for (unsigned long long i = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<unsigned long long>(gridDim.x) * blockDim.x)
        c += term[i] ? 1 : 0;
    for (int off = 16; off > 0; off >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, off);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

template <int INTEGRATOR>
__global__ void __launch_bounds__(128, 4) trace_noalloc(const __grid_constant__ grt::KParams kp) {
    extern __shared__ double smem[];
    grt::dev::Axes ax;
    grt::dev::KStore kk;
    grt::dev::stage_grid(kp, smem, INTEGRATOR, ax, kk);
    grt::dev::trace_body<INTEGRATOR, grt::dev::Fp64Rhs, true>(kp, ax, kk);
}

grt_status set_err(char* err, size_t len, const char* msg) {
    if (err && len) {
        std::strncpy(err, msg, len - 1);
        err[len - 1] = '\0';
    }
    return GRT_EINVAL;
}

}  // namespace

extern "C" grt_status grt_trace_device_noalloc(const grt_params* p, const grt_device_grid* grid,
                                               const grt_photon_soa* photons, uint64_t n, grt_run_stats* stats,
                                               void* stream_ptr, char* err, size_t err_len) {
    if (!p || !photons) return set_err(err, err_len, "null params or photons");
    if (grt_params_validate(p, err, err_len) != GRT_OK) return GRT_EINVAL;
    if (p->precision != GRT_PREC_FP64)
        return set_err(err, err_len, "grt_trace_device_noalloc runs the FP64 parity form only");
    const uint64_t nr = grid ? grid->nr : 0, nth = grid ? grid->ntheta : 0, nph = grid ? grid->nphi : 0;
    const uint64_t ncell = nr * nth * nph;
    if (ncell && nr + nth + nph > kMaxAxisValues)
        return set_err(err, err_len,
                       "grid axes too long for the allocation-free scratch: nr + ntheta + nphi must be <= 8160");
    if (ncell >= (1ull << 31)) return set_err(err, err_len, "grid has 2^31 or more cells");
    if (ncell && (!grid->r || !grid->theta || !grid->phi || !grid->rho || !grid->temperature || !grid->vel4 ||
                  !grid->mag4))
        return set_err(err, err_len, "null device grid array");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    void* scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) return set_err(err, err_len, "cudaGetSymbolAddress failed");
    auto* counters = reinterpret_cast<grt::KCounters*>(static_cast<unsigned char*>(scratch) + kCountersOffset);
    auto* meta = reinterpret_cast<GridMeta*>(static_cast<unsigned char*>(scratch) + kMetaOffset);
    auto* axes = reinterpret_cast<double*>(static_cast<unsigned char*>(scratch) + kAxesOffset);
    auto cuda_fail = [&](cudaError_t e) {
        set_err(err, err_len, cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? GRT_ENOMEM : GRT_ECUDA;
    };

    grt::KParams kp;
    std::memset(&kp, 0, sizeof(kp));
    GridMeta gm{0, 0, 0.0, INFINITY};
    if (ncell) {
        // 1. the cell-by-cell separability check and the axes, on the device
        int sms_prep = 148, dev_prep = 0;
        cudaGetDevice(&dev_prep);
        cudaDeviceGetAttribute(&sms_prep, cudaDevAttrMultiProcessorCount, dev_prep);
        const unsigned long long want_blocks = (ncell + 255) / 256;
        const unsigned blocks = static_cast<unsigned>(
            want_blocks < static_cast<unsigned long long>(sms_prep) * 8 ? want_blocks : sms_prep * 8ull);
        cudaError_t e = cudaMemsetAsync(&meta->separable, 0xFF, sizeof(int), stream);
        if (e == cudaSuccess) {
            noalloc_check_grid<<<blocks, 256, 0, stream>>>(grid->r, grid->theta, grid->phi, static_cast<int>(nr),
                                                           static_cast<int>(nth), static_cast<int>(nph), axes, meta);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&gm, meta, sizeof(gm), cudaMemcpyDeviceToHost, stream);
        // 2. the acceptance half-spans and radial reject bounds on the host,
        //    with the routine grt_upload_grid uses (glibc arithmetic), so both
        //    entry points accept and reject the same samples at cell edges
        std::lock_guard<std::mutex> lock(g_stage_mutex);
        const size_t nax = nr + nth + nph;
        double* ha = g_stage_host;
        if (e == cudaSuccess) e = cudaMemcpyAsync(ha, axes, nax * sizeof(double), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e);
        const double *ra = ha, *ta = ha + nr, *pa = ha + nr + nth;
        const bool sep = gm.separable != 0 && grt::axes::axes_stageable(ra, nr, ta, nth, pa, nph);
        gm.separable = sep ? 1 : 0;
        gm.r_reject_lo = 0.0;
        gm.r_reject_hi = INFINITY;
        if (sep) {
            double* hh = ha + nax;
            grt::axes::half_spans(ra, nr, 0, hh);
            grt::axes::half_spans(ta, nth, 1, hh + nr);
            grt::axes::half_spans(pa, nph, 2, hh + nr + nth);
            grt::axes::radial_reject_bounds(ra, nr, &gm.r_reject_lo, &gm.r_reject_hi);
            // returns once the pageable source is staged, so the buffer may be
            // reused after the lock is released
            e = cudaMemcpyAsync(axes + nax, hh, nax * sizeof(double), cudaMemcpyHostToDevice, stream);
            if (e != cudaSuccess) return cuda_fail(e);
        }
    }
    kp.a = p->spin;
    kp.M = p->mass;
    kp.rcp_ok = grt::rcp_params_ok(p->spin, p->mass);
    kp.r_min = p->r_term_min;
    kp.r_max = p->r_term_max;
    kp.atol = p->atol;
    kp.rtol = p->rtol;
    kp.min_scale = p->min_step_scale;
    kp.max_scale = p->max_step_scale;
    kp.safety = p->safety;
    kp.albedo = p->scattering_albedo;
    kp.length_scale = p->length_cm_per_code;
    kp.time_scale = p->time_s_per_code;
    kp.density_scale = p->density_g_cm3_per_code;
    kp.temperature_scale = p->temperature_k_per_code;
    kp.norm = p->superphoton_count_normalization;
    kp.energy = p->energy_per_cell_erg;
    kp.pl_slope = p->power_law_slope;
    kp.nu_min = p->nu_min_hz;
    kp.nu_max = p->nu_max_hz;
    kp.seed = p->scattering_seed + static_cast<uint64_t>(p->rank);
    kp.integrator = p->integrator;
    kp.image_mode = p->mode == GRT_MODE_IMAGE;
    kp.abs_on = p->absorption_enabled && ncell;
    kp.emis_on = p->emission_enabled && ncell;
    kp.scat_on = p->scattering_enabled && ncell;
    kp.generator = p->generator;
    kp.img0 = grt::make_kimage(p->camera_theta, p->camera_phi, p->camera_distance, p->camera_width,
                                p->camera_height, p->custom_frequency_hz, p->absorption_coefficient,
                                p->emission_coefficient);
    grt::KGrid& g = kp.grid;
    g.nr = static_cast<int>(nr);
    g.nth = static_cast<int>(nth);
    g.nph = static_cast<int>(nph);
    g.available = ncell > 0;
    g.separable = gm.separable;
    g.r_axis = axes;
    g.th_axis = axes + nr;
    g.ph_axis = axes + nr + nth;
    g.r_half = axes + nr + nth + nph;
    g.th_half = g.r_half + nr;
    g.ph_half = g.th_half + nth;
    if (ncell) {
        g.r3 = grid->r;
        g.th3 = grid->theta;
        g.ph3 = grid->phi;
        g.rho_raw = grid->rho;
        g.T_raw = grid->temperature;
        g.vel_raw = grid->vel4;
        g.mag_raw = grid->mag4;
    }
    g.vel_scale = p->four_velocity_cm_s_per_code;
    g.mag_scale = p->magnetic_gauss_per_code;
    g.r_reject_lo = gm.r_reject_lo;
    g.r_reject_hi = gm.r_reject_hi;
    kp.ph.id = photons->id;
    kp.ph.frequency = photons->frequency;
    kp.ph.emission_frame_energy = photons->emission_frame_energy;
    kp.ph.x0 = photons->x0; kp.ph.x1 = photons->x1; kp.ph.x2 = photons->x2; kp.ph.x3 = photons->x3;
    kp.ph.k0 = photons->k0; kp.ph.k1 = photons->k1; kp.ph.k2 = photons->k2; kp.ph.k3 = photons->k3;
    kp.ph.I = photons->I; kp.ph.Q = photons->Q; kp.ph.U = photons->U; kp.ph.V = photons->V;
    kp.ph.dlambda = photons->dlambda;
    kp.ph.theta_disp = photons->theta_disp;
    kp.ph.phi_disp = photons->phi_disp;
    kp.ph.terminate = photons->terminate;
    kp.ph.phase = photons->phase;
    kp.n = n;
    kp.counters = counters;
    kp.refill_threshold = 8;
    kp.grab = 32;

    grt_run_stats st;
    std::memset(&st, 0, sizeof(st));
    // initially terminated photons (counted into the cleared counter slot)
    unsigned long long terminated = 0;
    if (n) {
        cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(grt::KCounters), stream);
        if (e == cudaSuccess) {
            noalloc_count_terminated<<<256, 256, 0, stream>>>(photons->terminate, n, &counters->terminated);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&terminated, &counters->terminated, sizeof(terminated), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e);
    }
    const size_t smem = grt::dev_trace_smem_bytes(p->integrator, 128, gm.separable != 0, static_cast<int>(nr),
                                                  static_cast<int>(nth), static_cast<int>(nph));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t interval = p->output_interval ? p->output_interval : 1;
    const bool single = p->termination_percent >= 1.0;
    int64_t step = 0, steps_done = 0;
    unsigned long long max_term_step = 0;
    while (n && step < p->max_steps) {
        int64_t end = p->max_steps;
        if (!single) {
            int64_t next = static_cast<int64_t>(((static_cast<uint64_t>(step) + interval - 1) / interval) * interval);
            if (next > p->max_steps - 1) next = p->max_steps - 1;
            end = next + 1;
        }
        kp.step0 = step;
        kp.budget = end - step;
        const unsigned long long warps = static_cast<unsigned long long>(sms) * 4 * 4;
        kp.max_iterations = static_cast<unsigned long long>(kp.budget + 2) * 13ull * ((n + warps - 1) / warps + 32) +
                            (1ull << 20);
        grt::KCounters host;
        cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(grt::KCounters), stream);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(p->integrator == GRT_RK4 ? trace_noalloc<0> : trace_noalloc<1>,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e == cudaSuccess) {
            if (p->integrator == GRT_RK4) trace_noalloc<0><<<sms * 4, 128, smem, stream>>>(kp);
            else trace_noalloc<1><<<sms * 4, 128, smem, stream>>>(kp);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&host, counters, sizeof(host), cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cuda_fail(e);
        terminated += host.terminated;
        st.accepted_steps += host.accepted;
        st.rejected_attempts += host.rejected;
        st.photon_calls += host.calls;
        st.launches += 1;
        if (host.max_term_step > max_term_step) max_term_step = host.max_term_step;
        if (host.timed_out) {
            st.timed_out = 1;
            st.steps_done = steps_done;
            st.n_terminated = terminated;
            if (stats) *stats = st;
            set_err(err, err_len, "trace kernel hit its iteration limit");
            return GRT_ETIMEOUT;
        }
        step = end;
        steps_done = end;
        if (static_cast<double>(terminated) / static_cast<double>(n) >= p->termination_percent) break;
    }
    if (single && n && terminated >= n) {
        const int64_t last = max_term_step ? static_cast<int64_t>(max_term_step) - 1 : 0;
        int64_t s_out = static_cast<int64_t>(((static_cast<uint64_t>(last) + interval - 1) / interval) * interval);
        if (s_out > p->max_steps - 1) s_out = p->max_steps - 1;
        steps_done = s_out + 1;
    }
    st.steps_done = n ? steps_done : p->max_steps;
    st.n_terminated = terminated;
    if (stats) *stats = st;
    return GRT_OK;
}
