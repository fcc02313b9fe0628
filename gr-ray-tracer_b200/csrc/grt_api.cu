// C ABI of the hot path (include/grt.h): context, device buffers, the host
// step loop with the reference's termination semantics, and image products.
//
// Reference interfaces replaced (file:line within the reference project):
//   grt_upload_grid        ScatteringFluidGrid build (integrate_cart_ks.hpp:436-459)
//   grt_upload_photons     Photons device views (utils.hpp:40-133)
//   grt_init_image_photons initialize_photons_image (initialize_photons.hpp:82-170)
//   grt_run                integrate_geodesics step loop (integrate_cart_ks.hpp:468-527)
//   grt_get_image_products build_observation_products (observation.hpp:31-84)
//   grt_write_image_products_npz write_image_products (write_output.hpp:107-142)
//   grt_init_image_batch / grt_render_graph  batched images in one launch, CUDA graph (no reference counterpart)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <string>
#include <vector>

#include "grt.h"
#include "grt_grid_axes.h"
#include "grt_host.h"
#include "grt_kparams.h"
#include "grt_launch.h"
#include "grt_user_physics.h"

namespace {


template <class T>
struct DevBuf {
    T* ptr = nullptr;
    size_t count = 0;
    cudaError_t alloc(size_t n) {
        if (n <= count && ptr) return cudaSuccess;
        release();
        if (n == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T));
        if (e == cudaSuccess) count = n;
        else ptr = nullptr;
        return e;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
};

template <class T>
struct FieldView {
    T* ptr = nullptr;
};

// Byte offset of photon field k (grt_photon_soa order: 0 id, 1..17 the
// doubles, 18 terminate, 19 phase) in a block of n photons: the fields back
// to back, 146 bytes per photon, the 8-byte fields first.
size_t photon_field_offset(size_t n, int k) { return k <= 17 ? 8 * n * static_cast<size_t>(k) : 144 * n + n * (k - 18); }

// The photon SoA in one device block laid out by photon_field_offset; a host
// SoA in the same layout (grt_host_photon_layout) moves with one copy.
struct PhotonBufs {
    DevBuf<unsigned char> block;
    size_t n = 0;
    FieldView<uint64_t> id;
    FieldView<double> f[17];  // frequency .. phi_disp in grt_photon_soa order
    FieldView<uint8_t> term, phase;
    cudaError_t alloc(size_t count) {
        const cudaError_t e = block.alloc(146 * count);
        if (e != cudaSuccess) {
            release();
            return e;
        }
        n = count;
        unsigned char* b = block.ptr;
        id.ptr = reinterpret_cast<uint64_t*>(b);
        for (int q = 0; q < 17; ++q) f[q].ptr = reinterpret_cast<double*>(b + photon_field_offset(count, q + 1));
        term.ptr = b + photon_field_offset(count, 18);
        phase.ptr = b + photon_field_offset(count, 19);
        return cudaSuccess;
    }
    void release() {
        block.release();
        n = 0;
        id.ptr = nullptr;
        for (auto& v : f) v.ptr = nullptr;
        term.ptr = phase.ptr = nullptr;
    }
    grt::KPhotons view() const {
        grt::KPhotons k;
        k.id = id.ptr;
        double** d[17] = {&k.frequency, &k.emission_frame_energy, &k.x0, &k.x1, &k.x2, &k.x3,
                          &k.k0, &k.k1, &k.k2, &k.k3, &k.I, &k.Q, &k.U, &k.V,
                          &k.dlambda, &k.theta_disp, &k.phi_disp};
        for (int q = 0; q < 17; ++q) *d[q] = f[q].ptr;
        k.terminate = term.ptr;
        k.phase = phase.ptr;
        return k;
    }
};

double* const* soa_doubles(const grt_photon_soa* s, double* out[17]) {
    double* src[17] = {s->frequency, s->emission_frame_energy, s->x0, s->x1, s->x2, s->x3,
                       s->k0, s->k1, s->k2, s->k3, s->I, s->Q, s->U, s->V,
                       s->dlambda, s->theta_disp, s->phi_disp};
    for (int q = 0; q < 17; ++q) out[q] = src[q];
    return out;
}

// True when the 20 fields of s are one block in photon_field_offset's layout
// for n photons (the layout grt_host_photon_layout hands out).
bool soa_is_block(const grt_photon_soa* s, size_t n) {
    const unsigned char* b = reinterpret_cast<const unsigned char*>(s->id);
    if (!b) return false;
    double* d[17];
    soa_doubles(s, d);
    for (int q = 0; q < 17; ++q)
        if (reinterpret_cast<const unsigned char*>(d[q]) != b + photon_field_offset(n, q + 1)) return false;
    return s->terminate == b + photon_field_offset(n, 18) && s->phase == b + photon_field_offset(n, 19);
}

}  // namespace

struct grt_ctx {
    grt_params p;
    int device = 0;
    int sm_count = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    // grid
    bool grid_uploaded = false;
    bool fluid_available = false;
    bool separable = false;
    int nr = 0, nth = 0, nph = 0;
    double r_reject_lo = 0.0, r_reject_hi = 0.0;
    DevBuf<double> r_axis, th_axis, ph_axis, r_half, th_half, ph_half, r3, th3, ph3;
    DevBuf<double2> rho_t, vel, mag;
    DevBuf<double> cell_pos;               // [ncell][3] Cartesian KS cell positions (disk emission)
    std::vector<double> host_rho;          // code-unit density (disk packet counts)
    DevBuf<unsigned long long> disk_offsets;
    // photons
    size_t n = 0;
    PhotonBufs ph;
    unsigned long long initial_terminated = 0;
    // scratch: launch counters and products
    DevBuf<grt::KCounters> counters;
    grt::KCounters* host_counters = nullptr;  // pinned
    DevBuf<double> image, spectrum;
    DevBuf<unsigned long long> arrived;
    DevBuf<unsigned long long> scratch_u64;
    unsigned long long* host_u64 = nullptr;  // pinned
    grt_launch_config lc{128, 0, 8, 32, 1, 0, 0};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // images of the last grt_init_image_photons (one, cameras from p) or
    // grt_init_image_batch call; image k owns photon slots
    // [image_start[k], image_start[k+1])
    std::vector<grt_image_spec> images;
    std::vector<unsigned long long> image_start;
    uint64_t image_id_offset = 0;
    double forward_back = 0.0;  // > 0: line-of-sight forward rays from -forward_back * n
    bool random_screen = false;  // image rays at the reference's random screen positions
    uint64_t row0 = 0, nrows = 0;  // single image: pixel rows [row0, row0 + nrows) only (nrows 0 = all)
    bool batched = false;      // trace kernels read the per-image table
    bool have_images = false;  // photons came from an image init (a render can re-initialise them)
    DevBuf<grt::KImage> images_dev;
    DevBuf<unsigned long long> image_start_dev;
    // channel groups of the batch: images with the same camera and screen
    // share one geodesic per pixel (when scattering is off)
    bool share_channels = true;
    int ngroups = 0;
    bool groups_share = false;            // some group has two or more channels
    unsigned long long geodesics = 0;     // queue length with sharing
    DevBuf<unsigned long long> group_qstart_dev;
    // tile orders of the image-mode queue (queue position -> index): over
    // photon slots and over the geodesics of channel groups
    DevBuf<unsigned> order_ph, order_geo;
    // layout the tile orders were built for (image slot starts and widths,
    // group starts and widths): a new image set with the same layout reuses them
    std::vector<unsigned long long> order_layout;
    // per-SM first-claim counters of the trace launches (KParams::sm_claims)
    DevBuf<unsigned> sm_claims;
    bool order_ph_ok = false, order_geo_ok = false;
    DevBuf<int> group_chan_dev, chan_img_dev;
    DevBuf<unsigned long long> share_state;  // [geodesics] lead / finished channels (KParams::share_state)
    DevBuf<long long> calls_carry;           // [queue] calls taken in the backward-leg launch
    // output-step archives: gathered fields on the device, then in pinned host memory
    DevBuf<unsigned char> out_stage;
    unsigned char* host_out = nullptr;
    size_t host_out_bytes = 0;
    // per-image products of a batch: image k's I,Q,U,V at bimage + bimage_off[k]
    DevBuf<double> bimage, bspectrum;
    DevBuf<unsigned long long> barrived;
    std::vector<size_t> bimage_off;
    bool bproducts_valid = false;
    // per-cell multipliers on dtau / dI (differentiable RT)
    DevBuf<double> m_abs, m_emis;
    bool has_m_abs = false, has_m_emis = false;
    // checkpointed forward / adjoint
    DevBuf<double> ckpt, tape, dLdI, g_abs, g_emis;
    DevBuf<int> nckpt, adj_overflow;
    DevBuf<long long> call0;
    int adj_K = 0, adj_cap = 0;
    bool adj_ready = false;
    // render graph, valid while generation == graph_generation
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    uint64_t generation = 1, graph_generation = 0;
    // asynchronous renders (grt_render_async / grt_render_wait): the photon
    // upload and the products' copy-back run on copy_stream, the trace on
    // stream; one render in flight per context
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_uploaded = nullptr, ev_traced = nullptr, ev_done = nullptr;
    bool render_pending = false;
};

namespace {

grt_status fail(grt_ctx* c, grt_status s, const std::string& msg) {
    if (c) c->err = msg;
    return s;
}

grt_status cuda_fail(grt_ctx* c, cudaError_t e, const char* what) {
    return fail(c, e == cudaErrorMemoryAllocation ? GRT_ENOMEM : GRT_ECUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}

#define GRT_CUDA(ctx, call, what)                        \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
    } while (0)

// fluid_frame.hpp:28-48 on the host (glibc sin/cos, exactly the reference's
// arithmetic), then the [units] scale, as sample_scattering_fluid applies it
// per step (scattering.hpp:223-241).
void spherical_to_cartesian_vec(double r, double th, double ph, double spin, const double s[4], double scale,
                                double c[4]) {
    const double st = std::sin(th), ct = std::cos(th);
    const double sp = std::sin(ph), cp = std::cos(ph);
    const double radial_x = cp * st, radial_y = sp * st, radial_z = ct;
    const double theta_x = (r * cp - spin * sp) * ct;
    const double theta_y = (r * sp + spin * cp) * ct;
    const double theta_z = -r * st;
    const double phi_x = (-r * sp - spin * cp) * st;
    const double phi_y = (r * cp - spin * sp) * st;
    c[0] = s[0];
    c[1] = radial_x * s[1] + theta_x * s[2] + phi_x * s[3];
    c[2] = radial_y * s[1] + theta_y * s[2] + phi_y * s[3];
    c[3] = radial_z * s[1] + theta_z * s[2];
    for (int q = 0; q < 4; ++q) c[q] *= scale;
}

// Shared memory a trace block may spend on staged separable axes (the RK45
// stage slots take 42 KB of the 227 KB a block can have).
constexpr size_t kMaxStagedAxisBytes = 160 * 1024;

grt::KParams make_kparams(const grt_ctx* c) {
    const grt_params& p = c->p;
    grt::KParams k;
    std::memset(&k, 0, sizeof(k));
    k.a = p.spin;
    k.M = p.mass;
    k.r_min = p.r_term_min;
    k.r_max = p.r_term_max;
    k.atol = p.atol;
    k.rtol = p.rtol;
    k.min_scale = p.min_step_scale;
    k.max_scale = p.max_step_scale;
    k.safety = p.safety;
    k.albedo = p.scattering_albedo;
    k.length_scale = p.length_cm_per_code;
    k.time_scale = p.time_s_per_code;
    k.density_scale = p.density_g_cm3_per_code;
    k.temperature_scale = p.temperature_k_per_code;
    k.norm = p.superphoton_count_normalization;
    k.energy = p.energy_per_cell_erg;
    k.pl_slope = p.power_law_slope;
    k.nu_min = p.nu_min_hz;
    k.nu_max = p.nu_max_hz;
    k.seed = p.scattering_seed + static_cast<uint64_t>(p.rank);
    k.integrator = p.integrator;
    k.image_mode = p.mode == GRT_MODE_IMAGE;
    // integrate_cart_ks.hpp:446-452: physics flags are gated on fluid availability.
    k.abs_on = p.absorption_enabled && c->fluid_available;
    k.emis_on = p.emission_enabled && c->fluid_available;
    k.scat_on = p.scattering_enabled && c->fluid_available;
    k.generator = p.generator;
    // camera_plane_crossing basis (integrate_cart_ks.hpp:97-107), host libm.
    k.img0 = grt::make_kimage(p.camera_theta, p.camera_phi, p.camera_distance, p.camera_width,
                                p.camera_height, p.custom_frequency_hz, p.absorption_coefficient,
                                p.emission_coefficient);
    grt::KGrid& g = k.grid;
    g.nr = c->nr;
    g.nth = c->nth;
    g.nph = c->nph;
    g.available = c->fluid_available;
    g.separable = c->separable;
    g.r_axis = c->r_axis.ptr;
    g.th_axis = c->th_axis.ptr;
    g.ph_axis = c->ph_axis.ptr;
    g.r_half = c->r_half.ptr;
    g.th_half = c->th_half.ptr;
    g.ph_half = c->ph_half.ptr;
    g.r3 = c->r3.ptr;
    g.th3 = c->th3.ptr;
    g.ph3 = c->ph3.ptr;
    g.rho_t = c->rho_t.ptr;
    g.vel = c->vel.ptr;
    g.mag = c->mag.ptr;
    g.r_reject_lo = c->r_reject_lo;
    g.r_reject_hi = c->r_reject_hi;
    k.m_abs = c->has_m_abs ? c->m_abs.ptr : nullptr;
    k.m_emis = c->has_m_emis ? c->m_emis.ptr : nullptr;
    if (c->batched) {
        k.images = c->images_dev.ptr;
        k.image_start = c->image_start_dev.ptr;
        k.nimages = static_cast<int>(c->images.size());
    }
    k.ph = c->ph.view();
    k.n = c->n;
    // Frequency channels share their geodesic when nothing channel-specific
    // can change it: no scattering (its draws are keyed by each photon's id).
    if (c->batched && c->share_channels && c->groups_share && !k.scat_on) {
        k.ngroups = c->ngroups;
        k.group_qstart = c->group_qstart_dev.ptr;
        k.group_chan = c->group_chan_dev.ptr;
        k.chan_img = c->chan_img_dev.ptr;
        k.n = c->geodesics;
        k.share_state = c->share_state.ptr;
    }
    if (k.image_mode && c->have_images && !c->random_screen)
        k.order = k.ngroups > 0 ? (c->order_geo_ok ? c->order_geo.ptr : nullptr)
                                : (c->order_ph_ok ? c->order_ph.ptr : nullptr);
    k.calls_carry = c->calls_carry.ptr;
    k.counters = c->counters.ptr;
    k.refill_threshold = c->lc.refill_threshold;
    k.grab = c->lc.photons_per_grab;
    k.fp64_radius_sq = 16.0 * p.mass * p.mass + p.spin * p.spin;
    k.fp64_axis_sin2 = 0.01;
    // FP32 right-hand side for RK45 calls outside the fluid grid (lookup can
    // never accept radii above r_reject_hi); without a grid, everywhere.
    // (GRT_PREC_MIXED_GRID: inside the grid too, after emission)
    k.fp32_min_radius_sq = c->fluid_available && p.precision != GRT_PREC_MIXED_GRID
                               ? (std::isfinite(c->r_reject_hi) ? c->r_reject_hi * c->r_reject_hi : INFINITY)
                               : 0.0;
    k.renormalize = 1;
    k.rcp_ok = grt::rcp_params_ok(p.spin, p.mass);
    return k;
}

}  // namespace

extern "C" {

int32_t grt_abi_version(void) { return GRT_ABI_VERSION; }

const char* grt_build_info(void) {
    return "gr-ray-tracer-b200 hot path; sm_100a; FP64 parity kernels built with -fmad=false";
}

const char* grt_last_error(const grt_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

// Between grt_render_async and grt_render_wait the context's device buffers
// belong to the render in flight: calls that would enqueue work on them or
// read them are refused.
static grt_status rendering(grt_ctx* c) {
    return fail(c, GRT_ESTATE, "a render is in flight on this context (grt_render_wait first)");
}

grt_status grt_create(const grt_params* p, grt_ctx** out) {
    if (!p || !out) return GRT_EINVAL;
    *out = nullptr;
    char buf[512];
    if (grt_params_validate(p, buf, sizeof(buf)) != GRT_OK) return GRT_EINVAL;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GRT_ENODEV;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return GRT_ENODEV;
    if (prop.major < 10) return GRT_ENODEV;
    grt_ctx* c = new grt_ctx();
    c->p = *p;
    c->device = dev;
    c->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        c->counters.alloc(1) != cudaSuccess || c->sm_claims.alloc(grt::kSmClaimSlots) != cudaSuccess ||
        c->scratch_u64.alloc(4) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&c->host_counters), sizeof(grt::KCounters)) != cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void**>(&c->host_u64), 4 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_uploaded, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_traced, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_done, cudaEventDisableTiming) != cudaSuccess) {
        grt_destroy(c);
        return GRT_ECUDA;
    }
    c->stream = c->own_stream;
    *out = c;
    return GRT_OK;
}

void grt_destroy(grt_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    c->r_axis.release(); c->th_axis.release(); c->ph_axis.release();
    c->r_half.release(); c->th_half.release(); c->ph_half.release();
    c->r3.release(); c->th3.release(); c->ph3.release();
    c->rho_t.release(); c->vel.release(); c->mag.release();
    c->cell_pos.release(); c->disk_offsets.release();
    c->ph.release();
    c->counters.release();
    c->image.release(); c->spectrum.release(); c->arrived.release(); c->scratch_u64.release();
    c->images_dev.release(); c->image_start_dev.release();
    c->group_qstart_dev.release(); c->group_chan_dev.release(); c->chan_img_dev.release();
    c->order_ph.release(); c->order_geo.release(); c->sm_claims.release();
    c->m_abs.release(); c->m_emis.release();
    c->ckpt.release(); c->tape.release(); c->dLdI.release(); c->g_abs.release(); c->g_emis.release();
    c->nckpt.release(); c->adj_overflow.release(); c->call0.release();
    c->bimage.release(); c->bspectrum.release(); c->barrived.release();
    c->share_state.release(); c->calls_carry.release(); c->out_stage.release();
    if (c->host_out) cudaFreeHost(c->host_out);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->host_counters) cudaFreeHost(c->host_counters);
    if (c->host_u64) cudaFreeHost(c->host_u64);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->ev_uploaded) cudaEventDestroy(c->ev_uploaded);
    if (c->ev_traced) cudaEventDestroy(c->ev_traced);
    if (c->ev_done) cudaEventDestroy(c->ev_done);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

grt_status grt_set_params(grt_ctx* c, const grt_params* p) {
    if (c && c->render_pending) return rendering(c);
    if (!c || !p) return GRT_EINVAL;
    char buf[512];
    if (grt_params_validate(p, buf, sizeof(buf)) != GRT_OK) return fail(c, GRT_EINVAL, buf);
    c->p = *p;
    ++c->generation;
    return GRT_OK;
}

grt_status grt_set_stream(grt_ctx* c, void* stream) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
    ++c->generation;
    return GRT_OK;
}

grt_status grt_synchronize(grt_ctx* c) {
    if (!c) return GRT_EINVAL;
    GRT_CUDA(c, cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
    return GRT_OK;
}

grt_status grt_get_launch_config(const grt_ctx* c, grt_launch_config* cfg) {
    if (!c || !cfg) return GRT_EINVAL;
    *cfg = c->lc;
    return GRT_OK;
}

grt_status grt_set_launch_config(grt_ctx* c, const grt_launch_config* cfg) {
    if (c && c->render_pending) return rendering(c);
    if (!c || !cfg) return GRT_EINVAL;
    if (cfg->threads_per_block != 128)
        return fail(c, GRT_EINVAL, "threads_per_block must be 128 (the trace kernels' block size)");
    if (cfg->blocks_per_sm != 0 && (cfg->blocks_per_sm < 2 || cfg->blocks_per_sm > 4))
        return fail(c, GRT_EINVAL,
                    "blocks_per_sm must be 0 (automatic), 2, 3 or 4 (register caps 255, 170, 128)");
    if (cfg->refill_threshold < 1 || cfg->refill_threshold > 32)
        return fail(c, GRT_EINVAL, "refill_threshold must be in [1, 32]");
    if (cfg->photons_per_grab < 1 || cfg->photons_per_grab > (1 << 20))
        return fail(c, GRT_EINVAL, "photons_per_grab must be in [1, 2^20]");
    if (cfg->split_legs != 0 && cfg->split_legs != 1) return fail(c, GRT_EINVAL, "split_legs must be 0 or 1");
    if (cfg->max_iterations < 0) return fail(c, GRT_EINVAL, "max_iterations must be >= 0 (0 = automatic)");
    c->lc = *cfg;
    c->lc.pad = 0;
    ++c->generation;
    return GRT_OK;
}

grt_status grt_upload_grid(grt_ctx* c, size_t nr, size_t nth, size_t nph, const double* r, const double* th,
                           const double* ph, const double* rho, const double* T, const double* vel4,
                           const double* mag4) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    const size_t ncell = nr * nth * nph;
    ++c->generation;
    c->grid_uploaded = true;
    c->fluid_available = false;
    c->separable = false;
    c->nr = c->nth = c->nph = 0;
    if (ncell == 0) return GRT_OK;  // vacuum: fluid_available stays false
    if (!r || !th || !ph || !rho || !T || !vel4 || !mag4) return fail(c, GRT_EINVAL, "null grid array");
    if (nr > (1u << 30) || nth > (1u << 30) || nph > (1u << 30) || ncell > (1ull << 31))
        return fail(c, GRT_EINVAL, "grid too large for 32-bit cell indices");
    c->nr = static_cast<int>(nr);
    c->nth = static_cast<int>(nth);
    c->nph = static_cast<int>(nph);
    // Separable sorted coordinates -> per-axis binary-search lookup; otherwise
    // the reference's coordinate-descent scans over the full arrays.
    std::vector<double> ra(nr), ta(nth), pa(nph);
    for (size_t i = 0; i < nr; ++i) ra[i] = r[i * nth * nph];
    for (size_t j = 0; j < nth; ++j) ta[j] = th[j * nph];
    for (size_t k = 0; k < nph; ++k) pa[k] = ph[k];
    bool sep = true;
    for (size_t i = 0; i < nr && sep; ++i)
        for (size_t j = 0; j < nth && sep; ++j)
            for (size_t k = 0; k < nph && sep; ++k) {
                const size_t q = (i * nth + j) * nph + k;
                if (!(r[q] == ra[i]) || !(th[q] == ta[j]) || !(ph[q] == pa[k])) sep = false;
            }
    sep = sep && grt::axes::axes_stageable(ra.data(), nr, ta.data(), nth, pa.data(), nph);
    // the staged axes and half-spans (16 bytes per axis value) must fit in
    // shared memory beside the RK45 stage slots; longer axes use the general
    // lookup on the full coordinate arrays
    sep = sep && 16 * (nr + nth + nph) <= kMaxStagedAxisBytes;
    c->separable = sep;
    // Radii outside [lo, hi] fail within_radial_cell for every cell (margin
    // 0.6 > 0.500001 of the outermost log spacing), so lookup can stop early.
    c->r_reject_lo = 0.0;
    c->r_reject_hi = INFINITY;
    if (sep) grt::axes::radial_reject_bounds(ra.data(), nr, &c->r_reject_lo, &c->r_reject_hi);
    std::vector<double2> rt(ncell), uv(2 * ncell), bv(2 * ncell);
    std::vector<double> pos(3 * ncell);
    c->host_rho.assign(rho, rho + ncell);
    for (size_t q = 0; q < ncell; ++q) {
        rt[q] = make_double2(rho[q], T[q]);
        // spherical_kerr_schild_to_cartesian (fluid_frame.hpp:15-26), host libm
        const double st = std::sin(th[q]), ct = std::cos(th[q]), sp = std::sin(ph[q]), cp = std::cos(ph[q]);
        pos[3 * q] = (r[q] * cp - c->p.spin * sp) * st;
        pos[3 * q + 1] = (r[q] * sp + c->p.spin * cp) * st;
        pos[3 * q + 2] = r[q] * ct;
        double u[4], b[4];
        spherical_to_cartesian_vec(r[q], th[q], ph[q], c->p.spin, vel4 + 4 * q, c->p.four_velocity_cm_s_per_code, u);
        spherical_to_cartesian_vec(r[q], th[q], ph[q], c->p.spin, mag4 + 4 * q, c->p.magnetic_gauss_per_code, b);
        uv[2 * q] = make_double2(u[0], u[1]);
        uv[2 * q + 1] = make_double2(u[2], u[3]);
        bv[2 * q] = make_double2(b[0], b[1]);
        bv[2 * q + 1] = make_double2(b[2], b[3]);
    }
    GRT_CUDA(c, c->rho_t.alloc(ncell), "alloc rho_t");
    GRT_CUDA(c, c->vel.alloc(2 * ncell), "alloc vel");
    GRT_CUDA(c, c->mag.alloc(2 * ncell), "alloc mag");
    GRT_CUDA(c, c->r_axis.alloc(nr), "alloc axis");
    GRT_CUDA(c, c->th_axis.alloc(nth), "alloc axis");
    GRT_CUDA(c, c->ph_axis.alloc(nph), "alloc axis");
    GRT_CUDA(c, c->cell_pos.alloc(3 * ncell), "alloc positions");
    GRT_CUDA(c, cudaMemcpy(c->cell_pos.ptr, pos.data(), 3 * ncell * sizeof(double), cudaMemcpyHostToDevice),
             "H2D positions");
    GRT_CUDA(c, cudaMemcpy(c->rho_t.ptr, rt.data(), ncell * sizeof(double2), cudaMemcpyHostToDevice), "H2D grid");
    GRT_CUDA(c, cudaMemcpy(c->vel.ptr, uv.data(), 2 * ncell * sizeof(double2), cudaMemcpyHostToDevice), "H2D grid");
    GRT_CUDA(c, cudaMemcpy(c->mag.ptr, bv.data(), 2 * ncell * sizeof(double2), cudaMemcpyHostToDevice), "H2D grid");
    GRT_CUDA(c, cudaMemcpy(c->r_axis.ptr, ra.data(), nr * sizeof(double), cudaMemcpyHostToDevice), "H2D axis");
    GRT_CUDA(c, cudaMemcpy(c->th_axis.ptr, ta.data(), nth * sizeof(double), cudaMemcpyHostToDevice), "H2D axis");
    GRT_CUDA(c, cudaMemcpy(c->ph_axis.ptr, pa.data(), nph * sizeof(double), cudaMemcpyHostToDevice), "H2D axis");
    if (sep) {
        std::vector<double> rh(nr), th_h(nth), ph_h(nph);
        grt::axes::half_spans(ra.data(), nr, 0, rh.data());
        grt::axes::half_spans(ta.data(), nth, 1, th_h.data());
        grt::axes::half_spans(pa.data(), nph, 2, ph_h.data());
        GRT_CUDA(c, c->r_half.alloc(nr), "alloc half");
        GRT_CUDA(c, c->th_half.alloc(nth), "alloc half");
        GRT_CUDA(c, c->ph_half.alloc(nph), "alloc half");
        GRT_CUDA(c, cudaMemcpy(c->r_half.ptr, rh.data(), nr * sizeof(double), cudaMemcpyHostToDevice), "H2D half");
        GRT_CUDA(c, cudaMemcpy(c->th_half.ptr, th_h.data(), nth * sizeof(double), cudaMemcpyHostToDevice), "H2D half");
        GRT_CUDA(c, cudaMemcpy(c->ph_half.ptr, ph_h.data(), nph * sizeof(double), cudaMemcpyHostToDevice), "H2D half");
    }
    if (!sep) {
        GRT_CUDA(c, c->r3.alloc(ncell), "alloc r3");
        GRT_CUDA(c, c->th3.alloc(ncell), "alloc th3");
        GRT_CUDA(c, c->ph3.alloc(ncell), "alloc ph3");
        GRT_CUDA(c, cudaMemcpy(c->r3.ptr, r, ncell * sizeof(double), cudaMemcpyHostToDevice), "H2D r3");
        GRT_CUDA(c, cudaMemcpy(c->th3.ptr, th, ncell * sizeof(double), cudaMemcpyHostToDevice), "H2D th3");
        GRT_CUDA(c, cudaMemcpy(c->ph3.ptr, ph, ncell * sizeof(double), cudaMemcpyHostToDevice), "H2D ph3");
    }
    c->fluid_available = true;
    return GRT_OK;
}

grt_status grt_upload_grid_numpy_dir(grt_ctx* c, const char* dir) {
    if (c && c->render_pending) return rendering(c);
    if (!c || !dir) return GRT_EINVAL;
    namespace fs = std::filesystem;
    const fs::path root(dir);
    if (!fs::exists(root)) return fail(c, GRT_EIO, "NumPy directory does not exist: " + root.string());
    if (!fs::is_directory(root)) return fail(c, GRT_EIO, "NumPy input path is not a directory: " + root.string());
    const char* names[7] = {"r.npy", "theta.npy", "phi.npy", "rho.npy", "Tgas.npy", "vel.npy", "mag.npy"};
    std::string missing;
    for (const char* n : names)
        if (!fs::is_regular_file(root / n)) missing += (missing.empty() ? "" : ", ") + std::string(n);
    if (!missing.empty())
        return fail(c, GRT_EIO, "NumPy directory '" + root.string() + "' is missing required file(s): " + missing);
    std::vector<double> a[7];
    std::vector<size_t> shape[7];
    for (int q = 0; q < 7; ++q) {
        std::string e;
        if (!grt::npy_load_f64((root / names[q]).string(), shape[q], a[q], e)) return fail(c, GRT_EIO, e);
    }
    const std::vector<size_t>& s0 = shape[0];
    if (s0.size() != 3 || s0[0] == 0 || s0[1] == 0 || s0[2] == 0)
        return fail(c, GRT_EINVAL, "Coordinate grid must have shape (nr, ntheta, nphi): " + (root / names[0]).string());
    for (int q = 1; q < 7; ++q) {
        const size_t dims = q >= 5 ? 4 : 3;
        if (shape[q].size() != dims || shape[q][0] != s0[0] || shape[q][1] != s0[1] || shape[q][2] != s0[2])
            return fail(c, GRT_EINVAL, std::string("Grid field has incompatible dimensions: ") + (root / names[q]).string());
        if (dims == 4 && shape[q][3] != 4)
            return fail(c, GRT_EINVAL, std::string("Four-vector field must have four components: ") + (root / names[q]).string());
    }
    return grt_upload_grid(c, s0[0], s0[1], s0[2], a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(),
                           a[5].data(), a[6].data());
}

static grt_status count_initial_terminated(grt_ctx* c) {
    GRT_CUDA(c, cudaMemsetAsync(c->scratch_u64.ptr, 0, sizeof(unsigned long long), c->stream), "memset");
    GRT_CUDA(c, grt::launch_count_terminated(c->ph.term.ptr, c->n, c->scratch_u64.ptr, c->sm_count, c->stream),
             "count_terminated");
    GRT_CUDA(c, cudaMemcpyAsync(c->host_u64, c->scratch_u64.ptr, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                c->stream), "D2H count");
    GRT_CUDA(c, cudaStreamSynchronize(c->stream), "sync");
    c->initial_terminated = c->host_u64[0];
    return GRT_OK;
}

grt_status grt_upload_photons(grt_ctx* c, const grt_photon_soa* s, size_t n) {
    if (c && c->render_pending) return rendering(c);
    if (!c || (!s && n)) return GRT_EINVAL;
    if (n > (1ull << 40)) return fail(c, GRT_EINVAL, "photon count too large");
    const bool keep_images = c->have_images && n == c->n;  // same slots: photons keep their images
    c->adj_ready = false;
    GRT_CUDA(c, c->ph.alloc(n), "alloc photons");
    c->n = n;
    c->bproducts_valid = false;
    if (!keep_images) {
        ++c->generation;
        c->images.clear();
        c->image_start.clear();
        c->batched = false;
        c->have_images = false;
    }
    if (n == 0) {
        c->initial_terminated = 0;
        return GRT_OK;
    }
    double* src[17];
    soa_doubles(s, src);
    if (!s->id || !s->terminate || !s->phase) return fail(c, GRT_EINVAL, "null photon field");
    for (double* q : src)
        if (!q) return fail(c, GRT_EINVAL, "null photon field");
    if (soa_is_block(s, n)) {
        // the host block has the device block's layout: one transfer
        GRT_CUDA(c, cudaMemcpyAsync(c->ph.block.ptr, s->id, 146 * n, cudaMemcpyHostToDevice, c->stream), "H2D photons");
    } else {
        GRT_CUDA(c, cudaMemcpyAsync(c->ph.id.ptr, s->id, n * 8, cudaMemcpyHostToDevice, c->stream), "H2D id");
        for (int q = 0; q < 17; ++q)
            GRT_CUDA(c, cudaMemcpyAsync(c->ph.f[q].ptr, src[q], n * 8, cudaMemcpyHostToDevice, c->stream),
                     "H2D photons");
        GRT_CUDA(c, cudaMemcpyAsync(c->ph.term.ptr, s->terminate, n, cudaMemcpyHostToDevice, c->stream), "H2D term");
        GRT_CUDA(c, cudaMemcpyAsync(c->ph.phase.ptr, s->phase, n, cudaMemcpyHostToDevice, c->stream), "H2D phase");
    }
    if (keep_images && c->batched && c->groups_share && c->geodesics)
        GRT_CUDA(c, cudaMemsetAsync(c->share_state.ptr, 0, c->geodesics * sizeof(unsigned long long), c->stream),
                 "memset share state");
    return count_initial_terminated(c);
}

size_t grt_photon_count(const grt_ctx* c) { return c ? c->n : 0; }

uint64_t grt_geodesic_count(const grt_ctx* c) {
    if (!c) return 0;
    const bool scat = c->p.scattering_enabled && c->fluid_available;
    return c->batched && c->share_channels && c->groups_share && !scat ? c->geodesics : c->n;
}

size_t grt_photon_block_bytes(size_t n) { return 146 * n; }

grt_status grt_host_photon_layout(void* block, size_t n, grt_photon_soa* soa) {
    if (!soa || (!block && n)) return GRT_EINVAL;
    if (reinterpret_cast<uintptr_t>(block) % 8 != 0) return GRT_EINVAL;
    unsigned char* b = static_cast<unsigned char*>(block);
    soa->id = reinterpret_cast<uint64_t*>(b);
    double** d[17] = {&soa->frequency, &soa->emission_frame_energy, &soa->x0, &soa->x1, &soa->x2, &soa->x3,
                      &soa->k0, &soa->k1, &soa->k2, &soa->k3, &soa->I, &soa->Q, &soa->U, &soa->V,
                      &soa->dlambda, &soa->theta_disp, &soa->phi_disp};
    for (int q = 0; q < 17; ++q) *d[q] = reinterpret_cast<double*>(b + photon_field_offset(n, q + 1));
    soa->terminate = b + photon_field_offset(n, 18);
    soa->phase = b + photon_field_offset(n, 19);
    return GRT_OK;
}

grt_status grt_download_photons(grt_ctx* c, grt_photon_soa* s) {
    if (c && c->render_pending) return rendering(c);
    if (!c || !s) return GRT_EINVAL;
    const size_t n = c->n;
    if (n == 0) return GRT_OK;
    double* dst[17];
    soa_doubles(s, dst);
    if (soa_is_block(s, n)) {
        GRT_CUDA(c, cudaMemcpyAsync(s->id, c->ph.block.ptr, 146 * n, cudaMemcpyDeviceToHost, c->stream), "D2H");
        GRT_CUDA(c, cudaStreamSynchronize(c->stream), "sync");
        return GRT_OK;
    }
    if (s->id) GRT_CUDA(c, cudaMemcpyAsync(s->id, c->ph.id.ptr, n * 8, cudaMemcpyDeviceToHost, c->stream), "D2H");
    for (int q = 0; q < 17; ++q)
        if (dst[q]) GRT_CUDA(c, cudaMemcpyAsync(dst[q], c->ph.f[q].ptr, n * 8, cudaMemcpyDeviceToHost, c->stream), "D2H");
    if (s->terminate) GRT_CUDA(c, cudaMemcpyAsync(s->terminate, c->ph.term.ptr, n, cudaMemcpyDeviceToHost, c->stream), "D2H");
    if (s->phase) GRT_CUDA(c, cudaMemcpyAsync(s->phase, c->ph.phase.ptr, n, cudaMemcpyDeviceToHost, c->stream), "D2H");
    GRT_CUDA(c, cudaStreamSynchronize(c->stream), "sync");
    return GRT_OK;
}

}  // extern "C"

namespace {

grt_image_spec spec_from_params(const grt_params& p, uint64_t nx, uint64_t ny) {
    grt_image_spec sp;
    sp.camera_theta = p.camera_theta;
    sp.camera_phi = p.camera_phi;
    sp.camera_distance = p.camera_distance;
    sp.camera_width = p.camera_width;
    sp.camera_height = p.camera_height;
    sp.nx = nx;
    sp.ny = ny;
    sp.custom_frequency_hz = p.custom_frequency_hz;
    sp.absorption_coefficient = p.absorption_coefficient;
    sp.emission_coefficient = p.emission_coefficient;
    return sp;
}

// initialize_photons_image (initialize_photons.hpp:82-170) for every image of
// the context's image set, pixel-centre screen points.
grt_status launch_image_inits(grt_ctx* c) {
    const grt_params& p = c->p;
    // fresh rays: channel 0 leads every shared geodesic and none has finished
    if (c->batched && c->groups_share && c->geodesics)
        GRT_CUDA(c, cudaMemsetAsync(c->share_state.ptr, 0, c->geodesics * sizeof(unsigned long long), c->stream),
                 "memset share state");
    for (size_t k = 0; k < c->images.size(); ++k) {
        const grt_image_spec& sp = c->images[k];
        grt::InitImageArgs a;
        a.ph = c->ph.view();
        a.offset = c->image_start[k];
        a.nx = sp.nx;
        a.ny = sp.ny;
        a.row0 = c->nrows ? c->row0 : 0;
        a.nrows = c->nrows ? c->nrows : sp.ny;
        // ids: image k's pixel (ix, iy) is id_offset + start_k + iy * nx + ix
        a.id_offset = c->image_id_offset + c->image_start[k];
        a.W = sp.camera_width;
        a.H = sp.camera_height;
        // initialize_photons.hpp:94-108, evaluated on the host exactly as there.
        a.cx = sp.camera_distance * std::sin(sp.camera_theta) * std::cos(sp.camera_phi);
        a.cy = sp.camera_distance * std::sin(sp.camera_theta) * std::sin(sp.camera_phi);
        a.cz = sp.camera_distance * std::cos(sp.camera_theta);
        a.th_hat[0] = std::cos(sp.camera_theta) * std::cos(sp.camera_phi);
        a.th_hat[1] = std::cos(sp.camera_theta) * std::sin(sp.camera_phi);
        a.th_hat[2] = -std::sin(sp.camera_theta);
        a.ph_hat[0] = -std::sin(sp.camera_phi);
        a.ph_hat[1] = std::cos(sp.camera_phi);
        a.ph_hat[2] = 0.0;
        a.a = p.spin;
        a.M = p.mass;
        a.dlambda0 = p.initial_step * sp.camera_distance;
        a.forward = c->forward_back > 0.0;
        if (a.forward) {
            const double B = c->forward_back;
            a.bx = -B * std::sin(sp.camera_theta) * std::cos(sp.camera_phi);
            a.by = -B * std::sin(sp.camera_theta) * std::sin(sp.camera_phi);
            a.bz = -B * std::cos(sp.camera_theta);
            a.dlambda0 = p.initial_step * B;
            a.nu0 = sp.custom_frequency_hz;
        }
        // initialize_photons.hpp:115: the random pool is seeded 12345 + rank
        a.random_screen = c->random_screen ? 1 : 0;
        a.seed = 12345ull + static_cast<unsigned long long>(static_cast<long long>(p.rank));
        GRT_CUDA(c, grt::launch_init_image(a, c->stream), "init_image_pixels");
    }
    return GRT_OK;
}

// Appends the queue indices start .. start + nx ny - 1 of one row-major
// nx x ny pixel block in tile order: 8 x 4 tiles, left to right, top to
// bottom, each tile row by row (edge tiles are cut to the block).  A warp
// that claims 32 consecutive queue positions then traces one tile.  Measured
// on C2 (256 x 256, RK45): the trace 3.2% faster than with 32 x 1 row segments
// (4 x 8 and 16 x 2 tiles gained less; ordering by screen radius lost 5%).
void append_tile_order(std::vector<unsigned>& out, unsigned long long start, uint64_t nx, uint64_t ny) {
    constexpr uint64_t kTw = 8, kTh = 4;
    for (uint64_t ty = 0; ty < ny; ty += kTh)
        for (uint64_t tx = 0; tx < nx; tx += kTw)
            for (uint64_t y = ty; y < ty + kTh && y < ny; ++y)
                for (uint64_t x = tx; x < tx + kTw && x < nx; ++x)
                    out.push_back(static_cast<unsigned>(start + y * nx + x));
}

// Builds and uploads the tile orders of the image set just laid out.
grt_status set_tile_orders(grt_ctx* c, const std::vector<unsigned long long>& start,
                           const std::vector<unsigned long long>& qstart, const std::vector<int>& gchan,
                           const std::vector<int>& chan) {
    std::vector<unsigned long long> layout(start.begin(), start.end());
    for (const grt_image_spec& sp : c->images) layout.push_back(sp.nx);
    layout.push_back(~0ull);
    layout.insert(layout.end(), qstart.begin(), qstart.end());
    for (size_t g = 0; g + 1 < qstart.size(); ++g) layout.push_back(c->images[chan[gchan[g]]].nx);
    const bool usable = !c->random_screen && c->n < (1ull << 32);
    if (usable && layout == c->order_layout && c->order_ph_ok && (qstart.empty() || c->order_geo_ok))
        return GRT_OK;  // same layout: the orders on the device still hold
    c->order_ph_ok = c->order_geo_ok = false;
    c->order_layout.clear();
    if (!usable) return GRT_OK;
    std::vector<unsigned> ord;
    ord.reserve(c->n);
    for (size_t k = 0; k + 1 < start.size(); ++k)
        append_tile_order(ord, start[k], c->images[k].nx, (start[k + 1] - start[k]) / c->images[k].nx);
    GRT_CUDA(c, c->order_ph.alloc(ord.size()), "alloc queue order");
    GRT_CUDA(c, cudaMemcpy(c->order_ph.ptr, ord.data(), ord.size() * sizeof(unsigned), cudaMemcpyHostToDevice),
             "H2D queue order");
    c->order_ph_ok = ord.size() == c->n;
    if (!qstart.empty()) {
        ord.clear();
        for (size_t g = 0; g + 1 < qstart.size(); ++g) {
            const grt_image_spec& lead = c->images[chan[gchan[g]]];
            append_tile_order(ord, qstart[g], lead.nx, lead.ny);
        }
        GRT_CUDA(c, c->order_geo.alloc(ord.size()), "alloc queue order");
        GRT_CUDA(c, cudaMemcpy(c->order_geo.ptr, ord.data(), ord.size() * sizeof(unsigned), cudaMemcpyHostToDevice),
                 "H2D queue order");
        c->order_geo_ok = ord.size() == c->geodesics;
    }
    c->order_layout = std::move(layout);
    return GRT_OK;
}

grt_status set_image_set(grt_ctx* c, const grt_image_spec* specs, size_t nimages, uint64_t id_offset, bool batched,
                         double forward_back = 0.0, uint64_t row0 = 0, uint64_t nrows = 0,
                         bool random_screen = false) {
    unsigned long long total = 0;
    std::vector<unsigned long long> start(nimages + 1, 0);
    for (size_t k = 0; k < nimages; ++k) {
        const grt_image_spec& sp = specs[k];
        if (sp.nx == 0 || sp.ny == 0 || sp.nx > (1u << 20) || sp.ny > (1u << 20))
            return fail(c, GRT_EINVAL, "image " + std::to_string(k) + ": nx and ny must be in [1, 2^20]");
        if (!(sp.camera_distance > 0.0) || !(sp.camera_width > 0.0) || !(sp.camera_height > 0.0) ||
            !std::isfinite(sp.camera_theta) || !std::isfinite(sp.camera_phi))
            return fail(c, GRT_EINVAL, "image " + std::to_string(k) +
                                           ": camera distance, width and height must be positive and angles finite");
        start[k] = total;
        total += sp.nx * (nrows ? nrows : sp.ny);
        if (total > (1ull << 40)) return fail(c, GRT_EINVAL, "photon count too large");
    }
    start[nimages] = total;
    GRT_CUDA(c, c->ph.alloc(total), "alloc photons");
    ++c->generation;
    c->n = total;
    c->initial_terminated = 0;
    c->images.assign(specs, specs + nimages);
    c->image_start = start;
    c->image_id_offset = id_offset;
    c->forward_back = forward_back;
    c->random_screen = random_screen;
    c->row0 = row0;
    c->nrows = nrows;
    c->batched = batched;
    c->have_images = true;
    c->bproducts_valid = false;
    c->adj_ready = false;
    if (batched) {
        const grt_params& p = c->p;
        std::vector<grt::KImage> tab(nimages);
        for (size_t k = 0; k < nimages; ++k) {
            const grt_image_spec& sp = specs[k];
            tab[k] = grt::make_kimage(sp.camera_theta, sp.camera_phi, sp.camera_distance, sp.camera_width,
                                      sp.camera_height, sp.custom_frequency_hz, sp.absorption_coefficient,
                                      sp.emission_coefficient);
        }
        (void)p;
        GRT_CUDA(c, c->images_dev.alloc(nimages), "alloc image table");
        GRT_CUDA(c, c->image_start_dev.alloc(nimages + 1), "alloc image table");
        GRT_CUDA(c, cudaMemcpy(c->images_dev.ptr, tab.data(), nimages * sizeof(grt::KImage), cudaMemcpyHostToDevice),
                 "H2D image table");
        GRT_CUDA(c, cudaMemcpy(c->image_start_dev.ptr, start.data(), (nimages + 1) * sizeof(unsigned long long),
                               cudaMemcpyHostToDevice), "H2D image table");
        // channel groups: same camera plane and screen (exact parameter equality)
        std::vector<std::vector<int>> groups;
        for (size_t k = 0; k < nimages; ++k) {
            const grt_image_spec& a = specs[k];
            bool placed = false;
            for (auto& g : groups) {
                const grt_image_spec& b = specs[g[0]];
                if (a.camera_theta == b.camera_theta && a.camera_phi == b.camera_phi &&
                    a.camera_distance == b.camera_distance && a.camera_width == b.camera_width &&
                    a.camera_height == b.camera_height && a.nx == b.nx && a.ny == b.ny && g.size() < 32) {
                    g.push_back(static_cast<int>(k));
                    placed = true;
                    break;
                }
            }
            if (!placed) groups.push_back({static_cast<int>(k)});
        }
        std::vector<unsigned long long> qstart(groups.size() + 1, 0);
        std::vector<int> gchan(groups.size() + 1, 0), chan;
        c->groups_share = false;
        for (size_t g = 0; g < groups.size(); ++g) {
            qstart[g + 1] = qstart[g] + specs[groups[g][0]].nx * specs[groups[g][0]].ny;
            gchan[g + 1] = gchan[g] + static_cast<int>(groups[g].size());
            chan.insert(chan.end(), groups[g].begin(), groups[g].end());
            if (groups[g].size() > 1) c->groups_share = true;
        }
        c->ngroups = static_cast<int>(groups.size());
        c->geodesics = qstart.back();
        if (c->groups_share) GRT_CUDA(c, c->share_state.alloc(c->geodesics), "alloc share state");
        GRT_CUDA(c, c->group_qstart_dev.alloc(qstart.size()), "alloc groups");
        GRT_CUDA(c, c->group_chan_dev.alloc(gchan.size()), "alloc groups");
        GRT_CUDA(c, c->chan_img_dev.alloc(chan.size()), "alloc groups");
        GRT_CUDA(c, cudaMemcpy(c->group_qstart_dev.ptr, qstart.data(), qstart.size() * sizeof(unsigned long long),
                               cudaMemcpyHostToDevice), "H2D groups");
        GRT_CUDA(c, cudaMemcpy(c->group_chan_dev.ptr, gchan.data(), gchan.size() * sizeof(int), cudaMemcpyHostToDevice),
                 "H2D groups");
        GRT_CUDA(c, cudaMemcpy(c->chan_img_dev.ptr, chan.data(), chan.size() * sizeof(int), cudaMemcpyHostToDevice),
                 "H2D groups");
        const grt_status os = set_tile_orders(c, start, qstart, gchan, chan);
        if (os != GRT_OK) return os;
    } else {
        c->ngroups = 0;
        c->groups_share = false;
        const grt_status os = set_tile_orders(c, start, {}, {}, {});
        if (os != GRT_OK) return os;
    }
    return launch_image_inits(c);
}

// Launch-wide part of a build_observation_products (observation.hpp:31-84) launch.
grt::ProductsSet products_set(grt_ctx* c) {
    const grt_params& p = c->p;
    grt::ProductsSet set;
    std::memset(&set, 0, sizeof(set));
    set.ph = c->ph.view();
    set.bins = p.spectrum_bins;
    set.spec_min = p.spectrum_min_hz;
    set.spec_max = p.spectrum_max_hz;
    set.log_min = std::log10(p.spectrum_min_hz);
    set.log_max = std::log10(p.spectrum_max_hz);
    return set;
}

grt::ProductsImage products_image(unsigned long long offset, unsigned long long n, uint64_t nx, uint64_t ny, double W,
                                  double H, double* image, double* spectrum, unsigned long long* arrived) {
    grt::ProductsImage im;
    std::memset(&im, 0, sizeof(im));
    im.offset = offset;
    im.n = n;
    im.nx = nx;
    im.ny = ny;
    im.W = W;
    im.H = H;
    im.image = image;
    im.spectrum = spectrum;
    im.arrived = arrived;
    return im;
}

// Products of photon slots [offset, offset + n) as one image into device buffers.
grt_status launch_products(grt_ctx* c, unsigned long long offset, unsigned long long n, uint64_t nx, uint64_t ny,
                           double W, double H, double* image, double* spectrum, unsigned long long* arrived) {
    const size_t npix = nx * ny, bins = c->p.spectrum_bins;
    GRT_CUDA(c, cudaMemsetAsync(image, 0, 4 * npix * sizeof(double), c->stream), "memset");
    if (bins) GRT_CUDA(c, cudaMemsetAsync(spectrum, 0, bins * sizeof(double), c->stream), "memset");
    GRT_CUDA(c, cudaMemsetAsync(arrived, 0, sizeof(unsigned long long), c->stream), "memset");
    grt::ProductsSet set = products_set(c);
    set.nimages = 1;
    set.img[0] = products_image(offset, n, nx, ny, W, H, image, spectrum, arrived);
    GRT_CUDA(c, grt::launch_image_products(set, c->stream), "image_products");
    return GRT_OK;
}

// Products of every image of the image set into the per-image device buffers
// (contiguous, so three memsets clear them all), kProductsMaxImages images
// per launch.
grt_status launch_all_products(grt_ctx* c) {
    const size_t nimg = c->images.size(), bins = c->p.spectrum_bins;
    c->bimage_off.assign(nimg + 1, 0);
    for (size_t k = 0; k < nimg; ++k) c->bimage_off[k + 1] = c->bimage_off[k] + 4 * c->images[k].nx * c->images[k].ny;
    GRT_CUDA(c, c->bimage.alloc(c->bimage_off[nimg]), "alloc products");
    GRT_CUDA(c, c->bspectrum.alloc(nimg * bins), "alloc products");
    GRT_CUDA(c, c->barrived.alloc(nimg), "alloc products");
    if (nimg == 0) return GRT_OK;
    GRT_CUDA(c, cudaMemsetAsync(c->bimage.ptr, 0, c->bimage_off[nimg] * sizeof(double), c->stream), "memset");
    if (bins) GRT_CUDA(c, cudaMemsetAsync(c->bspectrum.ptr, 0, nimg * bins * sizeof(double), c->stream), "memset");
    GRT_CUDA(c, cudaMemsetAsync(c->barrived.ptr, 0, nimg * sizeof(unsigned long long), c->stream), "memset");
    for (size_t k0 = 0; k0 < nimg; k0 += grt::kProductsMaxImages) {
        grt::ProductsSet set = products_set(c);
        const size_t k1 = std::min(nimg, k0 + static_cast<size_t>(grt::kProductsMaxImages));
        for (size_t k = k0; k < k1; ++k) {
            const grt_image_spec& sp = c->images[k];
            set.img[k - k0] = products_image(c->image_start[k], c->image_start[k + 1] - c->image_start[k], sp.nx,
                                             sp.ny, sp.camera_width, sp.camera_height,
                                             c->bimage.ptr + c->bimage_off[k], c->bspectrum.ptr + k * bins,
                                             c->barrived.ptr + k);
        }
        set.nimages = static_cast<int>(k1 - k0);
        GRT_CUDA(c, grt::launch_image_products(set, c->stream), "image_products");
    }
    return GRT_OK;
}

// observation.hpp:51-58, on the host like the reference.
void fill_spectrum_frequencies(const grt_params& p, double* out) {
    const size_t bins = p.spectrum_bins;
    const double log_min = std::log10(p.spectrum_min_hz), log_max = std::log10(p.spectrum_max_hz);
    for (size_t b = 0; b < bins; ++b) {
        const double f = bins > 1 ? static_cast<double>(b) / static_cast<double>(bins - 1) : 0.0;
        out[b] = std::pow(10.0, log_min + f * (log_max - log_min));
    }
}

// Per-warp loop limit of a trace launch (GRT_ETIMEOUT beyond it): the launch
// shape's max_iterations
// when set, else a bound no launch that makes progress reaches: every photon
// may take `budget` calls of at most 13 attempts each, and every warp
// iteration is one RK45 attempt or RK4 step of at least one lane.
unsigned long long iteration_limit(const grt_ctx* c, const grt::KParams& kp, unsigned long long total, int blocks,
                                   int threads) {
    if (c->lc.max_iterations > 0) return static_cast<unsigned long long>(c->lc.max_iterations);
    const unsigned long long warps = static_cast<unsigned long long>(blocks) * (threads / 32);
    return static_cast<unsigned long long>(kp.budget + 2) * 13ull *
               ((total + warps - 1) / warps + static_cast<unsigned long long>(kp.grab)) +
           (1ull << 20);
}

// Image-mode rays are traced by the backward-leg launch, the packet generation
// at first fluid contact and the launch over the rest (trace_body LEG 1 and
// 2), unless the launch shape asks for one launch over whole rays.
bool split_legs(const grt_ctx* c) { return c->lc.split_legs != 0 && c->p.mode == GRT_MODE_IMAGE; }

// Device buffers a trace needs besides the photons; allocated before any
// launch or graph capture.
grt_status prepare_trace_buffers(grt_ctx* c, unsigned long long queue) {
    if (split_legs(c)) GRT_CUDA(c, c->calls_carry.alloc(queue), "alloc call carry");
    return GRT_OK;
}

// The trace of one chunk of the step loop: one launch over whole rays, or the
// backward-leg launch, the packet generation of the rays it stopped at their
// first fluid contact, and, with the queue head reset, the forward-leg launch
// over the same queue.
// Resident trace blocks per SM: the launch shape's, or with 0 (automatic)
// the fewest of 2, 3, 4 that keep every geodesic of the queue resident at
// once -- fewer blocks give each thread more registers (255, 170, 128) and
// spill less, and a workload that fits needs no more lanes.
int trace_blocks_per_sm(const grt_ctx* c, unsigned long long queue) {
    if (c->lc.blocks_per_sm) return c->lc.blocks_per_sm;
    for (int b = 2; b < 4; ++b)
        if (static_cast<unsigned long long>(c->sm_count) * b * 128 >= queue) return b;
    return 4;
}

// When every queue claim of a launch fits in its resident warps (C1, C2: no
// warp ever refills from the queue), the first claims are balanced over the
// SMs: at most ceil(claims / SMs) per SM (KParams::sm_quota).  Each launch
// zeroes the counters first, as a node of the render graph too.
cudaError_t launch_trace(const grt_ctx* c, const grt::KParams& kp_in, size_t smem) {
    const int bps = trace_blocks_per_sm(c, kp_in.n);
    grt::KParams kp = kp_in;
    const unsigned long long warps = static_cast<unsigned long long>(c->sm_count) * bps * 4;
    const unsigned long long claims = kp.grab > 0 ? (kp.n + kp.grab - 1) / kp.grab : 0;
    if (c->sm_claims.ptr && claims > 0 && claims <= warps) {
        kp.sm_claims = c->sm_claims.ptr;
        kp.sm_quota = static_cast<unsigned>((claims + c->sm_count - 1) / c->sm_count);
        const cudaError_t e0 =
            cudaMemsetAsync(kp.sm_claims, 0, grt::kSmClaimSlots * sizeof(unsigned), c->stream);
        if (e0 != cudaSuccess) return e0;
    }
    const grt_params& p = c->p;
    const bool mixed = p.precision != GRT_PREC_FP64;
    if (!split_legs(c)) {
        // disk mode: the whole-ray kernel without the image-mode code (leg 3)
        const int leg = p.mode == GRT_MODE_DISK && kp.ngroups == 0 ? 3 : 0;
        return grt::launch_trace(kp, mixed, leg, p.integrator, c->sm_count, bps, smem, c->stream);
    }
    cudaError_t e = cudaMemsetAsync(kp.calls_carry, 0, kp.n * sizeof(long long), c->stream);
    if (e == cudaSuccess)
        e = grt::launch_trace(kp, mixed, 1, p.integrator, c->sm_count, bps, smem, c->stream);
    if (e == cudaSuccess)
        e = grt::launch_generate_pending(
            kp, c->sm_count,
            grt::dev_trace_smem_bytes(0, 128, c->fluid_available && c->separable, c->nr, c->nth, c->nph), c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(&kp.counters->queue_head, 0, sizeof(unsigned long long), c->stream);
    if (e == cudaSuccess && kp.sm_quota)
        e = cudaMemsetAsync(kp.sm_claims, 0, grt::kSmClaimSlots * sizeof(unsigned), c->stream);
    if (e == cudaSuccess)
        e = grt::launch_trace(kp, mixed, 2, p.integrator, c->sm_count, bps, smem, c->stream);
    return e;
}

size_t trace_smem(const grt_ctx* c) {
    return grt::dev_trace_smem_bytes(c->p.integrator, 128, c->fluid_available && c->separable, c->nr, c->nth, c->nph);
}

// steps_done of a single-launch run (termination_percent = 1): the reference
// stops after the first output step at or after the last termination.
int64_t single_launch_steps_done(const grt_params& p, unsigned long long terminated, unsigned long long total,
                                 unsigned long long max_term_step) {
    if (terminated < total) return p.max_steps;
    const uint64_t interval = p.output_interval ? p.output_interval : 1;
    const int64_t last = max_term_step ? static_cast<int64_t>(max_term_step) - 1 : 0;
    int64_t s_out = static_cast<int64_t>(((static_cast<uint64_t>(last) + interval - 1) / interval) * interval);
    if (s_out > p.max_steps - 1) s_out = p.max_steps - 1;
    return s_out + 1;
}

}  // namespace

extern "C" {

grt_status grt_init_image_photons(grt_ctx* c, uint64_t nx, uint64_t ny, uint64_t id_offset) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    const grt_image_spec sp = spec_from_params(c->p, nx, ny);
    if (nx * ny == 0) {
        GRT_CUDA(c, c->ph.alloc(0), "alloc photons");
        c->n = 0;
        c->images.clear();
        c->image_start.clear();
        c->batched = false;
        c->have_images = false;
        ++c->generation;
        return GRT_OK;
    }
    return set_image_set(c, &sp, 1, id_offset, false);
}

grt_status grt_init_image_photons_random(grt_ctx* c, uint64_t n, uint64_t id_offset) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    if (n == 0) return grt_init_image_photons(c, 0, 0, id_offset);
    // one row of n rays: the slot layout only; products bin by arrival (u, v)
    // into output.image_nx x image_ny
    const grt_image_spec sp = spec_from_params(c->p, n, 1);
    return set_image_set(c, &sp, 1, id_offset, false, 0.0, 0, 0, true);
}

grt_status grt_init_image_rows(grt_ctx* c, uint64_t nx, uint64_t ny, uint64_t row0, uint64_t nrows,
                               uint64_t id_offset) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    if (nx == 0 || ny == 0 || nrows == 0 || row0 >= ny || nrows > ny - row0)
        return fail(c, GRT_EINVAL, "rows [row0, row0 + nrows) must lie inside the ny-row screen");
    const grt_image_spec sp = spec_from_params(c->p, nx, ny);
    return set_image_set(c, &sp, 1, id_offset, false, 0.0, row0, nrows);
}

grt_status grt_init_image_forward_photons(grt_ctx* c, uint64_t nx, uint64_t ny, double back_distance,
                                          uint64_t id_offset) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    if (!(back_distance > 0.0) || !std::isfinite(back_distance))
        return fail(c, GRT_EINVAL, "back_distance must be positive");
    if (nx * ny == 0) return fail(c, GRT_EINVAL, "nx and ny must be positive");
    const grt_image_spec sp = spec_from_params(c->p, nx, ny);
    return set_image_set(c, &sp, 1, id_offset, false, back_distance);
}

grt_status grt_init_disk_photons(grt_ctx* c, uint64_t id_offset, uint64_t* n_photons) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    if (!c->grid_uploaded || !c->fluid_available)
        return fail(c, GRT_ESTATE, "disk emission needs an uploaded fluid grid");
    const grt_params& p = c->p;
    const size_t ncell = c->host_rho.size();
    // build_superphoton_cell_offsets (initialize_photons.hpp:32-64), on the host like the reference
    std::vector<unsigned long long> off(ncell + 1);
    unsigned long long total = 0;
    for (size_t q = 0; q < ncell; ++q) {
        off[q] = total;
        const int count = grt::ComputeSuperphotonsPerCell(c->host_rho[q], p.superphoton_count_normalization);
        total += static_cast<unsigned long long>(count > 0 ? count : 0);
    }
    off[ncell] = total;
    if (total > (1ull << 36)) return fail(c, GRT_EINVAL, "disk packet count too large: " + std::to_string(total));
    GRT_CUDA(c, c->ph.alloc(total), "alloc photons");
    GRT_CUDA(c, c->disk_offsets.alloc(ncell + 1), "alloc offsets");
    GRT_CUDA(c, cudaMemcpy(c->disk_offsets.ptr, off.data(), (ncell + 1) * sizeof(unsigned long long),
                           cudaMemcpyHostToDevice), "H2D offsets");
    ++c->generation;
    c->n = total;
    c->images.clear();
    c->image_start.clear();
    c->batched = false;
    c->have_images = false;
    c->bproducts_valid = false;
    c->adj_ready = false;
    grt::DiskInitArgs a{};
    a.ph = c->ph.view();
    a.n = total;
    a.offsets = c->disk_offsets.ptr;
    a.ncell = ncell;
    a.pos = c->cell_pos.ptr;
    a.rho_t = c->rho_t.ptr;
    a.vel = c->vel.ptr;
    a.mag = c->mag.ptr;
    a.density_scale = p.density_g_cm3_per_code;
    a.temperature_scale = p.temperature_k_per_code;
    a.length_scale = p.length_cm_per_code;
    a.time_scale = p.time_s_per_code;
    a.a = p.spin;
    a.M = p.mass;
    a.generator = p.generator;
    a.energy = p.energy_per_cell_erg;
    a.pl_slope = p.power_law_slope;
    a.nu_min = p.nu_min_hz;
    a.nu_max = p.nu_max_hz;
    a.nu_custom = p.custom_frequency_hz;
    a.seed = p.scattering_seed + static_cast<uint64_t>(p.rank);
    a.id_offset = id_offset;
    a.dlambda0 = p.initial_step;
    GRT_CUDA(c, grt::launch_init_disk(a, c->stream), "init_disk_photons");
    c->initial_terminated = 0;
    if (total > 0) {
        grt_status st = count_initial_terminated(c);
        if (st != GRT_OK) return st;
    }
    if (n_photons) *n_photons = total;
    return GRT_OK;
}

grt_status grt_init_image_batch(grt_ctx* c, const grt_image_spec* specs, size_t nimages, uint64_t id_offset) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    if (!specs || nimages == 0) return fail(c, GRT_EINVAL, "an image batch needs at least one image");
    if (nimages > (1u << 20)) return fail(c, GRT_EINVAL, "too many images in one batch");
    return set_image_set(c, specs, nimages, id_offset, true);
}

size_t grt_batch_image_count(const grt_ctx* c) { return c && c->batched ? c->images.size() : 0; }

grt_status grt_set_channel_sharing(grt_ctx* c, int enable) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    c->share_channels = enable != 0;
    ++c->generation;
    return GRT_OK;
}

static bool products_complete(const grt_image_products* out) {
    return out->image_I && out->image_Q && out->image_U && out->image_V && out->spectrum_frequency_hz &&
           out->spectrum_I && out->arrived_count;
}

// Copies of image k's products into *out on stream st (the caller synchronises).
static grt_status enqueue_batch_products(grt_ctx* c, size_t image, grt_image_products* out, cudaStream_t st) {
    if (!products_complete(out)) return fail(c, GRT_EINVAL, "null image product buffer");
    const grt_image_spec& sp = c->images[image];
    const size_t npix = sp.nx * sp.ny, bins = c->p.spectrum_bins;
    const double* src = c->bimage.ptr + c->bimage_off[image];
    double* dst[4] = {out->image_I, out->image_Q, out->image_U, out->image_V};
    for (int q = 0; q < 4; ++q)
        GRT_CUDA(c, cudaMemcpyAsync(dst[q], src + q * npix, npix * sizeof(double), cudaMemcpyDeviceToHost, st),
                 "D2H image");
    GRT_CUDA(c, cudaMemcpyAsync(out->spectrum_I, c->bspectrum.ptr + image * bins, bins * sizeof(double),
                                cudaMemcpyDeviceToHost, st), "D2H spectrum");
    GRT_CUDA(c, cudaMemcpyAsync(out->arrived_count, c->barrived.ptr + image, sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, st), "D2H arrived");
    fill_spectrum_frequencies(c->p, out->spectrum_frequency_hz);
    return GRT_OK;
}

static grt_status ensure_batch_products(grt_ctx* c) {
    if (!c->batched) return fail(c, GRT_ESTATE, "no image batch (grt_init_image_batch)");
    if (!c->bproducts_valid) {
        grt_status st = launch_all_products(c);
        if (st != GRT_OK) return st;
        c->bproducts_valid = true;
    }
    return GRT_OK;
}

grt_status grt_get_batch_image_products(grt_ctx* c, size_t image, grt_image_products* out) {
    if (c && c->render_pending) return rendering(c);
    if (!c || !out) return GRT_EINVAL;
    grt_status st = ensure_batch_products(c);
    if (st != GRT_OK) return st;
    if (image >= c->images.size()) return fail(c, GRT_EINVAL, "image index out of range");
    st = enqueue_batch_products(c, image, out, c->stream);
    if (st != GRT_OK) return st;
    GRT_CUDA(c, cudaStreamSynchronize(c->stream), "products");
    return GRT_OK;
}

size_t grt_products_block_bytes(const grt_ctx* c) {
    if (!c || !c->have_images) return 0;
    size_t values = c->images.size() * (c->p.spectrum_bins + 1);
    for (const grt_image_spec& sp : c->images) values += 4 * sp.nx * sp.ny;
    return values * sizeof(double);
}

grt_status grt_copy_products_block(grt_ctx* c, void* dst, size_t bytes) {
    if (c && c->render_pending) return rendering(c);
    if (!c || !dst) return GRT_EINVAL;
    if (!c->have_images) return fail(c, GRT_ESTATE, "no image set (grt_init_image_photons or grt_init_image_batch)");
    if (bytes < grt_products_block_bytes(c)) return fail(c, GRT_EINVAL, "dst is smaller than grt_products_block_bytes");
    if (!c->bproducts_valid) {
        grt_status st = launch_all_products(c);
        if (st != GRT_OK) return st;
        c->bproducts_valid = true;
    }
    const size_t nimg = c->images.size(), bins = c->p.spectrum_bins;
    char* d = static_cast<char*>(dst);
    const size_t img_bytes = c->bimage_off[nimg] * sizeof(double), spec_bytes = nimg * bins * sizeof(double);
    GRT_CUDA(c, cudaMemcpyAsync(d, c->bimage.ptr, img_bytes, cudaMemcpyDefault, c->stream), "copy products");
    if (spec_bytes)
        GRT_CUDA(c, cudaMemcpyAsync(d + img_bytes, c->bspectrum.ptr, spec_bytes, cudaMemcpyDefault, c->stream),
                 "copy products");
    GRT_CUDA(c, cudaMemcpyAsync(d + img_bytes + spec_bytes, c->barrived.ptr, nimg * sizeof(unsigned long long),
                                cudaMemcpyDefault, c->stream), "copy products");
    return GRT_OK;
}

grt_status grt_get_all_batch_image_products(grt_ctx* c, grt_image_products* outs, size_t nimages) {
    if (c && c->render_pending) return rendering(c);
    if (!c || (!outs && nimages)) return GRT_EINVAL;
    grt_status st = ensure_batch_products(c);
    if (st != GRT_OK) return st;
    if (nimages != c->images.size()) return fail(c, GRT_EINVAL, "nimages must equal the batch's image count");
    for (size_t k = 0; k < nimages; ++k) {
        st = enqueue_batch_products(c, k, outs + k, c->stream);
        if (st != GRT_OK) return st;
    }
    GRT_CUDA(c, cudaStreamSynchronize(c->stream), "products");
    return GRT_OK;
}

}  // extern "C"

namespace {

// Where run_steps writes output-step archives (nullptr: none).
struct OutputPlan {
    std::string dir, name;
    std::vector<int> fields;
    uint64_t stride;
    int32_t rank;
};

grt_status write_output_step(grt_ctx* c, const OutputPlan& plan, int64_t step);

// The step loop of integrate_geodesics (integrate_cart_ks.hpp:468-527).
// Without output and with termination_percent = 1 one launch covers it; else
// launches end on the output steps, where the terminated fraction is checked
// (and, with a plan, an archive written).
grt_status run_steps(grt_ctx* c, grt_run_stats* stats, const OutputPlan* plan) {
    if (!c->grid_uploaded) return fail(c, GRT_ESTATE, "grt_run before grt_upload_grid");
    const grt_params& p = c->p;
    grt_run_stats st;
    std::memset(&st, 0, sizeof(st));
    c->bproducts_valid = false;
    c->adj_ready = false;
    if (c->n == 0) {
        st.steps_done = p.max_steps;
        if (stats) *stats = st;
        return GRT_OK;
    }
    grt::KParams kp = make_kparams(c);
    {
        const grt_status bs = prepare_trace_buffers(c, kp.n);
        if (bs != GRT_OK) return bs;
        kp.calls_carry = c->calls_carry.ptr;
    }
    const int threads = 128;
    const size_t smem = trace_smem(c);
    const int blocks = c->sm_count * trace_blocks_per_sm(c, kp.n);
    const unsigned long long total = c->n;
    unsigned long long terminated = c->initial_terminated;
    const uint64_t interval = p.output_interval ? p.output_interval : 1;
    // Chunks end on the reference's output steps (step % interval == 0 or the
    // last step), where it evaluates the termination fraction
    // (integrate_cart_ks.hpp:491-526).  With termination_percent = 1 the check
    // can only succeed once every photon has terminated, so one launch covers
    // the whole loop.
    const bool single = p.termination_percent >= 1.0 && !plan;
    int64_t step = 0;
    int64_t steps_done = 0;
    unsigned long long max_term_step = 0;
    float ms_total = 0.0f;
    while (step < p.max_steps) {
        int64_t end;
        if (single) {
            end = p.max_steps;
        } else {
            // next output step at or after `step`
            int64_t next = static_cast<int64_t>(((static_cast<uint64_t>(step) + interval - 1) / interval) * interval);
            if (next > p.max_steps - 1) next = p.max_steps - 1;
            end = next + 1;
        }
        kp.step0 = step;
        kp.budget = end - step;
        kp.max_iterations = iteration_limit(c, kp, total, blocks, threads);
        GRT_CUDA(c, cudaMemsetAsync(c->counters.ptr, 0, sizeof(grt::KCounters), c->stream), "memset counters");
        GRT_CUDA(c, cudaEventRecord(c->ev0, c->stream), "event");
        cudaError_t e = launch_trace(c, kp, smem);
        if (e != cudaSuccess) return cuda_fail(c, e, "trace launch");
        GRT_CUDA(c, cudaEventRecord(c->ev1, c->stream), "event");
        GRT_CUDA(c, cudaMemcpyAsync(c->host_counters, c->counters.ptr, sizeof(grt::KCounters), cudaMemcpyDeviceToHost,
                                    c->stream), "D2H counters");
        GRT_CUDA(c, cudaStreamSynchronize(c->stream), "trace kernel");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        ms_total += ms;
        const grt::KCounters& k = *c->host_counters;
        terminated += k.terminated;
        st.accepted_steps += k.accepted;
        st.rejected_attempts += k.rejected;
        st.photon_calls += k.calls;
        st.launches += split_legs(c) ? 3 : 1;
        if (k.max_term_step > max_term_step) max_term_step = k.max_term_step;
        if (k.timed_out) {
            st.timed_out = 1;
            st.steps_done = steps_done;
            st.trace_ms = ms_total;
            st.n_terminated = terminated;
            c->initial_terminated = terminated;  // a later run continues these photons
            if (stats) *stats = st;
            return fail(c, GRT_ETIMEOUT, "trace kernel hit its iteration limit");
        }
        step = end;
        steps_done = end;
        if (plan) {
            const grt_status ws = write_output_step(c, *plan, end - 1);
            if (ws != GRT_OK) return ws;
        }
        const double fraction = static_cast<double>(terminated) / static_cast<double>(total);
        if (fraction >= p.termination_percent) break;
    }
    if (single && terminated >= total) steps_done = single_launch_steps_done(p, terminated, total, max_term_step);
    st.steps_done = steps_done;
    st.n_terminated = terminated;
    st.trace_ms = ms_total;
    c->initial_terminated = terminated;
    if (stats) *stats = st;
    return GRT_OK;
}

}  // namespace

extern "C" {

grt_status grt_run(grt_ctx* c, grt_run_stats* stats) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    return run_steps(c, stats, nullptr);
}

grt_status grt_render_graph(grt_ctx* c, grt_run_stats* stats) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    if (!c->grid_uploaded) return fail(c, GRT_ESTATE, "grt_render_graph before grt_upload_grid");
    if (!c->have_images) return fail(c, GRT_ESTATE, "grt_render_graph needs grt_init_image_photons or grt_init_image_batch");
    const grt_params& p = c->p;
    if (!(p.termination_percent >= 1.0))
        return fail(c, GRT_EINVAL, "grt_render_graph needs termination_percent >= 1 (one trace launch)");
    if (!c->graph_exec || c->graph_generation != c->generation) {
        if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
        if (c->graph) cudaGraphDestroy(c->graph);
        c->graph_exec = nullptr;
        c->graph = nullptr;
        // allocations happen before the capture
        const size_t nimg = c->images.size(), bins = p.spectrum_bins;
        size_t pix = 0;
        for (const auto& sp : c->images) pix += 4 * sp.nx * sp.ny;
        GRT_CUDA(c, c->bimage.alloc(pix), "alloc products");
        GRT_CUDA(c, c->bspectrum.alloc(nimg * bins), "alloc products");
        GRT_CUDA(c, c->barrived.alloc(nimg), "alloc products");
        grt::KParams kp = make_kparams(c);
        {
            const grt_status bs = prepare_trace_buffers(c, kp.n);
            if (bs != GRT_OK) return bs;
            kp.calls_carry = c->calls_carry.ptr;
        }
        kp.step0 = 0;
        kp.budget = p.max_steps;
        kp.max_iterations = iteration_limit(c, kp, c->n, c->sm_count * trace_blocks_per_sm(c, kp.n), 128);
        const size_t smem = trace_smem(c);
        GRT_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed), "begin capture");
        grt_status gs = launch_image_inits(c);
        cudaError_t e = cudaSuccess;
        if (gs == GRT_OK) e = cudaMemsetAsync(c->counters.ptr, 0, sizeof(grt::KCounters), c->stream);
        // event-record nodes around the trace kernel time it inside the graph
        if (gs == GRT_OK && e == cudaSuccess) e = cudaEventRecordWithFlags(c->ev0, c->stream, cudaEventRecordExternal);
        if (gs == GRT_OK && e == cudaSuccess) e = launch_trace(c, kp, smem);
        if (gs == GRT_OK && e == cudaSuccess) e = cudaEventRecordWithFlags(c->ev1, c->stream, cudaEventRecordExternal);
        if (gs == GRT_OK && e == cudaSuccess) gs = launch_all_products(c);
        if (gs == GRT_OK && e == cudaSuccess)
            e = cudaMemcpyAsync(c->host_counters, c->counters.ptr, sizeof(grt::KCounters), cudaMemcpyDeviceToHost,
                                c->stream);
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(c->stream, &g);
        if (gs != GRT_OK) {
            if (g) cudaGraphDestroy(g);
            return gs;
        }
        if (e != cudaSuccess || ee != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return cuda_fail(c, e != cudaSuccess ? e : ee, "render graph capture");
        }
        c->graph = g;
        GRT_CUDA(c, cudaGraphInstantiate(&c->graph_exec, c->graph, 0), "graph instantiate");
        c->graph_generation = c->generation;
    }
    GRT_CUDA(c, cudaGraphLaunch(c->graph_exec, c->stream), "graph launch");
    GRT_CUDA(c, cudaStreamSynchronize(c->stream), "render graph");
    c->initial_terminated = 0;
    c->bproducts_valid = true;
    c->adj_ready = false;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    const grt::KCounters& k = *c->host_counters;
    grt_run_stats st;
    std::memset(&st, 0, sizeof(st));
    st.accepted_steps = k.accepted;
    st.rejected_attempts = k.rejected;
    st.photon_calls = k.calls;
    st.launches = split_legs(c) ? 3 : 1;
    st.n_terminated = k.terminated;
    st.trace_ms = ms;
    st.steps_done = single_launch_steps_done(p, k.terminated, c->n, k.max_term_step);
    if (k.timed_out) {
        st.timed_out = 1;
        if (stats) *stats = st;
        return fail(c, GRT_ETIMEOUT, "trace kernel hit its iteration limit");
    }
    if (stats) *stats = st;
    return GRT_OK;
}

// Enqueue one render of uploaded photons: the host photon block goes up on
// copy_stream; the trace launches and every image's products follow on stream
// once it has landed; the products go back on copy_stream once they are
// built.  Nothing synchronises here.
static grt_status enqueue_render(grt_ctx* c, const grt_photon_soa* s, grt_image_products* outs) {
    const size_t n = c->n, nimg = c->images.size();
    grt::KParams kp = make_kparams(c);
    kp.calls_carry = c->calls_carry.ptr;
    kp.step0 = 0;
    kp.budget = c->p.max_steps;
    kp.max_iterations = iteration_limit(c, kp, n, c->sm_count * trace_blocks_per_sm(c, kp.n), 128);
    GRT_CUDA(c, cudaMemcpyAsync(c->ph.block.ptr, s->id, grt_photon_block_bytes(n), cudaMemcpyHostToDevice,
                                c->copy_stream), "H2D photons");
    GRT_CUDA(c, cudaEventRecord(c->ev_uploaded, c->copy_stream), "event");
    GRT_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_uploaded, 0), "stream wait");
    if (c->groups_share && c->geodesics)
        GRT_CUDA(c, cudaMemsetAsync(c->share_state.ptr, 0, c->geodesics * sizeof(unsigned long long), c->stream),
                 "memset share state");
    // photons terminated before the trace count toward the stop rule
    GRT_CUDA(c, cudaMemsetAsync(c->scratch_u64.ptr + 1, 0, sizeof(unsigned long long), c->stream), "memset");
    GRT_CUDA(c, grt::launch_count_terminated(c->ph.term.ptr, n, c->scratch_u64.ptr + 1, c->sm_count, c->stream),
             "count_terminated");
    GRT_CUDA(c, cudaMemsetAsync(c->counters.ptr, 0, sizeof(grt::KCounters), c->stream), "memset counters");
    GRT_CUDA(c, cudaEventRecord(c->ev0, c->stream), "event");
    const cudaError_t e = launch_trace(c, kp, trace_smem(c));
    if (e != cudaSuccess) return cuda_fail(c, e, "trace launch");
    GRT_CUDA(c, cudaEventRecord(c->ev1, c->stream), "event");
    grt_status st = launch_all_products(c);
    if (st != GRT_OK) return st;
    GRT_CUDA(c, cudaMemcpyAsync(c->host_counters, c->counters.ptr, sizeof(grt::KCounters), cudaMemcpyDeviceToHost,
                                c->stream), "D2H counters");
    GRT_CUDA(c, cudaMemcpyAsync(c->host_u64 + 1, c->scratch_u64.ptr + 1, sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, c->stream), "D2H count");
    GRT_CUDA(c, cudaEventRecord(c->ev_traced, c->stream), "event");
    GRT_CUDA(c, cudaStreamWaitEvent(c->copy_stream, c->ev_traced, 0), "stream wait");
    for (size_t k = 0; k < nimg; ++k) {
        st = enqueue_batch_products(c, k, outs + k, c->copy_stream);
        if (st != GRT_OK) return st;
    }
    GRT_CUDA(c, cudaEventRecord(c->ev_done, c->copy_stream), "event");
    return GRT_OK;
}

grt_status grt_render_async(grt_ctx* c, const grt_photon_soa* s, grt_image_products* outs, size_t nimages) {
    if (!c || !s || (!outs && nimages)) return GRT_EINVAL;
    if (c->render_pending) return fail(c, GRT_ESTATE, "a render is in flight on this context (grt_render_wait)");
    if (!c->grid_uploaded) return fail(c, GRT_ESTATE, "grt_render_async before grt_upload_grid");
    if (!c->batched || !c->have_images || c->n == 0)
        return fail(c, GRT_ESTATE, "grt_render_async needs an image batch (grt_init_image_batch)");
    const grt_params& p = c->p;
    if (!(p.termination_percent >= 1.0))
        return fail(c, GRT_EINVAL, "grt_render_async needs termination_percent >= 1 (one trace launch)");
    if (nimages != c->images.size()) return fail(c, GRT_EINVAL, "nimages must equal the batch's image count");
    if (!soa_is_block(s, c->n))
        return fail(c, GRT_EINVAL,
                    "grt_render_async takes the batch's photons as one host block (grt_host_photon_layout, "
                    "grt_photon_count photons)");
    for (size_t k = 0; k < nimages; ++k)
        if (!products_complete(outs + k)) return fail(c, GRT_EINVAL, "null image product buffer");
    // allocations before anything is enqueued
    {
        const grt_status bs = prepare_trace_buffers(c, make_kparams(c).n);
        if (bs != GRT_OK) return bs;
        size_t pix = 0;
        for (const auto& sp : c->images) pix += 4 * sp.nx * sp.ny;
        GRT_CUDA(c, c->bimage.alloc(pix), "alloc products");
        GRT_CUDA(c, c->bspectrum.alloc(nimages * p.spectrum_bins), "alloc products");
        GRT_CUDA(c, c->barrived.alloc(nimages), "alloc products");
    }
    c->bproducts_valid = false;
    c->adj_ready = false;
    const grt_status st = enqueue_render(c, s, outs);
    if (st != GRT_OK) {
        // part of the render may be enqueued: let it drain before reporting
        cudaStreamSynchronize(c->stream);
        cudaStreamSynchronize(c->copy_stream);
        return st;
    }
    c->render_pending = true;
    return GRT_OK;
}

grt_status grt_render_wait(grt_ctx* c, grt_run_stats* stats) {
    if (!c) return GRT_EINVAL;
    if (!c->render_pending) return fail(c, GRT_ESTATE, "no render in flight on this context (grt_render_async)");
    c->render_pending = false;
    GRT_CUDA(c, cudaEventSynchronize(c->ev_done), "render");
    const grt_params& p = c->p;
    const grt::KCounters& k = *c->host_counters;
    const unsigned long long terminated = c->host_u64[1] + k.terminated;
    c->initial_terminated = terminated;
    c->bproducts_valid = true;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    grt_run_stats st;
    std::memset(&st, 0, sizeof(st));
    st.accepted_steps = k.accepted;
    st.rejected_attempts = k.rejected;
    st.photon_calls = k.calls;
    st.launches = split_legs(c) ? 3 : 1;
    st.n_terminated = terminated;
    st.trace_ms = ms;
    st.steps_done = single_launch_steps_done(p, terminated, c->n, k.max_term_step);
    if (k.timed_out) {
        st.timed_out = 1;
        if (stats) *stats = st;
        return fail(c, GRT_ETIMEOUT, "trace kernel hit its iteration limit");
    }
    if (stats) *stats = st;
    return GRT_OK;
}

grt_status grt_set_cell_multipliers(grt_ctx* c, const double* m_abs, const double* m_emis) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    const size_t ncell = static_cast<size_t>(c->nr) * c->nth * c->nph;
    if ((m_abs || m_emis) && (!c->grid_uploaded || !c->fluid_available || ncell == 0))
        return fail(c, GRT_ESTATE, "cell multipliers need an uploaded fluid grid");
    ++c->generation;
    c->adj_ready = false;
    c->has_m_abs = c->has_m_emis = false;
    if (m_abs) {
        GRT_CUDA(c, c->m_abs.alloc(ncell), "alloc multipliers");
        GRT_CUDA(c, cudaMemcpy(c->m_abs.ptr, m_abs, ncell * sizeof(double), cudaMemcpyHostToDevice), "H2D");
        c->has_m_abs = true;
    }
    if (m_emis) {
        GRT_CUDA(c, c->m_emis.alloc(ncell), "alloc multipliers");
        GRT_CUDA(c, cudaMemcpy(c->m_emis.ptr, m_emis, ncell * sizeof(double), cudaMemcpyHostToDevice), "H2D");
        c->has_m_emis = true;
    }
    return GRT_OK;
}

grt_status grt_forward_checkpointed(grt_ctx* c, int64_t K, grt_run_stats* stats) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    if (!c->grid_uploaded) return fail(c, GRT_ESTATE, "grt_forward_checkpointed before grt_upload_grid");
    const grt_params& p = c->p;
    if (K < 1 || K > (1 << 20)) return fail(c, GRT_EINVAL, "checkpoint_interval must be in [1, 2^20]");
    if (!(p.termination_percent >= 1.0))
        return fail(c, GRT_EINVAL, "the checkpointed forward needs termination_percent >= 1");
    if (p.precision != GRT_PREC_FP64) return fail(c, GRT_EINVAL, "the checkpointed forward runs the FP64 form");
    grt_run_stats st;
    std::memset(&st, 0, sizeof(st));
    c->adj_ready = false;
    c->bproducts_valid = false;
    const size_t n = c->n;
    const long long cap = (p.max_steps + K - 1) / K + 1;
    const double bytes = static_cast<double>(n) * static_cast<double>(cap) * 16.0 * 8.0;
    if (bytes > 32.0 * (1ull << 30))
        return fail(c, GRT_ENOMEM, "checkpoints would need " + std::to_string(bytes / (1ull << 30)) +
                                       " GiB; raise checkpoint_interval");
    const int threads = 128;
    const long long want_blocks = (static_cast<long long>(n) + threads - 1) / threads;
    const int blocks = static_cast<int>(std::max(1ll, std::min<long long>(want_blocks, 8ll * c->sm_count)));
    GRT_CUDA(c, c->ckpt.alloc(n * cap * 16), "alloc checkpoints");
    GRT_CUDA(c, c->nckpt.alloc(std::max<size_t>(n, 1)), "alloc checkpoints");
    GRT_CUDA(c, c->call0.alloc(std::max<size_t>(n, 1)), "alloc checkpoints");
    GRT_CUDA(c, c->adj_overflow.alloc(1), "alloc checkpoints");
    GRT_CUDA(c, c->tape.alloc(static_cast<size_t>(blocks) * threads * K * 6), "alloc tape");
    c->adj_K = static_cast<int>(K);
    c->adj_cap = static_cast<int>(cap);
    if (n == 0) {
        st.steps_done = p.max_steps;
        if (stats) *stats = st;
        c->adj_ready = true;
        return GRT_OK;
    }
    grt::KParams kp = make_kparams(c);
    kp.step0 = 0;
    kp.budget = p.max_steps;
    grt::AdjointArgs aa{};
    aa.ckpt = c->ckpt.ptr;
    aa.cap = c->adj_cap;
    aa.K = c->adj_K;
    aa.nckpt = c->nckpt.ptr;
    aa.call0 = c->call0.ptr;
    aa.overflow = c->adj_overflow.ptr;
    GRT_CUDA(c, cudaMemsetAsync(c->counters.ptr, 0, sizeof(grt::KCounters), c->stream), "memset");
    GRT_CUDA(c, cudaMemsetAsync(c->adj_overflow.ptr, 0, sizeof(int), c->stream), "memset");
    GRT_CUDA(c, cudaEventRecord(c->ev0, c->stream), "event");
    cudaError_t e = grt::launch_adjoint_forward(kp, aa, blocks, trace_smem(c), c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "adjoint forward launch");
    GRT_CUDA(c, cudaEventRecord(c->ev1, c->stream), "event");
    GRT_CUDA(c, cudaMemcpyAsync(c->host_counters, c->counters.ptr, sizeof(grt::KCounters), cudaMemcpyDeviceToHost,
                                c->stream), "D2H counters");
    int overflow = 0;
    GRT_CUDA(c, cudaMemcpyAsync(&overflow, c->adj_overflow.ptr, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
             "D2H");
    GRT_CUDA(c, cudaStreamSynchronize(c->stream), "adjoint forward");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    if (overflow) return fail(c, GRT_ECUDA, "checkpoint capacity exceeded");
    const grt::KCounters& k = *c->host_counters;
    st.photon_calls = k.calls;
    st.n_terminated = k.terminated + c->initial_terminated;
    st.launches = 1;
    st.trace_ms = ms;
    st.steps_done = p.max_steps;
    if (stats) *stats = st;
    c->adj_ready = true;
    return GRT_OK;
}

grt_status grt_adjoint_image_I(grt_ctx* c, const double* dL_dI, double* g_abs, double* g_emis) {
    if (c && c->render_pending) return rendering(c);
    if (!c || !dL_dI) return GRT_EINVAL;
    if (!c->adj_ready) return fail(c, GRT_ESTATE, "grt_adjoint_image_I needs a grt_forward_checkpointed first");
    if (c->batched) return fail(c, GRT_EINVAL, "the adjoint covers single-image runs");
    const grt_params& p = c->p;
    const size_t ncell = static_cast<size_t>(c->nr) * c->nth * c->nph;
    const size_t npix = p.image_nx * p.image_ny;
    GRT_CUDA(c, c->dLdI.alloc(std::max<size_t>(npix, 1)), "alloc");
    GRT_CUDA(c, c->g_abs.alloc(std::max<size_t>(ncell, 1)), "alloc");
    GRT_CUDA(c, c->g_emis.alloc(std::max<size_t>(ncell, 1)), "alloc");
    GRT_CUDA(c, cudaMemcpyAsync(c->dLdI.ptr, dL_dI, npix * sizeof(double), cudaMemcpyHostToDevice, c->stream), "H2D");
    GRT_CUDA(c, cudaMemsetAsync(c->g_abs.ptr, 0, std::max<size_t>(ncell, 1) * sizeof(double), c->stream), "memset");
    GRT_CUDA(c, cudaMemsetAsync(c->g_emis.ptr, 0, std::max<size_t>(ncell, 1) * sizeof(double), c->stream), "memset");
    GRT_CUDA(c, cudaMemsetAsync(c->adj_overflow.ptr, 0, sizeof(int), c->stream), "memset");
    if (c->n > 0 && ncell > 0) {
        grt::KParams kp = make_kparams(c);
        kp.step0 = 0;
        kp.budget = p.max_steps;
        grt::AdjointArgs aa{};
        aa.ckpt = c->ckpt.ptr;
        aa.cap = c->adj_cap;
        aa.K = c->adj_K;
        aa.nckpt = c->nckpt.ptr;
        aa.call0 = c->call0.ptr;
        aa.overflow = c->adj_overflow.ptr;
        aa.dL_dI = c->dLdI.ptr;
        aa.nx = p.image_nx;
        aa.ny = p.image_ny;
        aa.W = p.camera_width;
        aa.H = p.camera_height;
        aa.g_abs = c->g_abs.ptr;
        aa.g_emis = c->g_emis.ptr;
        aa.tape = c->tape.ptr;
        const int threads = 128;
        const size_t tape_threads = c->tape.count / (static_cast<size_t>(c->adj_K) * 6);
        const int blocks = static_cast<int>(std::max<size_t>(1, tape_threads / threads));
        cudaError_t e = grt::launch_adjoint_reverse(kp, aa, blocks, trace_smem(c), c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "adjoint reverse launch");
    }
    int overflow = 0;
    GRT_CUDA(c, cudaMemcpyAsync(&overflow, c->adj_overflow.ptr, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
             "D2H");
    if (g_abs && ncell)
        GRT_CUDA(c, cudaMemcpyAsync(g_abs, c->g_abs.ptr, ncell * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                 "D2H gradient");
    if (g_emis && ncell)
        GRT_CUDA(c, cudaMemcpyAsync(g_emis, c->g_emis.ptr, ncell * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                 "D2H gradient");
    GRT_CUDA(c, cudaStreamSynchronize(c->stream), "adjoint reverse");
    if (overflow) return fail(c, GRT_ECUDA, "adjoint tape capacity exceeded");
    return GRT_OK;
}

grt_status grt_get_image_products(grt_ctx* c, grt_image_products* out) {
    if (c && c->render_pending) return rendering(c);
    if (!c || !out) return GRT_EINVAL;
    const grt_params& p = c->p;
    const size_t npix = p.image_nx * p.image_ny, bins = p.spectrum_bins;
    if (!out->image_I || !out->image_Q || !out->image_U || !out->image_V || !out->spectrum_frequency_hz ||
        !out->spectrum_I || !out->arrived_count)
        return fail(c, GRT_EINVAL, "null image product buffer");
    GRT_CUDA(c, c->image.alloc(4 * npix), "alloc image");
    GRT_CUDA(c, c->spectrum.alloc(bins), "alloc spectrum");
    GRT_CUDA(c, c->arrived.alloc(1), "alloc arrived");
    grt_status st = launch_products(c, 0, c->n, p.image_nx, p.image_ny, p.camera_width, p.camera_height, c->image.ptr,
                                    c->spectrum.ptr, c->arrived.ptr);
    if (st != GRT_OK) return st;
    double* dst[4] = {out->image_I, out->image_Q, out->image_U, out->image_V};
    for (int q = 0; q < 4; ++q)
        GRT_CUDA(c, cudaMemcpyAsync(dst[q], c->image.ptr + q * npix, npix * sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream), "D2H image");
    GRT_CUDA(c, cudaMemcpyAsync(out->spectrum_I, c->spectrum.ptr, bins * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream), "D2H spectrum");
    GRT_CUDA(c, cudaMemcpyAsync(out->arrived_count, c->arrived.ptr, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                c->stream), "D2H arrived");
    fill_spectrum_frequencies(p, out->spectrum_frequency_hz);
    GRT_CUDA(c, cudaStreamSynchronize(c->stream), "products");
    return GRT_OK;
}

}  // extern "C"

namespace {

// write_image_products (write_output.hpp:107-142): one archive, written to a
// temporary name and renamed into place.
grt_status write_products_archive(grt_ctx* c, const std::string& output_dir, const std::string& file, size_t nx,
                                  size_t ny, size_t bins, const grt_image_products& out) {
    namespace fs = std::filesystem;
    std::error_code ec;
    fs::create_directories(output_dir, ec);
    const fs::path final_path = fs::path(output_dir) / file;
    const fs::path tmp = final_path.string() + ".tmp";
    grt::NpzOut z;
    if (!z.open(tmp.string())) return fail(c, GRT_EIO, "Failed to open output NumPy archive: " + tmp.string());
    const std::vector<size_t> img{ny, nx}, spec{bins}, one{1};
    bool ok = z.add("image_I", grt::npy_bytes("<f8", img, out.image_I, 8)) &&
              z.add("image_Q", grt::npy_bytes("<f8", img, out.image_Q, 8)) &&
              z.add("image_U", grt::npy_bytes("<f8", img, out.image_U, 8)) &&
              z.add("image_V", grt::npy_bytes("<f8", img, out.image_V, 8)) &&
              z.add("spectrum_frequency_hz", grt::npy_bytes("<f8", spec, out.spectrum_frequency_hz, 8)) &&
              z.add("spectrum_I", grt::npy_bytes("<f8", spec, out.spectrum_I, 8)) &&
              z.add("arrived_count", grt::npy_bytes("<u8", one, out.arrived_count, 8));
    ok = z.close() && ok;
    if (!ok) {
        fs::remove(tmp, ec);
        return fail(c, GRT_EIO, z.error().empty() ? std::string("Failed while writing NumPy archive") : z.error());
    }
    fs::rename(tmp, final_path, ec);
    if (ec) {
        fs::remove(tmp, ec);
        return fail(c, GRT_EIO, "Failed to publish output archive " + final_path.string());
    }
    return GRT_OK;
}

// Device pointer and element size of output field k (grt::kOutputFields order).
const void* output_field(const grt_ctx* c, int k, int& item) {
    item = 8;
    if (k == 0) return c->ph.id.ptr;
    if (k >= 1 && k <= 15) return c->ph.f[k - 1].ptr;  // frequency .. dlambda
    if (k == 16 || k == 17) {
        item = 1;
        return k == 16 ? static_cast<const void*>(c->ph.term.ptr) : static_cast<const void*>(c->ph.phase.ptr);
    }
    return c->ph.f[k - 3].ptr;  // 18, 19: theta_disp, phi_disp
}

// write_output_step (write_output.hpp:90-103) with add_photon_array's strided
// values (:26-59): the selected fields of photons 0, stride, 2*stride, ...
// gathered on the device into one staging buffer, one copy back, then one
// archive written under a temporary name and renamed into place.
grt_status write_output_step(grt_ctx* c, const OutputPlan& plan, int64_t step) {
    namespace fs = std::filesystem;
    const size_t n = c->n;
    const unsigned long long count = n == 0 ? 0 : 1 + (n - 1) / plan.stride;
    grt::GatherArgs g;
    std::memset(&g, 0, sizeof(g));
    unsigned long long bytes = 0;
    for (size_t q = 0; q < plan.fields.size(); ++q) {
        g.src[q] = output_field(c, plan.fields[q], g.item[q]);
        g.dst_off[q] = bytes;
        bytes += (count * g.item[q] + 7) / 8 * 8;
    }
    g.nfields = static_cast<int>(plan.fields.size());
    g.count = count;
    g.stride = plan.stride;
    if (bytes > 0) {
        GRT_CUDA(c, c->out_stage.alloc(bytes), "alloc output stage");
        if (c->host_out_bytes < bytes) {
            if (c->host_out) cudaFreeHost(c->host_out);
            c->host_out = nullptr;
            c->host_out_bytes = 0;
            GRT_CUDA(c, cudaMallocHost(reinterpret_cast<void**>(&c->host_out), bytes), "alloc output host stage");
            c->host_out_bytes = bytes;
        }
        g.dst = c->out_stage.ptr;
        GRT_CUDA(c, grt::launch_gather_fields(g, c->sm_count, c->stream), "gather_fields");
        GRT_CUDA(c, cudaMemcpyAsync(c->host_out, c->out_stage.ptr, bytes, cudaMemcpyDeviceToHost, c->stream),
                 "D2H output step");
        GRT_CUDA(c, cudaStreamSynchronize(c->stream), "output step");
    }
    std::error_code ec;
    fs::create_directories(plan.dir, ec);
    const fs::path final_path =
        fs::path(plan.dir) / (plan.name + "_step_" + std::to_string(step) + "_rank" + std::to_string(plan.rank) + ".npz");
    const fs::path tmp = final_path.string() + ".tmp";
    grt::NpzOut z;
    if (!z.open(tmp.string())) return fail(c, GRT_EIO, "Failed to open output NumPy archive: " + tmp.string());
    const std::vector<size_t> shape{static_cast<size_t>(count)};
    bool ok = true;
    for (size_t q = 0; q < plan.fields.size() && ok; ++q) {
        const int k = plan.fields[q];
        const char* descr = k == 0 ? "<u8" : (g.item[q] == 1 ? "|u1" : "<f8");
        ok = z.add(grt::kOutputFields[k], grt::npy_bytes(descr, shape, c->host_out ? c->host_out + g.dst_off[q] : nullptr,
                                                         static_cast<size_t>(g.item[q])));
    }
    ok = z.close() && ok;
    if (!ok) {
        fs::remove(tmp, ec);
        return fail(c, GRT_EIO, z.error().empty() ? std::string("Failed while writing NumPy archive") : z.error());
    }
    fs::rename(tmp, final_path, ec);
    if (ec) {
        fs::remove(tmp, ec);
        return fail(c, GRT_EIO, "Failed to publish output archive " + final_path.string() + ": " + ec.message());
    }
    return GRT_OK;
}

grt_status make_output_plan(grt_ctx* c, const char* output_dir, const char* name, const char* variables,
                            uint64_t stride, int32_t rank, OutputPlan& plan) {
    if (!output_dir || !name || !variables) return fail(c, GRT_EINVAL, "null output argument");
    if (!*output_dir) return fail(c, GRT_EINVAL, "output.directory must not be empty");
    if (!*name) return fail(c, GRT_EINVAL, "simulation.name must not be empty");
    if (stride == 0) return fail(c, GRT_EINVAL, "output.stride must be positive");
    std::string err;
    if (!grt::parse_output_variables(variables, plan.fields, err)) return fail(c, GRT_EINVAL, err);
    if (plan.fields.size() > static_cast<size_t>(grt::kGatherMaxFields))
        return fail(c, GRT_EINVAL, "too many output variables");
    plan.dir = output_dir;
    plan.name = name;
    plan.stride = stride;
    plan.rank = rank;
    return GRT_OK;
}

}  // namespace

extern "C" {

grt_status grt_write_image_products_npz(grt_ctx* c, const char* output_dir, const char* name) {
    if (c && c->render_pending) return rendering(c);
    if (!c || !output_dir || !name) return GRT_EINVAL;
    const grt_params& p = c->p;
    const size_t nx = p.image_nx, ny = p.image_ny, bins = p.spectrum_bins;
    std::vector<double> I(nx * ny), Q(nx * ny), U(nx * ny), V(nx * ny), sf(bins), si(bins);
    uint64_t arrived = 0;
    grt_image_products out{I.data(), Q.data(), U.data(), V.data(), sf.data(), si.data(), &arrived};
    grt_status s = grt_get_image_products(c, &out);
    if (s != GRT_OK) return s;
    return write_products_archive(c, output_dir, std::string(name) + "_image_products.npz", nx, ny, bins, out);
}

grt_status grt_write_batch_products_npz(grt_ctx* c, const char* output_dir, const char* name) {
    if (c && c->render_pending) return rendering(c);
    if (!c || !output_dir || !name) return GRT_EINVAL;
    if (!c->batched) return fail(c, GRT_ESTATE, "no image batch (grt_init_image_batch)");
    const size_t bins = c->p.spectrum_bins;
    for (size_t k = 0; k < c->images.size(); ++k) {
        const size_t nx = c->images[k].nx, ny = c->images[k].ny;
        std::vector<double> I(nx * ny), Q(nx * ny), U(nx * ny), V(nx * ny), sf(bins), si(bins);
        uint64_t arrived = 0;
        grt_image_products out{I.data(), Q.data(), U.data(), V.data(), sf.data(), si.data(), &arrived};
        grt_status s = grt_get_batch_image_products(c, k, &out);
        if (s != GRT_OK) return s;
        s = write_products_archive(c, output_dir,
                                   std::string(name) + "_image" + std::to_string(k) + "_image_products.npz", nx, ny,
                                   bins, out);
        if (s != GRT_OK) return s;
    }
    return GRT_OK;
}

grt_status grt_write_output_step_npz(grt_ctx* c, const char* output_dir, const char* name, int64_t step,
                                     int32_t rank, const char* variables, uint64_t stride) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    OutputPlan plan;
    const grt_status ps = make_output_plan(c, output_dir, name, variables, stride, rank, plan);
    if (ps != GRT_OK) return ps;
    return write_output_step(c, plan, step);
}

grt_status grt_run_with_output(grt_ctx* c, const char* output_dir, const char* name, const char* variables,
                               uint64_t stride, grt_run_stats* stats) {
    if (c && c->render_pending) return rendering(c);
    if (!c) return GRT_EINVAL;
    OutputPlan plan;
    grt_status s = make_output_plan(c, output_dir, name, variables, stride, c->p.rank, plan);
    if (s != GRT_OK) return s;
    s = run_steps(c, stats, &plan);
    if (s != GRT_OK) return s;
    // integrate_cart_ks.hpp:529-531: image mode ends with the image products
    if (c->p.mode == GRT_MODE_IMAGE)
        return c->batched ? grt_write_batch_products_npz(c, output_dir, name)
                          : grt_write_image_products_npz(c, output_dir, name);
    return GRT_OK;
}

}  // extern "C"
